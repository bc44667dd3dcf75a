"""The GPU path's single-precision log1p restatement (crest_b200/csrc/log1pf_libm.h)
equals the platform libm's log1pf -- what the reference's f32::ln_1p calls -- on
every one of the 2^32 float bit patterns."""

import ctypes as C
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def sweep(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("l1p") / "l1p_sweep.so")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I",
                    os.path.join(ROOT, "crest_b200", "csrc"), "-o", out, os.path.join(ROOT, "tests", "l1p_sweep.c"),
                    "-lm", "-lpthread"], check=True)
    lib = C.CDLL(out)
    lib.l1p_sweep.restype = C.c_uint64
    lib.l1p_sweep.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_uint32)]
    return lib


def test_log1pf_matches_libm_on_all_floats(sweep):
    first = C.c_uint32()
    bad = sweep.l1p_sweep(0, 1 << 32, os.cpu_count() or 1, C.byref(first))
    assert bad == 0, f"{bad} mismatches, first at bits {first.value:#010x}"
