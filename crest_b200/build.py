"""Build the CREST B200 CUDA library in-tree (nvcc, sm_100a)."""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcrest_gpu.so")
SOURCES = ["capi.cu", "capi_matrix.cu", "capi_static.cu", "k_fused.cu", "k_stream.cu", "k_sweep.cu", "k_gram.cu", "k_gram_tc.cu", "k_compact.cu", "k_groups.cu", "k_knn.cu", "k_csc.cu", "k_eig.cu", "synth.cu", "prof.cu"]
HEADERS = ["common.cuh", "kernels.cuh", "rowwarp.cuh", "host.cuh", "log1pf_libm.h", "synth_core.h", "prof.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "crest_gpu.h")]
    return any(os.path.exists(p) and os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False, jobs: int = 0) -> str:
    """Compile every .cu source for sm_100a and link libcrest_gpu.so (static cudart)."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "-I", CSRC, "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr",
              "--extended-lambda"] + (["-Xptxas", "-v"] if verbose else [])
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = common + ["-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    link = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *objs, "-lpthread"]
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
