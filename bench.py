"""Benchmark of the scale + PCA hot path: cells/s at 1,000,000 cells x 36,601
genes (seeded synthetic negative-binomial counts, ~1,500 non-zeros per cell,
50 clusters), HVG 2000, scale(max 10), 50 components, split-BF16 tensor-core
Gram with FP64 centring / eigensolve, projection.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One step = Gram pass over all cells (densify + bf16x3 tcgen05 SYRK + FP64
fold) + FP64 centring/eigensolve + projection pass, with the CSR matrix
resident in HBM (12 GB, larger than L2, so no flush is needed).  ``e2e`` is
the same step through the public API with host buffers: the pinned-host CSR
is uploaded and X_pca is read back inside the timed region.  Under torchrun
each rank holds its own 1M-cell shard (weak scaling); the FP64 Gram and
column sums are all-reduced over NCCL before the replicated eigensolve.
``--impl reference`` times the CPU restatement of the reference's Rust path
(threads = host cores) on the same workload: the same matrix, drawn on host
threads from the same generator, every cell in every step.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cells/s scale+PCA@1M cells, split-BF16 vs FP32 GPU at ≤0.01° angle; HBM GB/s"
UNIT = "cells/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="crest_b200", choices=["crest_b200", "reference"])
    ap.add_argument("--workload", default="1m")
    ap.add_argument("--cells", type=int, default=0, help="override the workload's cell count (testing)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return {"hbm_gbs": j["hbm_gbs"], "bf16_tflops": j["bf16_tflops"],
                "bf16_tflops_sustained": j.get("bf16_tflops_sustained", j["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes (read + write) of a kernel at the benchmark's launch
    size, from the committed ncu summary profiles/traffic.txt ("name bytes" lines)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#") and parts[0] == kernel:
                return float(parts[1])
    return None


def repo_libs_mapped():
    """Shared objects of this repository mapped into the process (from /proc/self/maps)."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(ROOT + os.sep):
                    out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------------ workload
def build_inputs(args, rank: int, device: str):
    """Generate the rank's shard: the named workload (or its first --cells cells),
    drawn on the GPU into page-locked host buffers ("gpu") or by the oracle's
    host-thread generator ("cpu", the reference arm).  Both draw the same matrix."""
    from crest_b200 import synth
    w = synth.WORKLOADS[args.workload]
    if rank:
        w = synth.Workload(w.name, w.n_cells, w.n_genes, w.n_clusters, w.dispersion, w.nnz_per_cell,
                           w.seed + 1000 * rank, w.chunk_cells)
    n_cells = min(args.cells or w.n_cells, w.n_cells)
    t0 = time.time()
    if device == "gpu":
        import torch

        def alloc(n, dt):
            t = torch.empty(int(n), dtype={np.uint32: torch.int32, np.float32: torch.float32}[dt], pin_memory=True)
            return t.numpy().view(dt)
        arrays = synth.make_workload(w, n_cells=n_cells, pinned_alloc=alloc)
    else:
        from oracle import synth as osynth
        arrays = osynth.make_workload(w, n_cells=n_cells)
    return w, n_cells, arrays, time.time() - t0


def workload_label(w, n_cells: int) -> str:
    """The workload as both arms name it in `config` (the method is in `dtype`)."""
    return (f"{w.name}: {n_cells} cells x {w.n_genes} genes per GPU, NB counts (~{w.nnz_per_cell:.0f} nnz/cell, "
            f"{w.n_clusters} clusters), HVG 2000, scale 10, 50 PCs")


def preprocess(bf, allreduce=None):
    import crest_b200 as cb
    from crest_b200 import pp
    bf = cb.pp.filter_cells(bf, min_genes=200)
    bf = cb.pp.filter_genes(bf, min_cells=3)
    cb.pp.normalize_total(bf, 1e4)
    cb.pp.log1p(bf)
    cb.pp.highly_variable_genes(bf, n_top_genes=2000)
    cb.pp.scale(bf, max_value=10)
    return bf


def pca_inputs(bf):
    from crest_b200 import _lib
    from crest_b200.tl import _scale_params
    mask = bf.var["highly_variable"].to_numpy().astype(bool)
    d = int(mask.sum())
    sub = np.full(bf.n_vars, -1, np.int32)
    sub[mask] = np.arange(d, dtype=np.int32)
    mean, std = _scale_params(bf, mask)
    cmap, gmap = bf._cell_map(), bf._gene_map()
    target, log = bf._transform()
    scale = _lib.Scale(1, _lib.ptr(mean), _lib.ptr(std), 10.0)
    return dict(d=d, sub=sub, mean=mean, std=std, cmap=cmap, gmap=gmap, target=target, log=log, scale=scale,
                n=bf.n_obs, n_vars=bf.n_vars, mask=mask)


# ------------------------------------------------------------------ reference arm
def cpu_prepare(indptr, indices, data, n_genes, threads):
    """QC filters, normalize_total, log1p, seurat HVG and scale of the oracle (the
    reference's CPU path restated: C kernels in its summation order + its numpy
    host math); the untimed preprocessing before the scale + PCA step."""
    from oracle import pipeline as op
    from crest_b200 import synth
    f = op.Frame(indptr, indices, data, n_genes, synth.gene_names(n_genes), threads=threads)
    f = op.filter_cells(f, min_genes=200)
    f = op.filter_genes(f, min_cells=3)
    op.normalize_total(f, 1e4)
    op.log1p(f)
    op.highly_variable_genes(f, n_top_genes=2000)
    op.scale(f, 10)
    return f


def cpu_step(f):
    """One scale + PCA step of the oracle over every kept cell: FP64 Gram pass,
    LAPACK eigensolve, projection pass.  Returns seconds."""
    from oracle import pipeline as op
    t0 = time.perf_counter()
    op.pca(f, n_comps=50)
    return time.perf_counter() - t0


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    oracle.build()
    threads = os.cpu_count() or 1
    w, n_cells, (indptr, indices, data), gen_s = build_inputs(args, 0, "cpu")
    t0 = time.time()
    f = cpu_prepare(indptr, indices, data, w.n_genes, threads)
    prep_s = time.time() - t0
    times = []
    for i in range(args.warmup + args.steps):
        dt = cpu_step(f)
        if i >= args.warmup:
            times.append(dt)
    t = float(np.mean(times))
    v = f.n_obs / t
    sample = (f"every cell of the workload ({f.n_obs} after QC) in every step: FP64 Gram pass, LAPACK "
              f"eigensolve, projection pass")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_label(w, n_cells), "cells_after_qc": f.n_obs,
                       "parallelism": f"{threads} cpu threads"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "generate_s": gen_s, "preprocess_s": prep_s, "native_so_loaded": repo_libs_mapped()}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def main_gpu(args):
    import torch
    import crest_b200 as cb
    from crest_b200 import _lib, tl
    import pandas as pd

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    _lib.call("crest_set_device", local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        from crest_b200 import dist as cdist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        cdist.enable()  # per-gene sums and the Gram are summed over ranks

    wl, n_gen, (indptr, indices, data), gen_s = build_inputs(args, rank, "gpu")
    from crest_b200 import synth
    names = synth.gene_names(wl.n_genes)
    bf = cb.BioFrame.from_csr(indptr, indices, data, wl.n_genes, var=pd.DataFrame({"gene_name": names}))
    t0 = time.time()
    _lib.profile_enable(True)  # the one-time passes (range index, cell totals) run here
    bf = preprocess(bf)
    prep_s = time.time() - t0
    tb_prep = _lib.profile_table()
    _lib.profile_enable(False)
    P = pca_inputs(bf)
    dm = bf.device_matrix()
    n_rows, k = P["n"], 50
    nnz = int(indptr[-1])
    X = torch.empty((n_rows, k), dtype=torch.float32, device="cuda")

    def step(plan):
        plan.accumulate(dm, P["cmap"], P["gmap"], P["target"], P["log"], P["sub"], P["n_vars"], P["scale"])
        n_tot = n_rows
        if dist is not None:  # one NCCL sum of the FP64 accumulators and the cell count
            gp, cp = plan.accumulators()
            cdist.sum_device(gp, P["d"] * P["d"])
            cdist.sum_device(cp, P["d"])
            n_tot = cdist.sum_count(n_rows)
        plan.solve(n_tot, k)
        plan.project(dm, P["cmap"], P["gmap"], P["target"], P["log"], P["sub"], P["n_vars"], P["scale"], n_rows,
                     device_ptr=X.data_ptr())

    def timed(precision, steps, warmup, profile=False, mark=False):
        plan = tl.PcaPlan(P["d"], precision)
        for _ in range(warmup):
            plan.reset()
            step(plan)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        if profile:
            _lib.profile_enable(True)
        # K steps timed as one interval, bracketed by a barrier and a sync
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        if mark:  # an NVTX range around the timed steps, for a profiler to select them
            torch.cuda.nvtx.range_push("crest_step")
        e0.record()
        for _ in range(steps):
            plan.reset()
            step(plan)
        e1.record()
        if mark:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        per = [e0.elapsed_time(e1) / steps]
        table = _lib.profile_table() if profile else {}
        if profile:
            _lib.profile_enable(False)
        stats = plan.stats()
        loadings = plan.results()[1]
        plan.close()
        ms = float(np.mean(per))
        if dist is not None:
            mt = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(mt, op=dist.ReduceOp.MAX)
            ms = float(mt.item())
        return ms, stats, table, loadings

    peaks = measured_peaks()
    with ClockSampler(local) as clk:
        ms, stats, _, L_bf = timed("bf16x3", args.steps, args.warmup, mark=True)
    clocks = clk.summary()
    value = n_rows * ws / (ms / 1e3)

    extra = {}
    # per-kernel device times: the same K steps again with a CUDA-event scope
    # around every launch (on its stream); the scopes' host cost makes this
    # pass a little slower, so the headline value comes from the pass above
    ms_prof, _, table, _ = timed("bf16x3", args.steps, 1, profile=True)
    extra["ms_per_step_profiled"] = ms_prof
    if not args.no_fp32:
        ms32, st32, tb32, L_32 = timed("fp32", max(2, args.steps // 2), 1)
        extra["fp32_cells_per_s"] = n_rows * ws / (ms32 / 1e3)
        extra["fp32_ms_per_step"] = ms32
        extra["speedup_bf16x3_vs_fp32"] = ms32 / ms
        # the Gram phase is the only part that differs between the two forms
        extra["speedup_gram_bf16x3_vs_fp32"] = st32["gram_ms"] / stats["gram_ms"]
    # accuracy of the product form against the FP64 Gram of the same run
    ms64, st64, _, L_64 = timed("fp64", 1, 0)
    from numpy.linalg import qr, svd
    qa, _ = qr(L_bf)
    qb, _ = qr(L_64)
    ang = float(np.degrees(np.arccos(np.clip(svd(qa.T @ qb, compute_uv=False), -1, 1))).max())
    extra["max_principal_angle_deg_vs_fp64"] = ang
    if not args.no_fp32:
        qc_, _ = qr(L_32)
        extra["fp32_max_principal_angle_deg_vs_fp64"] = float(
            np.degrees(np.arccos(np.clip(svd(qc_.T @ qb, compute_uv=False), -1, 1))).max())

    # memory-bound passes (HBM GB/s): QC and gene_stats over the whole CSR
    bytes_pass = nnz * 8 + (len(indptr)) * 8
    from crest_b200 import pp
    _lib.profile_enable(True)
    for _ in range(3):
        pp.calculate_qc_metrics(bf, inplace=False)
        pp.gene_stats(bf)
    tb_mem = _lib.profile_table()
    _lib.profile_enable(False)
    hbm = {}
    # bytes per launch: QC / gene_stats / cell totals read every entry once;
    # the one-time range index reads the gene ids and writes the row offsets
    n_ranges = max(2, -(-wl.n_genes // 4096))
    pass_bytes = {"qc_csr": bytes_pass, "gene_stats_csr": bytes_pass, "cell_totals_csr": bytes_pass,
                  "range_index_csr": nnz * 4 + len(indptr) * 8 + (len(indptr) - 1) * (n_ranges - 1) * 4}
    for kname, byts in pass_bytes.items():
        tb = tb_mem if kname in tb_mem else tb_prep
        if kname in tb:
            n_l, tot, mx = tb[kname]
            hbm[kname] = byts / (tot / n_l / 1e3) / 1e9
    if "project_csr" in table:
        n_l, tot, mx = table["project_csr"]
        hbm["project_csr"] = (bytes_pass + n_rows * k * 4 * 2) / (tot / n_l / 1e3) / 1e9
    if "extract_csr" in table:  # one CSR read per step; HVG entries and per-cell records written
        n_l, tot, mx = table["extract_csr"]
        hbm["extract_csr"] = bytes_pass / (tot / n_l / 1e3) / 1e9
    extra["hbm_gbs"] = hbm
    extra["hbm_frac"] = {kk: v / peaks["hbm_gbs"] for kk, v in hbm.items()}

    # roofline of the dominant kernel of the step
    # (the eigensolver is a fixed FP64 cost reported as time, not a roofline kernel)
    cand = {kk: v for kk, v in table.items() if not kk.startswith("eig_")}
    dom = max(cand.items(), key=lambda kv: kv[1][1]) if cand else None
    roof = None
    if dom:
        name, (n_l, tot, mx) = dom
        avg_s = tot / n_l / 1e3
        per_step = n_l / args.steps  # launches of this kernel in one step
        d = P["d"]
        if name.startswith("syrk"):
            flops = n_rows * d * (d + 1) / per_step  # algorithmic dense SYRK flops per launch
            ach = flops / avg_s / 1e12
            pk = peaks["bf16_tflops_sustained"]
            roof = {"kernel": name, "bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                    "frac": ach / pk, "traffic": ncu_traffic(name), "launches": n_l, "avg_ms": avg_s * 1e3,
                    "peak_source": peaks["source"] + " (bf16 sustained)",
                    "algorithmic": "n_cells*d*(d+1) flops per Gram pass / launches"}
        else:
            byts = bytes_pass / per_step
            ach = byts / avg_s / 1e9
            roof = {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": ach / peaks["hbm_gbs"], "traffic": ncu_traffic(name), "launches": n_l,
                    "avg_ms": avg_s * 1e3, "peak_source": peaks["source"]}
    launches = int(sum(v[0] for v in table.values()) / max(1, args.steps))

    # end to end through the public API with host buffers
    e2e = None
    if rank == 0 or ws > 1:
        times = []
        for i in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m = cb.core.DeviceMatrix(indptr, indices, data, wl.n_genes, "device")
            plan = tl.PcaPlan(P["d"], "bf16x3")
            plan.accumulate(m, P["cmap"], P["gmap"], P["target"], P["log"], P["sub"], P["n_vars"], P["scale"])
            plan.solve(n_rows, k)
            Xh = plan.project(m, P["cmap"], P["gmap"], P["target"], P["log"], P["sub"], P["n_vars"], P["scale"],
                              n_rows)
            plan.close()
            m.close()
            torch.cuda.synchronize()
            if i > 0:
                times.append(time.perf_counter() - t0)
        te = float(np.mean(times))
        h2d = nnz * 8 + len(indptr) * 8 + P["cmap"].nbytes + P["gmap"].nbytes
        e2e = {"value": n_rows * ws / te, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(Xh.nbytes), "ms_per_step": te * 1e3}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        # the oracle (the reference's CPU path restated) on this box's host
        # cores: one scale + PCA step over every cell of the same matrix
        import oracle
        oracle.build()
        threads = os.cpu_count() or 1
        f = cpu_prepare(indptr, indices, data, wl.n_genes, threads)
        dt = cpu_step(f)
        cpu = {"value": f.n_obs / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one scale+PCA step over all {f.n_obs} kept cells of this workload (FP64 Gram, "
                         f"LAPACK eigensolve, projection), the C port of the reference's Rust path"}
        del f

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic",
                "config": {"workload": workload_label(wl, n_gen), "gram": "split-BF16 (bf16x3) tcgen05",
                           "cells_after_qc": n_rows, "nnz": nnz, "hvg": P["d"], "l2": "inputs (12 GB) > L2",
                           "parallelism": f"dp{ws}" if ws > 1 else "1 GPU"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
                "kernels_ms_per_step": {kk: v[1] / max(1, args.steps) for kk, v in table.items()},
                "phases_ms": {"gram": stats["gram_ms"], "solve": stats["solve_ms"], "project": stats["project_ms"],
                              "eig_iters": stats["eig_iters"]},
                "generate_s": gen_s, "preprocess_s": prep_s}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return main_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
