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
    ap.add_argument("--no-fused", action="store_true")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the timed bf16x3 steps (for profiler launch lists): no CPU baseline, no FP32 / FP64 "
                         "legs, no memory-bound passes, no e2e")
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


def subspace_angle_deg(A, B):
    """Largest principal angle (degrees) between the column spaces of A and B."""
    qa, _ = np.linalg.qr(np.asarray(A, np.float64))
    qb, _ = np.linalg.qr(np.asarray(B, np.float64))
    return float(np.degrees(np.arccos(np.clip(np.linalg.svd(qa.T @ qb, compute_uv=False), -1, 1))).max())


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
    if args.kernels_only:
        args.no_cpu = args.no_fp32 = args.no_fused = True
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

    L2_BYTES = 126 << 20
    csr_bytes = nnz * 8 + (len(indptr)) * 8
    l2_flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda") if csr_bytes < 2 * L2_BYTES else None
    l2_note = (f"inputs ({csr_bytes / 1e9:.2f} GB) > L2" if l2_flush is None else
               f"L2 flushed before every timed step (inputs {csr_bytes / 1e6:.0f} MB)")

    def timed(precision, steps, warmup, profile=False, mark=False, keep_scores=False):
        plan = tl.PcaPlan(P["d"], precision)
        for _ in range(warmup):
            plan.reset()
            step(plan)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        if profile:
            _lib.profile_enable(True)
        # K steps timed as one interval, bracketed by a barrier and a sync; a
        # matrix smaller than L2 is timed step by step with L2 flushed in between
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        if mark:  # an NVTX range around the timed steps, for a profiler to select them
            torch.cuda.nvtx.range_push("crest_step")
        if l2_flush is None:
            e0.record()
            for _ in range(steps):
                plan.reset()
                step(plan)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
        else:
            tot = 0.0
            for _ in range(steps):
                l2_flush.zero_()
                e0.record()
                plan.reset()
                step(plan)
                e1.record()
                torch.cuda.synchronize()
                tot += e0.elapsed_time(e1)
            ms = tot / steps
        if mark:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        table = _lib.profile_table() if profile else {}
        if profile:
            _lib.profile_enable(False)
        stats = plan.stats()
        variance, loadings, total, _ = plan.results()
        plan.close()
        if dist is not None:
            mt = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(mt, op=dist.ReduceOp.MAX)
            ms = float(mt.item())
        res = {"ms": ms, "stats": stats, "table": table, "loadings": loadings, "variance_ratio": variance / total,
               "variance": variance}
        if keep_scores:
            res["X"] = X.cpu().numpy()
        return res

    want_parity = rank == 0 and ws == 1 and not args.no_cpu
    peaks = measured_peaks()
    with ClockSampler(local) as clk:
        r_bf = timed("bf16x3", args.steps, args.warmup, mark=True, keep_scores=want_parity)
    ms, stats = r_bf["ms"], r_bf["stats"]
    clocks = clk.summary()
    value = n_rows * ws / (ms / 1e3)

    extra = {}
    # per-kernel device times: the same K steps again with a CUDA-event scope
    # around every launch (on its stream); the scopes' host cost makes this
    # pass a little slower, so the headline value comes from the pass above
    r_prof = timed("bf16x3", args.steps, 1, profile=True)
    table = r_prof["table"]
    extra["ms_per_step_profiled"] = r_prof["ms"]
    r_32 = None
    if not args.no_fp32:
        r_32 = timed("fp32", max(2, args.steps // 2), 1, keep_scores=want_parity)
        extra["fp32_cells_per_s"] = n_rows * ws / (r_32["ms"] / 1e3)
        extra["fp32_ms_per_step"] = r_32["ms"]
        extra["speedup_bf16x3_vs_fp32"] = r_32["ms"] / ms
        # the Gram phase is the only part that differs between the two forms
        extra["speedup_gram_bf16x3_vs_fp32"] = r_32["stats"]["gram_ms"] / stats["gram_ms"]
    if args.kernels_only:
        print(json.dumps({"metric": METRIC, "value": n_rows * ws / (ms / 1e3), "unit": UNIT, "n_gpus": ws,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "kernels_ms_per_step": {kk: vv[1] / args.steps for kk, vv in table.items()},
                          "note": "kernels-only run"}))
        return 0
    # accuracy of the product and plain forms against the FP64 Gram of the same run
    r_64 = timed("fp64", 1, 0, keep_scores=want_parity)
    extra["max_principal_angle_deg_vs_fp64"] = subspace_angle_deg(r_bf["loadings"], r_64["loadings"])
    if r_32 is not None:
        extra["fp32_max_principal_angle_deg_vs_fp64"] = subspace_angle_deg(r_32["loadings"], r_64["loadings"])

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
    pass_bytes = {"qc_csr": bytes_pass, "gene_stats_csr": bytes_pass, "gene_stats_csc": bytes_pass,
                  "cell_totals_csr": bytes_pass,
                  "range_index_csr": nnz * 4 + len(indptr) * 8 + (len(indptr) - 1) * (n_ranges - 1) * 4}
    for kname, byts in pass_bytes.items():
        tb = tb_mem if kname in tb_mem else tb_prep
        if kname in tb:
            n_l, tot, mx = tb[kname]
            hbm[kname] = byts / (tot / n_l / 1e3) / 1e9
    if "extract_csr" in table:  # one CSR read per step, in launches of one upload chunk each
        n_l, tot, mx = table["extract_csr"]
        hbm["extract_csr"] = bytes_pass / (tot / max(1, args.steps) / 1e3) / 1e9
    if "densify" in table:  # the bf16 hi/lo tile rows written per step (compact-form reads not counted)
        n_l, tot, mx = table["densify"]
        d_pad = -(-P["d"] // 256) * 256
        hbm["densify_tile"] = n_rows * d_pad * 4 / (tot / max(1, args.steps) / 1e3) / 1e9
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
    def e2e_run(residency, host_in, host_out, reps=5):
        h_indptr, h_indices, h_data = host_in
        times, dev_bytes, Xh = [], 0, None
        phases = []
        for i in range(reps + 1):
            torch.cuda.synchronize()
            _lib.memory_stats(reset_high=True)
            base = _lib.memory_stats()[0]  # device memory the bench itself still holds
            t0 = time.perf_counter()
            m = cb.core.DeviceMatrix(h_indptr, h_indices, h_data, wl.n_genes, residency, chunk_cells=16384)
            t1 = time.perf_counter()
            plan = tl.PcaPlan(P["d"], "bf16x3")
            plan.accumulate(m, P["cmap"], P["gmap"], P["target"], P["log"], P["sub"], P["n_vars"], P["scale"])
            t2 = time.perf_counter()
            plan.solve(n_rows, k)
            t3 = time.perf_counter()
            Xh = plan.project(m, P["cmap"], P["gmap"], P["target"], P["log"], P["sub"], P["n_vars"], P["scale"],
                              n_rows, out=host_out)
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            dt = t4 - t0
            phases.append([t1 - t0, t2 - t1, t3 - t2, t4 - t3])
            dev_bytes = max(dev_bytes, _lib.memory_stats()[1] - base)
            plan.close()
            m.close()
            if i > 0:  # the first run is a warm-up
                times.append(dt)
        te = float(np.median(times))
        passes = 1  # streamed too: the projection reads the HVG entries the Gram pass packed on the device
        h2d = passes * (nnz * 8) + len(indptr) * 8 + 2 * P["cmap"].nbytes + 2 * P["gmap"].nbytes
        return {"value": n_rows * ws / te, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(Xh.nbytes), "ms_per_step": te * 1e3, "repeats": reps,
                "statistic": "median of the repeats", "host_inputs": "pinned",
                "ms_min": min(times) * 1e3, "ms_max": max(times) * 1e3, "residency": residency,
                "device_bytes": int(dev_bytes), "h2d_gbs_effective": h2d / te / 1e9,
                "phases_ms": dict(zip(["create", "accumulate", "solve", "project_and_read_back"],
                                      [round(float(np.median([p[j] for p in phases[1:]])) * 1e3, 2)
                                       for j in range(4)]))}

    e2e = e2e_streamed = pcie = None
    if rank == 0 or ws > 1:
        # the step's inputs live in pinned host memory (copied there once,
        # outside the timed region, as a serving process would hold them)
        host_in = tuple(torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
                        for a in (indptr, indices, data))
        # and the result is read back into a pinned buffer the caller reuses
        host_out = torch.empty((n_rows, k), dtype=torch.float32, pin_memory=True).numpy()
        e2e = e2e_run("device", host_in, host_out)
        e2e_streamed = e2e_run("host", host_in, host_out)
        del host_in, host_out
        chunk_bytes = max(int(indptr[min(i + 16384, n_gen)] - indptr[i]) for i in range(0, n_gen, 16384)) * 8
        e2e_streamed["chunk_bytes_max"] = chunk_bytes
        e2e_streamed["model"] = ("pinned host CSR, 16,384-cell chunks, two device buffers, copies on a second "
                                 "stream overlapped with the kernels; the Gram pass also packs each chunk's HVG "
                                 "entries (room for a quarter of the stored entries) so the projection does not "
                                 "stream the CSR again; device memory = two chunks + the packed HVG entries + the "
                                 "d x d Gram, its second-half copy and the eigensolver workspace")
        # H2D bandwidth of this box (pinned, one 1 GiB copy, CUDA events)
        hb = torch.empty(1 << 30, dtype=torch.uint8, pin_memory=True)
        db = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
        db.copy_(hb, non_blocking=True)
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record()
        for _ in range(3):
            db.copy_(hb, non_blocking=True)
        eb.record()
        torch.cuda.synchronize()
        pcie = 3 * (1 << 30) / (ea.elapsed_time(eb) / 1e3) / 1e9
        e2e_streamed["pcie_h2d_gbs_measured"] = pcie
        del hb, db

    cpu = parity = None
    if want_parity:
        # the oracle (the reference's CPU path restated) on this box's host
        # cores, on the same matrix: its preprocessing (untimed) checks the
        # GPU's QC / HVG results; one scale + PCA step over every kept cell
        # is the CPU baseline and the FP64 reference of the scores
        import oracle
        oracle.build()
        threads = os.cpu_count() or 1
        from oracle import pipeline as op
        f_raw = op.Frame(indptr, indices, data, wl.n_genes, synth.gene_names(wl.n_genes), threads=threads)
        oobs, ovar = op.qc_metrics(f_raw)
        gobs, gvar = pp.calculate_qc_metrics(cb.BioFrame.from_csr(indptr, indices, data, wl.n_genes,
                                                                  var=pd.DataFrame({"gene_name": names})),
                                             inplace=False)
        f = cpu_prepare(indptr, indices, data, wl.n_genes, threads)
        dt = cpu_step(f)
        cpu = {"value": f.n_obs / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"one scale+PCA step over all {f.n_obs} kept cells of this workload (FP64 Gram, "
                         f"LAPACK eigensolve, projection), the C port of the reference's Rust path"}
        parity = parity_block(bf, f, gobs, gvar, oobs, ovar, {"bf16x3": r_bf, "fp32": r_32, "fp64": r_64})
        del f, f_raw

    fused = None
    if rank == 0 and not args.no_fused:
        fused = fused_leg(torch, peaks)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic",
                "config": {"workload": workload_label(wl, n_gen), "gram": "split-BF16 (bf16x3) tcgen05",
                           "cells_after_qc": n_rows, "nnz": nnz, "hvg": P["d"], "l2": l2_note,
                           "gram_tile_cells": min(int(os.environ.get("CREST_TILE_CELLS", 262144)), n_rows),
                           "parallelism": f"dp{ws}" if ws > 1 else "1 GPU"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_streamed": e2e_streamed,
                "gpu_launches": launches, "clocks": clocks,
                "kernels_ms_per_step": {kk: v[1] / max(1, args.steps) for kk, v in table.items()},
                "phases_ms": {"gram": stats["gram_ms"], "solve": stats["solve_ms"], "project": stats["project_ms"],
                              "eig_iters": stats["eig_iters"]},
                "parity_vs_oracle": parity, "differentiation": fused,
                "generate_s": gen_s, "preprocess_s": prep_s, "native_so_loaded": repo_libs_mapped()}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def parity_block(bf, f, gobs, gvar, oobs, ovar, runs):
    """The GPU run against the oracle on the same 1M-cell matrix: QC integers,
    kept sets and the HVG set (bit-exact), dispersions_norm, and per Gram form
    the principal angles / score error / variance-ratio error of the scores."""
    from oracle import pipeline as op
    out = {"qc_equal": all(np.array_equal(gobs[c].to_numpy(), oobs[c]) for c in
                           ("n_genes_by_counts", "total_counts", "pct_counts_mt")) and
           all(np.array_equal(gvar[c].to_numpy(), ovar[c]) for c in ("n_cells_by_counts", "total_counts")),
           "kept_cells_equal": bool(np.array_equal(bf.obs["cell_id"].to_numpy(), f.cell_ids)),
           "kept_genes_equal": bool(np.array_equal(bf.var["gene_id"].to_numpy(), f.gene_ids)),
           "hvg_equal": bool(np.array_equal(bf.var["highly_variable"].to_numpy(),
                                            np.asarray(f.var["highly_variable"])))}
    dn, odn = bf.var["dispersions_norm"].to_numpy(), np.asarray(f.var["dispersions_norm"])
    ok = ~np.isnan(odn)
    out["dispersions_norm_max_abs_err"] = float(np.max(np.abs(dn[ok] - odn[ok]))) if ok.any() else 0.0
    R = f.obsm["X_pca"].astype(np.float64)
    ovr = f.uns["pca"]["variance"]
    for name, r in runs.items():
        if r is None or "X" not in r:
            continue
        X = r["X"].astype(np.float64)
        s = np.sign((X * R).sum(0))
        s[s == 0] = 1
        err = np.linalg.norm(X * s - R, axis=0) / np.linalg.norm(R, axis=0)
        v = np.asarray(ovr, np.float64)
        gaps = np.full(len(v), np.inf)
        gaps[:-1] = np.minimum(gaps[:-1], (v[:-1] - v[1:]) / v[:-1])
        gaps[1:] = np.minimum(gaps[1:], (v[:-1] - v[1:]) / v[:-1])
        sep = gaps >= 2e-3
        out[name] = {"max_principal_angle_deg": float(op.principal_angles_deg(X, R).max()),
                     "score_rel_err_separated_max": float(err[sep].max()) if sep.any() else None,
                     "separated_components": int(sep.sum()),
                     "variance_rel_err_max": float(np.max(np.abs(r["variance"] - v) / v))}
    return out


def fused_leg(torch, peaks):
    """The differentiation workload (50,000 cells x 2,000 HVG genes, ~200
    stored entries per cell, k = 50): fused forward and backward through the
    autograd Function, CUDA events over 5 repeats after 2 warm-ups."""
    from crest_b200 import synth
    from crest_b200.autograd import fused_scale_project
    n, d, k = 50_000, 2_000, 50
    p = synth.make_params(n, d, 20, 0.2, 200.0, seed=41)
    indptr, indices, data = synth.generate(p)
    rng = np.random.default_rng(42)
    sf = np.exp(rng.normal(0.0, 0.3, n)).astype(np.float32)
    W = np.linalg.qr(rng.standard_normal((d, k)))[0].astype(np.float32)
    cell = np.repeat(np.arange(n), np.diff(indptr))
    lg = np.log1p(data.astype(np.float64) / sf[cell])
    mean = np.bincount(indices, lg, d) / n
    std = np.sqrt(np.maximum((np.bincount(indices, lg * lg, d) - n * mean * mean) / (n - 1), 0.0))
    std[std == 0] = 1.0
    dev = torch.device("cuda")
    tv = torch.tensor(data, device=dev, requires_grad=True)
    ts = torch.tensor(sf, device=dev, requires_grad=True)
    tw = torch.tensor(W, device=dev, requires_grad=True)
    ti, tx = torch.tensor(indptr, device=dev), torch.tensor(indices.astype(np.int32), device=dev)
    tm, tsd = torch.tensor(mean, device=dev), torch.tensor(std, device=dev)
    g = torch.tensor(rng.standard_normal((n, k)).astype(np.float32), device=dev)
    fwd, bwd = [], []
    for i in range(7):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        out = fused_scale_project(tv, ts, tw, ti, tx, tm, tsd, 10.0)
        e[1].record()
        out.backward(g)
        e[2].record()
        torch.cuda.synchronize()
        if i >= 2:
            fwd.append(e[0].elapsed_time(e[1]))
            bwd.append(e[1].elapsed_time(e[2]))
        tv.grad = ts.grad = tw.grad = None
    nnz = int(indptr[-1])
    # algorithmic bytes: CSR (8 B per entry + indptr), size factors, W, mean/std, scores
    b_fwd = nnz * 8 + (n + 1) * 8 + n * 4 + d * k * 4 + d * 16 + n * k * 4
    b_bwd = b_fwd + nnz * 4 + n * 4 + d * k * 4  # + value, size-factor and W gradients
    f_ms, b_ms = float(np.median(fwd)), float(np.median(bwd))
    return {"workload": f"{n} cells x {d} HVG genes, {nnz} stored entries, k={k}",
            "forward_ms": f_ms, "backward_ms": b_ms,
            "forward_hbm_frac": b_fwd / (f_ms / 1e3) / 1e9 / peaks["hbm_gbs"],
            "backward_hbm_frac": b_bwd / (b_ms / 1e3) / 1e9 / peaks["hbm_gbs"],
            "note": "backward = per-gene entry histogram and scan, the entry pass (value and size-factor "
                    "gradients, each entry's scaled value and cell written into its gene's segment) and the "
                    "block-per-gene W gradient; bytes are the algorithmic minimum"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return main_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
