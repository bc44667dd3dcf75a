// Gene-range sweeps of a device-resident CSR matrix whose rows are sorted by
// gene id: the per-gene sums of QC (K1) and gene_stats (K2) without global
// atomics per entry.
//
// A range index splits every row at the gene ids b * S (S = 2^log2_s genes
// per range, b = 1 .. R-1): off[cell][b-1] is the first entry of the row
// (relative to its start) whose gene is >= b * S.  One CTA owns a
// contiguous block of cells and visits the ranges in turn; for range r its
// warps read each cell's window [off[r-1], off[r]) once (coalesced, read
// once from HBM over the whole sweep) and add into per-gene accumulators of
// the S genes of the range held in shared memory; at the end of the range
// the block adds the accumulators to the global per-gene sums (one atomic
// per gene and statistic, instead of one per entry).
//
// Building the index reads every gene id once and also reports whether all
// rows are sorted; an unsorted matrix keeps the entry-parallel kernels of
// k_stream.cu.  The QC sweep needs integral values (raw counts, below
// 2^24): the per-cell sums are then exact in any order, so windows may be
// summed independently; otherwise it reports that and the caller reruns the
// entry-ordered kernel.
#include <algorithm>

#include "kernels.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {

// ------------------------------------------------------------ range index
// Warp per cell.  Entry e's range is min(g >> log2_s, R-1); where the range
// grows from the previous entry's (0 before the first entry) the
// boundaries in between start at e.  Boundaries past the last entry start
// at the row's end.  A descending gene id anywhere in a row sets bit 0 of
// *unsorted, a gene id equal to its predecessor's (a duplicate entry) bit 1.
__global__ void __launch_bounds__(256) k_range_index(const int64_t *__restrict__ indptr,
                                                     const uint32_t *__restrict__ genes, int64_t n_cells,
                                                     int log2_s, int n_ranges, int32_t *__restrict__ off,
                                                     int *unsorted) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    const int nb = n_ranges - 1;
    for (int64_t cell = warp; cell < n_cells; cell += n_warps) {
        const int64_t lo = indptr[cell], hi = indptr[cell + 1];
        int32_t *o = off + cell * nb;
        uint32_t carry_g = 0;  // gene of the previous entry
        int carry_r = 0;       // its range (0 before the first entry)
        bool have_prev = false, bad = false, dup = false;
        constexpr int U = 8;
        for (int64_t s = lo; s < hi; s += 32 * U) {
            uint32_t g[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t e = s + u * 32 + lane;
                g[u] = e < hi ? __ldcs(genes + e) : 0u;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t base = s + u * 32;
                if (base >= hi) break;  // warp-uniform
                const int64_t e = base + lane;
                const bool valid = e < hi;
                const int r = valid ? min((int)(g[u] >> log2_s), n_ranges - 1) : 0;
                const uint32_t gp = __shfl_up_sync(kFull, g[u], 1);
                const int rp_up = __shfl_up_sync(kFull, r, 1);
                const uint32_t prev_g = lane == 0 ? carry_g : gp;
                const int prev_r = lane == 0 ? carry_r : rp_up;
                const bool has_prev = lane == 0 ? have_prev : true;
                if (valid && has_prev && g[u] <= prev_g) {
                    bad = bad || g[u] < prev_g;
                    dup = dup || g[u] == prev_g;
                }
                if (valid)
                    for (int b = prev_r + 1; b <= r; ++b) o[b - 1] = (int32_t)(e - lo);
                const int last = hi - 1 - base < 31 ? (int)(hi - 1 - base) : 31;
                carry_g = __shfl_sync(kFull, g[u], last);
                carry_r = __shfl_sync(kFull, r, last);
                have_prev = true;
            }
        }
        for (int b = carry_r + 1 + lane; b <= nb; b += 32) o[b - 1] = (int32_t)(hi - lo);
        const bool any_bad = __any_sync(kFull, bad), any_dup = __any_sync(kFull, dup);
        if ((any_bad || any_dup) && lane == 0) atomicOr(unsorted, (any_bad ? 1 : 0) | (any_dup ? 2 : 0));
    }
}

// One cell's window of the current range: entries [a, b) of the chunk.
struct Win {
    int64_t span, a, b;
};

// Window of range r of a row of nnz entries.
__device__ __forceinline__ void range_window(const int32_t *o, int r, int n_ranges, int64_t nnz, int64_t &a,
                                             int64_t &b) {
    a = r == 0 ? 0 : (int64_t)__ldg(o + r - 1);
    b = r == n_ranges - 1 ? nnz : (int64_t)__ldg(o + r);
}

// Up to kWinU * 32 entries of a window in registers (lane-strided).
constexpr int kWinU = 8;
struct WinBuf {
    uint32_t g[kWinU];
    float x[kWinU];
};
__device__ __forceinline__ void win_load(const DevChunk &c, int64_t s, int64_t hi, WinBuf &w) {
    const int lane = lane_id();
#pragma unroll
    for (int u = 0; u < kWinU; ++u) {
        const int64_t e = s + u * 32 + lane;
        const bool v = e < hi;
        w.g[u] = v ? __ldcs(c.genes + e) : 0u;
        w.x[u] = v ? __ldcs(c.values + e) : 0.0f;
    }
}

// Every window of range r of this warp's cells [c0 + warp, c1) (step
// n_warps): cell(w) once per window before its entries, entry(g, x, valid)
// for every lane of each 32-entry group, done(w) after them.  The windows'
// bounds are fetched 32 cells at a time (lane j reads the row bounds, the
// cell map and the range offsets of the j-th next cell of this warp, one
// round trip for 32 windows instead of three dependent loads per window),
// and the first kWinU * 32 entries of the next window are loaded before the
// current one is processed, so each warp keeps two windows of loads in
// flight.
template <class C, class E, class D>
__device__ __forceinline__ void sweep_range(const DevChunk &c, const RangeIndex &ix, int r, int64_t c0, int64_t c1,
                                            C &&cell, E &&entry, D &&done) {
    const int lane = lane_id();
    const int64_t step = blockDim.x >> 5;
    constexpr int64_t kSpan = kWinU * 32;
    int64_t batch = c0 + (threadIdx.x >> 5);  // this warp's first cell of the current batch
    int64_t m_span = 0, m_a = 0, m_b = 0;     // this lane's window of the batch
    unsigned pending = 0;                      // lanes whose windows are still to be visited
    auto fetch = [&]() {
        const int64_t i = batch + lane * step;
        bool ok = false;
        if (i < c1) {
            int64_t lo, hi;
            if (span_row(c, i, lo, hi) >= 0) {
                int64_t a, b;
                range_window(ix.off + (c.first_cell + i) * (ix.n_ranges - 1), r, ix.n_ranges, hi - lo, a, b);
                m_span = i;
                m_a = lo + a;
                m_b = lo + b;
                ok = true;
            }
        }
        pending = __ballot_sync(kFull, ok);
    };
    auto next = [&](Win &w) -> bool {
        for (;;) {
            if (pending) {
                const int j = __ffs(pending) - 1;
                pending &= pending - 1;
                w.span = __shfl_sync(kFull, m_span, j);
                w.a = __shfl_sync(kFull, m_a, j);
                w.b = __shfl_sync(kFull, m_b, j);
                return true;
            }
            batch += 32 * step;
            if (batch >= c1) return false;
            fetch();
        }
    };
    if (batch < c1) fetch();
    Win cur, nxt;
    WinBuf bc, bn;
    bool have = next(cur);
    if (have) win_load(c, cur.a, cur.b < cur.a + kSpan ? cur.b : cur.a + kSpan, bc);
    while (have) {
        const bool hn = next(nxt);
        if (hn) win_load(c, nxt.a, nxt.b < nxt.a + kSpan ? nxt.b : nxt.a + kSpan, bn);
        cell(cur);
        for (int64_t s = cur.a; s < cur.b; s += kSpan) {
            if (s != cur.a) win_load(c, s, cur.b, bc);  // windows longer than kSpan (rare)
#pragma unroll
            for (int u = 0; u < kWinU; ++u) {
                if (s + u * 32 >= cur.b) break;  // warp-uniform
                entry(bc.g[u], bc.x[u], s + u * 32 + lane < cur.b);
            }
        }
        done(cur);
        if (hn) {
            cur = nxt;
#pragma unroll
            for (int u = 0; u < kWinU; ++u) {
                bc.g[u] = bn.g[u];
                bc.x[u] = bn.x[u];
            }
        }
        have = hn;
    }
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Cells [c0, c1) of the piece for this CTA: an even split of the spans.
__device__ __forceinline__ void cta_cells(int64_t n_spans, int64_t &c0, int64_t &c1) {
    c0 = n_spans * (int64_t)blockIdx.x / gridDim.x;
    c1 = n_spans * (int64_t)(blockIdx.x + 1) / gridDim.x;
}

// ------------------------------------------------------------------- QC
// src/kernels.rs:164-195 for integral values.  Shared memory: per gene of
// the current range the count and the integer total as two u32 sums, one of
// the low and one of the high 16 bits of each value (values are below 2^24,
// a CTA holds at most 65,536 cells, so neither sum can wrap and the total is
// hi * 2^16 + lo exactly), then per-cell (t, f, n) of the CTA's cells.  Only
// 32-bit integer shared-memory atomics without a return value are used (the
// fast ones on this part); per-cell sums are integer lane sums.
// status bit 1: a non-integral value was seen.
constexpr int32_t kQcFlagBit = 1 << 30;  // kept gene indices stay below 2^30

__global__ void __launch_bounds__(kSweepThreads, 1)
    k_qc_sweep(DevChunk c, RangeIndex ix, const uint8_t *__restrict__ flag, uint32_t *__restrict__ gene_ncells,
               double *__restrict__ gene_total, RowOut ro, int *status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = 1 << ix.log2_s;
    uint32_t *s_lo = reinterpret_cast<uint32_t *>(smem);  // [S] sum of the low 16 bits
    uint32_t *s_hi = s_lo + S;                             // [S] sum of the high bits
    uint32_t *s_cnt = s_hi + S;                            // [S]
    // [S] gene_map of the range with the flag of the mapped gene in bit 30
    // (-1: dropped), one shared-memory read per entry for both
    int32_t *s_map = reinterpret_cast<int32_t *>(s_cnt + S);
    int64_t c0, c1;
    cta_cells(c.n_spans, c0, c1);
    const int64_t nc = c1 - c0;
    double *s_t = reinterpret_cast<double *>(s_map + S);     // [nc]
    double *s_f = s_t + nc;                                   // [nc]
    uint32_t *s_n = reinterpret_cast<uint32_t *>(s_f + nc);  // [nc]
    const int lane = lane_id();
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
        s_lo[i] = 0u;
        s_hi[i] = 0u;
        s_cnt[i] = 0u;
    }
    for (int64_t i = threadIdx.x; i < nc; i += blockDim.x) {
        s_t[i] = 0.0;
        s_f[i] = 0.0;
        s_n[i] = 0u;
    }
    __syncthreads();
    bool non_integral = false;
    for (int r = 0; r < ix.n_ranges; ++r) {
        const uint32_t g0 = (uint32_t)r << ix.log2_s;
        for (int i = threadIdx.x; i < S; i += blockDim.x) {
            const int64_t g = (int64_t)g0 + i;
            const int32_t m = g < c.n_gene_map ? __ldg(c.gene_map + g) : -1;
            s_map[i] = m >= 0 && flag[m] ? (m | kQcFlagBit) : m;
        }
        __syncthreads();
        uint64_t ts = 0, fs = 0;
        uint32_t n = 0;
        sweep_range(
            c, ix, r, c0, c1,
            [&](const Win &) {
                ts = 0;
                fs = 0;
                n = 0;
            },
            [&](uint32_t g, float x, bool valid) {
                const int j = (int)(g - g0);  // in [0, S) for a sorted row (any g < n_gene_map)
                const int32_t m = valid && (int64_t)g < c.n_gene_map ? s_map[j] : -1;
                if (m < 0 || x == 0.0f) return;
                const bool ok = x > 0.0f && x < 16777216.0f && x == rintf(x);
                non_integral = non_integral || !ok;
                const uint32_t xi = ok ? (uint32_t)x : 0u;
                ts += xi;
                if (m & kQcFlagBit) fs += xi;
                n += 1;
                atomicAdd(s_cnt + j, 1u);
                atomicAdd(s_lo + j, xi & 0xffffu);
                if (xi >> 16) atomicAdd(s_hi + j, xi >> 16);
            },
            [&](const Win &w) {
                const double t = (double)warp_sum_u64(ts), f = (double)warp_sum_u64(fs);
                const uint32_t k = __reduce_add_sync(kFull, n);
                if (lane == 0 && k) {  // one warp per cell: no race
                    const int64_t j = w.span - c0;
                    s_t[j] += t;
                    s_f[j] += f;
                    s_n[j] += k;
                }
            });
        __syncthreads();
        for (int i = threadIdx.x; i < S; i += blockDim.x) {
            const uint32_t k = s_cnt[i];
            if (k) {
                const int32_t m = s_map[i] & ~kQcFlagBit;  // counted entries have a mapped gene
                atomicAdd(gene_ncells + m, k);
                atomicAdd(gene_total + m, (double)(((uint64_t)s_hi[i] << 16) + s_lo[i]));
                s_cnt[i] = 0u;
                s_lo[i] = 0u;
                s_hi[i] = 0u;
            }
        }
        __syncthreads();
    }
    for (int64_t i = threadIdx.x; i < nc; i += blockDim.x) {
        int64_t lo, hi;
        const int64_t row = span_row(c, c0 + i, lo, hi);
        if (row < 0) continue;
        atomicAdd(ro.t + row, s_t[i]);
        atomicAdd(ro.n + row, s_n[i]);
        atomicAdd(ro.f + row, s_f[i]);
    }
    if (__any_sync(kFull, non_integral) && lane == 0) atomicOr(status, 1);
}

// ------------------------------------------------------------ gene_stats
// src/kernels.rs:144-160 with the per-cell totals over kept genes given
// (total[span]).  Shared memory per gene of the range: [x, x^2, expm1 x,
// expm1(x)^2] f64 and the entry count.  Entries of dropped genes are
// accumulated and discarded at the flush (no per-entry map lookup).
__global__ void __launch_bounds__(kSweepThreads, 1)
    k_gene_stats_sweep(DevChunk c, RangeIndex ix, const double *__restrict__ total, double *__restrict__ out) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = 1 << ix.log2_s;
    double *s_x = reinterpret_cast<double *>(smem);  // [4][S]
    uint32_t *s_cnt = reinterpret_cast<uint32_t *>(s_x + 4 * S);
    int64_t c0, c1;
    cta_cells(c.n_spans, c0, c1);
    for (int i = threadIdx.x; i < 4 * S; i += blockDim.x) s_x[i] = 0.0;
    for (int i = threadIdx.x; i < S; i += blockDim.x) s_cnt[i] = 0u;
    __syncthreads();
    for (int r = 0; r < ix.n_ranges; ++r) {
        const uint32_t g0 = (uint32_t)r << ix.log2_s;
        double scale = 1.0;
        sweep_range(
            c, ix, r, c0, c1,
            [&](const Win &w) {
                const double tot = c.target_sum > 0.0 ? __ldg(total + w.span) : 0.0;
                scale = tot > 0.0 ? c.target_sum / tot : 1.0;
            },
            [&](uint32_t g, float x, bool valid) {
                if (!valid || (int64_t)g >= c.n_gene_map) return;
                const double v = (double)transform_value(c, scale, x);
                const double ev = expm1(v);
                const int j = (int)(g - g0);
                atomicAdd(s_x + j, v);
                atomicAdd(s_x + S + j, __dmul_rn(v, v));
                atomicAdd(s_x + 2 * S + j, ev);
                atomicAdd(s_x + 3 * S + j, __dmul_rn(ev, ev));
                atomicAdd(s_cnt + j, 1u);
            },
            [&](const Win &) {});
        __syncthreads();
        for (int i = threadIdx.x; i < S; i += blockDim.x) {
            const uint32_t k = s_cnt[i];
            if (!k) continue;
            const int32_t m = __ldg(c.gene_map + (int64_t)g0 + i);
            if (m >= 0) {
                double *o = out + (size_t)m * 5;
                atomicAdd(o + 0, s_x[i]);
                atomicAdd(o + 1, s_x[S + i]);
                atomicAdd(o + 2, s_x[2 * S + i]);
                atomicAdd(o + 3, s_x[3 * S + i]);
                atomicAdd(o + 4, (double)k);
            }
            s_x[i] = s_x[S + i] = s_x[2 * S + i] = s_x[3 * S + i] = 0.0;
            s_cnt[i] = 0u;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ cell totals
// Per-span total of the kept-gene values (the normalisation total of
// src/kernels.rs:63-78): integral fast path, else the in-order f64 fold.
// Whether a gene is kept is read from a bit set in shared memory (one bit
// per store gene): a gather from the gene map in L1 costs about one cache
// wavefront per entry, the bit set a few bank cycles per 32 entries.
__global__ void __launch_bounds__(256) k_cell_totals(DevChunk c, double *__restrict__ total) {
    extern __shared__ uint32_t s_keep[];
    const int64_t n_words = (c.n_gene_map + 31) >> 5;
    for (int64_t w = threadIdx.x; w < n_words; w += blockDim.x) {
        uint32_t bits = 0;
        for (int b = 0; b < 32; ++b) {
            const int64_t g = (w << 5) + b;
            if (g < c.n_gene_map && __ldg(c.gene_map + g) >= 0) bits |= 1u << b;
        }
        s_keep[w] = bits;
    }
    __syncthreads();
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        span_row(c, i, lo, hi);
        uint64_t s = 0;  // exact while every kept value is an integer in [0, 2^24)
        bool ok = true;
        for_entries_x4<true>(c, lo, hi, [&](uint32_t g) { return ((s_keep[g >> 5] >> (g & 31)) & 1u) ? 0 : -1; },
                             [&](const int32_t (&m)[4], const float (&x)[4]) {
#pragma unroll
                                 for (int u = 0; u < 4; ++u) {
                                     if (m[u] < 0) continue;
                                     ok = ok && x[u] >= 0.0f && x[u] < 16777216.0f && x[u] == rintf(x[u]);
                                     s += (uint32_t)fminf(fmaxf(x[u], 0.0f), 16777215.0f);
                                 }
                             });
        double t;
        if (__all_sync(kFull, ok)) {
            t = (double)warp_sum_u64(s);
        } else {
            OrderedSum tot;
            for_entries<4, false>(c, lo, hi, [&](int32_t m, float x) { tot.add(m >= 0 ? (double)x : 0.0); });
            t = tot.acc;
        }
        if (lane == 0) total[i] = t;
    }
}

// ------------------------------------------------------------- launchers
int launch_range_index(const int64_t *indptr, const uint32_t *genes, int64_t n_cells, int log2_s, int n_ranges,
                       int32_t *off, int *unsorted, cudaStream_t st) {
    if (n_cells == 0 || n_ranges < 2) return CREST_OK;
    prof::Scope ps("range_index_csr", st);
    const int blocks = (int)std::min<int64_t>(ceil_div(n_cells, 8), (int64_t)device_sms() * 8);
    k_range_index<<<blocks, 256, 0, st>>>(indptr, genes, n_cells, log2_s, n_ranges, off, unsorted);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

size_t qc_sweep_smem(int log2_s, int64_t cells_per_cta) {
    return (size_t)(1 << log2_s) * 16 + (size_t)cells_per_cta * 20;
}

int sweep_ctas(int64_t n_spans, int64_t cell_cap) {
    int64_t p = device_sms();
    if (cell_cap > 0 && ceil_div(n_spans, p) > cell_cap) p = ceil_div(n_spans, cell_cap);
    if (p > n_spans) p = n_spans;
    return (int)(p < 1 ? 1 : p);
}

int launch_qc_sweep(const DevChunk &c, const RangeIndex &ix, const uint8_t *flag, uint32_t *gene_ncells,
                    double *gene_total, const RowOut &row, int *status, cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    CREST_REQUIRE(c.n_gene_map < kQcFlagBit, CREST_EINVAL, "QC sweep: at most 2^30 genes");
    const int64_t cap = std::min<int64_t>(((int64_t)kMaxSmem - (int64_t)(1 << ix.log2_s) * 16) / 20, 65536);
    const int ctas = sweep_ctas(c.n_spans, cap);
    const size_t smem = qc_sweep_smem(ix.log2_s, ceil_div(c.n_spans, ctas));
    CREST_REQUIRE(smem <= (size_t)kMaxSmem, CREST_EINVAL, "QC sweep: %zu B of shared memory", smem);
    CREST_TRY(ensure_smem_attr((const void *)k_qc_sweep, smem));
    prof::Scope ps("qc_csr", st);
    k_qc_sweep<<<ctas, kSweepThreads, smem, st>>>(c, ix, flag, gene_ncells, gene_total, row, status);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_gene_stats_sweep(const DevChunk &c, const RangeIndex &ix, const double *total, double *out,
                            cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    const size_t smem = (size_t)(1 << ix.log2_s) * 36;
    CREST_REQUIRE(smem <= (size_t)kMaxSmem, CREST_EINVAL, "gene_stats sweep: %zu B of shared memory", smem);
    CREST_TRY(ensure_smem_attr((const void *)k_gene_stats_sweep, smem));
    prof::Scope ps("gene_stats_csr", st);
    k_gene_stats_sweep<<<sweep_ctas(c.n_spans, 0), kSweepThreads, smem, st>>>(c, ix, total, out);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_cell_totals(const DevChunk &c, double *total, cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    const size_t smem = sizeof(uint32_t) * (size_t)ceil_div(c.n_gene_map, 32);
    CREST_REQUIRE(smem <= (size_t)kMaxSmem, CREST_EINVAL, "cell totals: %lld genes need a larger bit set",
                  (long long)c.n_gene_map);
    CREST_TRY(ensure_smem_attr((const void *)k_cell_totals, smem));
    prof::Scope ps("cell_totals_csr", st);
    const int blocks = (int)std::min<int64_t>(ceil_div(c.n_spans, 8), (int64_t)device_sms() * 8);
    k_cell_totals<<<blocks, 256, smem, st>>>(c, total);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
