// Memory-bound streaming passes over CSR chunks: QC sums (K1), lazy
// normalise + log1p + per-gene statistics (K2) and the score projection (K6).
//
// Layout: one warp per cell, grid-stride over the chunk's spans; every
// entry (4 B gene id + 4 B value) is read once from HBM with streaming
// loads, per-cell sums are formed in the reference's entry order
// (rowwarp.cuh), per-gene sums go to L2-resident accumulators.
#include "kernels.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {

// ----------------------------------------------------------------- QC (K1)
// src/kernels.rs:164-195.  Per kept cell: t = sum of non-zero values,
// n = their count, f = their sum over flagged genes; per mapped gene:
// ncells += 1, total += x.  Per-cell results go either to per-span slots
// (span_*; caller scatters) or are added at the cell's row (row_*).
__global__ void __launch_bounds__(256) k_qc(DevChunk c, const uint8_t *__restrict__ flag,
                                            uint32_t *__restrict__ gene_ncells,
                                            double *__restrict__ gene_total, int64_t *span_row_out,
                                            double *span_t, uint32_t *span_n, double *span_f,
                                            double *row_t, uint32_t *row_n, double *row_f) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        const int64_t row = span_row(c, i, lo, hi);
        if (row < 0) {
            if (span_row_out && lane == 0) span_row_out[i] = -1;
            continue;
        }
        const bool tf = c.target_sum > 0.0 || c.log1p;
        const double scale = tf ? cell_scale(c, lo, hi) : 1.0;
        OrderedSum t, f;
        uint32_t n = 0;
        for_entries<4>(c, lo, hi, [&](int32_t m, float x) {
            const float v = (tf && m >= 0) ? transform_value(c, scale, x) : x;
            const bool nz = m >= 0 && v != 0.0f;
            const bool fl = nz && flag[m];
            t.add(nz ? (double)v : 0.0);
            f.add(fl ? (double)v : 0.0);
            n += __popc(__ballot_sync(kFull, nz));
            if (nz) {
                atomicAdd(gene_ncells + m, 1u);
                atomicAdd(gene_total + m, (double)v);
            }
        });
        if (lane == 0) {
            if (span_row_out) {
                span_row_out[i] = row;
                span_t[i] = t.acc;
                span_n[i] = n;
                span_f[i] = f.acc;
            }
            if (row_t) {
                atomicAdd(row_t + row, t.acc);
                atomicAdd(row_n + row, n);
                atomicAdd(row_f + row, f.acc);
            }
        }
    }
}

// ----------------------------------------------------------- gene_stats (K2)
// src/kernels.rs:144-160.  out[m] += [x, x^2, expm1 x, expm1(x)^2, 1] of the
// transformed value x (f32 widened to f64).
__global__ void __launch_bounds__(256) k_gene_stats(DevChunk c, double *__restrict__ out) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        if (span_row(c, i, lo, hi) < 0) continue;
        const double scale = cell_scale(c, lo, hi);
        for_entries<4>(c, lo, hi, [&](int32_t m, float x) {
            if (m < 0) return;
            const double v = (double)transform_value(c, scale, x);
            const double ev = expm1(v);
            double *o = out + (size_t)m * 5;
            atomicAdd(o + 0, v);
            atomicAdd(o + 1, __dmul_rn(v, v));
            atomicAdd(o + 2, ev);
            atomicAdd(o + 3, __dmul_rn(ev, ev));
            atomicAdd(o + 4, 1.0);
        });
    }
}

// -------------------------------------------------------------- project (K6)
// src/kernels.rs:352-371.  For each kept cell: a[j] = sum over HVG entries
// (entry order) of s * V[sub, j] in f64 without fusing; out[row, j] += (f32)a[j].
// Lane l owns components l, l+32, ... (k <= 128).
template <int KPL>
__global__ void __launch_bounds__(256) k_project(DevChunk c, const int32_t *__restrict__ sub_map, DevScale t,
                                                 const double *__restrict__ V, int k, float *__restrict__ out,
                                                 int by_span) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        const int64_t row = span_row(c, i, lo, hi);
        if (row < 0) continue;
        const double scale = cell_scale(c, lo, hi);
        double acc[KPL];
#pragma unroll
        for (int q = 0; q < KPL; ++q) acc[q] = 0.0;
        for_entries<2>(c, lo, hi, [&](int32_t m, float x) {
            const int32_t sub = m >= 0 ? __ldg(sub_map + m) : -1;
            double s = 0.0;
            if (sub >= 0) s = scale_value(t, sub, transform_value(c, scale, x));
            unsigned mask = __ballot_sync(kFull, sub >= 0);
            while (mask) {
                const int src = __ffs(mask) - 1;
                mask &= mask - 1;
                const int32_t sj = __shfl_sync(kFull, sub, src);
                const double sv = __shfl_sync(kFull, s, src);
                const double *vr = V + (size_t)sj * k;
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int j = lane + 32 * q;
                    if (j < k) acc[q] = __dadd_rn(acc[q], __dmul_rn(sv, __ldg(vr + j)));
                }
            }
        });
        float *o = out + (size_t)(by_span ? i : row) * k;
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            const int j = lane + 32 * q;
            if (j < k) atomicAdd(o + j, __double2float_rn(acc[q]));
        }
    }
}

// ------------------------------------------------------------ launch glue
static int grid_for_spans(int64_t n_spans, int sms) {
    const int64_t warps_per_block = 8;
    int64_t blocks = ceil_div(n_spans, warps_per_block);
    const int64_t cap = (int64_t)sms * 16;  // grid-stride beyond 16 resident blocks per SM
    if (blocks > cap) blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

int launch_qc(const DevChunk &c, const uint8_t *flag, uint32_t *gene_ncells, double *gene_total,
              const SpanOut *span, const RowOut *row, cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    prof::Scope ps("qc_csr", st);
    k_qc<<<grid_for_spans(c.n_spans, device_sms()), 256, 0, st>>>(
        c, flag, gene_ncells, gene_total, span ? span->row : nullptr, span ? span->t : nullptr,
        span ? span->n : nullptr, span ? span->f : nullptr, row ? row->t : nullptr, row ? row->n : nullptr,
        row ? row->f : nullptr);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_gene_stats(const DevChunk &c, double *out, cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    prof::Scope ps("gene_stats_csr", st);
    k_gene_stats<<<grid_for_spans(c.n_spans, device_sms()), 256, 0, st>>>(c, out);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_project(const DevChunk &c, const int32_t *sub_map, const DevScale &t, const double *V, int k,
                   float *out, int by_span, cudaStream_t st) {
    if (c.n_spans == 0 || k == 0) return CREST_OK;
    CREST_REQUIRE(k <= 128, CREST_EINVAL, "project supports k <= 128 (got %d)", k);
    const int g = grid_for_spans(c.n_spans, device_sms());
    prof::Scope ps("project_csr", st);
    if (k <= 32)
        k_project<1><<<g, 256, 0, st>>>(c, sub_map, t, V, k, out, by_span);
    else if (k <= 64)
        k_project<2><<<g, 256, 0, st>>>(c, sub_map, t, V, k, out, by_span);
    else
        k_project<4><<<g, 256, 0, st>>>(c, sub_map, t, V, k, out, by_span);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// bias[g] = clip(-mean[g] / std[g]) (the scaled value of a zero entry).
__global__ void k_scale_bias(const double *mean, const double *std, double mv, int64_t d, double *bias) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < d) bias[g] = clip_mv(__ddiv_rn(-mean[g], std[g]), mv);
}

int launch_scale_bias(const double *mean, const double *std, double mv, int64_t d, double *bias, cudaStream_t st) {
    if (d == 0) return CREST_OK;
    k_scale_bias<<<(unsigned)ceil_div(d, 256), 256, 0, st>>>(mean, std, mv, d, bias);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
