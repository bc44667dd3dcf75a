// Memory-bound streaming passes over CSR chunks: QC sums (K1), lazy
// normalise + log1p + per-gene statistics (K2) and the score projection (K6).
//
// Layout: one warp per cell, grid-stride over the chunk's spans; every
// entry (4 B gene id + 4 B value) is read once from HBM with streaming
// loads, per-cell sums are formed in the reference's entry order
// (rowwarp.cuh), per-gene sums go to L2-resident accumulators.
#include <type_traits>

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
        double t_acc = 0.0, f_acc = 0.0;
        uint32_t n = 0;
        if (!tf) {
            // raw values: lane-private sums, exact (hence order-free) when
            // every non-zero value is an integer below 2^24
            double ts = 0.0, fs = 0.0;
            bool ok = true;
            for_entries<8>(c, lo, hi, [&](int32_t m, float x) {
                if (m < 0 || x == 0.0f) return;
                const double v = (double)x;
                ok = ok && small_integer(v);
                ts += v;
                if (flag[m]) fs += v;
                n += 1;
                atomicAdd(gene_ncells + m, 1u);
                atomicAdd(gene_total + m, v);
            });
            n = __reduce_add_sync(kFull, n);
            if (__all_sync(kFull, ok)) {
                t_acc = warp_sum(ts);
                f_acc = warp_sum(fs);
            } else {  // in entry order
                OrderedSum t, f;
                for_entries<4>(c, lo, hi, [&](int32_t m, float x) {
                    const bool nz = m >= 0 && x != 0.0f;
                    t.add(nz ? (double)x : 0.0);
                    f.add(nz && flag[m] ? (double)x : 0.0);
                });
                t_acc = t.acc;
                f_acc = f.acc;
            }
        } else {
            const double scale = cell_scale(c, lo, hi);
            OrderedSum t, f;
            for_entries<4>(c, lo, hi, [&](int32_t m, float x) {
                const float v = m >= 0 ? transform_value(c, scale, x) : x;
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
            t_acc = t.acc;
            f_acc = f.acc;
        }
        if (lane == 0) {
            if (span_row_out) {
                span_row_out[i] = row;
                span_t[i] = t_acc;
                span_n[i] = n;
                span_f[i] = f_acc;
            }
            if (row_t) {
                atomicAdd(row_t + row, t_acc);
                atomicAdd(row_n + row, n);
                atomicAdd(row_f + row, f_acc);
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
        for_entries<8>(c, lo, hi, [&](int32_t m, float x) {
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
// Lane l owns components l, l+32, ... (k <= 128).  One read of the cell's
// entries (four per lane, 16-byte loads) forms the normalisation total and
// queues the HVG entries (code, raw value) in entry order in a per-warp
// shared-memory queue.  Once the scale is known the queue is consumed in
// rounds of kProjStage entries: the lanes transform a round in parallel
// into a staging buffer, then the round is added U entries at a time with
// all V-row loads issued before the U ordered additions, so the L2 latency
// of the V gathers overlaps.  A cell with more than kProjQueue HVG entries
// (or whose total needs the in-order fold) reads its entries again.  Cells
// are handed out one at a time through a counter.
constexpr int kProjWarps = 32;
constexpr int kProjQueue = 512;
constexpr int kProjStage = 128;

template <bool SMAP>
constexpr size_t proj_smem_fixed() {
    return (size_t)kProjWarps * (kProjQueue * ((SMAP ? sizeof(int16_t) : sizeof(int32_t)) + sizeof(float)) +
                                 kProjStage * sizeof(double));
}

template <int KPL, bool SMAP>
__global__ void __launch_bounds__(kProjWarps * 32, 1) k_project(DevChunk c, const int32_t *__restrict__ code,
                                                                int32_t d, DevScale t, const double *__restrict__ V,
                                                                int k, float *__restrict__ out, int by_span,
                                                                unsigned int *counter) {
    constexpr int U = KPL >= 2 ? 4 : 8;
    using Q = typename std::conditional<SMAP, int16_t, int32_t>::type;
    extern __shared__ __align__(16) unsigned char smem[];
    const int wid = threadIdx.x >> 5, lane = lane_id();
    // [staged values (f64)] [queued raw values (f32)] [queued codes (Q)] [codes (int16), SMAP]
    double *q_val = reinterpret_cast<double *>(smem) + (size_t)wid * kProjStage;
    unsigned char *p1 = smem + sizeof(double) * kProjWarps * kProjStage;
    float *q_x = reinterpret_cast<float *>(p1) + (size_t)wid * kProjQueue;
    unsigned char *p2 = p1 + sizeof(float) * kProjWarps * kProjQueue;
    Q *q_code = reinterpret_cast<Q *>(p2) + (size_t)wid * kProjQueue;
    int16_t *s_code = reinterpret_cast<int16_t *>(smem + proj_smem_fixed<SMAP>());
    if (SMAP) copy_codes16(code, c.n_gene_map, s_code);
    __syncthreads();
    auto lookup = [&](uint32_t g) -> int32_t { return SMAP ? (int32_t)s_code[g] : __ldg(code + g); };
    const bool norm = c.target_sum > 0.0;
    for (;;) {
        int64_t i = 0;
        if (lane == 0) i = atomicAdd(counter, 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= c.n_spans) break;
        int64_t lo, hi;
        const int64_t row = span_row(c, i, lo, hi);
        if (row < 0) continue;
        double acc[KPL];
#pragma unroll
        for (int q = 0; q < KPL; ++q) acc[q] = 0.0;
        // add staged pairs (code q_code[base + e], value q_val[e]), e < n, in order
        auto drain = [&](int base, int n) {
            __syncwarp();
            int e = 0;
            for (; e + U <= n; e += U) {
                double vv[U][KPL];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double *vr = V + (size_t)q_code[base + e + u] * k;
#pragma unroll
                    for (int q = 0; q < KPL; ++q) {
                        const int j = lane + 32 * q;
                        vv[u][q] = j < k ? __ldg(vr + j) : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double sv = q_val[e + u];
#pragma unroll
                    for (int q = 0; q < KPL; ++q) acc[q] = __dadd_rn(acc[q], __dmul_rn(sv, vv[u][q]));
                }
            }
            for (; e < n; ++e) {
                const double *vr = V + (size_t)q_code[base + e] * k;
                const double sv = q_val[e];
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int j = lane + 32 * q;
                    if (j < k) acc[q] = __dadd_rn(acc[q], __dmul_rn(sv, __ldg(vr + j)));
                }
            }
            __syncwarp();
        };
        double tsum = 0.0;
        bool ok = true, ovf = false;
        int nq = 0;
        for_entries_x4<true, kProjDepth>(c, lo, hi, lookup, [&](const int32_t (&m)[4], const float (&x)[4]) {
            bool hv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (m[u] >= 0 && norm) {
                    ok = ok && x[u] == rintf(x[u]) && fabsf(x[u]) < 16777216.0f;
                    tsum += (double)x[u];
                }
                hv[u] = m[u] >= 0 && m[u] < d;
            }
            int cnt;
            int pos = nq + block_rank4(hv, cnt);
            if (cnt == 0) return;
            if (nq + cnt > kProjQueue) {
                ovf = true;
                return;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (hv[u]) {
                    q_code[pos] = (Q)m[u];
                    q_x[pos] = x[u];
                    ++pos;
                }
            nq += cnt;
        });
        double scale = 1.0;
        if (norm) {
            double total;
            if (__all_sync(kFull, ok)) {
                total = warp_sum(tsum);
            } else {
                OrderedSum ts;
                for_entries_by<4, false>(c, lo, hi, lookup,
                                         [&](int32_t m, float x) { ts.add(m >= 0 ? (double)x : 0.0); });
                total = ts.acc;
            }
            scale = total > 0.0 ? c.target_sum / total : 1.0;
        }
        if (!ovf) {
            for (int r0 = 0; r0 < nq; r0 += kProjStage) {
                const int n = nq - r0 < kProjStage ? nq - r0 : kProjStage;
                __syncwarp();
                for (int e = lane; e < n; e += 32)
                    q_val[e] = scale_value(t, q_code[r0 + e], transform_value(c, scale, q_x[r0 + e]));
                drain(r0, n);
            }
        } else {  // second read, draining whenever the staging buffer fills
            int ns = 0;
            __syncwarp();
            for_entries_by<8, true>(c, lo, hi, lookup, [&](int32_t m, float x) {
                const bool hv = m >= 0 && m < d;
                const unsigned mask = __ballot_sync(kFull, hv);
                if (!mask) return;
                if (ns + 32 > kProjStage) {
                    drain(0, ns);
                    ns = 0;
                }
                if (hv) {
                    const int pos = ns + __popc(mask & ((1u << lane) - 1u));
                    q_code[pos] = (Q)m;
                    q_val[pos] = scale_value(t, m, transform_value(c, scale, x));
                }
                ns += __popc(mask);
            });
            drain(0, ns);
        }
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

template <int KPL>
static int launch_project_k(const DevChunk &c, const int32_t *code, int64_t d, const DevScale &t, const double *V,
                            int k, float *out, int by_span, unsigned int *counter, cudaStream_t st) {
    CREST_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st));
    const int blocks = (int)std::min<int64_t>(ceil_div(c.n_spans, kProjWarps), device_sms());
    if (codes_in_smem(c.n_gene_map, d, proj_smem_fixed<true>())) {
        const size_t smem = proj_smem_fixed<true>() + 2 * (size_t)round_up(c.n_gene_map, 8);
        CREST_TRY(ensure_smem_attr((const void *)k_project<KPL, true>, smem));
        k_project<KPL, true><<<blocks, kProjWarps * 32, smem, st>>>(c, code, (int32_t)d, t, V, k, out, by_span,
                                                                     counter);
    } else {
        const size_t smem = proj_smem_fixed<false>();
        CREST_TRY(ensure_smem_attr((const void *)k_project<KPL, false>, smem));
        k_project<KPL, false><<<blocks, kProjWarps * 32, smem, st>>>(c, code, (int32_t)d, t, V, k, out, by_span,
                                                                      counter);
    }
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_project(const DevChunk &c, const int32_t *code, int64_t d, const DevScale &t, const double *V, int k,
                   float *out, int by_span, unsigned int *counter, cudaStream_t st) {
    if (c.n_spans == 0 || k == 0) return CREST_OK;
    CREST_REQUIRE(k <= 128, CREST_EINVAL, "project supports k <= 128 (got %d)", k);
    prof::Scope ps("project_csr", st);
    if (k <= 32) return launch_project_k<1>(c, code, d, t, V, k, out, by_span, counter, st);
    if (k <= 64) return launch_project_k<2>(c, code, d, t, V, k, out, by_span, counter, st);
    return launch_project_k<4>(c, code, d, t, V, k, out, by_span, counter, st);
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
