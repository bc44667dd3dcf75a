// K7: the differentiable normalise -> log1p -> scale -> project map and its
// backward, for training-style use of the PCA projection (no counterpart in
// the reference; the forward arithmetic is the reference's transform).
//
// Input: a CSR matrix over d genes (HVG columns already selected) with
// per-cell size factors sf, loadings W (d x k, row-major), fixed per-gene
// mean / std of the scale step and its clip value.  Per stored entry e of
// cell c and gene g (the size factor divides, y = x / sf):
//
//   y = x / sf_c                      (f32, correctly rounded)
//   l = log1pf(y)                     (f32, glibc's algorithm)
//   z = (l - mean_g) / std_g          (f64)
//   s = clip(z) - clip(-mean_g / std_g)
//   score[c, :] = sum_e s_e W[g_e, :] (f64 accumulation, stored as f32)
//
// Backward, given G = dL/dscore (n x k):
//   dL/ds_e  = G[c, :] . W[g_e, :]
//   dL/dz_e  = dL/ds_e  when -max <= z <= max (or no clipping), else 0
//   dL/dy_e  = dL/dz_e / (std_g (1 + y))
//   dL/dx_e  = dL/dy_e / sf_c
//   dL/dsf_c = - sum_e dL/dy_e y_e / sf_c
//   dL/dW[g, :] = sum over entries of gene g of s_e G[c_e, :]
// log1p and the scaled values are recomputed in the backward pass.  The W
// gradient is formed gene by gene: a per-gene histogram of the entries and
// its scan give every gene a segment, the entry pass writes (s_e, c_e) of
// each entry into its gene's segment (counting sort; the order inside a
// segment is not fixed), and one block per gene sums s_e G[c_e, :] over its
// segment in f64.
#include "host.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {
namespace {

struct FusedArgs {
    const int64_t *indptr;
    const int32_t *indices;
    const float *values;
    int64_t n, d;
    const float *sf;
    const float *W;
    int k;
    const double *mean, *std;
    double max_value;
    int *bad;  // set when a gene id is outside [0, d)
};

// (s, pass, y) of one entry; pass is the clip derivative (1 inside the band).
__device__ __forceinline__ double fused_value(const FusedArgs &a, int32_t g, float x, float sfc, float &y,
                                              double &pass) {
    y = __fdiv_rn(x, sfc);
    const float l = crest_log1pf(y);
    const double mu = __ldg(a.mean + g), sd = __ldg(a.std + g);
    const double z = __ddiv_rn(__dsub_rn((double)l, mu), sd);
    const double mv = a.max_value;
    pass = (mv > 0.0 && (z < -mv || z > mv)) ? 0.0 : 1.0;
    return __dsub_rn(clip_mv(z, mv), clip_mv(__ddiv_rn(-mu, sd), mv));
}

// Warp per cell; lane j of the warp owns score columns j, j + 32, ...  Each
// 32-entry segment is transformed lane-parallel, then folded into the
// scores in entry order.  (Loading the W rows of 8 entries ahead of their
// additions needs 80 registers and measured slower, 0.84 against 0.61 ms on
// the 50,000-cell workload: the occupancy it costs hides more latency.)
template <int KPL>
__global__ void __launch_bounds__(256) k_fused_fwd(FusedArgs a, float *__restrict__ scores) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < a.n; c += n_warps) {
        const int64_t lo = a.indptr[c], hi = a.indptr[c + 1];
        const float sfc = a.sf[c];
        double acc[KPL];
#pragma unroll
        for (int q = 0; q < KPL; ++q) acc[q] = 0.0;
        for (int64_t s0 = lo; s0 < hi; s0 += 32) {
            const int64_t e = s0 + lane;
            int32_t g = 0;
            double s = 0.0;
            if (e < hi) {
                g = __ldg(a.indices + e);
                if (g >= 0 && g < a.d) {
                    float y;
                    double pass;
                    s = fused_value(a, g, __ldg(a.values + e), sfc, y, pass);
                } else {  // out-of-range gene id: reported, contributes nothing
                    *a.bad = 1;
                    g = 0;
                }
            }
            const int cnt = hi - s0 < 32 ? (int)(hi - s0) : 32;
            for (int u = 0; u < cnt; ++u) {  // entry order
                const int32_t gu = __shfl_sync(kFull, g, u);
                const double su = __shfl_sync(kFull, s, u);
                const float *wr = a.W + (size_t)gu * a.k;
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int j = lane + 32 * q;
                    if (j < a.k) acc[q] = __dadd_rn(acc[q], __dmul_rn(su, (double)__ldg(wr + j)));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            const int j = lane + 32 * q;
            if (j < a.k) scores[c * a.k + j] = __double2float_rn(acc[q]);
        }
    }
}

// The W gradient loads the G rows of kGather entries before their products.
constexpr int kGather = 8;

// Per-gene entry counts: block-private counters in shared memory when d
// fits (kHistSmem genes), else global atomics; ids outside [0, d) are left
// out (the entry pass reports them).
constexpr int kHistSmem = 12288;

__global__ void __launch_bounds__(256) k_gene_hist(const int32_t *__restrict__ indices, int64_t nnz, int64_t d,
                                                   int32_t *__restrict__ count) {
    __shared__ int32_t s_cnt[kHistSmem];
    const bool priv = d <= kHistSmem;
    if (priv)
        for (int64_t g = threadIdx.x; g < d; g += blockDim.x) s_cnt[g] = 0;
    __syncthreads();
    const int64_t per = ceil_div(nnz, (int64_t)gridDim.x);
    const int64_t e0 = per * blockIdx.x, e1 = e0 + per < nnz ? e0 + per : nnz;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int32_t g = __ldg(indices + e);
        if (g < 0 || g >= d) continue;
        if (priv)
            atomicAdd(s_cnt + g, 1);
        else
            atomicAdd(count + g, 1);
    }
    __syncthreads();
    if (priv)
        for (int64_t g = threadIdx.x; g < d; g += blockDim.x)
            if (s_cnt[g]) atomicAdd(count + g, s_cnt[g]);
}

// Exclusive scan of the per-gene counts (one block): offsets[0..d].
__global__ void __launch_bounds__(1024) k_scan_counts(const int32_t *count, int64_t d, int64_t *offsets) {
    __shared__ int64_t part[1024];
    const int tid = threadIdx.x;
    const int64_t per = (d + 1023) / 1024, b0 = tid * per, b1 = b0 + per < d ? b0 + per : d;
    int64_t s = 0;
    for (int64_t i = b0; i < b1; ++i) s += count[i];
    part[tid] = s;
    __syncthreads();
    if (tid == 0) {
        int64_t run = 0;
        for (int i = 0; i < 1024; ++i) {
            const int64_t v = part[i];
            part[i] = run;
            run += v;
        }
        offsets[d] = run;
    }
    __syncthreads();
    int64_t run = part[tid];
    for (int64_t i = b0; i < b1; ++i) {
        offsets[i] = run;
        run += count[i];
    }
}

// W rows padded to kp = round_up(k, 4) floats (16-byte rows for vector loads).
__global__ void k_pad_rows(const float *__restrict__ W, int64_t d, int k, int kp, float *__restrict__ Wp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d * kp) return;
    const int64_t g = i / kp;
    const int j = (int)(i - g * kp);
    Wp[i] = j < k ? W[g * k + j] : 0.0f;
}

// One entry's contribution to the W gradient: s_e and its cell.
struct __align__(16) EntryCell {
    double s;
    int32_t cell;
    int32_t pad;
};

// Entry pass of the backward, warp per cell, lane per entry: dL/dx and
// dL/dsf, and (s_e, c) of every entry into its gene's segment.  The cell's
// row of G is held in shared memory as f64 (kp columns, zero-padded); the
// dot product with W[g, :] reads the W rows padded to kp (<= KP) columns,
// 16 bytes at a time.
template <int KP>
__global__ void __launch_bounds__(256) k_fused_bwd_entries(FusedArgs a, const float *__restrict__ G,
                                                           const float *__restrict__ Wp, int kp,
                                                           float *__restrict__ grad_x, float *__restrict__ grad_sf,
                                                           const int64_t *__restrict__ offsets,
                                                           int32_t *__restrict__ fill, EntryCell *__restrict__ by_gene) {
    __shared__ double g_row[8][KP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < a.n; c += n_warps) {
        __syncwarp();
        for (int j = lane; j < KP; j += 32) g_row[wid][j] = j < a.k ? (double)G[c * a.k + j] : 0.0;
        __syncwarp();
        const int64_t lo = a.indptr[c], hi = a.indptr[c + 1];
        const float sfc = a.sf[c];
        double dsf = 0.0;
        for (int64_t e = lo + lane; e < hi; e += 32) {
            const int32_t g = __ldg(a.indices + e);
            if (g < 0 || g >= a.d) {  // out-of-range gene id: reported, no gradient
                *a.bad = 1;
                grad_x[e] = 0.0f;
                continue;
            }
            const float x = __ldg(a.values + e);
            float y;
            double pass;
            const double s = fused_value(a, g, x, sfc, y, pass);
            const float4 *wr = reinterpret_cast<const float4 *>(Wp + (size_t)g * kp);
            double gs = 0.0;
#pragma unroll 4
            for (int j4 = 0; j4 < kp / 4; ++j4) {
                const float4 w = __ldg(wr + j4);
                const double *gr = g_row[wid] + 4 * j4;
                gs = fma(gr[0], (double)w.x, gs);
                gs = fma(gr[1], (double)w.y, gs);
                gs = fma(gr[2], (double)w.z, gs);
                gs = fma(gr[3], (double)w.w, gs);
            }
            const double dy = gs * pass / (__ldg(a.std + g) * (1.0 + (double)y));
            grad_x[e] = (float)(dy / (double)sfc);
            dsf -= dy * (double)y / (double)sfc;
            EntryCell ec;
            ec.s = s;
            ec.cell = (int32_t)c;
            ec.pad = 0;
            by_gene[offsets[g] + atomicAdd(fill + g, 1)] = ec;
        }
        dsf = warp_sum(dsf);
        if (lane == 0) grad_sf[c] = (float)dsf;
    }
}

// dL/dW[g, :] = sum over gene g's segment of s_e G[c_e, :], block per gene:
// the 8 warps take interleaved 32-entry pieces of the segment (one
// coalesced load of 32 (s, c) pairs per piece), lane j accumulates columns
// j, j + 32, ...; the G rows of kGather entries are loaded before their
// products are added.  The warps' partial sums are added in shared memory.
template <int KPL>
__global__ void __launch_bounds__(256) k_fused_bwd_w(int64_t d, int k, const int64_t *__restrict__ offsets,
                                                     const EntryCell *__restrict__ by_gene,
                                                     const float *__restrict__ G, float *__restrict__ grad_W) {
    __shared__ double part[8][32 * KPL];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t g = blockIdx.x; g < d; g += gridDim.x) {
        const int64_t t0 = offsets[g], t1 = offsets[g + 1];
        double acc[KPL];
#pragma unroll
        for (int q = 0; q < KPL; ++q) acc[q] = 0.0;
        for (int64_t b = t0 + 32 * wid; b < t1; b += 256) {
            const int cnt = t1 - b < 32 ? (int)(t1 - b) : 32;
            double s = 0.0;
            int32_t cell = 0;
            if (lane < cnt) {
                const EntryCell ec = by_gene[b + lane];
                s = ec.s;
                cell = ec.cell;
            }
            for (int u0 = 0; u0 < cnt; u0 += kGather) {
                float gv[kGather][KPL];
                double su[kGather];
#pragma unroll
                for (int t = 0; t < kGather; ++t) {
                    const int u = (u0 + t) & 31;
                    su[t] = __shfl_sync(kFull, s, u);
                    const int32_t cu = __shfl_sync(kFull, cell, u);
                    const float *gr = G + (size_t)cu * k;
#pragma unroll
                    for (int q = 0; q < KPL; ++q) {
                        const int j = lane + 32 * q;
                        gv[t][q] = (u0 + t < cnt && j < k) ? __ldg(gr + j) : 0.0f;
                    }
                }
#pragma unroll
                for (int t = 0; t < kGather; ++t)
#pragma unroll
                    for (int q = 0; q < KPL; ++q) acc[q] = fma(su[t], (double)gv[t][q], acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < KPL; ++q) part[wid][lane + 32 * q] = acc[q];
        __syncthreads();
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < 8; ++w) v += part[w][j];
            grad_W[g * k + j] = (float)v;
        }
        __syncthreads();
    }
}

int grid_warps(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 8), device_sms() * 16)); }

struct FusedWork {
    DevBuf by_gene, count, fill, offsets, wpad, bad;
};

FusedWork &fused_work(int dev) {
    static thread_local FusedWork ws[64];
    return ws[dev];
}

// Flag buffer of the current device, cleared; its value is read by bad_ids().
int arm_flag(FusedWork &w, FusedArgs &a, cudaStream_t st) {
    CREST_TRY(w.bad.ensure(sizeof(int)));
    CREST_CUDA_TRY(cudaMemsetAsync(w.bad.ptr, 0, sizeof(int), st));
    a.bad = w.bad.as<int>();
    return CREST_OK;
}

int bad_ids(FusedWork &w, cudaStream_t st) {
    int h = 0;
    CREST_CUDA_TRY(cudaMemcpyAsync(&h, w.bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    CREST_REQUIRE(h == 0, CREST_EINVAL, "fused map: indices must be gene ids in [0, d)");
    return CREST_OK;
}

int current_device(int *dev) {
    CREST_CUDA_TRY(cudaGetDevice(dev));
    CREST_REQUIRE(*dev >= 0 && *dev < 64, CREST_ERUNTIME, "device index %d out of range", *dev);
    return CREST_OK;
}

int check_fused(const FusedArgs &a) {
    CREST_REQUIRE(a.n >= 0 && a.d >= 0 && a.k >= 1 && a.k <= 128, CREST_EINVAL,
                  "fused map: need n, d >= 0 and 1 <= k <= 128 (k=%d)", a.k);
    CREST_REQUIRE(a.indptr && a.sf && a.W && a.mean && a.std, CREST_EINVAL, "fused map: NULL argument");
    return CREST_OK;
}

}  // namespace
}  // namespace crest

using namespace crest;

extern "C" int crest_fused_forward(const int64_t *indptr, const int32_t *indices, const float *values, int64_t n,
                                   int64_t d, const float *size_factors, const float *W, int64_t k,
                                   const double *mean, const double *std, double max_value, float *scores) {
    FusedArgs a{indptr, indices, values, n, d, size_factors, W, (int)k, mean, std, max_value, nullptr};
    CREST_TRY(check_fused(a));
    CREST_REQUIRE(scores, CREST_EINVAL, "fused map: NULL scores");
    CREST_TRY(require_device());
    if (n == 0) return CREST_OK;
    int dev = 0;
    CREST_TRY(current_device(&dev));
    FusedWork &w = fused_work(dev);
    cudaStream_t st = cudaStreamPerThread;
    CREST_TRY(arm_flag(w, a, st));
    {
        prof::Scope ps("fused_fwd", st);
        if (k <= 32)
            k_fused_fwd<1><<<grid_warps(n), 256, 0, st>>>(a, scores);
        else if (k <= 64)
            k_fused_fwd<2><<<grid_warps(n), 256, 0, st>>>(a, scores);
        else
            k_fused_fwd<4><<<grid_warps(n), 256, 0, st>>>(a, scores);
    }
    CREST_CUDA_TRY(cudaGetLastError());
    return bad_ids(w, st);
}

extern "C" int crest_fused_backward(const int64_t *indptr, const int32_t *indices, const float *values, int64_t n,
                                    int64_t d, const float *size_factors, const float *W, int64_t k,
                                    const double *mean, const double *std, double max_value,
                                    const float *grad_scores, float *grad_values, float *grad_sf, float *grad_W) {
    FusedArgs a{indptr, indices, values, n, d, size_factors, W, (int)k, mean, std, max_value, nullptr};
    CREST_TRY(check_fused(a));
    CREST_REQUIRE(grad_scores && grad_values && grad_sf && grad_W, CREST_EINVAL, "fused map: NULL gradient");
    CREST_TRY(require_device());
    int dev = 0;
    CREST_TRY(current_device(&dev));
    FusedWork &w = fused_work(dev);
    cudaStream_t st = cudaStreamPerThread;
    CREST_TRY(arm_flag(w, a, st));
    int64_t nnz = 0, p0 = 0;
    if (n > 0) {
        CREST_CUDA_TRY(cudaMemcpyAsync(&p0, indptr, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(&nnz, indptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaStreamSynchronize(st));
    }
    CREST_REQUIRE(p0 == 0 && nnz >= 0 && nnz < ((int64_t)1 << 31), CREST_EINVAL,
                  "fused map: indptr must start at 0 and hold < 2^31 entries");
    const int kp = (int)round_up(k, 4);
    CREST_TRY(w.by_gene.ensure(sizeof(EntryCell) * (size_t)std::max<int64_t>(nnz, 1)));
    CREST_TRY(w.count.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(d, 1)));
    CREST_TRY(w.fill.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(d, 1)));
    CREST_TRY(w.offsets.ensure(sizeof(int64_t) * (size_t)(d + 1)));
    CREST_TRY(w.wpad.ensure(sizeof(float) * (size_t)std::max<int64_t>(d * kp, 1)));
    if (d) {
        CREST_CUDA_TRY(cudaMemsetAsync(w.count.ptr, 0, sizeof(int32_t) * d, st));
        CREST_CUDA_TRY(cudaMemsetAsync(w.fill.ptr, 0, sizeof(int32_t) * d, st));
    }
    {
        prof::Scope ps("fused_bwd", st);
        if (d > 0) {
            if (nnz)
                k_gene_hist<<<(unsigned)std::min<int64_t>(ceil_div(nnz, 4096), device_sms() * 4), 256, 0, st>>>(
                    indices, nnz, d, w.count.as<int32_t>());
            k_scan_counts<<<1, 1024, 0, st>>>(w.count.as<int32_t>(), d, w.offsets.as<int64_t>());
            k_pad_rows<<<(unsigned)ceil_div(d * kp, 256), 256, 0, st>>>(W, d, (int)k, kp, w.wpad.as<float>());
        }
        if (n > 0) {
            const int g = grid_warps(n);
            auto entries = [&](auto kern) {
                kern<<<g, 256, 0, st>>>(a, grad_scores, w.wpad.as<float>(), kp, grad_values, grad_sf,
                                        w.offsets.as<int64_t>(), w.fill.as<int32_t>(), w.by_gene.as<EntryCell>());
            };
            if (kp <= 32)
                entries(k_fused_bwd_entries<32>);
            else if (kp <= 64)
                entries(k_fused_bwd_entries<64>);
            else
                entries(k_fused_bwd_entries<128>);
        }
        CREST_CUDA_TRY(cudaGetLastError());
    }
    if (d > 0) {
        prof::Scope ps("fused_bwd_w", st);
        const unsigned blocks = (unsigned)std::min<int64_t>(d, (int64_t)device_sms() * 8);
        if (k <= 32)
            k_fused_bwd_w<1><<<blocks, 256, 0, st>>>(d, (int)k, w.offsets.as<int64_t>(), w.by_gene.as<EntryCell>(),
                                                     grad_scores, grad_W);
        else if (k <= 64)
            k_fused_bwd_w<2><<<blocks, 256, 0, st>>>(d, (int)k, w.offsets.as<int64_t>(), w.by_gene.as<EntryCell>(),
                                                     grad_scores, grad_W);
        else
            k_fused_bwd_w<4><<<blocks, 256, 0, st>>>(d, (int)k, w.offsets.as<int64_t>(), w.by_gene.as<EntryCell>(),
                                                     grad_scores, grad_W);
        CREST_CUDA_TRY(cudaGetLastError());
    }
    return bad_ids(w, st);
}
