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
// log1p and the scaled values are recomputed in the backward pass; only the
// per-entry s_e of the stored entries is kept for the W gradient, which is
// formed gene by gene over a by-gene index of the entries (counting sort).
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

// Entry pass of the backward: dL/dx, dL/dsf, and s_e / cell of every entry
// for the W gradient; per-gene entry counts for the by-gene index.
template <int KPL>
__global__ void __launch_bounds__(256) k_fused_bwd_entries(FusedArgs a, const float *__restrict__ G,
                                                           float *__restrict__ grad_x, float *__restrict__ grad_sf,
                                                           double *__restrict__ s_out, int32_t *__restrict__ cell_out,
                                                           int32_t *__restrict__ gene_count) {
    __shared__ float g_row[8][32 * KPL];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < a.n; c += n_warps) {
        __syncwarp();
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            const int j = lane + 32 * q;
            g_row[wid][j] = j < a.k ? G[c * a.k + j] : 0.0f;
        }
        __syncwarp();
        const int64_t lo = a.indptr[c], hi = a.indptr[c + 1];
        const float sfc = a.sf[c];
        double dsf = 0.0;
        for (int64_t e = lo + lane; e < hi; e += 32) {
            const int32_t g = __ldg(a.indices + e);
            if (g < 0 || g >= a.d) {  // out-of-range gene id: reported, no gradient
                *a.bad = 1;
                grad_x[e] = 0.0f;
                s_out[e] = 0.0;
                cell_out[e] = (int32_t)c;
                continue;
            }
            const float x = __ldg(a.values + e);
            float y;
            double pass;
            const double s = fused_value(a, g, x, sfc, y, pass);
            const float *wr = a.W + (size_t)g * a.k;
            double gs = 0.0;
            for (int j = 0; j < a.k; ++j) gs = fma((double)g_row[wid][j], (double)__ldg(wr + j), gs);
            const double dy = gs * pass / (__ldg(a.std + g) * (1.0 + (double)y));
            grad_x[e] = (float)(dy / (double)sfc);
            dsf -= dy * (double)y / (double)sfc;
            s_out[e] = s;
            cell_out[e] = (int32_t)c;
            atomicAdd(gene_count + g, 1);
        }
        dsf = warp_sum(dsf);
        if (lane == 0) grad_sf[c] = (float)dsf;
    }
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

__global__ void k_scatter_by_gene(const int32_t *__restrict__ indices, int64_t nnz, int64_t d,
                                  const int64_t *__restrict__ offsets,
                                  int32_t *__restrict__ fill, int64_t *__restrict__ order) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const int32_t g = indices[e];
    if (g < 0 || g >= d) return;
    order[offsets[g] + atomicAdd(fill + g, 1)] = e;
}

// dL/dW[g, :] = sum over entries of gene g of s_e G[c_e, :], warp per gene.
template <int KPL>
__global__ void __launch_bounds__(256) k_fused_bwd_w(int64_t d, int k, const int64_t *__restrict__ offsets,
                                                     const int64_t *__restrict__ order, const double *__restrict__ s_e,
                                                     const int32_t *__restrict__ cell, const float *__restrict__ G,
                                                     float *__restrict__ grad_W) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = warp; g < d; g += n_warps) {
        double acc[KPL];
#pragma unroll
        for (int q = 0; q < KPL; ++q) acc[q] = 0.0;
        for (int64_t t = offsets[g]; t < offsets[g + 1]; ++t) {
            const int64_t e = order[t];
            const double s = s_e[e];
            const float *gr = G + (size_t)cell[e] * k;
#pragma unroll
            for (int q = 0; q < KPL; ++q) {
                const int j = lane + 32 * q;
                if (j < k) acc[q] = fma(s, (double)__ldg(gr + j), acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            const int j = lane + 32 * q;
            if (j < k) grad_W[g * k + j] = (float)acc[q];
        }
    }
}

int grid_warps(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 8), device_sms() * 16)); }

struct FusedWork {
    DevBuf s, cell, count, fill, offsets, order, bad;
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
    CREST_TRY(w.s.ensure(sizeof(double) * (size_t)std::max<int64_t>(nnz, 1)));
    CREST_TRY(w.cell.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1)));
    CREST_TRY(w.order.ensure(sizeof(int64_t) * (size_t)std::max<int64_t>(nnz, 1)));
    CREST_TRY(w.count.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(d, 1)));
    CREST_TRY(w.fill.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(d, 1)));
    CREST_TRY(w.offsets.ensure(sizeof(int64_t) * (size_t)(d + 1)));
    if (d) {
        CREST_CUDA_TRY(cudaMemsetAsync(w.count.ptr, 0, sizeof(int32_t) * d, st));
        CREST_CUDA_TRY(cudaMemsetAsync(w.fill.ptr, 0, sizeof(int32_t) * d, st));
    }
    if (n > 0) {
        prof::Scope ps("fused_bwd", st);
        const int g = grid_warps(n);
        if (k <= 32)
            k_fused_bwd_entries<1><<<g, 256, 0, st>>>(a, grad_scores, grad_values, grad_sf, w.s.as<double>(),
                                                      w.cell.as<int32_t>(), w.count.as<int32_t>());
        else if (k <= 64)
            k_fused_bwd_entries<2><<<g, 256, 0, st>>>(a, grad_scores, grad_values, grad_sf, w.s.as<double>(),
                                                      w.cell.as<int32_t>(), w.count.as<int32_t>());
        else
            k_fused_bwd_entries<4><<<g, 256, 0, st>>>(a, grad_scores, grad_values, grad_sf, w.s.as<double>(),
                                                      w.cell.as<int32_t>(), w.count.as<int32_t>());
        CREST_CUDA_TRY(cudaGetLastError());
    }
    if (d > 0) {
        prof::Scope ps("fused_bwd_w", st);
        k_scan_counts<<<1, 1024, 0, st>>>(w.count.as<int32_t>(), d, w.offsets.as<int64_t>());
        if (nnz)
            k_scatter_by_gene<<<(unsigned)ceil_div(nnz, 256), 256, 0, st>>>(indices, nnz, d, w.offsets.as<int64_t>(),
                                                                          w.fill.as<int32_t>(), w.order.as<int64_t>());
        const int g = grid_warps(d);
        if (k <= 32)
            k_fused_bwd_w<1><<<g, 256, 0, st>>>(d, (int)k, w.offsets.as<int64_t>(), w.order.as<int64_t>(),
                                                w.s.as<double>(), w.cell.as<int32_t>(), grad_scores, grad_W);
        else if (k <= 64)
            k_fused_bwd_w<2><<<g, 256, 0, st>>>(d, (int)k, w.offsets.as<int64_t>(), w.order.as<int64_t>(),
                                                w.s.as<double>(), w.cell.as<int32_t>(), grad_scores, grad_W);
        else
            k_fused_bwd_w<4><<<g, 256, 0, st>>>(d, (int)k, w.offsets.as<int64_t>(), w.order.as<int64_t>(),
                                                w.s.as<double>(), w.cell.as<int32_t>(), grad_scores, grad_W);
        CREST_CUDA_TRY(cudaGetLastError());
    }
    return bad_ids(w, st);
}
