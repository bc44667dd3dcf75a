// Gram accumulation over the HVG columns (K3 densify + K4 SYRK).
//
// src/kernels.rs:221-309 accumulates G += S^T S sparsely on the CPU.  On the
// GPU each tile of up to m_cap cells is densified into a gene-major tile in
// HBM/L2 (cells contiguous, the K dimension of the contraction) and
// contracted as a dense SYRK over the upper-triangular block tiles of G:
//
//  * FP64: T = S, CUDA-core DMUL+DADD accumulating straight into G in cell
//    order, which reproduces the reference's f64 sums bit for bit (the extra
//    terms are exact zeros);
//  * FP32 (plain form): T = Z = S + bias (the dense scaled matrix, centred by
//    construction), FP32 register-tiled SYRK, folded into G in FP64 with the
//    exact correction  S^T S = Z^T Z - bias c^T - c bias^T - n bias bias^T;
//  * BF16X3 (product form): same tile values split into bf16 hi/lo, contracted
//    on the tcgen05 tensor cores (k_gram_tc.cu) with the same FP64 fold.
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {

int syrk_bf16x3_fold(const GramWork &w, int64_t m, const DevScale &t, double *gram, cudaStream_t st);

size_t gram_tile_bytes(int precision, int64_t d_pad, int64_t m_cap) {
    const size_t n = (size_t)d_pad * (size_t)m_cap;
    if (precision == CREST_GRAM_FP64) return n * 8;
    if (precision == CREST_GRAM_FP32) return n * 4;
    return n * 4;  // two bf16 tiles
}

// ------------------------------------------------------------------ fill
// Every element of the tile: kept cell and gene < d -> value of a zero entry
// (0 for FP64, bias for the centred forms); dropped cell / padding -> 0.
template <class T>
__global__ void k_tile_fill(DevChunk c, int64_t d, int64_t d_pad, int64_t m_pad, const double *bias, T *tile,
                            int64_t *n_kept) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // cell column
    if (i >= m_pad) return;
    bool kept = false;
    if (i < c.n_spans) {
        const uint32_t cell = c.span_cell ? c.span_cell[i] : c.first_cell + (uint32_t)i;
        kept = (int64_t)cell < c.n_cell_map && c.cell_map[cell] >= 0;
    }
    if (kept && blockIdx.y == 0) atomicAdd((unsigned long long *)n_kept, 1ull);
    for (int64_t j = blockIdx.y; j < d_pad; j += gridDim.y) {
        double v = (kept && j < d && bias) ? bias[j] : 0.0;
        tile[(size_t)j * m_pad + i] = (T)v;
    }
}

__global__ void k_tile_fill_bf16x3(DevChunk c, int64_t d, int64_t d_pad, int64_t m_pad, const double *bias,
                                   __nv_bfloat16 *hi, __nv_bfloat16 *lo, int64_t *n_kept) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m_pad) return;
    bool kept = false;
    if (i < c.n_spans) {
        const uint32_t cell = c.span_cell ? c.span_cell[i] : c.first_cell + (uint32_t)i;
        kept = (int64_t)cell < c.n_cell_map && c.cell_map[cell] >= 0;
    }
    if (kept && blockIdx.y == 0) atomicAdd((unsigned long long *)n_kept, 1ull);
    for (int64_t j = blockIdx.y; j < d_pad; j += gridDim.y) {
        const double v = (kept && j < d && bias) ? bias[j] : 0.0;
        const __nv_bfloat16 h = __double2bfloat16(v);
        hi[(size_t)j * m_pad + i] = h;
        lo[(size_t)j * m_pad + i] = __double2bfloat16(v - (double)__bfloat162float(h));
    }
}

// --------------------------------------------------------------- scatter
// Warp per cell: stored HVG entries overwrite their tile element; colsum of
// S is accumulated in shared memory (f64) and flushed once per block.
template <int MODE>  // 0 FP64 (T = S), 1 FP32 (T = Z)
__global__ void __launch_bounds__(256) k_tile_scatter(DevChunk c, const int32_t *__restrict__ sub_map, DevScale t,
                                                      int64_t d, int64_t m_pad, void *tile,
                                                      double *__restrict__ colsum) {
    extern __shared__ double s_col[];
    const bool priv = MODE != 0 && d <= 4096;
    if (priv) {
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) s_col[j] = 0.0;
        __syncthreads();
    }
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        if (span_row(c, i, lo, hi) < 0) continue;
        const double scale = cell_scale(c, lo, hi);
        for_entries<4>(c, lo, hi, [&](int32_t m, float x) {
            const int32_t sub = m >= 0 ? __ldg(sub_map + m) : -1;
            if (sub < 0) return;
            const double s = scale_value(t, sub, transform_value(c, scale, x));
            const size_t at = (size_t)sub * m_pad + i;
            if (MODE == 0) {
                reinterpret_cast<double *>(tile)[at] = s;
            } else {
                const double z = t.scale ? __dadd_rn(s, __ldg(t.bias + sub)) : s;
                reinterpret_cast<float *>(tile)[at] = __double2float_rn(z);
                if (priv)
                    atomicAdd(s_col + sub, s);
                else
                    atomicAdd(colsum + sub, s);
            }
        });
    }
    if (priv) {
        __syncthreads();
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x)
            if (s_col[j] != 0.0) atomicAdd(colsum + j, s_col[j]);
    }
}

// BF16X3 needs both tiles; the lo tile sits right after the hi tile.
__global__ void __launch_bounds__(256) k_tile_scatter_bf16x3(DevChunk c, const int32_t *__restrict__ sub_map,
                                                             DevScale t, int64_t d, int64_t m_pad, int64_t d_pad,
                                                             __nv_bfloat16 *hi, __nv_bfloat16 *lo,
                                                             double *__restrict__ colsum) {
    extern __shared__ double s_col[];
    const bool priv = d <= 4096;
    if (priv) {
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) s_col[j] = 0.0;
        __syncthreads();
    }
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo_e, hi_e;
        if (span_row(c, i, lo_e, hi_e) < 0) continue;
        const double scale = cell_scale(c, lo_e, hi_e);
        for_entries<4>(c, lo_e, hi_e, [&](int32_t m, float x) {
            const int32_t sub = m >= 0 ? __ldg(sub_map + m) : -1;
            if (sub < 0) return;
            const double s = scale_value(t, sub, transform_value(c, scale, x));
            const double z = t.scale ? __dadd_rn(s, __ldg(t.bias + sub)) : s;
            const size_t at = (size_t)sub * m_pad + i;
            const __nv_bfloat16 h = __double2bfloat16(z);
            hi[at] = h;
            lo[at] = __double2bfloat16(z - (double)__bfloat162float(h));
            if (priv)
                atomicAdd(s_col + sub, s);
            else
                atomicAdd(colsum + sub, s);
        });
    }
    if (priv) {
        __syncthreads();
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x)
            if (s_col[j] != 0.0) atomicAdd(colsum + j, s_col[j]);
    }
    (void)d_pad;
}

int launch_densify(const DevChunk &c, const int32_t *sub_map, const DevScale &t, const GramWork &w,
                   cudaStream_t st) {
    CREST_REQUIRE(c.n_spans <= w.m_cap, CREST_EINVAL, "tile holds %lld cells, chunk has %lld",
                  (long long)w.m_cap, (long long)c.n_spans);
    const int64_t m_pad = round_up(c.n_spans > 0 ? c.n_spans : 1, 64);
    CREST_CUDA_TRY(cudaMemsetAsync(w.n_kept, 0, sizeof(int64_t), st));
    CREST_CUDA_TRY(cudaMemsetAsync(w.colsum_chunk, 0, sizeof(double) * (size_t)(w.d > 0 ? w.d : 1), st));
    const double *bias = (w.precision != CREST_GRAM_FP64 && t.scale) ? t.bias : nullptr;
    dim3 fg((unsigned)ceil_div(m_pad, 128), (unsigned)(w.d_pad < 64 ? w.d_pad : 64));
    {
    prof::Scope ps("tile_fill", st);
    if (w.precision == CREST_GRAM_FP64)
        k_tile_fill<double><<<fg, 128, 0, st>>>(c, w.d, w.d_pad, m_pad, bias, (double *)w.tile, w.n_kept);
    else if (w.precision == CREST_GRAM_FP32)
        k_tile_fill<float><<<fg, 128, 0, st>>>(c, w.d, w.d_pad, m_pad, bias, (float *)w.tile, w.n_kept);
    else {
        __nv_bfloat16 *hi = (__nv_bfloat16 *)w.tile;
        __nv_bfloat16 *lo = hi + (size_t)w.d_pad * (size_t)m_pad;
        k_tile_fill_bf16x3<<<fg, 128, 0, st>>>(c, w.d, w.d_pad, m_pad, bias, hi, lo, w.n_kept);
    }
    }
    CREST_CUDA_TRY(cudaGetLastError());
    if (c.n_spans == 0) return CREST_OK;
    const int64_t warps = 8;
    int64_t blocks = ceil_div(c.n_spans, warps);
    const int64_t cap = (int64_t)device_sms() * 8;
    if (blocks > cap) blocks = cap;
    const size_t smem = (w.d <= 4096) ? sizeof(double) * (size_t)w.d : 0;
    prof::Scope ps("tile_scatter", st);
    if (w.precision == CREST_GRAM_FP64) {
        k_tile_scatter<0><<<(unsigned)blocks, 256, 0, st>>>(c, sub_map, t, w.d, m_pad, w.tile, w.colsum_chunk);
    } else if (w.precision == CREST_GRAM_FP32) {
        if (smem > 48 * 1024)
            CREST_CUDA_TRY(cudaFuncSetAttribute(k_tile_scatter<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem));
        k_tile_scatter<1><<<(unsigned)blocks, 256, smem, st>>>(c, sub_map, t, w.d, m_pad, w.tile, w.colsum_chunk);
    } else {
        if (smem > 48 * 1024)
            CREST_CUDA_TRY(cudaFuncSetAttribute(k_tile_scatter_bf16x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem));
        __nv_bfloat16 *hi = (__nv_bfloat16 *)w.tile;
        __nv_bfloat16 *lo = hi + (size_t)w.d_pad * (size_t)m_pad;
        k_tile_scatter_bf16x3<<<(unsigned)blocks, 256, smem, st>>>(c, sub_map, t, w.d, m_pad, w.d_pad, hi, lo,
                                                                  w.colsum_chunk);
    }
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ------------------------------------------------------------ FP64 SYRK
// Upper-triangular 64x64 block tiles; each thread owns 4x4 outputs and
// accumulates G[a][b] + T[a][0]T[b][0] + T[a][1]T[b][1] + ... in cell order
// with separately rounded products, exactly like src/kernels.rs:303-305.
__device__ __forceinline__ void tri_decode(int64_t t, int64_t nb, int &bi, int &bj) {
    // t enumerates (bi <= bj) row-major: row bi has nb - bi tiles
    int r = 0;
    int64_t rem = t;
    while (rem >= nb - r) {
        rem -= nb - r;
        ++r;
    }
    bi = r;
    bj = r + (int)rem;
}

__global__ void __launch_bounds__(256) k_syrk_f64(const double *__restrict__ T, int64_t d, int64_t m_pad,
                                                  int64_t nb, double *__restrict__ G) {
    __shared__ double As[16][64 + 1];
    __shared__ double Bs[16][64 + 1];
    int bi, bj;
    tri_decode(blockIdx.x, nb, bi, bj);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t a0 = (int64_t)bi * 64, b0 = (int64_t)bj * 64;
    double acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t a = a0 + ty + 16 * p, b = b0 + tx + 16 * q;
            acc[p][q] = (a < d && b < d && a <= b) ? G[a * d + b] : 0.0;
        }
    // loader: 64 rows x 16 cols = 1024 doubles per panel; 4 per thread
    for (int64_t k0 = 0; k0 < m_pad; k0 += 16) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int idx = threadIdx.x + 256 * r;
            const int row = idx >> 4, col = idx & 15;
            As[col][row] = T[(a0 + row) * m_pad + k0 + col];
            Bs[col][row] = T[(b0 + row) * m_pad + k0 + col];
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double av[4], bv[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) av[p] = As[kk][ty + 16 * p];
#pragma unroll
            for (int q = 0; q < 4; ++q) bv[q] = Bs[kk][tx + 16 * q];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = __dadd_rn(acc[p][q], __dmul_rn(av[p], bv[q]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t a = a0 + ty + 16 * p, b = b0 + tx + 16 * q;
            if (a < d && b < d && a <= b) G[a * d + b] = acc[p][q];
        }
}

// colsum[j] += T[j][0] + T[j][1] + ... in cell order (FP64 form).
__global__ void k_colsum_f64(const double *__restrict__ T, int64_t d, int64_t m_pad, int64_t m,
                             double *__restrict__ colsum) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d) return;
    double acc = colsum[j];
    const double *r = T + (size_t)j * m_pad;
    for (int64_t i = 0; i < m; ++i) acc = __dadd_rn(acc, r[i]);
    colsum[j] = acc;
}

// ------------------------------------------------------------ FP32 SYRK
// 128x128 upper-triangular block tiles, 256 threads, 8x8 register tile per
// thread, K step 16 double-buffered through shared memory.  The FP32
// register accumulators are folded into FP64 (in shared memory) every
// kFoldSteps K steps, so FP32 rounding only ever spans kFoldSteps*16 cells;
// the epilogue adds the FP64 tile into G with the bias correction.
constexpr int kBM = 128, kBK = 16, kPadS = 4, kFoldSteps = 16;
constexpr size_t kSyrkF32Smem = sizeof(float) * 2 * 2 * kBK * (kBM + kPadS) + sizeof(double) * 64 * 256;

__global__ void __launch_bounds__(256) k_syrk_f32(const float *__restrict__ T, int64_t d, int64_t m_pad, int64_t nb,
                                                  const double *__restrict__ bias, const double *__restrict__ colsum_c,
                                                  const int64_t *__restrict__ n_kept, double *__restrict__ G) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float(*As)[kBK][kBM + kPadS] = reinterpret_cast<float(*)[kBK][kBM + kPadS]>(smem_raw);
    float(*Bs)[kBK][kBM + kPadS] = reinterpret_cast<float(*)[kBK][kBM + kPadS]>(smem_raw + sizeof(float) * 2 * kBK *
                                                                                                   (kBM + kPadS));
    double *acc64 = reinterpret_cast<double *>(smem_raw + sizeof(float) * 2 * 2 * kBK * (kBM + kPadS));
    int bi, bj;
    tri_decode(blockIdx.x, nb, bi, bj);
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int64_t a0 = (int64_t)bi * kBM, b0 = (int64_t)bj * kBM;
    float acc[8][8];
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            acc[p][q] = 0.0f;
            acc64[(p * 8 + q) * 256 + tid] = 0.0;
        }

    // loader: each panel is 128 rows x 16 floats = 512 float4; 2 per thread
    const int lrow = tid >> 2, lcol = (tid & 3) * 4;
    auto load = [&](int buf, int64_t k0) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int row = lrow + 64 * r;
            const float4 va = *reinterpret_cast<const float4 *>(T + (a0 + row) * m_pad + k0 + lcol);
            const float4 vb = *reinterpret_cast<const float4 *>(T + (b0 + row) * m_pad + k0 + lcol);
            As[buf][lcol + 0][row] = va.x;
            As[buf][lcol + 1][row] = va.y;
            As[buf][lcol + 2][row] = va.z;
            As[buf][lcol + 3][row] = va.w;
            Bs[buf][lcol + 0][row] = vb.x;
            Bs[buf][lcol + 1][row] = vb.y;
            Bs[buf][lcol + 2][row] = vb.z;
            Bs[buf][lcol + 3][row] = vb.w;
        }
    };
    auto fold = [&]() {
#pragma unroll
        for (int p = 0; p < 8; ++p)
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                acc64[(p * 8 + q) * 256 + tid] += (double)acc[p][q];
                acc[p][q] = 0.0f;
            }
    };
    load(0, 0);
    __syncthreads();
    int buf = 0, steps = 0;
    for (int64_t k0 = 0; k0 < m_pad; k0 += kBK) {
        if (k0 + kBK < m_pad) load(buf ^ 1, k0 + kBK);
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            float av[8], bv[8];
            const float4 a_lo = *reinterpret_cast<const float4 *>(&As[buf][kk][ty * 4]);
            const float4 a_hi = *reinterpret_cast<const float4 *>(&As[buf][kk][64 + ty * 4]);
            const float4 b_lo = *reinterpret_cast<const float4 *>(&Bs[buf][kk][tx * 4]);
            const float4 b_hi = *reinterpret_cast<const float4 *>(&Bs[buf][kk][64 + tx * 4]);
            av[0] = a_lo.x; av[1] = a_lo.y; av[2] = a_lo.z; av[3] = a_lo.w;
            av[4] = a_hi.x; av[5] = a_hi.y; av[6] = a_hi.z; av[7] = a_hi.w;
            bv[0] = b_lo.x; bv[1] = b_lo.y; bv[2] = b_lo.z; bv[3] = b_lo.w;
            bv[4] = b_hi.x; bv[5] = b_hi.y; bv[6] = b_hi.z; bv[7] = b_hi.w;
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int q = 0; q < 8; ++q) acc[p][q] = fmaf(av[p], bv[q], acc[p][q]);
        }
        if (++steps == kFoldSteps) {
            fold();
            steps = 0;
        }
        __syncthreads();
        buf ^= 1;
    }
    fold();
    const double nk = (double)*n_kept;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int64_t a = a0 + (p < 4 ? ty * 4 + p : 64 + ty * 4 + p - 4);
        if (a >= d) continue;
        const double ba = bias ? bias[a] : 0.0, ca = colsum_c[a];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int64_t b = b0 + (q < 4 ? tx * 4 + q : 64 + tx * 4 + q - 4);
            if (b >= d || b < a) continue;
            double v = acc64[(p * 8 + q) * 256 + tid];
            if (bias) {
                const double bb = bias[b], cb = colsum_c[b];
                v = v - ba * cb - ca * bb - nk * ba * bb;
            }
            G[a * d + b] += v;
        }
    }
}

__global__ void k_add_colsum(const double *__restrict__ src, int64_t d, double *__restrict__ dst) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < d) dst[j] += src[j];
}

int launch_syrk_fold(const GramWork &w, int64_t m, const DevScale &t, double *gram, double *colsum,
                     cudaStream_t st) {
    if (w.d == 0) return CREST_OK;
    const int64_t m_pad = round_up(m > 0 ? m : 1, 64);
    if (w.precision == CREST_GRAM_FP64) {
        const int64_t nb = ceil_div(w.d, 64);
        const int64_t tiles = nb * (nb + 1) / 2;
        prof::Scope ps("syrk_fp64", st);
        k_syrk_f64<<<(unsigned)tiles, 256, 0, st>>>((const double *)w.tile, w.d, m_pad, nb, gram);
        CREST_CUDA_TRY(cudaGetLastError());
        k_colsum_f64<<<(unsigned)ceil_div(w.d, 128), 128, 0, st>>>((const double *)w.tile, w.d, m_pad, m, colsum);
        CREST_CUDA_TRY(cudaGetLastError());
        return CREST_OK;
    }
    const double *bias = t.scale ? t.bias : nullptr;
    if (w.precision == CREST_GRAM_FP32) {
        const int64_t nb = w.d_pad / kBM;
        const int64_t tiles = nb * (nb + 1) / 2;
        prof::Scope ps("syrk_fp32", st);
        CREST_CUDA_TRY(
            cudaFuncSetAttribute(k_syrk_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSyrkF32Smem));
        k_syrk_f32<<<(unsigned)tiles, 256, kSyrkF32Smem, st>>>((const float *)w.tile, w.d, m_pad, nb, bias,
                                                              w.colsum_chunk, w.n_kept, gram);
        CREST_CUDA_TRY(cudaGetLastError());
    } else {
        CREST_TRY(syrk_bf16x3_fold(w, m_pad, t, gram, st));
    }
    k_add_colsum<<<(unsigned)ceil_div(w.d, 256), 256, 0, st>>>(w.colsum_chunk, w.d, colsum);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
