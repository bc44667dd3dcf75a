// Gram accumulation over the HVG columns (K3 densify + K4 SYRK).
//
// src/kernels.rs:221-309 accumulates G += S^T S sparsely on the CPU.  On the
// GPU each tile of up to m_cap cells is densified into a cell-major tile
// T[m_pad][d_pad] (one contiguous row of HVG genes per cell; the cells are
// the K dimension of the contraction) that stays L2-resident, and contracted
// as a dense SYRK over the upper-triangular block tiles of G:
//
//  * FP64: T = S, CUDA-core DMUL+DADD accumulating straight into G in cell
//    order, which reproduces the reference's f64 sums bit for bit (the extra
//    terms are exact zeros);
//  * FP32 (plain form): T = S + shift with shift = bias rounded to f32, i.e.
//    the dense scaled matrix Z (centred by construction) with its repeated
//    zero value stored exactly; FP32 register-tiled SYRK, folded into G in
//    FP64 with the exact correction S^T S = T^T T - shift c^T - c shift^T -
//    n shift shift^T;
//  * BF16X3 (product form): the same values split into bf16 hi/lo tiles,
//    contracted on the tcgen05 tensor cores (k_gram_tc.cu), same FP64 fold.
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
    return n * 4;  // hi and lo bf16 tiles
}

// ----------------------------------------------------------------- shift
// Tile value of a zero entry for the centred forms: bias rounded to the tile
// precision (f32, or bf16 so that hi = shift and lo = 0), i.e. every repeated
// zero is stored exactly and the rounding error left in the tile is that of
// the stored entries only.  The epilogues correct with the same rounded value.
__global__ void k_tile_shift(int precision, const double *__restrict__ bias, int64_t d, int64_t d_pad,
                             double *__restrict__ shift) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d_pad) return;
    double v = 0.0;
    if (bias && j < d) {
        v = bias[j];
        v = precision == CREST_GRAM_FP32 ? (double)__double2float_rn(v) : (double)__bfloat162float(__double2bfloat16(v));
    }
    shift[j] = v;
}

// ------------------------------------------------------------- densify
// Warp per cell row i of the tile (i < m_pad, padding rows included).  The
// row is built in a per-warp shared-memory buffer -- the zero-entry value of
// every gene (shift for kept cells, 0 for dropped / padding rows), then the
// cell's stored HVG entries -- and written out with 16-byte stores, so the
// densified tile costs one coalesced write per element.  The colsum of S
// (FP32 / BF16X3) is privatised per block in shared memory.
template <int MODE>  // 0 FP64 (T = S), 1 FP32 (T = S + shift), 2 BF16X3 (hi/lo of S + shift)
struct RowElem;
template <> struct RowElem<0> { using T = double; };
template <> struct RowElem<1> { using T = float; };
template <> struct RowElem<2> { using T = __nv_bfloat16; };

constexpr int kDensifyWarps = 8;

// bf16 split of a tile value (hi + lo ~ z to 2^-17 relative).  hi may come
// from a double rounding through f32: any nearby bf16 works, lo holds the rest.
__device__ __forceinline__ void split_bf16(double z, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(__double2float_rn(z));
    lo = __float2bfloat16_rn(__double2float_rn(z - (double)__bfloat162float(hi)));
}

template <int MODE>
__global__ void __launch_bounds__(kDensifyWarps * 32) k_densify(DevChunk c, const int32_t *__restrict__ sub_map,
                                                               DevScale t, const double *__restrict__ shift,
                                                               int64_t d, int64_t d_pad, int64_t m_pad, void *tile,
                                                               double *__restrict__ colsum, int64_t *n_kept) {
    using E = typename RowElem<MODE>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rows_per_warp = MODE == 2 ? 2 : 1;  // bf16: hi row then lo row
    // [shift row (tile type)] [per-warp row buffers] [colsum of S (f64)]
    E *shift_row = reinterpret_cast<E *>(smem);
    E *row = shift_row + d_pad + (size_t)wid * rows_per_warp * d_pad;
    double *s_col = reinterpret_cast<double *>(smem + sizeof(E) * (size_t)(1 + kDensifyWarps * rows_per_warp) * d_pad);
    const bool priv = MODE != 0;
    for (int64_t j = threadIdx.x; j < d_pad; j += blockDim.x) shift_row[j] = (E)((shift && j < d) ? shift[j] : 0.0);
    if (priv)
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) s_col[j] = 0.0;
    __syncthreads();
    const int64_t warp = (int64_t)blockIdx.x * kDensifyWarps + wid;
    const int64_t n_warps = (int64_t)gridDim.x * kDensifyWarps;
    const int64_t nvec = d_pad * (int64_t)sizeof(E) / 16;
    int kept_count = 0;
    for (int64_t i = warp; i < m_pad; i += n_warps) {
        int64_t lo = 0, hi = 0, r = -1;
        if (i < c.n_spans) r = span_row(c, i, lo, hi);
        const bool kept = r >= 0;
        // zero-entry value of each gene: the shift row (exact in the tile type) or 0
        {
            uint4 *dst = reinterpret_cast<uint4 *>(row);
            const uint4 *src = reinterpret_cast<const uint4 *>(shift_row);
            const uint4 zero = make_uint4(0, 0, 0, 0);
            for (int64_t v = lane; v < nvec; v += 32) {
                dst[v] = kept ? src[v] : zero;
                if (MODE == 2) dst[nvec + v] = zero;
            }
        }
        __syncwarp();
        if (kept) {
            kept_count += 1;
            const double scale = cell_scale(c, lo, hi);
            for_entries<4>(c, lo, hi, [&](int32_t m, float x) {
                const int32_t sub = m >= 0 ? __ldg(sub_map + m) : -1;
                if (sub < 0) return;
                const double s = scale_value(t, sub, transform_value(c, scale, x));
                if (MODE == 0) {
                    row[sub] = s;
                } else {
                    const double z = shift ? __dadd_rn(s, __ldg(shift + sub)) : s;
                    if (MODE == 1) {
                        row[sub] = (E)__double2float_rn(z);
                    } else {
                        __nv_bfloat16 h, l;
                        split_bf16(z, h, l);
                        row[sub] = h;
                        row[d_pad + sub] = l;
                    }
                    atomicAdd(s_col + sub, s);
                }
            });
        }
        __syncwarp();
        // coalesced 16-byte stores of the finished row(s)
        const uint4 *src = reinterpret_cast<const uint4 *>(row);
        uint4 *dst = reinterpret_cast<uint4 *>(reinterpret_cast<E *>(tile) + (size_t)i * d_pad);
        for (int64_t v = lane; v < nvec; v += 32) dst[v] = src[v];
        if (MODE == 2) {
            uint4 *dst_lo = reinterpret_cast<uint4 *>(reinterpret_cast<E *>(tile) + (size_t)m_pad * d_pad +
                                                      (size_t)i * d_pad);
            for (int64_t v = lane; v < nvec; v += 32) dst_lo[v] = src[nvec + v];
        }
        __syncwarp();
    }
    if (lane == 0 && kept_count) atomicAdd(reinterpret_cast<unsigned long long *>(n_kept), (unsigned long long)kept_count);
    if (priv) {
        __syncthreads();
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x)
            if (s_col[j] != 0.0) atomicAdd(colsum + j, s_col[j]);
    }
}

template <int MODE>
static int launch_densify_t(const DevChunk &c, const int32_t *sub_map, const DevScale &t, const double *shift,
                            const GramWork &w, int64_t m_pad, cudaStream_t st) {
    using E = typename RowElem<MODE>::T;
    const int rows_per_warp = MODE == 2 ? 2 : 1;
    const size_t smem = sizeof(E) * (size_t)(1 + kDensifyWarps * rows_per_warp) * w.d_pad +
                        (MODE != 0 ? sizeof(double) * (size_t)w.d : 0);
    CREST_REQUIRE(smem <= 220 * 1024, CREST_EINVAL, "d=%lld too large for the densify row buffers", (long long)w.d);
    CREST_CUDA_TRY(cudaFuncSetAttribute(k_densify<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int64_t blocks = ceil_div(m_pad, kDensifyWarps);
    const int64_t cap = (int64_t)device_sms() * 4;
    if (blocks > cap) blocks = cap;
    k_densify<MODE><<<(unsigned)blocks, kDensifyWarps * 32, smem, st>>>(c, sub_map, t, shift, w.d, w.d_pad, m_pad,
                                                                         w.tile, w.colsum_chunk, w.n_kept);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_densify(const DevChunk &c, const int32_t *sub_map, const DevScale &t, const GramWork &w,
                   cudaStream_t st) {
    CREST_REQUIRE(c.n_spans <= w.m_cap, CREST_EINVAL, "tile holds %lld cells, chunk has %lld",
                  (long long)w.m_cap, (long long)c.n_spans);
    const int64_t m_pad = round_up(c.n_spans > 0 ? c.n_spans : 1, 64);
    CREST_CUDA_TRY(cudaMemsetAsync(w.n_kept, 0, sizeof(int64_t), st));
    CREST_CUDA_TRY(cudaMemsetAsync(w.colsum_chunk, 0, sizeof(double) * (size_t)(w.d > 0 ? w.d : 1), st));
    const double *shift = nullptr;
    if (w.precision != CREST_GRAM_FP64 && t.scale) {
        k_tile_shift<<<(unsigned)ceil_div(w.d_pad, 256), 256, 0, st>>>(w.precision, t.bias, w.d, w.d_pad, w.shift);
        CREST_CUDA_TRY(cudaGetLastError());
        shift = w.shift;
    }
    prof::Scope ps("densify", st);
    if (w.precision == CREST_GRAM_FP64) return launch_densify_t<0>(c, sub_map, t, nullptr, w, m_pad, st);
    if (w.precision == CREST_GRAM_FP32) return launch_densify_t<1>(c, sub_map, t, shift, w, m_pad, st);
    return launch_densify_t<2>(c, sub_map, t, shift, w, m_pad, st);
}

// ------------------------------------------------------------ FP64 SYRK
// Upper-triangular 64x64 block tiles; each thread owns 4x4 outputs and
// accumulates G[a][b] + T[0][a]T[0][b] + T[1][a]T[1][b] + ... in cell order
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

__global__ void __launch_bounds__(256) k_syrk_f64(const double *__restrict__ T, int64_t d, int64_t d_pad,
                                                  int64_t m_pad, int64_t nb, double *__restrict__ G) {
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
    // loader: 16 cells x 64 genes = 1024 doubles per panel; 4 per thread, coalesced along genes
    for (int64_t k0 = 0; k0 < m_pad; k0 += 16) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int idx = threadIdx.x + 256 * r;
            const int kk = idx >> 6, g = idx & 63;
            As[kk][g] = T[(k0 + kk) * d_pad + a0 + g];
            Bs[kk][g] = T[(k0 + kk) * d_pad + b0 + g];
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

// colsum[j] += T[0][j] + T[1][j] + ... in cell order (FP64 form).
__global__ void k_colsum_f64(const double *__restrict__ T, int64_t d, int64_t d_pad, int64_t m,
                             double *__restrict__ colsum) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d) return;
    double acc = colsum[j];
    for (int64_t i = 0; i < m; ++i) acc = __dadd_rn(acc, T[i * d_pad + j]);
    colsum[j] = acc;
}

// ------------------------------------------------------------ FP32 SYRK
// 128x128 upper-triangular block tiles, 256 threads, 8x8 register tile per
// thread, K step 16 double-buffered through shared memory.  The FP32
// register accumulators are folded into FP64 (in shared memory) every
// kFoldSteps K steps, so FP32 rounding only ever spans kFoldSteps*16 cells;
// the epilogue adds the FP64 tile into G with the shift correction.
constexpr int kBM = 128, kBK = 16, kPadS = 4, kFoldSteps = 16;
constexpr size_t kSyrkF32Smem = sizeof(float) * 2 * 2 * kBK * (kBM + kPadS) + sizeof(double) * 64 * 256;

__global__ void __launch_bounds__(256) k_syrk_f32(const float *__restrict__ T, int64_t d, int64_t d_pad,
                                                  int64_t m_pad, int64_t nb, const double *__restrict__ shift,
                                                  const double *__restrict__ colsum_c,
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

    // loader: a panel is 16 cells x 128 genes = 512 float4 (rows contiguous along genes)
    const int lk = tid >> 5, lg = (tid & 31) * 4;
    auto load = [&](int buf, int64_t k0) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int kk = lk + 8 * r;
            const float4 va = *reinterpret_cast<const float4 *>(T + (k0 + kk) * d_pad + a0 + lg);
            const float4 vb = *reinterpret_cast<const float4 *>(T + (k0 + kk) * d_pad + b0 + lg);
            *reinterpret_cast<float4 *>(&As[buf][kk][lg]) = va;
            *reinterpret_cast<float4 *>(&Bs[buf][kk][lg]) = vb;
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
        const double ba = shift ? shift[a] : 0.0, ca = colsum_c[a];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int64_t b = b0 + (q < 4 ? tx * 4 + q : 64 + tx * 4 + q - 4);
            if (b >= d || b < a) continue;
            double v = acc64[(p * 8 + q) * 256 + tid];
            if (shift) {
                const double bb = shift[b], cb = colsum_c[b];
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
        {
            prof::Scope ps("syrk_fp64", st);
            k_syrk_f64<<<(unsigned)tiles, 256, 0, st>>>((const double *)w.tile, w.d, w.d_pad, m_pad, nb, gram);
        }
        CREST_CUDA_TRY(cudaGetLastError());
        k_colsum_f64<<<(unsigned)ceil_div(w.d, 128), 128, 0, st>>>((const double *)w.tile, w.d, w.d_pad, m, colsum);
        CREST_CUDA_TRY(cudaGetLastError());
        return CREST_OK;
    }
    const double *shift = t.scale ? w.shift : nullptr;  // the tile's exact zero-entry value
    if (w.precision == CREST_GRAM_FP32) {
        const int64_t nb = w.d_pad / kBM;
        const int64_t tiles = nb * (nb + 1) / 2;
        prof::Scope ps("syrk_fp32", st);
        CREST_CUDA_TRY(
            cudaFuncSetAttribute(k_syrk_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSyrkF32Smem));
        k_syrk_f32<<<(unsigned)tiles, 256, kSyrkF32Smem, st>>>((const float *)w.tile, w.d, w.d_pad, m_pad, nb, shift,
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
