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

#include <type_traits>

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

int launch_tile_shift(const GramWork &w, const DevScale &t, cudaStream_t st) {
    k_tile_shift<<<(unsigned)ceil_div(w.d_pad, 256), 256, 0, st>>>(w.precision, t.bias, w.d, w.d_pad, w.shift);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ------------------------------------------------------------- HVG codes
// code[g] for a store gene id g < n_gene_map: -1 when the gene is dropped,
// sub_map[gene_map[g]] in [0, d) for an HVG column, d for another kept gene
// (it still counts towards the cell total).  One table lookup per entry
// then serves both the normalisation total and the HVG selection.  The
// same codes follow as int16 (when d < 2^15 - 1), zero-padded to a multiple
// of 8, for the kernels that copy the table to shared memory.
__global__ void k_hvg_code(const int32_t *__restrict__ gene_map, int64_t n_gene_map,
                           const int32_t *__restrict__ sub_map, int64_t n_vars, int64_t d, int32_t *__restrict__ code) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= round_up(n_gene_map, 8)) return;
    int32_t v = -1;
    if (g < n_gene_map) {
        const int32_t m = gene_map[g];
        if (m >= 0) v = (m < n_vars && sub_map[m] >= 0) ? sub_map[m] : (int32_t)d;
        code[g] = v;
    }
    if (d < 32767) const_cast<int16_t *>(codes16(code, n_gene_map))[g] = (int16_t)v;
}

size_t hvg_code_bytes(int64_t n_gene_map) {
    return 4 * (size_t)round_up(n_gene_map, 4) + 2 * (size_t)round_up(n_gene_map, 8);
}

int launch_hvg_code(const DevChunk &c, const int32_t *sub_map, int64_t n_vars, int64_t d, int32_t *code,
                    cudaStream_t st) {
    if (c.n_gene_map <= 0) return CREST_OK;
    k_hvg_code<<<(unsigned)ceil_div(round_up(c.n_gene_map, 8), 256), 256, 0, st>>>(c.gene_map, c.n_gene_map, sub_map,
                                                                                   n_vars, d, code);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// Shared-memory copy of the codes as int16 (d < 2^15 - 1) when it fits next
// to the kernel's other buffers; the global int32 table otherwise.
bool codes_in_smem(int64_t n_gene_map, int64_t d, size_t other_smem) {
    return d < 32767 && other_smem + 2 * (size_t)round_up(n_gene_map, 8) <= (size_t)kMaxSmem;
}

// ------------------------------------------------------------- densify
// Warp per cell row i of the tile (i < m_pad, padding rows included),
// written straight into the (L2-resident) tile.  Rows are handed out one at
// a time through a counter, since cells differ in length.  One read of the
// cell's entries (four per lane, 16-byte loads): lanes add up the kept
// values (the normalisation total) and queue the HVG entries (code, raw
// value), in entry order, in a per-warp shared-memory queue.  Then the row
// is filled with the zero-entry value of every gene -- the shift for kept
// cells, 0 for dropped / padding rows -- with 16-byte stores and, after a
// warp barrier that orders the two sets of stores, the queued entries are
// transformed and stored.  A cell with more than kQueue HVG entries, or
// whose total needs the in-order fold, reads its entries a second time
// (rare: such cells are the longest of a tile and would otherwise set its
// duration).  The colsum of S (FP32 / BF16X3) is privatised per block in
// shared memory.  Duplicate (cell, column) entries, which a dense tile cannot
// hold (the reference's pairwise loop adds v1^2 + v1 v2 + v2^2 for two
// entries of one gene), are detected: a cell whose HVG columns are not
// strictly increasing is searched for a repeated column (bit 1 of *status),
// or flagged as unchecked when it overflowed the queue (bit 2).
template <int MODE>  // 0 FP64 (T = S), 1 FP32 (T = S + shift), 2 BF16X3 (hi/lo of S + shift)
struct RowElem;
template <> struct RowElem<0> { using T = double; };
template <> struct RowElem<1> { using T = float; };
template <> struct RowElem<2> { using T = __nv_bfloat16; };

constexpr int kDensifyWarps = 32;
constexpr int kQueue = 512;

// Queued codes are int16 when the code table itself is (SMAP), else int32.
template <int MODE, bool SMAP>
static size_t densify_smem_fixed(int64_t d, int64_t d_pad) {
    using E = typename RowElem<MODE>::T;
    using Q = typename std::conditional<SMAP, int16_t, int32_t>::type;
    const size_t priv = MODE != 0 ? sizeof(double) * (size_t)round_up(d, 2) + sizeof(E) * (size_t)d_pad : 0;
    return priv + (size_t)kDensifyWarps * kQueue * (sizeof(Q) + sizeof(float));
}

template <int MODE, bool SMAP>
__global__ void __launch_bounds__(kDensifyWarps * 32, 1) k_densify(DevChunk c, const int32_t *__restrict__ code,
                                                                   DevScale t, const double *__restrict__ shift,
                                                                   int64_t d, int64_t d_pad, int64_t m_pad,
                                                                   void *tile, double *__restrict__ colsum,
                                                                   int64_t *n_kept, unsigned int *counter,
                                                                   int *status) {
    using E = typename RowElem<MODE>::T;
    using Q = typename std::conditional<SMAP, int16_t, int32_t>::type;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr bool priv = MODE != 0;
    // [colsum of S (f64)] [shift row (tile type)]   (MODE != 0)
    // [queue values (f32)] [queue codes (Q)] [codes (int16), SMAP]
    double *s_col = reinterpret_cast<double *>(smem);
    E *shift_row = reinterpret_cast<E *>(smem + (priv ? sizeof(double) * (size_t)round_up(d, 2) : 0));
    unsigned char *qbase = reinterpret_cast<unsigned char *>(shift_row) + (priv ? sizeof(E) * (size_t)d_pad : 0);
    float *q_x = reinterpret_cast<float *>(qbase) + (size_t)wid * kQueue;
    Q *q_code = reinterpret_cast<Q *>(qbase + sizeof(float) * (size_t)kDensifyWarps * kQueue) + (size_t)wid * kQueue;
    int16_t *s_code = reinterpret_cast<int16_t *>(qbase + (sizeof(Q) + sizeof(float)) * (size_t)kDensifyWarps * kQueue);
    if (priv) {
        for (int64_t j = threadIdx.x; j < d_pad; j += blockDim.x) shift_row[j] = (E)((shift && j < d) ? shift[j] : 0.0);
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) s_col[j] = 0.0;
    }
    if (SMAP) copy_codes16(code, c.n_gene_map, s_code);
    __syncthreads();
    auto lookup = [&](uint32_t g) -> int32_t { return SMAP ? (int32_t)s_code[g] : __ldg(code + g); };
    const int32_t dd = (int32_t)d;
    const int64_t nvec = d_pad * (int64_t)sizeof(E) / 16;
    E *hi_plane = reinterpret_cast<E *>(tile);
    E *lo_plane = hi_plane + (size_t)m_pad * d_pad;  // BF16X3 only
    const uint4 zero = make_uint4(0, 0, 0, 0);
    const bool norm = c.target_sum > 0.0;
    int kept_count = 0;
    for (;;) {
        int64_t i = 0;
        if (lane == 0) i = atomicAdd(counter, 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= m_pad) break;
        int64_t lo = 0, hi = 0, r = -1;
        if (i < c.n_spans) r = span_row(c, i, lo, hi);
        const bool kept = r >= 0;
        // one pass: total of the kept values and the queue of HVG entries
        double tsum = 0.0;
        bool ok = true, ovf = false, ordered = true;
        int nq = 0;
        int32_t carry = -1;
        if (kept) {
            for_entries_x4<true, kDensifyDepth>(c, lo, hi, lookup, [&](const int32_t (&m)[4], const float (&x)[4]) {
                bool hv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (m[u] >= 0 && norm) {
                        ok = ok && x[u] == rintf(x[u]) && fabsf(x[u]) < 16777216.0f;
                        tsum += (double)x[u];
                    }
                    hv[u] = m[u] >= 0 && m[u] < dd;
                }
                int cnt;
                int pos = nq + block_rank4(hv, cnt);
                if (cnt == 0) return;
                order_check4(hv, m, carry, ordered);
                if (nq + cnt > kQueue) {
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
        }
        // fill the row with the zero-entry values
        E *row = hi_plane + (size_t)i * d_pad;
        {
            uint4 *dst = reinterpret_cast<uint4 *>(row);
            const uint4 *src = reinterpret_cast<const uint4 *>(shift_row);
            for (int64_t v = lane; v < nvec; v += 32) dst[v] = (priv && kept) ? src[v] : zero;
            if (MODE == 2) {
                uint4 *dlo = reinterpret_cast<uint4 *>(lo_plane + (size_t)i * d_pad);
                for (int64_t v = lane; v < nvec; v += 32) dlo[v] = zero;
            }
        }
        __syncwarp();  // orders the fill before the scattered entry stores; queue visible
        if (!kept) continue;
        kept_count += 1;
        if (!__all_sync(kFull, ordered)) {
            // columns not strictly increasing: look for a repeated column
            // among the queued entries (pairwise; such cells are rare)
            bool dup = false;
            if (!ovf) {
                for (int a = lane; a < nq; a += 32)
                    for (int b = 0; b < a; ++b) dup = dup || q_code[a] == q_code[b];
            }
            if (lane == 0) atomicOr(status, ovf ? 4 : 0);
            if (__any_sync(kFull, dup) && lane == 0) atomicOr(status, 2);
        }
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
        E *row_lo = lo_plane + (size_t)i * d_pad;
        auto put = [&](int32_t sub, float x) {
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
                    row_lo[sub] = l;
                }
                atomicAdd(s_col + sub, s);
            }
        };
        if (!ovf) {
            for (int e = lane; e < nq; e += 32) put((int32_t)q_code[e], q_x[e]);
        } else {
            for_entries_by<8, true>(c, lo, hi, lookup, [&](int32_t m, float x) {
                if (m >= 0 && m < dd) put(m, x);
            });
        }
        __syncwarp();  // queue reuse
    }
    if (lane == 0 && kept_count) atomicAdd(reinterpret_cast<unsigned long long *>(n_kept), (unsigned long long)kept_count);
    if (priv) {
        __syncthreads();
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x)
            if (s_col[j] != 0.0) atomicAdd(colsum + j, s_col[j]);
    }
}

template <int MODE, bool SMAP>
static int launch_densify_k(const DevChunk &c, const int32_t *code, const DevScale &t, const double *shift,
                            const GramWork &w, int64_t m_pad, size_t smem, cudaStream_t st) {
    CREST_TRY(ensure_smem_attr((const void *)k_densify<MODE, SMAP>, smem));
    int64_t blocks = ceil_div(m_pad, kDensifyWarps);
    const int64_t cap = (int64_t)device_sms();
    if (blocks > cap) blocks = cap;
    k_densify<MODE, SMAP><<<(unsigned)blocks, kDensifyWarps * 32, smem, st>>>(c, code, t, shift, w.d, w.d_pad, m_pad,
                                                                               w.tile, w.colsum_chunk, w.n_kept,
                                                                               w.counter, w.status);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

template <int MODE>
static int launch_densify_t(const DevChunk &c, const int32_t *code, const DevScale &t, const double *shift,
                            const GramWork &w, int64_t m_pad, cudaStream_t st) {
    const size_t fixed16 = densify_smem_fixed<MODE, true>(w.d, w.d_pad);
    if (codes_in_smem(c.n_gene_map, w.d, fixed16))
        return launch_densify_k<MODE, true>(c, code, t, shift, w, m_pad,
                                            fixed16 + 2 * (size_t)round_up(c.n_gene_map, 8), st);
    const size_t fixed = densify_smem_fixed<MODE, false>(w.d, w.d_pad);
    CREST_REQUIRE(fixed <= (size_t)kMaxSmem, CREST_EINVAL, "d=%lld too large for the densify shared buffers",
                  (long long)w.d);
    return launch_densify_k<MODE, false>(c, code, t, shift, w, m_pad, fixed, st);
}

int launch_densify(const DevChunk &c, const int32_t *code, const DevScale &t, const GramWork &w,
                   cudaStream_t st) {
    CREST_REQUIRE(c.n_spans <= w.m_cap, CREST_EINVAL, "tile holds %lld cells, chunk has %lld",
                  (long long)w.m_cap, (long long)c.n_spans);
    const int64_t m_pad = round_up(c.n_spans > 0 ? c.n_spans : 1, 64);
    CREST_CUDA_TRY(cudaMemsetAsync(w.n_kept, 0, 2 * sizeof(int64_t), st));  // kept count + work counter
    CREST_CUDA_TRY(cudaMemsetAsync(w.colsum_chunk, 0, sizeof(double) * (size_t)(w.d > 0 ? w.d : 1), st));
    const double *shift = nullptr;
    if (w.precision != CREST_GRAM_FP64 && t.scale) {
        CREST_TRY(launch_tile_shift(w, t, st));
        shift = w.shift;
    }
    prof::Scope ps("densify", st);
    if (w.precision == CREST_GRAM_FP64) return launch_densify_t<0>(c, code, t, nullptr, w, m_pad, st);
    if (w.precision == CREST_GRAM_FP32) return launch_densify_t<1>(c, code, t, shift, w, m_pad, st);
    return launch_densify_t<2>(c, code, t, shift, w, m_pad, st);
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
// register accumulators are folded into FP64 register sums every kFoldSteps
// K steps, so an FP32 rounding chain only ever spans kFoldSteps*16 cells:
// the error of a chain grows with its length times the partial's magnitude,
// and at 1M cells 256-cell chains left the top-50 subspace 0.03 degree from
// the FP64 Gram's; 32-cell chains keep it an order of magnitude closer.
// The epilogue adds the FP64 tile into G with the shift correction.
constexpr int kBM = 128, kBK = 16, kPadS = 4, kFoldSteps = 2;
constexpr size_t kSyrkF32Smem = sizeof(float) * 2 * 2 * kBK * (kBM + kPadS);

__global__ void __launch_bounds__(256, 1) k_syrk_f32(const float *__restrict__ T, int64_t d, int64_t d_pad,
                                                     int64_t m_pad, int64_t nb, const double *__restrict__ shift,
                                                     const double *__restrict__ colsum_c,
                                                     const int64_t *__restrict__ n_kept, double *__restrict__ G) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float(*As)[kBK][kBM + kPadS] = reinterpret_cast<float(*)[kBK][kBM + kPadS]>(smem_raw);
    float(*Bs)[kBK][kBM + kPadS] = reinterpret_cast<float(*)[kBK][kBM + kPadS]>(smem_raw + sizeof(float) * 2 * kBK *
                                                                                                   (kBM + kPadS));
    int bi, bj;
    tri_decode(blockIdx.x, nb, bi, bj);
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int64_t a0 = (int64_t)bi * kBM, b0 = (int64_t)bj * kBM;
    float acc[8][8];
    double acc64[8][8];
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            acc[p][q] = 0.0f;
            acc64[p][q] = 0.0;
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
                acc64[p][q] += (double)acc[p][q];
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
            double v = acc64[p][q];
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
                     cudaStream_t st, bool add_colsum) {
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
        CREST_TRY(ensure_smem_attr((const void *)k_syrk_f32, (size_t)kSyrkF32Smem));
        k_syrk_f32<<<(unsigned)tiles, 256, kSyrkF32Smem, st>>>((const float *)w.tile, w.d, w.d_pad, m_pad, nb, shift,
                                                              w.colsum_chunk, w.n_kept, gram);
        CREST_CUDA_TRY(cudaGetLastError());
    } else {
        CREST_TRY(syrk_bf16x3_fold(w, m_pad, t, gram, st));
    }
    if (add_colsum) {
        k_add_colsum<<<(unsigned)ceil_div(w.d, 256), 256, 0, st>>>(w.colsum_chunk, w.d, colsum);
        CREST_CUDA_TRY(cudaGetLastError());
    }
    return CREST_OK;
}

}  // namespace crest
