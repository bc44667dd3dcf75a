// Compact HVG form of a device-resident matrix for one scale + PCA step.
//
// The Gram pass (src/kernels.rs:227-309) and the projection pass (:352-371)
// both need, per cell, the normalisation total over kept genes and the
// cell's HVG entries in entry order; only about one stored entry in eight
// is an HVG entry.  k_extract16 streams the CSR once (16-byte loads, one
// warp per cell, the int16 code of every store gene in shared memory; the
// byte-class k_extract where that table does not fit): it adds
// up the kept values and writes the HVG entries (column, raw value) into the
// cell's slot of a compact array laid out like the CSR (slot of cell i =
// [indptr[i], indptr[i+1]), filled from the front), with the entry count and
// the normalisation factor per cell.  The densify kernel of every Gram tile
// and the projection then read only those entries.  Everything is formed
// again in every step; nothing is carried over between steps.
//
// Duplicate (cell, column) entries: the reference's pairwise loop gives
// v1^2 + v1 v2 + v2^2 on the diagonal for two entries of one gene, which a
// dense tile cannot represent.  The extract kernels check that every
// cell's HVG columns are strictly increasing (true for gene-sorted rows and a
// monotone column map; the check is skipped when the matrix's range index
// has shown every row strictly sorted and the column map is monotone); when
// some cell is not, k_dup_compact looks for a real duplicate with a per-warp
// bit set and the Gram pass reports an error.
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {

// --------------------------------------------------------- byte classes
// Byte g of cls: 0 dropped gene, 1 kept gene, 3 HVG column.
__global__ void k_gene_class(const int32_t *__restrict__ code, int64_t n_gene_map, int64_t d,
                             uint32_t *__restrict__ cls) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= ceil_div(n_gene_map, 4)) return;
    uint32_t v = 0;
    for (int j = 0; j < 4; ++j) {
        const int64_t g = w * 4 + j;
        if (g >= n_gene_map) break;
        const int32_t m = code[g];
        const uint32_t b = m < 0 ? 0u : (m < d ? 3u : 1u);
        v |= b << (8 * j);
    }
    cls[w] = v;
}

// words of the table, a multiple of four (whole 16-byte loads)
size_t gene_class_words(int64_t n_gene_map) { return (size_t)round_up(ceil_div(n_gene_map, 4), 4); }

int launch_gene_class(const int32_t *code, int64_t n_gene_map, int64_t d, uint32_t *cls, cudaStream_t st) {
    const int64_t nw = ceil_div(n_gene_map, 4);
    if (nw == 0) return CREST_OK;
    k_gene_class<<<(unsigned)ceil_div(nw, 256), 256, 0, st>>>(code, n_gene_map, d, cls);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ------------------------------------------------------------- extract
constexpr int kExtractWarps = 8;

__device__ __forceinline__ int64_t gene_class_words_dev(int64_t n_gene_map) {
    return round_up(ceil_div(n_gene_map, 4), 4);
}

template <int DEPTH>
__global__ void __launch_bounds__(kExtractWarps * 32, 4) k_extract(DevChunk c, const uint32_t *__restrict__ cls,
                                                                const int32_t *__restrict__ code, int32_t d,
                                                                int check_order, CompactHvg out) {
    extern __shared__ __align__(16) uint32_t s_cls[];
    const int64_t n16 = (int64_t)gene_class_words_dev(c.n_gene_map) / 4;
    for (int64_t j = threadIdx.x; j < n16; j += blockDim.x)
        reinterpret_cast<uint4 *>(s_cls)[j] = __ldg(reinterpret_cast<const uint4 *>(cls) + j);
    __syncthreads();
    const uint8_t *s_cls8 = reinterpret_cast<const uint8_t *>(s_cls);
    const int lane = lane_id();
    const int64_t warp = (int64_t)blockIdx.x * kExtractWarps + (threadIdx.x >> 5);
    const int64_t n_warps = (int64_t)gridDim.x * kExtractWarps;
    const bool norm = c.target_sum > 0.0;
    // lookup: -1 dropped gene, -2 kept gene outside the HVG columns, g for an HVG column
    auto lookup = [&](uint32_t g) -> int32_t {
        const uint32_t b = s_cls8[g];
        return b == 0u ? -1 : (b == 1u ? -2 : (int32_t)g);
    };
    bool ordered = true;
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        const int64_t row = span_row(c, i, lo, hi);
        const int64_t cell = c.first_cell + i;
        if (row < 0) {
            if (lane == 0) out.n[cell] = -1;
            continue;
        }
        int32_t *oc = out.code + lo;
        float *ox = out.x + lo;
        // kept values summed in FP32 per lane: exact while every value is a
        // non-negative integer and the lane's sum stays below 2^24 (then all
        // its partial sums do), which the end of the cell checks
        float fsum = 0.0f;
        bool integral = true;
        int nq = 0;
        int32_t carry = -1;
        for_entries_x4<true, DEPTH>(c, lo, hi, lookup, [&](const int32_t (&m)[4], const float (&x)[4]) {
            bool hv[4];
            int32_t col[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (norm) {
                    const bool kept = m[u] != -1;
                    fsum += kept ? x[u] : 0.0f;
                    integral = integral && (!kept || (x[u] == rintf(x[u]) && x[u] >= 0.0f));
                }
                hv[u] = m[u] >= 0;
                col[u] = hv[u] ? __ldg(code + m[u]) : 0;
            }
            int cnt;
            int pos = nq + block_rank4(hv, cnt);
            if (cnt == 0) return;
            if (check_order) order_check4(hv, col, carry, ordered);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (hv[u]) {
                    oc[pos] = col[u];
                    ox[pos] = x[u];
                    ++pos;
                }
            nq += cnt;
        });
        double scale = 1.0;
        if (norm) {
            double total;
            if (__all_sync(kFull, integral && fsum < 16777216.0f)) {
                total = warp_sum((double)fsum);  // integers: every order gives the in-order f64 sum
            } else {  // the reference's entry-order f64 sum
                OrderedSum ts;
                for_entries_by<4, false>(c, lo, hi, lookup, [&](int32_t m, float x) { ts.add(m != -1 ? (double)x : 0.0); });
                total = ts.acc;
            }
            scale = total > 0.0 ? c.target_sum / total : 1.0;
        }
        if (lane == 0) {
            out.n[cell] = nq;
            out.scale[cell] = scale;
        }
    }
    if (!__all_sync(kFull, ordered) && lane == 0) atomicOr(out.status, 1);
}

// ------------------------------------------------ extract, 16-bit codes
// The same pass with the int16 code of every store gene in shared memory
// (-1 dropped, d kept outside the HVG columns, else the HVG column), when
// d < 32767 and the table leaves room for two blocks per SM: one
// shared-memory load per entry gives both the class and the column.  Store
// ids past the gene map are clamped onto one extra dropped slot, so the
// full 128-entry blocks need no bounds checks; the loads of the next
// DEPTH blocks are in flight while one is processed.  Whether
// every kept value is a non-negative integer is tracked as the OR of the
// bit patterns of x - rint(x) and of the sign bit of x (zero for exactly
// those values).  The column-order check runs only when the rows are not
// known to be strictly gene-sorted under a monotone column map.
constexpr int kExtract16Warps = 8;

__host__ __device__ inline int64_t code16_slots(int64_t n_gene_map) { return round_up(n_gene_map + 1, 8); }

// The reference's entry-order f64 sum of a cell's kept values (the rare
// path: some kept value is not a small non-negative integer); out of line so
// that its registers do not weigh on the streaming loop.
__device__ __noinline__ double kept_total_ordered16(const DevChunk &c, int64_t lo, int64_t hi, const int16_t *s_code) {
    OrderedSum ts;
    for_entries_by<4, false>(c, lo, hi, [&](uint32_t g) { return s_code[g] < 0 ? -1 : 0; },
                             [&](int32_t m, float x) { ts.add(m != -1 ? (double)x : 0.0); });
    return ts.acc;
}

template <int DEPTH>
__global__ void __launch_bounds__(kExtract16Warps * 32, 3)
    k_extract16(DevChunk c, const int16_t *__restrict__ code16, int32_t d, int check_order, int known_int,
                CompactHvg out) {
    extern __shared__ __align__(16) int16_t s_code[];
    {
        const int64_t n_words = code16_slots(c.n_gene_map) / 8, n_src = round_up(c.n_gene_map, 8) / 8;
        for (int64_t j = threadIdx.x; j < n_words; j += blockDim.x)
            reinterpret_cast<uint4 *>(s_code)[j] =
                j < n_src ? __ldg(reinterpret_cast<const uint4 *>(code16) + j) : make_uint4(~0u, ~0u, ~0u, ~0u);
    }
    __syncthreads();
    const int lane = lane_id();
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t gclamp = (uint32_t)c.n_gene_map;  // a dropped slot
    const int64_t warp = (int64_t)blockIdx.x * kExtract16Warps + (threadIdx.x >> 5);
    const int64_t n_warps = (int64_t)gridDim.x * kExtract16Warps;
    const bool norm = c.target_sum > 0.0;
    const uintptr_t ga = reinterpret_cast<uintptr_t>(c.genes), va = reinterpret_cast<uintptr_t>(c.values);
    const bool vec = ((ga ^ va) & 15) == 0;
    bool ordered = true;
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        const int64_t row = span_row(c, i, lo, hi);
        const int64_t cell = c.first_cell + i;
        if (row < 0) {
            if (lane == 0) out.n[cell] = -1;
            continue;
        }
        int32_t *oc = out.code + lo;
        float *ox = out.x + lo;
        float fsum = 0.0f;  // kept values, exact while integral and below 2^24
        uint32_t bad = 0u;  // nonzero once a kept value is not a non-negative integer
        int nq = 0;
        int32_t carry = -1;
        // lane l holds entries 4l .. 4l + 3 of the block (padding: g = gclamp, x = 0)
        auto block = [&](const uint32_t(&g)[4], const float(&x)[4]) {
            int32_t v[4];
            bool hv[4];
            int before = 0, cnt = 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u] = s_code[min(g[u], gclamp)];
                if (norm) {
                    const float xk = v[u] >= 0 ? x[u] : 0.0f;
                    fsum += xk;
                    if (!known_int) bad |= __float_as_uint(xk - rintf(xk)) | (__float_as_uint(xk) & 0x80000000u);
                }
                hv[u] = (uint32_t)v[u] < (uint32_t)d;
                const unsigned bal = __ballot_sync(kFull, hv[u]);
                before += __popc(bal & lt);
                cnt += __popc(bal);
            }
            if (cnt == 0) return;  // warp-uniform
            if (check_order) order_check4(hv, v, carry, ordered);
            int pos = nq + before;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (hv[u]) {
                    oc[pos] = v[u];
                    ox[pos] = x[u];
                    ++pos;
                }
            nq += cnt;
        };
        int64_t b = lo;
        if (vec && lo < hi) {
            // up to 3 entries before the first 16-byte boundary, one per lane
            const int64_t head = (int64_t)((16 - ((ga + 4 * (uintptr_t)lo) & 15)) & 15) / 4;
            if (head > 0) {
                const int64_t hb = lo + head < hi ? lo + head : hi;
                uint32_t g[4] = {gclamp, gclamp, gclamp, gclamp};
                float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (lo + lane < hb) {
                    g[0] = __ldcs(c.genes + lo + lane);
                    x[0] = __ldcs(c.values + lo + lane);
                }
                block(g, x);
                b = hb;
            }
            // whole blocks, DEPTH of them loading ahead
            constexpr int NB = DEPTH + 1;
            const int64_t nfull = (hi - b) / 128;
            const uint4 *gp = reinterpret_cast<const uint4 *>(c.genes + b) + lane;
            const float4 *xp = reinterpret_cast<const float4 *>(c.values + b) + lane;
            uint4 gq[NB];
            float4 xq[NB];
#pragma unroll
            for (int k = 0; k < NB; ++k)
                if (k < nfull) {
                    gq[k] = __ldcs(gp + 32 * k);
                    xq[k] = __ldcs(xp + 32 * k);
                }
            for (int64_t t = 0; t < nfull; t += NB) {
#pragma unroll
                for (int k = 0; k < NB; ++k) {
                    if (t + k >= nfull) break;  // warp-uniform
                    const uint32_t g[4] = {gq[k].x, gq[k].y, gq[k].z, gq[k].w};
                    const float x[4] = {xq[k].x, xq[k].y, xq[k].z, xq[k].w};
                    if (t + k + NB < nfull) {
                        gq[k] = __ldcs(gp + 32 * (t + k + NB));
                        xq[k] = __ldcs(xp + 32 * (t + k + NB));
                    }
                    block(g, x);
                }
            }
            b += nfull * 128;
        }
        // the partial last block (or every block when genes and values are
        // not aligned alike), entry by entry
        for (; b < hi; b += 128) {
            uint32_t g[4];
            float x[4];
            const int64_t e = b + 4 * lane;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool ok = e + u < hi;
                g[u] = ok ? __ldcs(c.genes + e + u) : gclamp;
                x[u] = ok ? __ldcs(c.values + e + u) : 0.0f;
            }
            block(g, x);
        }
        double scale = 1.0;
        if (norm) {
            double total;
            if (__all_sync(kFull, bad == 0u && fsum < 16777216.0f)) {
                total = warp_sum((double)fsum);  // integers: every order gives the in-order f64 sum
            } else {
                total = kept_total_ordered16(c, lo, hi, s_code);
            }
            scale = total > 0.0 ? c.target_sum / total : 1.0;
        }
        if (lane == 0) {
            out.n[cell] = nq;
            out.scale[cell] = scale;
        }
    }
    if (!__all_sync(kFull, ordered) && lane == 0) atomicOr(out.status, 1);
}

int launch_extract(const DevChunk &c, const uint32_t *cls, const int32_t *code, int64_t d, const CompactHvg &out,
                   bool check_order, cudaStream_t st, bool known_int) {
    if (c.n_spans == 0) return CREST_OK;
    CREST_REQUIRE(!c.span_cell, CREST_EINVAL, "extract needs CSR chunks");
    if (d < 32767) {  // the int16 codes exist (launch_hvg_code)
        // one block loading ahead: two measured 4.58 against 4.49 ms at 1M cells
        const void *fn = (const void *)k_extract16<1>;
        const size_t smem = 2 * (size_t)code16_slots(c.n_gene_map);
        int per_sm = 0;
        if (smem <= (size_t)kMaxSmem) {
            CREST_TRY(ensure_smem_attr(fn, smem));
            CREST_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kExtract16Warps * 32, smem));
        }
        if (per_sm >= 2) {
            const int64_t blocks =
                std::min<int64_t>(ceil_div(c.n_spans, kExtract16Warps), (int64_t)device_sms() * per_sm);
            prof::Scope ps("extract_csr", st);
            k_extract16<1><<<(unsigned)blocks, kExtract16Warps * 32, smem, st>>>(
                c, codes16(code, c.n_gene_map), (int32_t)d, check_order ? 1 : 0, known_int ? 1 : 0, out);
            CREST_CUDA_TRY(cudaGetLastError());
            return CREST_OK;
        }
    }
    const size_t smem = 4 * gene_class_words(c.n_gene_map);
    CREST_REQUIRE(smem <= (size_t)kMaxSmem, CREST_EINVAL, "too many genes for the class table");
    CREST_TRY(ensure_smem_attr((const void *)k_extract<1>, smem));
    int per_sm = 0;
    CREST_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extract<1>, kExtractWarps * 32, smem));
    const int64_t blocks = std::min<int64_t>(ceil_div(c.n_spans, kExtractWarps), (int64_t)device_sms() * std::max(per_sm, 1));
    prof::Scope ps("extract_csr", st);
    k_extract<1><<<(unsigned)blocks, kExtractWarps * 32, smem, st>>>(c, cls, code, (int32_t)d, check_order ? 1 : 0,
                                                                     out);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ------------------------------------------------- exact duplicate check
// Warp per cell with a bit set of d columns in shared memory: a column met
// twice in one cell sets bit 1 of *status.
constexpr int kDupWarps = 8;

__global__ void __launch_bounds__(kDupWarps * 32) k_dup_compact(const int64_t *__restrict__ indptr,
                                                                int64_t n_cells, CompactHvg in, int32_t d) {
    extern __shared__ uint32_t s_bits[];
    const int lane = lane_id(), wid = threadIdx.x >> 5;
    const int nw = (d + 31) >> 5;
    uint32_t *bits = s_bits + (size_t)wid * nw;
    const int64_t warp = (int64_t)blockIdx.x * kDupWarps + wid;
    const int64_t n_warps = (int64_t)gridDim.x * kDupWarps;
    bool dup = false;
    for (int64_t i = warp; i < n_cells; i += n_warps) {
        const int n = in.n[i];
        if (n <= 0) continue;
        for (int j = lane; j < nw; j += 32) bits[j] = 0u;
        __syncwarp();
        const int32_t *cc = in.code + indptr[i];
        for (int e = lane; e < n; e += 32) {
            const int32_t col = cc[e];
            const uint32_t bit = 1u << (col & 31);
            if (atomicOr(bits + (col >> 5), bit) & bit) dup = true;
        }
        __syncwarp();
    }
    if (__any_sync(kFull, dup) && lane == 0) atomicOr(in.status, 2);
}

int launch_dup_compact(const int64_t *indptr, int64_t n_cells, const CompactHvg &in, int64_t d, cudaStream_t st) {
    if (n_cells == 0 || d == 0) return CREST_OK;
    const size_t smem = sizeof(uint32_t) * (size_t)kDupWarps * (size_t)((d + 31) / 32);
    CREST_REQUIRE(smem <= (size_t)kMaxSmem, CREST_EINVAL, "d=%lld too large for the duplicate check", (long long)d);
    CREST_TRY(ensure_smem_attr((const void *)k_dup_compact, smem));
    const int64_t blocks = std::min<int64_t>(ceil_div(n_cells, kDupWarps), (int64_t)device_sms() * 8);
    k_dup_compact<<<(unsigned)blocks, kDupWarps * 32, smem, st>>>(indptr, n_cells, in, (int32_t)d);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ------------------------------------------------------------- densify
// Tile row i < m_pad = cell cell0 + i of the compact form (padding rows past
// n_cells and dropped cells are rows of zeros).  The row is filled with the
// zero-entry value of every column (the shift; zeros for dropped / padding
// rows) with 16-byte stores, then the cell's entries are transformed and
// stored after a warp barrier -- the tile matches the CSR densify bit for
// bit.  The colsum of S is privatised per block in shared memory.
constexpr int kDensifyCWarps = 16;
constexpr int kDensifyU = 8;  // entry loads in flight per lane

template <int MODE> struct CElem;
template <> struct CElem<0> { using T = double; };
template <> struct CElem<1> { using T = float; };
template <> struct CElem<2> { using T = __nv_bfloat16; };

template <int MODE, int MINB, int DU>
__global__ void __launch_bounds__(kDensifyCWarps * 32, MINB) k_densify_compact(
    const int64_t *__restrict__ indptr, int64_t cell0, int64_t n_cells, CompactHvg in, double target_sum, int log1p,
    DevScale t, const double *__restrict__ shift, int64_t d, int64_t d_pad, int64_t m_pad, void *tile,
    double *__restrict__ colsum, long long *__restrict__ col_part, int64_t *n_kept) {
    using E = typename CElem<MODE>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool priv = MODE != 0;
    // column sums of the stored entries' scaled values in 32.32 fixed point
    // (native 64-bit integer shared atomics; exact, so the block's partial
    // does not depend on the order of the adds); |s| >= 2^12 goes straight
    // to the f64 global sum, so a block's total over a tile (at most 2^19
    // cells) stays below 2^31 and cannot overflow.  Each block writes its row of partials; k_colsum_reduce adds
    // them up in block order.
    // (Keeping each column's mean, std, bias and shift in shared memory
    // instead of four L1 gathers per entry measured slower: 6.76 against
    // 6.43 ms per 1M-cell step -- fewer long-scoreboard stalls, more
    // shared-memory and barrier stalls.)
    long long *s_col = reinterpret_cast<long long *>(smem);
    E *shift_row = reinterpret_cast<E *>(smem + (priv ? sizeof(double) * (size_t)round_up(d, 2) : 0));
    if (priv) {
        for (int64_t j = threadIdx.x; j < d_pad; j += blockDim.x) shift_row[j] = (E)((shift && j < d) ? shift[j] : 0.0);
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) s_col[j] = 0;
    }
    __syncthreads();
    const int lane = lane_id();
    const int64_t warp = (int64_t)blockIdx.x * kDensifyCWarps + (threadIdx.x >> 5);
    const int64_t n_warps = (int64_t)gridDim.x * kDensifyCWarps;
    const int64_t nvec = d_pad * (int64_t)sizeof(E) / 16;
    E *hi_plane = reinterpret_cast<E *>(tile);
    E *lo_plane = hi_plane + (size_t)m_pad * d_pad;  // BF16X3 only
    const uint4 zero = make_uint4(0, 0, 0, 0);
    DevChunk tc;  // only target_sum / log1p are read by transform_value
    tc.target_sum = target_sum;
    tc.log1p = log1p;
    int kept_count = 0;
    for (int64_t i = warp; i < m_pad; i += n_warps) {
        const int64_t cell = cell0 + i;
        const int n = i < n_cells ? in.n[cell] : -1;
        const bool kept = n >= 0;
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
        __syncwarp();  // orders the fill before the scattered entry stores
        if (!kept) continue;
        kept_count += 1;
        const double scale = in.scale[cell];
        const int64_t base = indptr[cell];
        E *row_lo = lo_plane + (size_t)i * d_pad;
        // the cell's entries in rounds of 32 x kDensifyU, every load of a
        // round issued before the first is used
        for (int e0 = 0; e0 < n; e0 += 32 * DU) {
            int32_t subs[DU];
            float xs[DU];
#pragma unroll
            for (int u = 0; u < DU; ++u) {
                const int e = e0 + 32 * u + lane;
                subs[u] = e < n ? __ldcs(in.code + base + e) : -1;
                xs[u] = e < n ? __ldcs(in.x + base + e) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < DU; ++u) {
            const int32_t sub = subs[u];
            if (sub < 0) continue;
            const double s = scale_value(t, sub, transform_value(tc, scale, xs[u]));
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
                if (fabs(s) < 4096.0)
                    atomicAdd(reinterpret_cast<unsigned long long *>(s_col + sub),
                              (unsigned long long)__double2ll_rn(s * 4294967296.0));
                else
                    atomicAdd(colsum + sub, s);
            }
            }
        }
    }
    if (lane == 0 && kept_count) atomicAdd(reinterpret_cast<unsigned long long *>(n_kept), (unsigned long long)kept_count);
    if (priv) {
        __syncthreads();
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) col_part[(int64_t)blockIdx.x * d + j] = s_col[j];
    }
}

// colsum[j] += (sum over blocks of part[b][j]) 2^-32: an exact integer sum,
// one warp per column (lanes over blocks).  With `pass`, the tile's finished
// column sum is also added there (the sum over the whole Gram pass).
__global__ void k_colsum_reduce(const long long *__restrict__ part, int nb, int64_t d, double *__restrict__ colsum,
                                double *__restrict__ pass) {
    const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= d) return;
    long long s = 0;
    for (int b = lane; b < nb; b += 32) s += part[(int64_t)b * d + j];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double v = colsum[j] + (double)s * 0x1.0p-32;
        colsum[j] = v;
        if (pass) pass[j] += v;
    }
}

// Two resident blocks of 16 warps per SM, eight entry loads per lane in
// flight (64 registers).  Three blocks with four loads each (40 registers)
// measured slower at 1M cells: 6.77 against 6.43 ms per step.
template <int MODE, int MINB, int DU>
static int densify_compact_t(const int64_t *indptr, int64_t cell0, int64_t n, const CompactHvg &in,
                             double target_sum, int log1p, const DevScale &t, const double *shift,
                             const GramWork &w, int64_t m_pad, cudaStream_t st, double *col_pass) {
    using E = typename CElem<MODE>::T;
    const auto kern = k_densify_compact<MODE, MINB, DU>;
    const size_t smem = MODE != 0 ? sizeof(double) * (size_t)round_up(w.d, 2) + sizeof(E) * (size_t)w.d_pad : 0;
    CREST_REQUIRE(smem <= (size_t)kMaxSmem, CREST_EINVAL, "d=%lld too large for the densify buffers", (long long)w.d);
    CREST_TRY(ensure_smem_attr((const void *)kern, smem));
    int per_sm = 0;
    CREST_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kDensifyCWarps * 32, smem));
    // the rows of the column-sum partials bound the block count
    const int64_t blocks = std::min<int64_t>(ceil_div(m_pad, kDensifyCWarps),
                                             std::min<int64_t>(w.colsum_rows, (int64_t)device_sms() * std::max(per_sm, 1)));
    kern<<<(unsigned)blocks, kDensifyCWarps * 32, smem, st>>>(indptr, cell0, n, in, target_sum, log1p, t, shift, w.d,
                                                              w.d_pad, m_pad, w.tile, w.colsum_chunk, w.colsum_part,
                                                              w.n_kept);
    CREST_CUDA_TRY(cudaGetLastError());
    if (MODE != 0 && w.d > 0) {
        k_colsum_reduce<<<(unsigned)ceil_div(w.d * 32, 256), 256, 0, st>>>(w.colsum_part, (int)blocks, w.d,
                                                                          w.colsum_chunk, col_pass);
        CREST_CUDA_TRY(cudaGetLastError());
    }
    return CREST_OK;
}

template <int MODE>
static int densify_compact_t(const int64_t *indptr, int64_t cell0, int64_t n, const CompactHvg &in,
                             double target_sum, int log1p, const DevScale &t, const double *shift,
                             const GramWork &w, int64_t m_pad, cudaStream_t st, double *col_pass) {
    return densify_compact_t<MODE, 2, kDensifyU>(indptr, cell0, n, in, target_sum, log1p, t, shift, w, m_pad, st,
                                                 col_pass);
}

int launch_densify_compact(const int64_t *indptr, int64_t cell0, int64_t n, const CompactHvg &in, double target_sum,
                           int log1p, const DevScale &t, const GramWork &w, cudaStream_t st, double *colsum_pass,
                           bool shift_ready) {
    CREST_REQUIRE(n <= w.m_cap, CREST_EINVAL, "tile holds %lld cells, piece has %lld", (long long)w.m_cap,
                  (long long)n);
    CREST_REQUIRE(n <= ((int64_t)1 << 19), CREST_EINVAL, "a Gram tile holds at most 2^19 cells (got %lld)",
                  (long long)n);
    const int64_t m_pad = round_up(n > 0 ? n : 1, 64);
    CREST_CUDA_TRY(cudaMemsetAsync(w.n_kept, 0, 2 * sizeof(int64_t), st));
    CREST_CUDA_TRY(cudaMemsetAsync(w.colsum_chunk, 0, sizeof(double) * (size_t)(w.d > 0 ? w.d : 1), st));
    const double *shift = nullptr;
    if (w.precision != CREST_GRAM_FP64 && t.scale) {
        if (!shift_ready) CREST_TRY(launch_tile_shift(w, t, st));  // the same for every tile of a pass
        shift = w.shift;
    }
    prof::Scope ps("densify", st);
    if (w.precision == CREST_GRAM_FP64)
        return densify_compact_t<0>(indptr, cell0, n, in, target_sum, log1p, t, nullptr, w, m_pad, st, colsum_pass);
    if (w.precision == CREST_GRAM_FP32)
        return densify_compact_t<1>(indptr, cell0, n, in, target_sum, log1p, t, shift, w, m_pad, st, colsum_pass);
    return densify_compact_t<2>(indptr, cell0, n, in, target_sum, log1p, t, shift, w, m_pad, st, colsum_pass);
}

// ------------------------------------------------------------ project
// Warp per cell: the cell's compact entries are transformed in rounds of
// STAGE (lanes in parallel, staged in shared memory), then added in entry
// order into KPL f64 accumulators per lane (component lane + 32 q), the V
// rows of U entries loaded before their ordered additions -- the same f64
// operations in the same order as src/kernels.rs:360-369, so the scores are
// bit-identical to the CSR projection.
//
// (Keeping the loadings rows of the most frequent columns in shared memory --
// one 1,024-thread CTA per SM instead of four 512-thread ones -- measured
// 7.5 ms against 5.1 ms at 1M cells: the pass is bound by each warp's
// dependent chains, not by the L2 reads of V.)
constexpr int kPCWarps = 16;
constexpr int kPCStage = 256;

template <int KPL>
__global__ void __launch_bounds__(kPCWarps * 32) k_project_compact(const int64_t *__restrict__ indptr,
                                                                   int64_t n_cells, const int64_t *__restrict__ cell_map,
                                                                   CompactHvg in, double target_sum, int log1p,
                                                                   DevScale t, const double *__restrict__ V, int k,
                                                                   float *__restrict__ out) {
    constexpr int U = KPL >= 2 ? 4 : 8, WARPS = kPCWarps, STAGE = kPCStage;
    __shared__ double s_val[WARPS][STAGE];
    __shared__ int32_t s_code[WARPS][STAGE];
    auto vrow = [&](int32_t c) -> const double * { return V + (size_t)c * k; };
    const int lane = lane_id(), wid = threadIdx.x >> 5;
    double *q_val = s_val[wid];
    int32_t *q_code = s_code[wid];
    const int64_t warp = (int64_t)blockIdx.x * WARPS + wid;
    const int64_t n_warps = (int64_t)gridDim.x * WARPS;
    DevChunk tc;
    tc.target_sum = target_sum;
    tc.log1p = log1p;
    for (int64_t i = warp; i < n_cells; i += n_warps) {
        const int n = in.n[i];
        if (n < 0) continue;
        const int64_t row = cell_map[i];
        const double scale = in.scale[i];
        const int64_t base = indptr[i];
        double acc[KPL];
#pragma unroll
        for (int q = 0; q < KPL; ++q) acc[q] = 0.0;
        for (int r0 = 0; r0 < n; r0 += STAGE) {
            const int m = n - r0 < STAGE ? n - r0 : STAGE;
            __syncwarp();
            for (int e = lane; e < m; e += 32) {
                const int32_t sub = __ldcs(in.code + base + r0 + e);
                q_code[e] = sub;
                q_val[e] = scale_value(t, sub, transform_value(tc, scale, __ldcs(in.x + base + r0 + e)));
            }
            __syncwarp();
            int e = 0;
            for (; e + U <= m; e += U) {
                double vv[U][KPL];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double *vr = vrow(q_code[e + u]);
#pragma unroll
                    for (int q = 0; q < KPL; ++q) {
                        const int j = lane + 32 * q;
                        vv[u][q] = j < k ? vr[j] : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double sv = q_val[e + u];
#pragma unroll
                    for (int q = 0; q < KPL; ++q) acc[q] = __dadd_rn(acc[q], __dmul_rn(sv, vv[u][q]));
                }
            }
            for (; e < m; ++e) {
                const double *vr = vrow(q_code[e]);
                const double sv = q_val[e];
#pragma unroll
                for (int q = 0; q < KPL; ++q) {
                    const int j = lane + 32 * q;
                    if (j < k) acc[q] = __dadd_rn(acc[q], __dmul_rn(sv, vr[j]));
                }
            }
        }
        float *o = out + (size_t)row * k;
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            const int j = lane + 32 * q;
            if (j < k) atomicAdd(o + j, __double2float_rn(acc[q]));
        }
    }
}

// The same pass for an even k above 32: lane l owns the column pairs
// (2l, 2l + 1) and (64 + 2l, 65 + 2l) (NP pairs), read as one 16-byte load
// each, so an entry costs NP row loads instead of 2 NP; the staged columns
// and values of 8 entries are read from shared memory as vectors.  Every
// column still sees the same f64 multiplies and additions in entry order.
template <int NP>
__global__ void __launch_bounds__(kPCWarps * 32) k_project_pairs(const int64_t *__restrict__ indptr,
                                                                 int64_t n_cells, const int64_t *__restrict__ cell_map,
                                                                 CompactHvg in, double target_sum, int log1p,
                                                                 DevScale t, const double *__restrict__ V, int k,
                                                                 float *__restrict__ out) {
    constexpr int U = 8, WARPS = kPCWarps, STAGE = kPCStage;
    __shared__ __align__(16) double s_val[WARPS][STAGE];
    __shared__ __align__(16) int32_t s_code[WARPS][STAGE];
    const int lane = lane_id(), wid = threadIdx.x >> 5;
    double *q_val = s_val[wid];
    int32_t *q_code = s_code[wid];
    const int64_t warp = (int64_t)blockIdx.x * WARPS + wid;
    const int64_t n_warps = (int64_t)gridDim.x * WARPS;
    bool ok[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) ok[p] = 64 * p + 2 * lane < k;
    DevChunk tc;
    tc.target_sum = target_sum;
    tc.log1p = log1p;
    for (int64_t i = warp; i < n_cells; i += n_warps) {
        const int n = in.n[i];
        if (n < 0) continue;
        const int64_t row = cell_map[i];
        const double scale = in.scale[i];
        const int64_t base = indptr[i];
        double2 acc[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) acc[p] = make_double2(0.0, 0.0);
        auto add = [&](double sv, const double2 &v, double2 &a) {
            a.x = __dadd_rn(a.x, __dmul_rn(sv, v.x));
            a.y = __dadd_rn(a.y, __dmul_rn(sv, v.y));
        };
        for (int r0 = 0; r0 < n; r0 += STAGE) {
            const int m = n - r0 < STAGE ? n - r0 : STAGE;
            __syncwarp();
            for (int e = lane; e < m; e += 32) {
                const int32_t sub = __ldcs(in.code + base + r0 + e);
                q_code[e] = sub;
                q_val[e] = scale_value(t, sub, transform_value(tc, scale, __ldcs(in.x + base + r0 + e)));
            }
            __syncwarp();
            int e = 0;
            for (; e + U <= m; e += U) {
                const int4 c0 = *reinterpret_cast<const int4 *>(q_code + e);
                const int4 c1 = *reinterpret_cast<const int4 *>(q_code + e + 4);
                const int32_t cc[U] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
                double2 vv[U][NP];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double2 *vr = reinterpret_cast<const double2 *>(V + (size_t)cc[u] * k) + lane;
#pragma unroll
                    for (int p = 0; p < NP; ++p) vv[u][p] = ok[p] ? __ldg(vr + 32 * p) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < U; u += 2) {
                    const double2 sv = *reinterpret_cast<const double2 *>(q_val + e + u);
#pragma unroll
                    for (int p = 0; p < NP; ++p) add(sv.x, vv[u][p], acc[p]);
#pragma unroll
                    for (int p = 0; p < NP; ++p) add(sv.y, vv[u + 1][p], acc[p]);
                }
            }
            for (; e < m; ++e) {
                const double2 *vr = reinterpret_cast<const double2 *>(V + (size_t)q_code[e] * k) + lane;
                const double sv = q_val[e];
#pragma unroll
                for (int p = 0; p < NP; ++p)
                    if (ok[p]) add(sv, __ldg(vr + 32 * p), acc[p]);
            }
        }
        float *o = out + (size_t)row * k;
#pragma unroll
        for (int p = 0; p < NP; ++p)
            if (ok[p]) {
                const int j = 64 * p + 2 * lane;
                atomicAdd(o + j, __double2float_rn(acc[p].x));
                atomicAdd(o + j + 1, __double2float_rn(acc[p].y));
            }
    }
}

template <class K>
static int project_launch(K kern, const int64_t *indptr, int64_t n_cells, const int64_t *cell_map,
                          const CompactHvg &in, double target_sum, int log1p, const DevScale &t, const double *V, int k,
                          float *out, cudaStream_t st) {
    int per_sm = 0;
    CREST_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPCWarps * 32, 0));
    const int64_t blocks = std::min<int64_t>(ceil_div(n_cells, kPCWarps), (int64_t)device_sms() * std::max(per_sm, 1));
    kern<<<(unsigned)blocks, kPCWarps * 32, 0, st>>>(indptr, n_cells, cell_map, in, target_sum, log1p, t, V, k, out);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

template <int KPL>
static int project_compact_k(const int64_t *indptr, int64_t n_cells, const int64_t *cell_map, const CompactHvg &in,
                             double target_sum, int log1p, const DevScale &t, const double *V, int k, float *out,
                             cudaStream_t st) {
    int per_sm = 0;
    CREST_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_project_compact<KPL>, kPCWarps * 32, 0));
    const int64_t blocks = std::min<int64_t>(ceil_div(n_cells, kPCWarps), (int64_t)device_sms() * std::max(per_sm, 1));
    k_project_compact<KPL><<<(unsigned)blocks, kPCWarps * 32, 0, st>>>(indptr, n_cells, cell_map, in, target_sum,
                                                                       log1p, t, V, k, out);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int launch_project_compact(const int64_t *indptr, int64_t n_cells, const int64_t *cell_map, const CompactHvg &in,
                           double target_sum, int log1p, const DevScale &t, const double *V, int k, int64_t d,
                           float *out, cudaStream_t st) {
    if (n_cells == 0 || k == 0) return CREST_OK;
    CREST_REQUIRE(k <= 128, CREST_EINVAL, "project supports k <= 128 (got %d)", k);
    (void)d;
    prof::Scope ps("project_compact", st);
    const bool pairs = k > 32 && k % 2 == 0 && (reinterpret_cast<uintptr_t>(V) & 15) == 0;
    if (pairs && k <= 64)
        return project_launch(k_project_pairs<1>, indptr, n_cells, cell_map, in, target_sum, log1p, t, V, k, out, st);
    if (pairs) return project_launch(k_project_pairs<2>, indptr, n_cells, cell_map, in, target_sum, log1p, t, V, k, out, st);
    if (k <= 32) return project_compact_k<1>(indptr, n_cells, cell_map, in, target_sum, log1p, t, V, k, out, st);
    if (k <= 64) return project_compact_k<2>(indptr, n_cells, cell_map, in, target_sum, log1p, t, V, k, out, st);
    return project_compact_k<4>(indptr, n_cells, cell_map, in, target_sum, log1p, t, V, k, out, st);
}

}  // namespace crest

namespace crest {

// ------------------------------------- compact form of a streamed matrix
// A streamed (host-resident) matrix has no CSR on the device to hold the
// compact form in place, so each chunk is extracted into a chunk-sized
// scratch (cell slots as in its chunk buffer) and the cells' HVG entries are
// then packed into one device array at running offsets: off[cell] = the
// entries of all earlier cells.  *total carries the offset from chunk to
// chunk; a cell whose entries would pass `cap` sets bit 3 of *status and is
// left out (the caller then projects from the CSR instead).

// Exclusive scan of the chunk's entry counts (one CTA, cells [c0, c0 + n)).
__global__ void __launch_bounds__(1024) k_compact_offsets(const int32_t *__restrict__ cnt, int64_t c0, int64_t n,
                                                          int64_t *__restrict__ off,
                                                          unsigned long long *__restrict__ total, int64_t cap,
                                                          int *__restrict__ status) {
    __shared__ long long warp_sums[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t per = (n + blockDim.x - 1) / blockDim.x, i0 = min(n, (int64_t)tid * per), i1 = min(n, i0 + per);
    long long mine = 0;
    for (int64_t i = i0; i < i1; ++i) mine += max(cnt[c0 + i], 0);
    long long incl = mine;  // inclusive scan over the block
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        long long w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += v;
        }
        warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const long long base = (long long)*total;
    long long run = base + (wid ? warp_sums[wid - 1] : 0) + incl - mine;
    for (int64_t i = i0; i < i1; ++i) {
        off[c0 + i] = run;
        run += max(cnt[c0 + i], 0);
    }
    __syncthreads();
    if (tid == 0) {
        const long long end = base + warp_sums[((blockDim.x >> 5)) - 1];
        if (end > cap) atomicOr(status, 8);
        *total = (unsigned long long)end;
    }
}

// Warp per cell: its n entries from the chunk scratch (slot at
// span_ptr[i] - base) to the packed array at off[cell].
__global__ void __launch_bounds__(256) k_compact_move(const int64_t *__restrict__ span_ptr, int64_t base, int64_t c0,
                                                      int64_t n, const int32_t *__restrict__ cnt,
                                                      const int64_t *__restrict__ off, const int32_t *__restrict__ sc,
                                                      const float *__restrict__ sx, int32_t *__restrict__ dc,
                                                      float *__restrict__ dx, int64_t cap) {
    const int lane = lane_id();
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int m = cnt[c0 + i];
        if (m <= 0) continue;
        const int64_t o = off[c0 + i], s = span_ptr[i] - base;
        if (o + m > cap) continue;
        for (int e = lane; e < m; e += 32) {
            dc[o + e] = sc[s + e];
            dx[o + e] = sx[s + e];
        }
    }
}

int launch_compact_pack(const DevChunk &c, const CompactHvg &scratch, const CompactHvg &packed, int64_t *off,
                        unsigned long long *total, int64_t cap, cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    k_compact_offsets<<<1, 1024, 0, st>>>(packed.n, c.first_cell, c.n_spans, off, total, cap, packed.status);
    CREST_CUDA_TRY(cudaGetLastError());
    const int64_t blocks = std::min<int64_t>(ceil_div(c.n_spans, 8), (int64_t)device_sms() * 8);
    k_compact_move<<<(unsigned)blocks, 256, 0, st>>>(c.span_ptr, c.base, c.first_cell, c.n_spans, packed.n, off,
                                                     scratch.code, scratch.x, packed.code, packed.x, cap);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
