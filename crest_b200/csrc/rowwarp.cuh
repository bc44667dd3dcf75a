// Warp-per-cell building blocks shared by the streaming kernels.
//
// One warp owns one cell (one span of the chunk).  Its entries are read
// either in segments of 32 consecutive entries (lane j holds entry s + j;
// for_entries) or in 128-entry blocks of four consecutive entries per lane
// with 16-byte loads (for_entries_x4, the single-pass kernels).  All
// per-cell f64 sums equal the reference's entry-order sums
// (src/kernels.rs:69-76, 170-183).  When every value of the cell is an
// integer below 2^24 (raw counts) all partial sums are exact, so per-lane
// partials and one shuffle tree give the identical result; otherwise the
// segments are folded lane by lane in entry order.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "log1pf_libm.h"

namespace crest {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Store row of span i, or -1 when the cell is dropped (ChunkView::cell,
// src/kernels.rs:65-68: cell ids beyond cell_map are dropped too).
__device__ __forceinline__ int64_t span_row(const DevChunk &c, int64_t i, int64_t &lo, int64_t &hi) {
    lo = c.span_ptr[i] - c.base;
    hi = c.span_ptr[i + 1] - c.base;
    const uint32_t cell = c.span_cell ? c.span_cell[i] : c.first_cell + (uint32_t)i;
    return (int64_t)cell < c.n_cell_map ? c.cell_map[cell] : -1;
}

// gene_map lookup; ids beyond the map are dropped (src/kernels.rs:71).
__device__ __forceinline__ int32_t map_gene(const DevChunk &c, uint32_t g) {
    return (int64_t)g < c.n_gene_map ? __ldg(c.gene_map + g) : -1;
}

// In-order fold of one segment: acc + v_0 + v_1 + ... + v_31 (lane order).
struct OrderedSum {
    double acc = 0.0;
    bool seq = false;  // warp-uniform: sequential fold required from now on
    __device__ __forceinline__ void add(double v) {
        const bool integral = (v == rint(v)) && fabs(v) < 16777216.0;
        if (!seq && __all_sync(kFull, integral)) {
            double s = v;
#pragma unroll
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
            acc = acc + s;
        } else {
            seq = true;
#pragma unroll
            for (int j = 0; j < 32; ++j) acc = __dadd_rn(acc, __shfl_sync(kFull, v, j));
        }
    }
};

// Visit the entries of [lo, hi) in segment order; f(mapped_gene, value) is
// called by all 32 lanes once per segment (warp-collective operations
// inside f are allowed).  Mapped gene is -1 for dropped or padding lanes.
// LAST: the final read of these entries in the kernel (streaming loads);
// earlier passes use cached loads so the next pass finds them in L2.
// for_entries_by: the same visit with the gene code taken from lookup(g)
// (g < n_gene_map guaranteed) instead of the chunk's gene_map.
template <int U, bool LAST, class L, class F>
__device__ __forceinline__ void for_entries_by(const DevChunk &c, int64_t lo, int64_t hi, L &&lookup, F &&f) {
    const int lane = lane_id();
    for (int64_t s = lo; s < hi; s += 32 * U) {
        uint32_t g[U];
        float x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t e = s + u * 32 + lane;
            const bool v = e < hi;
            g[u] = v ? (LAST ? __ldcs(c.genes + e) : __ldg(c.genes + e)) : 0u;
            x[u] = v ? (LAST ? __ldcs(c.values + e) : __ldg(c.values + e)) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (s + u * 32 >= hi) break;  // warp-uniform
            const int64_t e = s + u * 32 + lane;
            const int32_t m = (e < hi && (int64_t)g[u] < c.n_gene_map) ? lookup(g[u]) : -1;
            f(m, x[u]);
        }
    }
}

// Four entries per lane: lane l of a 128-entry block visits entries
// b + 4l .. b + 4l + 3 with one 16-byte load of gene ids and one of values,
// so a block is read in entry order lane by lane.  Entries before the first
// 16-byte boundary form a head block of at most 3 (lanes 0-2, one entry
// each); a partial last block is read entry by entry.  When genes and
// values do not share their alignment every block is read entry by entry.
// The loads of the next D blocks are in flight while a block is processed
// (D + 1 register buffers, indexed statically).
// f(m[4], x[4]) is called by all 32 lanes once per block; m = -1 marks
// dropped genes and empty slots.
template <bool LAST, int D = 1, class L, class F>
__device__ __forceinline__ void for_entries_x4(const DevChunk &c, int64_t lo, int64_t hi, L &&lookup, F &&f) {
    const int lane = lane_id();
    int32_t m[4];
    float x[4];
    const uintptr_t ga = reinterpret_cast<uintptr_t>(c.genes), va = reinterpret_cast<uintptr_t>(c.values);
    const bool vec = ((ga ^ va) & 15) == 0;
    int64_t b = lo;
    if (vec && lo < hi) {
        const int64_t head = (int64_t)((16 - ((ga + 4 * (uintptr_t)lo) & 15)) & 15) / 4;
        if (head > 0) {
            const int64_t hb = lo + head < hi ? lo + head : hi;
            const int64_t e = lo + lane;
            if (lane < 3 && e < hb) {
                const uint32_t g = LAST ? __ldcs(c.genes + e) : __ldg(c.genes + e);
                x[0] = LAST ? __ldcs(c.values + e) : __ldg(c.values + e);
                m[0] = (int64_t)g < c.n_gene_map ? lookup(g) : -1;
            } else {
                x[0] = 0.0f;
                m[0] = -1;
            }
            m[1] = m[2] = m[3] = -1;
            x[1] = x[2] = x[3] = 0.0f;
            f(m, x);
            b = hb;
        }
    }
    auto load = [&](int64_t bb, uint32_t (&g)[4], float (&v)[4]) {
        const int64_t e = bb + 4 * lane;
        if (vec && e + 3 < hi) {
            const uint4 g4 = LAST ? __ldcs(reinterpret_cast<const uint4 *>(c.genes + e))
                                  : __ldg(reinterpret_cast<const uint4 *>(c.genes + e));
            const float4 x4 = LAST ? __ldcs(reinterpret_cast<const float4 *>(c.values + e))
                                   : __ldg(reinterpret_cast<const float4 *>(c.values + e));
            g[0] = g4.x;
            g[1] = g4.y;
            g[2] = g4.z;
            g[3] = g4.w;
            v[0] = x4.x;
            v[1] = x4.y;
            v[2] = x4.z;
            v[3] = x4.w;
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool ok = e + u < hi;
                g[u] = ok ? (LAST ? __ldcs(c.genes + e + u) : __ldg(c.genes + e + u)) : 0u;
                v[u] = ok ? (LAST ? __ldcs(c.values + e + u) : __ldg(c.values + e + u)) : 0.0f;
            }
        }
    };
    constexpr int NB = D + 1;
    uint32_t gq[NB][4];
    float xq[NB][4];
#pragma unroll
    for (int k = 0; k < NB; ++k)
        if (b + 128 * k < hi) load(b + 128 * k, gq[k], xq[k]);
    for (; b < hi; b += 128 * NB) {
#pragma unroll
        for (int k = 0; k < NB; ++k) {
            const int64_t bb = b + 128 * k;
            if (bb >= hi) break;  // warp-uniform
            const int64_t e = bb + 4 * lane;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                x[u] = xq[k][u];
                m[u] = (e + u < hi && (int64_t)gq[k][u] < c.n_gene_map) ? lookup(gq[k][u]) : -1;
            }
            if (bb + 128 * NB < hi) load(bb + 128 * NB, gq[k], xq[k]);
            f(m, x);
        }
    }
}

// Entry-order position of this lane's first selected entry within a block
// visited by for_entries_x4, and the block's count of selected entries.
__device__ __forceinline__ int block_rank4(const bool (&sel)[4], int &count) {
    const unsigned lt = (1u << lane_id()) - 1u;
    int before = 0;
    count = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const unsigned bal = __ballot_sync(kFull, sel[u]);
        before += __popc(bal & lt);
        count += __popc(bal);
    }
    return before;
}

template <int U, bool LAST = true, class F>
__device__ __forceinline__ void for_entries(const DevChunk &c, int64_t lo, int64_t hi, F &&f) {
    for_entries_by<U, LAST>(c, lo, hi, [&](uint32_t g) { return (int32_t)__ldg(c.gene_map + g); }, f);
}

// Integer test of the fast paths: every partial sum of such values stays an
// exactly representable integer, so any summation order gives the in-order
// f64 result.
__device__ __forceinline__ bool small_integer(double v) { return v == rint(v) && fabs(v) < 16777216.0; }

// Warp sum of per-lane f64 partials (exact when they are integers).
__device__ __forceinline__ double warp_sum(double s) {
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    return s;
}

// Total of the kept-gene values of a cell when all of them are integers
// below 2^24 (raw counts): lanes keep private partial sums, one reduction at
// the end.  Returns false (and no total) when some value is not.
__device__ __forceinline__ bool integral_total(const DevChunk &c, int64_t lo, int64_t hi, double &out) {
    double s = 0.0;
    bool ok = true;
    for_entries<8, false>(c, lo, hi, [&](int32_t m, float x) {
        if (m < 0) return;
        const double v = (double)x;
        ok = ok && small_integer(v);
        s += v;
    });
    if (!__all_sync(kFull, ok)) return false;
    out = warp_sum(s);
    return true;
}

// Per-cell normalisation factor: target/total over kept genes, or 1
// (src/kernels.rs:69-78).
__device__ __forceinline__ double cell_scale(const DevChunk &c, int64_t lo, int64_t hi) {
    if (!(c.target_sum > 0.0)) return 1.0;
    double total;
    if (!integral_total(c, lo, hi, total)) {
        OrderedSum tot;
        for_entries<4, false>(c, lo, hi, [&](int32_t m, float x) { tot.add(m >= 0 ? (double)x : 0.0); });
        total = tot.acc;
    }
    return total > 0.0 ? c.target_sum / total : 1.0;
}

// The lazy transform of one value (src/kernels.rs:79-82).
__device__ __forceinline__ float transform_value(const DevChunk &c, double scale, float x) {
    float y = c.target_sum > 0.0 ? __double2float_rn(__dmul_rn((double)x, scale)) : x;
    return c.log1p ? crest_log1pf(y) : y;
}

// Transform::apply (src/kernels.rs:209-219).  bias[g] = clip(-mean/sd).
__device__ __forceinline__ double clip_mv(double z, double mv) {
    if (mv > 0.0) {
        if (z < -mv) return -mv;
        if (z > mv) return mv;
    }
    return z;
}
__device__ __forceinline__ double scale_value(const DevScale &t, int32_t g, float x) {
    if (!t.scale) return (double)x;
    const double z = __ddiv_rn(__dsub_rn((double)x, __ldg(t.mean + g)), __ldg(t.std + g));
    return __dsub_rn(clip_mv(z, t.max_value), __ldg(t.bias + g));
}

// Strictly increasing HVG columns of a cell, checked block by block of a
// for_entries_x4 visit: lane l holds entries 4l .. 4l+3 of the block, col[u]
// valid where sel[u].  carry = largest column seen in earlier blocks (-1).
__device__ __forceinline__ void order_check4(const bool (&sel)[4], const int32_t (&col)[4], int32_t &carry,
                                             bool &ok) {
    const int lane = lane_id();
    int32_t first = 0x7fffffff, last = -1;
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (sel[u]) {
            if (col[u] <= last) ok = false;
            if (first == 0x7fffffff) first = col[u];
            last = col[u];
        }
    int32_t incl = last;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl = max(incl, t);
    }
    int32_t prev = __shfl_up_sync(kFull, incl, 1);
    prev = lane == 0 ? carry : max(prev, carry);
    if (last >= 0 && first <= prev) ok = false;
    carry = max(carry, __shfl_sync(kFull, incl, 31));
}

// bf16 split of a Gram tile value (hi + lo ~ z to 2^-17 relative).  hi may
// come from a double rounding through f32: any nearby bf16 works, lo holds
// the rest.
__device__ __forceinline__ void split_bf16(double z, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(__double2float_rn(z));
    lo = __float2bfloat16_rn(__double2float_rn(z - (double)__bfloat162float(hi)));
}

}  // namespace crest
