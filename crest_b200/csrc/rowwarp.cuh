// Warp-per-cell building blocks shared by the streaming kernels.
//
// One warp owns one cell (one span of the chunk).  Its entries are read in
// segments of 32 consecutive entries (lane j holds entry s + j), several
// segments per iteration so each warp keeps more loads in flight.  All
// per-cell f64 sums equal the reference's entry-order sums
// (src/kernels.rs:69-76, 170-183).  When every value of the cell is an
// integer below 2^24 (raw counts) all partial sums are exact, so per-lane
// partials and one shuffle tree give the identical result; otherwise the
// segments are folded lane by lane in entry order.
#pragma once

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

}  // namespace crest
