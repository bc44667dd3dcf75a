// Host-side helpers shared by the C ABI translation units.
#pragma once

#include <stdlib.h>

#include <algorithm>

#include "kernels.cuh"

namespace crest {

inline int require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("no usable CUDA device (%s); the CREST GPU path has no CPU fallback",
                  e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
        return CREST_ENODEV;
    }
    return CREST_OK;
}

template <class T>
inline int upload(DevBuf &b, const T *src, int64_t n, cudaStream_t st) {
    CREST_TRY(b.ensure(sizeof(T) * (size_t)(n > 0 ? n : 1)));
    if (n > 0) CREST_CUDA_TRY(cudaMemcpyAsync(b.ptr, src, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice, st));
    return CREST_OK;
}
template <class T>
inline int zeros(DevBuf &b, int64_t n, cudaStream_t st) {
    CREST_TRY(b.ensure(sizeof(T) * (size_t)(n > 0 ? n : 1)));
    CREST_CUDA_TRY(cudaMemsetAsync(b.ptr, 0, sizeof(T) * (size_t)(n > 0 ? n : 1), st));
    return CREST_OK;
}

// Cells per Gram tile: one densify and one SYRK launch per tile, so larger
// tiles amortise the SYRK's prologue and its FP64 read-modify-write of the
// Gram, and the densify's tail.  At 1M cells (bf16x3, d = 2000) the step
// measured 50.2 / 43.0 / 42.1 / 41.2 ms with 8,192 / 32,768 / 65,536 /
// 131,072-cell tiles at the same accuracy (max angle 0.006 deg to FP64),
// and 40.0 ms (0.0065 deg) with 262,144-cell tiles over the whole resident
// matrix.  At most 2^19 (the densify's fixed-point column sums).
inline int64_t tile_cells_default() {
    const char *e = getenv("CREST_TILE_CELLS");
    int64_t v = e ? atoll(e) : 262144;
    if (v < 64) v = 64;
    if (v > ((int64_t)1 << 19)) v = (int64_t)1 << 19;
    return round_up(v, 64);
}

// A Gram tile workspace sized for d genes.
struct GramBufs {
    DevBuf tile, colsum_chunk, n_kept, shift, status, aux, colsum_part;
    int ensure(GramWork &w, int64_t d, int precision, int64_t m_cap) {
        w.d = d;
        // the tensor-core SYRK works on 256 x 256 blocks (pairs of SMs)
        w.d_pad = round_up(d > 0 ? d : 1, precision == CREST_GRAM_BF16X3 ? 256 : 128);
        w.m_cap = m_cap;
        w.precision = precision;
        CREST_TRY(tile.ensure(gram_tile_bytes(precision, w.d_pad, m_cap)));
        CREST_TRY(colsum_chunk.ensure(sizeof(double) * (size_t)w.d_pad));
        CREST_TRY(n_kept.ensure(2 * sizeof(int64_t)));  // kept count, then the work counter
        CREST_TRY(shift.ensure(sizeof(double) * (size_t)w.d_pad));
        CREST_TRY(status.ensure(sizeof(int)));
        w.tile = tile.ptr;
        w.colsum_chunk = colsum_chunk.as<double>();
        w.n_kept = n_kept.as<int64_t>();
        w.counter = reinterpret_cast<unsigned int *>(n_kept.as<int64_t>() + 1);
        w.part32 = nullptr;
        w.shift = shift.as<double>();
        w.status = status.as<int>();
        w.gram_aux = nullptr;
        w.colsum_rows = 2 * (int64_t)device_sms();
        CREST_TRY(colsum_part.ensure(sizeof(long long) * (size_t)w.colsum_rows * (size_t)w.d_pad));
        w.colsum_part = colsum_part.as<long long>();
        if (precision == CREST_GRAM_BF16X3 && d > 0) {
            const size_t bytes = sizeof(double) * (size_t)d * (size_t)d;
            const bool fresh = aux.cap < bytes;
            CREST_TRY(aux.ensure(bytes));
            if (fresh) CREST_CUDA_TRY(cudaMemset(aux.ptr, 0, bytes));
            w.gram_aux = aux.as<double>();
        }
        return CREST_OK;
    }
};

// Sub-chunk of spans [s0, s0 + n) of a staged chunk.
inline DevChunk slice(const DevChunk &c, int64_t s0, int64_t n) {
    DevChunk r = c;
    r.span_ptr = c.span_ptr + s0;
    if (c.span_cell) r.span_cell = c.span_cell + s0;
    else r.first_cell = c.first_cell + (uint32_t)s0;
    r.n_spans = n;
    return r;
}

// Chunk checks of the reference's binding (src/py.rs:162-193): lengths, one
// of cells / indptr, sorted cells, monotone indptr; gene_map values < n_vars.
int validate_chunk(const crest_chunk *c);
int check_maps(const crest_chunk *c, int64_t n_vars);

// Zero / read back the Gram work's duplicate-entry status: CREST_EINVAL when
// some cell holds an HVG column twice or could not be checked.
int gram_status_reset(const GramWork &w, cudaStream_t st);
int gram_status_check(const GramWork &w, cudaStream_t st);

// code: per-gene HVG codes from launch_hvg_code
int gram_over_chunk(const DevChunk &dc, const int32_t *code, const DevScale &ds, GramWork &w, double *gram,
                    double *colsum, cudaStream_t st);
// Per-gene HVG codes of a chunk's gene_map and sub_map into buf.
int stage_hvg_code(const DevChunk &dc, const int32_t *sub_map, int64_t n_vars, int64_t d, DevBuf &buf,
                   cudaStream_t st);

// Upload mean/std of d genes and derive bias = clip(-mean/std).
int stage_scale(DevBuf &mean, DevBuf &std_, DevBuf &bias, const crest_scale *t, int64_t d, DevScale &ds,
                cudaStream_t st);

}  // namespace crest
