// Shared device/host plumbing for the CREST B200 library: status codes,
// thread-local error text, CUDA error checks, a grow-only device arena and
// the device-side chunk descriptor every streaming kernel reads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "crest_gpu.h"

namespace crest {

// Last error message of the calling host thread (crest_last_error()).
void set_error(const char *fmt, ...);
const char *last_error();

struct Status {
    int code;
};

#define CREST_CUDA_TRY(expr)                                                                    \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess) {                                                                \
            ::crest::set_error("CUDA error %s at %s:%d: %s", cudaGetErrorName(_e), __FILE__,    \
                               __LINE__, cudaGetErrorString(_e));                               \
            (void)cudaGetLastError(); /* a non-sticky error must not fail the next call */      \
            return CREST_ECUDA;                                                                 \
        }                                                                                       \
    } while (0)

#define CREST_TRY(expr)              \
    do {                             \
        int _rc = (expr);            \
        if (_rc != CREST_OK) return _rc; \
    } while (0)

#define CREST_REQUIRE(cond, code, ...)          \
    do {                                        \
        if (!(cond)) {                          \
            ::crest::set_error(__VA_ARGS__);    \
            return (code);                      \
        }                                       \
    } while (0)

// A device buffer that only grows; used for per-call staging of chunk inputs.
// Device buffer that only grows.  Memory comes from a per-device
// stream-ordered pool that keeps what is returned to it (release threshold
// unbounded), so buffers freed by one call are handed to the next without
// new page mappings; plain cudaMalloc when no pool can be created.
struct DevBuf {
    void *ptr = nullptr;
    size_t cap = 0;
    bool pooled = false;
    int ensure(size_t bytes);
    void release();
    template <class T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

// Pinned host staging buffer that only grows.
struct HostBuf {
    void *ptr = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
    template <class T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Device view of one chunk of the raw count matrix (the reference's
// ChunkView, src/kernels.rs:24-32).  Entry e of span i lies in
// [span_ptr[i] - base, span_ptr[i+1] - base) of genes/values.  Spans map to
// store cells first_cell + i (CSR) or span_cell[i] (COO).
struct DevChunk {
    const uint32_t *genes;
    const float *values;
    const int64_t *span_ptr;   // [n_spans + 1]
    const uint32_t *span_cell; // [n_spans] or nullptr
    int64_t base;
    int64_t n_spans;
    uint32_t first_cell;
    const int64_t *cell_map;
    int64_t n_cell_map;
    const int32_t *gene_map;
    int64_t n_gene_map;
    double target_sum;
    int log1p;
};

// Scale transform parameters on the device (Transform, src/kernels.rs:201-219).
struct DevScale {
    int scale;
    const double *mean;  // [d]
    const double *std;   // [d]
    const double *bias;  // [d] clip(-mean/std): the value zeros map to
    double max_value;
};

}  // namespace crest
