// Synthetic count-matrix generator (GPU kernels over the per-draw definition
// of synth_core.h, which a host-thread generator shares to draw the same
// matrix).  Used to make the seeded inputs of the tests and the benchmark;
// not part of the preprocessing path.

#include "host.cuh"
#include "synth_core.h"

namespace crest {
namespace {

// Warp per cell; pass 0 counts the non-zeros, pass 1 writes them in gene order.
template <int PASS>
__global__ void __launch_bounds__(256) k_synth(crest_synth p, int64_t c0, int64_t n, int64_t *row_nnz,
                                               const int64_t *indptr, uint32_t *indices, float *data) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const double phi = p.dispersion, r = 1.0 / phi;
    for (int64_t i = warp; i < n; i += n_warps) {
        const int64_t c = c0 + i;
        const double lib = p.lib[c];
        const double *pr = p.prob + (int64_t)p.labels[c] * p.n_genes;
        int64_t cnt = 0, out = PASS ? indptr[c] - indptr[c0] : 0;
        for (int64_t g0 = 0; g0 < p.n_genes; g0 += 32) {
            const int64_t g = g0 + lane;
            uint32_t k = 0;
            if (g < p.n_genes) k = syn_count(lib * pr[g], phi, r, syn_uniform(p.seed, (uint64_t)c, (uint64_t)g));
            const unsigned nz = __ballot_sync(0xffffffffu, k != 0);
            if (PASS) {
                if (k) {
                    const int64_t at = out + __popc(nz & ((1u << lane) - 1u));
                    indices[at] = (uint32_t)g;
                    data[at] = (float)k;
                }
                out += __popc(nz);
            } else {
                cnt += __popc(nz);
            }
        }
        if (!PASS && lane == 0) row_nnz[i] = cnt;
    }
}

}  // namespace
}  // namespace crest

using namespace crest;

extern "C" {

/* GPU generator writing into host buffers: rows [c0, c1) with indptr
 * absolute (indptr[c0] may be non-zero; indices/data are indexed from
 * indptr[c0]).  All parameter arrays are host arrays. */
int crest_synth_gpu(const crest_synth *p, int64_t *row_nnz, const int64_t *indptr, uint32_t *indices, float *data) {
    CREST_REQUIRE(p && p->prob && p->labels && p->lib && p->dispersion > 0, CREST_EINVAL, "bad synth parameters");
    CREST_TRY(require_device());
    DevBuf prob, labels, lib, rn, ip, idx, val;
    cudaStream_t st = 0;
    const int64_t n = p->n_cells;
    auto cleanup = [&] {
        for (auto *b : {&prob, &labels, &lib, &rn, &ip, &idx, &val}) b->release();
    };
    int rc = upload(prob, p->prob, (int64_t)p->n_clusters * p->n_genes, st);
    if (!rc) rc = upload(labels, p->labels, n, st);
    if (!rc) rc = upload(lib, p->lib, n, st);
    if (rc) {
        cleanup();
        return rc;
    }
    crest_synth dp = *p;
    dp.prob = prob.as<double>();
    dp.labels = labels.as<int32_t>();
    dp.lib = lib.as<double>();
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 8), (int64_t)device_sms() * 32);
    if (!indices) {
        rc = rn.ensure(8 * (size_t)std::max<int64_t>(n, 1));
        if (!rc) {
            k_synth<0><<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(dp, 0, n, rn.as<int64_t>(), nullptr,
                                                                                nullptr, nullptr);
            if (cudaMemcpy(row_nnz, rn.ptr, 8 * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
                set_error("synth count pass failed: %s", cudaGetErrorString(cudaGetLastError()));
                rc = CREST_ECUDA;
            }
        }
        cleanup();
        return rc;
    }
    const int64_t nnz = indptr[n] - indptr[0];
    rc = upload(ip, indptr, n + 1, st);
    if (!rc) rc = idx.ensure(4 * (size_t)std::max<int64_t>(nnz, 1));
    if (!rc) rc = val.ensure(4 * (size_t)std::max<int64_t>(nnz, 1));
    if (!rc) {
        k_synth<1><<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(dp, 0, n, nullptr, ip.as<int64_t>(),
                                                                            idx.as<uint32_t>(), val.as<float>());
        if (cudaMemcpy(indices, idx.ptr, 4 * nnz, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(data, val.ptr, 4 * nnz, cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error("synth fill pass failed: %s", cudaGetErrorString(cudaGetLastError()));
            rc = CREST_ECUDA;
        }
    }
    cleanup();
    return rc;
}

}  // extern "C"
