// Exact k nearest neighbours of the rows of a dense n x d f32 matrix (the
// PCA scores), self excluded (src/knn.rs:337-371 knn, :136-152 knn_brute).
//
// One thread per query row; the candidate rows stream through shared memory
// in tiles of kTile rows that every thread of the block compares against its
// query (held in registers).  Every distance is computed exactly as the
// reference's final distances (src/knn.rs:48-66 sq_dist): f32 differences
// squared and added into eight partial sums over 8-wide chunks of the
// coordinates, the partials added in order, the remaining coordinates added
// one by one, every operation separately rounded.  A thread keeps its k best
// (squared distance, index) pairs sorted, candidates visited in index order,
// so ties keep the lower index; at the end the distances become square roots
// and each row is put in (distance, index) order, the reference's final sort
// (src/knn.rs:357-366).  All n rows are candidates: no approximation for any
// n (the reference switches to an IVF index above 20,000 rows).
#include "kernels.cuh"
#include "prof.cuh"

namespace crest {

constexpr int kKnnThreads = 128;
constexpr int kKnnTile = 128;
constexpr int kKnnMaxD = 128;
constexpr int kKnnMaxK = 64;

template <int D8>  // number of 8-wide chunks held in registers (d <= 8 * D8)
__global__ void __launch_bounds__(kKnnThreads) k_knn(const float *__restrict__ X, int64_t n, int d, int k,
                                                     uint32_t *__restrict__ out_idx, float *__restrict__ out_dist) {
    extern __shared__ float tile[];  // kKnnTile x d
    const int64_t q = (int64_t)blockIdx.x * kKnnThreads + threadIdx.x;
    const bool active = q < n;
    float xq[8 * D8];
#pragma unroll
    for (int j = 0; j < 8 * D8; ++j) xq[j] = (active && j < d) ? X[q * d + j] : 0.0f;
    const int full = d / 8;  // complete 8-wide chunks
    float best_d[kKnnMaxK];
    uint32_t best_i[kKnnMaxK];
    for (int j = 0; j < k; ++j) {
        best_d[j] = __int_as_float(0x7f800000);  // +inf
        best_i[j] = 0xffffffffu;
    }
    float worst = __int_as_float(0x7f800000);
    for (int64_t t0 = 0; t0 < n; t0 += kKnnTile) {
        const int m = (int)(n - t0 < (int64_t)kKnnTile ? n - t0 : (int64_t)kKnnTile);
        __syncthreads();
        for (int e = threadIdx.x; e < m * d; e += kKnnThreads) tile[e] = X[t0 * d + e];
        __syncthreads();
        if (!active) continue;
        for (int r = 0; r < m; ++r) {
            const int64_t c = t0 + r;
            const float *y = tile + r * d;
            float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ch = 0; ch < D8; ++ch) {
                if (ch < full) {
#pragma unroll
                    for (int l = 0; l < 8; ++l) {
                        const float dl = __fsub_rn(xq[8 * ch + l], y[8 * ch + l]);
                        acc[l] = __fadd_rn(acc[l], __fmul_rn(dl, dl));
                    }
                }
            }
            float s = 0.0f;
#pragma unroll
            for (int l = 0; l < 8; ++l) s = __fadd_rn(s, acc[l]);
#pragma unroll
            for (int j = 0; j < 8 * D8; ++j) {
                if (j >= 8 * full && j < d) {
                    const float dl = __fsub_rn(xq[j], y[j]);
                    s = __fadd_rn(s, __fmul_rn(dl, dl));
                }
            }
            if (c == q || !(s < worst)) continue;
            int p = k - 1;
            while (p > 0 && best_d[p - 1] > s) {
                best_d[p] = best_d[p - 1];
                best_i[p] = best_i[p - 1];
                --p;
            }
            best_d[p] = s;
            best_i[p] = (uint32_t)c;
            worst = best_d[k - 1];
        }
    }
    if (!active) return;
    // square roots, then (distance, index) order
    for (int j = 0; j < k; ++j) best_d[j] = best_i[j] == 0xffffffffu ? best_d[j] : __fsqrt_rn(best_d[j]);
    for (int j = 1; j < k; ++j) {
        const float dj = best_d[j];
        const uint32_t ij = best_i[j];
        int p = j;
        while (p > 0 && (best_d[p - 1] > dj || (best_d[p - 1] == dj && best_i[p - 1] > ij))) {
            best_d[p] = best_d[p - 1];
            best_i[p] = best_i[p - 1];
            --p;
        }
        best_d[p] = dj;
        best_i[p] = ij;
    }
    for (int j = 0; j < k; ++j) {
        out_idx[q * k + j] = best_i[j];
        out_dist[q * k + j] = best_d[j];
    }
}

int launch_knn(const float *X, int64_t n, int d, int k, uint32_t *idx, float *dist, cudaStream_t st) {
    CREST_REQUIRE(d >= 1 && d <= kKnnMaxD, CREST_EINVAL, "knn supports 1 <= d <= %d (got %d)", kKnnMaxD, d);
    CREST_REQUIRE(k >= 1 && k <= kKnnMaxK, CREST_EINVAL, "knn supports 1 <= k <= %d (got %d)", kKnnMaxK, k);
    if (n == 0) return CREST_OK;
    const size_t smem = sizeof(float) * (size_t)kKnnTile * (size_t)d;
    const unsigned blocks = (unsigned)ceil_div(n, kKnnThreads);
    prof::Scope ps("knn_exact", st);
    const int d8 = (d + 7) / 8;
#define CREST_KNN_CASE(N)                                                                   \
    if (d8 <= N) {                                                                          \
        CREST_TRY(ensure_smem_attr((const void *)k_knn<N>, smem));                          \
        k_knn<N><<<blocks, kKnnThreads, smem, st>>>(X, n, d, k, idx, dist);                 \
        CREST_CUDA_TRY(cudaGetLastError());                                                 \
        return CREST_OK;                                                                    \
    }
    CREST_KNN_CASE(2)
    CREST_KNN_CASE(4)
    CREST_KNN_CASE(7)
    CREST_KNN_CASE(10)
    CREST_KNN_CASE(16)
#undef CREST_KNN_CASE
    return CREST_EINVAL;
}

}  // namespace crest
