// K5: FP64 centring + top-k symmetric eigensolve on the GPU
// (src/kernels.rs:311-348 uses faer's dense self_adjoint_eigen on the CPU).
//
//   cov = (G - c c^T / n) / (n - 1)    (FP64, from the upper triangle of G)
//   total = trace(cov)
//   top-k eigenpairs, descending, clamped at 0, largest |loading| positive.
//
// d <= 160: cyclic Jacobi on the whole matrix in one CTA (matrix in shared
// memory, round-robin parallel ordering).
// d > 160: Chebyshev-filtered subspace iteration (Zhou & Saad, 2007) on a
// block of p = k + 32 (rounded to 16) vectors: Rayleigh-Ritz with the same
// Jacobi kernel on the p x p projected matrix, a degree-m Chebyshev filter
// that damps the spectrum below the smallest Ritz value, and classical
// Gram-Schmidt with re-orthogonalisation.  Stops when every wanted residual
// ||C v - theta v|| is below tol * theta_1.
#include <math.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"
#include "prof.cuh"

namespace crest {
namespace {

constexpr int kJacobiMax = 160;

// ------------------------------------------------------------ centring
__global__ void k_centre(const double *__restrict__ G, const double *__restrict__ c, int64_t d, double n,
                         double *__restrict__ C) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d * d) return;
    const int64_t i = idx / d, j = idx % d;
    const int64_t a = i <= j ? i : j, b = i <= j ? j : i;
    C[idx] = __ddiv_rn(__dsub_rn(G[a * d + b], __ddiv_rn(__dmul_rn(c[a], c[b]), n)), __dsub_rn(n, 1.0));
}

// total = sum_i cov[i][i] in index order (src/kernels.rs:323)
__global__ void k_trace(const double *__restrict__ C, int64_t d, double *total) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int64_t i = 0; i < d; ++i) s = __dadd_rn(s, C[i * d + i]);
    *total = s;
}

// Gershgorin upper bound of the spectrum: max_i sum_j |C[i][j]|
__global__ void k_row_abs_max(const double *__restrict__ C, int64_t d, double *out) {
    __shared__ double red[32];
    double best = 0.0;
    for (int64_t i = blockIdx.x; i < d; i += gridDim.x) {
        double s = 0.0;
        for (int64_t j = threadIdx.x; j < d; j += blockDim.x) s += fabs(C[i * d + j]);
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (threadIdx.x == 0) best = fmax(best, v);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        unsigned long long *p = reinterpret_cast<unsigned long long *>(out);
        atomicMax(p, (unsigned long long)__double_as_longlong(best));  // non-negative doubles order as integers
    }
}

// ------------------------------------------------------------------ GEMM
// Column-major FP64 GEMM: O = alpha * op(A) B + beta * X + gamma * Y.
struct Gemm {
    int M, N, K;
    const double *A;
    int lda;
    int tA;
    const double *B;
    int ldb;
    double *O;
    int ldo;
    double alpha;
    const double *X;
    double beta;
    const double *Y;
    double gamma;
};

__global__ void __launch_bounds__(256) k_gemm(Gemm g) {
    __shared__ double As[16][64 + 1];
    __shared__ double Bs[16][64 + 1];
    const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < g.K; k0 += 16) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int idx = tid + 256 * r;
            int mm, kk;
            if (!g.tA) {
                mm = idx & 63;
                kk = idx >> 6;
            } else {
                kk = idx & 15;
                mm = idx >> 4;
            }
            const int m = m0 + mm, k = k0 + kk;
            double v = 0.0;
            if (m < g.M && k < g.K) v = g.tA ? g.A[k + (int64_t)m * g.lda] : g.A[m + (int64_t)k * g.lda];
            As[kk][mm] = v;
            const int kb = idx & 15, nn = idx >> 4;
            const int n = n0 + nn, kB = k0 + kb;
            Bs[kb][nn] = (n < g.N && kB < g.K) ? g.B[kB + (int64_t)n * g.ldb] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) a[p] = As[kk][tx + 16 * p];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = Bs[kk][ty + 16 * q];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int m = m0 + tx + 16 * p, n = n0 + ty + 16 * q;
            if (m >= g.M || n >= g.N) continue;
            const int64_t o = m + (int64_t)n * g.ldo;
            double v = g.alpha * acc[p][q];
            if (g.X) v += g.beta * g.X[o];
            if (g.Y) v += g.gamma * g.Y[o];
            g.O[o] = v;
        }
}

int gemm(const Gemm &g, cudaStream_t st) {
    prof::Scope ps("eig_gemm_fp64", st);
    dim3 grid((unsigned)ceil_div(g.M, 64), (unsigned)ceil_div(g.N, 64));
    k_gemm<<<grid, 256, 0, st>>>(g);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ---------------------------------------------------------------- Jacobi
// Cyclic Jacobi on a symmetric n_in x n_in column-major matrix (padded to an
// even n with a decoupled zero row/column).  Round-robin ordering: n/2
// disjoint pairs per round, n-1 rounds per sweep; each round applies the
// row rotations, then the column rotations (Rutishauser's formulas, the
// rotation P with P_pp = P_qq = c, P_pq = s, P_qp = -s zeroes A'_pq in
// P^T A P).  On exit: vals[i] = A_ii, V (n x n, col-major, global) the
// accumulated rotations.
__global__ void __launch_bounds__(1024) k_jacobi(const double *__restrict__ Ain, int n_in, int n, double *V,
                                                 double *vals, int max_sweeps, int *sweeps_out) {
    extern __shared__ double S[];
    const int ld = n + 1;
    __shared__ double cs_[kJacobiMax / 2], sn_[kJacobiMax / 2];
    __shared__ int pp_[kJacobiMax / 2], qq_[kJacobiMax / 2];
    __shared__ double red[64];
    __shared__ int done;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int w = tid; w < n * n; w += nt) {
        const int r = w % n, c = w / n;
        S[r + c * ld] = (r < n_in && c < n_in) ? Ain[r + (int64_t)c * n_in] : 0.0;
        V[r + (int64_t)c * n] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    const int half = n / 2;
    int sweep = 0;
    for (; sweep < max_sweeps; ++sweep) {
        // convergence: off-diagonal mass relative to the whole matrix
        double off = 0.0, tot = 0.0;
        for (int w = tid; w < n * n; w += nt) {
            const int r = w % n, c = w / n;
            const double v = S[r + c * ld];
            tot += v * v;
            if (r != c) off += v * v;
        }
        for (int o = 16; o; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((tid & 31) == 0) {
            red[tid >> 5] = off;
            red[32 + (tid >> 5)] = tot;
        }
        __syncthreads();
        if (tid == 0) {
            double so = 0.0, sa = 0.0;
            for (int i = 0; i < (nt >> 5); ++i) {
                so += red[i];
                sa += red[32 + i];
            }
            done = (so <= 1e-30 * sa) || so == 0.0;
        }
        __syncthreads();
        if (done) break;
        for (int r = 0; r < n - 1; ++r) {
            if (tid < half) {
                // positions: 0 fixed, others rotate around the circle
                const int i = tid;
                const int a = (i == 0) ? 0 : ((i - 1 + r) % (n - 1)) + 1;
                const int b = ((n - 1 - i - 1 + r) % (n - 1)) + 1;
                const int p = a < b ? a : b, q = a < b ? b : a;
                const double apq = S[p + q * ld];
                double c = 1.0, s = 0.0;
                if (apq != 0.0) {
                    const double app = S[p + p * ld], aqq = S[q + q * ld];
                    const double tau = (aqq - app) / (2.0 * apq);
                    const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                    c = 1.0 / sqrt(1.0 + t * t);
                    s = t * c;
                }
                cs_[i] = c;
                sn_[i] = s;
                pp_[i] = p;
                qq_[i] = q;
            }
            __syncthreads();
            // rows p, q  <- P^T A
            for (int w = tid; w < half * n; w += nt) {
                const int i = w % half, j = w / half;
                const int p = pp_[i], q = qq_[i];
                const double c = cs_[i], s = sn_[i];
                if (s == 0.0) continue;
                const double x = S[p + j * ld], y = S[q + j * ld];
                S[p + j * ld] = c * x - s * y;
                S[q + j * ld] = s * x + c * y;
            }
            __syncthreads();
            // columns p, q  <- A P ;  V <- V P
            for (int w = tid; w < half * n; w += nt) {
                const int i = w % half, j = w / half;
                const int p = pp_[i], q = qq_[i];
                const double c = cs_[i], s = sn_[i];
                if (s == 0.0) continue;
                const double x = S[j + p * ld], y = S[j + q * ld];
                S[j + p * ld] = c * x - s * y;
                S[j + q * ld] = s * x + c * y;
                const double vx = V[j + (int64_t)p * n], vy = V[j + (int64_t)q * n];
                V[j + (int64_t)p * n] = c * vx - s * vy;
                V[j + (int64_t)q * n] = s * vx + c * vy;
            }
            __syncthreads();
        }
    }
    for (int i = tid; i < n; i += nt) vals[i] = S[i + i * ld];
    if (tid == 0 && sweeps_out) *sweeps_out = sweep;
}

int jacobi(const double *A, int n_in, double *V, double *vals, int *sweeps, cudaStream_t st) {
    const int n = n_in + (n_in & 1);
    CREST_REQUIRE(n <= kJacobiMax, CREST_EINVAL, "Jacobi size %d exceeds %d", n, kJacobiMax);
    const size_t smem = sizeof(double) * (size_t)n * (size_t)(n + 1);
    CREST_CUDA_TRY(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    prof::Scope ps("eig_jacobi", st);
    k_jacobi<<<1, 1024, smem, st>>>(A, n_in, n, V, vals, 40, sweeps);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ------------------------------------------------- order + emit results
// perm = indices of the n_in leading Jacobi values sorted descending
// (ties: lower index first); one thread per candidate.
__global__ void k_rank(const double *vals, int n_in, int *perm, double *sorted) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_in) return;
    const double v = vals[i];
    int r = 0;
    for (int j = 0; j < n_in; ++j) {
        const double u = vals[j];
        if (u > v || (u == v && j < i)) ++r;
    }
    perm[r] = i;
    sorted[r] = v;
}

// Column j of out (d x k row-major) = sign * col perm[j] of Vb (d x ldv
// col-major); vals[j] = max(sorted[j], 0).  sign makes the first entry of
// largest magnitude positive (sklearn svd_flip rule, src/kernels.rs:334-345).
__global__ void k_emit(const double *__restrict__ Vb, int64_t d, int64_t ldv, const int *perm,
                       const double *sorted, int64_t k, double *out_vals, double *out_vecs) {
    __shared__ double bv[32];
    __shared__ int bi[32];
    const int64_t j = blockIdx.x;
    const double *col = Vb + (int64_t)perm[j] * ldv;
    double best = -1.0;
    int besti = 0x7fffffff;
    for (int64_t r = threadIdx.x; r < d; r += blockDim.x) {
        const double a = fabs(col[r]);
        if (a > best) {  // rows visited in increasing order per thread
            best = a;
            besti = (int)r;
        }
    }
    for (int o = 16; o; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, besti, o);
        if (ob > best || (ob == best && oi < besti)) {
            best = ob;
            besti = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        bv[threadIdx.x >> 5] = best;
        bi[threadIdx.x >> 5] = besti;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = -1.0;
        int ib = 0x7fffffff;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (bv[w] > b || (bv[w] == b && bi[w] < ib)) {
                b = bv[w];
                ib = bi[w];
            }
        bi[0] = ib;
        bv[0] = b;
        out_vals[j] = fmax(sorted[j], 0.0);
    }
    __syncthreads();
    const double sign = (bv[0] > 0.0 && col[bi[0]] < 0.0) ? -1.0 : 1.0;
    for (int64_t r = threadIdx.x; r < d; r += blockDim.x) out_vecs[r * k + j] = col[r] * sign;
}

// --------------------------------------------------------- block kernels
__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // SplitMix64 finaliser (Steele et al. 2014)
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__global__ void k_random_block(double *V, int64_t n, uint64_t seed) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) V[i] = (double)(mix64(seed ^ (uint64_t)i) >> 11) * 0x1.0p-52 - 1.0;
}

// Classical Gram-Schmidt with one re-orthogonalisation pass, one CTA,
// column-major d x p block.  A column whose norm collapses below 1e-10 of
// its starting norm is replaced by a deterministic random vector and
// processed again.
__global__ void __launch_bounds__(1024) k_cgs2(double *Q, int64_t d, int p, uint64_t seed, int *n_replaced) {
    extern __shared__ double sh[];  // r[p] + red[32]
    double *rcoef = sh;
    double *red = sh + p;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    int replaced = 0;
    for (int j = 0; j < p; ++j) {
        double *y = Q + (int64_t)j * d;
        for (int attempt = 0; attempt < 3; ++attempt) {
            // starting norm
            double s = 0.0;
            for (int64_t r = tid; r < d; r += nt) s += y[r] * y[r];
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) red[wid] = s;
            __syncthreads();
            double n0 = 0.0;
            for (int w = 0; w < nw; ++w) n0 += red[w];
            __syncthreads();
            for (int pass = 0; pass < 2; ++pass) {
                // r_i = q_i . y for i < j  (warp per i)
                for (int i = wid; i < j; i += nw) {
                    const double *qi = Q + (int64_t)i * d;
                    double t = 0.0;
                    for (int64_t r = lane; r < d; r += 32) t += qi[r] * y[r];
                    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                    if (lane == 0) rcoef[i] = t;
                }
                __syncthreads();
                for (int64_t r = tid; r < d; r += nt) {
                    double v = y[r];
                    for (int i = 0; i < j; ++i) v -= rcoef[i] * Q[(int64_t)i * d + r];
                    y[r] = v;
                }
                __syncthreads();
            }
            s = 0.0;
            for (int64_t r = tid; r < d; r += nt) s += y[r] * y[r];
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) red[wid] = s;
            __syncthreads();
            double n1 = 0.0;
            for (int w = 0; w < nw; ++w) n1 += red[w];
            __syncthreads();
            if (n1 > 1e-20 * n0 && n1 > 0.0) {
                const double inv = 1.0 / sqrt(n1);
                for (int64_t r = tid; r < d; r += nt) y[r] *= inv;
                __syncthreads();
                break;
            }
            // deficient: draw a fresh direction and retry
            ++replaced;
            for (int64_t r = tid; r < d; r += nt)
                y[r] = (double)(mix64(seed ^ ((uint64_t)(j * 7 + attempt + 1) << 40) ^ (uint64_t)r) >> 11) *
                           0x1.0p-52 -
                       1.0;
            __syncthreads();
        }
    }
    if (tid == 0 && n_replaced) *n_replaced = replaced;
}

// r_i = || W_i - theta_i V_i || for i < k; out = max_i r_i (one block per column)
__global__ void k_residual(const double *__restrict__ W, const double *__restrict__ V, const double *theta,
                           int64_t d, double *out) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    const double th = theta[i];
    double s = 0.0;
    for (int64_t r = threadIdx.x; r < d; r += blockDim.x) {
        const double e = W[(int64_t)i * d + r] - th * V[(int64_t)i * d + r];
        s += e * e;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicMax(reinterpret_cast<unsigned long long *>(out), (unsigned long long)__double_as_longlong(sqrt(t)));
    }
}

// Permute the Ritz basis: dst[:, j] = src[:, perm[j]] for j < p.
__global__ void k_permute_cols(const double *src, double *dst, int64_t d, const int *perm, int p) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d * p) return;
    const int64_t r = idx % d, j = idx / d;
    dst[idx] = src[(int64_t)perm[j] * d + r];
}

// Symmetrise a p x p col-major matrix in place: H = (H + H^T)/2.
__global__ void k_symmetrise(double *H, int p) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= p * p) return;
    const int r = idx % p, c = idx / p;
    if (r < c) {
        const double v = 0.5 * (H[r + c * p] + H[c + r * p]);
        H[r + c * p] = v;
        H[c + r * p] = v;
    }
}

struct EigWork {
    DevBuf C, V, W, Y0, Y1, H, Q, vals, sorted, perm, scal;
};

}  // namespace

int eig_topk(const double *G, const double *colsum, int64_t d, int64_t n, int64_t k, double *out_vals,
             double *out_vecs, double *out_total, EigStats *stats, cudaStream_t st) {
    CREST_REQUIRE(d >= 1 && n >= 2, CREST_ERUNTIME, "need at least 2 cells and 1 gene");
    CREST_REQUIRE(k >= 0 && k <= d, CREST_EINVAL, "k=%lld must be in [0, d=%lld]", (long long)k, (long long)d);
    static thread_local EigWork w;
    const double nf = (double)n;
    CREST_TRY(w.C.ensure(sizeof(double) * (size_t)(d * d)));
    double *C = w.C.as<double>();
    k_centre<<<(unsigned)ceil_div(d * d, 256), 256, 0, st>>>(G, colsum, d, nf, C);
    CREST_CUDA_TRY(cudaGetLastError());
    k_trace<<<1, 32, 0, st>>>(C, d, out_total);
    CREST_CUDA_TRY(cudaGetLastError());
    if (stats) *stats = EigStats{0, 1, 0.0};
    if (k == 0) return CREST_OK;

    CREST_TRY(w.perm.ensure(sizeof(int) * 512));
    CREST_TRY(w.sorted.ensure(sizeof(double) * 512));
    CREST_TRY(w.vals.ensure(sizeof(double) * 512));
    CREST_TRY(w.scal.ensure(sizeof(double) * 8));
    int *perm = w.perm.as<int>();
    double *sorted = w.sorted.as<double>();
    double *jvals = w.vals.as<double>();

    if (d <= kJacobiMax) {  // whole matrix
        const int nn = (int)(d + (d & 1));
        CREST_TRY(w.Q.ensure(sizeof(double) * (size_t)nn * nn));
        CREST_TRY(jacobi(C, (int)d, w.Q.as<double>(), jvals, w.perm.as<int>() + 256, st));
        k_rank<<<(unsigned)ceil_div(d, 128), 128, 0, st>>>(jvals, (int)d, perm, sorted);
        CREST_CUDA_TRY(cudaGetLastError());
        k_emit<<<(unsigned)k, 256, 0, st>>>(w.Q.as<double>(), d, nn, perm, sorted, k, out_vals, out_vecs);
        CREST_CUDA_TRY(cudaGetLastError());
        if (stats) {
            int sweeps = 0;
            CREST_CUDA_TRY(cudaMemcpyAsync(&sweeps, w.perm.as<int>() + 256, sizeof(int), cudaMemcpyDeviceToHost, st));
            CREST_CUDA_TRY(cudaStreamSynchronize(st));
            stats->iters = sweeps;
        }
        return CREST_OK;
    }

    int p = (int)round_up(k + 32, 16);
    if (p > kJacobiMax) p = kJacobiMax;
    if (p > d) p = (int)d;
    CREST_REQUIRE(k <= p - 8, CREST_EINVAL, "n_comps=%lld too large for the block eigensolver (max %d)",
                  (long long)k, kJacobiMax - 8);
    const size_t blk = sizeof(double) * (size_t)d * (size_t)p;
    CREST_TRY(w.V.ensure(blk));
    CREST_TRY(w.W.ensure(blk));
    CREST_TRY(w.Y0.ensure(blk));
    CREST_TRY(w.Y1.ensure(blk));
    CREST_TRY(w.H.ensure(sizeof(double) * (size_t)p * p));
    CREST_TRY(w.Q.ensure(sizeof(double) * (size_t)p * p));
    double *V = w.V.as<double>(), *W = w.W.as<double>(), *Y0 = w.Y0.as<double>(), *Y1 = w.Y1.as<double>();
    double *H = w.H.as<double>(), *Q = w.Q.as<double>();
    double *scal = w.scal.as<double>();  // [0] gershgorin, [1] residual
    const int D = (int)d;
    const size_t cgs_smem = sizeof(double) * (size_t)(p + 32);

    // spectrum bound
    CREST_CUDA_TRY(cudaMemsetAsync(scal, 0, sizeof(double) * 2, st));
    k_row_abs_max<<<256, 256, 0, st>>>(C, d, scal);
    CREST_CUDA_TRY(cudaGetLastError());
    double bound = 0.0;
    CREST_CUDA_TRY(cudaMemcpyAsync(&bound, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    // start block
    k_random_block<<<(unsigned)ceil_div(d * p, 256), 256, 0, st>>>(V, d * p, 0x243f6a8885a308d3ull);
    CREST_CUDA_TRY(cudaGetLastError());
    k_cgs2<<<1, 1024, cgs_smem, st>>>(V, d, p, 0x13198a2e03707344ull, nullptr);
    CREST_CUDA_TRY(cudaGetLastError());
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    if (!(bound > 0.0)) {
        // zero covariance: every eigenvalue is 0; any orthonormal basis will do
        std::vector<int> hp(k);
        std::vector<double> hz(k, 0.0);
        for (int64_t i = 0; i < k; ++i) hp[i] = (int)i;
        CREST_CUDA_TRY(cudaMemcpyAsync(perm, hp.data(), sizeof(int) * k, cudaMemcpyHostToDevice, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(sorted, hz.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
        k_emit<<<(unsigned)k, 256, 0, st>>>(V, d, d, perm, sorted, k, out_vals, out_vecs);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_CUDA_TRY(cudaStreamSynchronize(st));
        return CREST_OK;
    }

    const double tol = 1e-11;
    const int max_outer = 80, degree = 12;
    std::vector<double> theta(p);
    int it = 0;
    double res = INFINITY;
    bool converged = false;
    for (; it < max_outer; ++it) {
        // Rayleigh-Ritz: W = C V, H = V^T W, H = Q diag(theta) Q^T
        CREST_TRY(gemm(Gemm{D, p, D, C, D, 0, V, D, W, D, 1.0, nullptr, 0.0, nullptr, 0.0}, st));
        CREST_TRY(gemm(Gemm{p, p, D, V, D, 1, W, D, H, p, 1.0, nullptr, 0.0, nullptr, 0.0}, st));
        k_symmetrise<<<(unsigned)ceil_div(p * p, 256), 256, 0, st>>>(H, p);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_TRY(jacobi(H, p, Q, jvals, nullptr, st));
        k_rank<<<(unsigned)ceil_div(p, 128), 128, 0, st>>>(jvals, p, perm, sorted);
        CREST_CUDA_TRY(cudaGetLastError());
        // V <- V Q_sorted, W <- W Q_sorted  (Q permuted into Y0 first)
        k_permute_cols<<<(unsigned)ceil_div(p * p, 256), 256, 0, st>>>(Q, H, p, perm, p);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_TRY(gemm(Gemm{D, p, p, V, D, 0, H, p, Y0, D, 1.0, nullptr, 0.0, nullptr, 0.0}, st));
        CREST_TRY(gemm(Gemm{D, p, p, W, D, 0, H, p, Y1, D, 1.0, nullptr, 0.0, nullptr, 0.0}, st));
        std::swap(V, Y0);
        std::swap(W, Y1);
        // residuals of the wanted pairs
        CREST_CUDA_TRY(cudaMemsetAsync(scal + 1, 0, sizeof(double), st));
        k_residual<<<(unsigned)k, 256, 0, st>>>(W, V, sorted, d, scal + 1);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_CUDA_TRY(cudaMemcpyAsync(theta.data(), sorted, sizeof(double) * p, cudaMemcpyDeviceToHost, st));
        double rmax = 0.0;
        CREST_CUDA_TRY(cudaMemcpyAsync(&rmax, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaStreamSynchronize(st));
        const double scale_ref = fmax(fabs(theta[0]), 1e-300);
        res = rmax / scale_ref;
        if (res <= tol) {
            converged = true;
            break;
        }
        if (it + 1 >= max_outer) break;
        // Chebyshev filter damping [lo, a], a = smallest Ritz value, reference point theta_0
        const double a = theta[p - 1], lo = -1e-12 * bound;
        if (!(a > lo) || !(theta[0] > a)) {
            // no usable gap estimate: plain subspace iteration step
            std::swap(V, W);
        } else {
            const double e = 0.5 * (a + lo), c = 0.5 * (a - lo);
            const double sigma1 = c / (theta[0] - e);
            double sigma = sigma1;
            // Y0 = V (previous), Y1 = sigma1/c (C V - e V) = sigma1/c (W - e V)
            // W already holds C V for the current V
            {
                // Y1 = (sigma1/c) * W + (-sigma1*e/c) * V
                CREST_TRY(gemm(Gemm{D, p, 0, C, D, 0, V, D, Y1, D, 0.0, W, sigma1 / c, V, -sigma1 * e / c}, st));
            }
            double *Yprev = V, *Ycur = Y1, *Ynext = Y0;
            for (int j = 2; j <= degree; ++j) {
                const double sigma_next = 1.0 / (2.0 / sigma1 - sigma);
                // Ynext = (2 sigma_next / c) (C Ycur - e Ycur) - sigma sigma_next Yprev
                CREST_TRY(gemm(Gemm{D, p, D, C, D, 0, Ycur, D, Ynext, D, 2.0 * sigma_next / c, Ycur,
                                    -2.0 * sigma_next * e / c, Yprev, -sigma * sigma_next},
                               st));
                sigma = sigma_next;
                double *t = Yprev;
                Yprev = Ycur;
                Ycur = Ynext;
                Ynext = t;
            }
            // make V the filtered block (V, Y0, Y1 are all free except Ycur)
            if (Ycur != V) {
                CREST_CUDA_TRY(cudaMemcpyAsync(V, Ycur, blk, cudaMemcpyDeviceToDevice, st));
            }
        }
        {
            prof::Scope ps("eig_cgs2", st);
            k_cgs2<<<1, 1024, cgs_smem, st>>>(V, d, p, 0x13198a2e03707344ull + (uint64_t)it, nullptr);
        }
        CREST_CUDA_TRY(cudaGetLastError());
    }
    if (stats) *stats = EigStats{it + 1, converged ? 1 : 0, res};
    // sorted Ritz pairs are already in order: identity permutation
    std::vector<int> ident(k);
    for (int64_t i = 0; i < k; ++i) ident[i] = (int)i;
    CREST_CUDA_TRY(cudaMemcpyAsync(perm, ident.data(), sizeof(int) * k, cudaMemcpyHostToDevice, st));
    k_emit<<<(unsigned)k, 256, 0, st>>>(V, d, d, perm, sorted, k, out_vals, out_vecs);
    CREST_CUDA_TRY(cudaGetLastError());
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    return CREST_OK;
}

}  // namespace crest
