// K5: FP64 centring + top-k symmetric eigensolve on the GPU
// (src/kernels.rs:311-348 uses faer's dense self_adjoint_eigen on the CPU).
//
//   cov = (G - c c^T / n) / (n - 1)    (FP64, from the upper triangle of G)
//   total = trace(cov)
//   top-k eigenpairs, descending, clamped at 0, largest |loading| positive.
//
// d <= 160: cyclic Jacobi on the whole matrix in one CTA (matrix in shared
// memory, round-robin parallel ordering).
//
// d > 160: Chebyshev-filtered subspace iteration (Zhou & Saad 2007) with
// locking, on a block of p = k + 14 (rounded up to 16) vectors:
//  * a short Lanczos run (full re-orthogonalisation) brackets the spectrum;
//    the filter damps [lambda_min, a] with a = the smallest active Ritz
//    value, so eigenvalues far from zero (scaled single-cell data: a dense
//    bulk near 1) still separate quickly;
//  * converged leading Ritz pairs are locked; the filter then acts on the
//    remaining columns only, keeping the dynamic range among active columns
//    small (one dominant component no longer swamps the bulk edge);
//  * the filter degree follows the estimated gap: enough growth per outer
//    step for the weakest wanted value, bounded so the block stays well
//    conditioned for Cholesky QR;
//  * orthonormalisation is shifted Cholesky QR (Fukaya et al. 2020) built
//    from split-K FP64 GEMMs (k_gemm, this file; no library GEMM), Rayleigh-
//    Ritz uses the same Jacobi kernel on the p x p projected matrix.
// Stops when every wanted residual ||C v - theta v|| <= tol * theta_1.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "kernels.cuh"
#include "prof.cuh"

namespace crest {
namespace {

constexpr int kJacobiMax = 160;
constexpr int kJacobiSmemV = 112;  // V also kept in shared memory up to this size
constexpr int kLanczos = 32;  // steps of the spectrum-bounds run

// ------------------------------------------------------------ centring
__global__ void k_centre(const double *__restrict__ G, const double *__restrict__ c, int64_t d, double n,
                         double *__restrict__ C) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d * d) return;
    const int64_t i = idx / d, j = idx % d;
    const int64_t a = i <= j ? i : j, b = i <= j ? j : i;
    C[idx] = __ddiv_rn(__dsub_rn(G[a * d + b], __ddiv_rn(__dmul_rn(c[a], c[b]), n)), __dsub_rn(n, 1.0));
}

// total = sum_i cov[i][i] in index order (src/kernels.rs:323): the diagonal
// is gathered 1024 entries at a time into shared memory by the whole block,
// then added up in order by one thread.
__global__ void __launch_bounds__(1024) k_trace(const double *__restrict__ C, int64_t d, double *total) {
    __shared__ double diag[1024];
    double s = 0.0;
    for (int64_t i0 = 0; i0 < d; i0 += 1024) {
        const int64_t i = i0 + threadIdx.x;
        if (i < d) diag[threadIdx.x] = C[i * d + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            const int64_t n = d - i0 < 1024 ? d - i0 : 1024;
            for (int64_t j = 0; j < n; ++j) s = __dadd_rn(s, diag[j]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = s;
}

// ------------------------------------------------------------------ GEMM
// Column-major FP64 GEMM: O = alpha * op(A) B + beta * X + gamma * Y, with an
// optional split of K over gridDim.z (partials to ws, then k_gemm_reduce).
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
    int tB = 0;  // 1: B is given transposed (element (k, n) at B[n + k ldb])
};

// 128 x 64 output tile per CTA (128 threads, 8 x 8 outputs each: rows
// 8 tr .. 8 tr + 7, columns 8 tc .. 8 tc + 7), K in steps of 8 staged
// through double-buffered shared memory with the next step's loads in
// registers.  gridDim.z splits K: each slice writes its partial product to
// ws (summed in slice order by k_gemm_reduce, so results do not depend on
// scheduling); without a split the epilogue is applied here.
constexpr int kGM = 128, kGN = 64, kGK = 8;

__global__ void __launch_bounds__(128) k_gemm(Gemm g, int kchunk, double *ws) {
    __shared__ __align__(16) double As[2][kGK][kGM];
    __shared__ __align__(16) double Bs[2][kGK][kGN];
    const int m0 = blockIdx.x * kGM, n0 = blockIdx.y * kGN;
    const int kb = blockIdx.z * kchunk, ke = min(g.K, kb + kchunk);
    const int tid = threadIdx.x, tr = tid >> 3, tc = tid & 7;
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    double ra[8], rb[4];
    // element r of this thread's share: A (m, k) and B (k, n) of the K step at k0
    auto a_mk = [&](int r, int &mm, int &kk) {
        const int e = tid + 128 * r;
        if (!g.tA) {
            mm = e & (kGM - 1);
            kk = e >> 7;
        } else {
            kk = e & (kGK - 1);
            mm = e >> 3;
        }
    };
    auto b_kn = [&](int r, int &kk, int &nn) {
        const int e = tid + 128 * r;
        if (!g.tB) {
            kk = e & (kGK - 1);
            nn = e >> 3;
        } else {
            nn = e & (kGN - 1);
            kk = e >> 6;
        }
    };
    auto gload = [&](int k0) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            int mm, kk;
            a_mk(r, mm, kk);
            const int m = m0 + mm, k = k0 + kk;
            ra[r] = (m < g.M && k < ke) ? (g.tA ? g.A[k + (int64_t)m * g.lda] : g.A[m + (int64_t)k * g.lda]) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            int kk, nn;
            b_kn(r, kk, nn);
            const int n = n0 + nn, k = k0 + kk;
            rb[r] = (n < g.N && k < ke) ? (g.tB ? g.B[n + (int64_t)k * g.ldb] : g.B[k + (int64_t)n * g.ldb]) : 0.0;
        }
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            int mm, kk;
            a_mk(r, mm, kk);
            As[buf][kk][mm] = ra[r];
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            int kk, nn;
            b_kn(r, kk, nn);
            Bs[buf][kk][nn] = rb[r];
        }
    };
    int buf = 0;
    if (kb < ke) {
        gload(kb);
        sstore(0);
    }
    __syncthreads();
    for (int k0 = kb; k0 < ke; k0 += kGK) {
        const bool more = k0 + kGK < ke;
        if (more) gload(k0 + kGK);
#pragma unroll
        for (int kk = 0; kk < kGK; ++kk) {
            double a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; i += 2) {
                const double2 va = *reinterpret_cast<const double2 *>(&As[buf][kk][tr * 8 + i]);
                const double2 vb = *reinterpret_cast<const double2 *>(&Bs[buf][kk][tc * 8 + i]);
                a[i] = va.x;
                a[i + 1] = va.y;
                b[i] = vb.x;
                b[i + 1] = vb.y;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (more) sstore(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int m = m0 + tr * 8 + i, n = n0 + tc * 8 + j;
            if (m >= g.M || n >= g.N) continue;
            if (ws) {
                ws[((int64_t)blockIdx.z * g.N + n) * g.M + m] = acc[i][j];
                continue;
            }
            const int64_t o = m + (int64_t)n * g.ldo;
            double v = g.alpha * acc[i][j];
            if (g.X) v += g.beta * g.X[o];
            if (g.Y) v += g.gamma * g.Y[o];
            g.O[o] = v;
        }
}

__global__ void k_gemm_reduce(Gemm g, int ksplit, const double *__restrict__ ws) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)g.M * g.N) return;
    const int m = (int)(idx % g.M), n = (int)(idx / g.M);
    double s = 0.0;
    for (int z = 0; z < ksplit; ++z) s += ws[((int64_t)z * g.N + n) * g.M + m];
    const int64_t o = m + (int64_t)n * g.ldo;
    double v = g.alpha * s;
    if (g.X) v += g.beta * g.X[o];
    if (g.Y) v += g.gamma * g.Y[o];
    g.O[o] = v;
}

// Tall-skinny products O = alpha op(A) B + beta X + gamma Y with B (K x N,
// N <= 64) column-major and op(A) = A (M x K) or A^T (A given K x M), all
// column-major (the filter and Rayleigh-Ritz products C V and V^T W of the
// subspace iteration): FP64 tensor-core MMAs (m8n8k4).
//
// CTA tile 64 x BN (BN = 16 NF), eight warps as 4 (M) x 2 (N), each warp
// 16 x 8 NF outputs = 2 x NF fragments of 8 x 8.  K in steps of 16 through an
// ST-stage cp.async ring (more stages for narrow B, where the product streams
// A at little arithmetic per byte); shared-memory rows are padded so that
// each half-warp's 8-byte fragment loads fall in 16 distinct 8-byte slots
// (row strides of 68 and 20 doubles are 4 mod 16; op(A) = A^T is staged
// [m][k] like B).  K is split over gridDim.z = the cluster's z extent: every
// slice leaves its partial tile in its own shared memory, and after a cluster
// barrier slice r sums rows [64 r / ks, 64 (r + 1) / ks) of all slices'
// partials in slice order (distributed shared memory), so results do not
// depend on scheduling.
namespace dm {
constexpr int kBK = 16;
constexpr int kBS = kBK + 4;  // [n][k] (and A^T's [m][k]) staging: k stride 20
constexpr int kMaxSplit = 16;

// Tile shapes: WM x WN warps, each FM x FN fragments of 8 x 8; 4 x 2 warps of
// 2 x NF fragments (tile 64 x 16 NF) with six, four and three stages for
// NF = 1, 2, 4.  (Two by two warps of 4 x 4 fragments at 128 threads, three
// CTAs per SM, measured 12 % slower on the 2000 x 2000 x 63 products.)
template <int KIND>
struct Cfg {
    static constexpr int WM = 4, WN = 2;
    static constexpr int FM = 2, FN = KIND == 0 ? 1 : KIND == 1 ? 2 : 4;
    static constexpr int BM = WM * FM * 8, BN = WN * FN * 8;
    static constexpr int THREADS = 32 * WM * WN;
    static constexpr int ST = KIND == 0 ? 6 : KIND == 1 ? 4 : 3;
    static constexpr int AS = BM + 4;  // A staging [k][m]: m stride, 4 mod 16
    static constexpr int AStage = BM * kBS > kBK * AS ? BM * kBS : kBK * AS;
    static constexpr int BStage = BN * kBS;
    static constexpr size_t smem = sizeof(double) * (size_t)ST * (AStage + BStage);
    static_assert((size_t)ST * (AStage + BStage) >= (size_t)BM * BN, "partial tile must fit the ring");
    static_assert(AS % 16 == 4 && kBS % 16 == 4, "fragment loads must not conflict");
};

__device__ __forceinline__ void cp16(void *smem, const void *gmem, bool ok) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = ok ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// generic address of the same shared-memory location in cluster CTA `rank`
__device__ __forceinline__ const double *cluster_ptr(const double *p, unsigned rank) {
    uint64_t r;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(reinterpret_cast<uint64_t>(p)), "r"(rank));
    return reinterpret_cast<const double *>(r);
}

template <int KIND, bool TA>
__global__ void __launch_bounds__(Cfg<KIND>::THREADS, 2) k_gemm_dmma(Gemm g, int kchunk) {
    using C = Cfg<KIND>;
    constexpr int BM = C::BM, BN = C::BN, ST = C::ST, FM = C::FM, FN = C::FN, T = C::THREADS;
    extern __shared__ __align__(16) double sm[];
    double *As = sm, *Bs = sm + ST * C::AStage;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp % C::WM, wn = warp / C::WM;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * kchunk, ke = min(g.K, kb + kchunk);
    const int ntiles = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;

    auto load = [&](int t, int stage) {
        const int k0 = kb + t * kBK;
        double *as = As + stage * C::AStage, *bs = Bs + stage * C::BStage;
        // A: 16 k x BM m in chunks of two m ([k][m]), or of two k for A^T ([m][k])
        for (int c = tid; c < 8 * BM; c += T) {
            if (!TA) {
                const int kk = c / (BM / 2), mm = (c % (BM / 2)) * 2;
                const int m = m0 + mm, k = k0 + kk;
                const bool ok = m < g.M && k < ke;
                cp16(as + kk * C::AS + mm, ok ? g.A + m + (int64_t)k * g.lda : g.A, ok);
            } else {
                const int mm = c >> 3, kk = (c & 7) * 2;
                const int m = m0 + mm, k = k0 + kk;
                const bool ok = m < g.M && k < ke;
                cp16(as + mm * kBS + kk, ok ? g.A + k + (int64_t)m * g.lda : g.A, ok);
            }
        }
        // B: BN n x 16 k in chunks of two k
        for (int c = tid; c < 8 * BN; c += T) {
            const int nn = c >> 3, kk = (c & 7) * 2;
            const int n = n0 + nn, k = k0 + kk;
            const bool ok = n < g.N && k < ke;
            cp16(bs + nn * kBS + kk, ok ? g.B + k + (int64_t)n * g.ldb : g.B, ok);
        }
    };

    double acc[FM][FN][2];
#pragma unroll
    for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < ST - 1; ++s) {
        if (s < ntiles) load(s, s);
        cp_commit();
    }
    const int ar = lane >> 2, ac = lane & 3;  // fragment row / column of this lane
    for (int t = 0; t < ntiles; ++t) {
        cp_wait<ST - 2>();
        __syncthreads();
        if (t + ST - 1 < ntiles) load(t + ST - 1, (t + ST - 1) % ST);
        cp_commit();
        const double *as =
            As + (t % ST) * C::AStage + (TA ? (wm * FM * 8 + ar) * kBS + ac : wm * FM * 8 + ar + ac * C::AS);
        const double *bs = Bs + (t % ST) * C::BStage + (wn * FN * 8 + ar) * kBS + ac;
#pragma unroll
        for (int k4 = 0; k4 < kBK; k4 += 4) {
            double a[FM], b[FN];
#pragma unroll
            for (int i = 0; i < FM; ++i) a[i] = TA ? as[i * 8 * kBS + k4] : as[k4 * C::AS + i * 8];
#pragma unroll
            for (int j = 0; j < FN; ++j) b[j] = bs[j * 8 * kBS + k4];
#pragma unroll
            for (int i = 0; i < FM; ++i)
#pragma unroll
                for (int j = 0; j < FN; ++j) dmma(acc[i][j], a[i], b[j]);
        }
    }
    cp_wait<0>();

    auto out = [&](int m, int n, double v) {
        if (m >= g.M || n >= g.N) return;
        const int64_t o = m + (int64_t)n * g.ldo;
        double r = g.alpha * v;
        if (g.X) r += g.beta * g.X[o];
        if (g.Y) r += g.gamma * g.Y[o];
        g.O[o] = r;
    };
    const int ks = (int)gridDim.z;
    if (ks == 1) {
#pragma unroll
        for (int i = 0; i < FM; ++i)
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    out(m0 + wm * FM * 8 + i * 8 + ar, n0 + wn * FN * 8 + j * 8 + ac * 2 + h, acc[i][j][h]);
        return;
    }
    // partial tile [m][n] in this CTA's ring, then the cluster-wide row split
    __syncthreads();
    double *part = sm;
#pragma unroll
    for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h)
                part[(wm * FM * 8 + i * 8 + ar) * BN + wn * FN * 8 + j * 8 + ac * 2 + h] = acc[i][j][h];
    cluster_sync_all();
    const int r = (int)blockIdx.z, rows = (BM + ks - 1) / ks;
    const int e0 = min(BM, r * rows) * BN, e1 = min(BM, (r + 1) * rows) * BN;
    const double *src[kMaxSplit];
#pragma unroll
    for (int z = 0; z < kMaxSplit; ++z) src[z] = z < ks ? cluster_ptr(part, (unsigned)z) : part;
    for (int e = e0 + tid; e < e1; e += T) {
        double v = 0.0;
#pragma unroll
        for (int z = 0; z < kMaxSplit; ++z)
            if (z < ks) v += src[z][e];
        out(m0 + e / BN, n0 + e % BN, v);
    }
    cluster_sync_all();  // no CTA leaves while another reads its partial
}
}  // namespace dm

struct GemmWs {
    DevBuf ws;
};

static bool dmma_enabled() {  // CREST_EIG_DMMA=0: CUDA-core kernel for every product
    static const bool on = [] {
        const char *e = getenv("CREST_EIG_DMMA");
        return !(e && e[0] == '0');
    }();
    return on;
}

static bool dmma_fits(const Gemm &g) {
    auto al = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
    return !g.tB && g.N >= 1 && g.N <= 64 && g.M >= 1 && g.K >= dm::kBK && !(g.K & 1) && !(g.lda & 1) &&
           !(g.ldb & 1) && (g.tA || !(g.M & 1)) && al(g.A) && al(g.B);
}

template <int KIND, bool TA>
static int launch_dmma(const Gemm &g, cudaStream_t st) {
    using C = dm::Cfg<KIND>;
    const void *fn = (const void *)dm::k_gemm_dmma<KIND, TA>;
    CREST_TRY(ensure_smem_attr(fn, C::smem));
    static bool nonportable = [fn] {
        const bool ok = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
        (void)cudaGetLastError();
        return ok;
    }();
    const int mt = (int)ceil_div(g.M, C::BM), nt = (int)ceil_div(g.N, C::BN);
    // K split = the cluster's z extent: about two CTAs per SM, slices of at
    // least 64, a power of two up to 16 (8 without non-portable clusters)
    const int want = std::max(1, std::min((2 * device_sms()) / (mt * nt), g.K / (4 * dm::kBK)));
    int ks = 1;
    while (ks * 2 <= want && ks * 2 <= (nonportable ? dm::kMaxSplit : 8)) ks *= 2;
    auto launch = [&](int z) {
        const int kc = z > 1 ? (int)round_up(ceil_div(g.K, z), dm::kBK) : g.K;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(mt, nt, z);
        cfg.blockDim = dim3(C::THREADS);
        cfg.dynamicSmemBytes = C::smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 1;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = z;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, dm::k_gemm_dmma<KIND, TA>, g, kc);
    };
    cudaError_t e = launch(ks);
    if (e != cudaSuccess && ks > 1) {  // a cluster shape that cannot be placed: a power of two up to 8
        (void)cudaGetLastError();
        int z = 1;
        while (z * 2 <= std::min(ks, 8)) z *= 2;
        e = launch(z);
    }
    CREST_CUDA_TRY(e);
    return CREST_OK;
}

static int gemm_dmma(const Gemm &g, GemmWs &, cudaStream_t st) {
    if (g.N <= 16) return g.tA ? launch_dmma<0, true>(g, st) : launch_dmma<0, false>(g, st);
    if (g.N <= 32) return g.tA ? launch_dmma<1, true>(g, st) : launch_dmma<1, false>(g, st);
    return g.tA ? launch_dmma<2, true>(g, st) : launch_dmma<2, false>(g, st);
}

int gemm(const Gemm &g, GemmWs &w, cudaStream_t st) {
    prof::Scope ps("eig_gemm_fp64", st);
    if (dmma_fits(g) && dmma_enabled()) return gemm_dmma(g, w, st);
    const int mt = (int)ceil_div(g.M, kGM), nt = (int)ceil_div(g.N, kGN);
    int ksplit = 1;
    if (g.K > 0) {  // about one CTA per SM, slices of at least 64
        const int want = (int)ceil_div(device_sms(), mt * nt);
        ksplit = std::max(1, std::min(want, (int)ceil_div(g.K, 64)));
    }
    if (ksplit == 1) {
        k_gemm<<<dim3(mt, nt, 1), 128, 0, st>>>(g, std::max(g.K, 1), nullptr);
        CREST_CUDA_TRY(cudaGetLastError());
        return CREST_OK;
    }
    const int kchunk = (int)round_up(ceil_div(g.K, ksplit), kGK);
    ksplit = (int)ceil_div(g.K, kchunk);
    CREST_TRY(w.ws.ensure(sizeof(double) * (size_t)ksplit * g.M * g.N));
    k_gemm<<<dim3(mt, nt, ksplit), 128, 0, st>>>(g, kchunk, w.ws.as<double>());
    CREST_CUDA_TRY(cudaGetLastError());
    k_gemm_reduce<<<(unsigned)ceil_div((int64_t)g.M * g.N, 256), 256, 0, st>>>(g, ksplit, w.ws.as<double>());
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// ---------------------------------------------------------------- Jacobi
// Cyclic Jacobi on a symmetric n_in x n_in column-major matrix (padded to an
// even n with a decoupled zero row/column).  Round-robin ordering: n/2
// disjoint pairs per round, n-1 rounds per sweep.  The rotation of pair
// (p, q) is P with P_pp = P_qq = c, P_pq = s, P_qp = -s (Rutishauser's
// formulas), chosen so that (P^T A P)_pq = 0.  The pairs of a round
// partition the indices, so A' = J^T A J splits into independent 2x2 blocks
// (rows of pair i, columns of pair j): each thread updates whole blocks,
// R_i^T M R_j, and one round costs two barriers.  A rotation is skipped when
// |A_pq| <= n u sqrt(|A_pp A_qq|), u = 2^-52 (or below 1e-18 ||A||_F): below
// that level a rotation only moves rounding noise around.  The solver stops
// after a sweep without rotations.  The rotations accumulate in V (shared
// memory when n <= 112, else the n x n global scratch Vwork).  The padding
// row/column never couples, so the leading n_in x n_in block of V holds the
// eigenvectors.  On exit: vals[i] = A_ii, Vout (n_in x n_in, col-major).
template <bool V_SMEM>
__global__ void __launch_bounds__(512) k_jacobi(const double *__restrict__ Ain, int n_in, int n, double *Vwork,
                                                 double *Vout, double *vals, int max_sweeps, int *sweeps_out) {
    extern __shared__ double S[];
    const int ld = n + 1;
    double *V = V_SMEM ? S + (size_t)n * ld : Vwork;
    __shared__ double cs_[kJacobiMax / 2], sn_[kJacobiMax / 2];
    __shared__ int pp_[kJacobiMax / 2], qq_[kJacobiMax / 2];
    __shared__ double red[32];
    __shared__ int rotated;
    __shared__ double floor_abs;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int w = tid; w < n * n; w += nt) {
        const int r = w % n, c = w / n;
        S[r + c * ld] = (r < n_in && c < n_in) ? Ain[r + (int64_t)c * n_in] : 0.0;
        V[r + (int64_t)c * n] = (r == c) ? 1.0 : 0.0;
    }
    // ||A||_F (invariant under the rotations) for the absolute skip floor
    double ss = 0.0;
    for (int w = tid; w < n * n; w += nt) {
        const double v = S[(w % n) + (w / n) * ld];
        ss += v * v;
    }
    for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((tid & 31) == 0) red[tid >> 5] = ss;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int i = 0; i < (nt >> 5); ++i) t += red[i];
        floor_abs = 1e-18 * sqrt(t);
        rotated = 0;
    }
    __syncthreads();
    const int half = n / 2;
    const double eps = (double)n * 0x1.0p-52, eps2 = eps * eps;
    int sweep = 0;
    for (; sweep < max_sweeps; ++sweep) {
        for (int r = 0; r < n - 1; ++r) {
            for (int i = tid; i < half; i += nt) {
                const int a = (i == 0) ? 0 : ((i - 1 + r) % (n - 1)) + 1;
                const int b = ((n - 2 - i + r) % (n - 1)) + 1;
                const int p = a < b ? a : b, q = a < b ? b : a;
                const double apq = S[p + q * ld], app = S[p + p * ld], aqq = S[q + q * ld];
                double c = 1.0, s = 0.0;
                if (fabs(apq) > floor_abs && apq * apq > eps2 * fabs(app * aqq)) {
                    // t = sign(tau) / (|tau| + sqrt(1 + tau^2)), tau = (aqq - app) / (2 apq),
                    // written with one square root and one division
                    const double dd = aqq - app, two = 2.0 * apq;
                    const double r = sqrt(fma(dd, dd, two * two));
                    const double t = (dd >= 0.0 ? two : -two) / (fabs(dd) + r);
                    c = rsqrt(fma(t, t, 1.0));
                    s = t * c;
                    rotated = 1;
                }
                cs_[i] = c;
                sn_[i] = s;
                pp_[i] = p;
                qq_[i] = q;
            }
            __syncthreads();
            // Warp w owns the row pairs bi = w, w + nw, ...; lane l owns the
            // column pairs bj = l, l + 32, ... and the rows j = l, l + 32, ...
            // of V, so every rotation parameter is read once into registers.
            {
                const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
                double cj[3], sj[3];
                int uj[3], vj[3];
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    const int bj = lane + 32 * t;
                    const bool in = bj < half;
                    cj[t] = in ? cs_[bj] : 1.0;
                    sj[t] = in ? sn_[bj] : 0.0;
                    uj[t] = in ? pp_[bj] : 0;
                    vj[t] = in ? qq_[bj] : 0;
                }
                for (int bi = wid; bi < half; bi += nw) {
                    const double ci = cs_[bi], si = sn_[bi];
                    const int p = pp_[bi], q = qq_[bi];
#pragma unroll
                    for (int t = 0; t < 3; ++t) {
                        const int bj = lane + 32 * t;
                        if (bj >= half || (si == 0.0 && sj[t] == 0.0)) continue;
                        const int u = uj[t], v = vj[t];
                        const double m00 = S[p + u * ld], m01 = S[p + v * ld];
                        const double m10 = S[q + u * ld], m11 = S[q + v * ld];
                        // rows: [c -s; s c] M
                        const double r00 = ci * m00 - si * m10, r01 = ci * m01 - si * m11;
                        const double r10 = si * m00 + ci * m10, r11 = si * m01 + ci * m11;
                        // columns: R [c s; -s c]
                        double n00 = cj[t] * r00 - sj[t] * r01, n01 = sj[t] * r00 + cj[t] * r01;
                        double n10 = cj[t] * r10 - sj[t] * r11, n11 = sj[t] * r10 + cj[t] * r11;
                        if (bi == bj) {  // the rotated pair itself: zero by construction
                            n01 = 0.0;
                            n10 = 0.0;
                        }
                        S[p + u * ld] = n00;
                        S[p + v * ld] = n01;
                        S[q + u * ld] = n10;
                        S[q + v * ld] = n11;
                    }
                    // V <- V J for the columns of pair bi
                    if (si != 0.0) {
                        for (int j = lane; j < n; j += 32) {
                            const double vx = V[j + (int64_t)p * n], vy = V[j + (int64_t)q * n];
                            V[j + (int64_t)p * n] = ci * vx - si * vy;
                            V[j + (int64_t)q * n] = si * vx + ci * vy;
                        }
                    }
                }
            }
            __syncthreads();
        }
        const bool any = rotated != 0;
        __syncthreads();
        if (tid == 0) rotated = 0;
        if (!any) break;
        __syncthreads();
    }
    __syncthreads();
    for (int i = tid; i < n; i += nt) vals[i] = S[i + i * ld];
    for (int w = tid; w < n_in * n_in; w += nt) Vout[w] = V[(w % n_in) + (int64_t)(w / n_in) * n];
    if (tid == 0 && sweeps_out) *sweeps_out = sweep;
}

// V: n_in x n_in eigenvectors (col-major); Vwork: (n_in+1)^2 doubles of
// global scratch, used when the rotations do not fit in shared memory.
// Threads of the Jacobi CTA (CREST_JACOBI_THREADS, a multiple of 32 in [64, 512]).
static int jacobi_threads() {
    const char *e = getenv("CREST_JACOBI_THREADS");
    int v = e ? atoi(e) : 512;
    v = (v / 32) * 32;
    return v < 64 ? 64 : (v > 512 ? 512 : v);
}

int jacobi(const double *A, int n_in, double *Vwork, double *V, double *vals, int *sweeps, cudaStream_t st,
           int max_sweeps = 40) {
    const int n = n_in + (n_in & 1);
    CREST_REQUIRE(n <= kJacobiMax, CREST_EINVAL, "Jacobi size %d exceeds %d", n, kJacobiMax);
    prof::Scope ps("eig_jacobi", st);
    const int nt = jacobi_threads();
    if (n <= kJacobiSmemV) {
        const size_t smem = sizeof(double) * ((size_t)n * (n + 1) + (size_t)n * n);
        CREST_TRY(ensure_smem_attr((const void *)k_jacobi<true>, (size_t)smem));
        k_jacobi<true><<<1, nt, smem, st>>>(A, n_in, n, nullptr, V, vals, max_sweeps, sweeps);
    } else {
        const size_t smem = sizeof(double) * (size_t)n * (size_t)(n + 1);
        CREST_TRY(ensure_smem_attr((const void *)k_jacobi<false>, (size_t)smem));
        k_jacobi<false><<<1, nt, smem, st>>>(A, n_in, n, Vwork, V, vals, max_sweeps, sweeps);
    }
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

// Block reduction helper (sum over the CTA), result valid in every thread.
__device__ double block_sum(double v, double *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w];
    return s;
}

// Classical Gram-Schmidt with one re-orthogonalisation pass, one CTA, on
// columns [j0, p) of a column-major d x p block (columns < j0 are already
// orthonormal).  A column whose norm collapses below 1e-10 of its starting
// norm is replaced by a deterministic random vector and processed again.
// Fallback orthonormalisation when Cholesky QR meets a rank-deficient block.
__global__ void __launch_bounds__(1024) k_cgs2(double *Q, int64_t d, int j0, int p, uint64_t seed) {
    extern __shared__ double sh[];  // r[p] + red[32]
    double *rcoef = sh;
    double *red = sh + p;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    for (int j = j0; j < p; ++j) {
        double *y = Q + (int64_t)j * d;
        for (int attempt = 0; attempt < 3; ++attempt) {
            double s = 0.0;
            for (int64_t r = tid; r < d; r += nt) s += y[r] * y[r];
            const double n0 = block_sum(s, red);
            for (int pass = 0; pass < 2; ++pass) {
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
            const double n1 = block_sum(s, red);
            if (n1 > 1e-20 * n0 && n1 > 0.0) {
                const double inv = 1.0 / sqrt(n1);
                for (int64_t r = tid; r < d; r += nt) y[r] *= inv;
                __syncthreads();
                break;
            }
            for (int64_t r = tid; r < d; r += nt)
                y[r] = (double)(mix64(seed ^ ((uint64_t)(j * 7 + attempt + 1) << 40) ^ (uint64_t)r) >> 11) *
                           0x1.0p-52 -
                       1.0;
            __syncthreads();
        }
    }
}

// Cholesky QR factor for a block Y with Gram matrix B = Y^T Y (p x p).  The
// Gram matrix is first equilibrated, B' = D B D with D = diag(B)^-1/2 (column
// scaling leaves the span unchanged and removes the norm disparity a
// Chebyshev filter creates), shifted by shift_coef * ||B'||_2 (bounded by
// trace(B') = p), and factored B' = L L^T.  Rinv = D L^-T (upper triangular),
// so Y Rinv has orthonormal columns.  One CTA; L, L^-1 and a 16-row panel in
// shared memory.  Both the factorisation and the inverse go by 16 x 16
// blocks: the diagonal block by one warp, the panel and the trailing update
// by the whole block, three barriers per block column.  *fail = 1 (and
// Rinv = I, leaving Y unchanged) when a column is zero or a pivot is not
// positive.
constexpr int kCholNb = 16;

// The same factor for p <= 64 with one barrier per step: the matrix stays
// in shared memory, every thread reads the step's pivot itself, and the
// trailing update uses the unscaled column (A_ij -= A_ik A_jk / A_kk); L^-1
// follows by right-looking substitution on the identity, rows scaled at the
// end.  Rinv and the failure flag have the meaning of k_chol_inv's.
constexpr int kCholSmall = 64;

__global__ void __launch_bounds__(256) k_chol_inv_small(const double *__restrict__ B, int p, double shift_coef,
                                                        double *__restrict__ Rinv, int *fail) {
    extern __shared__ double chol_smem[];
    auto A = reinterpret_cast<double(*)[kCholSmall + 1]>(chol_smem);  // [i][j], lower triangle
    auto R = A + kCholSmall;                                          // right-hand sides -> L^-1, [i][c]
    __shared__ double dsc[kCholSmall], rl[kCholSmall];
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int i = tid; i < p; i += nt) {
        const double b = B[i + (int64_t)i * p];
        if (!(b > 0.0)) bad = 1;
        dsc[i] = b > 0.0 ? 1.0 / sqrt(b) : 1.0;
    }
    __syncthreads();
    const double shift = shift_coef * (double)p;
    for (int w = tid; w < p * p; w += nt) {
        const int i = w % p, j = w / p;
        A[i][j] = (i == j) ? 1.0 + shift : B[w] * dsc[i] * dsc[j];
        R[i][j] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < p; ++k) {
        const double akk = A[k][k];
        const double piv = akk > 0.0 ? akk : 1.0;
        const double rp = 1.0 / piv;
        const int m = p - k - 1;
        for (int w = tid; w < m * m; w += nt) {
            const int i = k + 1 + w % m, j = k + 1 + w / m;
            if (i >= j) A[i][j] -= A[i][k] * A[j][k] * rp;
        }
        if (tid == 0) {
            if (!(akk > 0.0)) bad = 1;
            rl[k] = 1.0 / sqrt(piv);
        }
        __syncthreads();
    }
    // L X = I with L_ik = A_ik rl_k: row i of X is R_i rl_i once rows < i are applied
    for (int i = 0; i < p; ++i) {
        const int m = p - i - 1, n = i + 1;
        const double ri = rl[i];
        for (int w = tid; w < m * n; w += nt) {
            const int t = i + 1 + w % m, c = w / m;
            R[t][c] -= (A[t][i] * ri) * (R[i][c] * ri);
        }
        __syncthreads();
    }
    // Rinv = D (L^-1)^T, or the identity (Y left as it is) when the factor failed
    for (int w = tid; w < p * p; w += nt) {
        const int r = w % p, c = w / p;
        Rinv[w] = bad ? (r == c ? 1.0 : 0.0) : (r <= c ? dsc[r] * R[c][r] * rl[c] : 0.0);
    }
    if (tid == 0 && bad) *fail = 1;
}

__global__ void __launch_bounds__(512) k_chol_inv(const double *__restrict__ B, int p, double shift_coef,
                                                  double *__restrict__ Rinv, int *fail) {
    extern __shared__ double sm[];
    double *L = sm;                     // p x p, col-major (lower triangle used)
    double *X = sm + (size_t)p * p;     // L^-1, col-major
    double *T = X + (size_t)p * p;      // kCholNb x p panel
    __shared__ double dsc[kJacobiMax];
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int i = tid; i < p; i += nt) {
        const double b = B[i + (int64_t)i * p];
        if (!(b > 0.0)) bad = 1;
        dsc[i] = b > 0.0 ? 1.0 / sqrt(b) : 1.0;
    }
    __syncthreads();
    const double shift = shift_coef * (double)p;
    for (int w = tid; w < p * p; w += nt) {
        const int r = w % p, c = w / p;
        L[w] = (r == c) ? 1.0 + shift : B[w] * dsc[r] * dsc[c];
        X[w] = 0.0;
    }
    __syncthreads();
    // ---- B' = L L^T, right-looking by block columns
    for (int k0 = 0; k0 < p; k0 += kCholNb) {
        const int kb = min(kCholNb, p - k0);
        if (wid == 0) {  // diagonal block, unblocked, lane i owns row k0 + i
            for (int j = 0; j < kb; ++j) {
                const int jj = k0 + j;
                double piv = L[jj + jj * p];
                if (!(piv > 0.0)) {
                    if (lane == 0) bad = 1;
                    piv = 1.0;
                }
                const double r = sqrt(piv);
                __syncwarp();
                if (lane == j) L[jj + jj * p] = r;
                if (lane > j && lane < kb) L[k0 + lane + jj * p] /= r;
                __syncwarp();
                if (lane > j && lane < kb) {
                    const int i = k0 + lane;
                    const double lij = L[i + jj * p];
                    for (int c = j + 1; c <= lane; ++c) L[i + (k0 + c) * p] -= lij * L[k0 + c + jj * p];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // panel below the diagonal block: L21 = A21 L11^-T, one row per thread
        for (int i = k0 + kb + tid; i < p; i += nt) {
            for (int j = 0; j < kb; ++j) {
                double v = L[i + (k0 + j) * p];
                for (int t = 0; t < j; ++t) v -= L[i + (k0 + t) * p] * L[k0 + j + (k0 + t) * p];
                L[i + (k0 + j) * p] = v / L[k0 + j + (k0 + j) * p];
            }
        }
        __syncthreads();
        // trailing lower triangle: A22 -= L21 L21^T
        const int r0 = k0 + kb, rem = p - r0;
        for (int w = tid; w < rem * rem; w += nt) {
            const int i = r0 + w % rem, j = r0 + w / rem;
            if (i < j) continue;
            double v = L[i + j * p];
            for (int t = 0; t < kb; ++t) v -= L[i + (k0 + t) * p] * L[j + (k0 + t) * p];
            L[i + j * p] = v;
        }
        __syncthreads();
    }
    // ---- X = L^-1 by block rows: X_II = L_II^-1, X_IC = -X_II sum_K L_IK X_KC
    for (int i0 = 0; i0 < p; i0 += kCholNb) {
        const int ib = min(kCholNb, p - i0);
        if (wid == 0 && lane < ib) {  // diagonal block, lane c owns column i0 + c
            const int c = lane;
            for (int i = c; i < ib; ++i) {
                double v = (i == c) ? 1.0 : 0.0;
                for (int t = c; t < i; ++t) v -= L[i0 + i + (i0 + t) * p] * X[i0 + t + (i0 + c) * p];
                X[i0 + i + (i0 + c) * p] = v / L[i0 + i + (i0 + i) * p];
            }
        }
        for (int w = tid; w < ib * i0; w += nt) {  // T[ii][c] = sum_{t=c}^{i0-1} L[i0+ii][t] X[t][c]
            const int ii = w % ib, c = w / ib;
            double v = 0.0;
            for (int t = c; t < i0; ++t) v += L[i0 + ii + t * p] * X[t + c * p];
            T[ii + c * kCholNb] = v;
        }
        __syncthreads();
        for (int w = tid; w < ib * i0; w += nt) {
            const int ii = w % ib, c = w / ib;
            double v = 0.0;
            for (int t = 0; t <= ii; ++t) v += X[i0 + ii + (i0 + t) * p] * T[t + c * kCholNb];
            X[i0 + ii + c * p] = -v;
        }
        __syncthreads();
    }
    // Rinv = D (L^-1)^T, or the identity (Y left as it is) when the factor failed
    for (int w = tid; w < p * p; w += nt) {
        const int r = w % p, c = w / p;
        Rinv[w] = bad ? (r == c ? 1.0 : 0.0) : dsc[r] * X[c + r * p];
    }
    if (tid == 0 && bad) *fail = 1;
}

// r_i = || W_i - theta_i V_i || for the given columns; rmax[i] per column.
__global__ void k_residual(const double *__restrict__ W, const double *__restrict__ V, const double *theta,
                           int64_t d, double *res) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    const double th = theta[i];
    double s = 0.0;
    for (int64_t r = threadIdx.x; r < d; r += blockDim.x) {
        const double e = W[(int64_t)i * d + r] - th * V[(int64_t)i * d + r];
        s += e * e;
    }
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) res[i] = sqrt(t);
}

// Permute the Ritz basis: dst[:, j] = src[:, perm[j]] for j < p.
__global__ void k_permute_cols(const double *src, double *dst, int64_t d, const int *perm, int p) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d * p) return;
    const int64_t r = idx % d, j = idx / d;
    dst[idx] = src[(int64_t)perm[j] * d + r];
}

// S = C - e I (d x d, col-major; S may be a copy of C made just before).
__global__ void k_shift_diag(double *S, int64_t d, double e) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d) S[i + i * d] -= e;
}

// Z[:, j] = (theta[j] - t) V[:, j] for j < nl (d x nl, col-major).
__global__ void k_scale_cols(const double *V, const double *theta, double t, int64_t d, int nl, double *Z) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= d * nl) return;
    Z[idx] = (theta[idx / d] - t) * V[idx];
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

// y = C x for a symmetric d x d C (column-major; reads column i for y_i).
__global__ void k_symv(const double *__restrict__ C, int64_t d, const double *__restrict__ x, double *__restrict__ y) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= d) return;
    const double *col = C + i * d;
    double s = 0.0;
    for (int64_t j = lane; j < d; j += 32) s += col[j] * x[j];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[i] = s;
}

// One Lanczos step after w = C v_j: alpha_j = v_j.w, w -= alpha v_j + beta v_{j-1},
// full re-orthogonalisation (twice) against V[:, 0..j], beta_j = |w|,
// v_{j+1} = w / beta_j.  One CTA; V is d x (kLanczos + 1) col-major.
__global__ void __launch_bounds__(1024) k_lanczos_step(double *V, int64_t d, int j, double *w, double *ab) {
    __shared__ double red[32];
    __shared__ double coef[kLanczos + 1];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    const double *vj = V + (int64_t)j * d;
    double s = 0.0;
    for (int64_t r = tid; r < d; r += nt) s += vj[r] * w[r];
    const double alpha = block_sum(s, red);
    const double beta_prev = j > 0 ? ab[kLanczos + j - 1] : 0.0;
    for (int64_t r = tid; r < d; r += nt) {
        double v = w[r] - alpha * vj[r];
        if (j > 0) v -= beta_prev * V[(int64_t)(j - 1) * d + r];
        w[r] = v;
    }
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
        for (int i = wid; i <= j; i += nw) {
            const double *qi = V + (int64_t)i * d;
            double t = 0.0;
            for (int64_t r = lane; r < d; r += 32) t += qi[r] * w[r];
            for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) coef[i] = t;
        }
        __syncthreads();
        for (int64_t r = tid; r < d; r += nt) {
            double v = w[r];
            for (int i = 0; i <= j; ++i) v -= coef[i] * V[(int64_t)i * d + r];
            w[r] = v;
        }
        __syncthreads();
    }
    s = 0.0;
    for (int64_t r = tid; r < d; r += nt) s += w[r] * w[r];
    const double beta = sqrt(block_sum(s, red));
    double *vn = V + (int64_t)(j + 1) * d;
    const double inv = beta > 0.0 ? 1.0 / beta : 0.0;
    for (int64_t r = tid; r < d; r += nt) vn[r] = w[r] * inv;
    if (tid == 0) {
        ab[j] = alpha;
        ab[kLanczos + j] = beta;
    }
}

// All L Lanczos steps in one cooperative launch (one CTA per SM).  CTA b
// owns rows [r0, r1) of C and of the basis: it keeps those rows of C in
// shared memory as FP32 (the run only brackets the spectrum: FP32 products
// move the extreme Ritz values by ~1e-7 relative, far inside the guard the
// filter interval keeps) and its slice of the basis in FP64, so only the
// current vector crosses the grid.  Per step, three grid barriers:
//   1. w' = C v_j / beta_{j-1} on the owned rows (v_j = w / beta_{j-1} is
//      normalised on the fly), and the partial dots of those rows with
//      v_0..v_j;
//   2. h = the sum of the partials over CTAs (a fixed shuffle tree);
//      w' -= V h on the owned rows, and the second Gram-Schmidt pass's
//      partials;
//   3. the same subtraction again, w' published for the next product, and
//      the partial squared norm.
// alpha_j is the first-pass coefficient of v_j.  Every sum runs in a fixed
// order, so the run is deterministic.  Each barrier wait is bounded (about
// one second of %globaltimer); on expiry the CTA raises *err and every later
// barrier is skipped, so the launch always ends.
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier on counters that only grow (zeroed before the launch).  CTAs
// arrive on the counter of their group of 16 (one 128-byte line each, so
// arrivals do not all queue on one address); the last arrival of a group
// adds one to the top counter, and barrier number `phase` is passed once the
// top counter reaches phase x groups.
constexpr int kBarGroup = 16;

__device__ void grid_barrier(unsigned *bar, unsigned &phase, unsigned nblk, int *err) {
    __syncthreads();
    ++phase;
    if (threadIdx.x == 0) {
        volatile int *e = err;
        if (!*e) {
            const unsigned n_groups = (nblk + kBarGroup - 1) / kBarGroup, g = blockIdx.x / kBarGroup;
            const unsigned in_group = min((unsigned)kBarGroup, nblk - g * kBarGroup);
            unsigned *top = bar, *mine = bar + 32 * (1 + g);
            __threadfence();
            if (atomicAdd(mine, 1u) == phase * in_group - 1) atomicAdd(top, 1u);
            const unsigned target = phase * n_groups;
            const unsigned long long t0 = gtimer();
            for (;;) {
                unsigned v;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(top) : "memory");
                if (v >= target) break;
                if (*e || gtimer() - t0 > 1000000000ull) {
                    atomicExch(err, 1);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

struct LanczosArgs {
    const double *C;
    int64_t d;
    int L;
    int rows;      // rows per CTA (the last CTAs may own fewer)
    const double *z0;  // the normalised start vector
    double *w;     // d: the current (unnormalised) vector, published each step
    double *part;  // gridDim.x x 3 x (kLanczos + 1)
    double *ab;    // alpha [0, kLanczos), beta [kLanczos, 2 kLanczos)
    unsigned *bar;
    int *err;
};

constexpr int kLzP = kLanczos + 1;

size_t lanczos_smem(int64_t d, int rows) {
    return sizeof(float) * (size_t)rows * d + sizeof(double) * ((size_t)d + (size_t)kLzP * rows + rows);
}

__global__ void __launch_bounds__(512) k_lanczos(LanczosArgs a) {
    extern __shared__ __align__(16) unsigned char lz_smem[];
    __shared__ double coef[kLzP], red[16];
    __shared__ double scal;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    const unsigned nb = gridDim.x, b = blockIdx.x;
    const int64_t d = a.d;
    const int64_t r0 = min(d, (int64_t)b * a.rows), r1 = min(d, r0 + a.rows);
    const int R = (int)(r1 - r0);
    double *wv = reinterpret_cast<double *>(lz_smem);  // d: the vector being multiplied
    double *zs = wv + d;                               // kLzP x rows: owned slice of the basis
    double *wl = zs + (size_t)kLzP * a.rows;           // rows: owned slice of w'
    float *cs = reinterpret_cast<float *>(wl + a.rows);  // rows x d: owned rows of C
    for (int64_t e = tid; e < (int64_t)R * d; e += nt) cs[e] = (float)a.C[r0 * d + e];
    for (int64_t e = tid; e < d; e += nt) wv[e] = a.z0[e];
    if (tid == 0) scal = 1.0;  // the start vector plays the role of w with beta = 1
    double *part = a.part + (size_t)b * 3 * kLzP;
    unsigned phase = 0;
    __syncthreads();
    for (int j = 0; j < a.L; ++j) {
        if (j > 0)
            for (int64_t e = tid; e < d; e += nt) wv[e] = __ldcg(a.w + e);
        __syncthreads();
        const double inv = 1.0 / scal;
        for (int rr = tid; rr < R; rr += nt) zs[j * a.rows + rr] = wv[r0 + rr] * inv;
        for (int rr = wid; rr < R; rr += nw) {
            const float *row = cs + (size_t)rr * d;
            double t0 = 0.0, t1 = 0.0;
            int64_t i = lane;
            for (; i + 32 < d; i += 64) {
                t0 += (double)row[i] * wv[i];
                t1 += (double)row[i + 32] * wv[i + 32];
            }
            if (i < d) t0 += (double)row[i] * wv[i];
            double t = t0 + t1;
            for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) wl[rr] = t * inv;
        }
        __syncthreads();
        for (int pass = 0; pass < 3; ++pass) {
            double *pp = part + pass * kLzP;
            if (pass < 2) {  // partial dots of the owned rows with v_0..v_j
                for (int i = wid; i <= j; i += nw) {
                    double t = 0.0;
                    for (int rr = lane; rr < R; rr += 32) t += zs[i * a.rows + rr] * wl[rr];
                    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                    if (lane == 0) pp[i] = t;
                }
            } else {
                double t = 0.0;
                for (int rr = tid; rr < R; rr += nt) t += wl[rr] * wl[rr];
                for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (lane == 0) red[wid] = t;
                __syncthreads();
                if (tid == 0) {
                    double s2 = 0.0;
                    for (int i = 0; i < nw; ++i) s2 += red[i];
                    pp[0] = s2;
                }
            }
            grid_barrier(a.bar, phase, nb, a.err);
            if (pass == 2) break;
            // coefficients: warp w sums those of i = w, w + 16, ... (lanes over
            // CTAs, a fixed shuffle tree), all of its loads issued at once
            {
                constexpr int kI = (kLzP + 15) / 16, kC = 8;  // i per warp, CTAs per lane (<= 256 CTAs)
                double v[kI][kC];
#pragma unroll
                for (int q = 0; q < kI; ++q)
#pragma unroll
                    for (int t = 0; t < kC; ++t) {
                        const int i = wid + 16 * q;
                        const unsigned c = lane + 32 * t;
                        v[q][t] = (i <= j && c < nb) ? __ldcg(a.part + ((size_t)c * 3 + pass) * kLzP + i) : 0.0;
                    }
#pragma unroll
                for (int q = 0; q < kI; ++q) {
                    double s2 = 0.0;
#pragma unroll
                    for (int t = 0; t < kC; ++t) s2 += v[q][t];
                    for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                    if (lane == 0 && wid + 16 * q <= j) coef[wid + 16 * q] = s2;
                }
            }
            __syncthreads();
            if (pass == 0 && b == 0 && tid == 0) a.ab[j] = coef[j];
            for (int rr = tid; rr < R; rr += nt) {
                double v = wl[rr];
                for (int i = 0; i <= j; ++i) v -= coef[i] * zs[i * a.rows + rr];
                wl[rr] = v;
                if (pass == 1) a.w[r0 + rr] = v;  // published before the last barrier of the step
            }
            __syncthreads();
        }
        if (wid == 0) {
            double v[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const unsigned c = lane + 32 * t;
                v[t] = c < nb ? __ldcg(a.part + ((size_t)c * 3 + 2) * kLzP) : 0.0;
            }
            double s2 = 0.0;
#pragma unroll
            for (int t = 0; t < 8; ++t) s2 += v[t];
            for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            const double beta = sqrt(s2);
            if (lane == 0) {
                scal = beta > 0.0 ? beta : 1.0;
                if (b == 0) a.ab[kLanczos + j] = beta;
            }
        }
        __syncthreads();
    }
}

// Lanczos tridiagonal T (L x L, col-major) from alpha = ab[0..L), beta = ab[kLanczos..).
__global__ void k_tridiag(const double *ab, int L, double *T) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= L * L) return;
    const int i = idx % L, j = idx / L;
    T[idx] = (i == j) ? ab[i] : ((i == j + 1 || j == i + 1) ? ab[kLanczos + min(i, j)] : 0.0);
}

struct EigWork {
    DevBuf C, Cs, V, W, Y0, Y1, H, Q, vals, sorted, perm, scal, lz, lw, lw2, lpart, lbar, lab, res, rinv, fail;
    GemmWs g;
};

// The cooperative Lanczos launch; CREST_ERUNTIME (nothing launched) when the
// device cannot hold one CTA per SM of it.
int lanczos_coop(EigWork &w, const double *C, int64_t d, int L, cudaStream_t st) {
    static const bool off = [] {
        const char *e = getenv("CREST_EIG_COOP");
        return e && e[0] == '0';
    }();
    if (off) return CREST_ERUNTIME;
    // at most 256 CTAs: each lane of the coefficient sums reads 8 CTAs' partials
    const int nb = (int)std::min<int64_t>(std::min(device_sms(), 256), std::max<int64_t>(1, d / 4));
    const int rows = (int)ceil_div(d, nb);
    const size_t smem = lanczos_smem(d, rows);
    if (smem > (size_t)kMaxSmem || ensure_smem_attr((const void *)k_lanczos, smem) != CREST_OK) {
        (void)cudaGetLastError();
        return CREST_ERUNTIME;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos, 512, smem) != cudaSuccess || per_sm < 1) {
        (void)cudaGetLastError();
        return CREST_ERUNTIME;
    }
    CREST_TRY(w.lw2.ensure(sizeof(double) * (size_t)d));
    CREST_TRY(w.lpart.ensure(sizeof(double) * (size_t)nb * 3 * (kLanczos + 1)));
    // the top counter, then one 128-byte line per group of CTAs
    const size_t bar_bytes = sizeof(unsigned) * 32 * (1 + (size_t)ceil_div(nb, kBarGroup));
    CREST_TRY(w.lbar.ensure(bar_bytes));
    CREST_CUDA_TRY(cudaMemsetAsync(w.lbar.ptr, 0, bar_bytes, st));
    CREST_CUDA_TRY(cudaMemsetAsync(w.fail.as<int>() + 3, 0, sizeof(int), st));
    LanczosArgs a{C, d, L, rows, w.lz.as<double>(), w.lw2.as<double>(), w.lpart.as<double>(),
                  w.lab.as<double>(), w.lbar.as<unsigned>(), w.fail.as<int>() + 3};
    void *args[] = {&a};
    if (cudaLaunchCooperativeKernel((const void *)k_lanczos, dim3(nb), dim3(512), args, smem, st) != cudaSuccess) {
        (void)cudaGetLastError();
        return CREST_ERUNTIME;
    }
    return CREST_OK;
}

// Orthonormalise columns [j0, j0+q) of the d x p block Y against its first
// j0 columns (already orthonormal) and among themselves: shifted Cholesky QR
// passes (Fukaya et al. 2020), CGS2 on the device when Cholesky fails.
int orthonormalise(EigWork &w, double *Y, int64_t d, int j0, int q, bool shifted, uint64_t seed, cudaStream_t st) {
    const int D = (int)d;
    double *Ya = Y + (int64_t)j0 * d;
    double *T = w.Y1.as<double>();  // scratch d x p
    double *B = w.H.as<double>();
    double *Rinv = w.Q.as<double>();
    int *fail = w.fail.as<int>();
    const size_t csmem = sizeof(double) * (2 * (size_t)q * q + (size_t)kCholNb * q);
    CREST_TRY(ensure_smem_attr((const void *)k_chol_inv, (size_t)csmem));
    CREST_CUDA_TRY(cudaMemsetAsync(fail, 0, sizeof(int), st));
    // all passes are queued without a host round trip: a failed factor leaves
    // the block unchanged and raises the flag, checked once at the end
    const int passes = shifted ? 3 : 2;
    for (int pass = 0; pass < passes; ++pass) {
        if (j0 > 0) {  // remove the locked directions (twice for orthogonality)
            for (int rep = 0; rep < 2; ++rep) {
                CREST_TRY(gemm(Gemm{j0, q, D, Y, D, 1, Ya, D, B, j0, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
                CREST_TRY(gemm(Gemm{D, q, j0, Y, D, 0, B, j0, Ya, D, -1.0, Ya, 1.0, nullptr, 0.0}, w.g, st));
            }
        }
        CREST_TRY(gemm(Gemm{q, q, D, Ya, D, 1, Ya, D, B, q, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
        // shift = 11 (d q + q (q + 1)) u ||B'||_2 on the first pass of the shifted form
        const double shift_coef = (shifted && pass == 0) ? 11.0 * ((double)d * q + (double)q * (q + 1)) * 0x1.0p-53 : 0.0;
        {
            prof::Scope ps("eig_cholqr", st);
            constexpr size_t small_smem = sizeof(double) * 2 * kCholSmall * (kCholSmall + 1);
            if (q <= kCholSmall && ensure_smem_attr((const void *)k_chol_inv_small, small_smem) == CREST_OK)
                k_chol_inv_small<<<1, 256, small_smem, st>>>(B, q, shift_coef, Rinv, fail);
            else
                k_chol_inv<<<1, 512, csmem, st>>>(B, q, shift_coef, Rinv, fail);
        }
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_TRY(gemm(Gemm{D, q, q, Ya, D, 0, Rinv, q, T, D, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(Ya, T, sizeof(double) * (size_t)d * q, cudaMemcpyDeviceToDevice, st));
    }
    int hf = 0;
    CREST_CUDA_TRY(cudaMemcpyAsync(&hf, fail, sizeof(int), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    if (hf) {  // rank-deficient block: Gram-Schmidt with random replacements
        prof::Scope ps("eig_cgs2", st);
        k_cgs2<<<1, 1024, sizeof(double) * (size_t)(j0 + q + 32), st>>>(Y, d, j0, j0 + q, seed);
        CREST_CUDA_TRY(cudaGetLastError());
    }
    return CREST_OK;
}

}  // namespace

int eig_topk(const double *G, const double *colsum, int64_t d, int64_t n, int64_t k, double *out_vals,
             double *out_vecs, double *out_total, EigStats *stats, cudaStream_t st) {
    CREST_REQUIRE(d >= 1 && n >= 2, CREST_ERUNTIME, "need at least 2 cells and 1 gene");
    CREST_REQUIRE(k >= 0 && k <= d, CREST_EINVAL, "k=%lld must be in [0, d=%lld]", (long long)k, (long long)d);
    int dev = 0;
    CREST_CUDA_TRY(cudaGetDevice(&dev));
    CREST_REQUIRE(dev >= 0 && dev < 64, CREST_ERUNTIME, "device index %d out of range", dev);
    static thread_local EigWork ws[64];  // per host thread and device
    EigWork &w = ws[dev];
    const double nf = (double)n;
    CREST_TRY(w.C.ensure(sizeof(double) * (size_t)(d * d)));
    CREST_TRY(w.Cs.ensure(sizeof(double) * (size_t)(d * d)));
    double *C = w.C.as<double>();
    {
        prof::Scope ps("eig_centre", st);
        k_centre<<<(unsigned)ceil_div(d * d, 256), 256, 0, st>>>(G, colsum, d, nf, C);
    }
    CREST_CUDA_TRY(cudaGetLastError());
    k_trace<<<1, 1024, 0, st>>>(C, d, out_total);
    CREST_CUDA_TRY(cudaGetLastError());
    if (stats) *stats = EigStats{0, 1, 0.0};
    if (k == 0) return CREST_OK;

    CREST_TRY(w.perm.ensure(sizeof(int) * 512));
    CREST_TRY(w.sorted.ensure(sizeof(double) * 512));
    CREST_TRY(w.vals.ensure(sizeof(double) * 512));
    CREST_TRY(w.scal.ensure(sizeof(double) * 8));
    CREST_TRY(w.res.ensure(sizeof(double) * 512));
    CREST_TRY(w.fail.ensure(sizeof(int) * 4));
    int *perm = w.perm.as<int>();
    double *sorted = w.sorted.as<double>();
    double *jvals = w.vals.as<double>();

    if (d <= kJacobiMax) {  // whole matrix
        const int nn = (int)(d + (d & 1));
        CREST_TRY(w.Q.ensure(sizeof(double) * (size_t)nn * nn));
        CREST_TRY(w.Y0.ensure(sizeof(double) * (size_t)nn * nn));
        CREST_TRY(jacobi(C, (int)d, w.Y0.as<double>(), w.Q.as<double>(), jvals, w.perm.as<int>() + 256, st));
        k_rank<<<(unsigned)ceil_div(d, 128), 128, 0, st>>>(jvals, (int)d, perm, sorted);
        CREST_CUDA_TRY(cudaGetLastError());
        k_emit<<<(unsigned)k, 256, 0, st>>>(w.Q.as<double>(), d, d, perm, sorted, k, out_vals, out_vecs);
        CREST_CUDA_TRY(cudaGetLastError());
        if (stats) {
            int sweeps = 0;
            CREST_CUDA_TRY(cudaMemcpyAsync(&sweeps, w.perm.as<int>() + 256, sizeof(int), cudaMemcpyDeviceToHost, st));
            CREST_CUDA_TRY(cudaStreamSynchronize(st));
            stats->iters = sweeps;
        }
        return CREST_OK;
    }

    int p = (int)round_up(k + 14, 16);
    if (p > kJacobiSmemV) p = kJacobiSmemV;
    if (p > d) p = (int)d;
    CREST_REQUIRE(k <= p - 8, CREST_EINVAL, "n_comps=%lld too large for the block eigensolver (max %d)",
                  (long long)k, kJacobiSmemV - 8);
    const int D = (int)d;
    const size_t blk = sizeof(double) * (size_t)d * (size_t)p;
    CREST_TRY(w.V.ensure(blk));
    CREST_TRY(w.W.ensure(blk));
    CREST_TRY(w.Y0.ensure(blk));
    CREST_TRY(w.Y1.ensure(blk));
    CREST_TRY(w.H.ensure(sizeof(double) * (size_t)p * p));
    CREST_TRY(w.Q.ensure(sizeof(double) * (size_t)p * p));
    CREST_TRY(w.lz.ensure(sizeof(double) * (size_t)d * (kLanczos + 1)));
    CREST_TRY(w.lw.ensure(sizeof(double) * (size_t)d));
    CREST_TRY(w.lab.ensure(sizeof(double) * 2 * kLanczos));
    double *V = w.V.as<double>(), *W = w.W.as<double>(), *Y0 = w.Y0.as<double>();
    double *H = w.H.as<double>(), *Q = w.Q.as<double>();

    // ---- spectrum bounds by Lanczos (full re-orthogonalisation)
    double lam_lo, lam_hi;
    {
        double *LZ = w.lz.as<double>(), *lw = w.lw.as<double>(), *lab = w.lab.as<double>();
        k_random_block<<<(unsigned)ceil_div(d, 256), 256, 0, st>>>(LZ, d, 0x452821e638d01377ull);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_TRY(w.res.ensure(sizeof(double) * 512));
        // normalise v0: one CGS2 pass over a single column
        k_cgs2<<<1, 1024, sizeof(double) * 64, st>>>(LZ, d, 0, 1, 1);
        CREST_CUDA_TRY(cudaGetLastError());
        const int L = (int)std::min<int64_t>(kLanczos, d - 1);
        {
            prof::Scope ps("eig_lanczos", st);
            if (lanczos_coop(w, C, d, L, st) != CREST_OK) {  // one launch per step instead
                for (int j = 0; j < L; ++j) {
                    k_symv<<<(unsigned)ceil_div(d * 32, 256), 256, 0, st>>>(C, d, LZ + (int64_t)j * d, lw);
                    k_lanczos_step<<<1, 1024, 0, st>>>(LZ, d, j, lw, lab);
                }
            }
        }
        CREST_CUDA_TRY(cudaGetLastError());
        // Ritz values of T and the last components of its eigenvectors
        k_tridiag<<<(unsigned)ceil_div(L * L, 256), 256, 0, st>>>(lab, L, H);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_TRY(jacobi(H, L, Y0, Q, jvals, nullptr, st));
        std::vector<double> hab(2 * kLanczos), tw(L), tz((size_t)L * L);
        CREST_CUDA_TRY(cudaMemcpyAsync(hab.data(), lab, sizeof(double) * 2 * kLanczos, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(tw.data(), jvals, sizeof(double) * L, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(tz.data(), Q, sizeof(double) * L * L, cudaMemcpyDeviceToHost, st));
        int lz_err = 0;
        CREST_CUDA_TRY(cudaMemcpyAsync(&lz_err, w.fail.as<int>() + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaStreamSynchronize(st));
        CREST_REQUIRE(!lz_err, CREST_ERUNTIME, "Lanczos grid barrier timed out");
        int imin = 0, imax = 0;
        for (int i = 1; i < L; ++i) {
            if (tw[i] < tw[imin]) imin = i;
            if (tw[i] > tw[imax]) imax = i;
        }
        const double bL = hab[kLanczos + L - 1];
        const double rmin = fabs(bL * tz[(size_t)(L - 1) + (size_t)imin * L]);  // col-major
        const double rmax = fabs(bL * tz[(size_t)(L - 1) + (size_t)imax * L]);
        lam_hi = tw[imax] + rmax;
        // a guard below the smallest Ritz value: eigenvalues a little below
        // the damped interval only slow convergence, they cannot be chosen
        lam_lo = tw[imin] - rmin - 1e-3 * (tw[imax] - tw[imin]);
        if (lam_lo < 0.0) lam_lo = 0.0 - 1e-12 * fabs(lam_hi);
    }
    if (!(lam_hi > 0.0)) {
        // zero covariance: every eigenvalue is 0; any orthonormal basis will do
        k_random_block<<<(unsigned)ceil_div(d * p, 256), 256, 0, st>>>(V, d * p, 0x243f6a8885a308d3ull);
        k_cgs2<<<1, 1024, sizeof(double) * (size_t)(p + 32), st>>>(V, d, 0, p, 3);
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

    // ---- start block
    k_random_block<<<(unsigned)ceil_div(d * p, 256), 256, 0, st>>>(V, d * p, 0x243f6a8885a308d3ull);
    CREST_CUDA_TRY(cudaGetLastError());
    CREST_TRY(orthonormalise(w, V, d, 0, p, false, 11, st));

    const double tol = 1e-11;
    const int max_outer = 60;
    std::vector<double> theta(p), hres(p);
    int locked = 0, it = 0;
    double res_max = INFINITY;
    bool converged = false;
    for (; it < max_outer; ++it) {
        const int q = p - locked;
        double *Va = V + (int64_t)locked * d, *Wa = W + (int64_t)locked * d;
        // Rayleigh-Ritz on the active columns: Wa = C Va, H = Va^T Wa
        CREST_TRY(gemm(Gemm{D, q, D, C, D, 0, Va, D, Wa, D, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
        CREST_TRY(gemm(Gemm{q, q, D, Va, D, 1, Wa, D, H, q, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
        k_symmetrise<<<(unsigned)ceil_div(q * q, 256), 256, 0, st>>>(H, q);
        CREST_CUDA_TRY(cudaGetLastError());
        // While the wanted residuals are far from converged the Ritz vectors
        // only have to span the block (the filter acts on the subspace), so
        // two sweeps stand in for the full diagonalisation; the Ritz values
        // (diagonal of the partly rotated H) only set the filter interval.
        CREST_TRY(jacobi(H, q, Y0, Q, jvals, nullptr, st, res_max > 1e-5 ? 2 : 40));
        k_rank<<<(unsigned)ceil_div(q, 128), 128, 0, st>>>(jvals, q, perm, sorted + locked);
        CREST_CUDA_TRY(cudaGetLastError());
        k_permute_cols<<<(unsigned)ceil_div(q * q, 256), 256, 0, st>>>(Q, H, q, perm, q);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_TRY(gemm(Gemm{D, q, q, Va, D, 0, H, q, Y0, D, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(Va, Y0, sizeof(double) * (size_t)d * q, cudaMemcpyDeviceToDevice, st));
        CREST_TRY(gemm(Gemm{D, q, q, Wa, D, 0, H, q, Y0, D, 1.0, nullptr, 0.0, nullptr, 0.0}, w.g, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(Wa, Y0, sizeof(double) * (size_t)d * q, cudaMemcpyDeviceToDevice, st));
        k_residual<<<(unsigned)q, 256, 0, st>>>(Wa, Va, sorted + locked, d, w.res.as<double>() + locked);
        CREST_CUDA_TRY(cudaGetLastError());
        CREST_CUDA_TRY(cudaMemcpyAsync(theta.data(), sorted, sizeof(double) * p, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(hres.data(), w.res.as<double>(), sizeof(double) * p, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaStreamSynchronize(st));
        const double scale_ref = fmax(fabs(theta[0]), 1e-300);
        // lock the leading converged pairs (in order) and deflate them: their
        // eigenvalues move to lam_lo, the edge of every damped interval, so
        // the filter never amplifies what leaks back into the active block
        const int l0 = locked;
        while (locked < k && hres[locked] <= tol * scale_ref) ++locked;
        if (locked > l0 && locked < k) {
            const int nl = locked - l0;
            double *Vl = V + (int64_t)l0 * d;
            k_scale_cols<<<(unsigned)ceil_div(d * nl, 256), 256, 0, st>>>(Vl, sorted + l0, lam_lo, d, nl, Y0);
            CREST_CUDA_TRY(cudaGetLastError());
            Gemm g{D, D, nl, Y0, D, 0, Vl, D, C, D, -1.0, C, 1.0, nullptr, 0.0};
            g.tB = 1;
            CREST_TRY(gemm(g, w.g, st));
        }
        res_max = 0.0;
        for (int i = 0; i < k; ++i) res_max = fmax(res_max, hres[i] / scale_ref);
        if (locked >= k) {
            converged = true;
            break;
        }
        if (it + 1 >= max_outer) break;
        // Chebyshev filter on the active columns, damping [lam_lo, a]
        const int qa = p - locked;
        Va = V + (int64_t)locked * d;
        Wa = W + (int64_t)locked * d;
        const double a = theta[p - 1], top = theta[locked];
        const double e = 0.5 * (a + lam_lo), c = 0.5 * (a - lam_lo);
        if (!(c > 0.0) || !(top > a)) {
            // no usable interval: one power step
            CREST_CUDA_TRY(cudaMemcpyAsync(Va, Wa, sizeof(double) * (size_t)d * qa, cudaMemcpyDeviceToDevice, st));
        } else {
            // degree: growth 2e4 of the weakest wanted value over the damped
            // interval, capped so that no eigenvalue of the active operator
            // grows by more than 1e8 (the filtered block stays within reach of
            // shifted Cholesky QR).  Until a pair is locked the largest
            // eigenvalue is bounded by the Lanczos estimate, afterwards by the
            // leading active Ritz value plus its residual.
            double bound = top + hres[locked];
            if (locked == 0) bound = fmax(bound, lam_hi);
            const double xk = (theta[k - 1] - e) / c, xb = (bound - e) / c;
            const double gk = acosh(fmax(xk, 1.0 + 1e-12)), gb = acosh(fmax(xb, 1.0 + 1e-12));
            int m = (int)ceil(log(2e4) / fmax(gk, 1e-6));
            const int m_cap = (int)floor(log(1e8) / fmax(gb, 1e-6));
            m = std::max(2, std::min(m, std::min(m_cap, 60)));
            const double sigma1 = c / (top - e);
            double sigma = sigma1;
            double *Yprev = Va, *Ycur = w.Y1.as<double>();
            // Y1 = (sigma1/c) (C Va - e Va); Wa already holds C Va
            CREST_TRY(gemm(Gemm{D, qa, 0, C, D, 0, Va, D, Ycur, D, 0.0, Wa, sigma1 / c, Va, -sigma1 * e / c}, w.g, st));
            // the three-term step with the shift folded into a copy of C:
            // Y_{j+1} = (2 s'/c) (C - e I) Y_j - s s' Y_{j-1}, written over
            // Y_{j-1} (one product with beta, no separate element-wise pass)
            double *Cs = w.Cs.as<double>();
            if (m >= 2) {
                CREST_CUDA_TRY(cudaMemcpyAsync(Cs, C, sizeof(double) * (size_t)(d * d), cudaMemcpyDeviceToDevice, st));
                k_shift_diag<<<(unsigned)ceil_div(d, 256), 256, 0, st>>>(Cs, d, e);
                CREST_CUDA_TRY(cudaGetLastError());
            }
            for (int j = 2; j <= m; ++j) {
                const double sigma_next = 1.0 / (2.0 / sigma1 - sigma);
                CREST_TRY(gemm(Gemm{D, qa, D, Cs, D, 0, Ycur, D, Yprev, D, 2.0 * sigma_next / c, Yprev,
                                    -sigma * sigma_next, nullptr, 0.0},
                               w.g, st));
                sigma = sigma_next;
                double *t = Yprev;
                Yprev = Ycur;
                Ycur = t;
            }
            if (Ycur != Va)
                CREST_CUDA_TRY(
                    cudaMemcpyAsync(Va, Ycur, sizeof(double) * (size_t)d * qa, cudaMemcpyDeviceToDevice, st));
        }
        CREST_TRY(orthonormalise(w, V, d, locked, qa, true, 1000 + it, st));
    }
    if (stats) *stats = EigStats{it + 1, converged ? 1 : 0, res_max};
    // V columns 0..k-1 are the wanted Ritz vectors: locked ones (descending,
    // in locking order) then the active ones; order them by value once more
    k_rank<<<(unsigned)ceil_div(k, 128), 128, 0, st>>>(sorted, (int)k, perm, jvals);
    CREST_CUDA_TRY(cudaGetLastError());
    k_emit<<<(unsigned)k, 256, 0, st>>>(V, d, d, perm, jvals, k, out_vals, out_vecs);
    CREST_CUDA_TRY(cudaGetLastError());
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    return CREST_OK;
}

}  // namespace crest
