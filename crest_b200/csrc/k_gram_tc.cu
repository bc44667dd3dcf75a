// Product-form Gram (K4): split-BF16 ("bf16x3") SYRK on the sm_100a tcgen05
// tensor cores.
//
// Each tile value z = hi + lo (hi = bf16(z), lo = bf16(z - hi)) is stored as
// two gene-major bf16 tiles.  One CTA owns one 128x128 upper-triangular block
// (a-genes x b-genes) of G and contracts the chunk's cells (K):
//
//   G_ab += sum_k hi_a hi_b + hi_a lo_b + lo_a hi_b      (FP32 in TMEM)
//
// Warp roles (10 warps):
//   warp 0     TMA producer: 64-cell stages of A_hi, A_lo (and B_hi, B_lo off
//              the diagonal) into a 3-deep 128B-swizzled shared-memory ring;
//   warp 1     allocates all 512 TMEM columns (four 128x128 FP32 accumulators)
//              and issues the tcgen05.mma instructions from one thread;
//   warps 2-9  fold each stage's FP32 accumulator into FP64 registers while
//              the MMAs run into the next accumulator, so FP32 accumulation
//              never spans more than 64 cells (12 MMAs; the tensor core's
//              FP32 adder does not round to nearest, so long FP32 chains drift),
//              and finally add the FP64 block into G with the bias correction
//              S^T S = Z^T Z - bias c^T - c bias^T - n bias bias^T.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on
// timeout the kernel records an error code, stops issuing work and still
// releases its TMEM before returning.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "prof.cuh"

namespace crest {
namespace {

constexpr int kTile = 128;         // M = N of one block
constexpr int kStageCells = 64;    // K per stage: 64 bf16 = 128 B rows (one swizzle atom)
constexpr int kStages = 3;
constexpr int kAccBufs = 4;        // TMEM accumulators (4 x 128 columns)
constexpr int kOperandBytes = kTile * kStageCells * 2;  // 16 KB
constexpr int kStageBytes = 4 * kOperandBytes;          // A_hi, A_lo, B_hi, B_lo
constexpr int kThreads = 320;
constexpr uint32_t kTmemCols = 512;
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s

// instruction descriptor, kind::f16: D f32 (bit 4), A bf16 (bits 7-9 = 1),
// B bf16 (bits 10-12 = 1), both K-major, N>>3 at bit 17, M>>4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTile >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false (and an error code in *err) after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (!mbar_try(bar, parity)) {
        if (globaltimer() - t0 > kWaitNs) {
            atomicCAS(err, 0, code);
            return false;
        }
        if (*(volatile int *)err) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// UMMA shared-memory descriptor: K-major, 128B swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tri_decode(int t, int nb, int &bi, int &bj) {
    int r = 0, rem = t;
    while (rem >= nb - r) {
        rem -= nb - r;
        ++r;
    }
    bi = r;
    bj = r + rem;
}

struct TcArgs {
    int64_t d, d_pad;
    int n_stages;          // K stages in this launch (m_pad / 64)
    int nb;                // 128-blocks along d_pad
    const double *bias;    // [d] or nullptr
    const double *colsum;  // [d] colsum of S for this chunk
    const int64_t *n_kept;
    double *G;             // [d x d]
    int *err;
};

__global__ void __launch_bounds__(kThreads, 1) k_syrk_bf16x3(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
    extern __shared__ uint8_t smem_dyn[];
    __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], acc_full[kAccBufs], acc_empty[kAccBufs];
    __shared__ uint32_t tmem_base_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int bi, bj;
    tri_decode(blockIdx.x, a.nb, bi, bj);
    const bool diag = bi == bj;
    // 1024-B aligned operand ring
    const uint32_t raw = smem_u32(smem_dyn);
    uint8_t *ring = smem_dyn + (((raw + 1023u) & ~1023u) - raw);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < kAccBufs; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 8);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            const uint32_t bytes = diag ? 2 * kOperandBytes : 4 * kOperandBytes;
            const int ya = bi * kTile, yb = bj * kTile, lo_off = (int)a.d_pad;
            for (int i = 0; i < a.n_stages; ++i) {
                const int s = i % kStages;
                if (i >= kStages && !mbar_wait(&empty_bar[s], ((i / kStages) - 1) & 1, a.err, 1)) break;
                uint8_t *st = ring + (size_t)s * kStageBytes;
                mbar_expect_tx(&full_bar[s], bytes);
                const int x = i * kStageCells;
                tma_load_2d(st, &tmap, &full_bar[s], x, ya);
                tma_load_2d(st + kOperandBytes, &tmap, &full_bar[s], x, lo_off + ya);
                if (!diag) {
                    tma_load_2d(st + 2 * kOperandBytes, &tmap, &full_bar[s], x, yb);
                    tma_load_2d(st + 3 * kOperandBytes, &tmap, &full_bar[s], x, lo_off + yb);
                }
            }
            // drain: every stage release (tcgen05.commit arrival) lands before the CTA exits
            for (int i = max(0, a.n_stages - kStages); i < a.n_stages; ++i)
                if (!mbar_wait(&empty_bar[i % kStages], (i / kStages) & 1, a.err, 5)) break;
        }
    } else if (warp == 1) {
        // --------------------------------------------------------- MMA issuer
        if (lane == 0) {
            for (int i = 0; i < a.n_stages; ++i) {
                const int buf = i % kAccBufs;
                if (i >= kAccBufs && !mbar_wait(&acc_empty[buf], ((i / kAccBufs) - 1) & 1, a.err, 2)) break;
                const uint32_t d_tmem = tmem + (uint32_t)(buf * kTile);
                {
                    const int s = i % kStages;
                    if (!mbar_wait(&full_bar[s], (i / kStages) & 1, a.err, 3)) break;
                    tc_fence_after();
                    const uint32_t st = smem_u32(ring + (size_t)s * kStageBytes);
                    const uint32_t a_hi = st, a_lo = st + kOperandBytes;
                    const uint32_t b_hi = diag ? a_hi : st + 2 * kOperandBytes;
                    const uint32_t b_lo = diag ? a_lo : st + 3 * kOperandBytes;
#pragma unroll
                    for (int kk = 0; kk < kStageCells / 16; ++kk) {
                        const uint32_t off = kk * 32;  // 16 bf16 along K inside the 128-B row
                        const uint32_t first = kk == 0 ? 0u : 1u;
                        umma_bf16(d_tmem, umma_desc(a_hi + off), umma_desc(b_hi + off), first);
                        umma_bf16(d_tmem, umma_desc(a_hi + off), umma_desc(b_lo + off), 1u);
                        umma_bf16(d_tmem, umma_desc(a_lo + off), umma_desc(b_hi + off), 1u);
                    }
                    umma_commit(&empty_bar[s]);  // stage reusable once these MMAs complete
                }
                umma_commit(&acc_full[buf]);
            }
        }
    } else {
        // ----------------------------------------------------------- epilogue
        const int q = warp & 3;              // TMEM lane quadrant this warp may access
        const int h = (warp - 2) >> 2;       // column half: 0 -> 0..63, 1 -> 64..127
        const int row = q * 32 + lane;
        double acc[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) acc[j] = 0.0;
        bool ok = true;
        for (int p = 0; p < a.n_stages; ++p) {
            const int buf = p % kAccBufs;
            // one lane waits, the warp reconverges before the .sync.aligned TMEM loads
            int got = 0;
            if (lane == 0) got = mbar_wait(&acc_full[buf], (p / kAccBufs) & 1, a.err, 4) ? 1 : 0;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * kTile + h * 64);
            float v[32];
            tmem_ld32(taddr, v);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[j] += (double)v[j];
            tmem_ld32(taddr + 32, v);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[32 + j] += (double)v[j];
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);
        }
        if (ok) {
            const int64_t ga = (int64_t)bi * kTile + row;
            if (ga < a.d) {
                const double nk = (double)*a.n_kept;
                const double ba = a.bias ? a.bias[ga] : 0.0, ca = a.colsum[ga];
                double *grow = a.G + ga * a.d;
#pragma unroll
                for (int j = 0; j < 64; ++j) {
                    const int64_t gb = (int64_t)bj * kTile + h * 64 + j;
                    if (gb >= a.d || gb < ga) continue;
                    double v = acc[j];
                    if (a.bias) {
                        const double bb = a.bias[gb], cb = a.colsum[gb];
                        v = v - ba * cb - ca * bb - nk * ba * bb;
                    }
                    grow[gb] += v;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// --------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

struct ErrFlag {
    int *dev = nullptr;
};

}  // namespace

static ErrFlag g_tc_err[64];

// Device error word of the current device (0 = no bounded wait has timed out).
int *tc_error_word() {
    int dev = 0;
    cudaGetDevice(&dev);
    ErrFlag &f = g_tc_err[dev & 63];
    if (!f.dev) {
        if (cudaMalloc(&f.dev, sizeof(int)) != cudaSuccess) return nullptr;
        cudaMemset(f.dev, 0, sizeof(int));
    }
    return f.dev;
}

int tc_check_error() {
    int *e = tc_error_word();
    if (!e) return CREST_OK;
    int h = 0;
    CREST_CUDA_TRY(cudaMemcpy(&h, e, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        cudaMemset(e, 0, sizeof(int));
        set_error("tensor-core Gram: a bounded pipeline wait timed out (code %d)", h);
        return CREST_ETIMEOUT;
    }
    return CREST_OK;
}

int syrk_bf16x3_fold(const GramWork &w, int64_t m_pad, const DevScale &t, double *gram, cudaStream_t st) {
    CREST_REQUIRE(m_pad % kStageCells == 0 && w.d_pad % kTile == 0, CREST_EINVAL, "bad tensor-core tile shape");
    auto enc = encode_fn();
    CREST_REQUIRE(enc != nullptr, CREST_ECUDA, "cuTensorMapEncodeTiled is unavailable");
    int *err = tc_error_word();
    CREST_REQUIRE(err != nullptr, CREST_ENOMEM, "could not allocate the pipeline error word");
    // hi rows [0, d_pad) then lo rows [d_pad, 2 d_pad), cells contiguous
    CUtensorMap map;
    cuuint64_t dims[2] = {(cuuint64_t)m_pad, (cuuint64_t)(2 * w.d_pad)};
    cuuint64_t strides[1] = {(cuuint64_t)m_pad * 2};
    cuuint32_t box[2] = {kStageCells, kTile};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, w.tile, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    CREST_REQUIRE(r == CUDA_SUCCESS, CREST_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    TcArgs a;
    a.d = w.d;
    a.d_pad = w.d_pad;
    a.n_stages = (int)(m_pad / kStageCells);
    a.nb = (int)(w.d_pad / kTile);
    a.bias = t.scale ? t.bias : nullptr;
    a.colsum = w.colsum_chunk;
    a.n_kept = w.n_kept;
    a.G = gram;
    a.err = err;
    const size_t smem = 1024 + (size_t)kStages * kStageBytes;
    CREST_CUDA_TRY(cudaFuncSetAttribute(k_syrk_bf16x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int tiles = a.nb * (a.nb + 1) / 2;
    prof::Scope ps("syrk_bf16x3_tcgen05", st);
    k_syrk_bf16x3<<<tiles, kThreads, smem, st>>>(map, a);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
