// Product-form Gram (K4): split-BF16 ("bf16x3") SYRK on the sm_100a tcgen05
// tensor cores.
//
// Each tile value z = hi + lo (hi = bf16(z), lo = bf16(z - hi)) is stored in
// two cell-major bf16 tiles (one row of genes per cell), so both operands are
// MN-major for the tensor core.  One CTA owns one 128x128 upper-triangular
// block (a-genes x b-genes) of G and contracts the chunk's cells (K):
//
//   G_ab += sum_k hi_a hi_b + hi_a lo_b + lo_a hi_b      (FP32 in TMEM)
//
// Warp roles (10 warps):
//   warp 0     TMA producer: 64-cell stages of A_hi, A_lo (and B_hi, B_lo off
//              the diagonal) into a 3-deep 128B-swizzled shared-memory ring;
//   warp 1     allocates all 512 TMEM columns (four 128x128 FP32 accumulators)
//              and issues the tcgen05.mma instructions from one thread;
//   warps 2-9  fold each period's FP32 accumulator (fold stages of 64 cells,
//              2 by default) into FP64 register sums while the
//              MMAs run into the next accumulator, so the tensor core's FP32
//              accumulation never spans more than one period (12 MMAs per
//              stage; long FP32 chains in the tensor core drift, measured
//              1.2e-5 relative over 512 cells); at the end the block goes
//              through shared memory to a coalesced FP64 update of G with the
//              shift correction S^T S = Z^T Z - shift c^T - c shift^T - n shift shift^T.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on
// timeout the kernel records an error code, stops issuing work and still
// releases its TMEM before returning.
#include <cuda.h>
#include <stdlib.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "prof.cuh"

namespace crest {
namespace {

constexpr int kTile = 128;         // M = N of one block
constexpr int kStageCells = 64;    // K per stage (cells)
constexpr int kHalf = 64;          // genes per TMA box / MN swizzle atom: 64 bf16 = 128 B
constexpr int kStages = 3;
constexpr int kAccBufs = 4;        // TMEM accumulators (4 x 128 columns)
constexpr int kBoxBytes = kHalf * kStageCells * 2;     // 8 KB: 64 genes x 64 cells
constexpr int kOperandBytes = 2 * kBoxBytes;           // 16 KB: 128 genes x 64 cells
constexpr int kStageBytes = 4 * kOperandBytes;          // A_hi, A_lo, B_hi, B_lo
constexpr int kEpiWarps = 8;      // 2 per TMEM lane quadrant, 64 accumulator columns each
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr uint32_t kTmemCols = 512;
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s: the limit of every pipeline wait

// instruction descriptor, kind::f16: D f32 (bit 4), A bf16 (bits 7-9 = 1),
// B bf16 (bits 10-12 = 1), A and B MN-major (bits 15, 16), N>>3 at bit 17,
// M>>4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                            ((uint32_t)(kTile >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);

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

// try_wait suspends the thread until the phase completes or the hint (ns)
// expires, so a waiting role costs no issue slots and wakes on completion.
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Bounded wait: false (and an error code in *err) after `limit` ns (kWaitNs
// unless a test shortens it).  The error word (global memory) is only looked
// at on the slow path, every 64 polls, so another role's failure also ends
// this wait.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          unsigned long long limit) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (uint32_t n = 1;; ++n) {
        if (mbar_try(bar, parity)) return true;
        if ((n & 63u) == 0) {
            if (globaltimer() - t0 > limit) {
                atomicCAS(err, 0, code);
                return false;
            }
            if (*(volatile int *)err) return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// UMMA shared-memory descriptor of an MN-major operand with 128B swizzle:
// 64-element MN atoms (128 B rows, one row per K index), atoms along MN
// kBoxBytes apart (leading byte offset), groups of 8 K rows 1024 B apart
// (stride byte offset).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kBoxBytes >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
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
    int m_pad;             // cells in the tile (row offset of the lo tile)
    int fold;              // stages accumulated in FP32 before each FP64 fold
    int nb;                // 128-blocks along d_pad
    const double *bias;    // [d] or nullptr
    const double *colsum;  // [d] colsum of S for this chunk
    const int64_t *n_kept;
    double *G;             // [d x d]
    int *err;
    unsigned long long wait_ns;  // limit of every pipeline wait
    int stall_stage;       // test hook: the producer leaves this stage's loads out (-1: none)
};

// Bounded mbarrier wait made by lane 0 and broadcast, so the calling warp
// stays converged (the .sync.aligned tcgen05 instructions need the whole warp).
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          unsigned long long limit) {
    int got = 0;
    if ((threadIdx.x & 31) == 0) got = mbar_wait(bar, parity, err, code, limit) ? 1 : 0;
    return __shfl_sync(0xffffffffu, got, 0) != 0;
}

// Epilogue warps (2 .. 9): fold each period's FP32 accumulator into FP64
// registers, then update block (bi, bj) of G through shared memory (the
// operand ring, idle once the last accumulator has been seen).
__device__ __forceinline__ void tc_epilogue(const TcArgs &a, int bi, int bj, uint32_t tmem, uint8_t *ring,
                                            uint64_t *acc_full, uint64_t *acc_empty, int n_periods, int *epi_ok_sh) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int &epi_ok = *epi_ok_sh;
    auto warp_wait = [&](uint64_t *bar, uint32_t parity, int code) -> bool {
        return ::crest::warp_wait(bar, parity, a.err, code, a.wait_ns);
    };
    const int q = warp & 3;              // TMEM lane quadrant this warp may access
    const int h = (warp - 2) >> 2;       // column group: 64 h .. 64 h + 63
    const int row = q * 32 + lane;
    double acc[64];                      // FP64 sums of the periods
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.0;
    bool ok = true;
    for (int p = 0; p < n_periods; ++p) {
        const int buf = p % kAccBufs;
        if (!warp_wait(&acc_full[buf], (p / kAccBufs) & 1, 4)) {
            ok = false;
            break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * kTile + h * 64);
#pragma unroll
        for (int g = 0; g < 4; ++g) {  // 16 columns at a time keeps the register footprint down
            float v[16];
            tmem_ld16(taddr + 16 * g, v);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[16 * g + j] += (double)v[j];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[buf]);  // accumulator read out
    }
    // Stage the FP64 block in the operand ring (idle once the last
    // accumulator has been seen: every MMA has read its operands), then
    // update G row by row with coalesced accesses.
    double *stage = reinterpret_cast<double *>(ring);
    constexpr int kPitch = kTile + 1;
    if (!ok) atomicExch(&epi_ok, 0);
    if (ok) {
#pragma unroll
        for (int j = 0; j < 64; ++j) stage[row * kPitch + h * 64 + j] = acc[j];
    }
    asm volatile("bar.sync 1, %0;" ::"r"(kEpiWarps * 32) : "memory");  // the epilogue warps
    if (epi_ok) {
        const int e = warp - 2;
        const double nk = (double)*a.n_kept;
        for (int r = e; r < kTile; r += kEpiWarps) {
            const int64_t ga = (int64_t)bi * kTile + r;
            if (ga >= a.d) break;
            const double ba = a.bias ? a.bias[ga] : 0.0, ca = a.colsum[ga];
            double *grow = a.G + ga * a.d;
            for (int cc = lane; cc < kTile; cc += 32) {
                const int64_t gb = (int64_t)bj * kTile + cc;
                if (gb >= a.d || gb < ga) continue;
                double v = stage[r * kPitch + cc];
                if (a.bias) v = v - ba * a.colsum[gb] - ca * a.bias[gb] - nk * ba * a.bias[gb];
                grow[gb] += v;
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads, 1) k_syrk_bf16x3(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
    extern __shared__ uint8_t smem_dyn[];
    __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], acc_full[kAccBufs], acc_empty[kAccBufs];
    __shared__ uint32_t tmem_base_sh;
    __shared__ int epi_ok;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int bi, bj;
    tri_decode(blockIdx.x, a.nb, bi, bj);
    const bool diag = bi == bj;
    // 1024-B aligned operand ring
    const uint32_t raw = smem_u32(smem_dyn);
    uint8_t *ring = smem_dyn + (((raw + 1023u) & ~1023u) - raw);

    if (threadIdx.x == 0) {
        epi_ok = 1;
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < kAccBufs; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiWarps);
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

    // Waits are made by lane 0 and broadcast, so every role warp stays
    // converged (the .sync.aligned tcgen05 instructions need the whole warp).
    auto warp_wait = [&](uint64_t *bar, uint32_t parity, int code) -> bool {
        int got = 0;
        if (lane == 0) got = mbar_wait(bar, parity, a.err, code, a.wait_ns) ? 1 : 0;
        return __shfl_sync(0xffffffffu, got, 0) != 0;
    };
    const int n_periods = (a.n_stages + a.fold - 1) / a.fold;

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        const uint32_t bytes = diag ? 2 * kOperandBytes : 4 * kOperandBytes;
        const int xa = bi * kTile, xb = bj * kTile, lo_off = a.m_pad;
        int issued = 0;
        for (int i = 0; i < a.n_stages; ++i) {
            const int s = i % kStages;
            if (i >= kStages && !warp_wait(&empty_bar[s], ((i / kStages) - 1) & 1, 1)) break;
            if (lane == 0 && i == a.stall_stage) {
                mbar_expect_tx(&full_bar[s], bytes);  // armed, never filled: the consumer's wait runs out
            } else if (lane == 0) {
                uint8_t *st = ring + (size_t)s * kStageBytes;
                mbar_expect_tx(&full_bar[s], bytes);
                const int y = i * kStageCells;  // first cell of the stage
                // operand = two 64-gene boxes side by side (MN atoms kBoxBytes apart)
                tma_load_2d(st, &tmap, &full_bar[s], xa, y);
                tma_load_2d(st + kBoxBytes, &tmap, &full_bar[s], xa + kHalf, y);
                tma_load_2d(st + kOperandBytes, &tmap, &full_bar[s], xa, lo_off + y);
                tma_load_2d(st + kOperandBytes + kBoxBytes, &tmap, &full_bar[s], xa + kHalf, lo_off + y);
                if (!diag) {
                    tma_load_2d(st + 2 * kOperandBytes, &tmap, &full_bar[s], xb, y);
                    tma_load_2d(st + 2 * kOperandBytes + kBoxBytes, &tmap, &full_bar[s], xb + kHalf, y);
                    tma_load_2d(st + 3 * kOperandBytes, &tmap, &full_bar[s], xb, lo_off + y);
                    tma_load_2d(st + 3 * kOperandBytes + kBoxBytes, &tmap, &full_bar[s], xb + kHalf, lo_off + y);
                }
            }
            __syncwarp();
            issued = i + 1;
        }
        // drain: every stage release (tcgen05.commit arrival) lands before the CTA exits
        for (int i = max(0, issued - kStages); i < issued; ++i)
            if (!warp_wait(&empty_bar[i % kStages], (i / kStages) & 1, 5)) break;
    } else if (warp == 1) {
        // --------------------------------------------------------- MMA issuer
        bool ok = true;
        for (int p = 0; p < n_periods && ok; ++p) {
            const int buf = p % kAccBufs;
            if (p >= kAccBufs && !warp_wait(&acc_empty[buf], ((p / kAccBufs) - 1) & 1, 2)) break;
            const uint32_t d_tmem = tmem + (uint32_t)(buf * kTile);
            const int i0 = p * a.fold, i1 = min(a.n_stages, i0 + a.fold);
            for (int i = i0; i < i1; ++i) {
                const int s = i % kStages;
                if (!warp_wait(&full_bar[s], (i / kStages) & 1, 3)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                if (lane == 0) {
                    const uint32_t st = smem_u32(ring + (size_t)s * kStageBytes);
                    const uint32_t a_hi = st, a_lo = st + kOperandBytes;
                    const uint32_t b_hi = diag ? a_hi : st + 2 * kOperandBytes;
                    const uint32_t b_lo = diag ? a_lo : st + 3 * kOperandBytes;
#pragma unroll
                    for (int kk = 0; kk < kStageCells / 16; ++kk) {
                        const uint32_t off = kk * 16 * 128;  // 16 K rows of 128 B = two 8-row groups
                        const uint32_t first = (i == i0 && kk == 0) ? 0u : 1u;
                        umma_bf16(d_tmem, umma_desc(a_hi + off), umma_desc(b_hi + off), first);
                        umma_bf16(d_tmem, umma_desc(a_hi + off), umma_desc(b_lo + off), 1u);
                        umma_bf16(d_tmem, umma_desc(a_lo + off), umma_desc(b_hi + off), 1u);
                    }
                    umma_commit(&empty_bar[s]);  // stage reusable once these MMAs complete
                }
                __syncwarp();
            }
            if (ok && lane == 0) umma_commit(&acc_full[buf]);
            __syncwarp();
        }
    } else {
        // ----------------------------------------------------------- epilogue
        tc_epilogue(a, bi, bj, tmem, ring, acc_full, acc_empty, n_periods, &epi_ok);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// ------------------------------------------------------ CTA-pair form
// The same contraction on pairs of SMs (tcgen05 cta_group::2): a cluster of
// two CTAs owns a 256 x 256 block (bi, bj) of G, M = 256 rows split 128 per
// CTA, N = 256 columns whose B operand is split 128 per CTA, so every CTA
// stages 128 a-genes and 128 b-genes per stage -- the operand bytes per
// output halve against one CTA per 128 x 128 block, which is what bounded
// that form (L2 -> shared memory).  Each CTA's TMEM holds its 128 rows x 256
// columns of the FP32 accumulator, two of them (all 512 columns).  The
// cells of a launch are split in two halves (pairs 2t and 2t + 1 of tile t)
// so the 36 blocks of d = 2048 keep 144 SMs busy; half 1 adds into a second
// FP64 Gram (gram_aux), folded into G once per pass.
//
// Roles: warp 0 of each CTA loads its own operand halves (TMA, cta_group::2
// form, completing on the leader CTA's full barrier, which the leader's
// producer arms with both CTAs' bytes); warp 1 of the leader issues the
// MMAs and the commits, multicast to both CTAs' barriers; warps 2-9 of both
// CTAs read their TMEM rows every period (fold stages of 64 cells) and add
// them into FP32 register sums (one row, 128 columns per thread), and
// release the accumulator on the leader's barrier (local and remote
// arrivals).  FP32 register sums over a launch's periods are correctly
// rounded adds of at most 32 period results; the FP64 update of G at the
// end applies the shift correction once (in half 0).
namespace pair {

constexpr int kN = 256;                       // block edge (M = N)
constexpr int kHalfRows = 128;                // rows (and B columns) per CTA
constexpr int kStageBytes = 4 * kOperandBytes;  // A_hi, A_lo, B_hi, B_lo of this CTA: 64 KB
constexpr int kAccCols = 256;
constexpr int kAccBufs = 2;

__device__ __forceinline__ uint32_t cta_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// shared::cluster address of the same shared-memory location in CTA `rank`
__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ bool try_cluster(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Bounded wait (as mbar_wait) with cluster-scope acquire.
__device__ __forceinline__ bool wait(uint64_t *bar, uint32_t parity, int *err, int code, unsigned long long limit) {
    if (try_cluster(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (uint32_t n = 1;; ++n) {
        if (try_cluster(bar, parity)) return true;
        if ((n & 63u) == 0) {
            if (globaltimer() - t0 > limit) {
                atomicCAS(err, 0, code);
                return false;
            }
            if (*(volatile int *)err) return false;
        }
    }
}

__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          unsigned long long limit) {
    int got = 0;
    if ((threadIdx.x & 31) == 0) got = wait(bar, parity, err, code, limit) ? 1 : 0;
    return __shfl_sync(0xffffffffu, got, 0) != 0;
}

// TMA load into this CTA's shared memory, completing on the barrier at the
// shared::cluster address bar (the leader's).
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

// instruction descriptor: as kIdesc with M = 256 (the pair), N = 256
constexpr uint32_t kIdesc2 = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                             ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(kN >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kIdesc2), "r"(accumulate), "r"(0u));
}

// arrive on barrier `bar` (same offset) in both CTAs once this thread's MMAs complete
__device__ __forceinline__ void commit_both(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"((uint16_t)3)
        : "memory");
}

struct Args {
    int64_t d, d_pad;
    int n_stages;          // 64-cell stages of the launch
    int m_pad;             // cells in the tile (row offset of the lo plane)
    int fold;              // stages per FP32 TMEM period
    int nb;                // 256-blocks along d_pad
    const double *bias;    // [d] or nullptr
    const double *colsum;  // [d]
    const int64_t *n_kept;
    double *G, *G_aux;     // [d x d]: cell halves 0 and 1
    int *err;
    unsigned long long wait_ns;  // limit of every pipeline wait
    int stall_stage;       // test hook: the leader's producer leaves this stage out (-1: none)
};

__global__ void __launch_bounds__(kThreads, 1) k_syrk_pair(const __grid_constant__ CUtensorMap tmap, Args a) {
    extern __shared__ uint8_t smem_dyn[];
    __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], acc_full[kAccBufs], acc_empty[kAccBufs];
    __shared__ uint32_t tmem_base_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cta_rank();
    const bool leader = rank == 0;
    const int pair_id = blockIdx.x >> 1;
    const int t = pair_id >> 1, half = pair_id & 1;
    int bi, bj;
    tri_decode(t, a.nb, bi, bj);
    const bool diag = bi == bj;
    const int s_lo = half == 0 ? 0 : a.n_stages / 2, s_hi = half == 0 ? a.n_stages / 2 : a.n_stages;
    const int n_my = s_hi - s_lo;
    const int n_periods = (n_my + a.fold - 1) / a.fold;
    const uint32_t raw = smem_u32(smem_dyn);
    uint8_t *ring = smem_dyn + (((raw + 1023u) & ~1023u) - raw);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < kAccBufs; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * kEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    cluster_sync();  // barriers initialised and TMEM allocated in both CTAs
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        // ------------------------------------------------------ producer
        const uint32_t bytes_cta = diag ? 2 * kOperandBytes : 4 * kOperandBytes;
        const int xa = bi * kN + (int)rank * kHalfRows, xb = bj * kN + (int)rank * kHalfRows, lo_off = a.m_pad;
        int issued = 0;
        for (int i = 0; i < n_my; ++i) {
            const int s = i % kStages;
            if (i >= kStages && !warp_wait(&empty_bar[s], ((i / kStages) - 1) & 1, a.err, 11, a.wait_ns)) break;
            if (lane == 0 && leader && i == a.stall_stage) {
                mbar_expect_tx(&full_bar[s], 2 * bytes_cta);  // armed, never filled (test hook)
            } else if (lane == 0) {
                uint8_t *st = ring + (size_t)s * kStageBytes;
                const uint32_t fb = mapa(smem_u32(&full_bar[s]), 0);
                if (leader) mbar_expect_tx(&full_bar[s], 2 * bytes_cta);
                const int y = (s_lo + i) * kStageCells;
                tma_load(st, &tmap, fb, xa, y);
                tma_load(st + kBoxBytes, &tmap, fb, xa + kHalf, y);
                tma_load(st + kOperandBytes, &tmap, fb, xa, lo_off + y);
                tma_load(st + kOperandBytes + kBoxBytes, &tmap, fb, xa + kHalf, lo_off + y);
                if (!diag) {
                    tma_load(st + 2 * kOperandBytes, &tmap, fb, xb, y);
                    tma_load(st + 2 * kOperandBytes + kBoxBytes, &tmap, fb, xb + kHalf, y);
                    tma_load(st + 3 * kOperandBytes, &tmap, fb, xb, lo_off + y);
                    tma_load(st + 3 * kOperandBytes + kBoxBytes, &tmap, fb, xb + kHalf, lo_off + y);
                }
            }
            __syncwarp();
            issued = i + 1;
        }
        // drain: the last stages' releases (MMA commits) land before exit
        for (int i = max(0, issued - kStages); i < issued; ++i)
            if (!warp_wait(&empty_bar[i % kStages], (i / kStages) & 1, a.err, 15, a.wait_ns)) break;
    } else if (warp == 1) {
        // --------------------------------------------- MMA issuer (leader)
        if (leader) {
            bool ok = true;
            for (int p = 0; p < n_periods && ok; ++p) {
                const int buf = p % kAccBufs;
                if (p >= kAccBufs && !warp_wait(&acc_empty[buf], ((p / kAccBufs) - 1) & 1, a.err, 12, a.wait_ns)) break;
                const uint32_t d_tmem = tmem + (uint32_t)(buf * kAccCols);
                const int i0 = p * a.fold, i1 = min(n_my, i0 + a.fold);
                for (int i = i0; i < i1; ++i) {
                    const int s = i % kStages;
                    if (!warp_wait(&full_bar[s], (i / kStages) & 1, a.err, 13, a.wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    if (lane == 0) {
                        const uint32_t st = smem_u32(ring + (size_t)s * kStageBytes);
                        const uint32_t a_hi = st, a_lo = st + kOperandBytes;
                        const uint32_t b_hi = diag ? a_hi : st + 2 * kOperandBytes;
                        const uint32_t b_lo = diag ? a_lo : st + 3 * kOperandBytes;
#pragma unroll
                        for (int kk = 0; kk < kStageCells / 16; ++kk) {
                            const uint32_t off = kk * 16 * 128;
                            const uint32_t first = (i == i0 && kk == 0) ? 0u : 1u;
                            mma(d_tmem, umma_desc(a_hi + off), umma_desc(b_hi + off), first);
                            mma(d_tmem, umma_desc(a_hi + off), umma_desc(b_lo + off), 1u);
                            mma(d_tmem, umma_desc(a_lo + off), umma_desc(b_hi + off), 1u);
                        }
                        commit_both(&empty_bar[s]);
                    }
                    __syncwarp();
                }
                if (ok && lane == 0) commit_both(&acc_full[buf]);
                __syncwarp();
            }
        }
    } else {
        // ------------------------------------------------------ epilogue
        const int q = warp & 3;         // TMEM lane quadrant of this warp
        const int h = (warp - 2) >> 2;  // columns 128 h .. 128 h + 127
        const int row = q * 32 + lane;
        float acc[128];
#pragma unroll
        for (int j = 0; j < 128; ++j) acc[j] = 0.0f;
        bool ok = true;
        const uint32_t empty_leader[2] = {mapa(smem_u32(&acc_empty[0]), 0), mapa(smem_u32(&acc_empty[1]), 0)};
        for (int p = 0; p < n_periods; ++p) {
            const int buf = p % kAccBufs;
            if (!warp_wait(&acc_full[buf], (p / kAccBufs) & 1, a.err, 14, a.wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * kAccCols + h * 128);
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                float v[16];
                tmem_ld16(taddr + 16 * g, v);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[16 * g + j] += v[j];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) arrive_cluster(empty_leader[buf]);
        }
        // the ring is idle: every MMA (which reads both CTAs' stages) has
        // completed before the last accumulator was committed
        float *stage = reinterpret_cast<float *>(ring);
        constexpr int kPitch = kN + 1;
        if (ok) {
#pragma unroll
            for (int j = 0; j < 128; ++j) stage[row * kPitch + h * 128 + j] = acc[j];
        }
        asm volatile("bar.sync 1, %0;" ::"r"(kEpiWarps * 32) : "memory");
        if (ok && !*(volatile int *)a.err) {
            const int e = warp - 2;
            const bool corr = half == 0 && a.bias;
            double *G = half == 0 ? a.G : a.G_aux;
            const double nk = (double)*a.n_kept;
            // kRmwRows rows per pass, every load of a pass issued before the
            // first add: 8 kRmwRows independent G reads in flight per lane;
            // G goes through L2 as evict-first so that it does not push the
            // next tile's operands out
            constexpr int kRmwRows = 4;
            for (int r0 = e; r0 < kHalfRows; r0 += kRmwRows * kEpiWarps) {
                double gv[kRmwRows][8];
#pragma unroll
                for (int u = 0; u < kRmwRows; ++u) {
                    const int64_t ga = (int64_t)bi * kN + (int64_t)rank * kHalfRows + r0 + u * kEpiWarps;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int64_t gb = (int64_t)bj * kN + lane + 32 * c;
                        gv[u][c] = (ga < a.d && gb < a.d && gb >= ga) ? __ldcs(G + ga * a.d + gb) : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < kRmwRows; ++u) {
                    const int r = r0 + u * kEpiWarps;
                    const int64_t ga = (int64_t)bi * kN + (int64_t)rank * kHalfRows + r;
                    if (ga >= a.d) continue;
                    const double ba = corr ? a.bias[ga] : 0.0, ca = corr ? a.colsum[ga] : 0.0;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int cc = lane + 32 * c;
                        const int64_t gb = (int64_t)bj * kN + cc;
                        if (gb >= a.d || gb < ga) continue;
                        double v = (double)stage[r * kPitch + cc];
                        if (corr) v = v - ba * a.colsum[gb] - ca * a.bias[gb] - nk * ba * a.bias[gb];
                        __stcs(G + ga * a.d + gb, gv[u][c] + v);
                    }
                }
            }
        }
    }
    tc_fence_before();
    cluster_sync();  // both CTAs done with TMEM, barriers and shared memory
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

}  // namespace pair

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

// FP32 accumulation period in stages of kStageCells cells (CREST_TC_FOLD,
// default 128 cells; at 1M cells periods of 64, 128 and 256 cells all keep
// the top-50 subspace within 0.007 degree of the FP64 Gram, 512 cells drift
// past 0.01 degree).
// Failure-injection hook for tests (host side, read at every launch):
// CREST_TC_INJECT_STALL=1 makes the producer arm the last stage of the launch
// without loading it and shortens every pipeline wait to 5 ms, so the MMA
// issuer's wait runs out, the kernel records the error and returns with its
// TMEM released; the next call reports CREST_ETIMEOUT.  Off by default.
void tc_test_hooks(int n_stages, unsigned long long &wait_ns, int &stall_stage) {
    const char *e = getenv("CREST_TC_INJECT_STALL");
    const bool on = e && e[0] == '1' && n_stages > 0;
    wait_ns = on ? 5000000ull : kWaitNs;
    stall_stage = on ? n_stages - 1 : -1;
}

// CTA-pair SYRK (default) or one CTA per 128 x 128 block (CREST_TC_PAIR=0).
bool tc_pair_enabled() {
    const char *e = getenv("CREST_TC_PAIR");
    return !(e && e[0] == '0');
}

int tc_fold_stages() {
    const char *e = getenv("CREST_TC_FOLD");
    int v = e ? atoi(e) : 128 / kStageCells;
    return v < 1 ? 1 : (v > 64 ? 64 : v);
}

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
    // cell rows of d_pad genes: hi rows [0, m_pad) then lo rows [m_pad, 2 m_pad)
    CUtensorMap map;
    cuuint64_t dims[2] = {(cuuint64_t)w.d_pad, (cuuint64_t)(2 * m_pad)};
    cuuint64_t strides[1] = {(cuuint64_t)w.d_pad * 2};
    cuuint32_t box[2] = {kHalf, kStageCells};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, w.tile, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    CREST_REQUIRE(r == CUDA_SUCCESS, CREST_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    TcArgs a;
    a.d = w.d;
    a.d_pad = w.d_pad;
    a.n_stages = (int)(m_pad / kStageCells);
    a.m_pad = (int)m_pad;
    a.nb = (int)(w.d_pad / kTile);
    a.fold = tc_fold_stages();
    a.bias = t.scale ? w.shift : nullptr;  // bf16-rounded bias: the exact tile value of zeros
    a.colsum = w.colsum_chunk;
    a.n_kept = w.n_kept;
    a.G = gram;
    a.err = err;
    tc_test_hooks(a.n_stages, a.wait_ns, a.stall_stage);
    if (tc_pair_enabled() && w.gram_aux && w.d_pad % pair::kN == 0) {
        pair::Args b;
        b.d = w.d;
        b.d_pad = w.d_pad;
        b.n_stages = a.n_stages;
        b.m_pad = a.m_pad;
        b.fold = a.fold;
        b.nb = (int)(w.d_pad / pair::kN);
        b.bias = a.bias;
        b.colsum = a.colsum;
        b.n_kept = a.n_kept;
        b.G = gram;
        b.G_aux = w.gram_aux;
        b.err = err;
        b.wait_ns = a.wait_ns;
        b.stall_stage = a.stall_stage < 0 ? -1 : (a.stall_stage - a.n_stages / 2);  // in the second cell half
        const size_t smem = 1024 + (size_t)kStages * pair::kStageBytes;
        prof::Scope ps("syrk_bf16x3_tcgen05_pair", st);
        CREST_TRY(ensure_smem_attr((const void *)pair::k_syrk_pair, smem));
        const int tiles = b.nb * (b.nb + 1) / 2;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(tiles * 4), 1, 1);  // two cell halves x two CTAs per tile
        cfg.blockDim = dim3(kThreads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CREST_CUDA_TRY(cudaLaunchKernelEx(&cfg, pair::k_syrk_pair, map, b));
        return CREST_OK;
    }
    const size_t smem = 1024 + (size_t)kStages * kStageBytes;
    prof::Scope ps("syrk_bf16x3_tcgen05", st);
    CREST_TRY(ensure_smem_attr((const void *)k_syrk_bf16x3, (size_t)smem));
    const int tiles = a.nb * (a.nb + 1) / 2;
    k_syrk_bf16x3<<<tiles, kThreads, smem, st>>>(map, a);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

// gram += aux; aux = 0 (the second cell half of the CTA-pair SYRK).
__global__ void k_gram_fold(double *__restrict__ gram, double *__restrict__ aux, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = aux[i];
    if (v != 0.0) {
        gram[i] += v;
        aux[i] = 0.0;
    }
}

int gram_aux_fold(const GramWork &w, double *gram, cudaStream_t st) {
    if (!w.gram_aux || w.d == 0) return CREST_OK;
    const int64_t n = w.d * w.d;
    k_gram_fold<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(gram, w.gram_aux, n);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
