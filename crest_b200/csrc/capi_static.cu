// crest_qc_static: the QC pass of one chunk without any device allocation.
//
// Some callers cannot let a library allocate device memory on their behalf:
// a host application that hands the GPU a fixed memory budget up front and
// accounts for every byte, or a latency-sensitive loop that must not meet
// the implicit device synchronisation of cudaFree or the unbounded latency
// of a first cudaMalloc.  crest_qc (capi.cu) grows per-device buffers on
// demand; this variant runs the same kernel on a fixed scratch area that is
// part of the library image instead.
//
// Scratch: one file-scope __device__ array (kScratchBytes, about 12 MB) per
// device, carved into the chunk's entries, spans, maps and the kernel's
// outputs.  Limits: nnz <= kMaxEntries, spans (cells of the chunk) <=
// kMaxSpans, n_gene_map and n_vars <= kMaxGenes; larger chunks are rejected
// with CREST_EINVAL.  CSR chunks (indptr) only.
//
// Set-up: every call looks the array's address up on the current device
// with cudaGetSymbolAddress; the first call on a device also loads this
// file's device code there, so it should come before any stream capture the
// caller runs.  (Looking it up each time, instead of caching it, keeps the
// address right after a device reset re-creates the context.)
//
// Zero state: the per-gene accumulators are cleared with cudaMemsetAsync at
// the start of every call; everything else in the scratch is written before
// it is read.  Calls on one device share the scratch, so overlapping calls
// would race: all calls are serialised by one process-wide lock and each
// returns only after its results are back on the host.  The copies run on
// the per-thread default stream with pageable host memory and end in a
// stream synchronisation, so no call may overlap a global-mode stream
// capture on any thread.
#include <mutex>

#include "host.cuh"

namespace crest {
namespace {

constexpr int64_t kMaxEntries = int64_t(1) << 20;
constexpr int64_t kMaxSpans = int64_t(1) << 16;
constexpr int64_t kMaxGenes = int64_t(1) << 16;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// byte offsets inside the scratch
constexpr size_t kOffGenes = 0;
constexpr size_t kOffValues = kOffGenes + align256(4 * kMaxEntries);
constexpr size_t kOffSpanPtr = kOffValues + align256(4 * kMaxEntries);
constexpr size_t kOffCellMap = kOffSpanPtr + align256(8 * (kMaxSpans + 1));
constexpr size_t kOffGeneMap = kOffCellMap + align256(8 * kMaxSpans);
constexpr size_t kOffFlag = kOffGeneMap + align256(4 * kMaxGenes);
constexpr size_t kOffSpanRow = kOffFlag + align256(kMaxGenes);
constexpr size_t kOffSpanT = kOffSpanRow + align256(8 * kMaxSpans);
constexpr size_t kOffSpanN = kOffSpanT + align256(8 * kMaxSpans);
constexpr size_t kOffSpanF = kOffSpanN + align256(4 * kMaxSpans);
constexpr size_t kOffGeneN = kOffSpanF + align256(8 * kMaxSpans);
constexpr size_t kOffGeneT = kOffGeneN + align256(4 * kMaxGenes);
constexpr size_t kScratchBytes = kOffGeneT + align256(8 * kMaxGenes);

static __device__ __align__(256) unsigned char g_qc_scratch[kScratchBytes];

std::mutex g_lock;  // serialises every call (scratch and host staging)

// Host-side copies of the per-span and per-gene results (guarded by g_lock).
struct HostStage {
    int64_t row[kMaxSpans];
    double t[kMaxSpans];
    uint32_t n[kMaxSpans];
    double f[kMaxSpans];
    uint32_t gene_n[kMaxGenes];
    double gene_t[kMaxGenes];
};
HostStage g_stage;

// Device address of the scratch on the current device.  In host code the
// array's name only stands for it; a kernel must be given this address.
int scratch_base(unsigned char **out) {
    void *p = nullptr;
    CREST_CUDA_TRY(cudaGetSymbolAddress(&p, g_qc_scratch));
    CREST_REQUIRE(p != nullptr, CREST_ECUDA, "cudaGetSymbolAddress returned NULL for the QC scratch");
    *out = static_cast<unsigned char *>(p);
    return CREST_OK;
}

}  // namespace
}  // namespace crest

using namespace crest;

extern "C" int crest_qc_static(const crest_chunk *chunk, const uint8_t *flag, int64_t n_vars, double *cell_total,
                               uint32_t *cell_ngenes, double *cell_flag, int64_t n_rows, uint32_t *gene_ncells,
                               double *gene_total) {
    CREST_TRY(validate_chunk(chunk));
    CREST_TRY(check_maps(chunk, n_vars));
    CREST_REQUIRE(chunk->indptr != nullptr, CREST_EINVAL, "crest_qc_static takes CSR chunks (indptr) only");
    CREST_REQUIRE(n_vars == 0 || (flag && gene_ncells && gene_total), CREST_EINVAL, "NULL per-gene output");
    const int64_t nnz = chunk->nnz, n_spans = chunk->n_indptr - 1;
    CREST_REQUIRE(nnz <= kMaxEntries, CREST_EINVAL,
                  "crest_qc_static: chunk has %lld entries, the static scratch holds at most %lld",
                  (long long)nnz, (long long)kMaxEntries);
    CREST_REQUIRE(n_spans <= kMaxSpans, CREST_EINVAL,
                  "crest_qc_static: chunk has %lld cells, the static scratch holds at most %lld",
                  (long long)n_spans, (long long)kMaxSpans);
    CREST_REQUIRE(chunk->n_gene_map <= kMaxGenes && n_vars <= kMaxGenes, CREST_EINVAL,
                  "crest_qc_static: %lld store genes / %lld kept genes, the static scratch holds at most %lld",
                  (long long)chunk->n_gene_map, (long long)n_vars, (long long)kMaxGenes);
    CREST_TRY(require_device());
    std::lock_guard<std::mutex> lock(g_lock);
    unsigned char *b = nullptr;
    CREST_TRY(scratch_base(&b));
    cudaStream_t st = cudaStreamPerThread;

    // The chunk's spans are cells first_cell .. first_cell + n_spans - 1, so
    // their rows are one contiguous slice of cell_map; cells past its end
    // are dropped (src/kernels.rs:65-68), i.e. the slice is just shorter.
    const int64_t fc = chunk->first_cell;
    const int64_t n_map = std::max<int64_t>(0, std::min<int64_t>(n_spans, chunk->n_cell_map - fc));
    if (nnz) {
        CREST_CUDA_TRY(cudaMemcpyAsync(b + kOffGenes, chunk->genes, 4 * nnz, cudaMemcpyHostToDevice, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(b + kOffValues, chunk->values, 4 * nnz, cudaMemcpyHostToDevice, st));
    }
    CREST_CUDA_TRY(cudaMemcpyAsync(b + kOffSpanPtr, chunk->indptr, 8 * chunk->n_indptr, cudaMemcpyHostToDevice, st));
    if (n_map)
        CREST_CUDA_TRY(cudaMemcpyAsync(b + kOffCellMap, chunk->cell_map + fc, 8 * n_map, cudaMemcpyHostToDevice, st));
    if (chunk->n_gene_map)
        CREST_CUDA_TRY(cudaMemcpyAsync(b + kOffGeneMap, chunk->gene_map, 4 * chunk->n_gene_map,
                                       cudaMemcpyHostToDevice, st));
    if (n_vars) {
        CREST_CUDA_TRY(cudaMemcpyAsync(b + kOffFlag, flag, n_vars, cudaMemcpyHostToDevice, st));
        CREST_CUDA_TRY(cudaMemsetAsync(b + kOffGeneN, 0, 4 * n_vars, st));
        CREST_CUDA_TRY(cudaMemsetAsync(b + kOffGeneT, 0, 8 * n_vars, st));
    }

    DevChunk dc;
    dc.genes = reinterpret_cast<const uint32_t *>(b + kOffGenes);
    dc.values = reinterpret_cast<const float *>(b + kOffValues);
    dc.span_ptr = reinterpret_cast<const int64_t *>(b + kOffSpanPtr);
    dc.span_cell = nullptr;
    dc.base = chunk->indptr[0];
    dc.n_spans = n_spans;
    dc.first_cell = 0;  // span i reads cell_map slice entry i
    dc.cell_map = reinterpret_cast<const int64_t *>(b + kOffCellMap);
    dc.n_cell_map = n_map;
    dc.gene_map = reinterpret_cast<const int32_t *>(b + kOffGeneMap);
    dc.n_gene_map = chunk->n_gene_map;
    dc.target_sum = chunk->target_sum;
    dc.log1p = chunk->log1p ? 1 : 0;
    SpanOut so{reinterpret_cast<int64_t *>(b + kOffSpanRow), reinterpret_cast<double *>(b + kOffSpanT),
               reinterpret_cast<uint32_t *>(b + kOffSpanN), reinterpret_cast<double *>(b + kOffSpanF)};
    CREST_TRY(launch_qc(dc, reinterpret_cast<const uint8_t *>(b + kOffFlag), reinterpret_cast<uint32_t *>(b + kOffGeneN),
                        reinterpret_cast<double *>(b + kOffGeneT), &so, nullptr, st));

    HostStage &h = g_stage;
    if (n_spans) {
        CREST_CUDA_TRY(cudaMemcpyAsync(h.row, so.row, 8 * n_spans, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(h.t, so.t, 8 * n_spans, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(h.n, so.n, 4 * n_spans, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(h.f, so.f, 8 * n_spans, cudaMemcpyDeviceToHost, st));
    }
    if (n_vars) {
        CREST_CUDA_TRY(cudaMemcpyAsync(h.gene_n, b + kOffGeneN, 4 * n_vars, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(h.gene_t, b + kOffGeneT, 8 * n_vars, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    // every row is checked before anything is added: a failing call leaves
    // the caller's outputs untouched
    for (int64_t i = 0; i < n_spans; ++i)
        CREST_REQUIRE(h.row[i] < n_rows, CREST_EINVAL, "output sizes do not match the maps");
    for (int64_t i = 0; i < n_spans; ++i) {
        const int64_t r = h.row[i];
        if (r < 0) continue;
        cell_total[r] += h.t[i];
        cell_ngenes[r] += h.n[i];
        cell_flag[r] += h.f[i];
    }
    for (int64_t g = 0; g < n_vars; ++g) {
        gene_ncells[g] += h.gene_n[g];
        gene_total[g] += h.gene_t[g];
    }
    return CREST_OK;
}
