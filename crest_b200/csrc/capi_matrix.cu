// Device-resident matrix and PCA plan (layer 2 of the C ABI).
//
// The matrix is either copied to HBM once (residency DEVICE; in chunks of
// whole cells on a copy stream, the Gram pass consuming each chunk as it
// arrives) or streamed
// from host memory in fixed cell chunks through two device buffers on a copy
// stream, the copy of chunk i+1 overlapping the kernels of chunk i
// (residency HOST; the reference's out-of-core model, crest/core.py:54-62 and
// docs/memory_model.md, with device memory bounded by two chunks plus the
// accumulators).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "host.cuh"

struct crest_matrix {
    int device = 0;
    int64_t n_cells = 0, n_genes = 0, nnz = 0;
    int residency = CREST_MEM_DEVICE;
    int64_t chunk_cells = 16384;
    std::vector<int64_t> h_indptr;
    const uint32_t *h_indices = nullptr;
    const float *h_data = nullptr;
    bool registered = false;
    crest::DevBuf d_indptr, d_indices, d_data;
    cudaStream_t compute = nullptr, copy = nullptr;
    // device residency: the CSR arrays are copied in chunks of whole cells on
    // the copy stream; chunk u covers cells [up_end[u-1], up_end[u]) and is on
    // the device once up_ev[u] has completed.  up_waited: the compute stream
    // already waits for every chunk.
    std::vector<int64_t> up_end;
    std::vector<cudaEvent_t> up_ev;
    size_t up_issued = 0;  // chunks whose copies have been queued (in order)
    bool up_waited = true;
    crest::DevBuf buf_idx[2], buf_val[2];
    cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    // per-pass staging
    crest::DevBuf cell_map, gene_map, flag, sub_map, code, counter, mean, std_, bias;
    crest::DevBuf out[5];
    // gene-range index of a device-resident matrix (built on first use):
    // range_state 0 = not built, 1 = rows sorted (index valid), -1 = unsorted;
    // rows_strict: sorted with no gene id stored twice in a row
    int range_state = 0;
    bool rows_strict = false;
    int range_log2_s = 12, n_ranges = 0;
    crest::DevBuf range_off, status;
    int qc_integral = 1;  // cleared once the QC sweep meets a non-integral value
    // set once a QC sweep with every store gene mapped met only integers in
    // [0, 2^24): every stored value is then a small non-negative integer
    bool values_small_int = false;
    // per-cell kept-gene totals of a device-resident matrix for the gene_map
    // they were formed with
    crest::DevBuf totals;
    std::vector<int32_t> totals_key;
    bool totals_valid = false;
    // compact HVG form of the last Gram pass over a device-resident matrix
    // (read by the projection of the same maps); compact_off once its
    // buffers could not be allocated (the passes then read the CSR)
    crest::DevBuf cmp_code, cmp_x, cmp_n, cmp_scale, cmp_status, cls;
    bool compact_off = false, cmp_valid = false;
    // streamed matrices: the compact form packed at running offsets (cmp_off)
    // through a chunk-sized scratch; cmp_packed marks that layout
    crest::DevBuf cmp_off, cmp_sc, cmp_sx, cmp_total;
    bool cmp_packed = false;
    int64_t cmp_cap = 0;
    std::vector<int64_t> cmp_cell_map;
    std::vector<int32_t> cmp_gene_map, cmp_sub_map;
    double cmp_target = 0.0;
    int64_t cmp_d = -1;
    // gene-major copy of a device-resident matrix for per-gene statistics
    // (built on first use; csc_state -1 once it could not be built)
    crest::CscMatrix csc;
    int csc_state = 0;
};

struct crest_pca {
    int device = 0;
    int64_t d = 0, k = 0, n = 0;
    int precision = CREST_GRAM_BF16X3;
    crest::DevBuf gram, colsum, vals, vecs, total, shift, xbuf;
    crest::GramBufs gb;
    crest::GramWork w;
    crest_pca_stats stats;
};

namespace crest {
namespace {

constexpr int64_t kUploadCells = 131072;  // cells per upload chunk (a multiple of the Gram tile)

// Queue the copies of upload chunks [up_issued, upto).  Chunks are queued a
// little ahead of their use rather than all at matrix creation: copies from
// pageable memory made later (the maps of a pass) then do not wait behind
// the whole matrix on the copy engine.
int issue_uploads(crest_matrix *m, size_t upto) {
    upto = std::min(upto, m->up_ev.size());
    for (; m->up_issued < upto; ++m->up_issued) {
        const size_t u = m->up_issued;
        const int64_t c0 = u ? m->up_end[u - 1] : 0, c1 = m->up_end[u];
        const int64_t e0 = m->h_indptr[c0], e1 = m->h_indptr[c1];
        if (e1 > e0) {
            CREST_CUDA_TRY(cudaMemcpyAsync(m->d_indices.as<uint32_t>() + e0, m->h_indices + e0, 4 * (size_t)(e1 - e0),
                                           cudaMemcpyHostToDevice, m->copy));
            CREST_CUDA_TRY(cudaMemcpyAsync(m->d_data.as<float>() + e0, m->h_data + e0, 4 * (size_t)(e1 - e0),
                                           cudaMemcpyHostToDevice, m->copy));
        }
        CREST_CUDA_TRY(cudaEventRecord(m->up_ev[u], m->copy));
    }
    return CREST_OK;
}

// The compute stream waits for every upload chunk (once per matrix).
int wait_upload(crest_matrix *m) {
    if (m->up_waited || m->up_ev.empty()) return CREST_OK;
    CREST_TRY(issue_uploads(m, m->up_ev.size()));
    CREST_CUDA_TRY(cudaStreamWaitEvent(m->compute, m->up_ev.back(), 0));
    m->up_waited = true;
    return CREST_OK;
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t st;
    explicit Timer(cudaStream_t s) : st(s) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, st);
    }
    double stop() {
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
    ~Timer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

int bind_device(int dev) {
    CREST_TRY(require_device());
    CREST_CUDA_TRY(cudaSetDevice(dev));
    return CREST_OK;
}

// Stage cell_map (n_cells) and gene_map (n_genes) of one pass; every mapped
// row must be < n_rows and every mapped var < n_vars (outputs are sized so).
int stage_maps(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map, int64_t n_rows = -1,
               int64_t n_vars = -1) {
    CREST_REQUIRE(cell_map && gene_map, CREST_EINVAL, "cell_map / gene_map are NULL");
    if (n_rows >= 0)
        for (int64_t i = 0; i < m->n_cells; ++i)
            CREST_REQUIRE(cell_map[i] < n_rows, CREST_EINVAL, "cell_map holds row %lld but n_rows is %lld",
                          (long long)cell_map[i], (long long)n_rows);
    if (n_vars >= 0)
        for (int64_t i = 0; i < m->n_genes; ++i)
            CREST_REQUIRE(gene_map[i] < n_vars, CREST_EINVAL, "gene_map holds var %d but n_vars is %lld",
                          (int)gene_map[i], (long long)n_vars);
    CREST_TRY(upload(m->cell_map, cell_map, m->n_cells, m->compute));
    CREST_TRY(upload(m->gene_map, gene_map, m->n_genes, m->compute));
    return CREST_OK;
}

DevChunk base_chunk(crest_matrix *m, double target_sum, int log1p) {
    DevChunk c;
    c.genes = nullptr;
    c.values = nullptr;
    c.span_ptr = m->d_indptr.as<int64_t>();
    c.span_cell = nullptr;
    c.base = 0;
    c.n_spans = 0;
    c.first_cell = 0;
    c.cell_map = m->cell_map.as<int64_t>();
    c.n_cell_map = m->n_cells;
    c.gene_map = m->gene_map.as<int32_t>();
    c.n_gene_map = m->n_genes;
    c.target_sum = target_sum;
    c.log1p = log1p ? 1 : 0;
    return c;
}

// Run fn(chunk) over consecutive cell pieces of at most max_cells cells on
// the compute stream.  Streaming residency copies each piece's entries into
// one of two device buffers on the copy stream first.
template <class F>
int for_each_piece(crest_matrix *m, const DevChunk &proto, int64_t max_cells, F &&fn) {
    const int64_t n = m->n_cells;
    if (m->residency == CREST_MEM_DEVICE) {
        for (int64_t s0 = 0; s0 < n; s0 += max_cells) {
            DevChunk c = proto;
            c.genes = m->d_indices.as<uint32_t>();
            c.values = m->d_data.as<float>();
            c.span_ptr = m->d_indptr.as<int64_t>() + s0;
            c.first_cell = (uint32_t)s0;
            c.base = 0;
            c.n_spans = std::min(max_cells, n - s0);
            CREST_TRY(fn(c));
        }
        return CREST_OK;
    }
    const int64_t piece = std::min(max_cells, m->chunk_cells);
    int slot = 0;
    for (int64_t s0 = 0; s0 < n; s0 += piece, slot ^= 1) {
        const int64_t s1 = std::min(n, s0 + piece);
        const int64_t e0 = m->h_indptr[s0], e1 = m->h_indptr[s1];
        const size_t ne = (size_t)(e1 - e0);
        CREST_TRY(m->buf_idx[slot].ensure(4 * std::max<size_t>(ne, 1)));
        CREST_TRY(m->buf_val[slot].ensure(4 * std::max<size_t>(ne, 1)));
        // the buffer is free once the kernels that read it last have finished
        CREST_CUDA_TRY(cudaStreamWaitEvent(m->copy, m->ev_free[slot], 0));
        if (ne) {
            CREST_CUDA_TRY(cudaMemcpyAsync(m->buf_idx[slot].ptr, m->h_indices + e0, 4 * ne, cudaMemcpyHostToDevice,
                                           m->copy));
            CREST_CUDA_TRY(cudaMemcpyAsync(m->buf_val[slot].ptr, m->h_data + e0, 4 * ne, cudaMemcpyHostToDevice,
                                           m->copy));
        }
        CREST_CUDA_TRY(cudaEventRecord(m->ev_ready[slot], m->copy));
        CREST_CUDA_TRY(cudaStreamWaitEvent(m->compute, m->ev_ready[slot], 0));
        DevChunk c = proto;
        c.genes = m->buf_idx[slot].as<uint32_t>();
        c.values = m->buf_val[slot].as<float>();
        c.span_ptr = m->d_indptr.as<int64_t>() + s0;
        c.first_cell = (uint32_t)s0;
        c.base = e0;
        c.n_spans = s1 - s0;
        CREST_TRY(fn(c));
        CREST_CUDA_TRY(cudaEventRecord(m->ev_free[slot], m->compute));
    }
    return CREST_OK;
}

// The gene-range index of a device-resident matrix, built on first use;
// false when the matrix is streamed or has a row that is not sorted.
int range_index(crest_matrix *m, RangeIndex &ix, bool &ok) {
    ok = false;
    if (m->residency != CREST_MEM_DEVICE || m->n_cells == 0 || m->n_genes == 0) return CREST_OK;
    if (m->range_state == 0) {
        const int R = (int)std::max<int64_t>(2, ceil_div(m->n_genes, (int64_t)1 << m->range_log2_s));
        CREST_TRY(m->range_off.ensure((size_t)m->n_cells * (R - 1) * sizeof(int32_t)));
        CREST_TRY(m->status.ensure(sizeof(int)));
        CREST_CUDA_TRY(cudaMemsetAsync(m->status.ptr, 0, sizeof(int), m->compute));
        CREST_TRY(launch_range_index(m->d_indptr.as<int64_t>(), m->d_indices.as<uint32_t>(), m->n_cells,
                                     m->range_log2_s, R, m->range_off.as<int32_t>(), m->status.as<int>(),
                                     m->compute));
        int unsorted = 0;
        CREST_CUDA_TRY(cudaMemcpyAsync(&unsorted, m->status.ptr, sizeof(int), cudaMemcpyDeviceToHost, m->compute));
        CREST_CUDA_TRY(cudaStreamSynchronize(m->compute));
        m->n_ranges = R;
        m->range_state = (unsorted & 1) ? -1 : 1;
        m->rows_strict = unsorted == 0;
        if (unsorted & 1) m->range_off.release();
    }
    if (m->range_state != 1) return CREST_OK;
    ix.log2_s = m->range_log2_s;
    ix.n_ranges = m->n_ranges;
    ix.off = m->range_off.as<int32_t>();
    ok = true;
    return CREST_OK;
}

// The gene-major copy of a device-resident matrix, built on first use;
// false when the matrix is streamed, the copy does not fit, or
// CREST_GENE_MAJOR=0 (then the per-gene passes use the gene-range sweep or
// the entry-parallel kernels).
int gene_major(crest_matrix *m, bool &ok) {
    ok = false;
    if (m->residency != CREST_MEM_DEVICE || m->n_cells == 0 || m->n_genes == 0 || m->csc_state < 0) return CREST_OK;
    const char *e = getenv("CREST_GENE_MAJOR");
    if (e && e[0] == '0') return CREST_OK;
    if (m->csc_state == 0) {
        const int rc = build_csc(m->d_indptr.as<int64_t>(), m->d_indices.as<uint32_t>(), m->d_data.as<float>(),
                                 m->n_cells, m->n_genes, m->nnz, m->csc, m->compute);
        if (rc == CREST_ENOMEM || rc == CREST_EINVAL) {  // no room / unsupported shape: keep the CSR passes
            m->csc.release();
            cudaGetLastError();
            m->csc_state = -1;
            return CREST_OK;
        }
        CREST_TRY(rc);
        m->csc_state = 1;
    }
    ok = true;
    return CREST_OK;
}

// Per-cell kept-gene totals of a device-resident matrix for the staged
// gene_map (cached until the map changes).
int cell_totals(crest_matrix *m, const int32_t *gene_map, const DevChunk &proto, const double **out) {
    const bool same = m->totals_valid && m->totals_key.size() == (size_t)m->n_genes &&
                      std::equal(m->totals_key.begin(), m->totals_key.end(), gene_map);
    if (!same) {
        m->totals_valid = false;
        CREST_TRY(m->totals.ensure(sizeof(double) * std::max<int64_t>(m->n_cells, 1)));
        DevChunk c = proto;
        c.genes = m->d_indices.as<uint32_t>();
        c.values = m->d_data.as<float>();
        c.first_cell = 0;
        c.base = 0;
        c.n_spans = m->n_cells;
        CREST_TRY(launch_cell_totals(c, m->totals.as<double>(), m->compute));
        m->totals_key.assign(gene_map, gene_map + m->n_genes);
        m->totals_valid = true;
    }
    *out = m->totals.as<double>();
    return CREST_OK;
}

CompactHvg compact_view(crest_matrix *m) {
    return CompactHvg{m->cmp_code.as<int32_t>(), m->cmp_x.as<float>(), m->cmp_n.as<int32_t>(),
                      m->cmp_scale.as<double>(), m->cmp_status.as<int>()};
}

void compact_release(crest_matrix *m) {
    for (auto *b : {&m->cmp_code, &m->cmp_x, &m->cmp_n, &m->cmp_scale, &m->cmp_status, &m->cls, &m->cmp_off,
                    &m->cmp_sc, &m->cmp_sx, &m->cmp_total})
        b->release();
    m->cmp_valid = false;
}

// Buffers of the packed compact form of a streamed matrix: room for a
// quarter of the stored entries (HVG entries are about one in eight for
// 2,000 of 30,000+ genes); compact_off when they do not fit.
int streamed_compact_prepare(crest_matrix *m, int64_t d, bool &ok, cudaStream_t st) {
    ok = false;
    m->cmp_valid = false;
    if (m->residency != CREST_MEM_HOST || m->compact_off || m->n_cells == 0) return CREST_OK;
    if (4 * gene_class_words(std::max<int64_t>(m->n_genes, 1)) > (size_t)kMaxSmem) return CREST_OK;
    const char *e = getenv("CREST_STREAM_COMPACT");  // 0: the projection streams the CSR again
    if (e && e[0] == '0') return CREST_OK;
    int64_t piece_max = 1;
    for (int64_t s0 = 0; s0 < m->n_cells; s0 += m->chunk_cells) {
        const int64_t s1 = std::min(m->n_cells, s0 + m->chunk_cells);
        piece_max = std::max(piece_max, m->h_indptr[s1] - m->h_indptr[s0]);
    }
    m->cmp_cap = m->nnz / 4 + 1024;
    const size_t n = (size_t)m->n_cells;
    if (m->cmp_code.ensure(4 * (size_t)m->cmp_cap) || m->cmp_x.ensure(4 * (size_t)m->cmp_cap) ||
        m->cmp_n.ensure(4 * n) || m->cmp_scale.ensure(8 * n) || m->cmp_off.ensure(8 * n) ||
        m->cmp_status.ensure(sizeof(int)) || m->cmp_total.ensure(8) || m->cmp_sc.ensure(4 * (size_t)piece_max) ||
        m->cmp_sx.ensure(4 * (size_t)piece_max) || m->cls.ensure(4 * gene_class_words(std::max<int64_t>(m->n_genes, 1)))) {
        compact_release(m);
        cudaGetLastError();
        m->compact_off = true;
        return CREST_OK;
    }
    CREST_TRY(launch_gene_class(m->code.as<int32_t>(), m->n_genes, d, m->cls.as<uint32_t>(), st));
    CREST_CUDA_TRY(cudaMemsetAsync(m->cmp_status.ptr, 0, sizeof(int), st));
    CREST_CUDA_TRY(cudaMemsetAsync(m->cmp_total.ptr, 0, 8, st));
    ok = true;
    return CREST_OK;
}

// One streamed chunk: its compact form into the scratch, then packed.
int streamed_compact_chunk(crest_matrix *m, const DevChunk &c, int64_t d, cudaStream_t st) {
    const CompactHvg scratch{m->cmp_sc.as<int32_t>(), m->cmp_sx.as<float>(), m->cmp_n.as<int32_t>(),
                             m->cmp_scale.as<double>(), m->cmp_status.as<int>()};
    CREST_TRY(launch_extract(c, m->cls.as<uint32_t>(), m->code.as<int32_t>(), d, scratch, true, st));
    return launch_compact_pack(c, scratch, compact_view(m), m->cmp_off.as<int64_t>(),
                               m->cmp_total.as<unsigned long long>(), m->cmp_cap, st);
}

// One read of the device-resident CSR into the compact HVG form (k_extract);
// done = false when the matrix is streamed or the buffers do not fit, in
// which case the Gram and projection passes read the CSR themselves.
int compact_pass(crest_matrix *m, const DevChunk &proto, int64_t d, bool &done, cudaStream_t st) {
    done = false;
    m->cmp_valid = false;
    if (m->residency != CREST_MEM_DEVICE || m->compact_off || m->n_cells == 0) return CREST_OK;
    // the extract kernel keeps one class byte per gene in shared memory
    if (4 * gene_class_words(std::max<int64_t>(m->n_genes, 1)) > (size_t)kMaxSmem) return CREST_OK;
    const size_t nnz = (size_t)std::max<int64_t>(m->nnz, 1), n = (size_t)m->n_cells;
    if (m->cmp_code.ensure(4 * nnz) || m->cmp_x.ensure(4 * nnz) || m->cmp_n.ensure(4 * n) ||
        m->cmp_scale.ensure(8 * n) || m->cmp_status.ensure(sizeof(int)) ||
        m->cls.ensure(4 * gene_class_words(std::max<int64_t>(m->n_genes, 1)))) {
        compact_release(m);
    m->csc.release();
        cudaGetLastError();
        m->compact_off = true;
        return CREST_OK;
    }
    CREST_TRY(launch_gene_class(m->code.as<int32_t>(), m->n_genes, d, m->cls.as<uint32_t>(), st));
    CREST_CUDA_TRY(cudaMemsetAsync(m->cmp_status.ptr, 0, sizeof(int), st));
    done = true;
    return CREST_OK;
}

// Compact form of cells [c0, c1) (after compact_pass), once the upload
// chunk(s) holding them are on the device.
int compact_extract(crest_matrix *m, const DevChunk &proto, int64_t d, int64_t c0, int64_t c1, bool check_order,
                    cudaStream_t st) {
    DevChunk c = proto;
    c.genes = m->d_indices.as<uint32_t>();
    c.values = m->d_data.as<float>();
    c.span_ptr = m->d_indptr.as<int64_t>() + c0;
    c.first_cell = (uint32_t)c0;
    c.base = 0;
    c.n_spans = c1 - c0;
    return launch_extract(c, m->cls.as<uint32_t>(), m->code.as<int32_t>(), d, compact_view(m), check_order, st,
                          m->values_small_int);
}

// True when the HVG column of a store gene (sub_map[gene_map[g]], as
// launch_hvg_code forms it) strictly increases with g over the HVG genes.
bool columns_monotone(const int32_t *gene_map, int64_t n_genes, const int32_t *sub_map, int64_t n_vars) {
    int32_t last = -1;
    for (int64_t g = 0; g < n_genes; ++g) {
        const int32_t k = gene_map[g];
        if (k < 0 || k >= n_vars || sub_map[k] < 0) continue;
        if (sub_map[k] <= last) return false;
        last = sub_map[k];
    }
    return true;
}

// Duplicate-column check of the compact form: only cells whose columns were
// not strictly increasing need the exact search.
int compact_dup_check(crest_matrix *m, int64_t d, cudaStream_t st) {
    int h = 0;
    CREST_CUDA_TRY(cudaMemcpyAsync(&h, m->cmp_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    if (!(h & 1)) return CREST_OK;
    CREST_TRY(launch_dup_compact(m->d_indptr.as<int64_t>(), m->n_cells, compact_view(m), d, st));
    CREST_CUDA_TRY(cudaMemcpyAsync(&h, m->cmp_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    CREST_REQUIRE(!(h & 2), CREST_EINVAL,
                  "a cell holds the same HVG column twice (duplicate (cell, gene) entries): the dense Gram tile "
                  "cannot represent the reference's pairwise sum; merge duplicates first");
    return CREST_OK;
}

bool compact_matches(const crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map, const int32_t *sub_map,
                     int64_t n_vars, double target_sum, int64_t d) {
    return m->cmp_valid && m->cmp_d == d && m->cmp_target == target_sum &&
           m->cmp_sub_map.size() == (size_t)n_vars &&
           std::equal(m->cmp_cell_map.begin(), m->cmp_cell_map.end(), cell_map) &&
           std::equal(m->cmp_gene_map.begin(), m->cmp_gene_map.end(), gene_map) &&
           std::equal(m->cmp_sub_map.begin(), m->cmp_sub_map.end(), sub_map);
}

// shift[j] = sum_a (colsum[a] / n) V[a][j] (crest/tl.py:72-76): one block per
// component, each thread a strided partial sum, then a block reduction.
__global__ void __launch_bounds__(256) k_init_scores(const double *__restrict__ colsum, const double *__restrict__ V,
                                                     int64_t d, int64_t k, double n, double *__restrict__ shift) {
    __shared__ double part[8];
    const int64_t j = blockIdx.x;
    double s = 0.0;
    for (int64_t a = threadIdx.x; a < d; a += blockDim.x) s += (colsum[a] / n) * V[a * k + j];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        shift[j] = t;
    }
}

__global__ void k_fill_scores(const double *__restrict__ shift, int64_t n_rows, int64_t k, float *__restrict__ X) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n_rows * k) return;
    X[idx] = -__double2float_rn(shift[idx % k]);
}

}  // namespace
}  // namespace crest

using namespace crest;

extern "C" {

int crest_matrix_create(crest_matrix **out, const int64_t *indptr, const uint32_t *indices, const float *data,
                        int64_t n_cells, int64_t n_genes, int32_t residency, int64_t chunk_cells) {
    CREST_REQUIRE(out, CREST_EINVAL, "out is NULL");
    *out = nullptr;
    CREST_REQUIRE(indptr && n_cells >= 0 && n_genes >= 0, CREST_EINVAL, "invalid matrix shape");
    CREST_REQUIRE(indptr[0] == 0, CREST_EINVAL, "indptr[0] must be 0");
    for (int64_t i = 0; i < n_cells; ++i)
        CREST_REQUIRE(indptr[i] <= indptr[i + 1], CREST_EINVAL, "indptr must be non-decreasing");
    const int64_t nnz = indptr[n_cells];
    CREST_REQUIRE(nnz == 0 || (indices && data), CREST_EINVAL, "indices / data are NULL");
    CREST_REQUIRE(residency == CREST_MEM_DEVICE || residency == CREST_MEM_HOST, CREST_EINVAL, "bad residency");
    CREST_TRY(require_device());
    crest_matrix *m = new crest_matrix();
    cudaGetDevice(&m->device);
    m->n_cells = n_cells;
    m->n_genes = n_genes;
    m->nnz = nnz;
    m->residency = residency;
    m->chunk_cells = chunk_cells > 0 ? chunk_cells : 16384;
    m->h_indptr.assign(indptr, indptr + n_cells + 1);
    auto fail = [&](int rc) {
        crest_matrix_free(m);
        return rc;
    };
    if (cudaStreamCreateWithFlags(&m->compute, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&m->copy, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("stream creation failed");
        return fail(CREST_ECUDA);
    }
    for (int i = 0; i < 2; ++i) {
        cudaEventCreateWithFlags(&m->ev_ready[i], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&m->ev_free[i], cudaEventDisableTiming);
    }
    int rc = upload(m->d_indptr, indptr, n_cells + 1, m->compute);
    if (rc) return fail(rc);
    if (residency == CREST_MEM_DEVICE) {
        // chunked copies on the copy stream, left running: the Gram pass
        // extracts each chunk as soon as it has arrived (the caller's arrays
        // must stay valid until the first operation on the matrix returns)
        rc = m->d_indices.ensure(4 * (size_t)std::max<int64_t>(nnz, 1));
        if (!rc) rc = m->d_data.ensure(4 * (size_t)std::max<int64_t>(nnz, 1));
        if (rc) return fail(rc);
        m->h_indices = indices;
        m->h_data = data;
        for (int64_t c0 = 0; c0 < n_cells || (c0 == 0 && n_cells == 0); c0 += kUploadCells) {
            cudaEvent_t ev = nullptr;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
                set_error("matrix upload failed: %s", cudaGetErrorString(cudaGetLastError()));
                return fail(CREST_ECUDA);
            }
            m->up_ev.push_back(ev);
            m->up_end.push_back(std::min(n_cells, c0 + kUploadCells));
            if (n_cells == 0) break;
        }
        m->up_waited = false;
        rc = issue_uploads(m, 1);  // the first chunk now, the rest as passes consume them
        if (rc) return fail(rc);
    } else {
        m->h_indices = indices;
        m->h_data = data;
        // pin the caller's buffers when they are not pinned already
        cudaPointerAttributes at;
        if (nnz > 0 && cudaPointerGetAttributes(&at, indices) == cudaSuccess && at.type == cudaMemoryTypeUnregistered) {
            if (cudaHostRegister((void *)indices, 4 * (size_t)nnz, cudaHostRegisterReadOnly) == cudaSuccess &&
                cudaHostRegister((void *)data, 4 * (size_t)nnz, cudaHostRegisterReadOnly) == cudaSuccess)
                m->registered = true;
            cudaGetLastError();
        }
        cudaGetLastError();
    }
    if (cudaStreamSynchronize(m->compute) != cudaSuccess) {
        set_error("matrix upload failed: %s", cudaGetErrorString(cudaGetLastError()));
        return fail(CREST_ECUDA);
    }
    *out = m;
    return CREST_OK;
}

int crest_matrix_free(crest_matrix *m) {
    if (!m) return CREST_OK;
    cudaSetDevice(m->device);
    if (m->compute) cudaStreamSynchronize(m->compute);
    if (m->copy) cudaStreamSynchronize(m->copy);
    if (m->registered) {
        cudaHostUnregister((void *)m->h_indices);
        cudaHostUnregister((void *)m->h_data);
    }
    m->d_indptr.release();
    m->d_indices.release();
    m->d_data.release();
    for (int i = 0; i < 2; ++i) {
        m->buf_idx[i].release();
        m->buf_val[i].release();
        if (m->ev_ready[i]) cudaEventDestroy(m->ev_ready[i]);
        if (m->ev_free[i]) cudaEventDestroy(m->ev_free[i]);
    }
    for (cudaEvent_t ev : m->up_ev) cudaEventDestroy(ev);
    m->up_ev.clear();
    for (auto *b : {&m->cell_map, &m->gene_map, &m->flag, &m->sub_map, &m->mean, &m->std_, &m->bias, &m->range_off,
                    &m->status, &m->totals})
        b->release();
    compact_release(m);
    for (auto &b : m->out) b.release();
    if (m->compute) cudaStreamDestroy(m->compute);
    if (m->copy) cudaStreamDestroy(m->copy);
    delete m;
    return CREST_OK;
}

int crest_matrix_info(const crest_matrix *m, int64_t *n_cells, int64_t *n_genes, int64_t *nnz) {
    CREST_REQUIRE(m, CREST_EINVAL, "matrix is NULL");
    if (n_cells) *n_cells = m->n_cells;
    if (n_genes) *n_genes = m->n_genes;
    if (nnz) *nnz = m->nnz;
    return CREST_OK;
}

int crest_matrix_qc(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map, const uint8_t *flag,
                    int64_t n_rows, int64_t n_vars, double *cell_total, uint32_t *cell_ngenes, double *cell_flag,
                    uint32_t *gene_ncells, double *gene_total) {
    CREST_REQUIRE(m, CREST_EINVAL, "matrix is NULL");
    CREST_TRY(bind_device(m->device));
    CREST_TRY(wait_upload(m));
    CREST_TRY(stage_maps(m, cell_map, gene_map, n_rows, n_vars));
    cudaStream_t st = m->compute;
    CREST_TRY(upload(m->flag, flag, n_vars, st));
    CREST_TRY(zeros<double>(m->out[0], n_rows, st));
    CREST_TRY(zeros<uint32_t>(m->out[1], n_rows, st));
    CREST_TRY(zeros<double>(m->out[2], n_rows, st));
    CREST_TRY(zeros<uint32_t>(m->out[3], n_vars, st));
    CREST_TRY(zeros<double>(m->out[4], n_vars, st));
    RowOut ro{m->out[0].as<double>(), m->out[1].as<uint32_t>(), m->out[2].as<double>()};
    const DevChunk proto = base_chunk(m, 0.0, 0);
    RangeIndex ix;
    bool swept = false;
    CREST_TRY(range_index(m, ix, swept));
    swept = swept && m->qc_integral;
    if (swept) {  // gene-range sweep over the whole resident matrix
        DevChunk c = proto;
        c.genes = m->d_indices.as<uint32_t>();
        c.values = m->d_data.as<float>();
        c.n_spans = m->n_cells;
        CREST_CUDA_TRY(cudaMemsetAsync(m->status.ptr, 0, sizeof(int), st));
        CREST_TRY(launch_qc_sweep(c, ix, m->flag.as<uint8_t>(), m->out[3].as<uint32_t>(), m->out[4].as<double>(),
                                  ro, m->status.as<int>(), st));
        int status = 0;
        CREST_CUDA_TRY(cudaMemcpyAsync(&status, m->status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaStreamSynchronize(st));
        // the sweep visits the mapped cells' entries of mapped genes only
        if (!status && std::all_of(gene_map, gene_map + m->n_genes, [](int32_t g) { return g >= 0; }) &&
            std::all_of(cell_map, cell_map + m->n_cells, [](int64_t r) { return r >= 0; }))
            m->values_small_int = true;
        if (status) {  // a non-integral value: redo in entry order
            m->qc_integral = 0;
            swept = false;
            CREST_TRY(zeros<double>(m->out[0], n_rows, st));
            CREST_TRY(zeros<uint32_t>(m->out[1], n_rows, st));
            CREST_TRY(zeros<double>(m->out[2], n_rows, st));
            CREST_TRY(zeros<uint32_t>(m->out[3], n_vars, st));
            CREST_TRY(zeros<double>(m->out[4], n_vars, st));
        }
    }
    if (!swept)
        CREST_TRY(for_each_piece(m, proto, m->n_cells, [&](const DevChunk &c) {
            return launch_qc(c, m->flag.as<uint8_t>(), m->out[3].as<uint32_t>(), m->out[4].as<double>(), nullptr, &ro,
                             st);
        }));
    if (n_rows) {
        CREST_CUDA_TRY(cudaMemcpyAsync(cell_total, m->out[0].ptr, 8 * n_rows, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(cell_ngenes, m->out[1].ptr, 4 * n_rows, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(cell_flag, m->out[2].ptr, 8 * n_rows, cudaMemcpyDeviceToHost, st));
    }
    if (n_vars) {
        CREST_CUDA_TRY(cudaMemcpyAsync(gene_ncells, m->out[3].ptr, 4 * n_vars, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(gene_total, m->out[4].ptr, 8 * n_vars, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    return CREST_OK;
}

int crest_matrix_gene_stats(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map, double target_sum,
                            int32_t log1p, int64_t n_vars, double *out) {
    CREST_REQUIRE(m && out, CREST_EINVAL, "NULL argument");
    CREST_TRY(bind_device(m->device));
    CREST_TRY(wait_upload(m));
    CREST_TRY(stage_maps(m, cell_map, gene_map, -1, n_vars));
    cudaStream_t st = m->compute;
    CREST_TRY(zeros<double>(m->out[0], n_vars * 5, st));
    const DevChunk proto = base_chunk(m, target_sum, log1p);
    RangeIndex ix;
    bool swept = false;
    CREST_TRY(range_index(m, ix, swept));
    bool by_gene = false;
    CREST_TRY(gene_major(m, by_gene));
    if (by_gene) {  // segmented reductions over the gene-major copy
        const double *total = nullptr;
        if (target_sum > 0.0) CREST_TRY(cell_totals(m, gene_map, proto, &total));
        DevChunk c = proto;
        c.n_spans = m->n_cells;
        CREST_TRY(launch_gene_stats_csc(c, m->csc, total, m->out[0].as<double>(), st));
    } else if (swept) {  // gene-range sweep over the whole resident matrix
        const double *total = nullptr;
        if (target_sum > 0.0) CREST_TRY(cell_totals(m, gene_map, proto, &total));
        DevChunk c = proto;
        c.genes = m->d_indices.as<uint32_t>();
        c.values = m->d_data.as<float>();
        c.n_spans = m->n_cells;
        CREST_TRY(launch_gene_stats_sweep(c, ix, total, m->out[0].as<double>(), st));
    } else {
        CREST_TRY(for_each_piece(m, proto, m->n_cells,
                                 [&](const DevChunk &c) { return launch_gene_stats(c, m->out[0].as<double>(), st); }));
    }
    if (n_vars) CREST_CUDA_TRY(cudaMemcpyAsync(out, m->out[0].ptr, 40 * n_vars, cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    return CREST_OK;
}

int crest_matrix_group_gene_sums(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map, double target_sum,
                                 int32_t log1p, const uint32_t *group_of_row, int64_t n_group_rows, int64_t n_groups,
                                 int64_t n_vars, const double *clip, double *sum, double *sumsq, double *nnz) {
    CREST_REQUIRE(m && sum && n_groups >= 0, CREST_EINVAL, "NULL argument");
    CREST_TRY(bind_device(m->device));
    CREST_TRY(wait_upload(m));
    int64_t n_rows = 0;
    for (int64_t i = 0; i < m->n_cells; ++i) n_rows = std::max<int64_t>(n_rows, cell_map[i] + 1);
    CREST_REQUIRE(n_group_rows >= n_rows && (n_group_rows == 0 || group_of_row), CREST_EINVAL,
                  "sum, sumsq, nnz must be (n_groups, n_vars); group_of_row (n_rows,)");
    for (int64_t r = 0; r < n_group_rows; ++r)
        CREST_REQUIRE(group_of_row[r] == 0xffffffffu || (int64_t)group_of_row[r] < n_groups, CREST_EINVAL,
                      "group id out of range");
    CREST_TRY(stage_maps(m, cell_map, gene_map, -1, n_vars));
    cudaStream_t st = m->compute;
    const int64_t ne = n_groups * n_vars;
    CREST_TRY(upload(m->out[3], group_of_row, n_group_rows, st));
    const double *dclip = nullptr;
    if (clip) {
        CREST_TRY(upload(m->out[4], clip, ne, st));
        dclip = m->out[4].as<double>();
    }
    CREST_TRY(zeros<double>(m->out[0], ne, st));
    if (sumsq) CREST_TRY(zeros<double>(m->out[1], ne, st));
    if (nnz) CREST_TRY(zeros<double>(m->out[2], ne, st));
    const DevChunk proto = base_chunk(m, target_sum, log1p);
    CREST_TRY(for_each_piece(m, proto, m->n_cells, [&](const DevChunk &c) {
        return launch_group_gene_sums(c, m->out[3].as<uint32_t>(), n_vars, dclip, m->out[0].as<double>(),
                                      sumsq ? m->out[1].as<double>() : nullptr, nnz ? m->out[2].as<double>() : nullptr,
                                      st);
    }));
    std::vector<double> h0(ne), h1(sumsq ? ne : 0), h2(nnz ? ne : 0);
    if (ne) {
        CREST_CUDA_TRY(cudaMemcpyAsync(h0.data(), m->out[0].ptr, 8 * ne, cudaMemcpyDeviceToHost, st));
        if (sumsq) CREST_CUDA_TRY(cudaMemcpyAsync(h1.data(), m->out[1].ptr, 8 * ne, cudaMemcpyDeviceToHost, st));
        if (nnz) CREST_CUDA_TRY(cudaMemcpyAsync(h2.data(), m->out[2].ptr, 8 * ne, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < ne; ++i) sum[i] += h0[i];
    for (int64_t i = 0; sumsq && i < ne; ++i) sumsq[i] += h1[i];
    for (int64_t i = 0; nnz && i < ne; ++i) nnz[i] += h2[i];
    return CREST_OK;
}

int crest_pca_create(crest_pca **out, int64_t d, int32_t precision) {
    CREST_REQUIRE(out, CREST_EINVAL, "out is NULL");
    *out = nullptr;
    CREST_REQUIRE(d >= 1, CREST_EINVAL, "need at least 1 gene");
    CREST_REQUIRE(precision >= CREST_GRAM_FP64 && precision <= CREST_GRAM_BF16X3, CREST_EINVAL,
                  "unknown Gram precision %d", precision);
    CREST_TRY(require_device());
    crest_pca *p = new crest_pca();
    cudaGetDevice(&p->device);
    p->d = d;
    p->precision = precision;
    memset(&p->stats, 0, sizeof p->stats);
    int rc = zeros<double>(p->gram, d * d, 0);
    if (!rc) rc = zeros<double>(p->colsum, d, 0);
    // a first tile; crest_pca_accumulate sizes it for the matrix it reads
    if (!rc) rc = p->gb.ensure(p->w, d, precision, std::min<int64_t>(tile_cells_default(), 16384));
    if (!rc && cudaDeviceSynchronize() != cudaSuccess) {
        set_error("PCA plan set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
        rc = CREST_ECUDA;
    }
    if (rc) {
        crest_pca_free(p);
        return rc;
    }
    *out = p;
    return CREST_OK;
}

int crest_pca_free(crest_pca *p) {
    if (!p) return CREST_OK;
    cudaSetDevice(p->device);
    cudaDeviceSynchronize();
    for (auto *b : {&p->gram, &p->colsum, &p->vals, &p->vecs, &p->total, &p->shift, &p->xbuf}) b->release();
    p->gb.tile.release();
    p->gb.colsum_chunk.release();
    p->gb.n_kept.release();
    p->gb.shift.release();
    p->gb.status.release();
    p->gb.aux.release();
    delete p;
    return CREST_OK;
}

int crest_pca_accumulate(crest_pca *p, crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map,
                         double target_sum, int32_t log1p, const int32_t *sub_map, int64_t n_vars,
                         const crest_scale *scale) {
    CREST_REQUIRE(p && m, CREST_EINVAL, "NULL plan or matrix");
    CREST_TRY(bind_device(m->device));
    for (int64_t i = 0; i < n_vars; ++i)
        CREST_REQUIRE(sub_map[i] < p->d, CREST_EINVAL, "sub_map must have length n_vars and values < d");
    cudaStream_t st = m->compute;
    Timer t(st);
    CREST_TRY(stage_maps(m, cell_map, gene_map, -1, n_vars));
    CREST_TRY(upload(m->sub_map, sub_map, n_vars, st));
    DevScale ds;
    CREST_TRY(stage_scale(m->mean, m->std_, m->bias, scale, p->d, ds, st));
    const DevChunk proto = base_chunk(m, target_sum, log1p);
    CREST_TRY(stage_hvg_code(proto, m->sub_map.as<int32_t>(), n_vars, p->d, m->code, st));
    CREST_TRY(gram_status_reset(p->w, st));
    // a resident matrix already on the device is one range of tiles; while its
    // upload is in flight the tiles follow the upload chunks
    const bool resident = m->residency == CREST_MEM_DEVICE && m->up_waited;
    {  // tiles: the default size for a resident matrix, at most one upload chunk while
       // uploading, one stored chunk of a streamed matrix
        const int64_t cap = resident ? tile_cells_default()
                            : m->residency == CREST_MEM_DEVICE ? std::min<int64_t>(tile_cells_default(), kUploadCells)
                                                               : std::min<int64_t>(tile_cells_default(), m->chunk_cells);
        CREST_TRY(p->gb.ensure(p->w, p->d, p->precision, std::min(cap, round_up(std::max<int64_t>(m->n_cells, 1), 64))));
    }
    bool compact = false;
    CREST_TRY(compact_pass(m, proto, p->d, compact, st));
    if (compact) m->cmp_packed = false;
    if (compact) {  // per upload chunk: its compact HVG form, then its Gram tiles
        const CompactHvg ch = compact_view(m);
        // the zero-entry tile value is the same for every tile of the pass;
        // the densify kernel adds each tile's column sums to the pass's
        const bool reduced = p->precision != CREST_GRAM_FP64;
        if (reduced && ds.scale) CREST_TRY(launch_tile_shift(p->w, ds, st));
        // strictly gene-sorted rows (known once the range index exists) under a
        // monotone column map give strictly increasing columns in every cell
        const bool check_order = !(m->rows_strict && columns_monotone(gene_map, m->n_genes, sub_map, n_vars));
        int64_t u0 = 0;
        const size_t n_ranges = resident ? 1 : m->up_end.size();
        for (size_t u = 0; u < n_ranges && u0 < m->n_cells; ++u) {
            const int64_t u1 = resident ? m->n_cells : m->up_end[u];
            if (!m->up_waited) {
                CREST_TRY(issue_uploads(m, u + 2));  // keep the next chunk's copy queued
                CREST_CUDA_TRY(cudaStreamWaitEvent(st, m->up_ev[u], 0));
            }
            CREST_TRY(compact_extract(m, proto, p->d, u0, u1, check_order, st));
            for (int64_t s0 = u0; s0 < u1; s0 += p->w.m_cap) {
                const int64_t n = std::min(p->w.m_cap, u1 - s0);
                CREST_TRY(launch_densify_compact(m->d_indptr.as<int64_t>(), s0, n, ch, target_sum, log1p, ds, p->w,
                                                 st, reduced ? p->colsum.as<double>() : nullptr, true));
                CREST_TRY(launch_syrk_fold(p->w, n, ds, p->gram.as<double>(), p->colsum.as<double>(), st, !reduced));
            }
            u0 = u1;
        }
        m->up_waited = true;
    } else {
        CREST_TRY(wait_upload(m));
        bool packed = false;  // streamed: also keep the packed compact form for the projection
        CREST_TRY(streamed_compact_prepare(m, p->d, packed, st));
        CREST_TRY(for_each_piece(m, proto, p->w.m_cap, [&](const DevChunk &c) {
            CREST_TRY(gram_over_chunk(c, m->code.as<int32_t>(), ds, p->w, p->gram.as<double>(),
                                      p->colsum.as<double>(), st));
            return packed ? streamed_compact_chunk(m, c, p->d, st) : CREST_OK;
        }));
        if (packed) {
            int h = 0;
            CREST_CUDA_TRY(cudaMemcpyAsync(&h, m->cmp_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
            CREST_CUDA_TRY(cudaStreamSynchronize(st));
            compact = !(h & 8);  // every cell's entries fitted: the projection reads the packed form
            m->cmp_packed = compact;
        }
    }
    CREST_TRY(gram_aux_fold(p->w, p->gram.as<double>(), st));
    p->stats.gram_ms = t.stop();
    CREST_CUDA_TRY(cudaGetLastError());
    if (compact && !m->cmp_packed) CREST_TRY(compact_dup_check(m, p->d, st));
    CREST_TRY(gram_status_check(p->w, st));
    if (p->precision == CREST_GRAM_BF16X3) CREST_TRY(tc_check_error());
    if (compact) {  // the projection of the same maps reads this form
        m->cmp_cell_map.assign(cell_map, cell_map + m->n_cells);
        m->cmp_gene_map.assign(gene_map, gene_map + m->n_genes);
        m->cmp_sub_map.assign(sub_map, sub_map + n_vars);
        m->cmp_target = target_sum;
        m->cmp_d = p->d;
        m->cmp_valid = true;
    }
    return CREST_OK;
}

int crest_pca_reset(crest_pca *p) {
    CREST_REQUIRE(p, CREST_EINVAL, "plan is NULL");
    CREST_TRY(bind_device(p->device));
    CREST_CUDA_TRY(cudaMemset(p->gram.ptr, 0, sizeof(double) * (size_t)(p->d * p->d)));
    CREST_CUDA_TRY(cudaMemset(p->colsum.ptr, 0, sizeof(double) * (size_t)p->d));
    if (p->w.gram_aux) CREST_CUDA_TRY(cudaMemset(p->w.gram_aux, 0, sizeof(double) * (size_t)(p->d * p->d)));
    p->k = 0;
    return CREST_OK;
}

int crest_pca_accumulators(crest_pca *p, double **gram_dev, double **colsum_dev) {
    CREST_REQUIRE(p, CREST_EINVAL, "plan is NULL");
    if (gram_dev) *gram_dev = p->gram.as<double>();
    if (colsum_dev) *colsum_dev = p->colsum.as<double>();
    return CREST_OK;
}

int crest_pca_gram(crest_pca *p, double *gram) {
    CREST_REQUIRE(p && gram, CREST_EINVAL, "NULL argument");
    CREST_TRY(bind_device(p->device));
    CREST_CUDA_TRY(cudaDeviceSynchronize());
    CREST_CUDA_TRY(cudaMemcpy(gram, p->gram.ptr, 8 * (size_t)(p->d * p->d), cudaMemcpyDeviceToHost));
    return CREST_OK;
}

int crest_pca_solve(crest_pca *p, int64_t n, int64_t k) {
    CREST_REQUIRE(p, CREST_EINVAL, "plan is NULL");
    CREST_REQUIRE(n >= 2, CREST_ERUNTIME, "need at least 2 cells and 1 gene");
    CREST_REQUIRE(k >= 1 && k <= p->d && k <= 128, CREST_EINVAL, "k=%lld must be in [1, min(d, 128)]", (long long)k);
    CREST_TRY(bind_device(p->device));
    cudaStream_t st = 0;
    CREST_TRY(p->vals.ensure(8 * (size_t)k));
    CREST_TRY(p->vecs.ensure(8 * (size_t)(p->d * k)));
    CREST_TRY(p->total.ensure(8));
    CREST_TRY(p->shift.ensure(8 * (size_t)k));
    Timer t(st);
    EigStats es{};
    CREST_TRY(eig_topk(p->gram.as<double>(), p->colsum.as<double>(), p->d, n, k, p->vals.as<double>(),
                       p->vecs.as<double>(), p->total.as<double>(), &es, st));
    k_init_scores<<<(unsigned)k, 256, 0, st>>>(p->colsum.as<double>(), p->vecs.as<double>(), p->d, k,
                                                           (double)n, p->shift.as<double>());
    CREST_CUDA_TRY(cudaGetLastError());
    p->stats.solve_ms = t.stop();
    p->stats.eig_iters = es.iters;
    p->stats.eig_converged = es.converged;
    p->stats.eig_residual = es.residual;
    p->k = k;
    p->n = n;
    CREST_REQUIRE(es.converged, CREST_ERUNTIME, "eigensolver did not converge (residual %.3g after %d iterations)",
                  es.residual, es.iters);
    return CREST_OK;
}

int crest_pca_results(crest_pca *p, double *variance, double *loadings, double *total, double *colsum) {
    CREST_REQUIRE(p, CREST_EINVAL, "plan is NULL");
    CREST_TRY(bind_device(p->device));
    CREST_CUDA_TRY(cudaDeviceSynchronize());  // the plan's streams may be non-blocking
    if (variance && p->k) CREST_CUDA_TRY(cudaMemcpy(variance, p->vals.ptr, 8 * p->k, cudaMemcpyDeviceToHost));
    if (loadings && p->k) CREST_CUDA_TRY(cudaMemcpy(loadings, p->vecs.ptr, 8 * p->d * p->k, cudaMemcpyDeviceToHost));
    if (total) {  // the total is reduced by crest_pca_solve; 0 before it
        *total = 0.0;
        if (p->total.ptr) CREST_CUDA_TRY(cudaMemcpy(total, p->total.ptr, 8, cudaMemcpyDeviceToHost));
    }
    if (colsum && p->d) CREST_CUDA_TRY(cudaMemcpy(colsum, p->colsum.ptr, 8 * p->d, cudaMemcpyDeviceToHost));
    return CREST_OK;
}

int crest_pca_project(crest_pca *p, crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map,
                      double target_sum, int32_t log1p, const int32_t *sub_map, int64_t n_vars,
                      const crest_scale *scale, int64_t n_rows, float *out, int32_t out_mem) {
    CREST_REQUIRE(p && m && out, CREST_EINVAL, "NULL argument");
    CREST_REQUIRE(p->k >= 1, CREST_EINVAL, "crest_pca_solve must run before crest_pca_project");
    CREST_TRY(bind_device(m->device));
    CREST_TRY(wait_upload(m));
    for (int64_t i = 0; i < n_vars; ++i)
        CREST_REQUIRE(sub_map[i] < p->d, CREST_EINVAL, "sub_map must have length n_vars and values < d");
    cudaStream_t st = m->compute;
    Timer t(st);
    CREST_TRY(stage_maps(m, cell_map, gene_map, n_rows, n_vars));
    CREST_TRY(upload(m->sub_map, sub_map, n_vars, st));
    DevScale ds;
    CREST_TRY(stage_scale(m->mean, m->std_, m->bias, scale, p->d, ds, st));
    float *X = out;
    if (out_mem != CREST_MEM_DEVICE) {
        CREST_TRY(p->xbuf.ensure(4 * (size_t)std::max<int64_t>(n_rows * p->k, 1)));
        X = p->xbuf.as<float>();
    }
    if (n_rows > 0 && p->k > 0)
        k_fill_scores<<<(unsigned)ceil_div(n_rows * p->k, 256), 256, 0, st>>>(p->shift.as<double>(), n_rows, p->k, X);
    CREST_CUDA_TRY(cudaGetLastError());
    const DevChunk proto = base_chunk(m, target_sum, log1p);
    if (compact_matches(m, cell_map, gene_map, sub_map, n_vars, target_sum, p->d)) {
        const int64_t *start = m->cmp_packed ? m->cmp_off.as<int64_t>() : m->d_indptr.as<int64_t>();
        CREST_TRY(launch_project_compact(start, m->n_cells, m->cell_map.as<int64_t>(), compact_view(m), target_sum,
                                         log1p, ds, p->vecs.as<double>(), (int)p->k, p->d, X, st));
    } else {
        CREST_TRY(stage_hvg_code(proto, m->sub_map.as<int32_t>(), n_vars, p->d, m->code, st));
        CREST_TRY(m->counter.ensure(sizeof(unsigned int)));
        CREST_TRY(for_each_piece(m, proto, m->n_cells, [&](const DevChunk &c) {
            return launch_project(c, m->code.as<int32_t>(), p->d, ds, p->vecs.as<double>(), (int)p->k, X, 0,
                                  m->counter.as<unsigned int>(), st);
        }));
    }
    if (out_mem != CREST_MEM_DEVICE && n_rows > 0 && p->k > 0)
        CREST_CUDA_TRY(cudaMemcpyAsync(out, X, 4 * (size_t)(n_rows * p->k), cudaMemcpyDeviceToHost, st));
    p->stats.project_ms = t.stop();
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

int crest_pca_stats_get(const crest_pca *p, crest_pca_stats *stats) {
    CREST_REQUIRE(p && stats, CREST_EINVAL, "NULL argument");
    *stats = p->stats;
    return CREST_OK;
}

}  // extern "C"
