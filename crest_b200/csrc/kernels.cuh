// Launch interfaces of the CREST B200 kernels (host side).
#pragma once

#include "common.cuh"

namespace crest {

int device_sms();  // SM count of the current device (cached per device)
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per kernel, device
// and size instead of before every launch.
int ensure_smem_attr(const void *kernel, size_t bytes);

struct SpanOut {  // per-span QC results (per-chunk API)
    int64_t *row;
    double *t;
    uint32_t *n;
    double *f;
};
struct RowOut {  // per-row QC results added at the cell's row (matrix API)
    double *t;
    uint32_t *n;
    double *f;
};

int launch_qc(const DevChunk &c, const uint8_t *flag, uint32_t *gene_ncells, double *gene_total,
              const SpanOut *span, const RowOut *row, cudaStream_t st);
int launch_gene_stats(const DevChunk &c, double *out, cudaStream_t st);
// Gene-major copy of a device-resident CSR matrix (k_csc.cu): column g holds
// (cell, raw value) of its entries in [col_ptr[g], col_ptr[g + 1]); segments
// of at most 16384 entries of one gene start at seg_lo[s] (gene seg_gene[s]).
struct CscMatrix {
    DevBuf col_ptr, col_cell, col_val, seg_lo, seg_gene;
    DevBuf cell_scale;  // per store cell: its normalisation factor, or -1 when dropped
    int64_t n_segs = 0, n_genes = 0;
    void release() {
        for (auto *b : {&col_ptr, &col_cell, &col_val, &seg_lo, &seg_gene, &cell_scale}) b->release();
        n_segs = n_genes = 0;
    }
};
int build_csc(const int64_t *indptr, const uint32_t *genes, const float *values, int64_t n_cells, int64_t n_genes,
              int64_t nnz, CscMatrix &out, cudaStream_t st);
// gene_stats of a whole matrix (c: the matrix as one chunk, for its maps and
// transform) from its gene-major copy, given the per-cell kept-gene totals.
int launch_gene_stats_csc(const DevChunk &c, CscMatrix &m, const double *total, double *out, cudaStream_t st);

// Exact k nearest neighbours (self excluded) of the rows of X (n x d f32, device).
int launch_knn(const float *X, int64_t n, int d, int k, uint32_t *idx, float *dist, cudaStream_t st);
// Per (group, var) sums of the transformed values (sumsq / nnz / clip may be NULL).
int launch_group_gene_sums(const DevChunk &c, const uint32_t *group_of_row, int64_t n_vars, const double *clip,
                           double *sum, double *sumsq, double *nnz, cudaStream_t st);
// Gene-range index of a device-resident CSR matrix with rows sorted by gene
// id: off[cell * (n_ranges - 1) + b - 1] = first entry of the row (relative
// to its start) with gene >= b << log2_s, b = 1 .. n_ranges - 1.
struct RangeIndex {
    int log2_s;
    int n_ranges;
    const int32_t *off;
};
constexpr int kSweepThreads = 768;
// Builds the index; ORs into *unsorted bit 0 if some row is not sorted by
// gene, bit 1 if some row holds a gene id twice in a row.
int launch_range_index(const int64_t *indptr, const uint32_t *genes, int64_t n_cells, int log2_s, int n_ranges,
                       int32_t *off, int *unsorted, cudaStream_t st);
// Per-gene QC sums and per-row (t, n, f) of a piece whose spans are matrix
// cells first_cell + i.  Integral values only: bit 1 of *status is set
// otherwise and the results must be discarded.
int launch_qc_sweep(const DevChunk &c, const RangeIndex &ix, const uint8_t *flag, uint32_t *gene_ncells,
                    double *gene_total, const RowOut &row, int *status, cudaStream_t st);
// gene_stats of a piece given its per-span kept-gene totals.
int launch_gene_stats_sweep(const DevChunk &c, const RangeIndex &ix, const double *total, double *out,
                            cudaStream_t st);
// total[i] = sum of the kept-gene values of span i (normalisation total).
int launch_cell_totals(const DevChunk &c, double *total, cudaStream_t st);

// out row index: the cell's row, or the span index when by_span != 0
// code: per-gene HVG codes from launch_hvg_code (d = number of HVG columns)
// counter: one device word of scratch (zeroed here) for dynamic scheduling.
int launch_project(const DevChunk &c, const int32_t *code, int64_t d, const DevScale &t, const double *V, int k,
                   float *out, int by_span, unsigned int *counter, cudaStream_t st);
// code[g] (g < c.n_gene_map): -1 dropped gene, sub_map[gene_map[g]] in [0, d)
// for an HVG column, d for another kept gene.
int launch_hvg_code(const DevChunk &c, const int32_t *sub_map, int64_t n_vars, int64_t d, int32_t *code,
                    cudaStream_t st);
// Bytes of the code table of n_gene_map genes: int32 codes, then an int16
// copy (16-byte aligned, zero-padded to a multiple of 8 entries).
size_t hvg_code_bytes(int64_t n_gene_map);
__host__ __device__ inline const int16_t *codes16(const int32_t *code, int64_t n_gene_map) {
    return reinterpret_cast<const int16_t *>(code + round_up(n_gene_map, 4));
}
// Block-wide copy of the int16 codes into shared memory with 16-byte loads.
__device__ inline void copy_codes16(const int32_t *code, int64_t n_gene_map, int16_t *dst) {
    const uint4 *src = reinterpret_cast<const uint4 *>(codes16(code, n_gene_map));
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    const int64_t n = round_up(n_gene_map, 8) / 8;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) d4[j] = __ldg(src + j);
}
// Largest dynamic shared memory a kernel here asks for (bytes).
constexpr int kMaxSmem = 227 * 1024;
// Blocks of 128 entries whose loads are in flight while one is processed
// (for_entries_x4) in the densify and projection passes.
constexpr int kDensifyDepth = 1;
constexpr int kProjDepth = 1;
bool codes_in_smem(int64_t n_gene_map, int64_t d, size_t other_smem);
int launch_scale_bias(const double *mean, const double *std, double mv, int64_t d, double *bias, cudaStream_t st);

// ------------------------------------------------------------------ Gram
// One Gram tile job: the chunk's kept cells become the K dimension of a
// dense, gene-major tile T[d_pad][m_pad] (cells contiguous) that holds the
// scaled matrix restricted to the HVG columns.  FP64 keeps S itself (zero
// where nothing is stored) so the SYRK reproduces the reference's sums;
// FP32/BF16x3 hold Z = S - shift (shift = -bias, i.e. the dense scaled
// matrix), which keeps the reduced-precision products centred.
struct GramWork {
    int64_t d, d_pad;
    int64_t m_cap;          // max cells per tile (multiple of 64)
    int precision;
    void *tile;             // FP64: double; FP32: float; BF16X3: hi then lo (bf16)
    double *colsum_chunk;   // [d] FP64 column sums of S for the current tile
    int64_t *n_kept;        // [1] kept cells in the current tile
    unsigned int *counter;  // [1] next tile row to densify (dynamic scheduling)
    float *part32;          // [d_pad * d_pad] FP32 partial (FP32 / BF16X3)
    double *shift;          // [d_pad] tile value of a zero entry: bias rounded to the tile's
                            // precision, so the (repeated) zeros are stored exactly
    int *status;            // [1] bit 1: a cell holds one column twice; bit 2: a cell could not
                            // be checked (unsorted, more HVG entries than the densify queue)
    double *gram_aux;       // [d x d] BF16X3: Gram of the second cell half of each tile (CTA-pair
                            // SYRK), zero between passes; folded by gram_aux_fold
    long long *colsum_part;  // [colsum_rows x d] per-block column sums (32.32 fixed point)
    int64_t colsum_rows;
};

size_t gram_tile_bytes(int precision, int64_t d_pad, int64_t m_cap);
// Densify spans [0, c.n_spans) of a chunk (n_spans <= m_cap) into the tile
// and accumulate its colsum / kept count.
int launch_densify(const DevChunk &c, const int32_t *code, const DevScale &t, const GramWork &w,
                   cudaStream_t st);
// gram (d x d row-major, upper triangle) += T T^T of the current tile; adds
// colsum_chunk to colsum.
int launch_syrk_fold(const GramWork &w, int64_t m, const DevScale &t, double *gram, double *colsum,
                     cudaStream_t st, bool add_colsum = true);
// Non-zero error word of the tensor-core Gram pipeline -> CREST_ETIMEOUT (and cleared).
int tc_check_error();
// gram += gram_aux, gram_aux = 0: once at the end of every Gram pass.
int gram_aux_fold(const GramWork &w, double *gram, cudaStream_t st);
// shift[j] = bias[j] rounded to the tile precision (the stored value of zeros).
int launch_tile_shift(const GramWork &w, const DevScale &t, cudaStream_t st);

// ------------------------------------------------- compact HVG form (k_compact.cu)
// HVG entries of every cell of a device-resident CSR matrix, in entry order,
// in the cell's CSR slot: entry e < n[i] of cell i is (code[indptr[i] + e],
// x[indptr[i] + e]); n[i] = -1 for a dropped cell; scale[i] = target/total.
struct CompactHvg {
    int32_t *code;   // [nnz] HVG column
    float *x;        // [nnz] raw value
    int32_t *n;      // [n_cells]
    double *scale;   // [n_cells]
    int *status;     // bit 0: some cell's columns not strictly increasing; bit 1: a duplicate column
};
// Kept / HVG class byte per store gene from the code table (for the byte-class
// extract kernel; words of four genes, a multiple of four words).
size_t gene_class_words(int64_t n_gene_map);
int launch_gene_class(const int32_t *code, int64_t n_gene_map, int64_t d, uint32_t *cls, cudaStream_t st);
// One read of a whole CSR matrix (c.base == 0, CSR spans) into the compact form.
// check_order = false when every row is known to be strictly gene-sorted and
// the HVG columns increase with the gene id (the columns of every cell are
// then strictly increasing and need no check).
// known_int: every stored value is known to be an integer in [0, 2^24)
// (the per-entry integrality test of the kept totals is then skipped).
int launch_extract(const DevChunk &c, const uint32_t *cls, const int32_t *code, int64_t d, const CompactHvg &out,
                   bool check_order, cudaStream_t st, bool known_int = false);
// Exact duplicate-column check of every cell (sets bit 1 of *in.status).
int launch_dup_compact(const int64_t *indptr, int64_t n_cells, const CompactHvg &in, int64_t d, cudaStream_t st);
// Densify cells [cell0, cell0 + n) of the compact form into the Gram tile.
// colsum_pass: also add the tile's column sums there (reduced precisions);
// shift_ready: launch_tile_shift already ran for this pass.
int launch_densify_compact(const int64_t *indptr, int64_t cell0, int64_t n, const CompactHvg &in, double target_sum,
                           int log1p, const DevScale &t, const GramWork &w, cudaStream_t st,
                           double *colsum_pass = nullptr, bool shift_ready = false);
// Streamed matrices: the HVG entries of chunk c (extracted into `scratch`,
// slots as in the chunk buffer) packed into `packed` at running offsets
// off[cell]; *total is the running entry count (bit 3 of *packed.status when
// it would pass cap).
int launch_compact_pack(const DevChunk &c, const CompactHvg &scratch, const CompactHvg &packed, int64_t *off,
                        unsigned long long *total, int64_t cap, cudaStream_t st);
// out[cell_map[i]] += scores of cell i (bit-identical to launch_project);
// cell i's entries start at start[i] (indptr, or the packed offsets).
int launch_project_compact(const int64_t *indptr, int64_t n_cells, const int64_t *cell_map, const CompactHvg &in,
                           double target_sum, int log1p, const DevScale &t, const double *V, int k, int64_t d,
                           float *out, cudaStream_t st);

// ------------------------------------------------------------ eigensolver
struct EigStats {
    int iters;
    int converged;
    double residual;
};
// cov = (G - c c^T / n) / (n - 1) from the upper triangle of G; top-k
// eigenpairs (descending, clamped at 0; largest |loading| positive) and
// trace.  vals [k], vecs [d x k] row-major, total [1]: device pointers.
int eig_topk(const double *G, const double *colsum, int64_t d, int64_t n, int64_t k, double *vals, double *vecs,
             double *total, EigStats *stats, cudaStream_t st);

}  // namespace crest
