/*
 * crest_gpu.h -- C ABI of the B200 (sm_100a) implementation of CREST's
 * chunked preprocessing-to-PCA path.
 *
 * Two layers:
 *
 *  1. Per-chunk entry points that mirror the reference's native module
 *     `crest.crest` (PyO3, src/py.rs).  Each takes one chunk of the raw count
 *     matrix in the reference's chunk protocol (the 9-tuple of
 *     BioFrame.iter_ctx, crest/core.py:265-278) plus the function's own
 *     arguments, and ACCUMULATES (+=) into caller-allocated outputs exactly
 *     like the reference.  Buffers live in host memory, as numpy arrays do
 *     for the reference.
 *
 *  2. A device-resident matrix + PCA plan API used by the Python package's
 *     whole-pass functions: the CSR matrix is copied to HBM once (or streamed
 *     from pinned host memory in fixed cell chunks) and accumulators stay on
 *     the GPU across chunks.
 *
 * All functions return CREST_OK (0) or a negative status; crest_last_error()
 * gives the message of the calling thread's last failure.  CREST_EINVAL is
 * what the reference raises as ValueError, CREST_ERUNTIME what it raises as
 * RuntimeError.  No function falls back to a CPU implementation: without a
 * usable CUDA device every compute entry point returns CREST_ENODEV.
 */
#ifndef CREST_GPU_H
#define CREST_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CREST_OK = 0,
    CREST_ERUNTIME = -1,   /* computation failed (reference: RuntimeError)   */
    CREST_ECUDA = -5,      /* CUDA runtime error                              */
    CREST_ENOMEM = -12,    /* device or pinned allocation failed              */
    CREST_ENODEV = -19,    /* no usable CUDA device                           */
    CREST_EINVAL = -22,    /* invalid argument (reference: ValueError)        */
    CREST_ETIMEOUT = -110  /* a bounded device wait gave up                   */
};

/* Precision of the Gram accumulation. */
enum {
    CREST_GRAM_FP64 = 0,   /* FP64 dense SYRK in the reference's summation order  */
    CREST_GRAM_FP32 = 1,   /* plain form: FP32 SYRK on CUDA cores, FP64 per chunk  */
    CREST_GRAM_BF16X3 = 2  /* product form: split-BF16 tcgen05 SYRK, FP32 in TMEM  */
};

/* Where a buffer lives. */
enum { CREST_MEM_HOST = 0, CREST_MEM_DEVICE = 1 };

/*
 * One chunk in the reference's chunk protocol (crest/core.py:265-278,
 * src/py.rs:162-189, docs/development.md "The chunk protocol"):
 *   genes u32[nnz], values f32[nnz], cell_map i64[n_store_cells],
 *   gene_map i32[n_store_genes], target_sum, log1p, and either cells u32[nnz]
 *   (COO, non-decreasing) or indptr i64[n_indptr] (CSR for cells
 *   first_cell .. first_cell + n_indptr - 2, absolute offsets).
 * Exactly one of `cells` / `indptr` is non-NULL.
 */
typedef struct crest_chunk {
    const uint32_t *genes;
    const float *values;
    int64_t nnz;
    const int64_t *cell_map;
    int64_t n_cell_map;
    const int32_t *gene_map;
    int64_t n_gene_map;
    double target_sum;
    int32_t log1p;
    const uint32_t *cells;
    const int64_t *indptr;
    int64_t n_indptr;
    uint32_t first_cell;
} crest_chunk;

/* The scale transform of crest.pp.scale (src/kernels.rs:201-219). */
typedef struct crest_scale {
    int32_t scale;        /* 0: values used as they are                         */
    const double *mean;   /* [d] per-gene log-scale mean (NULL when scale == 0)  */
    const double *std;    /* [d] per-gene std, ddof=1, zeros replaced by 1       */
    double max_value;     /* clip at +-max_value; <= 0: no clipping              */
} crest_scale;

/* Per-call timings and eigensolver diagnostics. */
typedef struct crest_pca_stats {
    double gram_ms;       /* device time of the Gram pass                         */
    double solve_ms;      /* centring + eigensolve                                */
    double project_ms;    /* projection pass                                      */
    int32_t eig_iters;    /* outer Rayleigh-Ritz iterations                       */
    int32_t eig_converged;
    double eig_residual;  /* max_i ||C v_i - l_i v_i|| / l_1 over the k pairs     */
} crest_pca_stats;

const char *crest_last_error(void);
int crest_version(void);
/* Device memory held by the library's allocations on the current device:
 * bytes in use now and the high-water mark since the last reset (reset_high
 * != 0 resets it after reading).  Buffers come from a stream-ordered pool
 * that keeps freed memory for reuse, so the driver's free-memory figure
 * does not show a call's working set. */
int crest_memory_stats(int64_t *used, int64_t *used_high, int32_t reset_high);
/* Number of CUDA devices (0 without a driver); never fails. */
int crest_device_count(void);
/* Select the device used by this thread's subsequent calls. */
int crest_set_device(int device);

/* ---------------------------------------------------------------- layer 1
 * Mirrors of the reference's per-chunk native functions.  n_rows / n_vars
 * are max(cell_map)+1 / max(gene_map)+1 as computed by src/py.rs:187-193.
 */

/* qc: src/py.rs:234-248, src/kernels.rs:164-195.  Per kept cell: total,
 * genes detected (x != 0) and total in flagged genes; per kept gene: cells
 * detected and total.  Outputs are accumulated. */
int crest_qc(const crest_chunk *chunk, const uint8_t *flag, int64_t n_vars, double *cell_total,
             uint32_t *cell_ngenes, double *cell_flag, int64_t n_rows, uint32_t *gene_ncells,
             double *gene_total);

/* group_gene_sums: src/py.rs:311-338, src/kernels.rs:388-442.  Per (group,
 * var) sum, sum of squares and count of the transformed stored values of
 * kept cells; group_of_row[row] is the group of a cell's row (0xffffffff: no
 * group), n_group_rows >= n_rows; clip (n_groups x n_vars, may be NULL) caps
 * each value first.  sum / sumsq / nnz are (n_groups x n_vars) row-major and
 * accumulated; sumsq and nnz may be NULL. */
int crest_group_gene_sums(const crest_chunk *chunk, const uint32_t *group_of_row, int64_t n_group_rows,
                          int64_t n_groups, int64_t n_vars, const double *clip, double *sum, double *sumsq,
                          double *nnz);
/* group_gene_totals: src/py.rs:340-357 (pseudobulk sums only). */
int crest_group_gene_totals(const crest_chunk *chunk, const uint32_t *group_of_row, int64_t n_group_rows,
                            int64_t n_groups, int64_t n_vars, double *sum);

/* knn_graph: src/py.rs:52-72, src/knn.rs:337-371.  k nearest neighbours of
 * every row of data (n x d f32, row-major, host), self excluded, ascending
 * Euclidean distance, ties by index; k is reduced to min(k, n - 1) (at least
 * 1 when n > 1).  indices / distances are (n x k') with k' that value.  The
 * search is exhaustive for every n (exact neighbours); d <= 128, k' <= 64. */
int crest_knn_graph(const float *data, int64_t n, int64_t d, int64_t k, uint32_t *indices, float *distances);

/* crest_qc_static: no counterpart in the reference.  Same arguments and
 * results as crest_qc, computed without allocating device memory: the
 * kernel runs on a fixed scratch array compiled into the library (about
 * 12 MB per device), for callers that must not have a library allocate (or
 * free, with its implicit device synchronisation) device memory for them.
 * Limits: CSR chunks (indptr) only, nnz <= 2^20, cells per chunk <= 2^16,
 * n_gene_map and n_vars <= 2^16; larger chunks return CREST_EINVAL.  Every
 * call looks the scratch up on the current device (cudaGetSymbolAddress);
 * the first call on a device also loads the library's device code there and
 * should precede any stream capture.  Calls are serialised process-wide
 * (they share the scratch) and return after the results are on the host;
 * they copy through pageable host memory on the per-thread default stream,
 * so no call may overlap a global-mode stream capture on any thread. */
int crest_qc_static(const crest_chunk *chunk, const uint8_t *flag, int64_t n_vars, double *cell_total,
                    uint32_t *cell_ngenes, double *cell_flag, int64_t n_rows, uint32_t *gene_ncells,
                    double *gene_total);

/* gene_stats: src/py.rs:221-232, src/kernels.rs:144-160.  out is
 * (n_vars, 5) row-major: [sum x, sum x^2, sum expm1 x, sum expm1(x)^2, nnz]. */
int crest_gene_stats(const crest_chunk *chunk, int64_t n_vars, double *out);

/* gram_accumulate: src/py.rs:270-287, src/kernels.rs:221-309.  gram (d, d)
 * row-major, upper triangle accumulated; colsum (d). */
int crest_gram_accumulate(const crest_chunk *chunk, const int32_t *sub_map, int64_t n_vars,
                          const crest_scale *scale, int64_t d, double *gram, double *colsum,
                          int32_t precision);

/* pca_from_gram: src/py.rs:386-399, src/kernels.rs:311-348.  Writes the k
 * eigenvalues (descending, clamped at 0), loadings (d, k) row-major with the
 * largest |loading| of each column positive, and the total variance.
 * k must already be min(k, d). */
int crest_pca_from_gram(const double *gram, const double *colsum, int64_t d, int64_t n, int64_t k,
                        double *variance, double *loadings, double *total, crest_pca_stats *stats);

/* project: src/py.rs:289-309, src/kernels.rs:350-371.  out[row] += S_row V
 * (FP64 accumulation, added as f32). */
int crest_project(const crest_chunk *chunk, const int32_t *sub_map, int64_t n_vars,
                  const double *loadings, int64_t d, int64_t k, const crest_scale *scale, float *out,
                  int64_t n_rows);

/* ---------------------------------------------------------------- layer 2 */
typedef struct crest_matrix crest_matrix;
typedef struct crest_pca crest_pca;

/* A CSR count matrix (cells x genes): indptr i64[n_cells+1] (indptr[0] == 0),
 * indices u32[nnz], data f32[nnz], all in host memory.
 * residency CREST_MEM_DEVICE copies it to HBM once: the copy of indices /
 * data runs asynchronously in chunks of 131,072 cells (from pinned memory it
 * overlaps the first Gram pass, which consumes each chunk as it arrives), so
 * indices and data must stay valid and unchanged until the first operation
 * on the matrix has returned (or until crest_matrix_free); indptr is copied
 * before this call returns.  CREST_MEM_HOST keeps it in (ideally pinned)
 * host memory and streams chunks of chunk_cells cells through two device
 * buffers on every pass. */
int crest_matrix_create(crest_matrix **out, const int64_t *indptr, const uint32_t *indices,
                        const float *data, int64_t n_cells, int64_t n_genes, int32_t residency,
                        int64_t chunk_cells);
int crest_matrix_free(crest_matrix *m);
int crest_matrix_info(const crest_matrix *m, int64_t *n_cells, int64_t *n_genes, int64_t *nnz);

/* Whole-matrix QC pass (crest/pp.py:25-45 loop).  Outputs in host memory,
 * overwritten (not accumulated). */
int crest_matrix_qc(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map,
                    const uint8_t *flag, int64_t n_rows, int64_t n_vars, double *cell_total,
                    uint32_t *cell_ngenes, double *cell_flag, uint32_t *gene_ncells,
                    double *gene_total);

/* Whole-matrix gene_stats pass (crest/pp.py:115-120).  out (n_vars, 5). */
int crest_matrix_gene_stats(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map,
                            double target_sum, int32_t log1p, int64_t n_vars, double *out);

/* group_gene_sums over a whole matrix (same arguments and results as
 * crest_group_gene_sums, with the matrix's cell_map / gene_map). */
int crest_matrix_group_gene_sums(crest_matrix *m, const int64_t *cell_map, const int32_t *gene_map, double target_sum,
                                 int32_t log1p, const uint32_t *group_of_row, int64_t n_group_rows, int64_t n_groups,
                                 int64_t n_vars, const double *clip, double *sum, double *sumsq, double *nnz);

/* PCA plan (crest/tl.py:37-91): Gram pass, centring + eigensolve, projection. */
int crest_pca_create(crest_pca **out, int64_t d, int32_t precision);
int crest_pca_free(crest_pca *p);
/* Gram pass over the whole matrix into the plan's device accumulators. */
int crest_pca_accumulate(crest_pca *p, crest_matrix *m, const int64_t *cell_map,
                         const int32_t *gene_map, double target_sum, int32_t log1p,
                         const int32_t *sub_map, int64_t n_vars, const crest_scale *scale);
/* Zero the plan's accumulators (start a new Gram pass). */
int crest_pca_reset(crest_pca *p);
/* Device pointers of the FP64 accumulators (gram d*d, colsum d), e.g. for
 * an all-reduce across ranks before crest_pca_solve. */
int crest_pca_accumulators(crest_pca *p, double **gram_dev, double **colsum_dev);
/* Copy of the FP64 Gram accumulator (d x d row-major, upper triangle
 * meaningful) to a host buffer: the `gram` the reference's gram_accumulate
 * leaves in the caller's array (src/py.rs:270-287). */
int crest_pca_gram(crest_pca *p, double *gram);
/* Centring + top-k eigensolve on the device; n = number of cells. */
int crest_pca_solve(crest_pca *p, int64_t n, int64_t k);
/* Results of the solve (host): variance (k), loadings (d, k), total,
 * colsum (d); any pointer may be NULL. */
int crest_pca_results(crest_pca *p, double *variance, double *loadings, double *total,
                      double *colsum);
/* Projection pass: out (n_rows, k) f32 = -shift + S V, in host or device
 * memory per out_mem. */
int crest_pca_project(crest_pca *p, crest_matrix *m, const int64_t *cell_map,
                      const int32_t *gene_map, double target_sum, int32_t log1p,
                      const int32_t *sub_map, int64_t n_vars, const crest_scale *scale,
                      int64_t n_rows, float *out, int32_t out_mem);
int crest_pca_stats_get(const crest_pca *p, crest_pca_stats *stats);

/* ------------------------------------------------------- differentiation
 * The normalise -> log1p -> scale -> project map of a CSR matrix over d
 * genes (HVG columns already selected) and its gradient, for the autograd
 * hook of the Python package.  No counterpart in the reference; the forward
 * arithmetic is its transform (src/kernels.rs:79-82, 209-219, 352-371) with
 * the normalisation written as a per-cell size factor that DIVIDES:
 *   y = x / sf[c] (f32), l = log1pf(y), s = clip((l - mean)/std) - clip(-mean/std),
 *   scores[c, :] = sum over the cell's entries of s W[g, :]  (f64 sums, f32 out).
 * All pointers are DEVICE memory of the current device: indptr i64[n+1]
 * (indptr[0] = 0), indices i32[nnz] in [0, d), values f32[nnz], size_factors
 * f32[n], W f32[d, k] row-major (1 <= k <= 128), mean/std f64[d],
 * scores f32[n, k].  A gene id outside [0, d) returns CREST_EINVAL. */
int crest_fused_forward(const int64_t *indptr, const int32_t *indices, const float *values, int64_t n,
                        int64_t d, const float *size_factors, const float *W, int64_t k,
                        const double *mean, const double *std, double max_value, float *scores);
/* Gradients of L given grad_scores = dL/dscores (f32[n, k]): grad_values
 * f32[nnz], grad_sf f32[n], grad_W f32[d, k] (all overwritten).  log1p and
 * the scaled values are recomputed, not stored by the forward. */
int crest_fused_backward(const int64_t *indptr, const int32_t *indices, const float *values, int64_t n,
                         int64_t d, const float *size_factors, const float *W, int64_t k,
                         const double *mean, const double *std, double max_value,
                         const float *grad_scores, float *grad_values, float *grad_sf, float *grad_W);

/* ---------------------------------------------------------------- timing
 * Optional per-kernel device timing with CUDA events around each launch on
 * its stream (no counterpart in the reference, which has no GPU code).
 */
int crest_profile_enable(int on);  /* clears the table; on != 0 starts timing */
int crest_profile_count(void);     /* distinct kernels timed so far            */
int crest_profile_entry(int i, char *name, int cap, long long *launches, double *total_ms, double *max_ms);

/* ---------------------------------------------------------------- inputs
 * Seeded synthetic counts for tests and benchmarks (not part of the
 * reference's API; it has no counterpart there).  Gene g of cell c is
 * negative-binomial with mean lib[c] * prob[labels[c]][g] and dispersion
 * `dispersion`.  Call once with indices == NULL to get row_nnz, build
 * indptr from it, then call again to fill indices/data (gene-sorted rows).
 */
typedef struct crest_synth {
    int64_t n_cells, n_genes;
    int32_t n_clusters;
    double dispersion;
    uint64_t seed;
    const double *prob;    /* [n_clusters * n_genes], rows sum to 1 */
    const int32_t *labels; /* [n_cells]                              */
    const double *lib;     /* [n_cells] expected total count         */
} crest_synth;
int crest_synth_gpu(const crest_synth *p, int64_t *row_nnz, const int64_t *indptr, uint32_t *indices, float *data);

#ifdef __cplusplus
}
#endif

#endif /* CREST_GPU_H */
