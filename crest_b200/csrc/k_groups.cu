// Per (group, gene) sums of the transformed matrix: the streaming pass behind
// differential expression (rank_genes_groups t-test) and pseudobulk totals
// (src/kernels.rs:388-442 group_gene_sums; src/py.rs:311-357).
//
// For every stored entry of a kept cell whose row has a group
// (group_of_row[row] != 0xffffffff) and whose gene is kept:
//   x = the lazily transformed value (normalize_total / log1p, f32),
//   x = min(x, clip[group][gene]) when a clip table is given (seurat_v3),
//   sum[group][gene] += x, sumsq += x * x, nnz += 1        (f64)
// One warp per cell (the cell's normalisation factor from its kept-gene
// total, as every pass here), then one f64 atomic per entry and statistic
// into the (n_groups x n_vars) outputs; the outputs are small enough to stay
// in L2.  The reference sums each (group, gene) in entry order; here the
// order of the atomics is not fixed, so results agree to rounding.
#include "kernels.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {

__global__ void __launch_bounds__(256) k_group_gene_sums(DevChunk c, const uint32_t *__restrict__ group_of_row,
                                                         int64_t n_vars, const double *__restrict__ clip,
                                                         double *__restrict__ sum, double *__restrict__ sumsq,
                                                         double *__restrict__ nnz) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < c.n_spans; i += n_warps) {
        int64_t lo, hi;
        const int64_t row = span_row(c, i, lo, hi);
        if (row < 0) continue;
        const uint32_t grp = __ldg(group_of_row + row);
        if (grp == 0xffffffffu) continue;
        const double scale = cell_scale(c, lo, hi);
        const int64_t base = (int64_t)grp * n_vars;
        for_entries<8>(c, lo, hi, [&](int32_t m, float xf) {
            if (m < 0) return;
            const int64_t at = base + m;
            double x = (double)transform_value(c, scale, xf);
            if (clip) x = fmin(x, __ldg(clip + at));
            atomicAdd(sum + at, x);
            if (sumsq) atomicAdd(sumsq + at, __dmul_rn(x, x));
            if (nnz) atomicAdd(nnz + at, 1.0);
        });
    }
}

int launch_group_gene_sums(const DevChunk &c, const uint32_t *group_of_row, int64_t n_vars, const double *clip,
                           double *sum, double *sumsq, double *nnz, cudaStream_t st) {
    if (c.n_spans == 0) return CREST_OK;
    prof::Scope ps("group_gene_sums_csr", st);
    int64_t blocks = ceil_div(c.n_spans, 8);
    const int64_t cap = (int64_t)device_sms() * 16;
    if (blocks > cap) blocks = cap;
    k_group_gene_sums<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(c, group_of_row, n_vars, clip, sum,
                                                                              sumsq, nnz);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
