// Gene-major (CSC) copy of a device-resident CSR matrix and the per-gene
// statistics read from it (src/kernels.rs:144-160 gene_stats).
//
// Per-gene sums over cells are a scatter in the CSR layout: every stored
// entry adds four f64 values at its gene, and without a native f64 atomic in
// shared memory that scatter ran at 0.07 of HBM bandwidth.  In the CSC copy
// each gene's entries are contiguous, so the sums become segmented reductions
// with no atomics per entry: a CTA reduces a segment of one gene's column
// (cell ids and raw values, coalesced), taking each cell's normalisation
// factor from the cached per-cell totals (a gather from L2), and adds its five
// partial sums to the gene's outputs once.
//
// The copy is built once per matrix (it holds raw counts; maps and transforms
// are applied when it is read): a per-gene count (shared-memory histograms of
// blocks of cells), a host prefix sum, then a scatter in which each block of
// cells reserves one run per gene with a global atomic and places its entries
// with shared-memory atomics.  Entry order within a column follows that
// reservation order, so per-gene sums are added in no fixed order (as with
// atomics); they agree with the reference's to rounding.  Entries whose gene
// id is past the matrix's gene count are left out (every gene map drops them).
#include <vector>

#include "host.cuh"
#include "prof.cuh"
#include "rowwarp.cuh"

namespace crest {

constexpr int kCscThreads = 1024;
constexpr int kCscBlockCells = 128;
constexpr int64_t kSegEntries = 16384;

// cells [c0, c1) of a block, one warp per cell: f(gene, value, cell)
template <class F>
__device__ __forceinline__ void block_entries(const int64_t *__restrict__ indptr, const uint32_t *__restrict__ genes,
                                              const float *__restrict__ values, int64_t c0, int64_t c1, F &&f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t cell = c0 + warp; cell < c1; cell += nw) {
        const int64_t lo = indptr[cell], hi = indptr[cell + 1];
        for (int64_t e = lo + lane; e < hi; e += 32) f(__ldg(genes + e), values ? __ldg(values + e) : 0.0f, cell);
    }
}

// count[g] += entries of gene g (blocks of 8 x kCscBlockCells cells)
__global__ void __launch_bounds__(kCscThreads, 1) k_col_count(const int64_t *__restrict__ indptr,
                                                              const uint32_t *__restrict__ genes, int64_t n_cells,
                                                              int64_t n_genes, unsigned long long *__restrict__ count) {
    extern __shared__ uint32_t hist[];
    const int64_t span = (int64_t)kCscBlockCells * 8;
    for (int64_t b0 = (int64_t)blockIdx.x * span; b0 < n_cells; b0 += (int64_t)gridDim.x * span) {
        const int64_t b1 = b0 + span < n_cells ? b0 + span : n_cells;
        for (int64_t g = threadIdx.x; g < n_genes; g += blockDim.x) hist[g] = 0u;
        __syncthreads();
        block_entries(indptr, genes, nullptr, b0, b1, [&](uint32_t g, float, int64_t) {
            if ((int64_t)g < n_genes) atomicAdd(hist + g, 1u);
        });
        __syncthreads();
        for (int64_t g = threadIdx.x; g < n_genes; g += blockDim.x)
            if (hist[g]) atomicAdd(count + g, (unsigned long long)hist[g]);
        __syncthreads();
    }
}

// cursor[g]: entries of gene g placed so far, relative to col_ptr[g].
__global__ void __launch_bounds__(kCscThreads, 1)
    k_col_scatter(const int64_t *__restrict__ indptr, const uint32_t *__restrict__ genes,
                  const float *__restrict__ values, int64_t n_cells, int64_t n_genes,
                  const int64_t *__restrict__ col_ptr, uint32_t *__restrict__ cursor, uint32_t *__restrict__ col_cell,
                  float *__restrict__ col_val) {
    extern __shared__ uint32_t slot[];  // per gene: entries of the block, then the next free offset of its run
    for (int64_t b0 = (int64_t)blockIdx.x * kCscBlockCells; b0 < n_cells; b0 += (int64_t)gridDim.x * kCscBlockCells) {
        const int64_t b1 = b0 + kCscBlockCells < n_cells ? b0 + kCscBlockCells : n_cells;
        for (int64_t g = threadIdx.x; g < n_genes; g += blockDim.x) slot[g] = 0u;
        __syncthreads();
        block_entries(indptr, genes, nullptr, b0, b1, [&](uint32_t g, float, int64_t) {
            if ((int64_t)g < n_genes) atomicAdd(slot + g, 1u);
        });
        __syncthreads();
        for (int64_t g = threadIdx.x; g < n_genes; g += blockDim.x) {  // one run per gene present
            const uint32_t k = slot[g];
            if (k) slot[g] = atomicAdd(cursor + g, k);
        }
        __syncthreads();
        block_entries(indptr, genes, values, b0, b1, [&](uint32_t g, float x, int64_t cell) {
            if ((int64_t)g >= n_genes) return;
            const int64_t pos = __ldg(col_ptr + g) + atomicAdd(slot + g, 1u);
            col_cell[pos] = (uint32_t)cell;
            col_val[pos] = x;
        });
        __syncthreads();
    }
}

// Per store cell: target / total of its kept genes (1 without
// normalisation, or when the total is 0), or -1 for a dropped cell -- one
// 8-byte gather per entry in the gene-major pass instead of the cell map's
// and the totals' (each entry of a sparse gene's column meets a new sector).
__global__ void k_cell_scale(DevChunk c, int64_t n_cells, const double *__restrict__ total, double *__restrict__ cs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cells) return;
    double v = -1.0;
    if (i < c.n_cell_map && c.cell_map[i] >= 0) {
        v = 1.0;
        if (c.target_sum > 0.0) {
            const double t = total[i];
            v = t > 0.0 ? c.target_sum / t : 1.0;
        }
    }
    cs[i] = v;
}

// Five sums of one segment of a gene's column per CTA: out[m * 5 + s] +=
// (x, x^2, expm1 x, expm1(x)^2, 1) over the segment's entries of kept
// cells, x the transformed value.
__global__ void __launch_bounds__(256) k_gene_stats_csc(DevChunk c, const int64_t *__restrict__ seg_lo,
                                                        const int32_t *__restrict__ seg_gene, int64_t n_segs,
                                                        const int64_t *__restrict__ col_ptr,
                                                        const uint32_t *__restrict__ col_cell,
                                                        const float *__restrict__ col_val,
                                                        const double *__restrict__ cell_scale, double *__restrict__ out) {
    __shared__ double red[5][8];
    for (int64_t s = blockIdx.x; s < n_segs; s += gridDim.x) {
        const int32_t g = seg_gene[s];
        const int32_t m = g < c.n_gene_map ? __ldg(c.gene_map + g) : -1;
        if (m < 0) continue;  // uniform over the block
        const int64_t e0 = seg_lo[s];
        const int64_t e1 = (s + 1 < n_segs && seg_gene[s + 1] == g) ? seg_lo[s + 1] : col_ptr[g + 1];
        double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            const uint32_t cell = __ldcs(col_cell + e);
            const float x = __ldcs(col_val + e);
            const double scale = __ldg(cell_scale + cell);
            if (scale < 0.0) continue;  // dropped cell
            const double v = (double)transform_value(c, scale, x);
            const double ev = expm1(v);
            a[0] += v;
            a[1] += __dmul_rn(v, v);
            a[2] += ev;
            a[3] += __dmul_rn(ev, ev);
            a[4] += 1.0;
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) a[q] = warp_sum(a[q]);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < 5; ++q) red[q][w] = a[q];
        __syncthreads();
        if (threadIdx.x < 5) {
            double t = 0.0;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[threadIdx.x][i];
            if (t != 0.0) atomicAdd(out + (size_t)m * 5 + threadIdx.x, t);
        }
        __syncthreads();
    }
}

int build_csc(const int64_t *indptr, const uint32_t *genes, const float *values, int64_t n_cells, int64_t n_genes,
              int64_t nnz, CscMatrix &out, cudaStream_t st) {
    CREST_REQUIRE(4 * (size_t)n_genes <= (size_t)kMaxSmem, CREST_EINVAL, "too many genes for the CSC build");
    CREST_TRY(out.col_ptr.ensure(8 * (size_t)(n_genes + 1)));
    CREST_TRY(out.col_cell.ensure(4 * (size_t)std::max<int64_t>(nnz, 1)));
    CREST_TRY(out.col_val.ensure(4 * (size_t)std::max<int64_t>(nnz, 1)));
    DevBuf cursor;  // per-gene counts (u64), then per-gene placement cursors (u32)
    CREST_TRY(cursor.ensure(8 * (size_t)std::max<int64_t>(n_genes, 1)));
    CREST_CUDA_TRY(cudaMemsetAsync(cursor.ptr, 0, 8 * (size_t)n_genes, st));
    const size_t smem = 4 * (size_t)n_genes;
    CREST_TRY(ensure_smem_attr((const void *)k_col_count, smem));
    CREST_TRY(ensure_smem_attr((const void *)k_col_scatter, smem));
    const int grid = device_sms();
    {
        prof::Scope ps("csc_build", st);
        k_col_count<<<grid, kCscThreads, smem, st>>>(indptr, genes, n_cells, n_genes,
                                                      cursor.as<unsigned long long>());
        CREST_CUDA_TRY(cudaGetLastError());
    }
    std::vector<unsigned long long> cnt(n_genes);
    CREST_CUDA_TRY(cudaMemcpyAsync(cnt.data(), cursor.ptr, 8 * (size_t)n_genes, cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int64_t> ptr(n_genes + 1, 0);
    for (int64_t g = 0; g < n_genes; ++g) {
        CREST_REQUIRE(cnt[g] < (1ull << 32), CREST_EINVAL, "gene %lld has 2^32 or more entries", (long long)g);
        ptr[g + 1] = ptr[g] + (int64_t)cnt[g];
    }
    std::vector<int64_t> seg_lo;
    std::vector<int32_t> seg_gene;
    for (int64_t g = 0; g < n_genes; ++g)
        for (int64_t e = ptr[g]; e < ptr[g + 1]; e += kSegEntries) {
            seg_lo.push_back(e);
            seg_gene.push_back((int32_t)g);
        }
    out.n_segs = (int64_t)seg_lo.size();
    CREST_TRY(upload(out.col_ptr, ptr.data(), n_genes + 1, st));
    CREST_TRY(upload(out.seg_lo, seg_lo.data(), out.n_segs, st));
    CREST_TRY(upload(out.seg_gene, seg_gene.data(), out.n_segs, st));
    CREST_CUDA_TRY(cudaMemsetAsync(cursor.ptr, 0, 4 * (size_t)n_genes, st));
    {
        prof::Scope ps("csc_build", st);
        k_col_scatter<<<grid, kCscThreads, smem, st>>>(indptr, genes, values, n_cells, n_genes,
                                                        out.col_ptr.as<int64_t>(), cursor.as<uint32_t>(),
                                                        out.col_cell.as<uint32_t>(), out.col_val.as<float>());
        CREST_CUDA_TRY(cudaGetLastError());
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    cursor.release();
    out.n_genes = n_genes;
    return CREST_OK;
}

int launch_gene_stats_csc(const DevChunk &c, CscMatrix &m, const double *total, double *out, cudaStream_t st) {
    if (m.n_segs == 0) return CREST_OK;
    CREST_TRY(m.cell_scale.ensure(8 * (size_t)std::max<int64_t>(c.n_spans, 1)));
    prof::Scope ps("gene_stats_csc", st);
    if (c.n_spans)
        k_cell_scale<<<(unsigned)ceil_div(c.n_spans, 256), 256, 0, st>>>(c, c.n_spans, total,
                                                                          m.cell_scale.as<double>());
    const int64_t blocks = std::min<int64_t>(m.n_segs, (int64_t)device_sms() * 8);
    k_gene_stats_csc<<<(unsigned)blocks, 256, 0, st>>>(c, m.seg_lo.as<int64_t>(), m.seg_gene.as<int32_t>(), m.n_segs,
                                                        m.col_ptr.as<int64_t>(), m.col_cell.as<uint32_t>(),
                                                        m.col_val.as<float>(), m.cell_scale.as<double>(), out);
    CREST_CUDA_TRY(cudaGetLastError());
    return CREST_OK;
}

}  // namespace crest
