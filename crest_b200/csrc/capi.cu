// C ABI of the CREST B200 library: argument validation (the checks of
// src/py.rs), host <-> device staging, chunk streaming and pass orchestration.
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "host.cuh"

namespace crest {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}
const char *last_error() { return g_err.c_str(); }

// Failure-injection hook for tests (host side): CREST_INJECT_ALLOC_FAIL=N
// makes the N-th device allocation from now on fail as if the device were
// out of memory (read on every allocation; off by default).
static bool injected_alloc_failure() {
    static std::mutex mu;
    static long countdown = 0;
    static std::string seen;
    std::lock_guard<std::mutex> lock(mu);
    const char *e = getenv("CREST_INJECT_ALLOC_FAIL");
    const std::string v = e ? e : "";
    if (v != seen) {  // a new setting re-arms the countdown
        seen = v;
        countdown = v.empty() ? 0 : atol(v.c_str());
    }
    if (countdown <= 0) return false;
    return --countdown == 0;
}

// The library's memory pool of the current device (nullptr: none).
cudaMemPool_t device_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64];
    static bool tried[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!tried[dev]) {
        tried[dev] = true;
        int supported = 0;
        cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev);
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (supported && cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
            uint64_t keep = ~(uint64_t)0;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            pools[dev] = pool;
        }
        cudaGetLastError();
    }
    return pools[dev];
}

int DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && ptr) return CREST_OK;
    release();
    size_t want = bytes < 256 ? 256 : bytes;
    if (injected_alloc_failure()) {
        set_error("device allocation of %zu bytes failed: out of memory (injected)", want);
        return CREST_ENOMEM;
    }
    cudaMemPool_t pool = device_pool();
    cudaError_t e;
    if (pool) {  // ordered on the legacy stream, which is idle here: usable on every stream after the sync
        e = cudaMallocFromPoolAsync(&ptr, want, pool, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    } else {
        e = cudaMalloc(&ptr, want);
    }
    if (e != cudaSuccess) {
        if (ptr && pool) cudaFreeAsync(ptr, 0);
        ptr = nullptr;
        cap = 0;
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
        return CREST_ENOMEM;
    }
    cap = want;
    pooled = pool != nullptr;
    return CREST_OK;
}
void DevBuf::release() {
    if (ptr) {
        if (pooled) {  // as cudaFree: the device is idle before the memory goes back to the pool
            cudaDeviceSynchronize();
            cudaFreeAsync(ptr, 0);
            cudaStreamSynchronize(0);
        } else {
            cudaFree(ptr);
        }
    }
    ptr = nullptr;
    cap = 0;
    pooled = false;
}
int HostBuf::ensure(size_t bytes) {
    if (bytes <= cap && ptr) return CREST_OK;
    release();
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMallocHost(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cap = 0;
        cudaGetLastError();
        set_error("pinned allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
        return CREST_ENOMEM;
    }
    cap = want;
    return CREST_OK;
}
void HostBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}

int device_sms() {
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cache[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = v > 0 ? v : 1;
    }
    return cache[dev];
}

int ensure_smem_attr(const void *kernel, size_t bytes) {
    int dev = 0;
    CREST_CUDA_TRY(cudaGetDevice(&dev));
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void *, int>, size_t>> done;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &e : done)
        if (e.first.first == kernel && e.first.second == dev && e.second >= bytes) return CREST_OK;
    CREST_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    for (auto &e : done)
        if (e.first.first == kernel && e.first.second == dev) {
            e.second = bytes;
            return CREST_OK;
        }
    done.push_back({{kernel, dev}, bytes});
    return CREST_OK;
}

// ------------------------------------------------------------------ context
// Per-device staging state of the per-chunk API.  The reference's native
// functions are called sequentially from one Python thread; a mutex keeps
// concurrent callers correct.
struct Ctx {
    std::mutex mu;
    bool ready = false;
    cudaStream_t st = nullptr;
    DevBuf genes, values, span_ptr, span_cell, cell_map, gene_map, flag, sub_map, code, counter;
    DevBuf out0, out1, out2, out3, out4, out5;
    DevBuf mean, std_, bias, gram, colsum, vecs, vals, total, loadings;
    GramBufs gb;
};

static Ctx g_ctx[64];

static int get_ctx(Ctx **out) {
    CREST_TRY(require_device());
    int dev = 0;
    CREST_CUDA_TRY(cudaGetDevice(&dev));
    Ctx &c = g_ctx[dev & 63];
    if (!c.ready) {
        CREST_CUDA_TRY(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
        c.ready = true;
    }
    *out = &c;
    return CREST_OK;
}

// ------------------------------------------------------- chunk validation
// src/py.rs:162-189: lengths, exactly one of cells/indptr, sorted cells,
// monotone indptr spanning the chunk.
int validate_chunk(const crest_chunk *c) {
    CREST_REQUIRE(c != nullptr, CREST_EINVAL, "chunk is NULL");
    CREST_REQUIRE(c->nnz >= 0 && c->n_cell_map >= 0 && c->n_gene_map >= 0, CREST_EINVAL, "negative length");
    CREST_REQUIRE(c->nnz == 0 || (c->genes && c->values), CREST_EINVAL, "genes/values are NULL");
    CREST_REQUIRE((c->cells == nullptr) != (c->indptr == nullptr), CREST_EINVAL,
                  "pass exactly one of cells / indptr");
    if (c->cells) {
        for (int64_t i = 1; i < c->nnz; ++i)
            CREST_REQUIRE(c->cells[i - 1] <= c->cells[i], CREST_EINVAL, "chunk must be sorted by cell");
    } else {
        const int64_t *p = c->indptr;
        CREST_REQUIRE(c->n_indptr >= 1, CREST_EINVAL, "indptr must be non-decreasing and span the chunk");
        for (int64_t i = 1; i < c->n_indptr; ++i)
            CREST_REQUIRE(p[i - 1] <= p[i], CREST_EINVAL, "indptr must be non-decreasing and span the chunk");
        CREST_REQUIRE(p[c->n_indptr - 1] - p[0] == c->nnz, CREST_EINVAL,
                      "indptr must be non-decreasing and span the chunk");
    }
    return CREST_OK;
}

// Host-side span list of a chunk: CSR uses indptr as is; COO runs of equal
// cell ids become spans (ChunkView::cell_spans, src/kernels.rs:36-59).
struct HostSpans {
    std::vector<int64_t> ptr;
    std::vector<uint32_t> cell;
    int64_t base = 0;
    int64_t n = 0;
};

static void make_spans(const crest_chunk *c, HostSpans &s) {
    s.ptr.clear();
    s.cell.clear();
    if (c->indptr) {
        s.n = c->n_indptr - 1;
        s.base = c->indptr[0];
        return;
    }
    s.base = 0;
    int64_t p = 0;
    while (p < c->nnz) {
        const uint32_t cell = c->cells[p];
        int64_t q = p + 1;
        while (q < c->nnz && c->cells[q] == cell) ++q;
        s.ptr.push_back(p);
        s.cell.push_back(cell);
        p = q;
    }
    s.ptr.push_back(c->nnz);
    s.n = (int64_t)s.cell.size();
}

static uint32_t span_cell_host(const crest_chunk *c, const HostSpans &s, int64_t i) {
    return c->indptr ? c->first_cell + (uint32_t)i : s.cell[i];
}

// Uploads the chunk entries, spans and maps; fills a DevChunk.
static int stage_chunk(Ctx &x, const crest_chunk *c, const HostSpans &s, DevChunk &dc) {
    cudaStream_t st = x.st;
    CREST_TRY(upload(x.genes, c->genes, c->nnz, st));
    CREST_TRY(upload(x.values, c->values, c->nnz, st));
    if (c->indptr) {
        CREST_TRY(upload(x.span_ptr, c->indptr, c->n_indptr, st));
    } else {
        CREST_TRY(upload(x.span_ptr, s.ptr.data(), (int64_t)s.ptr.size(), st));
        CREST_TRY(upload(x.span_cell, s.cell.data(), (int64_t)s.cell.size(), st));
    }
    CREST_TRY(upload(x.cell_map, c->cell_map, c->n_cell_map, st));
    CREST_TRY(upload(x.gene_map, c->gene_map, c->n_gene_map, st));
    dc.genes = x.genes.as<uint32_t>();
    dc.values = x.values.as<float>();
    dc.span_ptr = x.span_ptr.as<int64_t>();
    dc.span_cell = c->indptr ? nullptr : x.span_cell.as<uint32_t>();
    dc.base = s.base;
    dc.n_spans = s.n;
    dc.first_cell = c->first_cell;
    dc.cell_map = x.cell_map.as<int64_t>();
    dc.n_cell_map = c->n_cell_map;
    dc.gene_map = x.gene_map.as<int32_t>();
    dc.n_gene_map = c->n_gene_map;
    dc.target_sum = c->target_sum;
    dc.log1p = c->log1p ? 1 : 0;
    return CREST_OK;
}

int check_maps(const crest_chunk *c, int64_t n_vars) {
    int32_t mx = -1;
    for (int64_t i = 0; i < c->n_gene_map; ++i) mx = std::max(mx, c->gene_map[i]);
    CREST_REQUIRE((int64_t)mx + 1 <= n_vars, CREST_EINVAL, "gene_map holds var %d but n_vars is %lld", (int)mx,
                  (long long)n_vars);
    return CREST_OK;
}

// Stage the scale transform (mean/std/bias) of d genes.
int stage_scale(DevBuf &mean, DevBuf &std_, DevBuf &bias, const crest_scale *t, int64_t d, DevScale &ds,
                       cudaStream_t st) {
    ds.scale = (t && t->scale) ? 1 : 0;
    ds.max_value = t ? t->max_value : 0.0;
    ds.mean = ds.std = ds.bias = nullptr;
    if (!ds.scale) return CREST_OK;
    CREST_REQUIRE(t->mean && t->std, CREST_EINVAL, "scale=True needs mean and std");
    CREST_TRY(upload(mean, t->mean, d, st));
    CREST_TRY(upload(std_, t->std, d, st));
    CREST_TRY(bias.ensure(sizeof(double) * (size_t)(d > 0 ? d : 1)));
    CREST_TRY(launch_scale_bias(mean.as<double>(), std_.as<double>(), ds.max_value, d, bias.as<double>(), st));
    ds.mean = mean.as<double>();
    ds.std = std_.as<double>();
    ds.bias = bias.as<double>();
    return CREST_OK;
}

static int check_sub_map(const int32_t *sub_map, int64_t n_vars, int64_t d) {
    CREST_REQUIRE(sub_map || n_vars == 0, CREST_EINVAL, "sub_map is NULL");
    for (int64_t i = 0; i < n_vars; ++i)
        CREST_REQUIRE(sub_map[i] < d, CREST_EINVAL, "sub_map must have length n_vars and values < d");
    return CREST_OK;
}

int stage_hvg_code(const DevChunk &dc, const int32_t *sub_map, int64_t n_vars, int64_t d, DevBuf &buf,
                   cudaStream_t st) {
    CREST_TRY(buf.ensure(std::max<size_t>(hvg_code_bytes(dc.n_gene_map), 16)));
    return launch_hvg_code(dc, sub_map, n_vars, d, buf.as<int32_t>(), st);
}

int gram_status_reset(const GramWork &w, cudaStream_t st) {
    CREST_CUDA_TRY(cudaMemsetAsync(w.status, 0, sizeof(int), st));
    return CREST_OK;
}

int gram_status_check(const GramWork &w, cudaStream_t st) {
    int h = 0;
    CREST_CUDA_TRY(cudaMemcpyAsync(&h, w.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    CREST_REQUIRE(!(h & 2), CREST_EINVAL,
                  "a cell holds the same HVG column twice (duplicate (cell, gene) entries): the dense Gram tile "
                  "cannot represent the reference's pairwise sum; merge duplicates first");
    CREST_REQUIRE(!(h & 4), CREST_EINVAL,
                  "a cell with more than 512 HVG entries is not sorted by column, so duplicate entries could not "
                  "be ruled out: sort each cell's entries by gene");
    return CREST_OK;
}

int gram_over_chunk(const DevChunk &dc, const int32_t *code, const DevScale &ds, GramWork &w,
                           double *gram, double *colsum, cudaStream_t st) {
    for (int64_t s0 = 0; s0 < dc.n_spans; s0 += w.m_cap) {
        const int64_t n = std::min(w.m_cap, dc.n_spans - s0);
        const DevChunk sc = slice(dc, s0, n);
        CREST_TRY(launch_densify(sc, code, ds, w, st));
        CREST_TRY(launch_syrk_fold(w, n, ds, gram, colsum, st));
    }
    return CREST_OK;
}

}  // namespace crest

using namespace crest;

// =================================================================== ABI
extern "C" {

const char *crest_last_error(void) { return last_error(); }
int crest_version(void) { return 1; }

int crest_memory_stats(int64_t *used, int64_t *used_high, int32_t reset_high) {
    CREST_TRY(crest::require_device());
    cudaMemPool_t pool = crest::device_pool();
    uint64_t u = 0, h = 0;
    if (pool) {
        CREST_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
        CREST_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &h));
        if (reset_high) {
            uint64_t zero = 0;
            CREST_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
        }
    }
    if (used) *used = (int64_t)u;
    if (used_high) *used_high = (int64_t)h;
    return CREST_OK;
}

int crest_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int crest_set_device(int device) {
    CREST_TRY(require_device());
    CREST_CUDA_TRY(cudaSetDevice(device));
    return CREST_OK;
}

int crest_qc(const crest_chunk *chunk, const uint8_t *flag, int64_t n_vars, double *cell_total,
             uint32_t *cell_ngenes, double *cell_flag, int64_t n_rows, uint32_t *gene_ncells,
             double *gene_total) {
    CREST_TRY(validate_chunk(chunk));
    CREST_TRY(check_maps(chunk, n_vars));
    CREST_REQUIRE(n_vars == 0 || (flag && gene_ncells && gene_total), CREST_EINVAL, "NULL per-gene output");
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    HostSpans s;
    make_spans(chunk, s);
    DevChunk dc;
    CREST_TRY(stage_chunk(*x, chunk, s, dc));
    cudaStream_t st = x->st;
    CREST_TRY(upload(x->flag, flag, n_vars, st));
    CREST_TRY(zeros<uint32_t>(x->out0, n_vars, st));
    CREST_TRY(zeros<double>(x->out1, n_vars, st));
    CREST_TRY(x->out2.ensure(sizeof(int64_t) * (size_t)std::max<int64_t>(s.n, 1)));
    CREST_TRY(x->out3.ensure(sizeof(double) * (size_t)std::max<int64_t>(s.n, 1)));
    CREST_TRY(x->out4.ensure(sizeof(uint32_t) * (size_t)std::max<int64_t>(s.n, 1)));
    CREST_TRY(x->out5.ensure(sizeof(double) * (size_t)std::max<int64_t>(s.n, 1)));
    SpanOut so{x->out2.as<int64_t>(), x->out3.as<double>(), x->out4.as<uint32_t>(), x->out5.as<double>()};
    CREST_TRY(launch_qc(dc, x->flag.as<uint8_t>(), x->out0.as<uint32_t>(), x->out1.as<double>(), &so, nullptr, st));
    std::vector<uint32_t> gn(n_vars);
    std::vector<double> gt(n_vars), st_t(s.n), st_f(s.n);
    std::vector<int64_t> srow(s.n);
    std::vector<uint32_t> st_n(s.n);
    if (n_vars) {
        CREST_CUDA_TRY(cudaMemcpyAsync(gn.data(), x->out0.ptr, 4 * n_vars, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(gt.data(), x->out1.ptr, 8 * n_vars, cudaMemcpyDeviceToHost, st));
    }
    if (s.n) {
        CREST_CUDA_TRY(cudaMemcpyAsync(srow.data(), x->out2.ptr, 8 * s.n, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(st_t.data(), x->out3.ptr, 8 * s.n, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(st_n.data(), x->out4.ptr, 4 * s.n, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(st_f.data(), x->out5.ptr, 8 * s.n, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < s.n; ++i) {
        const int64_t r = srow[i];
        if (r < 0) continue;
        CREST_REQUIRE(r < n_rows, CREST_EINVAL, "output sizes do not match the maps");
        cell_total[r] += st_t[i];
        cell_ngenes[r] += st_n[i];
        cell_flag[r] += st_f[i];
    }
    for (int64_t g = 0; g < n_vars; ++g) {
        gene_ncells[g] += gn[g];
        gene_total[g] += gt[g];
    }
    return CREST_OK;
}

int crest_gene_stats(const crest_chunk *chunk, int64_t n_vars, double *out) {
    CREST_TRY(validate_chunk(chunk));
    CREST_TRY(check_maps(chunk, n_vars));
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    HostSpans s;
    make_spans(chunk, s);
    DevChunk dc;
    CREST_TRY(stage_chunk(*x, chunk, s, dc));
    cudaStream_t st = x->st;
    CREST_TRY(zeros<double>(x->out1, n_vars * 5, st));
    CREST_TRY(launch_gene_stats(dc, x->out1.as<double>(), st));
    std::vector<double> o(n_vars * 5);
    if (n_vars)
        CREST_CUDA_TRY(cudaMemcpyAsync(o.data(), x->out1.ptr, 40 * n_vars, cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < n_vars * 5; ++i) out[i] += o[i];
    return CREST_OK;
}

int crest_gram_accumulate(const crest_chunk *chunk, const int32_t *sub_map, int64_t n_vars,
                          const crest_scale *scale, int64_t d, double *gram, double *colsum,
                          int32_t precision) {
    CREST_TRY(validate_chunk(chunk));
    CREST_TRY(check_maps(chunk, n_vars));
    CREST_REQUIRE(d >= 0 && gram && colsum, CREST_EINVAL, "gram must be (d, d)");
    CREST_REQUIRE(precision >= CREST_GRAM_FP64 && precision <= CREST_GRAM_BF16X3, CREST_EINVAL,
                  "unknown Gram precision %d", precision);
    CREST_TRY(check_sub_map(sub_map, n_vars, d));
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    HostSpans s;
    make_spans(chunk, s);
    DevChunk dc;
    CREST_TRY(stage_chunk(*x, chunk, s, dc));
    cudaStream_t st = x->st;
    CREST_TRY(upload(x->sub_map, sub_map, n_vars, st));
    DevScale ds;
    CREST_TRY(stage_scale(x->mean, x->std_, x->bias, scale, d, ds, st));
    CREST_TRY(upload(x->gram, gram, d * d, st));
    CREST_TRY(upload(x->colsum, colsum, d, st));
    GramWork w;
    const int64_t m_cap = std::min<int64_t>(tile_cells_default(), round_up(std::max<int64_t>(s.n, 1), 64));
    CREST_TRY(x->gb.ensure(w, d, precision, m_cap));
    CREST_TRY(stage_hvg_code(dc, x->sub_map.as<int32_t>(), n_vars, d, x->code, st));
    CREST_TRY(gram_status_reset(w, st));
    if (w.gram_aux) CREST_CUDA_TRY(cudaMemsetAsync(w.gram_aux, 0, sizeof(double) * (size_t)(d * d), st));
    CREST_TRY(gram_over_chunk(dc, x->code.as<int32_t>(), ds, w, x->gram.as<double>(), x->colsum.as<double>(), st));
    CREST_TRY(gram_aux_fold(w, x->gram.as<double>(), st));
    CREST_TRY(gram_status_check(w, st));  // the caller's gram / colsum stay untouched on error
    if (precision == CREST_GRAM_BF16X3) CREST_TRY(tc_check_error());
    if (d) {
        CREST_CUDA_TRY(cudaMemcpyAsync(gram, x->gram.ptr, 8 * d * d, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(colsum, x->colsum.ptr, 8 * d, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    return CREST_OK;
}

int crest_pca_from_gram(const double *gram, const double *colsum, int64_t d, int64_t n, int64_t k,
                        double *variance, double *loadings, double *total, crest_pca_stats *stats) {
    CREST_REQUIRE(gram && colsum && total, CREST_EINVAL, "gram must be (d, d)");
    CREST_REQUIRE(n >= 2 && d >= 1, CREST_ERUNTIME, "need at least 2 cells and 1 gene");
    CREST_REQUIRE(k >= 0 && k <= d, CREST_EINVAL, "k must be in [0, d]");
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    cudaStream_t st = x->st;
    CREST_TRY(upload(x->gram, gram, d * d, st));
    CREST_TRY(upload(x->colsum, colsum, d, st));
    CREST_TRY(x->vals.ensure(sizeof(double) * (size_t)std::max<int64_t>(k, 1)));
    CREST_TRY(x->vecs.ensure(sizeof(double) * (size_t)std::max<int64_t>(d * k, 1)));
    CREST_TRY(x->total.ensure(sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    EigStats es{};
    int rc = eig_topk(x->gram.as<double>(), x->colsum.as<double>(), d, n, k, x->vals.as<double>(),
                      x->vecs.as<double>(), x->total.as<double>(), &es, st);
    cudaEventRecord(e1, st);
    if (rc != CREST_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
    }
    if (k) {
        CREST_CUDA_TRY(cudaMemcpyAsync(variance, x->vals.ptr, 8 * k, cudaMemcpyDeviceToHost, st));
        CREST_CUDA_TRY(cudaMemcpyAsync(loadings, x->vecs.ptr, 8 * d * k, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaMemcpyAsync(total, x->total.ptr, 8, cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->solve_ms = ms;
        stats->eig_iters = es.iters;
        stats->eig_converged = es.converged;
        stats->eig_residual = es.residual;
    }
    CREST_REQUIRE(es.converged, CREST_ERUNTIME, "eigensolver did not converge (residual %.3g after %d iterations)",
                  es.residual, es.iters);
    return CREST_OK;
}

int crest_group_gene_sums(const crest_chunk *chunk, const uint32_t *group_of_row, int64_t n_group_rows,
                          int64_t n_groups, int64_t n_vars, const double *clip, double *sum, double *sumsq,
                          double *nnz) {
    CREST_TRY(validate_chunk(chunk));
    CREST_TRY(check_maps(chunk, n_vars));
    CREST_REQUIRE(n_groups >= 0 && sum && (n_groups * n_vars == 0 || group_of_row), CREST_EINVAL,
                  "sum, sumsq, nnz must be (n_groups, n_vars); group_of_row (n_rows,)");
    int64_t n_rows = 0;
    for (int64_t i = 0; i < chunk->n_cell_map; ++i) n_rows = std::max<int64_t>(n_rows, chunk->cell_map[i] + 1);
    CREST_REQUIRE(n_group_rows >= n_rows, CREST_EINVAL,
                  "sum, sumsq, nnz must be (n_groups, n_vars); group_of_row (n_rows,)");
    for (int64_t r = 0; r < n_group_rows; ++r)
        CREST_REQUIRE(group_of_row[r] == 0xffffffffu || (int64_t)group_of_row[r] < n_groups, CREST_EINVAL,
                      "group id out of range");
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    HostSpans s;
    make_spans(chunk, s);
    DevChunk dc;
    CREST_TRY(stage_chunk(*x, chunk, s, dc));
    cudaStream_t st = x->st;
    const int64_t ne = n_groups * n_vars;
    CREST_TRY(upload(x->out5, group_of_row, n_group_rows, st));
    const double *dclip = nullptr;
    if (clip) {
        CREST_TRY(upload(x->out4, clip, ne, st));
        dclip = x->out4.as<double>();
    }
    CREST_TRY(zeros<double>(x->out0, ne, st));
    if (sumsq) CREST_TRY(zeros<double>(x->out1, ne, st));
    if (nnz) CREST_TRY(zeros<double>(x->out2, ne, st));
    CREST_TRY(launch_group_gene_sums(dc, x->out5.as<uint32_t>(), n_vars, dclip, x->out0.as<double>(),
                                     sumsq ? x->out1.as<double>() : nullptr, nnz ? x->out2.as<double>() : nullptr,
                                     st));
    std::vector<double> h0(ne), h1(sumsq ? ne : 0), h2(nnz ? ne : 0);
    if (ne) {
        CREST_CUDA_TRY(cudaMemcpyAsync(h0.data(), x->out0.ptr, 8 * ne, cudaMemcpyDeviceToHost, st));
        if (sumsq) CREST_CUDA_TRY(cudaMemcpyAsync(h1.data(), x->out1.ptr, 8 * ne, cudaMemcpyDeviceToHost, st));
        if (nnz) CREST_CUDA_TRY(cudaMemcpyAsync(h2.data(), x->out2.ptr, 8 * ne, cudaMemcpyDeviceToHost, st));
    }
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < ne; ++i) sum[i] += h0[i];
    for (int64_t i = 0; sumsq && i < ne; ++i) sumsq[i] += h1[i];
    for (int64_t i = 0; nnz && i < ne; ++i) nnz[i] += h2[i];
    return CREST_OK;
}

int crest_group_gene_totals(const crest_chunk *chunk, const uint32_t *group_of_row, int64_t n_group_rows,
                            int64_t n_groups, int64_t n_vars, double *sum) {
    return crest_group_gene_sums(chunk, group_of_row, n_group_rows, n_groups, n_vars, nullptr, sum, nullptr,
                                 nullptr);
}

int crest_knn_graph(const float *data, int64_t n, int64_t d, int64_t k, uint32_t *indices, float *distances) {
    CREST_REQUIRE(n >= 0 && d >= 1 && k >= 0 && (n == 0 || data), CREST_EINVAL, "data must be (n, d) with d >= 1");
    const int64_t kk = n > 1 ? std::max<int64_t>(1, std::min(k, n - 1)) : 0;
    if (kk == 0) return CREST_OK;
    CREST_REQUIRE(indices && distances, CREST_EINVAL, "NULL output");
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    cudaStream_t st = x->st;
    CREST_TRY(upload(x->out0, data, n * d, st));
    CREST_TRY(x->out1.ensure(sizeof(uint32_t) * (size_t)(n * kk)));
    CREST_TRY(x->out2.ensure(sizeof(float) * (size_t)(n * kk)));
    CREST_TRY(launch_knn(x->out0.as<float>(), n, (int)d, (int)kk, x->out1.as<uint32_t>(), x->out2.as<float>(), st));
    CREST_CUDA_TRY(cudaMemcpyAsync(indices, x->out1.ptr, 4 * (size_t)(n * kk), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaMemcpyAsync(distances, x->out2.ptr, 4 * (size_t)(n * kk), cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    return CREST_OK;
}

int crest_project(const crest_chunk *chunk, const int32_t *sub_map, int64_t n_vars, const double *loadings,
                  int64_t d, int64_t k, const crest_scale *scale, float *out, int64_t n_rows) {
    CREST_TRY(validate_chunk(chunk));
    CREST_TRY(check_maps(chunk, n_vars));
    CREST_REQUIRE(k >= 0 && k <= 128, CREST_EINVAL, "loadings must be (d, k) with k <= 128");
    CREST_REQUIRE(loadings || d * k == 0, CREST_EINVAL, "loadings must be (d, k)");
    CREST_TRY(check_sub_map(sub_map, n_vars, d));
    Ctx *x;
    CREST_TRY(get_ctx(&x));
    std::lock_guard<std::mutex> lock(x->mu);
    HostSpans s;
    make_spans(chunk, s);
    DevChunk dc;
    CREST_TRY(stage_chunk(*x, chunk, s, dc));
    cudaStream_t st = x->st;
    CREST_TRY(upload(x->sub_map, sub_map, n_vars, st));
    DevScale ds;
    CREST_TRY(stage_scale(x->mean, x->std_, x->bias, scale, d, ds, st));
    CREST_TRY(upload(x->loadings, loadings, d * k, st));
    CREST_TRY(zeros<float>(x->out3, s.n * k, st));
    CREST_TRY(stage_hvg_code(dc, x->sub_map.as<int32_t>(), n_vars, d, x->code, st));
    CREST_TRY(x->counter.ensure(sizeof(unsigned int)));
    CREST_TRY(launch_project(dc, x->code.as<int32_t>(), d, ds, x->loadings.as<double>(), (int)k,
                             x->out3.as<float>(), 1, x->counter.as<unsigned int>(), st));
    std::vector<float> part(s.n * k);
    if (!part.empty())
        CREST_CUDA_TRY(cudaMemcpyAsync(part.data(), x->out3.ptr, 4 * s.n * k, cudaMemcpyDeviceToHost, st));
    CREST_CUDA_TRY(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < s.n; ++i) {
        const uint32_t cell = span_cell_host(chunk, s, i);
        if ((int64_t)cell >= chunk->n_cell_map) continue;
        const int64_t r = chunk->cell_map[cell];
        if (r < 0) continue;
        CREST_REQUIRE(r < n_rows, CREST_EINVAL, "out must be (n_rows, k)");
        for (int64_t j = 0; j < k; ++j) out[r * k + j] += part[i * k + j];
    }
    return CREST_OK;
}

}  // extern "C"
