/*
 * CPU ORACLE -- test infrastructure only.
 *
 * A plain-C restatement of the reference's streaming CPU kernels
 * (src/kernels.rs of harshameghadri/CREST).  It exists to check the CUDA
 * product path and to serve as the timed CPU baseline; nothing in the
 * product imports, links or calls it.
 *
 * Parity pinning: the reference crate cannot be compiled here (no Rust
 * toolchain, no crates registry), so this restatement is pinned by the
 * reference's own known-answer tests restated in tests/test_oracle.py
 * (src/kernels.rs:565-578 materialise KAT, src/kernels.rs:580-633 scaled
 * Gram vs dense covariance) and by golden vectors produced by running the
 * reference's unmodified Python orchestration (crest/pp.py, crest/tl.py)
 * on top of this library (tests/golden/make_golden.py).
 *
 * Everything follows the reference's summation order:
 *  - cells are grouped into "parts" exactly like ChunkView::parts
 *    (src/kernels.rs:88-102), with `n_threads` standing in for
 *    rayon::current_num_threads(); per-part partial arrays are merged in
 *    part order (src/kernels.rs:157-159, 186-194);
 *  - per-cell transforms use libm log1pf / expm1 as Rust's f32::ln_1p and
 *    f64::exp_m1 do on Linux (src/kernels.rs:81, 148);
 *  - products are never fused (Rust does not contract a*b+c); build with
 *    -ffp-contract=off.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    const uint32_t *genes;   /* [nnz] store gene ids                     */
    const float *values;     /* [nnz]                                    */
    int64_t nnz;
    const int64_t *cell_map; /* [n_cell_map] store cell -> row, -1 = drop */
    int64_t n_cell_map;
    const int32_t *gene_map; /* [n_gene_map] store gene -> var, -1 = drop */
    int64_t n_gene_map;
    double target_sum;
    int32_t log1p;
    const uint32_t *cells;   /* [nnz] COO cell ids, or NULL              */
    const int64_t *indptr;   /* [n_indptr] CSR row pointer, or NULL      */
    int64_t n_indptr;
    uint32_t first_cell;
} oc_chunk;

typedef struct { uint32_t cell; int64_t lo, hi; } span_t;
typedef struct { int64_t first, last; } part_t; /* span index range [first, last) */

/* ------------------------------------------------------------------ spans
 * ChunkView::cell_spans, src/kernels.rs:36-59. */
static span_t *cell_spans(const oc_chunk *v, int64_t *n_out) {
    span_t *out;
    int64_t n = 0;
    if (v->indptr) {
        int64_t m = v->n_indptr > 0 ? v->n_indptr - 1 : 0;
        int64_t base = v->n_indptr > 0 ? v->indptr[0] : 0;
        out = (span_t *)malloc(sizeof(span_t) * (size_t)(m > 0 ? m : 1));
        for (int64_t i = 0; i < m; i++) {
            out[i].cell = v->first_cell + (uint32_t)i;
            out[i].lo = v->indptr[i] - base;
            out[i].hi = v->indptr[i + 1] - base;
        }
        n = m;
    } else {
        out = (span_t *)malloc(sizeof(span_t) * (size_t)(v->nnz > 0 ? v->nnz : 1));
        int64_t p = 0;
        while (p < v->nnz) {
            uint32_t c = v->cells[p];
            int64_t q = p + 1;
            while (q < v->nnz && v->cells[q] == c) q++;
            out[n].cell = c; out[n].lo = p; out[n].hi = q; n++;
            p = q;
        }
    }
    *n_out = n;
    return out;
}

/* ChunkView::parts, src/kernels.rs:88-102: about 4 x threads parts of
 * similar entry counts. */
static part_t *make_parts(const oc_chunk *v, const span_t *sp, int64_t ns, int n_threads, int64_t *np_out) {
    int64_t total = v->nnz > 1 ? v->nnz : 1;
    int64_t n_parts = (int64_t)n_threads * 4;
    if (total / 8192 + 1 < n_parts) n_parts = total / 8192 + 1;
    if (n_parts < 1) n_parts = 1;
    part_t *parts = (part_t *)malloc(sizeof(part_t) * (size_t)(ns + 1));
    int64_t np = 1;
    parts[0].first = 0; parts[0].last = 0;
    int64_t acc = 0;
    for (int64_t i = 0; i < ns; i++) {
        if (acc * n_parts >= total * np && parts[np - 1].last > parts[np - 1].first) {
            parts[np].first = i; parts[np].last = i; np++;
        }
        acc += sp[i].hi - sp[i].lo;
        parts[np - 1].last = i + 1;
    }
    *np_out = np;
    return parts;
}

/* ------------------------------------------------------------------ cell
 * ChunkView::cell, src/kernels.rs:63-85.  Returns the row or -1. */
static int64_t cell_entries(const oc_chunk *v, const span_t *s, uint32_t *bg, float *bx, int64_t *nb) {
    *nb = 0;
    if ((int64_t)s->cell >= v->n_cell_map) return -1;
    int64_t row = v->cell_map[s->cell];
    if (row < 0) return -1;
    double total = 0.0;
    int64_t n = 0;
    for (int64_t e = s->lo; e < s->hi; e++) {
        uint32_t g = v->genes[e];
        int32_t m = (int64_t)g < v->n_gene_map ? v->gene_map[g] : -1;
        if (m >= 0) {
            bg[n] = (uint32_t)m;
            bx[n] = v->values[e];
            total += (double)v->values[e];
            n++;
        }
    }
    if (v->target_sum > 0.0 || v->log1p) {
        double scale = (v->target_sum > 0.0 && total > 0.0) ? v->target_sum / total : 1.0;
        for (int64_t i = 0; i < n; i++) {
            float y = v->target_sum > 0.0 ? (float)((double)bx[i] * scale) : bx[i];
            bx[i] = v->log1p ? log1pf(y) : y;
        }
    }
    *nb = n;
    return row;
}

static int64_t max_span_len(const span_t *sp, int64_t ns) {
    int64_t m = 1;
    for (int64_t i = 0; i < ns; i++) if (sp[i].hi - sp[i].lo > m) m = sp[i].hi - sp[i].lo;
    return m;
}

/* ------------------------------------------------------------------ pool */
typedef struct {
    void (*fn)(void *ctx, int64_t item);
    void *ctx;
    int64_t n_items;
    int64_t next;
    pthread_mutex_t mu;
} pool_t;

static void *pool_worker(void *arg) {
    pool_t *p = (pool_t *)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        int64_t it = p->next++;
        pthread_mutex_unlock(&p->mu);
        if (it >= p->n_items) break;
        p->fn(p->ctx, it);
    }
    return NULL;
}

static void run_pool(int n_threads, int64_t n_items, void (*fn)(void *, int64_t), void *ctx) {
    pool_t p;
    p.fn = fn; p.ctx = ctx; p.n_items = n_items; p.next = 0;
    pthread_mutex_init(&p.mu, NULL);
    int nt = n_threads < 1 ? 1 : n_threads;
    if (nt > 256) nt = 256;
    if ((int64_t)nt > n_items) nt = (int)(n_items > 0 ? n_items : 1);
    pthread_t th[256];
    for (int i = 1; i < nt; i++) pthread_create(&th[i], NULL, pool_worker, &p);
    pool_worker(&p);
    for (int i = 1; i < nt; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&p.mu);
}

/* ------------------------------------------------------------------ qc
 * src/kernels.rs:164-195 */
typedef struct {
    const oc_chunk *v; const span_t *sp; const part_t *parts; int64_t maxlen;
    const uint8_t *flag; int64_t ng;
    /* per part outputs */
    int64_t *cell_row; double *cell_t; uint32_t *cell_n; double *cell_f; /* indexed by span */
    uint32_t **gn; double **gt;
} qc_ctx;

static void qc_part(void *c_, int64_t ip) {
    qc_ctx *c = (qc_ctx *)c_;
    const part_t *pt = &c->parts[ip];
    uint32_t *bg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)c->maxlen);
    float *bx = (float *)malloc(sizeof(float) * (size_t)c->maxlen);
    uint32_t *gn = (uint32_t *)calloc((size_t)(c->ng > 0 ? c->ng : 1), sizeof(uint32_t));
    double *gt = (double *)calloc((size_t)(c->ng > 0 ? c->ng : 1), sizeof(double));
    for (int64_t i = pt->first; i < pt->last; i++) {
        int64_t nb;
        int64_t row = cell_entries(c->v, &c->sp[i], bg, bx, &nb);
        c->cell_row[i] = row;
        if (row < 0) continue;
        double t = 0.0, f = 0.0;
        uint32_t n = 0;
        for (int64_t e = 0; e < nb; e++) {
            float x = bx[e];
            if (x == 0.0f) continue;
            t += (double)x;
            n += 1;
            if (c->flag[bg[e]]) f += (double)x;
            gn[bg[e]] += 1;
            gt[bg[e]] += (double)x;
        }
        c->cell_t[i] = t; c->cell_n[i] = n; c->cell_f[i] = f;
    }
    c->gn[ip] = gn; c->gt[ip] = gt;
    free(bg); free(bx);
}

int oc_qc(const oc_chunk *v, int n_threads, const uint8_t *flag, double *cell_total, uint32_t *cell_ngenes,
          double *cell_flag, uint32_t *gene_ncells, double *gene_total, int64_t ng) {
    int64_t ns, np;
    span_t *sp = cell_spans(v, &ns);
    part_t *parts = make_parts(v, sp, ns, n_threads, &np);
    qc_ctx c;
    c.v = v; c.sp = sp; c.parts = parts; c.maxlen = max_span_len(sp, ns); c.flag = flag; c.ng = ng;
    size_t nsz = (size_t)(ns > 0 ? ns : 1);
    c.cell_row = (int64_t *)malloc(sizeof(int64_t) * nsz);
    c.cell_t = (double *)malloc(sizeof(double) * nsz);
    c.cell_n = (uint32_t *)malloc(sizeof(uint32_t) * nsz);
    c.cell_f = (double *)malloc(sizeof(double) * nsz);
    c.gn = (uint32_t **)calloc((size_t)np, sizeof(uint32_t *));
    c.gt = (double **)calloc((size_t)np, sizeof(double *));
    run_pool(n_threads, np, qc_part, &c);
    for (int64_t ip = 0; ip < np; ip++) {
        for (int64_t i = parts[ip].first; i < parts[ip].last; i++) {
            int64_t r = c.cell_row[i];
            if (r < 0) continue;
            cell_total[r] += c.cell_t[i];
            cell_ngenes[r] += c.cell_n[i];
            cell_flag[r] += c.cell_f[i];
        }
        for (int64_t g = 0; g < ng; g++) { gene_ncells[g] += c.gn[ip][g]; gene_total[g] += c.gt[ip][g]; }
        free(c.gn[ip]); free(c.gt[ip]);
    }
    free(c.gn); free(c.gt); free(c.cell_row); free(c.cell_t); free(c.cell_n); free(c.cell_f);
    free(parts); free(sp);
    return 0;
}

/* ------------------------------------------------------------------ gene_stats
 * src/kernels.rs:144-160 */
typedef struct {
    const oc_chunk *v; const span_t *sp; const part_t *parts; int64_t maxlen; int64_t nv;
    double **acc;
} gs_ctx;

static void gs_part(void *c_, int64_t ip) {
    gs_ctx *c = (gs_ctx *)c_;
    const part_t *pt = &c->parts[ip];
    uint32_t *bg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)c->maxlen);
    float *bx = (float *)malloc(sizeof(float) * (size_t)c->maxlen);
    double *acc = (double *)calloc((size_t)(c->nv > 0 ? c->nv * 5 : 1), sizeof(double));
    for (int64_t i = pt->first; i < pt->last; i++) {
        int64_t nb;
        if (cell_entries(c->v, &c->sp[i], bg, bx, &nb) < 0) continue;
        for (int64_t e = 0; e < nb; e++) {
            double x = (double)bx[e];
            double ex = expm1(x);
            double *o = acc + (size_t)bg[e] * 5;
            o[0] += x;
            o[1] += x * x;
            o[2] += ex;
            o[3] += ex * ex;
            o[4] += 1.0;
        }
    }
    c->acc[ip] = acc;
    free(bg); free(bx);
}

int oc_gene_stats(const oc_chunk *v, int n_threads, double *out, int64_t nv) {
    int64_t ns, np;
    span_t *sp = cell_spans(v, &ns);
    part_t *parts = make_parts(v, sp, ns, n_threads, &np);
    gs_ctx c;
    c.v = v; c.sp = sp; c.parts = parts; c.maxlen = max_span_len(sp, ns); c.nv = nv;
    c.acc = (double **)calloc((size_t)np, sizeof(double *));
    run_pool(n_threads, np, gs_part, &c);
    for (int64_t ip = 0; ip < np; ip++) {
        for (int64_t i = 0; i < nv * 5; i++) out[i] += c.acc[ip][i];
        free(c.acc[ip]);
    }
    free(c.acc); free(parts); free(sp);
    return 0;
}

/* ------------------------------------------------------------------ transform
 * Transform::apply, src/kernels.rs:209-219 */
typedef struct { int scale; const double *mean; const double *std; double max_value; } oc_transform;

static inline double clipv(double z, double mv) {
    if (mv > 0.0) { if (z < -mv) return -mv; if (z > mv) return mv; }
    return z;
}
static inline double tf_apply(const oc_transform *t, int64_t g, float x) {
    if (!t->scale) return (double)x;
    double mu = t->mean[g], sd = t->std[g];
    return clipv(((double)x - mu) / sd, t->max_value) - clipv(-mu / sd, t->max_value);
}

/* ------------------------------------------------------------------ gram
 * src/kernels.rs:227-309 */
typedef struct {
    const oc_chunk *v; const span_t *sp; const part_t *parts; int64_t maxlen;
    const int32_t *sub_map; const oc_transform *t;
    /* per part compacted rows */
    int64_t **ends; int64_t *n_rows; uint32_t **eg; double **ev; int64_t *n_ent;
} gc_ctx;

static void gc_part(void *c_, int64_t ip) {
    gc_ctx *c = (gc_ctx *)c_;
    const part_t *pt = &c->parts[ip];
    uint32_t *bg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)c->maxlen);
    float *bx = (float *)malloc(sizeof(float) * (size_t)c->maxlen);
    int64_t cap = 1024, nrow = 0, cnt = 0, rcap = 64;
    uint32_t *eg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)cap);
    double *ev = (double *)malloc(sizeof(double) * (size_t)cap);
    int64_t *ends = (int64_t *)malloc(sizeof(int64_t) * (size_t)rcap);
    for (int64_t i = pt->first; i < pt->last; i++) {
        int64_t nb;
        if (cell_entries(c->v, &c->sp[i], bg, bx, &nb) < 0) continue;
        int64_t s = cnt;
        for (int64_t e = 0; e < nb; e++) {
            int32_t m = c->sub_map[bg[e]];
            if (m >= 0) {
                if (cnt == cap) {
                    cap *= 2;
                    eg = (uint32_t *)realloc(eg, sizeof(uint32_t) * (size_t)cap);
                    ev = (double *)realloc(ev, sizeof(double) * (size_t)cap);
                }
                eg[cnt] = (uint32_t)m;
                ev[cnt] = tf_apply(c->t, m, bx[e]);
                cnt++;
            }
        }
        if (cnt > s) {
            int sorted = 1;
            for (int64_t q = s + 1; q < cnt; q++) if (eg[q - 1] > eg[q]) { sorted = 0; break; }
            if (!sorted) { /* stable insertion sort by gene (Rust sort_by_key is stable) */
                for (int64_t q = s + 1; q < cnt; q++) {
                    uint32_t kg = eg[q]; double kv = ev[q];
                    int64_t r = q;
                    while (r > s && eg[r - 1] > kg) { eg[r] = eg[r - 1]; ev[r] = ev[r - 1]; r--; }
                    eg[r] = kg; ev[r] = kv;
                }
            }
            if (nrow == rcap) { rcap *= 2; ends = (int64_t *)realloc(ends, sizeof(int64_t) * (size_t)rcap); }
            ends[nrow++] = cnt;
        }
    }
    c->ends[ip] = ends; c->n_rows[ip] = nrow; c->eg[ip] = eg; c->ev[ip] = ev; c->n_ent[ip] = cnt;
    free(bg); free(bx);
}

typedef struct {
    const int64_t *starts; int64_t n_starts; const uint32_t *eg; const double *ev;
    const int64_t *bounds; int64_t d; double *gram;
} gb_ctx;

static void gb_block(void *c_, int64_t ib) {
    gb_ctx *c = (gb_ctx *)c_;
    int64_t lo = c->bounds[ib], hi = c->bounds[ib + 1], d = c->d;
    for (int64_t w = 0; w + 1 < c->n_starts; w++) {
        const uint32_t *rg = c->eg + c->starts[w];
        const double *rv = c->ev + c->starts[w];
        int64_t len = c->starts[w + 1] - c->starts[w];
        /* partition_point(|g| g < lo) */
        int64_t a0 = 0, a1 = len;
        while (a0 < a1) { int64_t mid = (a0 + a1) / 2; if ((int64_t)rg[mid] < lo) a0 = mid + 1; else a1 = mid; }
        for (int64_t k = a0; k < len; k++) {
            int64_t a = rg[k];
            if (a >= hi) break;
            double va = rv[k];
            double *out = c->gram + (size_t)a * (size_t)d;
            for (int64_t m = k; m < len; m++) out[rg[m]] += va * rv[m];
        }
    }
}

int oc_gram_accumulate(const oc_chunk *v, int n_threads, const int32_t *sub_map, int64_t d, int scale,
                       const double *mean, const double *std, double max_value, double *gram, double *colsum) {
    oc_transform t = {scale, mean, std, max_value};
    int64_t ns, np;
    span_t *sp = cell_spans(v, &ns);
    part_t *parts = make_parts(v, sp, ns, n_threads, &np);
    gc_ctx c;
    c.v = v; c.sp = sp; c.parts = parts; c.maxlen = max_span_len(sp, ns); c.sub_map = sub_map; c.t = &t;
    c.ends = (int64_t **)calloc((size_t)np, sizeof(int64_t *));
    c.n_rows = (int64_t *)calloc((size_t)np, sizeof(int64_t));
    c.eg = (uint32_t **)calloc((size_t)np, sizeof(uint32_t *));
    c.ev = (double **)calloc((size_t)np, sizeof(double *));
    c.n_ent = (int64_t *)calloc((size_t)np, sizeof(int64_t));
    run_pool(n_threads, np, gc_part, &c);
    /* concatenate parts in order */
    int64_t tot_ent = 0, tot_rows = 0;
    for (int64_t ip = 0; ip < np; ip++) { tot_ent += c.n_ent[ip]; tot_rows += c.n_rows[ip]; }
    uint32_t *eg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(tot_ent > 0 ? tot_ent : 1));
    double *ev = (double *)malloc(sizeof(double) * (size_t)(tot_ent > 0 ? tot_ent : 1));
    int64_t *starts = (int64_t *)malloc(sizeof(int64_t) * (size_t)(tot_rows + 1));
    int64_t off = 0, ri = 0;
    starts[ri++] = 0;
    for (int64_t ip = 0; ip < np; ip++) {
        for (int64_t r = 0; r < c.n_rows[ip]; r++) starts[ri++] = c.ends[ip][r] + off;
        memcpy(eg + off, c.eg[ip], sizeof(uint32_t) * (size_t)c.n_ent[ip]);
        memcpy(ev + off, c.ev[ip], sizeof(double) * (size_t)c.n_ent[ip]);
        off += c.n_ent[ip];
        free(c.ends[ip]); free(c.eg[ip]); free(c.ev[ip]);
    }
    for (int64_t e = 0; e < tot_ent; e++) colsum[eg[e]] += ev[e];
    /* work-balanced row blocks, src/kernels.rs:262-281 */
    uint64_t *work = (uint64_t *)calloc((size_t)(d > 0 ? d : 1), sizeof(uint64_t));
    for (int64_t w = 0; w < tot_rows; w++) {
        int64_t len = starts[w + 1] - starts[w];
        for (int64_t k = 0; k < len; k++) work[eg[starts[w] + k]] += (uint64_t)(len - k);
    }
    uint64_t total = 0;
    for (int64_t g = 0; g < d; g++) total += work[g];
    int64_t parts_n = (int64_t)n_threads * 2;
    if (parts_n < 1) parts_n = 1;
    int64_t *bounds = (int64_t *)malloc(sizeof(int64_t) * (size_t)(parts_n + 2));
    int64_t nb = 0;
    bounds[nb++] = 0;
    uint64_t acc = 0;
    for (int64_t g = 0; g < d; g++) {
        acc += work[g];
        if (acc * (uint64_t)parts_n >= total * (uint64_t)nb && nb < parts_n && g + 1 < d) bounds[nb++] = g + 1;
    }
    bounds[nb++] = d;
    /* dedup consecutive equal bounds */
    int64_t nd = 0;
    for (int64_t i = 0; i < nb; i++) if (nd == 0 || bounds[nd - 1] != bounds[i]) bounds[nd++] = bounds[i];
    gb_ctx b = {starts, tot_rows + 1, eg, ev, bounds, d, gram};
    run_pool(n_threads, nd - 1, gb_block, &b);
    free(bounds); free(work); free(starts); free(eg); free(ev);
    free(c.ends); free(c.n_rows); free(c.eg); free(c.ev); free(c.n_ent); free(parts); free(sp);
    return 0;
}

/* ------------------------------------------------------------------ project
 * src/kernels.rs:352-371 */
typedef struct {
    const oc_chunk *v; const span_t *sp; const part_t *parts; int64_t maxlen;
    const int32_t *sub_map; const oc_transform *t; const double *vv; int64_t k;
    int64_t *rows; double *acc; /* per span */
} pj_ctx;

static void pj_part(void *c_, int64_t ip) {
    pj_ctx *c = (pj_ctx *)c_;
    const part_t *pt = &c->parts[ip];
    uint32_t *bg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)c->maxlen);
    float *bx = (float *)malloc(sizeof(float) * (size_t)c->maxlen);
    int64_t k = c->k;
    for (int64_t i = pt->first; i < pt->last; i++) {
        int64_t nb;
        int64_t row = cell_entries(c->v, &c->sp[i], bg, bx, &nb);
        c->rows[i] = row;
        if (row < 0) continue;
        double *a = c->acc + (size_t)i * (size_t)k;
        for (int64_t j = 0; j < k; j++) a[j] = 0.0;
        for (int64_t e = 0; e < nb; e++) {
            int32_t m = c->sub_map[bg[e]];
            if (m >= 0) {
                double s = tf_apply(c->t, m, bx[e]);
                const double *vr = c->vv + (size_t)m * (size_t)k;
                for (int64_t j = 0; j < k; j++) a[j] += s * vr[j];
            }
        }
    }
    free(bg); free(bx);
}

int oc_project(const oc_chunk *v, int n_threads, const int32_t *sub_map, int scale, const double *mean,
               const double *std, double max_value, const double *loadings, int64_t k, float *out) {
    oc_transform t = {scale, mean, std, max_value};
    int64_t ns, np;
    span_t *sp = cell_spans(v, &ns);
    part_t *parts = make_parts(v, sp, ns, n_threads, &np);
    pj_ctx c;
    c.v = v; c.sp = sp; c.parts = parts; c.maxlen = max_span_len(sp, ns); c.sub_map = sub_map; c.t = &t;
    c.vv = loadings; c.k = k;
    c.rows = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ns > 0 ? ns : 1));
    c.acc = (double *)malloc(sizeof(double) * (size_t)((ns > 0 ? ns : 1) * (k > 0 ? k : 1)));
    run_pool(n_threads, np, pj_part, &c);
    for (int64_t ip = 0; ip < np; ip++)
        for (int64_t i = parts[ip].first; i < parts[ip].last; i++) {
            int64_t r = c.rows[i];
            if (r < 0) continue;
            for (int64_t j = 0; j < k; j++) out[r * k + j] += (float)c.acc[i * k + j];
        }
    free(c.rows); free(c.acc); free(parts); free(sp);
    return 0;
}

/* ------------------------------------------------------------------ materialize
 * src/kernels.rs:123-139 (only used to check the lazy transform). */
int64_t oc_materialize(const oc_chunk *v, int n_threads, uint32_t *rows, uint32_t *genes, float *vals, int64_t cap) {
    (void)n_threads; /* parts are concatenated in order: a sequential walk gives the same output */
    int64_t ns;
    span_t *sp = cell_spans(v, &ns);
    int64_t maxlen = max_span_len(sp, ns);
    uint32_t *bg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)maxlen);
    float *bx = (float *)malloc(sizeof(float) * (size_t)maxlen);
    int64_t n = 0;
    for (int64_t i = 0; i < ns; i++) {
        int64_t nb;
        int64_t row = cell_entries(v, &sp[i], bg, bx, &nb);
        if (row < 0) continue;
        for (int64_t e = 0; e < nb; e++) {
            if (n < cap) { rows[n] = (uint32_t)row; genes[n] = bg[e]; vals[n] = bx[e]; }
            n++;
        }
    }
    free(bg); free(bx); free(sp);
    return n;
}

/* ------------------------------------------------------------------ group_gene_sums
 * src/kernels.rs:388-442.  The reference materialises the chunk and lets
 * each thread own a block of genes, walking the entries in order; every
 * (group, gene) total is therefore an entry-order sum, which a sequential
 * walk reproduces.  clip (n_groups x nv) may be NULL, sumsq / nnz too. */
int oc_group_gene_sums(const oc_chunk *v, const uint32_t *group_of_row, int64_t nv, const double *clip, double *sum,
                       double *sumsq, double *nnz) {
    int64_t ns;
    span_t *sp = cell_spans(v, &ns);
    int64_t maxlen = max_span_len(sp, ns);
    uint32_t *bg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)maxlen);
    float *bx = (float *)malloc(sizeof(float) * (size_t)maxlen);
    for (int64_t i = 0; i < ns; i++) {
        int64_t nb;
        int64_t row = cell_entries(v, &sp[i], bg, bx, &nb);
        if (row < 0) continue;
        uint32_t grp = group_of_row[row];
        if (grp == 0xffffffffu) continue;
        for (int64_t e = 0; e < nb; e++) {
            int64_t at = (int64_t)grp * nv + bg[e];
            double x = (double)bx[e];
            if (clip && clip[at] < x) x = clip[at];
            sum[at] += x;
            if (sumsq) sumsq[at] += x * x;
            if (nnz) nnz[at] += 1.0;
        }
    }
    free(bg); free(bx); free(sp);
    return 0;
}

/* ------------------------------------------------------------------ knn
 * src/knn.rs: exact k nearest neighbours (self excluded) of the rows of an
 * n x d f32 matrix.  Distances follow sq_dist (src/knn.rs:48-66): f32
 * differences squared into eight partial sums over 8-wide chunks, partials
 * added in order, remaining coordinates one by one, no contraction (built
 * with -ffp-contract=off); the k best by (distance, index) after the square
 * root, as the reference's final re-sort (src/knn.rs:357-366).  Exhaustive
 * for every n: the exact answer the reference's brute force approximates
 * through GEMM-tile distances for its candidate selection. */
static float knn_sq(const float *a, const float *b, int64_t d) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t full = d - d % 8;
    for (int64_t c = 0; c < full; c += 8)
        for (int l = 0; l < 8; l++) {
            float t = a[c + l] - b[c + l];
            acc[l] += t * t;
        }
    float s = 0.0f;
    for (int l = 0; l < 8; l++) s += acc[l];
    for (int64_t j = full; j < d; j++) {
        float t = a[j] - b[j];
        s += t * t;
    }
    return s;
}

typedef struct {
    const float *x;
    int64_t n, d, k;
    uint32_t *idx;
    float *dist;
} knn_job;

static void knn_rows(void *c_, int64_t i) {
    knn_job *c = (knn_job *)c_;
    const int64_t k = c->k;
    float *bd = c->dist + i * k;
    uint32_t *bi = c->idx + i * k;
    for (int64_t j = 0; j < k; j++) { bd[j] = INFINITY; bi[j] = 0xffffffffu; }
    for (int64_t j = 0; j < c->n; j++) {
        if (j == i) continue;
        float s = knn_sq(c->x + i * c->d, c->x + j * c->d, c->d);
        if (!(s < bd[k - 1])) continue;
        int64_t p = k - 1;
        while (p > 0 && bd[p - 1] > s) { bd[p] = bd[p - 1]; bi[p] = bi[p - 1]; p--; }
        bd[p] = s;
        bi[p] = (uint32_t)j;
    }
    for (int64_t j = 0; j < k; j++) if (bi[j] != 0xffffffffu) bd[j] = sqrtf(bd[j]);
    for (int64_t j = 1; j < k; j++) {  /* (distance, index) order */
        float dj = bd[j];
        uint32_t ij = bi[j];
        int64_t p = j;
        while (p > 0 && (bd[p - 1] > dj || (bd[p - 1] == dj && bi[p - 1] > ij))) { bd[p] = bd[p - 1]; bi[p] = bi[p - 1]; p--; }
        bd[p] = dj;
        bi[p] = ij;
    }
}

int oc_knn(const float *x, int64_t n, int64_t d, int64_t k, uint32_t *idx, float *dist, int n_threads) {
    knn_job c = {x, n, d, k, idx, dist};
    run_pool(n_threads, n, knn_rows, &c);
    return 0;
}
