/*
 * CPU ORACLE -- test infrastructure only.
 *
 * Host-thread generator of the seeded synthetic count matrices (the same
 * per-(cell, gene) draw as the product's GPU generator, one shared
 * definition in crest_b200/csrc/synth_core.h), so tests and the CPU
 * baseline get their inputs without loading the product library.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

#include "synth_core.h"

typedef struct {
    int64_t n_cells, n_genes;
    int32_t n_clusters;
    double dispersion;
    uint64_t seed;
    const double *prob;    /* [n_clusters x n_genes] */
    const int32_t *labels; /* [n_cells] */
    const double *lib;     /* [n_cells] */
} oc_synth_params;

typedef struct {
    const oc_synth_params *p;
    int64_t c0, c1;
    int64_t *row_nnz;
    const int64_t *indptr;
    uint32_t *indices;
    float *data;
} synth_job;

static void *synth_rows(void *arg) {
    const synth_job *j = (const synth_job *)arg;
    const oc_synth_params *p = j->p;
    const double phi = p->dispersion, r = 1.0 / phi;
    for (int64_t c = j->c0; c < j->c1; ++c) {
        const double lib = p->lib[c];
        const double *pr = p->prob + (int64_t)p->labels[c] * p->n_genes;
        int64_t at = j->indices ? j->indptr[c] : 0, cnt = 0;
        for (int64_t g = 0; g < p->n_genes; ++g) {
            const uint32_t k = syn_count(lib * pr[g], phi, r, syn_uniform(p->seed, (uint64_t)c, (uint64_t)g));
            if (!k) continue;
            if (j->indices) {
                j->indices[at] = (uint32_t)g;
                j->data[at] = (float)k;
                ++at;
            }
            ++cnt;
        }
        if (!j->indices) j->row_nnz[c] = cnt;
    }
    return NULL;
}

/* indices == NULL: row_nnz[c] = non-zeros of cell c.  Otherwise indptr
 * (n_cells + 1, from those counts) is given and indices / data are filled
 * in gene order.  Returns 0, or -22 for bad parameters. */
int oc_synth(const oc_synth_params *p, int64_t *row_nnz, const int64_t *indptr, uint32_t *indices, float *data,
             int threads) {
    if (!p || !p->prob || !p->labels || !p->lib || !(p->dispersion > 0.0)) return -22;
    if (indices ? (!indptr || !data) : !row_nnz) return -22;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    synth_job jobs[256];
    const int64_t per = (p->n_cells + threads - 1) / threads;
    int n = 0;
    for (int t = 0; t < threads; ++t) {
        const int64_t a = t * per, b = a + per < p->n_cells ? a + per : p->n_cells;
        if (a >= b) break;
        jobs[n] = (synth_job){p, a, b, row_nnz, indptr, indices, data};
        ++n;
    }
    for (int t = 1; t < n; ++t) pthread_create(&th[t], NULL, synth_rows, &jobs[t]);
    if (n > 0) synth_rows(&jobs[0]);
    for (int t = 1; t < n; ++t) pthread_join(th[t], NULL);
    return 0;
}
