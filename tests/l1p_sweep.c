/* Test helper: compares crest_log1pf (the GPU path's restatement) with the
 * platform libm log1pf over a range of float bit patterns, multi-threaded. */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <string.h>
#include "log1pf_libm.h"

typedef struct { uint64_t lo, hi, bad; uint32_t first_bad; } job_t;

static void *run(void *p) {
    job_t *j = (job_t *)p;
    for (uint64_t b = j->lo; b < j->hi; b++) {
        float x = l1p_from((uint32_t)b);
        float r = log1pf(x), m = crest_log1pf(x);
        if (l1p_bits(r) != l1p_bits(m) && !(isnan(r) && isnan(m))) {
            if (j->bad == 0) j->first_bad = (uint32_t)b;
            j->bad++;
        }
    }
    return NULL;
}

/* returns the number of mismatching inputs in [lo, hi); *first gets the first one */
uint64_t l1p_sweep(uint64_t lo, uint64_t hi, int threads, uint32_t *first) {
    pthread_t th[64];
    job_t js[64];
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    uint64_t span = (hi - lo + (uint64_t)threads - 1) / (uint64_t)threads;
    for (int i = 0; i < threads; i++) {
        js[i].lo = lo + span * (uint64_t)i;
        js[i].hi = js[i].lo + span > hi ? hi : js[i].lo + span;
        if (js[i].lo > hi) js[i].lo = hi;
        js[i].bad = 0; js[i].first_bad = 0;
        pthread_create(&th[i], NULL, run, &js[i]);
    }
    uint64_t bad = 0;
    *first = 0;
    for (int i = 0; i < threads; i++) {
        pthread_join(th[i], NULL);
        if (js[i].bad && bad == 0) *first = js[i].first_bad;
        bad += js[i].bad;
    }
    return bad;
}
