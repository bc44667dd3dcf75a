// Per-kernel device timing (see prof.cuh) and its C ABI.
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "prof.cuh"

namespace crest {
namespace prof {
namespace {

struct Pending {
    std::string name;
    cudaEvent_t a, b;
};
struct Entry {
    std::string name;
    long long launches = 0;
    double total_ms = 0.0, max_ms = 0.0;
};

std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free;
std::vector<Entry> g_table;

cudaEvent_t take() {
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void collect_locked() {
    for (auto &p : g_pending) {
        cudaEventSynchronize(p.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        Entry *e = nullptr;
        for (auto &x : g_table)
            if (x.name == p.name) e = &x;
        if (!e) {
            g_table.push_back(Entry{p.name});
            e = &g_table.back();
        }
        e->launches += 1;
        e->total_ms += ms;
        if (ms > e->max_ms) e->max_ms = ms;
        g_free.push_back(p.a);
        g_free.push_back(p.b);
    }
    g_pending.clear();
}

}  // namespace

bool enabled() { return g_on; }

Scope::Scope(const char *name, cudaStream_t st) : st_(st) {
    if (!g_on) return;
    std::lock_guard<std::mutex> l(g_mu);
    name_ = name;
    a_ = take();
    cudaEventRecord(a_, st);
}

Scope::~Scope() {
    if (!a_) return;
    std::lock_guard<std::mutex> l(g_mu);
    cudaEvent_t b = take();
    cudaEventRecord(b, st_);
    g_pending.push_back(Pending{name_, a_, b});
}

}  // namespace prof
}  // namespace crest

using namespace crest::prof;

extern "C" {

/* Turn per-kernel timing on (1) or off (0); either way the table is cleared. */
int crest_profile_enable(int on) {
    std::lock_guard<std::mutex> l(g_mu);
    collect_locked();
    g_table.clear();
    g_on = on != 0;
    return 0;
}

/* Number of distinct kernels timed so far (waits for pending launches). */
int crest_profile_count(void) {
    std::lock_guard<std::mutex> l(g_mu);
    collect_locked();
    return (int)g_table.size();
}

/* Entry i: kernel name, launches, total and longest launch time (ms). */
int crest_profile_entry(int i, char *name, int cap, long long *launches, double *total_ms, double *max_ms) {
    std::lock_guard<std::mutex> l(g_mu);
    collect_locked();
    if (i < 0 || i >= (int)g_table.size()) return CREST_EINVAL;
    const Entry &e = g_table[i];
    if (name && cap > 0) {
        strncpy(name, e.name.c_str(), (size_t)cap - 1);
        name[cap - 1] = 0;
    }
    if (launches) *launches = e.launches;
    if (total_ms) *total_ms = e.total_ms;
    if (max_ms) *max_ms = e.max_ms;
    return CREST_OK;
}

}  // extern "C"
