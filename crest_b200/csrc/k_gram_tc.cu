// Product-form Gram: split-BF16 (bf16x3) SYRK on the tcgen05 tensor cores.
#include "kernels.cuh"

namespace crest {

int syrk_bf16x3_fold(const GramWork &w, int64_t m, const DevScale &t, double *gram, cudaStream_t st) {
    (void)w; (void)m; (void)t; (void)gram; (void)st;
    set_error("the bf16x3 tensor-core Gram is not available in this build");
    return CREST_EINVAL;
}

}  // namespace crest
