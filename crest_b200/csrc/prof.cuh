// Optional per-kernel device timing: CUDA events recorded around each launch
// on the launching stream, accumulated by kernel name.  Off by default; the
// benchmark turns it on to measure kernel durations inside its timed region.
#pragma once

#include <cuda_runtime.h>

namespace crest {
namespace prof {

bool enabled();

// Records a start event now and a stop event when it goes out of scope.
class Scope {
  public:
    Scope(const char *name, cudaStream_t st);
    ~Scope();

  private:
    const char *name_ = nullptr;
    cudaEvent_t a_ = nullptr;
    cudaStream_t st_;
};

}  // namespace prof
}  // namespace crest
