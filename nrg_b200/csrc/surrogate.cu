// Gated MLP surrogate (placeholder until the tensor-core kernels land).
#include "surrogate.hpp"

namespace nrg {

struct Surrogate {
  bool ready = false;
};

Surrogate* surrogate_create(const DevMech&) { return new Surrogate(); }
void surrogate_destroy(Surrogate* s) { delete s; }
bool surrogate_ready(const Surrogate* s) { return s && s->ready; }

cudaError_t surrogate_step(Surrogate*, const StepArgs&, const LaunchCfg&, int*, unsigned long long*,
                           cudaStream_t, const FallbackFn&) {
  return cudaErrorNotSupported;
}

}  // namespace nrg
