// Chemistry-step kernels, variant "ref": finite-difference Jacobian as the reference (DDPST MITER=2), FP64 LU.
#include "chem_kernels.cuh"

namespace nrg {

void upload_mechanism_ref(const DevMech& m, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_mech, &m, sizeof(DevMech), 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_chem_ref(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                              unsigned long long* counters, cudaStream_t s) {
  return launch_variant<9, 9, 24, kJacFD, double, false>(a, cfg, queue, counters, s);
}

}  // namespace nrg
