// Chemistry-step kernels, variant "mixed": analytic Jacobian, FP32 LU with FP64 residual refinement.
#include "chem_kernels.cuh"

namespace nrg {

void upload_mechanism_mixed(const DevMech& m, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_mech, &m, sizeof(DevMech), 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_chem_mixed(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                              unsigned long long* counters, cudaStream_t s, int n_int, int spec, int n_species,
                              int n_reactions) {
  // the mechanism's inert species (third bodies only) are not integrated;
  // spec: the generated specialised code the parsed mechanism matches (0: none)
  if (n_species != 9 || n_reactions != 24) return cudaErrorNotSupported;
  if (n_int == 8 && spec == kSpecKeromnes)
    return launch_variant<9, 8, 24, kJacAnalytic, float, kSpecKeromnes>(a, cfg, queue, counters, s);
  if (n_int == 8) return launch_variant<9, 8, 24, kJacAnalytic, float, 0>(a, cfg, queue, counters, s);
  if (n_int == 9) return launch_variant<9, 9, 24, kJacAnalytic, float, 0>(a, cfg, queue, counters, s);
  return cudaErrorNotSupported;
}

}  // namespace nrg
