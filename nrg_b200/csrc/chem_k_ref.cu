// Chemistry-step kernels, variant "ref": finite-difference Jacobian as the reference (DDPST MITER=2), FP64 LU.
#include "chem_kernels.cuh"

namespace nrg {

void upload_mechanism_ref(const DevMech& m, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_mech, &m, sizeof(DevMech), 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_chem_ref(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                              unsigned long long* counters, cudaStream_t s, int n_species, int n_reactions) {
  // H2/air mechanisms of the reference's task set-ups: KEROMNES (all shapes),
  // ZHANG, TEREZA, KONNOV (thread-per-cell grid)
  if (n_species == 9 && n_reactions == 24)
    return launch_variant<9, 9, 24, kJacFD, double, 0>(a, cfg, queue, counters, s);
  if (n_species == 9 && n_reactions == 28) return launch_grid<9, 9, 28, kJacFD, double>(a, cfg, queue, counters, s);
  if (n_species == 10 && n_reactions == 24)
    return launch_grid<10, 10, 24, kJacFD, double>(a, cfg, queue, counters, s);
  if (n_species == 13 && n_reactions == 71)
    return launch_grid<13, 13, 71, kJacFD, double>(a, cfg, queue, counters, s);
  if (n_species == 17 && n_reactions == 25)
    return launch_grid<17, 17, 25, kJacFD, double>(a, cfg, queue, counters, s);
  return cudaErrorNotSupported;
}

}  // namespace nrg
