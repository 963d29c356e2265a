// Chemistry-step kernels, variant "fast": analytic Jacobian, FP64 LU.
#include "chem_kernels.cuh"

namespace nrg {

void upload_mechanism_fast(const DevMech& m, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_mech, &m, sizeof(DevMech), 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_chem_fast(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                              unsigned long long* counters, cudaStream_t s, int n_int, bool spec, int n_species,
                              int n_reactions) {
  // the mechanism's inert species (third bodies only) are not integrated;
  // spec: the parsed mechanism matches the generated specialised code
  if (n_species == 9 && n_reactions == 24) {
    if (n_int == gen::kSpecN && spec)
      return launch_variant<9, gen::kSpecN, 24, kJacAnalytic, double, true>(a, cfg, queue, counters, s);
    if (n_int == 8) return launch_variant<9, 8, 24, kJacAnalytic, double, false>(a, cfg, queue, counters, s);
    if (n_int == 9) return launch_variant<9, 9, 24, kJacAnalytic, double, false>(a, cfg, queue, counters, s);
  }
  if (n_species == 9 && n_reactions == 28 && n_int == 8)
    return launch_grid<9, 8, 28, kJacAnalytic, double>(a, cfg, queue, counters, s);
  if (n_species == 10 && n_reactions == 24 && n_int == 10)
    return launch_grid<10, 10, 24, kJacAnalytic, double>(a, cfg, queue, counters, s);
  if (n_species == 13 && n_reactions == 71 && n_int == 13)
    return launch_grid<13, 13, 71, kJacAnalytic, double>(a, cfg, queue, counters, s);
  return cudaErrorNotSupported;
}

}  // namespace nrg
