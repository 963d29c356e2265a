// Chemistry-step kernels, variant "fast": analytic Jacobian, FP64 LU.
#include "chem_kernels.cuh"

namespace nrg {

void upload_mechanism_fast(const DevMech& m, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_mech, &m, sizeof(DevMech), 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_chem_fast(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                              unsigned long long* counters, cudaStream_t s, int n_int, int spec, int n_species,
                              int n_reactions) {
  // the mechanism's inert species (third bodies only) are not integrated;
  // spec: the generated specialised code the parsed mechanism matches (0: none)
  constexpr int kA = kJacAnalytic;
  if (n_species == 9 && n_reactions == 24) {
    if (n_int == 8 && spec == kSpecKeromnes)
      return launch_variant<9, 8, 24, kA, double, kSpecKeromnes>(a, cfg, queue, counters, s);
    if (n_int == 8) return launch_variant<9, 8, 24, kA, double, 0>(a, cfg, queue, counters, s);
    if (n_int == 9) return launch_variant<9, 9, 24, kA, double, 0>(a, cfg, queue, counters, s);
  }
  if (n_species == 9 && n_reactions == 28 && n_int == 8)
    return spec == kSpecZhang ? launch_grid<9, 8, 28, kA, double, kSpecZhang>(a, cfg, queue, counters, s)
                              : launch_grid<9, 8, 28, kA, double>(a, cfg, queue, counters, s);
  if (n_species == 10 && n_reactions == 24 && n_int == 10)
    return spec == kSpecTereza ? launch_grid<10, 10, 24, kA, double, kSpecTereza>(a, cfg, queue, counters, s)
                               : launch_grid<10, 10, 24, kA, double>(a, cfg, queue, counters, s);
  if (n_species == 13 && n_reactions == 71 && n_int == 13)
    return spec == kSpecKonnov ? launch_grid<13, 13, 71, kA, double, kSpecKonnov>(a, cfg, queue, counters, s)
                               : launch_grid<13, 13, 71, kA, double>(a, cfg, queue, counters, s);
  if (n_species == 17 && n_reactions == 25 && n_int == 15)
    return spec == kSpecAcetylene ? launch_grid<17, 15, 25, kA, double, kSpecAcetylene>(a, cfg, queue, counters, s)
                                  : launch_grid<17, 15, 25, kA, double>(a, cfg, queue, counters, s);
  return cudaErrorNotSupported;
}

}  // namespace nrg
