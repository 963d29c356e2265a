// Species predictor of the low-Mach solver (transport.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nrg {

constexpr int kPredictorMaxSpecies = 16;
constexpr int kPredictorMaxParticlePhases = 4;

// Cell fields: 0-based (i, j, k) with the ghost layer, extents e[d] = n[d] + 2
// for active directions and 1 otherwise, cell at i + e0 * (j + e1 * k),
// species s at [s * ld + cell].  Face velocity of component d: the
// reference's face field v_f%pr(d)%cells(dims, 0:n+2, ...), element
// (c, i, j, k) at c + dims * (i + f0 * (j + f1 * k)), f[d] = e[d] + 1 for
// active directions; face i is the low face of cell i.  Interior: lo..hi.
struct PredictorArgs {
  int dims = 0, coord = 0, n_part = 0;
  long e[3] = {1, 1, 1}, f[3] = {1, 1, 1}, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  long ld = 0;
  double dx = 0.0, inv_dx = 0.0, dt = 0.0;
  double W[kPredictorMaxSpecies] = {};
  const double* rho = nullptr;
  const double* Y = nullptr;
  const double* v_f[3] = {nullptr, nullptr, nullptr};
  const double* x_center = nullptr;
  const int8_t* bc = nullptr;
  const double* Y_prod_diff = nullptr;
  const double* Y_prod_chem = nullptr;
  const double* Y_prod_part[kPredictorMaxParticlePhases] = {};
  double* rho_old = nullptr;
  double* Y_old = nullptr;
  double* rho_int = nullptr;
  double* Y_int = nullptr;
  // written by the commit kernel
  double* rho_out = nullptr;
  double* Y_out = nullptr;
};

// Fills e, f, lo, hi from the interior cell counts; false on bad sizes.
bool predictor_grid(PredictorArgs& a, int dims, const int n_cells[3]);
// Both kernels on stream s; cudaErrorNotSupported for a species count
// without an instantiation.
cudaError_t launch_species_predictor(int n_species, const PredictorArgs& a, cudaStream_t s);
// Interior cells the kernels touch (with the ghost layer excluded).
long predictor_interior_cells(const PredictorArgs& a);

}  // namespace nrg
