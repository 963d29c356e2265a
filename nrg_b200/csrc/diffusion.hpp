// Mixture-averaged diffusion coefficients (diffusion.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nrg {

constexpr int kDiffMaxSpecies = 16;
constexpr int kDiffMaxPairs = kDiffMaxSpecies * (kDiffMaxSpecies - 1) / 2;

// Flat cells, species-major fields at [k * ld + c].  Pair tables in the order
// (0,1), (0,2), ..., (1,2), ...: bdc = binary diffusivity constant,
// pair_ok = bdc > 0 and both well depths > 0, pair_u = index of the pair's
// sqrt(eps_i * eps_j) in uniq_sq (the distinct values, first-seen order):
// pairs with equal values share one collision-integral evaluation.
struct DiffusivityArgs {
  long n = 0, ld = 0;
  int N = 0;
  const double* T = nullptr;
  const double* p = nullptr;
  const double* Y = nullptr;
  const double* m_mix = nullptr;
  const int8_t* bc = nullptr;
  double* D = nullptr;
  double W[kDiffMaxSpecies] = {};
  double bdc[kDiffMaxPairs] = {};
  double uniq_sq[kDiffMaxPairs] = {};
  int n_uniq = 0;
  unsigned char pair_ok[kDiffMaxPairs] = {};
  unsigned char pair_u[kDiffMaxPairs] = {};
};

cudaError_t launch_mixture_diffusivity(const DiffusivityArgs& a, cudaStream_t s);

}  // namespace nrg
