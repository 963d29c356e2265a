// Mixture-averaged diffusion coefficients on the device: the per-cell
// transport-property kernel of the Fickian diffusion solver
// (fickean_diffusion_solver.f90:358-395, calculate_diffusivity_coeff, over
// thermophysical_properties_class.f90:560-577 calculate_omega, :737-762
// binary_diffusion_coefficient, :768-814
// mixture_averaged_diffusion_coefficients).
//
// One thread per cell.  The collision integral is evaluated once per distinct
// sqrt(eps_i * eps_j) of the mechanism (equal inputs give equal bits; the
// H2/air decks repeat well depths, e.g. 36 pairs but 17 distinct values for
// KEROMNES).  The binary coefficients are then formed pair by pair in the
// order i < j and each one is added to both species' accumulators at once:
// for species i the contributions then arrive in increasing partner order,
// which is the reference's loop order, so only the pair's value is ever held
// (no N x N matrix per cell).  The accumulators and mass fractions live in
// shared memory [species][thread].  Compiled with --fmad=false; pow and exp
// are CUDA's, so results match the host restatement to a few ulp, not bit for
// bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "diffusion.hpp"

namespace nrg {

namespace {

// calculate_omega(T_red, 1, 1): Neufeld, Janzen and Aziz (1972) fit of the
// (1,1) collision integral with the coefficients set in set_properties.
__device__ __noinline__ double omega11(double T_red) {
  const double c1 = 1.06036, c2 = 0.15610, c3 = 0.19300, c4 = 0.47635, c5 = 1.03587, c6 = 1.52996,
               c7 = 1.76474, c8 = 3.89411;
  if (T_red < 70.0) return c1 / pow(T_red, c2) + c3 / exp(c4 * T_red) + c5 / exp(c6 * T_red) + c7 / exp(c8 * T_red);
  return c1 / pow(T_red, c2);
}

}  // namespace

__global__ void __launch_bounds__(128) k_mixture_diffusivity(DiffusivityArgs a) {
  extern __shared__ double sm[];
  const int t = threadIdx.x, BS = blockDim.x, N = a.N;
  const long c = (long)blockIdx.x * BS + t;
  if (c >= a.n) return;
  double* sY = sm + t;
  double* sA = sm + (long)N * BS + t;
  double* sO = sm + (long)2 * N * BS + t;
  const double T = a.T[c], p = a.p[c], mm = a.m_mix[c];
  const bool valid = (!a.bc || a.bc[c] == 0) && N > 0 && T > 0.0 && p > 0.0 && mm > 0.0;
  if (!valid) {
    for (int k = 0; k < N; ++k) a.D[(long)k * a.ld + c] = 0.0;
    return;
  }
  for (int k = 0; k < N; ++k) {
    sY[k * BS] = a.Y[(long)k * a.ld + c];
    sA[k * BS] = 0.0;
  }
  const double T15 = pow(T, 1.5);
  for (int u = 0; u < a.n_uniq; ++u) sO[u * BS] = omega11(T / a.uniq_sq[u]);
  int q = 0;
  for (int i = 0; i < N - 1; ++i) {
    for (int j = i + 1; j < N; ++j, ++q) {
      if (!a.pair_ok[q]) continue;  // bdc <= 0 or a well depth <= 0: D_ij = 0
      const double om = sO[a.pair_u[q] * BS];
      if (om <= 0.0) continue;
      const double Dij = a.bdc[q] * T15 / (p * om);
      if (Dij <= 0.0 || a.W[i] <= 0.0 || a.W[j] <= 0.0) continue;
      const double Yi = sY[i * BS], Yj = sY[j * BS];
      double ai = sA[i * BS];
      ai = ai + (1.0 - Yi) * a.W[i] * Yj / (Dij * a.W[j]);
      ai = ai + Yi * Yj / Dij;
      sA[i * BS] = ai;
      double aj = sA[j * BS];
      aj = aj + (1.0 - Yj) * a.W[j] * Yi / (Dij * a.W[i]);
      aj = aj + Yj * Yi / Dij;
      sA[j * BS] = aj;
    }
  }
  for (int k = 0; k < N; ++k) {
    const double Yk = sY[k * BS], acc = sA[k * BS];
    double d = 0.0;
    if (a.W[k] > 0.0 && acc > 1.0e-10) d = (1.0 - Yk) * a.W[k] / (acc * mm);
    a.D[(long)k * a.ld + c] = d;
  }
}

cudaError_t launch_mixture_diffusivity(const DiffusivityArgs& a, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const size_t per_thread = (size_t)(2 * a.N + a.n_uniq) * sizeof(double);
  const int BS = per_thread * 128 <= 48 * 1024 ? 128 : 64;
  const size_t smem = per_thread * BS;
  cudaError_t e = cudaFuncSetAttribute(k_mixture_diffusivity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long grid = (a.n + BS - 1) / BS;
  if (grid > 0x7fffffffL) return cudaErrorInvalidValue;
  k_mixture_diffusivity<<<(unsigned)grid, BS, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace nrg
