// Species predictor of the low-Mach solver on the device: the explicit
// convective update of rho*Y_k that brackets the chemistry step in the
// operator split (fds_low_mach_solver.f90:785-954,
// calculate_interm_Y_predictor, with charm_face_value :4979-5009 and
// eos_corrected_species_face_vector :5011-5070), so that rho, Y and the
// chemistry sources stay on the GPU across the split.
//
// Two kernels.  k_predictor: a CTA takes a TX x TY tile of cells of one
// k-plane, stages rho*Y_k, sum_k rho*Y_k / W_k and the most abundant species
// of the tile and a two-cell halo in shared memory, computes every x and y
// face of the tile once (CHARM-limited face values with the equation-of-state
// correction, times the face velocity; both cells of a face use the same
// bits), then each thread updates its cell: rho*Y_k + dt * (flux divergence
// + sources), clipped at zero and renormalised into rho_int / Y_int, with
// rho_old / Y_old = the old values.  z faces (3-D) are computed per cell
// from global memory.  k_predictor_commit: rho = rho_int, Y = Y_int, after
// every cell's fluxes have seen the old values.  Operations are the
// reference's, in its order, never fused (the file is compiled with
// --fmad=false), so results equal the oracle's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "transport.hpp"

namespace nrg {

namespace {

constexpr int kTX = 32;

// charm_face_value without branches: both candidates are formed from safe
// operands and the reference's choice selects one, so the selected value has
// the reference's bits and the N + 1 face values of a face can overlap.
__device__ __forceinline__ double charm(double a0, double a1, double a2, double a3, double v) {
  const bool pos = v > 0.0;
  const double phi_loc = a2 - a1;
  const double up_pos = a1 - a0, up_neg = a3 - a2;
  const double phi_up = pos ? up_pos : up_neg;
  const bool has_loc = phi_loc != 0.0;
  const double r = has_loc ? phi_up / (has_loc ? phi_loc : 1.0) : 0.0;
  const bool lim = r > 1.0e-10;
  const double s = 1.0 / (lim ? r : 1.0);
  const double B_r = lim ? s * (3.0 * s + 1.0) / (s + 1.0) / (s + 1.0) : 0.0;
  const double h = B_r * 0.5 * phi_up;
  return pos ? a1 + h : a2 - h;
}

// Per staged cell: rho*Y_k, sum_k rho*Y_k / W_k (species order, from 0.0) and
// the index of the largest rho*Y_k (first of equals; -DBL_MAX start).
template <int N>
__device__ __forceinline__ void cell_terms(const PredictorArgs& a, long c, double* rY, double& row, int& gam) {
  const double rho = a.rho[c];
  row = 0.0;
  gam = 0;
  double mx = -DBL_MAX;
#pragma unroll
  for (int s = 0; s < N; ++s) {
    rY[s] = rho * a.Y[(long)s * a.ld + c];
    row = row + rY[s] / a.W[s];
    if (rY[s] > mx) {
      mx = rY[s];
      gam = s;
    }
  }
}

// CHARM face fluxes with the EOS correction from four staged cells (low to
// high along the face normal) read through `at(n, s)`; upwind cell index 1 or
// 2 of the four for v > 0 or not.
template <int N, class RY, class ROW>
__device__ __forceinline__ void charm_face_flux(const double* W, RY at, ROW row_at, int gam, double v, double* F) {
  double phi[N];
#pragma unroll
  for (int s = 0; s < N; ++s) phi[s] = charm(at(0, s), at(1, s), at(2, s), at(3, s), v);
  const double row_face = charm(row_at(0), row_at(1), row_at(2), row_at(3), v);
  double q[N];
#pragma unroll
  for (int s = 0; s < N; ++s) q[s] = phi[s] / W[s];
  double sum_not_gamma = 0.0;
#pragma unroll
  for (int s = 0; s < N; ++s) sum_not_gamma = s != gam ? sum_not_gamma + q[s] : sum_not_gamma;
  double pg = 0.0;
#pragma unroll
  for (int s = 0; s < N; ++s)
    if (s == gam) pg = W[s] * (row_face - sum_not_gamma);
#pragma unroll
  for (int s = 0; s < N; ++s) F[s] = (s == gam ? pg : phi[s]) * v;
}

}  // namespace

template <int N, bool Z3>
__global__ void __launch_bounds__(256, Z3 ? 1 : (N == 9 ? 3 : 2)) k_predictor(PredictorArgs a) {
  extern __shared__ double sm[];
  const int TY = blockDim.y;
  const bool two_d = a.dims >= 2;
  const int RX = kTX + 4, RY = two_d ? TY + 4 : 1;
  const int nst = RX * RY;
  double* s_rY = sm;                     // [N][RY][RX]
  double* s_row = s_rY + N * nst;        // [RY][RX]
  double* s_fx = s_row + nst;            // [N][TY][kTX + 1]
  double* s_fy = s_fx + N * TY * (kTX + 1);  // [N][TY + 1][kTX]
  int* s_gam = reinterpret_cast<int*>(s_fy + (two_d ? N * (TY + 1) * kTX : 0));  // [RY][RX]

  const int tid = threadIdx.y * kTX + threadIdx.x, nthr = kTX * TY;
  const long i0 = a.lo[0] + (long)blockIdx.x * kTX;
  const long j0 = a.lo[1] + (long)blockIdx.y * TY;
  const long k = a.lo[2] + blockIdx.z;
  const long e0 = a.e[0], e1 = a.e[1];

  // stage the tile and its halo (cells outside the array stay unused): first
  // the raw rho and Y_k (loads only, so a thread's cells are all in flight at
  // once), then, by the same thread, rho*Y_k, sum rho*Y_k / W_k and the most
  // abundant species in place
#pragma unroll 2
  for (int q = tid; q < nst; q += nthr) {
    const int rx = q % RX, ry = q / RX;
    const long i = i0 - 2 + rx, j = two_d ? j0 - 2 + ry : j0;
    if (i < 0 || i >= e0 || j < 0 || j >= e1) continue;
    const long c = i + e0 * (j + e1 * k);
    s_row[q] = a.rho[c];
#pragma unroll
    for (int s = 0; s < N; ++s) s_rY[s * nst + q] = a.Y[(long)s * a.ld + c];
  }
  for (int q = tid; q < nst; q += nthr) {
    const int rx = q % RX, ry = q / RX;
    const long i = i0 - 2 + rx, j = two_d ? j0 - 2 + ry : j0;
    if (i < 0 || i >= e0 || j < 0 || j >= e1) continue;
    const double rho = s_row[q];
    double row = 0.0, mx = -DBL_MAX;
    int gam = 0;
#pragma unroll
    for (int s = 0; s < N; ++s) {
      const double rY = rho * s_rY[s * nst + q];
      s_rY[s * nst + q] = rY;
      row = row + rY / a.W[s];
      if (rY > mx) {
        mx = rY;
        gam = s;
      }
    }
    s_row[q] = row;
    s_gam[q] = gam;
  }
  __syncthreads();

  // faces, x then y in one job list: x face (fi, fj) is the low face of
  // cell (i0 + fi, j0 + fj), its four stencil cells are staged columns
  // fi .. fi + 3 of row fj + 2; y faces likewise along the rows
  const long f0 = a.f[0], f1 = a.f[1];
  const int nxf = (kTX + 1) * TY, nyf = two_d ? kTX * (TY + 1) : 0;
  for (int q = tid; q < nxf + nyf; q += nthr) {
    const bool xf = q < nxf;
    const int r = xf ? q : q - nxf;
    const int fi = xf ? r % (kTX + 1) : r % kTX, fj = xf ? r / (kTX + 1) : r / kTX;
    const long i = i0 + fi, j = j0 + fj;
    if (xf ? (i > a.hi[0] + 1 || j > a.hi[1]) : (i > a.hi[0] || j > a.hi[1] + 1)) continue;
    const int d = xf ? 0 : 1;
    const double v = a.v_f[d][d + a.dims * (i + f0 * (j + f1 * k))];
    const bool edge = xf ? (i == a.lo[0] || i == a.hi[0] + 1) : (j == a.lo[1] || j == a.hi[1] + 1);
    const int st = xf ? 1 : RX;
    const int b = xf ? (two_d ? fj + 2 : 0) * RX + fi : fj * RX + fi + 2;
    double* out = xf ? s_fx + fj * (kTX + 1) + fi : s_fy + fj * kTX + fi;
    const int ostride = xf ? TY * (kTX + 1) : (TY + 1) * kTX;
    double F[N];
    if (edge) {
      const int up = b + (v > 0.0 ? 1 : 2) * st;
#pragma unroll
      for (int s = 0; s < N; ++s) F[s] = s_rY[s * nst + up] * v;
    } else {
      charm_face_flux<N>(a.W, [&](int n, int s) { return s_rY[s * nst + b + n * st]; },
                         [&](int n) { return s_row[b + n * st]; }, s_gam[b + (v > 0.0 ? 1 : 2) * st], v, F);
    }
#pragma unroll
    for (int s = 0; s < N; ++s) out[s * ostride] = F[s];
  }
  __syncthreads();

  // cell update
  const int tx = threadIdx.x, ty = threadIdx.y;
  const long i = i0 + tx, j = j0 + ty;
  if (i > a.hi[0] || j > a.hi[1]) return;
  const long c = i + e0 * (j + e1 * k);
  if (a.bc && a.bc[c] != 0) return;
  double l1 = 1.0, l2 = 1.0, l3 = 1.0;
  if (a.coord == 1) {
    l1 = a.x_center[i] - 0.5 * a.dx;
    l2 = a.x_center[i];
    l3 = a.x_center[i] + 0.5 * a.dx;
  } else if (a.coord == 2) {
    const double l = a.x_center[i] - 0.5 * a.dx, m = a.x_center[i], r = a.x_center[i] + 0.5 * a.dx;
    l1 = l * l;
    l2 = m * m;
    l3 = r * r;
  }
  const int me = (two_d ? ty + 2 : 0) * RX + tx + 2;
  double rhs[N];
#pragma unroll
  for (int s = 0; s < N; ++s) {
    const double fr = s_fx[(s * TY + ty) * (kTX + 1) + tx + 1], fl = s_fx[(s * TY + ty) * (kTX + 1) + tx];
    double d = (fr * l3 - fl * l1) * a.inv_dx;
    if (a.coord != 0) d = d / l2;  // cartesian: l2 = 1, and x / 1 == x
    rhs[s] = 0.0 - d;
  }
  if (two_d) {
#pragma unroll
    for (int s = 0; s < N; ++s) {
      const double fr = s_fy[(s * (TY + 1) + ty + 1) * kTX + tx], fl = s_fy[(s * (TY + 1) + ty) * kTX + tx];
      rhs[s] = rhs[s] - (fr * 1.0 - fl * 1.0) * a.inv_dx;
    }
  }
  if (Z3) {
    // z faces from global memory: low face kf = k (cells k-1 | k), high face kf = k + 1
    const long pz = e0 * e1;
    double Fz[2][N];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const long kf = k + side;
      const double v = a.v_f[2][2 + a.dims * (i + f0 * (j + f1 * kf))];
      if (kf == a.lo[2] || kf == a.hi[2] + 1) {
        const long cu = c + (v > 0.0 ? kf - 1 - k : kf - k) * pz;
        const double rho = a.rho[cu];
#pragma unroll
        for (int s = 0; s < N; ++s) Fz[side][s] = rho * a.Y[(long)s * a.ld + cu] * v;
      } else {
        double rY[4][N], row[4];
        int gam[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) cell_terms<N>(a, c + (kf - 2 + n - k) * pz, rY[n], row[n], gam[n]);
        charm_face_flux<N>(a.W, [&](int n, int s) { return rY[n][s]; }, [&](int n) { return row[n]; },
                           gam[v > 0.0 ? 1 : 2], v, Fz[side]);
      }
    }
#pragma unroll
    for (int s = 0; s < N; ++s) rhs[s] = rhs[s] - (Fz[1][s] * 1.0 - Fz[0][s] * 1.0) * a.inv_dx;
  }
  double rYn[N];
  double summ = 0.0;
#pragma unroll
  for (int s = 0; s < N; ++s) {
    const long o = (long)s * a.ld + c;
    double x = s_rY[s * nst + me] + rhs[s] * a.dt;
    if (a.Y_prod_diff) x = x + a.Y_prod_diff[o] * a.dt;
    if (a.Y_prod_chem) x = x + a.Y_prod_chem[o] * a.dt;
    for (int p = 0; p < a.n_part; ++p) x = x + a.Y_prod_part[p][o] * a.dt;
    x = x > 0.0 ? x : 0.0;
    rYn[s] = x;
    summ = summ + x;
  }
  a.rho_old[c] = a.rho[c];
#pragma unroll
  for (int s = 0; s < N; ++s) a.Y_old[(long)s * a.ld + c] = a.Y[(long)s * a.ld + c];
  if (summ > DBL_MIN) {
    a.rho_int[c] = summ;
#pragma unroll
    for (int s = 0; s < N; ++s) a.Y_int[(long)s * a.ld + c] = rYn[s] / summ;
  }
}

}  // namespace nrg

namespace nrg {

// rho = rho_int, Y = Y_int on the interior cells with bc == 0
// (fds_low_mach_solver.f90:940-953; rho_old and Y_old were written by
// k_predictor from the same old values).
template <int N>
__global__ void k_predictor_commit(PredictorArgs a) {
  const long nx = a.hi[0] - a.lo[0] + 1, ny = a.hi[1] - a.lo[1] + 1, nz = a.hi[2] - a.lo[2] + 1;
  const long total = nx * ny * nz;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const long i = a.lo[0] + q % nx, j = a.lo[1] + (q / nx) % ny, k = a.lo[2] + q / (nx * ny);
    const long c = i + a.e[0] * (j + a.e[1] * k);
    if (a.bc && a.bc[c] != 0) continue;
    a.rho_out[c] = a.rho_int[c];
#pragma unroll
    for (int s = 0; s < N; ++s) a.Y_out[(long)s * a.ld + c] = a.Y_int[(long)s * a.ld + c];
  }
}

bool predictor_grid(PredictorArgs& a, int dims, const int n_cells[3]) {
  if (dims < 1 || dims > 3) return false;
  a.dims = dims;
  for (int d = 0; d < 3; ++d) {
    const bool act = d < dims;
    if (act && n_cells[d] < 1) return false;
    a.e[d] = act ? (long)n_cells[d] + 2 : 1;
    a.f[d] = act ? a.e[d] + 1 : 1;
    a.lo[d] = act ? 1 : 0;
    a.hi[d] = act ? n_cells[d] : 0;
  }
  return true;
}

long predictor_interior_cells(const PredictorArgs& a) {
  return (a.hi[0] - a.lo[0] + 1) * (a.hi[1] - a.lo[1] + 1) * (a.hi[2] - a.lo[2] + 1);
}

template <int N>
static cudaError_t launch_n(const PredictorArgs& a, cudaStream_t s) {
  const int TY = a.dims >= 2 ? 8 : 1;
  const bool two_d = a.dims >= 2;
  const int RX = 32 + 4, RY = two_d ? TY + 4 : 1, nst = RX * RY;
  const size_t doubles = (size_t)N * nst + nst + (size_t)N * TY * 33 + (two_d ? (size_t)N * (TY + 1) * 32 : 0);
  const size_t smem = doubles * sizeof(double) + (size_t)nst * sizeof(int);
  auto kern = a.dims == 3 ? k_predictor<N, true> : k_predictor<N, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  const long nx = a.hi[0] - a.lo[0] + 1, ny = a.hi[1] - a.lo[1] + 1, nz = a.hi[2] - a.lo[2] + 1;
  const dim3 grid((unsigned)((nx + 31) / 32), (unsigned)((ny + TY - 1) / TY), (unsigned)nz);
  if (grid.y > 65535u || grid.z > 65535u) return cudaErrorInvalidValue;
  kern<<<grid, dim3(32, TY), smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long total = nx * ny * nz;
  const long blocks = std::min<long>((total + 255) / 256, 2147483647L);  // a block per 256 cells
  k_predictor_commit<N><<<(unsigned)std::max<long>(blocks, 1), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_species_predictor(int n_species, const PredictorArgs& a, cudaStream_t s) {
  switch (n_species) {
    case 9: return launch_n<9>(a, s);
    case 10: return launch_n<10>(a, s);
    case 13: return launch_n<13>(a, s);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace nrg
