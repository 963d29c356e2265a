// Gated MLP surrogate of the per-cell chemistry increment.
//
// Training and the GEMM-chain inference path use one BF16 tensor-core GEMM
// (tcgen05.mma, FP32 accumulator in TMEM) with a fused bias/GELU epilogue; the
// gate decides per cell whether the prediction is used or the cell goes to
// the FP64 integrator:
//   * skip rule of the reference (T < 305 K or bc /= 0): zero sources;
//   * training hull: every raw feature inside the training min/max widened by
//     hull_margin of its range;
//   * element conservation: the network's dY has an element residual
//     |sum_k a_ek (W_e / W_k) dY_k| <= raw_elem_tol for H, O, N (element mass
//     fraction units); it is then projected orthogonally onto the conserving
//     increments in FP64 and the residual of what is written must be
//     <= elem_tol;
//   * temperature: the network's dT agrees within dT_tol with the FP64 energy
//     closure of its own dY, and |dT| <= dT_max.
// Rejected cells are compacted in cell order (so neighbouring cells stay
// neighbours for the integrator) and integrated by the FP64 kernel.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "chem_bdf.cuh"
#include "surrogate.hpp"
#include "order.hpp"
#include "tc_sm100.cuh"

namespace nrg {

// ------------------------------------------------------------------ GEMM
struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16* A;
  long sam, sak;
  const __nv_bfloat16* B;
  long sbk, sbn;
  float* C;  // fp32 result (may be null)
  long ldc;
  const float* bias;   // per column (may be null)
  __nv_bfloat16* H;    // bf16 activation output (may be null)
  long ldh;
  int gelu;            // H = bf16(gelu(C)) when set, else bf16(C)
};

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// C[M, N] = sum_k A[m, k] B[k, n] (+ bias, GELU) on the tensor cores, for
// training (forward, weight and activation gradients) and the GEMM-chain
// inference path.  One 128-thread CTA per 128-row x BN-column tile (BN = N
// rounded up to 16, at most 128): K advances in chunks of 64, each staged in
// shared memory in the K-major no-swizzle core-matrix layout by all threads
// (16-byte vector loads where K is the contiguous direction, element loads
// that transpose otherwise), then multiplied by one thread with
// tcgen05.mma (kind::f16, FP32 accumulator in 128 TMEM columns); two
// buffers, so the next chunk is staged while the tensor core reads the
// previous one.  gridDim.z > 1 splits K (the weight gradients, K = batch):
// each CTA adds its partial tile to C with atomics (C zeroed beforehand, no
// bias or GELU then).  Every mbarrier wait is bounded; a timeout sets *err
// and the CTA stops.
constexpr uint64_t kTcWaitNs = 1000000000ull;  // 1 s per MMA wait (this GEMM and k_mlp_tc)
constexpr int kTgBK = 64;
constexpr uint32_t kTgBuf = 128 * kTgBK * 2;  // one operand chunk: 128 rows x 64 bf16 = 16 KB
constexpr uint32_t kTgSmem = 4 * kTgBuf + 64;  // A0 A1 B0 B1, barriers, TMEM slot

__device__ __forceinline__ void tg_stage(unsigned char* dst, const __nv_bfloat16* src, long s_row, long s_k,
                                         long row0, long rows, long k0, long kend) {
  // dst: 128 rows x kTgBK, row r = operand row row0 + r, column kk = k0 + kk
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  const bool vec = s_k == 1 && (s_row % 8) == 0 && ((reinterpret_cast<uintptr_t>(src) & 15) == 0) &&
                   k0 + kTgBK <= kend;
  if (vec) {
    for (int e = threadIdx.x; e < 128 * (kTgBK / 8); e += blockDim.x) {
      const int r = e / (kTgBK / 8), kc = e % (kTgBK / 8);
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (row0 + r < rows) v = *reinterpret_cast<const uint4*>(src + (row0 + r) * s_row + k0 + kc * 8);
      *reinterpret_cast<uint4*>(dst + tc::kmajor_off(r, kc, kTgBK)) = v;
    }
  } else {
    // consecutive threads take consecutive rows (coalesced when rows are the
    // contiguous direction, as in the transposed operands of the gradients)
    for (int e = threadIdx.x; e < 128 * kTgBK; e += blockDim.x) {
      const int r = e % 128, kk = e / 128;
      const long row = row0 + r, k = k0 + kk;
      const __nv_bfloat16 v = (row < rows && k < kend) ? src[row * s_row + k * s_k] : zero;
      *reinterpret_cast<__nv_bfloat16*>(dst + tc::kmajor_off(r, kk >> 3, kTgBK) + (kk & 7) * 2) = v;
    }
  }
}

__global__ void __launch_bounds__(128, 1) k_gemm_tc(GemmArgs g, long k_per_cta, unsigned int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* bufA[2] = {sm, sm + kTgBuf};
  unsigned char* bufB[2] = {sm + 2 * kTgBuf, sm + 3 * kTgBuf};
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + 4 * kTgBuf);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 4 * kTgBuf + 32);
  const int tid = threadIdx.x, wq = tid >> 5;
  const long m0 = (long)blockIdx.x * 128, n0 = (long)blockIdx.y * 128;
  const long kb = (long)blockIdx.z * k_per_cta, ke = min((long)g.K, kb + k_per_cta);
  const int bn = (int)(((min(128L, (long)g.N - n0) + 15) / 16) * 16);
  if (tid == 0) {
    tc::mbar_init(tc::smem_u32(&mbar[0]), 1);
    tc::mbar_init(tc::smem_u32(&mbar[1]), 1);
    tc::mbar_init_fence();
  }
  if (tid < 32) tc::tmem_alloc(tc::smem_u32(tslot), 128);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  // B operand rows are the output columns n: element (n, k) = B[k * sbk + n * sbn]
  const uint32_t idesc = tc::idesc_bf16_f32(128, (uint32_t)bn);
  const long nch = (ke - kb + kTgBK - 1) / kTgBK;
  uint32_t parity[2] = {0u, 0u};
  bool ok = true;
  for (long c = 0; c < nch && ok; ++c) {
    const int b = (int)(c & 1);
    if (c >= 2) {  // the MMAs that read this buffer two chunks ago are done
      ok = tc::bar_and(1, 128, tc::mbar_wait(tc::smem_u32(&mbar[b]), parity[b], kTcWaitNs));
      parity[b] ^= 1u;
      if (!ok) break;
    }
    const long k0 = kb + c * kTgBK;
    tg_stage(bufA[b], g.A, g.sam, g.sak, m0, g.M, k0, ke);
    tg_stage(bufB[b], g.B, g.sbn, g.sbk, n0, g.N, k0, ke);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a = tc::smem_u32(bufA[b]), bb = tc::smem_u32(bufB[b]);
#pragma unroll
      for (int s = 0; s < kTgBK / 16; ++s)
        tc::mma_bf16(tbase, tc::smem_desc(a + s * 256, 128, kTgBK * 16), tc::smem_desc(bb + s * 256, 128, kTgBK * 16),
                     idesc, (c > 0 || s > 0) ? 1u : 0u);
      tc::commit(tc::smem_u32(&mbar[b]));
    }
  }
  // the last chunk's MMAs (and with them all earlier ones) complete
  if (ok && nch > 0) {
    const int b = (int)((nch - 1) & 1);
    ok = tc::bar_and(1, 128, tc::mbar_wait(tc::smem_u32(&mbar[b]), parity[b], kTcWaitNs));
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1u);
  } else if (nch > 0) {
    tc::fence_after_sync();
    const long m = m0 + tid;
    const bool split = gridDim.z > 1;
    for (int j0 = 0; j0 < bn; j0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tbase + ((uint32_t)(wq * 32) << 16) + (uint32_t)j0, r);
      tc::tmem_ld_wait();
      if (m >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const long n = n0 + j0 + j;
        if (n >= g.N) continue;
        float v = __uint_as_float(r[j]);
        if (split) {
          atomicAdd(&g.C[m * g.ldc + n], v);
          continue;
        }
        if (g.bias) v += g.bias[n];
        if (g.C) g.C[m * g.ldc + n] = v;
        if (g.H) g.H[m * g.ldh + n] = __float2bfloat16(g.gelu ? gelu_f(v) : v);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 128);
  }
}

// Launches the tensor-core GEMM; K split over CTAs when the output is a
// single tile and K is long (the weight gradients).
static cudaError_t gemm(const GemmArgs& g, cudaStream_t st, unsigned int* err) {
  if (g.M <= 0 || g.N <= 0) return cudaSuccess;
  dim3 grid((unsigned)((g.M + 127) / 128), (unsigned)((g.N + 127) / 128), 1);
  long kpc = g.K;
  if (grid.x * grid.y < 16 && g.K > 4 * kTgBK) {
    if (g.bias || g.H || !g.C) return cudaErrorInvalidValue;  // split K adds partial tiles only
    const long chunks = (g.K + kTgBK - 1) / kTgBK;
    const long z = std::min<long>(chunks, 64);
    kpc = ((chunks + z - 1) / z) * kTgBK;
    grid.z = (unsigned)((g.K + kpc - 1) / kpc);
    cudaError_t e = cudaSuccess;
    if (g.ldc == g.N) {
      e = cudaMemsetAsync(g.C, 0, sizeof(float) * (size_t)g.N * (size_t)g.M, st);
    } else {
      for (long m = 0; m < g.M && e == cudaSuccess; ++m)
        e = cudaMemsetAsync(g.C + m * g.ldc, 0, sizeof(float) * (size_t)g.N, st);
    }
    if (e != cudaSuccess) return e;
  }
  k_gemm_tc<<<grid, 128, kTgSmem, st>>>(g, kpc, err);
  return cudaGetLastError();
}

// ------------------------------------------------------- small kernels
__global__ void k_loss_grad(long B, const float* O, const float* Y, float* dOf, __nv_bfloat16* dOb,
                            double* loss) {
  double part = 0.0;
  const float scale = 2.0f / (float)(B * kMlpOut);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < B * kMlpOutPad; i += (long)gridDim.x * blockDim.x) {
    const long b = i / kMlpOutPad;
    const int j = (int)(i % kMlpOutPad);
    float d = 0.f;
    if (j < kMlpOut) {
      const float e = O[b * kMlpOutPad + j] - Y[b * kMlpOut + j];
      part += (double)e * e;
      d = scale * e;
    }
    dOf[i] = d;
    dOb[i] = __float2bfloat16(d);
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, part / (double)(B * kMlpOut));
}

__global__ void k_gelu_back(long n, const float* dH, const float* Z, float* dZf, __nv_bfloat16* dZb) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float d = dH[i] * gelu_grad_f(Z[i]);
    dZf[i] = d;
    dZb[i] = __float2bfloat16(d);
  }
}

// db[c] = sum over rows of M[r][c] (one block per column)
__global__ void k_colsum(long rows, int ncols, const float* M, float* db) {
  const int c = blockIdx.x;
  float s = 0.f;
  for (long r = threadIdx.x; r < rows; r += blockDim.x) s += M[r * ncols + c];
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) db[c] = s;
  }
}

__global__ void k_adam(long n, float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

__global__ void k_to_bf16(long n, const float* x, __nv_bfloat16* y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

__global__ void k_gather_rows(long nb, const int* idx, const __nv_bfloat16* X, const float* Y,
                              __nv_bfloat16* Xb, float* Yb) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nb; i += (long)gridDim.x * blockDim.x) {
    const long r = idx[i];
#pragma unroll
    for (int j = 0; j < kMlpInPad; ++j) Xb[i * kMlpInPad + j] = X[r * kMlpInPad + j];
#pragma unroll
    for (int j = 0; j < kMlpOut; ++j) Yb[i * kMlpOut + j] = Y[r * kMlpOut + j];
  }
}

// Raw features of a cell: T, log(p/1 atm), Y_1..Y_9, log10(dt).
template <int N>
__device__ __forceinline__ void cell_features(double T, double rho, const double (&y)[N], double dt, float* f) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) s += y[k] / c_mech.W[k];
  const double p = rho * 8.31446261815324 * T * s;
  f[0] = (float)T;
  f[1] = (float)log(p / 101325.0);
#pragma unroll
  for (int k = 0; k < N; ++k) f[2 + k] = (float)y[k];
  f[11] = (float)log10(dt);
}

__global__ void k_features(long n, long ld, double dt, const double* dt_cells, const double* T, const double* rho,
                           const double* Y, const MlpNorm* nm, float* xraw, __nv_bfloat16* x) {
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    double y[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) y[k] = Y[k * ld + c];
    float f[kMlpIn];
    cell_features<9>(T[c], rho[c], y, dt_cells ? dt_cells[c] : dt, f);
    if (xraw)
#pragma unroll
      for (int j = 0; j < kMlpIn; ++j) xraw[c * kMlpIn + j] = f[j];
    if (x) {
#pragma unroll
      for (int j = 0; j < kMlpInPad; ++j)
        x[c * kMlpInPad + j] = __float2bfloat16(j < kMlpIn ? net_input(*nm, j, f[j]) : 0.f);
    }
  }
}

// Gate and outputs.  flag[c] = 1 sends the cell to the FP64 fallback.
struct GateCfg {
  double elem_tol;      // element residual of the dY that is written (after projection)
  double raw_elem_tol;  // element residual of the network's own dY
  double dT_tol, dT_max;
  double dt_max;        // cells with a longer step go to FP64: the bounds above were calibrated up to it
  // committee check: with a partner network (index >= 0), a cell is accepted
  // only if the partner predicts every dY_k within agree_Y and dT within
  // agree_T of this network
  int partner;
  double agree_Y, agree_T;
};

// Element residual max_e |sum_k a_ek (W_e / W_k) dY_k| (element mass fraction)
// for H, O, N.
__device__ __forceinline__ double element_residual(const double (&dY)[9]) {
  const double We[3] = {1.00794e-3, 15.9994e-3, 14.0067e-3};
  double m = 0.0;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) r += c_mech.elem[e][k] * We[e] / c_mech.W[k] * dY[k];
    m = fmax(m, fabs(r));
  }
  return m;
}

// Orthogonal projector onto the element-conserving increments
// {dY : sum_k a_ek dY_k / W_k = 0 for H, O, N}: P = I - sum_q q q^T over an
// orthonormal basis q of the rows a_e / W (Gram-Schmidt; elements absent from
// the mechanism drop out).
__device__ void element_projector(double (*P)[9]) {
  double q[3][9];
  int nq = 0;
  for (int e = 0; e < 3; ++e) {
    double v[9], n0 = 0.0;
    for (int k = 0; k < 9; ++k) {
      v[k] = c_mech.elem[e][k] / c_mech.W[k];
      n0 += v[k] * v[k];
    }
    for (int i = 0; i < nq; ++i) {
      double d = 0.0;
      for (int k = 0; k < 9; ++k) d += q[i][k] * v[k];
      for (int k = 0; k < 9; ++k) v[k] -= d * q[i][k];
    }
    double nn = 0.0;
    for (int k = 0; k < 9; ++k) nn += v[k] * v[k];
    if (!(n0 > 0.0) || nn <= 1e-24 * n0) continue;
    const double r = 1.0 / sqrt(nn);
    for (int k = 0; k < 9; ++k) q[nq][k] = v[k] * r;
    ++nq;
  }
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) {
      double x = i == j ? 1.0 : 0.0;
      for (int b = 0; b < nq; ++b) x -= q[b][i] * q[b][j];
      P[i][j] = x;
    }
}

// Skip rule of the reference (T < 305 K or a boundary marker): zero sources,
// T unchanged.  Returns true for a skipped cell.
__device__ __forceinline__ bool write_if_skipped(const StepArgs& a, long c, double T0) {
  if (reference_cell_active(T0, a.bc, c)) return false;
  write_skipped_cell(a, c, 9, T0);
  return true;
}

// Per-block copy of what the gate's energy closure reads: NASA-7 enthalpy
// coefficients pre-divided by their powers (b_i = a_i / (i + 1), i < 5, and
// a_5), cp coefficients a_0..a_4, both sets of each species, and 1 / W.
struct GateThermo {
  double h[9][2][6];
  double cp[9][2][5];
  double invW[9];
};

__device__ void gate_thermo_init(GateThermo* g) {
  for (int i = threadIdx.x; i < 9 * 2; i += blockDim.x) {
    const int k = i >> 1, set = i & 1;
    const double* a = c_mech.a[k][set];
    for (int j = 0; j < 5; ++j) {
      g->h[k][set][j] = a[j] / (double)(j + 1);
      g->cp[k][set][j] = a[j];
    }
    g->h[k][set][5] = a[5];
    if (set == 0) g->invW[k] = c_mech.invW[k];
  }
}

// h_k(T) * ... as the reference's specie_enthalpy (per mole, times R in the
// tables): t (b0 + t (b1 + t (b2 + t (b3 + t b4)))) + a5, t = min(T, 6000 K).
__device__ __forceinline__ double gate_enthalpy(const GateThermo& g, int k, double T) {
  const double t = fmin(T, 6000.0);
  const double* b = g.h[k][t >= 1000.0 ? 1 : 0];
  return fma(t, fma(t, fma(t, fma(t, fma(t, b[4], b[3]), b[2]), b[1]), b[0]), b[5]);
}

// Energy closure of the gate: the reference's constant-density closure
// (cpm_solver.f90:517,549; calculate_temperature, thermophysical_properties_
// class.f90:409-452 -- Newton with cp frozen at the start temperature, at
// most 1000 iterations, |step| < 1e-8 K) unrolled over the nine species in
// registers, started at T_start (the network's temperature).  The gate
// compares its result with the network's temperature change within dT_tol,
// so it agrees with the integrator's closure to far below that tolerance
// rather than to its last bit.
__device__ __forceinline__ double gate_closure(const GateThermo& g, double T0, double T_start,
                                               const double (&Y0)[9], const double (&dY)[9], double dE) {
  const double RG = 8.31446261815324;
  double X[9], s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) s0 += Y0[k] * g.invW[k];
  const double W0 = 1.0 / s0;
  double e0 = 0.0, h0 = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double x = Y0[k] * g.invW[k] * W0;
    e0 += gate_enthalpy(g, k, T0) * x;
    h0 += c_mech.h_ref[k] * x;
  }
  e0 -= RG * T0;
  const double e1 = (e0 - h0) / W0 + dE;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    X[k] = Y0[k] + dY[k];
    s1 += X[k] * g.invW[k];
  }
  const double W1 = 1.0 / s1;
  double hc = 0.0, cp = 0.0;
  double temp = fmin(T_start, 6000.0);
  const int set = temp >= 1000.0 ? 1 : 0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    X[k] = X[k] * g.invW[k] * W1;
    hc += c_mech.h_ref[k] * X[k];
    const double* a = g.cp[k][set];
    cp += fma(temp, fma(temp, fma(temp, fma(temp, a[4], a[3]), a[2]), a[1]), a[0]) * X[k];
  }
  const double ei = e1 * W1, rcp = 1.0 / cp;
  for (int it = 0; it < 1000; ++it) {
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) e += gate_enthalpy(g, k, temp) * X[k];
    e -= RG * temp;
    const double res = (ei - (e - hc)) * rcp;
    temp += res;
    if (fabs(res) < (double)1e-08f) break;
  }
  return temp;
}

// Gate of one active cell on its network outputs o (normalised units): hull
// of the raw features f, element residuals, FP64 projection, energy closure.
// Writes the sources of an accepted cell and returns whether it was accepted.
// Each test returns as soon as it fails; the cell's mass fractions are read
// again (from cache) for the closure rather than kept live across the tests.
__device__ __forceinline__ bool gate_active_cell(const StepArgs& a, long c, double T0, double rho, double dt,
                                                 const float (&f)[kMlpIn], const float (&o)[kMlpOut],
                                                 const MlpNorm* nm, const GateCfg& gc, const double (*P)[9],
                                                 const GateThermo& th, const float* op, const MlpNorm* pnm) {
  if (!(dt <= gc.dt_max)) return false;
  bool in = true;
  const float margin = nm->hull_margin;
#pragma unroll
  for (int j = 0; j < kMlpIn; ++j) {
    const float lo0 = nm->x_min[j], hi0 = nm->x_max[j], span = hi0 - lo0;
    in = in && (f[j] >= lo0 - margin * span) && (f[j] <= hi0 + margin * span);
  }
  if (!in) return false;
  const double sc = (double)target_scale(f[11], nm->dt_pow);
  double dYn[9];
  bool fin = true;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    dYn[k] = (double)o[k] * (double)nm->y_sd[k] * sc;
    fin = fin && isfinite(dYn[k]);
  }
  const double dT_net = (double)o[9] * (double)nm->y_sd[9] * sc;
  if (!fin || !isfinite(dT_net) || !(fabs(dT_net) <= gc.dT_max)) return false;
  if (op) {  // committee check against the partner network's prediction
    const double psc = (double)target_scale(f[11], pnm->dt_pow);
    bool agree = fabs((double)op[9] * (double)pnm->y_sd[9] * psc - dT_net) <= gc.agree_T;
#pragma unroll
    for (int k = 0; k < 9; ++k) agree = agree && fabs((double)op[k] * (double)pnm->y_sd[k] * psc - dYn[k]) <= gc.agree_Y;
    if (!agree) return false;
  }
  if (!(element_residual(dYn) <= gc.raw_elem_tol)) return false;
  // the written increment conserves H, O and N: projection in FP64
  double dY[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    double x = 0.0;
#pragma unroll
    for (int j = 0; j < 9; ++j) x = fma(P[i][j], dYn[j], x);
    dY[i] = x;
  }
  if (!(element_residual(dY) <= gc.elem_tol)) return false;
  const double rho_dt = rho / dt;
  double E = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) E -= c_mech.h_ref[k] * (dY[k] * th.invW[k]) * rho_dt;
  double y0[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) y0[k] = a.Y[k * a.ld + c];
  // the Newton iteration of the closure starts at the network's temperature
  const double T1 = gate_closure(th, T0, T0 + dT_net, y0, dY, E * dt / rho);
  if (!(fabs((T1 - T0) - dT_net) <= gc.dT_tol)) return false;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    // the integrator's relation Y_prod = Y_prod2 W / dt, evaluated the same
    // way, so that a host can rebuild Y_prod from Y_prod2 bit for bit
    const double y2 = dY[k] * rho * th.invW[k];
    a.Y_prod2[k * a.ld + c] = y2;
    a.Y_prod[k * a.ld + c] = y2 * c_mech.W[k] / dt;
  }
  a.E_f_prod[c] = E;
  if (a.T_after) a.T_after[c] = T1;
  if (a.status) a.status[c] = kCellSurrogate;
  return true;
}

__device__ __forceinline__ void count_surrogate(unsigned long long n_sur, unsigned long long* counters) {
  if (!counters) return;
  for (int o = 16; o > 0; o >>= 1) n_sur += __shfl_down_sync(0xffffffffu, n_sur, o);
  if ((threadIdx.x & 31) == 0 && n_sur) atomicAdd(&counters[6], n_sur);
}

// O: the network outputs of every active cell, output j of cell c at
// O[j * o_ld + c] (o_ld > 0) or O[c * 16 + j] (o_ld == 0).
// The networks of one step: an active cell goes to the enabled network of
// highest index whose routing band [lo, hi) -- the temperature range of its
// training hull -- holds its temperature, and is gated with that network's
// standardisation and settings.  Network 0 is the main one; the others
// cover narrower bands (a flame's preheat zone, the low-temperature part of
// its front) and take precedence there.
// gc: the gate for steps up to gc.dt_max (and the committee partner); xb:
// bounds for longer steps, band b for dt in (previous band's dt_max,
// xb[b].dt_max] (dt_max 0: unused).
struct GateNet {
  const MlpNorm* nm;
  GateCfg gc;
  double lo, hi;
  int on;
  GateCfg xb[kGateBands - 1];
  double dt_lo, dt_hi;  // routing step band (dt_lo, dt_hi]
};

// The gate settings for a step of length dt (the committee fields are gc's).
__device__ __forceinline__ GateCfg gate_for_dt(const GateNet& g, double dt) {
  if (dt <= g.gc.dt_max) return g.gc;
  double prev = g.gc.dt_max;
#pragma unroll
  for (int b = 0; b < kGateBands - 1; ++b) {
    const GateCfg& x = g.xb[b];
    if (x.dt_max > prev && dt <= x.dt_max) {
      GateCfg r = x;
      r.partner = g.gc.partner;
      r.agree_Y = g.gc.agree_Y;
      r.agree_T = g.gc.agree_T;
      return r;
    }
    if (x.dt_max > prev) prev = x.dt_max;
  }
  return g.gc;  // dt above every band: gate_active_cell rejects it
}
struct GateNets {
  GateNet net[kMaxNets];
};

// The enabled network of highest index whose temperature band [lo, hi) and
// step band (dt_lo, dt_hi] hold the cell, or -1.
__device__ __forceinline__ int route_of(const GateNets& g, double T, double dt) {
#pragma unroll
  for (int i = kMaxNets - 1; i >= 0; --i)
    if (g.net[i].on && T >= g.net[i].lo && T < g.net[i].hi && dt > g.net[i].dt_lo && dt <= g.net[i].dt_hi) return i;
  return -1;
}

// OP (may be null): the partner networks' outputs for the cells routed to a
// network that has a partner, planar like O with o_ld.
__global__ void __launch_bounds__(128, 3) k_gate(StepArgs a, const float* O, const float* OP, long o_ld, GateNets nets,
                                              unsigned char* flag, unsigned long long* counters) {
  __shared__ double P[9][9];
  __shared__ GateThermo th;
  if (threadIdx.x == 0) element_projector(P);
  gate_thermo_init(&th);
  __syncthreads();
  unsigned long long n_sur = 0;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < a.n; c += (long)gridDim.x * blockDim.x) {
    const double T0 = a.T[c];
    if (write_if_skipped(a, c, T0)) {
      flag[c] = 0;
      continue;
    }
    const int net = route_of(nets, T0, a.dt_cells ? a.dt_cells[c] : a.dt);
    if (net < 0) {  // no network for this temperature and step: FP64
      flag[c] = 1;
      continue;
    }
    const double rho = a.rho[c];
    const double dt = a.dt_cells ? a.dt_cells[c] : a.dt;
    float f[kMlpIn], o[kMlpOut];
    {
      double y0[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) y0[k] = a.Y[k * a.ld + c];
      cell_features<9>(T0, rho, y0, dt, f);
    }
#pragma unroll
    for (int j = 0; j < kMlpOut; ++j) o[j] = o_ld > 0 ? O[j * o_ld + c] : O[c * kMlpOutPad + j];
    const int pn = nets.net[net].gc.partner;
    float op[kMlpOut];
    const bool with_partner = OP && o_ld > 0 && pn >= 0 && pn < kMaxNets && nets.net[pn].on;
    if (with_partner) {
#pragma unroll
      for (int j = 0; j < kMlpOut; ++j) op[j] = OP[j * o_ld + c];
    }
    const GateCfg gc = gate_for_dt(nets.net[net], dt);
    const bool acc = gate_active_cell(a, c, T0, rho, dt, f, o, nets.net[net].nm, gc, P, th,
                                      with_partner ? op : nullptr, with_partner ? nets.net[pn].nm : nullptr);
    n_sur += acc;
    flag[c] = acc ? 0 : 1;
  }
  count_surrogate(n_sur, counters);
}

// ------------------------------------------------- tcgen05 inference
// The network of the surrogate step runs in its own kernel, k_mlp_tc, and the
// FP64 gate in a wide grid after it (k_gate, above), so that the gate's
// latency-bound FP64 work (energy-closure Newton, element projection) runs
// with many warps per SM instead of inside the tensor-core kernel.
//
// k_mlp_tc: persistent CTAs of three warpgroups; each warpgroup streams its
// own 128-cell tiles (thread t of the group owns cell t of the tile, which is
// TMEM lane t).  Per tile: features are standardised into a bf16 K-major
// operand in shared memory, one thread issues the layer's tcgen05.mma
// (M = 128, A = activations, B = weights, both in shared memory; FP32
// accumulator in this group's 128 TMEM columns) and commits to the group's
// mbarrier; the epilogue reads the thread's accumulator row with tcgen05.ld,
// adds the bias, applies GELU and writes the next layer's bf16 operand.  The
// weights (104 KB) stay in shared memory for the kernel's lifetime; while one
// group runs its epilogue the others' MMAs run.  Tiles without an active cell
// skip the network.  Every wait is bounded: on a timeout the group stops
// issuing MMAs, writes NaN outputs for its remaining cells (the gate sends
// them to the FP64 integrator) and records the event in *err.
constexpr int kTcGroups = 3;
constexpr uint32_t kTcW0 = 0;                             // layer 0: 128 x 16
constexpr uint32_t kTcW1 = 4096;                          // layers 1-3: 128 x 128
constexpr uint32_t kTcW4 = kTcW1 + 3 * 32768;             // layer 4: 16 x 128
constexpr uint32_t kTcAct = kTcW4 + 4096;                 // per group 128 x 128 bf16
constexpr uint32_t kTcBias = kTcAct + kTcGroups * 32768;  // fp32, 4 x 128 + 16
constexpr uint32_t kTcMisc = kTcBias + (4 * kMlpHid + kMlpOutPad) * 4;
constexpr uint32_t kTcSmem = kTcMisc + 256;
constexpr uint32_t kTcTmemCols = 512;  // a power of two holding 128 columns per group
static_assert(kTcGroups * 128 <= (int)kTcTmemCols, "TMEM columns of the groups");
static_assert(kTcSmem <= 227u * 1024u, "shared memory of one CTA");

struct TcArgs {
  StepArgs a;
  const MlpNorm* nm;
  const __nv_bfloat16* wb;  // bf16 parameters (per layer W[out][in_pad], then b)
  const float* w;           // fp32 parameters (biases read from here)
  long offW[kMlpLayers], offb[kMlpLayers];
  float* out;    // network outputs (normalised units)
  long out_ld;   // > 0: output j of cell c at out[j * out_ld + c] (kMlpOut values); 0: out[c * 16 + j]
  int active;    // 1: only the cells the step integrates (skip rule) that route to network `net`, or to a
                 // network whose partner `net` is (those outputs go to out_partner); 0: every cell
  int net;
  GateNets routes;
  float* out_partner;
  unsigned int* err;  // bit 0: an MMA wait timed out
  // when set: the kernel's cells are list[0 .. *list_count) (indices into a)
  // instead of every cell of a
  const int* list;
  const int* list_count;
};

__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 r;
  r.x = pack_bf16(__float2bfloat16(v[0]), __float2bfloat16(v[1]));
  r.y = pack_bf16(__float2bfloat16(v[2]), __float2bfloat16(v[3]));
  r.z = pack_bf16(__float2bfloat16(v[4]), __float2bfloat16(v[5]));
  r.w = pack_bf16(__float2bfloat16(v[6]), __float2bfloat16(v[7]));
  return r;
}

__device__ __forceinline__ void store_outputs(const TcArgs& p, long c, const float* o, bool valid, bool partner) {
  const float nan = __int_as_float(0x7fc00000);
  if (p.out_ld > 0) {
    float* dst = partner ? p.out_partner : p.out;
#pragma unroll
    for (int j = 0; j < kMlpOut; ++j) dst[j * p.out_ld + c] = valid ? o[j] : nan;
  } else {
#pragma unroll
    for (int j = 0; j < kMlpOutPad; ++j) p.out[c * kMlpOutPad + j] = !valid ? nan : (j < kMlpOut ? o[j] : 0.f);
  }
}

__global__ void __launch_bounds__(128 * kTcGroups, 1) k_mlp_tc(TcArgs p) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const StepArgs& a = p.a;
  const int tid = threadIdx.x, g = tid >> 7, t = tid & 127, wq = t >> 5;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kTcMisc);         // [kTcGroups]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTcMisc + 32);
  uint32_t* vote = reinterpret_cast<uint32_t*>(sm + kTcMisc + 64);    // [group][parity][warp]
  float* bias = reinterpret_cast<float*>(sm + kTcBias);

  // weights into the K-major canonical layout, biases, barriers, TMEM
  for (int i = tid; i < kMlpHid * 2; i += blockDim.x) {
    const int n = i >> 1, kc = i & 1;
    *reinterpret_cast<uint4*>(sm + kTcW0 + tc::kmajor_off(n, kc, 16)) =
        *reinterpret_cast<const uint4*>(p.wb + p.offW[0] + n * 16 + kc * 8);
  }
  for (int l = 1; l <= 3; ++l)
    for (int i = tid; i < kMlpHid * 16; i += blockDim.x) {
      const int n = i >> 4, kc = i & 15;
      *reinterpret_cast<uint4*>(sm + kTcW1 + (l - 1) * 32768 + tc::kmajor_off(n, kc, 128)) =
          *reinterpret_cast<const uint4*>(p.wb + p.offW[l] + n * 128 + kc * 8);
    }
  for (int i = tid; i < kMlpOutPad * 16; i += blockDim.x) {
    const int n = i >> 4, kc = i & 15;
    *reinterpret_cast<uint4*>(sm + kTcW4 + tc::kmajor_off(n, kc, 128)) =
        *reinterpret_cast<const uint4*>(p.wb + p.offW[4] + n * 128 + kc * 8);
  }
  for (int i = tid; i < 4 * kMlpHid + kMlpOutPad; i += blockDim.x)
    bias[i] = i < 4 * kMlpHid ? p.w[p.offb[i / kMlpHid] + i % kMlpHid] : p.w[p.offb[4] + (i - 4 * kMlpHid)];
  if (tid == 0) {
    for (int i = 0; i < kTcGroups; ++i) tc::mbar_init(tc::smem_u32(&mbar[i]), 1);
    tc::mbar_init_fence();
  }
  if (tid < 32) tc::tmem_alloc(tc::smem_u32(tslot), kTcTmemCols);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;

  const uint32_t bar_id = 1 + g;
  unsigned char* actp = sm + kTcAct + g * 32768;
  const uint32_t act = tc::smem_u32(actp);
  const uint32_t wsm = tc::smem_u32(sm);
  const uint32_t mb = tc::smem_u32(&mbar[g]);
  const uint32_t d_tmem = tbase + (uint32_t)g * 128u;
  const uint32_t my_tmem = d_tmem + ((uint32_t)(wq * 32) << 16);
  constexpr uint32_t kIdHid = tc::idesc_bf16_f32(128, 128), kIdOut = tc::idesc_bf16_f32(128, 16);
  uint32_t phase = 0;
  bool aborted = false;
  const long nitems = p.list ? (long)*p.list_count : a.n;
  const long ntiles = (nitems + 127) / 128;
  int par = 0;
  for (long tile = (long)blockIdx.x * kTcGroups + g; tile < ntiles; tile += (long)gridDim.x * kTcGroups, par ^= 1) {
    const long idx = tile * 128 + t;
    const long c = p.list ? (idx < nitems ? (long)p.list[idx] : -1L) : idx;
    bool need = false, for_partner = false;
    float f[kMlpIn];
#pragma unroll
    for (int j = 0; j < kMlpIn; ++j) f[j] = 0.f;
    if (c >= 0 && c < a.n) {
      const double T0 = a.T[c];
      if (p.active) {
        const int r = reference_cell_active(T0, a.bc, c) ? route_of(p.routes, T0, a.dt_cells ? a.dt_cells[c] : a.dt)
                                                         : -1;
        for_partner = r >= 0 && r != p.net && p.out_partner && p.routes.net[r].gc.partner == p.net;
        need = r == p.net || for_partner;
      } else {
        need = true;
      }
      if (need) {
        double y0[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) y0[k] = a.Y[k * a.ld + c];
        cell_features<9>(T0, a.rho[c], y0, a.dt_cells ? a.dt_cells[c] : a.dt, f);
      }
    }
    float o[kMlpOutPad];
    if (aborted) {
      if (need) store_outputs(p, c, o, false, for_partner);
      continue;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, need);
    if ((t & 31) == 0) vote[(g * 2 + par) * 4 + wq] = bal;
    tc::bar_sync(bar_id, 128);
    const uint32_t* vv = vote + (g * 2 + par) * 4;
    if ((vv[0] | vv[1] | vv[2] | vv[3]) == 0u) continue;

    // layer 0 operand: 16 standardised bf16 features of this thread's cell
    {
      float xs[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) xs[j] = (need && j < kMlpIn) ? net_input(*p.nm, j, f[j]) : 0.f;
      *reinterpret_cast<uint4*>(actp + tc::kmajor_off(t, 0, 16)) = pack8(xs);
      *reinterpret_cast<uint4*>(actp + tc::kmajor_off(t, 1, 16)) = pack8(xs + 8);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    tc::bar_sync(bar_id, 128);
    if (t == 0) {
      tc::fence_after_sync();
      tc::mma_bf16(d_tmem, tc::smem_desc(act, 128, 256), tc::smem_desc(wsm + kTcW0, 128, 256), kIdHid, 0);
      tc::commit(mb);
    }
    bool ok = true;
    for (int l = 0; l < 4 && ok; ++l) {
      // epilogue of layer l: bias + GELU -> bf16 operand of layer l + 1
      ok = __all_sync(0xffffffffu, tc::mbar_wait(mb, phase, kTcWaitNs));  // tcgen05.ld is warp-wide
      phase ^= 1u;
      tc::fence_after_sync();
      if (ok) {
        const float* bl = bias + l * kMlpHid;
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
          uint32_t r[32];
          tc::tmem_ld32(my_tmem + q * 32, r);
          tc::tmem_ld_wait();
          float h[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) h[j] = gelu_f(__uint_as_float(r[j]) + bl[q * 32 + j]);
#pragma unroll
          for (int i = 0; i < 4; ++i)
            *reinterpret_cast<uint4*>(actp + tc::kmajor_off(t, q * 4 + i, 128)) = pack8(h + 8 * i);
        }
      }
      tc::fence_async_smem();
      tc::fence_before_sync();
      ok = tc::bar_and(bar_id, 128, ok);
      if (ok && t == 0) {
        tc::fence_after_sync();
        const bool last = l == 3;
        const uint32_t wl = last ? wsm + kTcW4 : wsm + kTcW1 + (uint32_t)l * 32768u;
#pragma unroll
        for (int s = 0; s < 8; ++s)
          tc::mma_bf16(d_tmem, tc::smem_desc(act + s * 256, 128, 2048), tc::smem_desc(wl + s * 256, 128, 2048),
                       last ? kIdOut : kIdHid, s > 0);
        tc::commit(mb);
      }
    }
    if (ok) {
      ok = __all_sync(0xffffffffu, tc::mbar_wait(mb, phase, kTcWaitNs));
      phase ^= 1u;
      tc::fence_after_sync();
      if (ok) {
        uint32_t r[16];
        tc::tmem_ld16(my_tmem, r);
        tc::tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < kMlpOutPad; ++j) o[j] = __uint_as_float(r[j]) + bias[4 * kMlpHid + j];
      }
      tc::fence_before_sync();
      ok = tc::bar_and(bar_id, 128, ok);
    }
    if (!ok) {
      aborted = true;
      if (t == 0) atomicOr(p.err, 1u);
    }
    if (need) store_outputs(p, c, o, ok, for_partner);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, kTcTmemCols);
  }
}

// Order-preserving compaction of flagged cells: per-block counts, a single
// block scan of the counts, then an in-block ballot scan for the scatter.
constexpr int kCompactBlock = 1024;

__global__ void k_flag_count(long n, const unsigned char* flag, int* block_count) {
  const long i = (long)blockIdx.x * kCompactBlock + threadIdx.x;
  const int f = (i < n) ? (int)flag[i] : 0;
  const int cnt = __syncthreads_count(f);
  if (threadIdx.x == 0) block_count[blockIdx.x] = cnt;
}

// Exclusive scan of nb block counts by one block (any multiple of 32 threads up
// to 1024); the total goes to *total (and is added to counters[7]).
__device__ void scan_counts_body(int nb, const int* block_count, int* block_off, int* total,
                                 unsigned long long* counters) {
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? block_count[i] : 0;
    // inclusive warp scan, then across warps
    int x = v;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    __shared__ int wsum[32];
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      int s = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    const int incl = x + (w > 0 ? wsum[w - 1] : 0);
    if (i < nb) block_off[i] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *total = carry;
    if (counters) atomicAdd(&counters[7], (unsigned long long)carry);  // steps of two streams may add at once
  }
}

__global__ void k_scan_counts(int nb, const int* block_count, int* block_off, int* total,
                              unsigned long long* counters) {
  scan_counts_body(nb, block_count, block_off, total, counters);
}

// ------------------------------------------------ per-network cell lists
// The tensor-core kernel of network i runs over the list of the cells it has
// to answer, so its tiles are full and a network with a narrow band does not
// scan the whole field.  Bit i of a cell's mask: the cell routes to network
// i, or to a network whose committee partner i is.
__device__ __forceinline__ unsigned route_mask(const StepArgs& a, const GateNets& nets, long c) {
  const double T0 = a.T[c];
  if (!reference_cell_active(T0, a.bc, c)) return 0u;
  const int r = route_of(nets, T0, a.dt_cells ? a.dt_cells[c] : a.dt);
  if (r < 0) return 0u;
  unsigned m = 1u << r;
  const int q = nets.net[r].gc.partner;
  if (q >= 0 && q < kMaxNets && q != r && nets.net[q].on) m |= 1u << q;
  return m;
}

__global__ void k_route_count(StepArgs a, GateNets nets, unsigned char* mask, int nb, int* block_count) {
  const long c = (long)blockIdx.x * kCompactBlock + threadIdx.x;
  const unsigned m = c < a.n ? route_mask(a, nets, c) : 0u;
  if (c < a.n) mask[c] = (unsigned char)m;
  for (int i = 0; i < kMaxNets; ++i) {
    const int cnt = __syncthreads_count((int)((m >> i) & 1u));
    if (threadIdx.x == 0) block_count[i * nb + blockIdx.x] = cnt;
  }
}

__global__ void k_route_scan(int nb, const int* block_count, int* block_off, int* total) {
  scan_counts_body(nb, block_count + (long)blockIdx.x * nb, block_off + (long)blockIdx.x * nb, total + blockIdx.x,
                   nullptr);
}

// list[i * cap + j]: the j-th cell (in cell order) of network i's list
__global__ void k_route_scatter(long n, const unsigned char* mask, int nb, const int* block_off, long cap,
                                int* list) {
  const long c = (long)blockIdx.x * kCompactBlock + threadIdx.x;
  const unsigned m = c < n ? mask[c] : 0u;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ int wcount[kCompactBlock / 32];
  for (int i = 0; i < kMaxNets; ++i) {
    const int f = (int)((m >> i) & 1u);
    if (!__syncthreads_or(f)) continue;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcount[w] = __popc(bal);
    __syncthreads();
    int before = 0;
    for (int q = 0; q < w; ++q) before += wcount[q];
    if (f) list[(long)i * cap + block_off[i * nb + blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u))] = (int)c;
  }
}

__global__ void k_compact(long n, const unsigned char* flag, const int* block_off, int* list) {
  const long i = (long)blockIdx.x * kCompactBlock + threadIdx.x;
  const int f = (i < n) ? (int)flag[i] : 0;
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ int wcount[kCompactBlock / 32];
  if (lane == 0) wcount[w] = __popc(bal);
  __syncthreads();
  int before = 0;
  for (int q = 0; q < w; ++q) before += wcount[q];
  if (f) list[block_off[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u))] = (int)i;
}

// Raw training targets: dY_k = Y_prod_k dt / rho and dT = T_after - T.
__global__ void k_targets(long n, long ld, double dt, const double* dt_cells, const double* T, const double* rho,
                          const double* Y_prod, const double* T_after, float dt_pow, float* y) {
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    const double d = dt_cells ? dt_cells[c] : dt;
    const double sc = (double)target_scale((float)log10(d), dt_pow);
#pragma unroll
    for (int k = 0; k < 9; ++k) y[c * kMlpOut + k] = (float)(Y_prod[k * ld + c] * d / rho[c] / sc);
    y[c * kMlpOut + 9] = (float)((T_after[c] - T[c]) / sc);
  }
}

// Per-column mean, standard deviation, min and max (one block per column).
__global__ void k_colstats(long rows, int ncols, const float* M, double* out) {
  const int c = blockIdx.x;
  double s = 0.0, q = 0.0, lo = 1e300, hi = -1e300;
  for (long r = threadIdx.x; r < rows; r += blockDim.x) {
    const double v = M[r * ncols + c];
    s += v;
    q += v * v;
    lo = v < lo ? v : lo;
    hi = v > hi ? v : hi;
  }
  __shared__ double sh[4][32];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    q += __shfl_down_sync(0xffffffffu, q, o);
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { sh[0][w] = s; sh[1][w] = q; sh[2][w] = lo; sh[3][w] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0, Q = 0, L = 1e300, H = -1e300;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      S += sh[0][i]; Q += sh[1][i]; L = fmin(L, sh[2][i]); H = fmax(H, sh[3][i]);
    }
    const double mu = S / (double)rows;
    out[c * 4 + 0] = mu;
    out[c * 4 + 1] = sqrt(fmax(Q / (double)rows - mu * mu, 0.0));
    out[c * 4 + 2] = L;
    out[c * 4 + 3] = H;
  }
}

// Network inputs before standardisation (log transform of the chosen species).
__global__ void k_transform(long n, const float* xraw, float log_mask, float log_eps, float* xt) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * kMlpIn; i += (long)gridDim.x * blockDim.x)
    xt[i] = net_feature(log_mask, log_eps, (int)(i % kMlpIn), xraw[i]);
}

__global__ void k_standardize(long n, const float* xraw, const float* yraw, const MlpNorm* nm,
                              __nv_bfloat16* x, float* y) {
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j < kMlpInPad; ++j)
      x[c * kMlpInPad + j] = __float2bfloat16(j < kMlpIn ? net_input(*nm, j, xraw[c * kMlpIn + j]) : 0.f);
#pragma unroll
    for (int j = 0; j < kMlpOut; ++j) y[c * kMlpOut + j] = yraw[c * kMlpOut + j] / nm->y_sd[j];
  }
}

// -------------------------------------------------------------- state
struct Surrogate {
  bool ready = false;
  bool uploaded = false;
  GateCfg gate{1e-6, 5e-6, 0.2, 5.0, 1e-6, -1, 0.0, 0.0};
  GateCfg xgate[kGateBands - 1] = {};  // bounds for longer steps (dt_max 0: unused)
  MlpNorm norm{};
  MlpNorm* d_norm = nullptr;
  // parameters: fp32 master, Adam moments, bf16 working copies, gradients
  float* w = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* gr = nullptr;
  __nv_bfloat16* wb = nullptr;
  long n_params = 0;
  long offW[kMlpLayers], offb[kMlpLayers];
  long step = 0;
  // activation buffers (grow-only)
  long cap = 0;
  __nv_bfloat16 *X = nullptr, *H[kMlpLayers] = {}, *dHb = nullptr;
  float *Z[kMlpLayers] = {}, *O = nullptr, *dOf = nullptr, *dHf = nullptr, *dZf = nullptr;
  __nv_bfloat16* dOb = nullptr;
  float* Yb = nullptr;
  int* idx = nullptr;
  double* d_loss = nullptr;
  // inference buffers (features, two activation buffers, outputs)
  long icap = 0;
  __nv_bfloat16 *iX = nullptr, *iH[2] = {nullptr, nullptr};
  float* iO = nullptr;
  // the tensor-core network kernel (default) or the GEMM chain (one k_gemm_tc
  // launch per layer), then the gate
  bool fused = true;
  int num_sms = 0;
  unsigned int* d_err = nullptr;  // bit 0: an MMA wait of the tensor-core kernel timed out
  unsigned int* h_err = nullptr;  // pinned
  // gate / compaction buffers; gO: network outputs of the tensor-core kernel
  // (kMlpOut planes of gcap floats)
  long gcap = 0;
  float* gO = nullptr;
  float* gP = nullptr;  // partner networks' outputs (committee check), same layout
  // routing band [band_lo, band_hi) when set (band_set), else the hull's T range
  bool band_set = false;
  double band_lo = 0.0, band_hi = 0.0;
  // routing step band (dt_band_lo, dt_band_hi]
  double dt_band_lo = 0.0, dt_band_hi = 1e300;
  unsigned char* flag = nullptr;
  int *block_count = nullptr, *block_off = nullptr, *list = nullptr, *n_list = nullptr;
  // per-network cell lists of the tensor-core kernel (kMaxNets lists of gcap)
  unsigned char* rmask = nullptr;
  int *rlist = nullptr, *rblock_count = nullptr, *rblock_off = nullptr, *rcount = nullptr;
  // fallback cells in temperature order (order.hpp) or in cell order
  bool order_cells = true;
  OrderScratch order;
  // a second set of the per-step scratch above (lists, outputs, order), so
  // that two chunks of a field go through surrogate_gate / surrogate_fallback
  // at once on two streams (surrogate_reserve_lane1)
  struct Lane {
    long cap = 0;
    float *gO = nullptr, *gP = nullptr;
    int *block_count = nullptr, *block_off = nullptr, *list = nullptr, *n_list = nullptr;
    unsigned char* rmask = nullptr;
    int *rlist = nullptr, *rblock_count = nullptr, *rblock_off = nullptr, *rcount = nullptr;
    OrderScratch order;
  } lane1;
};

// The scratch of lane 0 (the fields of Surrogate) or lane 1 (Surrogate::lane1).
struct LaneRef {
  long cap;
  float *gO, *gP;
  int *block_count, *block_off, *list, *n_list;
  unsigned char* rmask;
  int *rlist, *rblock_count, *rblock_off, *rcount;
  OrderScratch* order;
};

static LaneRef lane_ref(Surrogate* s, int lane) {
  if (lane == 1) {
    Surrogate::Lane& L = s->lane1;
    return LaneRef{L.cap, L.gO, L.gP, L.block_count, L.block_off, L.list, L.n_list, L.rmask, L.rlist,
                   L.rblock_count, L.rblock_off, L.rcount, &L.order};
  }
  return LaneRef{s->gcap, s->gO, s->gP, s->block_count, s->block_off, s->list, s->n_list, s->rmask, s->rlist,
                 s->rblock_count, s->rblock_off, s->rcount, &s->order};
}

static void free_lane1(Surrogate* s) {
  Surrogate::Lane& L = s->lane1;
  cudaFree(L.gO); cudaFree(L.gP); cudaFree(L.block_count); cudaFree(L.block_off); cudaFree(L.list);
  cudaFree(L.n_list); cudaFree(L.rmask); cudaFree(L.rlist); cudaFree(L.rblock_count); cudaFree(L.rblock_off);
  cudaFree(L.rcount);
  order_free(&L.order);
  L.gO = L.gP = nullptr;
  L.block_count = L.block_off = L.list = L.n_list = L.rlist = L.rblock_count = L.rblock_off = L.rcount = nullptr;
  L.rmask = nullptr;
  L.cap = 0;
}

static long param_layout(Surrogate* s) {
  long off = 0;
  for (int l = 0; l < kMlpLayers; ++l) {
    s->offW[l] = off;
    off += (long)mlp_out(l) * mlp_in(l);
    s->offb[l] = off;
    off += mlp_out(l);
  }
  return off;
}

int surrogate_param_count() {
  int off = 0;
  for (int l = 0; l < kMlpLayers; ++l) off += mlp_out(l) * mlp_in(l) + mlp_out(l);
  return off;
}

void surrogate_upload_tables(const DevMech& dm, cudaStream_t st) {
  cudaMemcpyToSymbolAsync(c_mech, &dm, sizeof(DevMech), 0, cudaMemcpyHostToDevice, st);
}

Surrogate* surrogate_create(const DevMech& dm) {
  Surrogate* s = new Surrogate();
  s->n_params = param_layout(s);
  (void)dm;  // the gate's tables are put in place with the handle's (surrogate_upload_tables)
  const size_t P = (size_t)s->n_params;
  if (cudaMalloc(&s->w, P * 4) != cudaSuccess || cudaMalloc(&s->m, P * 4) != cudaSuccess ||
      cudaMalloc(&s->v, P * 4) != cudaSuccess || cudaMalloc(&s->gr, P * 4) != cudaSuccess ||
      cudaMalloc(&s->wb, P * 2) != cudaSuccess || cudaMalloc(&s->d_norm, sizeof(MlpNorm)) != cudaSuccess ||
      cudaMalloc(&s->d_loss, sizeof(double)) != cudaSuccess || cudaMalloc(&s->d_err, 4) != cudaSuccess ||
      cudaMallocHost(&s->h_err, 4) != cudaSuccess) {
    cudaGetLastError();
    s->uploaded = false;
    return s;
  }
  cudaMemset(s->d_err, 0, 4);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTgSmem);
  cudaMemset(s->w, 0, P * 4);
  cudaMemset(s->m, 0, P * 4);
  cudaMemset(s->v, 0, P * 4);
  cudaMemset(s->wb, 0, P * 2);
  s->uploaded = true;
  return s;
}

static void free_act(Surrogate* s) {
  cudaFree(s->X);
  for (int l = 0; l < kMlpLayers; ++l) {
    cudaFree(s->H[l]);
    cudaFree(s->Z[l]);
    s->H[l] = nullptr;
    s->Z[l] = nullptr;
  }
  cudaFree(s->dHb); cudaFree(s->O); cudaFree(s->dOf); cudaFree(s->dHf); cudaFree(s->dZf); cudaFree(s->dOb);
  cudaFree(s->Yb); cudaFree(s->idx);
  s->X = s->dHb = s->dOb = nullptr;
  s->O = s->dOf = s->dHf = s->dZf = s->Yb = nullptr;
  s->idx = nullptr;
  s->cap = 0;
}

void surrogate_destroy(Surrogate* s) {
  if (!s) return;
  free_act(s);
  cudaFree(s->w); cudaFree(s->m); cudaFree(s->v); cudaFree(s->gr); cudaFree(s->wb); cudaFree(s->d_norm);
  cudaFree(s->iX); cudaFree(s->iH[0]); cudaFree(s->iH[1]); cudaFree(s->iO);
  cudaFree(s->d_loss); cudaFree(s->flag); cudaFree(s->gO); cudaFree(s->gP); cudaFree(s->block_count); cudaFree(s->block_off);
  cudaFree(s->list);
  cudaFree(s->n_list);
  cudaFree(s->rmask); cudaFree(s->rlist); cudaFree(s->rblock_count); cudaFree(s->rblock_off); cudaFree(s->rcount);
  order_free(&s->order);
  free_lane1(s);
  cudaFree(s->d_err);
  cudaFreeHost(s->h_err);
  delete s;
}

bool surrogate_ready(const Surrogate* s) { return s && s->ready && s->uploaded; }
void surrogate_set_ready(Surrogate* s, bool r) { s->ready = r; }
void surrogate_set_cell_order(Surrogate* s, bool by_temperature) { s->order_cells = by_temperature; }
void surrogate_set_gate(Surrogate* s, double elem_tol, double raw_elem_tol, double dT_tol, double dT_max) {
  const GateCfg g0 = s->gate;
  s->gate = GateCfg{elem_tol, raw_elem_tol, dT_tol, dT_max, g0.dt_max, g0.partner, g0.agree_Y, g0.agree_T};
}
void surrogate_set_gate_dt(Surrogate* s, double dt_max) { s->gate.dt_max = dt_max; }
void surrogate_set_dt_band(Surrogate* s, double dt_lo, double dt_hi) {
  s->dt_band_lo = dt_lo;
  s->dt_band_hi = dt_hi;
}
void surrogate_set_gate_band(Surrogate* s, int band, double dt_max, double elem_tol, double raw_elem_tol,
                             double dT_tol, double dT_max) {
  if (band < 1 || band >= kGateBands) return;
  s->xgate[band - 1] = GateCfg{elem_tol, raw_elem_tol, dT_tol, dT_max, dt_max, -1, 0.0, 0.0};
}

static GateNet gate_net(const Surrogate* s, double lo, double hi) {
  GateNet g{};
  g.nm = s->d_norm;
  g.gc = s->gate;
  g.lo = lo;
  g.hi = hi;
  g.on = 1;
  for (int b = 0; b < kGateBands - 1; ++b) g.xb[b] = s->xgate[b];
  g.dt_lo = s->dt_band_lo;
  g.dt_hi = s->dt_band_hi;
  return g;
}
void surrogate_set_band(Surrogate* s, bool set, double lo, double hi) {
  s->band_set = set;
  s->band_lo = lo;
  s->band_hi = hi;
}
void surrogate_set_partner(Surrogate* s, int partner, double agree_Y, double agree_T) {
  s->gate.partner = partner;
  s->gate.agree_Y = agree_Y;
  s->gate.agree_T = agree_T;
}

static std::string ck(cudaError_t e, const char* what) {
  return e == cudaSuccess ? std::string() : std::string(what) + ": " + cudaGetErrorString(e);
}

static std::string ensure_act(Surrogate* s, long n) {
  if (n <= s->cap) return "";
  free_act(s);
  const long np = (n + 63) / 64 * 64;
  std::string e;
  e = ck(cudaMalloc(&s->X, np * kMlpInPad * 2), "alloc X");
  if (!e.empty()) return e;
  for (int l = 0; l < kMlpLayers; ++l) {
    if ((e = ck(cudaMalloc(&s->H[l], np * mlp_out(l) * 2), "alloc H")).size()) return e;
    if ((e = ck(cudaMalloc(&s->Z[l], np * mlp_out(l) * 4), "alloc Z")).size()) return e;
  }
  if ((e = ck(cudaMalloc(&s->O, np * kMlpOutPad * 4), "alloc O")).size()) return e;
  if ((e = ck(cudaMalloc(&s->dOf, np * kMlpOutPad * 4), "alloc dO")).size()) return e;
  if ((e = ck(cudaMalloc(&s->dOb, np * kMlpOutPad * 2), "alloc dO")).size()) return e;
  if ((e = ck(cudaMalloc(&s->dHf, np * kMlpHid * 4), "alloc dH")).size()) return e;
  if ((e = ck(cudaMalloc(&s->dHb, np * kMlpHid * 2), "alloc dH")).size()) return e;
  if ((e = ck(cudaMalloc(&s->dZf, np * kMlpHid * 4), "alloc dZ")).size()) return e;
  if ((e = ck(cudaMalloc(&s->Yb, np * kMlpOut * 4), "alloc Y")).size()) return e;
  if ((e = ck(cudaMalloc(&s->idx, np * 4), "alloc idx")).size()) return e;
  s->cap = np;
  return "";
}

static std::string ensure_infer(Surrogate* s, long n) {
  if (n <= s->icap) return "";
  cudaFree(s->iX); cudaFree(s->iH[0]); cudaFree(s->iH[1]); cudaFree(s->iO);
  s->iX = s->iH[0] = s->iH[1] = nullptr;
  s->iO = nullptr;
  s->icap = 0;
  const long np = (n + 63) / 64 * 64;
  std::string e;
  if ((e = ck(cudaMalloc(&s->iX, np * kMlpInPad * 2), "alloc X")).size()) return e;
  if ((e = ck(cudaMalloc(&s->iH[0], np * kMlpHid * 2), "alloc H")).size()) return e;
  if ((e = ck(cudaMalloc(&s->iH[1], np * kMlpHid * 2), "alloc H")).size()) return e;
  if ((e = ck(cudaMalloc(&s->iO, np * kMlpOutPad * 4), "alloc O")).size()) return e;
  s->icap = np;
  return "";
}

static std::string ensure_gate(Surrogate* s, long n) {
  if (n <= s->gcap) return "";
  cudaFree(s->flag); cudaFree(s->block_count); cudaFree(s->block_off); cudaFree(s->list); cudaFree(s->n_list);
  cudaFree(s->rmask); cudaFree(s->rlist); cudaFree(s->rblock_count); cudaFree(s->rblock_off); cudaFree(s->rcount);
  s->rmask = nullptr;
  s->rlist = s->rblock_count = s->rblock_off = s->rcount = nullptr;
  cudaFree(s->gO);
  cudaFree(s->gP);
  s->gO = s->gP = nullptr;
  const long nb = (n + kCompactBlock - 1) / kCompactBlock;
  std::string e;
  if ((e = ck(cudaMalloc(&s->gO, sizeof(float) * kMlpOut * (size_t)n), "alloc outputs")).size()) return e;
  if ((e = ck(cudaMalloc(&s->gP, sizeof(float) * kMlpOut * (size_t)n), "alloc partner outputs")).size()) return e;
  if ((e = ck(cudaMalloc(&s->flag, n), "alloc flag")).size()) return e;
  if ((e = ck(cudaMalloc(&s->block_count, nb * 4), "alloc counts")).size()) return e;
  if ((e = ck(cudaMalloc(&s->block_off, nb * 4), "alloc offsets")).size()) return e;
  if ((e = ck(cudaMalloc(&s->list, n * 4), "alloc list")).size()) return e;
  if ((e = ck(cudaMalloc(&s->n_list, 4), "alloc count")).size()) return e;
  if ((e = ck(cudaMalloc(&s->rmask, n), "alloc route masks")).size()) return e;
  if ((e = ck(cudaMalloc(&s->rlist, sizeof(int) * kMaxNets * (size_t)n), "alloc network lists")).size()) return e;
  if ((e = ck(cudaMalloc(&s->rblock_count, sizeof(int) * kMaxNets * nb), "alloc network counts")).size()) return e;
  if ((e = ck(cudaMalloc(&s->rblock_off, sizeof(int) * kMaxNets * nb), "alloc network offsets")).size()) return e;
  if ((e = ck(cudaMalloc(&s->rcount, sizeof(int) * kMaxNets), "alloc network totals")).size()) return e;
  if ((e = order_reserve(&s->order, n)).size()) return e;
  s->gcap = n;
  return "";
}

std::string surrogate_init(Surrogate* s, unsigned long long seed, cudaStream_t st) {
  std::vector<float> h((size_t)s->n_params, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kMlpLayers; ++l) {
    const int fan_in = l == 0 ? kMlpIn : kMlpHid;
    const float bound = std::sqrt(6.0f / (float)fan_in) * (l == kMlpLayers - 1 ? 0.25f : 1.0f);
    std::uniform_real_distribution<float> U(-bound, bound);
    for (int o = 0; o < mlp_out(l); ++o)
      for (int i = 0; i < mlp_in(l); ++i) {
        const bool live = (l == 0 ? i < kMlpIn : true) && (l == kMlpLayers - 1 ? o < kMlpOut : true);
        h[s->offW[l] + (long)o * mlp_in(l) + i] = live ? U(rng) : 0.f;
      }
  }
  s->step = 0;
  std::string e = surrogate_set_params(s, h.data(), st);
  if (!e.empty()) return e;
  cudaMemsetAsync(s->m, 0, s->n_params * 4, st);
  cudaMemsetAsync(s->v, 0, s->n_params * 4, st);
  return ck(cudaStreamSynchronize(st), "init");
}

std::string surrogate_set_norm(Surrogate* s, const MlpNorm& norm) {
  s->norm = norm;
  return ck(cudaMemcpy(s->d_norm, &norm, sizeof(MlpNorm), cudaMemcpyHostToDevice), "norm upload");
}

MlpNorm surrogate_get_norm(const Surrogate* s) { return s->norm; }

std::string surrogate_get_params(Surrogate* s, float* host, cudaStream_t st) {
  std::string e = ck(cudaMemcpyAsync(host, s->w, s->n_params * 4, cudaMemcpyDeviceToHost, st), "params D2H");
  if (!e.empty()) return e;
  return ck(cudaStreamSynchronize(st), "params D2H");
}

std::string surrogate_set_params(Surrogate* s, const float* host, cudaStream_t st) {
  std::string e = ck(cudaMemcpyAsync(s->w, host, s->n_params * 4, cudaMemcpyHostToDevice, st), "params H2D");
  if (!e.empty()) return e;
  k_to_bf16<<<64, 256, 0, st>>>(s->n_params, s->w, s->wb);
  return ck(cudaStreamSynchronize(st), "params H2D");
}

std::string surrogate_features(Surrogate* s, long n, long ld, double dt, const double* dt_cells, const double* T,
                               const double* rho, const double* Y, float* xraw, __nv_bfloat16* x,
                               cudaStream_t st) {
  if (n <= 0) return "";
  k_features<<<std::min<long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(n, ld, dt, dt_cells, T, rho, Y, s->d_norm,
                                                                      xraw, x);
  return ck(cudaGetLastError(), "features");
}

// Forward over n rows of bf16 features; keeps H/Z for backward.
static cudaError_t forward(Surrogate* s, long n, const __nv_bfloat16* x, float* out, cudaStream_t st) {
  const __nv_bfloat16* in = x;
  for (int l = 0; l < kMlpLayers; ++l) {
    GemmArgs g{};
    g.M = (int)n;
    g.N = mlp_out(l);
    g.K = mlp_in(l);
    g.A = in;
    g.sam = mlp_in(l);
    g.sak = 1;
    g.B = s->wb + s->offW[l];
    g.sbk = 1;
    g.sbn = mlp_in(l);
    g.bias = s->w + s->offb[l];
    const bool last = l == kMlpLayers - 1;
    g.C = last ? out : s->Z[l];
    g.ldc = mlp_out(l);
    g.H = last ? nullptr : s->H[l];
    g.ldh = mlp_out(l);
    g.gelu = 1;
    cudaError_t e = gemm(g, st, s->d_err);
    if (e != cudaSuccess) return e;
    in = s->H[l];
  }
  return cudaSuccess;
}

std::string surrogate_forward(Surrogate* s, long n, const __nv_bfloat16* x, float* out, cudaStream_t st) {
  std::string e = ensure_act(s, n);
  if (!e.empty()) return e;
  e = ck(forward(s, n, x, out, st), "forward");
  if (!e.empty()) return e;
  return ck(cudaStreamSynchronize(st), "forward");
}

// Inference forward: bf16 activations ping-pong, no pre-activations kept.
static cudaError_t forward_infer(Surrogate* s, long n, const __nv_bfloat16* x, float* out, cudaStream_t st) {
  const __nv_bfloat16* in = x;
  for (int l = 0; l < kMlpLayers; ++l) {
    GemmArgs g{};
    g.M = (int)n;
    g.N = mlp_out(l);
    g.K = mlp_in(l);
    g.A = in;
    g.sam = mlp_in(l);
    g.sak = 1;
    g.B = s->wb + s->offW[l];
    g.sbk = 1;
    g.sbn = mlp_in(l);
    g.bias = s->w + s->offb[l];
    const bool last = l == kMlpLayers - 1;
    g.C = last ? out : nullptr;
    g.ldc = mlp_out(l);
    g.H = last ? nullptr : s->iH[l & 1];
    g.ldh = mlp_out(l);
    g.gelu = 1;
    cudaError_t e = gemm(g, st, s->d_err);
    if (e != cudaSuccess) return e;
    in = s->iH[l & 1];
  }
  return cudaSuccess;
}

// Gradients of the MSE over B rows (x in s->X-like layout, y normalised).
static cudaError_t backward(Surrogate* s, long B, const __nv_bfloat16* x, const float* y, cudaStream_t st) {
  cudaError_t e = forward(s, B, x, s->O, st);
  if (e != cudaSuccess) return e;
  k_loss_grad<<<std::min<long>((B * kMlpOutPad + 255) / 256, 1024), 256, 0, st>>>(B, s->O, y, s->dOf, s->dOb,
                                                                                   s->d_loss);
  const __nv_bfloat16* dZb = s->dOb;
  const float* dZf = s->dOf;
  for (int l = kMlpLayers - 1; l >= 0; --l) {
    const __nv_bfloat16* Hin = l == 0 ? x : s->H[l - 1];
    // dW[out][in] = sum_b dZ[b][out] Hin[b][in]
    GemmArgs g{};
    g.M = mlp_out(l);
    g.N = mlp_in(l);
    g.K = (int)B;
    g.A = dZb;
    g.sam = 1;
    g.sak = mlp_out(l);
    g.B = Hin;
    g.sbk = mlp_in(l);
    g.sbn = 1;
    g.C = s->gr + s->offW[l];
    g.ldc = mlp_in(l);
    if ((e = gemm(g, st, s->d_err)) != cudaSuccess) return e;
    k_colsum<<<mlp_out(l), 256, 0, st>>>(B, mlp_out(l), dZf, s->gr + s->offb[l]);
    if (l == 0) break;
    // dH[b][in] = sum_out dZ[b][out] W[out][in]
    GemmArgs h{};
    h.M = (int)B;
    h.N = mlp_in(l);
    h.K = mlp_out(l);
    h.A = dZb;
    h.sam = mlp_out(l);
    h.sak = 1;
    h.B = s->wb + s->offW[l];
    h.sbk = mlp_in(l);
    h.sbn = 1;
    h.C = s->dHf;
    h.ldc = mlp_in(l);
    if ((e = gemm(h, st, s->d_err)) != cudaSuccess) return e;
    const long cnt = B * kMlpHid;
    k_gelu_back<<<std::min<long>((cnt + 255) / 256, 4096), 256, 0, st>>>(cnt, s->dHf, s->Z[l - 1], s->dZf,
                                                                         s->dHb);
    dZb = s->dHb;
    dZf = s->dZf;
  }
  return cudaGetLastError();
}

std::string surrogate_grad(Surrogate* s, long n, const __nv_bfloat16* x, const float* y, float* grads_host,
                           double* loss, cudaStream_t st) {
  std::string e = ensure_act(s, n);
  if (!e.empty()) return e;
  cudaMemsetAsync(s->d_loss, 0, sizeof(double), st);
  if ((e = ck(backward(s, n, x, y, st), "backward")).size()) return e;
  if (grads_host) cudaMemcpyAsync(grads_host, s->gr, s->n_params * 4, cudaMemcpyDeviceToHost, st);
  if (loss) cudaMemcpyAsync(loss, s->d_loss, sizeof(double), cudaMemcpyDeviceToHost, st);
  return ck(cudaStreamSynchronize(st), "grad");
}

std::string surrogate_train(Surrogate* s, long n, const __nv_bfloat16* x, const float* y, int epochs, int batch,
                            float lr, unsigned long long seed, float* loss_per_epoch, cudaStream_t st) {
  if (n < batch || batch < 64 || (batch % 64)) return "need n >= batch, batch a multiple of 64";
  std::string e = ensure_act(s, batch);
  if (!e.empty()) return e;
  std::vector<int> perm((size_t)n);
  for (long i = 0; i < n; ++i) perm[i] = (int)i;
  std::mt19937_64 rng(seed);
  // two permutation buffers: the next epoch's order is drawn on the host
  // and copied in while the GPU still runs the current epoch
  int* d_perm = nullptr;
  if ((e = ck(cudaMalloc(&d_perm, 2 * n * 4), "alloc perm")).size()) return e;
  __nv_bfloat16* Xb = nullptr;
  if ((e = ck(cudaMalloc(&Xb, (long)batch * kMlpInPad * 2), "alloc batch")).size()) {
    cudaFree(d_perm);
    return e;
  }
  const long steps = n / batch;
  const double total = (double)steps * epochs;
  long t_local = 0;
  std::shuffle(perm.begin(), perm.end(), rng);
  cudaMemcpyAsync(d_perm, perm.data(), n * 4, cudaMemcpyHostToDevice, st);
  for (int ep = 0; ep < epochs; ++ep) {
    const int* cur = d_perm + (ep & 1) * n;
    cudaMemsetAsync(s->d_loss, 0, sizeof(double), st);
    for (long it = 0; it < steps; ++it) {
      k_gather_rows<<<(batch + 255) / 256, 256, 0, st>>>(batch, cur + it * batch, x, y, Xb, s->Yb);
      cudaError_t ce = backward(s, batch, Xb, s->Yb, st);
      if (ce != cudaSuccess) {
        cudaFree(d_perm);
        cudaFree(Xb);
        return ck(ce, "train step");
      }
      s->step += 1;
      // cosine decay from lr to lr/20 over the run
      const double frac = (double)(t_local++) / total;
      const float lr_t = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.141592653589793 * frac))));
      const float b1 = 0.9f, b2 = 0.999f;
      const float bc1 = 1.f - std::pow(b1, (float)s->step), bc2 = 1.f - std::pow(b2, (float)s->step);
      k_adam<<<64, 256, 0, st>>>(s->n_params, s->w, s->gr, s->m, s->v, s->wb, lr_t, b1, b2, 1e-8f, bc1, bc2);
    }
    if (ep + 1 < epochs) {  // the next epoch's order, drawn while this one runs
      std::shuffle(perm.begin(), perm.end(), rng);
      cudaMemcpyAsync(d_perm + ((ep + 1) & 1) * n, perm.data(), n * 4, cudaMemcpyHostToDevice, st);
    }
    double L = 0.0;
    cudaMemcpyAsync(&L, s->d_loss, sizeof(double), cudaMemcpyDeviceToHost, st);
    if ((e = ck(cudaStreamSynchronize(st), "train epoch")).size()) {
      cudaFree(d_perm);
      cudaFree(Xb);
      return e;
    }
    if (loss_per_epoch) loss_per_epoch[ep] = (float)(L / (double)steps);
  }
  cudaFree(d_perm);
  cudaFree(Xb);
  return "";
}

std::string surrogate_prepare(Surrogate* s, long n, long ld, double dt, const double* dt_cells, const double* T,
                              const double* rho, const double* Y, const double* Y_prod, const double* T_after,
                              const PrepareOpts& o, __nv_bfloat16* x, float* y, cudaStream_t st) {
  if (n <= 0) return "no training states";
  float *xraw = nullptr, *xt = nullptr, *yraw = nullptr;
  double* stats = nullptr;
  std::string e;
  auto release = [&]() {
    cudaFree(xraw);
    cudaFree(xt);
    cudaFree(yraw);
    cudaFree(stats);
  };
  if ((e = ck(cudaMalloc(&xraw, n * kMlpIn * 4), "alloc raw features")).size()) return e;
  if ((e = ck(cudaMalloc(&xt, n * kMlpIn * 4), "alloc network inputs")).size()) { release(); return e; }
  if ((e = ck(cudaMalloc(&yraw, n * kMlpOut * 4), "alloc raw targets")).size()) { release(); return e; }
  if ((e = ck(cudaMalloc(&stats, (2 * kMlpIn + kMlpOut) * 4 * 8), "alloc stats")).size()) { release(); return e; }
  const float log_mask = (float)(o.log_mask & 0x1ffu);
  const int grid = (int)std::min<long>((n + 255) / 256, 148 * 16);
  k_features<<<grid, 256, 0, st>>>(n, ld, dt, dt_cells, T, rho, Y, s->d_norm, xraw, nullptr);
  k_transform<<<grid, 256, 0, st>>>(n, xraw, log_mask, o.log_eps, xt);
  k_targets<<<grid, 256, 0, st>>>(n, ld, dt, dt_cells, T, rho, Y_prod, T_after, o.dt_pow, yraw);
  k_colstats<<<kMlpIn, 1024, 0, st>>>(n, kMlpIn, xraw, stats);
  k_colstats<<<kMlpIn, 1024, 0, st>>>(n, kMlpIn, xt, stats + kMlpIn * 4);
  k_colstats<<<kMlpOut, 1024, 0, st>>>(n, kMlpOut, yraw, stats + 2 * kMlpIn * 4);
  std::vector<double> hs((2 * kMlpIn + kMlpOut) * 4);
  cudaMemcpyAsync(hs.data(), stats, hs.size() * 8, cudaMemcpyDeviceToHost, st);
  if ((e = ck(cudaStreamSynchronize(st), "training statistics")).empty()) {
    MlpNorm nm{};
    for (int j = 0; j < kMlpIn; ++j) {
      nm.x_min[j] = (float)hs[j * 4 + 2];                       // hull: raw features
      nm.x_max[j] = (float)hs[j * 4 + 3];
      nm.x_mu[j] = (float)hs[(kMlpIn + j) * 4 + 0];             // scaling: network inputs
      nm.x_sd[j] = (float)std::max(hs[(kMlpIn + j) * 4 + 1], 1e-12);
    }
    const double* ys = hs.data() + 2 * kMlpIn * 4;
    double sd_max = 0.0;
    for (int j = 0; j < kMlpOut - 1; ++j) sd_max = std::max(sd_max, ys[j * 4 + 1]);
    for (int j = 0; j < kMlpOut; ++j) {
      // one scale for all dY_k makes the loss an absolute-error loss, the
      // measure of the tolerance |dY_k| <= const
      const double sdj = (o.common_dY_scale && j < kMlpOut - 1) ? sd_max : ys[j * 4 + 1];
      nm.y_sd[j] = (float)std::max(sdj, 1e-30);
    }
    nm.hull_margin = o.hull_margin;
    nm.dt_pow = o.dt_pow;
    nm.log_mask = log_mask;
    nm.log_eps = o.log_eps;
    e = surrogate_set_norm(s, nm);
    if (e.empty()) {
      k_standardize<<<grid, 256, 0, st>>>(n, xraw, yraw, s->d_norm, x, y);
      e = ck(cudaStreamSynchronize(st), "standardize");
    }
  }
  release();
  return e;
}

std::string surrogate_reserve(Surrogate* s, long n) {
  if (!s->fused) {
    std::string e = ensure_infer(s, n);
    if (!e.empty()) return e;
  }
  return ensure_gate(s, n);
}

static TcArgs tc_args(Surrogate* s, const StepArgs& a, float* out, long out_ld, int active,
                      const GateNets* routes = nullptr, int net = 0, float* out_partner = nullptr) {
  TcArgs p{};
  if (routes) p.routes = *routes;
  p.net = net;
  p.out_partner = out_partner;
  p.a = a;
  p.nm = s->d_norm;
  p.wb = s->wb;
  p.w = s->w;
  for (int l = 0; l < kMlpLayers; ++l) {
    p.offW[l] = s->offW[l];
    p.offb[l] = s->offb[l];
  }
  p.out = out;
  p.out_ld = out_ld;
  p.active = active;
  p.err = s->d_err;
  return p;
}

static cudaError_t launch_tc(Surrogate* s, const TcArgs& p, cudaStream_t st) {
  const long ntiles = (p.a.n + 127) / 128;
  const int grid = (int)std::max<long>(1, std::min<long>(s->num_sms > 0 ? s->num_sms : 148,
                                                         (ntiles + kTcGroups - 1) / kTcGroups));
  k_mlp_tc<<<grid, 128 * kTcGroups, kTcSmem, st>>>(p);
  return cudaGetLastError();
}

// The FP64 gate over the n cells of a, in a grid of 128-thread blocks.
static cudaError_t launch_gate(Surrogate* s, const StepArgs& a, const float* O, const float* OP, long o_ld,
                               const GateNets& nets, unsigned long long* counters, cudaStream_t st,
                               unsigned char* flag) {
  // one resident wave of blocks (three per SM), each looping over cells: the
  // block's set-up (projector, thermo tables) is paid once per block
  const int sms = s->num_sms > 0 ? s->num_sms : 148;
  const long grid = std::min<long>((a.n + 127) / 128, (long)sms * 3);
  k_gate<<<(unsigned)std::max<long>(grid, 1), 128, 0, st>>>(a, O, OP, o_ld, nets, flag, counters);
  return cudaGetLastError();
}

// Temperature range of a network's training hull (widened by its margin).
static void hull_T(const Surrogate* s, double* lo_out, double* hi_out) {
  const double lo = s->norm.x_min[0], hi = s->norm.x_max[0], m = (double)s->norm.hull_margin * (hi - lo);
  *lo_out = lo - m;
  *hi_out = hi + m;
}

std::string surrogate_infer(Surrogate* s, const StepArgs& a, float* out, cudaStream_t st) {
  if (a.n <= 0) return "";
  std::string e = ck(launch_tc(s, tc_args(s, a, out, 0, 0), st), "tensor-core inference");
  if (!e.empty()) return e;
  if ((e = ck(cudaStreamSynchronize(st), "tensor-core inference")).size()) return e;
  return surrogate_check(s, st);
}

std::string surrogate_check(Surrogate* s, cudaStream_t st) {
  if (!s) return "";
  cudaMemcpyAsync(s->h_err, s->d_err, 4, cudaMemcpyDeviceToHost, st);
  std::string e = ck(cudaStreamSynchronize(st), "surrogate error word");
  if (!e.empty()) return e;
  if (*s->h_err) {
    cudaMemsetAsync(s->d_err, 0, 4, st);
    cudaStreamSynchronize(st);
    return "a tensor-core wait of the MLP kernel timed out; the affected cells were integrated in FP64";
  }
  return "";
}

void surrogate_set_fused(Surrogate* s, bool fused) { s->fused = fused; }

std::string surrogate_reserve_lane1(Surrogate* s, long n) {
  Surrogate::Lane& L = s->lane1;
  if (n <= L.cap) return "";
  free_lane1(s);
  const long nb = (n + kCompactBlock - 1) / kCompactBlock;
  std::string e;
  if ((e = ck(cudaMalloc(&L.gO, sizeof(float) * kMlpOut * (size_t)n), "alloc outputs")).size()) return e;
  if ((e = ck(cudaMalloc(&L.gP, sizeof(float) * kMlpOut * (size_t)n), "alloc partner outputs")).size()) return e;
  if ((e = ck(cudaMalloc(&L.block_count, nb * 4), "alloc counts")).size()) return e;
  if ((e = ck(cudaMalloc(&L.block_off, nb * 4), "alloc offsets")).size()) return e;
  if ((e = ck(cudaMalloc(&L.list, n * 4), "alloc list")).size()) return e;
  if ((e = ck(cudaMalloc(&L.n_list, 4), "alloc count")).size()) return e;
  if ((e = ck(cudaMalloc(&L.rmask, n), "alloc route masks")).size()) return e;
  if ((e = ck(cudaMalloc(&L.rlist, sizeof(int) * kMaxNets * (size_t)n), "alloc network lists")).size()) return e;
  if ((e = ck(cudaMalloc(&L.rblock_count, sizeof(int) * kMaxNets * nb), "alloc network counts")).size()) return e;
  if ((e = ck(cudaMalloc(&L.rblock_off, sizeof(int) * kMaxNets * nb), "alloc network offsets")).size()) return e;
  if ((e = ck(cudaMalloc(&L.rcount, sizeof(int) * kMaxNets), "alloc network totals")).size()) return e;
  if ((e = order_reserve(&L.order, n)).size()) return e;
  L.cap = n;
  return "";
}

bool surrogate_fused(const Surrogate* s) { return s && s->fused; }

cudaError_t surrogate_gate(Surrogate* const* nets_in, const StepArgs& a, long flag_off,
                           unsigned long long* counters, cudaStream_t st, cudaEvent_t* ph, int lane) {
  Surrogate* s = nets_in[0];
  const LaneRef R = lane_ref(s, lane);
  // buffers are reserved by surrogate_reserve (lane 1: surrogate_reserve_lane1)
  // before any graph capture
  if (flag_off < 0 || flag_off + a.n > s->gcap || a.n > R.cap || (!s->fused && (lane != 0 || a.n > s->icap)))
    return cudaErrorMemoryAllocation;
  const long n = a.n;
  unsigned char* flag = s->flag + flag_off;
  cudaError_t e;
  GateNets nets{};
  nets.net[0] = gate_net(s, -1e300, 1e300);
  if (s->fused) {
    // routing bands: the hulls' temperature ranges; network 0 also takes
    // what lies above its hull (its hull test then sends it to FP64)
    for (int i = 0; i < kMaxNets; ++i) {
      Surrogate* si = nets_in[i];
      if (!si || !surrogate_ready(si)) continue;
      double lo, hi;
      hull_T(si, &lo, &hi);
      if (i == 0) hi = 1e300;
      if (si->band_set) {
        lo = si->band_lo;
        hi = si->band_hi;
      }
      nets.net[i] = gate_net(si, lo, hi);
    }
    // each network's cells listed once, then the network outputs of the
    // listed cells, planar, then the wide FP64 gate
    const int nb = (int)((n + kCompactBlock - 1) / kCompactBlock);
    if (n > 0) {
      k_route_count<<<nb, kCompactBlock, 0, st>>>(a, nets, R.rmask, nb, R.rblock_count);
      k_route_scan<<<kMaxNets, 1024, 0, st>>>(nb, R.rblock_count, R.rblock_off, R.rcount);
      k_route_scatter<<<nb, kCompactBlock, 0, st>>>(n, R.rmask, nb, R.rblock_off, R.cap, R.rlist);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    for (int i = 0; i < kMaxNets; ++i) {
      if (!nets.net[i].on) continue;
      TcArgs p = tc_args(nets_in[i], a, R.gO, n, 1, &nets, i, R.gP);
      p.list = R.rlist + (size_t)i * R.cap;
      p.list_count = R.rcount + i;
      if ((e = launch_tc(nets_in[i], p, st)) != cudaSuccess) return e;
    }
    if ((e = launch_gate(s, a, R.gO, R.gP, n, nets, counters, st, flag)) != cudaSuccess) return e;
  } else {
    k_features<<<std::min<long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(n, a.ld, a.dt, a.dt_cells, a.T, a.rho,
                                                                        a.Y, s->d_norm, nullptr, s->iX);
    if ((e = forward_infer(s, n, s->iX, s->iO, st)) != cudaSuccess) return e;
    if ((e = launch_gate(s, a, s->iO, nullptr, 0, nets, counters, st, flag)) != cudaSuccess) return e;
  }
  if (ph) cudaEventRecord(ph[1], st);
  return cudaSuccess;
}

cudaError_t surrogate_fallback(Surrogate* const* nets_in, const StepArgs& a, long flag_off,
                               unsigned long long* counters, cudaStream_t st, const FallbackFn& fallback, int lane) {
  Surrogate* s = nets_in[0];
  const LaneRef R = lane_ref(s, lane);
  if (flag_off < 0 || flag_off + a.n > s->gcap || a.n > R.cap) return cudaErrorMemoryAllocation;
  const long n = a.n;
  const unsigned char* flag = s->flag + flag_off;
  cudaError_t e;
  if (s->order_cells) {
    // rejected cells grouped by temperature: the fallback's warps then hold
    // cells with similar BDF paths
    if ((e = order_cells_by_temperature(n, a.T, a.bc, flag, R.order, R.list, R.n_list,
                                        counters ? counters + 7 : nullptr, st)) != cudaSuccess)
      return e;
  } else {
    const int nb = (int)((n + kCompactBlock - 1) / kCompactBlock);
    k_flag_count<<<nb, kCompactBlock, 0, st>>>(n, flag, R.block_count);
    k_scan_counts<<<1, 1024, 0, st>>>(nb, R.block_count, R.block_off, R.n_list, counters);
    k_compact<<<nb, kCompactBlock, 0, st>>>(n, flag, R.block_off, R.list);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  StepArgs fa = a;
  fa.cell_list = R.list;
  fa.n_list_dev = R.n_list;
  fa.n_list = (int)n;  // upper bound for the grid; the kernel reads the device count
  return fallback(fa, st);
}

cudaError_t surrogate_step(Surrogate* const* nets_in, const StepArgs& a, const LaunchCfg& cfg, int* queue,
                           unsigned long long* counters, cudaStream_t st, const FallbackFn& fallback,
                           cudaEvent_t* ph) {
  (void)cfg;
  (void)queue;
  cudaError_t e = surrogate_gate(nets_in, a, 0, counters, st, ph, 0);
  if (e != cudaSuccess) return e;
  return surrogate_fallback(nets_in, a, 0, counters, st, fallback, 0);
}

// Bounded-wait probe: one warp waits on an mbarrier that nothing arrives at,
// with the same bounded wait the tensor-core kernel uses, and reports that the
// wait gave up (and after how long) instead of hanging.
__global__ void k_bounded_wait_probe(unsigned long long limit_ns, int* timed_out, unsigned long long* waited_ns) {
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t mb = tc::smem_u32(&bar);
  if (threadIdx.x == 0) tc::mbar_init(mb, 1);
  __syncwarp();
  const uint64_t t0 = tc::globaltimer_ns();
  const bool ok = tc::mbar_wait(mb, 0, limit_ns);  // phase 0 never completes
  const uint64_t t1 = tc::globaltimer_ns();
  if (threadIdx.x == 0) {
    *timed_out = ok ? 0 : 1;
    *waited_ns = t1 - t0;
  }
}

std::string bounded_wait_probe(unsigned long long limit_ns, int* timed_out, double* waited_ms) {
  int* d_flag = nullptr;
  unsigned long long* d_ns = nullptr;
  std::string err;
  if (cudaMalloc(&d_flag, sizeof(int)) != cudaSuccess || cudaMalloc(&d_ns, sizeof(unsigned long long)) != cudaSuccess)
    err = "cudaMalloc";
  if (err.empty()) {
    k_bounded_wait_probe<<<1, 32>>>(limit_ns, d_flag, d_ns);
    int f = 0;
    unsigned long long ns = 0;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&f, d_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&ns, d_ns, sizeof(ns), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) err = cudaGetErrorString(e);
    if (timed_out) *timed_out = f;
    if (waited_ms) *waited_ms = (double)ns * 1e-6;
  }
  cudaFree(d_flag);
  cudaFree(d_ns);
  return err;
}

}  // namespace nrg
