// MLP surrogate of the per-cell chemistry increment: shapes, activation and
// feature/target definitions shared by the training and inference kernels.
//
//   input  (12): T, log(p / 1 atm), Y_1..Y_9, log10(dt); the species picked by
//                log_mask enter as log10(Y_k + log_eps); each input is
//                standardised by the training-set mean and standard
//                deviation; padded to 16
//   hidden     : 4 layers x 128, GELU (tanh form)
//   output (10): dY_1..dY_9 and dT, divided by (dt / 1e-6)^dt_pow and then by
//                the training-set standard deviation; padded to 16
// Weights and activations are BF16, accumulation FP32.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace nrg {

constexpr int kMlpIn = 12, kMlpInPad = 16, kMlpHid = 128, kMlpOut = 10, kMlpOutPad = 16;
constexpr int kMlpLayers = 5;
__host__ __device__ constexpr int mlp_in(int l) { return l == 0 ? kMlpInPad : kMlpHid; }
__host__ __device__ constexpr int mlp_out(int l) { return l == kMlpLayers - 1 ? kMlpOutPad : kMlpHid; }

// Feature / target scaling and the training hull.
struct MlpNorm {
  float x_mu[kMlpIn], x_sd[kMlpIn];    // of the network inputs (after the log transform)
  float x_min[kMlpIn], x_max[kMlpIn];  // raw-feature range of the training states
  float y_sd[kMlpOut];
  float hull_margin;                   // fraction of the range added on both sides
  float dt_pow;                        // targets are divided by (dt / 1e-6)^dt_pow
  float log_mask;                      // bit k set: Y_k enters as log10(Y_k + log_eps)
  float log_eps;
};

// Network input j (before standardisation) from raw feature j.
__host__ __device__ __forceinline__ float net_feature(float log_mask, float log_eps, int j, float f) {
  const unsigned m = (unsigned)log_mask;
  if (j >= 2 && j < 2 + 9 && ((m >> (j - 2)) & 1u)) return log10f(fmaxf(f, 0.f) + log_eps);
  return f;
}

// Standardised network input j from raw feature j.
__host__ __device__ __forceinline__ float net_input(const MlpNorm& nm, int j, float f) {
  return (net_feature(nm.log_mask, nm.log_eps, j, f) - nm.x_mu[j]) / nm.x_sd[j];
}

// Target scale of a sample with step dt: (dt / 1e-6)^dt_pow, from log10(dt).
__host__ __device__ __forceinline__ float target_scale(float log10_dt, float dt_pow) {
  return dt_pow == 0.f ? 1.f : exp10f(dt_pow * (log10_dt + 6.0f));
}

__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float gelu_f(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanh_fast(u));
}

__device__ __forceinline__ float gelu_grad_f(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float t = tanh_fast(u);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}

}  // namespace nrg
