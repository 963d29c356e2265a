// Gated MLP surrogate of the per-cell chemistry increment (host interface).
#pragma once

#include <functional>
#include <string>

#include <cuda_runtime.h>

#include "chem_device.cuh"
#include "chem_kernels.hpp"
#include "mlp.cuh"

namespace nrg {

struct Surrogate;

// Networks of one handle: 0 the main one, the others for narrower
// temperature bands (routing in surrogate_step).
constexpr int kMaxNets = 8;
// gate settings per network: one for steps up to its dt bound and up to
// kGateBands - 1 more for longer steps
constexpr int kGateBands = 4;

using FallbackFn = std::function<cudaError_t(const StepArgs&, cudaStream_t)>;

Surrogate* surrogate_create(const DevMech& dm);
// The gate's copy of the mechanism tables (per translation unit).
void surrogate_upload_tables(const DevMech& dm, cudaStream_t st);
void surrogate_destroy(Surrogate* s);
bool surrogate_ready(const Surrogate* s);

// Allocates the inference and compaction buffers for n cells (call outside
// stream capture).
std::string surrogate_reserve(Surrogate* s, long n);
// One warp waits on an mbarrier nothing arrives at, with the bounded wait of
// the tensor-core kernel (limit_ns); reports whether the wait gave up.
std::string bounded_wait_probe(unsigned long long limit_ns, int* timed_out, double* waited_ms);

// Enqueues features -> MLP -> gate/outputs -> compaction -> FP64 fallback
// on the cells the gate rejects.  nets: kMaxNets networks, nets[0] the main
// one (ready; it owns the step's buffers), the others may be null or not
// ready; each active cell goes to the ready network of highest index whose
// hull's temperature range holds it.  counters[6] / [7] receive surrogate /
// fallback cell counts.
// ph (may be null): events recorded at phase boundaries: ph[1] after the
// network and the gate kernel; the fallback callback records ph[2] / ph[3]
// around the integrator.
cudaError_t surrogate_step(Surrogate* const* nets, const StepArgs& a, const LaunchCfg& cfg, int* queue,
                           unsigned long long* counters, cudaStream_t st, const FallbackFn& fallback,
                           cudaEvent_t* ph);
// The two halves of surrogate_step, for callers that stream a field in
// chunks: surrogate_gate runs the networks and the gate on a.n cells whose
// accept/reject flags go to positions [flag_off, flag_off + a.n) of the
// step's flag array (accepted and skipped cells are final after it);
// surrogate_fallback then integrates the a.n cells at a's pointers whose
// flags sit at [flag_off, flag_off + a.n) and were set by surrogate_gate
// calls before it.
// lane: which of the two sets of per-step scratch the call uses (0 always
// exists; 1 after surrogate_reserve_lane1, fused inference only), so that
// calls on two streams with different lanes may run at once.
cudaError_t surrogate_gate(Surrogate* const* nets, const StepArgs& a, long flag_off,
                           unsigned long long* counters, cudaStream_t st, cudaEvent_t* ph, int lane = 0);
cudaError_t surrogate_fallback(Surrogate* const* nets, const StepArgs& a, long flag_off,
                               unsigned long long* counters, cudaStream_t st, const FallbackFn& fallback,
                               int lane = 0);
// Scratch of lane 1 for chunks of up to n cells (before any graph capture).
std::string surrogate_reserve_lane1(Surrogate* s, long n);
// Whether the tensor-core inference path is selected (the default).
bool surrogate_fused(const Surrogate* s);

// ---- training / inspection (device pointers unless stated)
std::string surrogate_init(Surrogate* s, unsigned long long seed, cudaStream_t st);
std::string surrogate_set_norm(Surrogate* s, const MlpNorm& norm);
MlpNorm surrogate_get_norm(const Surrogate* s);
// flattened fp32 parameters, per layer W[out][in_pad] then b[out]
int surrogate_param_count();
std::string surrogate_get_params(Surrogate* s, float* host, cudaStream_t st);
std::string surrogate_set_params(Surrogate* s, const float* host, cudaStream_t st);
// raw features (n x 12 fp32) and standardised padded bf16 features (n x 16)
std::string surrogate_features(Surrogate* s, long n, long ld, double dt, const double* dt_cells,
                               const double* T, const double* rho, const double* Y, float* xraw,
                               __nv_bfloat16* x, cudaStream_t st);
// network outputs (n x 16 fp32, normalised units) for bf16 features
std::string surrogate_forward(Surrogate* s, long n, const __nv_bfloat16* x, float* out, cudaStream_t st);
// gradient of the mean squared error over one batch (no update)
std::string surrogate_grad(Surrogate* s, long n, const __nv_bfloat16* x, const float* y, float* grads_host,
                           double* loss, cudaStream_t st);
// Adam training over n samples; loss_per_epoch (host) may be null
std::string surrogate_train(Surrogate* s, long n, const __nv_bfloat16* x, const float* y, int epochs, int batch,
                            float lr, unsigned long long seed, float* loss_per_epoch, cudaStream_t st);
// Choices made when the training arrays are prepared.
struct PrepareOpts {
  float hull_margin;    // fraction of each raw feature's range added on both sides of the hull
  float dt_pow;         // targets are divided by (dt / 1e-6)^dt_pow
  unsigned log_mask;    // bit k: Y_k enters the network as log10(Y_k + log_eps)
  float log_eps;
  int common_dY_scale;  // 1: one scale for all dY_k; 0: each its own standard deviation
};
// raw features and targets of integrated training states, fitted
// standardisation and training hull, standardised bf16 x (n x 16) and y (n x 10)
std::string surrogate_prepare(Surrogate* s, long n, long ld, double dt, const double* dt_cells, const double* T,
                              const double* rho, const double* Y, const double* Y_prod, const double* T_after,
                              const PrepareOpts& opts, __nv_bfloat16* x, float* y, cudaStream_t st);
void surrogate_set_ready(Surrogate* s, bool ready);
// Fallback cells grouped by temperature (default) or in cell order.
void surrogate_set_cell_order(Surrogate* s, bool by_temperature);
// Inference path of surrogate_step: the tensor-core network kernel (default)
// or the GEMM chain (one tcgen05 GEMM launch per layer), either followed by
// the gate kernel.
void surrogate_set_fused(Surrogate* s, bool fused);
// Features + MLP on tcgen05 over the n cells of a (no gate): out is n x 16
// fp32 network outputs in normalised units; synchronises.
std::string surrogate_infer(Surrogate* s, const StepArgs& a, float* out, cudaStream_t st);
// Reads and clears the tensor-core kernel's error word (after the step's work).
std::string surrogate_check(Surrogate* s, cudaStream_t st);
void surrogate_set_gate(Surrogate* s, double elem_tol, double raw_elem_tol, double dT_tol, double dT_max);
// Longest step (s) whose cells the gate may accept.
void surrogate_set_gate_dt(Surrogate* s, double dt_max);
// Routing step band (dt_lo, dt_hi] of a network (default (0, 1e300]): cells
// whose step lies outside it are not routed to it.
void surrogate_set_dt_band(Surrogate* s, double dt_lo, double dt_hi);
// Gate bounds of band b (1 .. kGateBands - 1) for steps in (the previous
// band's dt_max, dt_max]; band 0 is surrogate_set_gate / surrogate_set_gate_dt.
// dt_max 0 leaves the band unused.
void surrogate_set_gate_band(Surrogate* s, int band, double dt_max, double elem_tol, double raw_elem_tol,
                             double dT_tol, double dT_max);
// Committee check of a network: partner (-1: none), agreement bounds.
void surrogate_set_partner(Surrogate* s, int partner, double agree_Y, double agree_T);
// Routing band [lo, hi) of a network (set = false: its hull's T range).
void surrogate_set_band(Surrogate* s, bool set, double lo, double hi);

}  // namespace nrg
