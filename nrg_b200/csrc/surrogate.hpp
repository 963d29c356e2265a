// Gated MLP surrogate of the per-cell chemistry increment (host interface).
#pragma once

#include <functional>

#include <cuda_runtime.h>

#include "chem_device.cuh"
#include "chem_kernels.hpp"

namespace nrg {

struct Surrogate;

using FallbackFn = std::function<cudaError_t(const StepArgs&, cudaStream_t)>;

Surrogate* surrogate_create(const DevMech& dm);
void surrogate_destroy(Surrogate* s);
bool surrogate_ready(const Surrogate* s);

// Enqueues gate + inference + compaction + FP64 fallback for the cells that
// fail the gate.  counters[6] / [7] receive surrogate / fallback cell counts.
cudaError_t surrogate_step(Surrogate* s, const StepArgs& a, const LaunchCfg& cfg, int* queue,
                           unsigned long long* counters, cudaStream_t st, const FallbackFn& fallback);

}  // namespace nrg
