// Kernel templates of the chemistry step (included by the per-variant
// translation units chem_k_*.cu, which instantiate them).
//
//   k_chem_plain  -- one thread per cell, grid covers all cells.
//   k_chem_queue  -- persistent grid; every lane pulls cells from a device
//                    work queue and is refilled as soon as its cell reaches
//                    t = dt, so lanes never wait for the slowest cell of a
//                    warp.  Block size, blocks per SM and the number of cells
//                    a lane reserves per queue fetch are autotuned on the host.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "chem_bdf.cuh"
#include "chem_kernels.hpp"
#include "chem_warp.cuh"

namespace nrg {

namespace cg = cooperative_groups;

// Counter slots (unsigned long long): cells integrated, steps, RHS
// evaluations, Jacobians, linear solves, cells not ok.
enum { kCntCells = 0, kCntSteps, kCntRhs, kCntJac, kCntSolve, kCntBad, kCntSlots };

__device__ __forceinline__ void block_flush_counters(unsigned long long* counters,
                                                     unsigned long long v[kCntSlots]) {
  __shared__ unsigned long long s_cnt[kCntSlots];
  if (threadIdx.x < kCntSlots) s_cnt[threadIdx.x] = 0;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kCntSlots; ++i) {
    unsigned long long x = v[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(&s_cnt[i], x);
  }
  __syncthreads();
  if (threadIdx.x < kCntSlots && s_cnt[threadIdx.x]) atomicAdd(&counters[threadIdx.x], s_cnt[threadIdx.x]);
}

template <int N, int R, int JAC, typename LUT, int BS, int NF, int SPEC>
__global__ void __launch_bounds__(BS, 1) k_chem_plain(StepArgs a, unsigned long long* counters) {
  extern __shared__ __align__(16) char smem[];
  const long li = (long)blockIdx.x * BS + threadIdx.x;
  const long nl = a.cell_list ? (long)(a.n_list_dev ? *a.n_list_dev : a.n_list) : a.n;
  const long cid = (a.cell_list && li < nl) ? (long)a.cell_list[li] : li;
  unsigned long long v[kCntSlots] = {0, 0, 0, 0, 0, 0};
  CellState<N, R, LUT, BS, NF, SPEC> c;
  c.bind(smem, threadIdx.x);
  if (li < nl) {
    if (cell_begin<N, R, JAC>(c, a, cid)) {
      int st;
      while ((st = cell_advance<N, R, JAC, LUT>(c, a.mxstep)) == 0) {
      }
      cell_finish<N, JAC>(c, a, cid, st);
      v[kCntCells] = 1;
      v[kCntSteps] = c.nstep;
      v[kCntRhs] = c.nfe;
      v[kCntJac] = c.nje;
      v[kCntSolve] = c.nsolve;
      v[kCntBad] = st != kCellOk;
    }
  }
  if (counters) block_flush_counters(counters, v);
}

template <int N, int R, int JAC, typename LUT, int BS, int NF, int SPEC>
__global__ void __launch_bounds__(BS, 1) k_chem_queue(StepArgs a, int* queue, int chunk,
                                                       unsigned long long* counters) {
  extern __shared__ __align__(16) char smem[];
  unsigned long long v[kCntSlots] = {0, 0, 0, 0, 0, 0};
  CellState<N, R, LUT, BS, NF, SPEC> c;
  c.bind(smem, threadIdx.x);
  long cur = 0, left = 0, cid = 0;  // logical index, cells still reserved, cell id
  const long nl = a.cell_list ? (long)(a.n_list_dev ? *a.n_list_dev : a.n_list) : a.n;
  bool have = false;
  for (;;) {
    if (!have) {
      if (left == 0) {
        // warp-aggregated reservation of `chunk` cells per requesting lane
        cg::coalesced_group g = cg::coalesced_threads();
        long base = 0;
        if (g.thread_rank() == 0) base = (long)atomicAdd(queue, (int)(g.size() * chunk));
        base = g.shfl(base, 0);
        cur = base + (long)g.thread_rank() * chunk;
        left = chunk;
      } else {
        ++cur;
      }
      --left;
      if (cur >= nl) break;
      cid = a.cell_list ? (long)a.cell_list[cur] : cur;
      have = cell_begin<N, R, JAC>(c, a, cid);
      if (!have) continue;
    }
    const int st = cell_advance<N, R, JAC, LUT>(c, a.mxstep);
    if (st) {
      cell_finish<N, JAC>(c, a, cid, st);
      v[kCntCells] += 1;
      v[kCntSteps] += c.nstep;
      v[kCntRhs] += c.nfe;
      v[kCntJac] += c.nje;
      v[kCntSolve] += c.nsolve;
      v[kCntBad] += st != kCellOk;
      have = false;
    }
  }
  if (counters) block_flush_counters(counters, v);
}

template <int N, int R, int JAC, typename LUT, int BS, int NF, int SPEC>
static cudaError_t launch_bs(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                             unsigned long long* counters, cudaStream_t s) {
  const size_t smem = (size_t)BS * SmemStore<N, R, LUT, BS>::kBytesPerThread;
  cudaError_t e;
  if (cfg.kernel == kKernelThreadQueue) {
    e = cudaFuncSetAttribute(k_chem_queue<N, R, JAC, LUT, BS, NF, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = cfg.grid > 0 ? cfg.grid : 148;
    k_chem_queue<N, R, JAC, LUT, BS, NF, SPEC><<<grid, BS, smem, s>>>(a, queue, cfg.chunk, counters);
  } else {
    e = cudaFuncSetAttribute(k_chem_plain<N, R, JAC, LUT, BS, NF, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    const long nl = a.cell_list ? (long)a.n_list : a.n;
    const long grid = (nl + BS - 1) / BS;
    if (grid > 0) k_chem_plain<N, R, JAC, LUT, BS, NF, SPEC><<<(unsigned)grid, BS, smem, s>>>(a, counters);
  }
  return cudaGetLastError();
}


__host__ __device__ constexpr size_t warp_tables_bytes() { return (sizeof(DevMech) + 15) / 16 * 16; }

// Warp-per-cell persistent kernel: every warp pulls `chunk` cells at a time
// from the work queue and integrates them one after the other.
template <int N, int R, int JAC, typename LUT, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, WARPS == 4 ? 4 : 1) k_chem_warp(StepArgs a, int* queue, int chunk,
                                                         unsigned long long* counters) {
  // dynamic shared memory: the mechanism tables, then one scratch per warp
  extern __shared__ __align__(16) char wsmem[];
  DevMech& sM = *reinterpret_cast<DevMech*>(wsmem);
  WarpSmem<N, R, LUT>* sm = reinterpret_cast<WarpSmem<N, R, LUT>*>(wsmem + warp_tables_bytes());
  {
    // lanes read per-reaction and per-species entries at different addresses,
    // which __constant__ memory would serialize: work from a shared copy
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(a.mech);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sM);
    for (int i = threadIdx.x; i < (int)(sizeof(DevMech) / 8); i += WARPS * 32) dst[i] = src[i];
    __syncthreads();
  }
  unsigned long long v[kCntSlots] = {0, 0, 0, 0, 0, 0};
  WarpCell<N, R, LUT> c;
  c.M = &sM;
  c.lane = threadIdx.x & 31;
  c.sm = &sm[threadIdx.x >> 5];
  const long nl = a.cell_list ? (long)(a.n_list_dev ? *a.n_list_dev : a.n_list) : a.n;
  long cur = 0, left = 0;
  for (;;) {
    if (left == 0) {
      int base = 0;
      if (c.lane == 0) base = atomicAdd(queue, chunk);
      cur = __shfl_sync(kFullMask, base, 0);
      left = chunk;
    } else {
      ++cur;
    }
    --left;
    if (cur >= nl) break;
    const long cid = a.cell_list ? (long)a.cell_list[cur] : cur;
    if (!warp_cell_begin(c, a, cid)) continue;
    int st;
    while ((st = warp_cell_advance<N, R, JAC>(c, a.mxstep)) == 0) {
    }
    warp_cell_finish(c, a, cid, st);
    if (c.lane == 0) {
      v[kCntCells] += 1;
      v[kCntSteps] += c.nstep;
      v[kCntRhs] += c.nfe;
      v[kCntJac] += c.nje;
      v[kCntSolve] += c.nsolve;
      v[kCntBad] += st != kCellOk;
    }
  }
  if (counters) block_flush_counters(counters, v);
}

template <int N, int R, int JAC, typename LUT, int WARPS>
static cudaError_t launch_warp(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                               unsigned long long* counters, cudaStream_t s) {
  const size_t smem = warp_tables_bytes() + WARPS * sizeof(WarpSmem<N, R, LUT>);
  cudaError_t e = cudaFuncSetAttribute(k_chem_warp<N, R, JAC, LUT, WARPS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int grid = cfg.grid;
  if (grid <= 0) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chem_warp<N, R, JAC, LUT, WARPS>, WARPS * 32, smem);
    grid = sms * (per_sm > 0 ? per_sm : 1);
  }
  k_chem_warp<N, R, JAC, LUT, WARPS><<<grid, WARPS * 32, smem, s>>>(a, queue, cfg.chunk, counters);
  return cudaGetLastError();
}

// Launches one (JAC, LUT) variant: cfg.kernel selects thread-per-cell (grid
// or work queue, 32- or 64-thread blocks) or warp-per-cell (128- or 256-thread
// blocks).  With 32-thread blocks every warp is its own block, so an SM slot
// is handed to a new block as soon as the warp's cells are done instead of
// waiting for the slowest warp of a larger block.  NF mechanism species, NI of
// them integrated by the thread-per-cell kernels (the translation unit's
// tables are numbered over those NI); the warp kernel integrates all NF from
// the full tables it copies to shared memory.  SPEC != 0: the thread kernels
// use that generated mechanism-specialised RHS and iteration matrix.
template <int NF, int NI, int R, int JAC, typename LUT, int SPEC>
static cudaError_t launch_variant(const StepArgs& a, const LaunchCfg& cfg, int* queue,
                                  unsigned long long* counters, cudaStream_t s) {
  if (cfg.kernel == kKernelWarpQueue) {
    switch (cfg.block) {
      case 128: return launch_warp<NF, R, JAC, LUT, 4>(a, cfg, queue, counters, s);
      case 256: return launch_warp<NF, R, JAC, LUT, 8>(a, cfg, queue, counters, s);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (cfg.block) {
    case 32: return launch_bs<NI, R, JAC, LUT, 32, NF, SPEC>(a, cfg, queue, counters, s);
    case 64: return launch_bs<NI, R, JAC, LUT, 64, NF, SPEC>(a, cfg, queue, counters, s);
    default: return cudaErrorInvalidValue;
  }
}

// The thread-per-cell grid kernel only (the shape used for the mechanisms
// other than the default one, which get no queue / warp variants).
template <int NF, int NI, int R, int JAC, typename LUT, int SPEC = 0>
static cudaError_t launch_grid(const StepArgs& a, const LaunchCfg& cfg, int* queue, unsigned long long* counters,
                               cudaStream_t s) {
  if (cfg.kernel != kKernelThreadGrid) return cudaErrorNotSupported;
  switch (cfg.block) {
    case 32: return launch_bs<NI, R, JAC, LUT, 32, NF, SPEC>(a, cfg, queue, counters, s);
    case 64: return launch_bs<NI, R, JAC, LUT, 64, NF, SPEC>(a, cfg, queue, counters, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace nrg
