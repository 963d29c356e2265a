// Temperature order of the integrator's cells: a stable least-significant-
// digit radix sort of (key, cell) pairs over three 8-bit digits.  Per pass:
// digit counts per 8192-cell tile, exclusive scans over the tiles of each
// digit and over the digits, then a stable scatter (tile order, then warp order, then lane order).
// Small HBM-bound kernels next to the integrator's step.
#include <climits>

#include "chem_device.cuh"
#include "order.hpp"

namespace nrg {
namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr int kRounds = kOrderTile / kThreads;
constexpr int kDigits = 1 << kOrderDigitBits;
static_assert(kOrderTile % kThreads == 0, "a tile is a whole number of block-wide rounds");
static_assert(kDigits <= kThreads, "one thread per digit in the column scans");
static_assert(kOrderKeyBits % kOrderDigitBits == 0, "whole digits");

__device__ __forceinline__ uint32_t order_key(double T, int8_t bcv) {
  if (!(T >= kSkipBelowK) || bcv != 0) return 0u;  // skipped by the step (also NaN T)
  return 1u + (uint32_t)fmin((T - kSkipBelowK) * 1024.0, (double)((1u << kOrderKeyBits) - 2u));
}

// Items of one pass: the cells themselves (first pass; keys computed from T,
// cells filtered by flag) or the previous pass's (key, cell) pairs.
struct PassIn {
  long n;            // item bound of the first pass
  const int* count;  // items of the later passes (device), nullptr in the first
  const double* T;
  const int8_t* bc;
  const unsigned char* flag;
  const uint32_t* keys;
  const int* vals;
  int shift;
};

__device__ __forceinline__ long pass_items(const PassIn& p) { return p.count ? (long)*p.count : p.n; }

__device__ __forceinline__ bool load_item(const PassIn& p, long i, long nitems, uint32_t* key, int* val) {
  if (i >= nitems) return false;
  if (p.keys == nullptr) {
    if (p.flag && p.flag[i] == 0) return false;
    *key = order_key(p.T[i], p.bc ? p.bc[i] : (int8_t)0);
    *val = (int)i;
  } else {
    *key = p.keys[i];
    *val = p.vals[i];
  }
  return true;
}

// Digit counts of one tile, written to counts[digit * tiles + tile].  Every
// warp runs all rounds, so the warp-wide votes see all 32 lanes.
__global__ void __launch_bounds__(kThreads) k_rs_count(PassIn p, int* counts, int tiles) {
  __shared__ int sh[kDigits];
  if (threadIdx.x < kDigits) sh[threadIdx.x] = 0;
  __syncthreads();
  const long nitems = pass_items(p);
  const long base = (long)blockIdx.x * kOrderTile;
  const unsigned lane = threadIdx.x & 31u;
  for (int r = 0; r < kRounds; ++r) {
    uint32_t key = 0;
    int val = 0;
    const bool take = load_item(p, base + (long)r * kThreads + threadIdx.x, nitems, &key, &val);
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (take) {
      const int d = (int)((key >> p.shift) & (kDigits - 1));
      const unsigned peers = __match_any_sync(m, d);
      if (lane == (unsigned)(__ffs(peers) - 1)) atomicAdd(&sh[d], __popc(peers));
    }
  }
  __syncthreads();
  if (threadIdx.x < kDigits) counts[(long)threadIdx.x * tiles + blockIdx.x] = sh[threadIdx.x];
}

// Block-wide exclusive scan of one int per thread (blockDim.x a multiple of
// 32, at most 1024; wsum holds blockDim.x / 32 ints); returns the thread's
// exclusive prefix and sets *sum to the block total.
__device__ __forceinline__ int block_exclusive_scan(int v, int* wsum, int* sum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int z = lane < nw ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += y;
    }
    if (lane < nw) wsum[lane] = z;
  }
  __syncthreads();
  const int incl = x + (w > 0 ? wsum[w - 1] : 0);
  *sum = wsum[nw - 1];
  __syncthreads();  // wsum is reused by the next call
  return incl - v;
}

// Per digit (one block each): exclusive scan of its tile counts in place
// (coalesced over the tiles) and the digit's total to digit_base[digit].
__global__ void __launch_bounds__(kThreads) k_rs_scan_tiles(int* counts, int tiles, int* digit_base) {
  __shared__ int wsum[kWarps];
  int* row = counts + (long)blockIdx.x * tiles;
  int carry = 0;
  for (int base = 0; base < tiles; base += kThreads) {
    const int i = base + threadIdx.x;
    const int v = i < tiles ? row[i] : 0;
    int sum = 0;
    const int ex = block_exclusive_scan(v, wsum, &sum);
    if (i < tiles) row[i] = carry + ex;
    carry += sum;
  }
  if (threadIdx.x == 0) digit_base[blockIdx.x] = carry;
}

// Exclusive scan of the digit totals in place (one block of kDigits threads);
// the grand total goes to *total and *total2 (may be null) and is added to
// *counter (may be null).
__global__ void __launch_bounds__(kDigits) k_rs_scan_digits(int* digit_base, int* total, int* total2,
                                                            unsigned long long* counter) {
  __shared__ int wsum[kDigits / 32];
  const int v = digit_base[threadIdx.x];
  int sum = 0;
  const int ex = block_exclusive_scan(v, wsum, &sum);
  digit_base[threadIdx.x] = ex;
  if (threadIdx.x == 0) {
    *total = sum;
    if (total2) *total2 = sum;
    if (counter) atomicAdd(counter, (unsigned long long)sum);  // orders on two streams may add at once
  }
}

// Stable scatter of one tile: an item's slot is its tile's offset for its
// digit, plus the items of that digit in earlier iterations of the tile
// loop, earlier warps of this iteration and earlier lanes of its warp.
__global__ void __launch_bounds__(kThreads) k_rs_scatter(PassIn p, const int* offsets, const int* digit_base,
                                                         int tiles, uint32_t* keys_out, int* vals_out) {
  __shared__ int s_off[kDigits];
  __shared__ int s_w[kWarps][kDigits];
  const int t = threadIdx.x;
  const unsigned lane = t & 31u;
  const int w = t >> 5;
  if (t < kDigits) s_off[t] = digit_base[t] + offsets[(long)t * tiles + blockIdx.x];
  const long nitems = pass_items(p);
  const long base = (long)blockIdx.x * kOrderTile;
  for (int r = 0; r < kRounds; ++r) {
    for (int j = t; j < kWarps * kDigits; j += kThreads) (&s_w[0][0])[j] = 0;
    __syncthreads();
    uint32_t key = 0;
    int val = 0;
    const bool take = load_item(p, base + (long)r * kThreads + t, nitems, &key, &val);
    const unsigned m = __ballot_sync(0xffffffffu, take);
    int d = 0, rank = 0;
    if (take) {
      d = (int)((key >> p.shift) & (kDigits - 1));
      const unsigned peers = __match_any_sync(m, d);
      rank = __popc(peers & ((1u << lane) - 1u));
      if (lane == (unsigned)(__ffs(peers) - 1)) s_w[w][d] = __popc(peers);
    }
    __syncthreads();
    int tot = 0;
    if (t < kDigits) {
      for (int q = 0; q < kWarps; ++q) {
        const int c = s_w[q][t];
        s_w[q][t] = tot;
        tot += c;
      }
    }
    __syncthreads();
    if (take) {
      const int pos = s_off[d] + s_w[w][d] + rank;
      if (keys_out) keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    if (t < kDigits) s_off[t] += tot;
  }
}

}  // namespace

std::string order_reserve(OrderScratch* o, long n) {
  if (n <= o->cap) return "";
  if (n > (long)INT_MAX) return "temperature order: more cells than an int index holds";
  order_free(o);
  const long tiles = (n + kOrderTile - 1) / kOrderTile;
  const size_t b = sizeof(int) * (size_t)n;
  if (cudaMalloc(&o->keys[0], b) != cudaSuccess || cudaMalloc(&o->keys[1], b) != cudaSuccess ||
      cudaMalloc(&o->vals[0], b) != cudaSuccess || cudaMalloc(&o->vals[1], b) != cudaSuccess ||
      cudaMalloc(&o->counts, sizeof(int) * (size_t)kDigits * tiles) != cudaSuccess ||
      cudaMalloc(&o->digit_base, sizeof(int) * kDigits) != cudaSuccess ||
      cudaMalloc(&o->total, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    order_free(o);
    return "temperature order: cudaMalloc of the sort scratch failed";
  }
  o->cap = n;
  return "";
}

void order_free(OrderScratch* o) {
  for (int i = 0; i < 2; ++i) {
    cudaFree(o->keys[i]);
    cudaFree(o->vals[i]);
    o->keys[i] = nullptr;
    o->vals[i] = nullptr;
  }
  cudaFree(o->counts);
  cudaFree(o->digit_base);
  cudaFree(o->total);
  o->counts = nullptr;
  o->digit_base = nullptr;
  o->total = nullptr;
  o->cap = 0;
}

cudaError_t order_cells_by_temperature(long n, const double* T, const int8_t* bc, const unsigned char* flag,
                                       OrderScratch* o, int* list, int* count, unsigned long long* counter,
                                       cudaStream_t s) {
  if (n < 0 || !o || n > o->cap || !list || !count || (n > 0 && !T)) return cudaErrorInvalidValue;
  if (n == 0) return cudaMemsetAsync(count, 0, sizeof(int), s);
  const int tiles = (int)((n + kOrderTile - 1) / kOrderTile);
  for (int pass = 0; pass < kOrderPasses; ++pass) {
    PassIn p{};
    p.n = n;
    p.shift = pass * kOrderDigitBits;
    if (pass == 0) {
      p.T = T;
      p.bc = bc;
      p.flag = flag;
    } else {
      p.count = o->total;
      p.keys = o->keys[(pass - 1) & 1];
      p.vals = o->vals[(pass - 1) & 1];
    }
    const bool last = pass == kOrderPasses - 1;
    k_rs_count<<<tiles, kThreads, 0, s>>>(p, o->counts, tiles);
    k_rs_scan_tiles<<<kDigits, kThreads, 0, s>>>(o->counts, tiles, o->digit_base);
    k_rs_scan_digits<<<1, kDigits, 0, s>>>(o->digit_base, o->total, last ? count : nullptr,
                                           pass == 0 ? counter : nullptr);
    k_rs_scatter<<<tiles, kThreads, 0, s>>>(p, o->counts, o->digit_base, tiles,
                                            last ? nullptr : o->keys[pass & 1], last ? list : o->vals[pass & 1]);
  }
  return cudaGetLastError();
}

}  // namespace nrg
