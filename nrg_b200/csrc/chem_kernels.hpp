// Host-visible declarations of the chemistry kernels' launch interface.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace nrg {

struct DevMech;

// Arguments of one chemistry step over n cells.  Species arrays are
// species-major: element (k, c) lives at [k * ld + c].
struct StepArgs {
  long n;
  long ld;
  double dt;
  const double* T;
  const double* rho;
  const double* Y;
  const int8_t* bc;   // may be null: every cell interior
  double* Y_prod;
  double* Y_prod2;
  double* E_f_prod;
  double* T_after;    // may be null
  uint8_t* status;    // may be null
  int mxstep;
  const DevMech* mech;     // device copy of the mechanism tables (global memory)
  const double* dt_cells;  // per-cell step (training pairs); null: dt for every cell
  const int* cell_list;    // integrate only these cells (gated fallback); null: 0..n-1
  int n_list;              // number of entries in cell_list (grid bound when n_list_dev is set)
  const int* n_list_dev;   // device-side entry count of cell_list (may be null)
  double eps = 0.0;        // relative tolerance of the integrator; 0: the mechanism's (the reference's 1e-9)
  int lu_rolled = 0;       // thread-per-cell kernels: the LU factorisation as a loop (same bits)
};

// Chemistry sources applied to the state, then the state equation.
struct ApplyStateArgs {
  long n, ld;
  int dims;                 // velocity components in v
  double dt;
  const double* rho;
  const double* Y_prod;     // may be null (state equation only)
  const double* E_f_prod;   // may be null
  const int8_t* bc;         // may be null
  double* Y;                // in/out, species-major
  double* E_f;              // in/out (total energy per mass)
  const double* v;          // dims x ld (may be null when dims == 0)
  double* T;                // in: Newton start; out
  double* p;
  double* gamma;
  double* cp_mass;          // optional outputs from here on
  double* h_s;
  double* h_full;
  double* v_s;
  double* mix_mol_mass;
  uint8_t* status;          // 0 skipped (bc), 1 ok, 2 negative gamma, p or rho
};
cudaError_t launch_apply_state(int n_species, const ApplyStateArgs& a, cudaStream_t s);

enum KernelKind { kKernelThreadGrid = 0, kKernelThreadQueue = 1, kKernelWarpQueue = 2 };

struct LaunchCfg {
  int kernel = kKernelThreadGrid;  // KernelKind
  int block = 32;                  // threads per block
  int grid = 0;                   // persistent grid (0: fill the GPU)
  int chunk = 1;                  // cells reserved per queue fetch (per lane or per warp)
  int lu_rolled = 0;              // thread-per-cell kernels: LU as a loop instead of unrolled
};

// full: tables over all species; reduced: the same with reaction lists
// numbered over the reacting species (thread-per-cell fast / mixed variants)
void upload_mechanism(const DevMech& full, const DevMech& reduced, cudaStream_t s);

// jac: 0 finite-difference (reference DDPST), 1 analytic.  mixed: float LU.
// queue must point at a zeroed device int for the work-queue kernels.
// Mechanism sizes (species, reactions) with compiled kernels: KEROMNES
// (9, 24; every launch shape), ZHANG (9, 28), TEREZA (10, 24), KONNOV
// (13, 71) (thread-per-cell grid, reference and analytic-Jacobian modes).
bool supported_mechanism(int n_species, int n_reactions);
// The number (1..) of the generated mechanism-specialised code whose reaction
// lists equal the reduced ones, 0 when none does.
int match_specialised(const DevMech& reduced);
cudaError_t launch_chem(int n_species, int n_int, int spec, int n_reactions, int jac, bool mixed, const StepArgs& a,
                        const LaunchCfg& cfg, int* queue, unsigned long long* counters,
                        cudaStream_t s);

// Shared memory one cell of the given mechanism size occupies.
int smem_bytes_per_cell(int n_species, int n_reactions, bool mixed);

cudaError_t launch_fp64_peak(double* out, int blocks, int threads, int iters, cudaStream_t s);

}  // namespace nrg
