// Device-side mechanism tables and per-cell chemistry for the NRG step.
//
// Layout: one thread integrates one cell.  Mechanism constants live in
// __constant__ memory: every lane of a warp walks the same reaction at the same
// time, so each table read is a broadcast.  Cell fields are SoA in HBM
// (species-major, cell-minor) so a warp's loads/stores of one species are
// coalesced 256-byte transactions.
#pragma once

#include <cstdint>

#include "chem_kernels.hpp"

namespace nrg {

constexpr int kMaxSpecies = 24;
constexpr int kMaxReactions = 96;
constexpr int kMaxOrd = 5;  // MXORD for Gear (MINT = 2)
constexpr int kMaxSpecUpd = 64;  // reactions touching one species

// Per-reaction update list entry: species (0-based) and whether the
// occurrence is a reactant (Zdot -= f, += r) or a product (Zdot -= r, += f).
// Entries are ordered species-major, reactants before products, which is the
// accumulation order of the reference RHS (chemical_kinetics_solver.f90:528-535).
struct DevMech {
  int N, R;
  int type[kMaxReactions];
  int nl[kMaxReactions], nr[kMaxReactions];
  int left[kMaxReactions][3], right[kMaxReactions][3];  // 0-based, -1 = M
  int nupd[kMaxReactions];
  int upd_k[kMaxReactions][6];
  int upd_prod[kMaxReactions][6];
  double A[kMaxReactions], beta[kMaxReactions], E[kMaxReactions];
  double A_low[kMaxReactions], beta_low[kMaxReactions], E_low[kMaxReactions];
  double troe[kMaxReactions][4];
  double dnu[kMaxReactions];
  double eff_t[kMaxSpecies][kMaxReactions];  // third-body efficiency, species-major
  double a[kMaxSpecies][2][7];  // NASA-7 times R
  double W[kMaxSpecies];
  double invW[kMaxSpecies];
  double h_ref[kMaxSpecies];   // h_k(T_ref)
  // integrator constants (host-computed so host and device agree bit-for-bit)
  double el[13 * 12], tq[3 * 12];
  double eps, ewt, hmax, uround;
  double sqrt_uround, br, bl, bp, facmin;
  // per-species update lists in reaction order, entry-major so that lanes
  // owning consecutive species read consecutive words: (r << 1) | 1 for a
  // product occurrence of species k in reaction r, (r << 1) for a reactant one
  int sp_n[kMaxSpecies];
  int sp_list[kMaxSpecUpd][kMaxSpecies];
  // element composition for conservation checks (H, O, N) in atoms/molecule
  double elem[3][kMaxSpecies];
  // Integrated species.  Species that appear in no reaction (third bodies
  // only, N2 in the H2/air mechanisms) have a zero right-hand side; the
  // thread-per-cell integrators of the analytic-Jacobian and mixed modes
  // integrate only the NI others.  In the copy of the tables those kernels
  // use, left/right/upd_k hold integrated indices; every per-species array
  // above stays indexed by mechanism species.
  int NI;
  int full_of[kMaxSpecies];   // integrated index -> mechanism species
  int n_inert;
  int inert_of[kMaxSpecies];  // the inert species (mechanism index)
};

// Per-cell status byte written by the integrator.
enum CellStatus : uint8_t {
  kCellSkipped = 0,   // T < 305 K or bc /= 0: zero sources (reference rule)
  kCellOk = 1,
  kCellMxstep = 2,    // MXSTEP reached; state at the current T returned
  kCellFatal = 3,     // step size vanished / too many retries / singular
  kCellNonfinite = 4, // non-finite input or output
  kCellSurrogate = 5  // accepted surrogate prediction (gated path)
};

// Skip rule of the reference (chemical_kinetics_solver.f90:228-231): a cell
// colder than 305 K, or one carrying a boundary marker, is not integrated.
// A NaN temperature counts as cold.
constexpr double kSkipBelowK = 305.0;

__device__ __forceinline__ bool reference_cell_active(double T, const int8_t* bc, long c) {
  return (T >= kSkipBelowK) && (bc == nullptr || bc[c] == 0);
}

// Outputs of a skipped cell (:341-346): zero species and energy sources,
// Y_prod2 left as the caller had it, the temperature after the step equal to
// the one before.  Every path of the step (integrators, surrogate, the
// no-allocation step) writes skipped cells through this one function.
__device__ __forceinline__ void write_skipped_cell(const StepArgs& a, long c, int n_species, double T) {
  for (int k = 0; k < n_species; ++k) a.Y_prod[k * a.ld + c] = 0.0;
  a.E_f_prod[c] = 0.0;
  if (a.T_after) a.T_after[c] = T;
  if (a.status) a.status[c] = kCellSkipped;
}

}  // namespace nrg
