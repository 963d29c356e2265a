// The table_approximated mode of the chemistry step (host interface).
//
// The reference tabulates the per-step concentration change Y_prod2 of a
// 1-D flame against temperature (write_chemical_kinetics_table,
// chemical_kinetics_solver.f90:542-607), reads the table back at set-up
// (read_chemical_kinetics_table, :608-650) and, in this mode, replaces the
// stiff integration of every cell by a linear interpolation in T
// (interpolate_chemical_kinetics, :651-685; the mode's output branches
// :256-262, :314-315, :323-325, :334-335).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "chem_kernels.hpp"

namespace nrg {

// Rows of a table: T[i] and the N species values Y[k * rows + i].
struct ChemTable {
  long rows = 0;
  std::vector<double> T, Y;
};

// Reads a table file of n_species species (empty string on success).
std::string read_chem_table(const std::string& path, int n_species, ChemTable* out);

// Writes the rows first..last of one row of cells: T_at(i), Y2_at(k, i).
// The header names the species.  Empty string on success.
template <class FT, class FY>
std::string write_chem_table(const std::string& path, const std::vector<std::string>& species, int first, int last,
                             FT T_at, FY Y2_at);

// Fortran E14.7 output of one value (14 characters, no terminator needed).
void format_e14_7(double x, char out[15]);

// Whether the nodes are finite and non-decreasing, so that the last
// interval holding a temperature is found by bisection.
bool table_nodes_sorted(const std::vector<double>& T);

// Bucket index of sorted nodes: the range [T_0, T_{rows-1}] cut into nb equal
// buckets; a temperature T in bucket j = floor((T - T_0) * inv_w) (clamped to
// [0, nb - 1]) has between lo[j] and hi[j] nodes <= T, so the bisection for
// its interval starts from that range instead of the whole table.
struct TableIndex {
  std::vector<int> lo, hi;
  double t0 = 0.0, inv_w = 0.0;
};

// Builds the index of sorted nodes (false, and no index, for fewer than two
// distinct nodes or more than 2^31 - 1 rows).  The bucket bounds are widened
// by a millionth of a bucket, more than the rounding of the device's bucket
// arithmetic, so the true node count always lies in [lo[j], hi[j]].
bool build_table_index(const std::vector<double>& T, int n_buckets, TableIndex* out);

// Device copy of a table for the step kernel.
struct TableArgs {
  long rows;
  const double* T;   // rows
  const double* Y;   // N x rows, species-major
  int sorted;        // table_nodes_sorted
  const int2* idx;   // TableIndex as (lo, hi) pairs, or null
  int nb;            // buckets of idx
  double t0, inv_w;  // TableIndex::t0, inv_w
};

// One chemistry step in table mode over a.n cells (a.cell_list unused):
// skip rule, interpolation, outputs, optional T_after and status; adds the
// active and non-finite cells to counters[0] and counters[5].
cudaError_t launch_table_step(int n_species, const StepArgs& a, const TableArgs& t, unsigned long long* counters,
                              cudaStream_t s);

void upload_mechanism_table(const DevMech& m, cudaStream_t s);

// ------------------------------------------------------------ definitions
template <class FT, class FY>
std::string write_chem_table(const std::string& path, const std::vector<std::string>& species, int first, int last,
                             FT T_at, FY Y2_at) {
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return "cannot write " + path;
  std::string head = "T";
  for (const std::string& s : species) head += "  r(" + s + ")";
  bool ok = std::fprintf(f, "%s\n", head.c_str()) > 0;
  char fld[15];
  const int N = (int)species.size();
  for (int i = first; i <= last && ok; ++i) {
    format_e14_7(T_at(i), fld);
    ok = std::fwrite(fld, 1, 14, f) == 14;
    for (int k = 0; k < N && ok; ++k) {
      format_e14_7(Y2_at(k, i), fld);
      ok = std::fwrite(fld, 1, 14, f) == 14;
    }
    ok = ok && std::fputc('\n', f) != EOF;
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? std::string() : "short write to " + path;
}

}  // namespace nrg
