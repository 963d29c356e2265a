// The table_approximated mode of the chemistry step: the table file reader
// and writer (host) and the step kernel (device).  Compiled without FMA
// contraction, so the interpolation and the sources round exactly as the
// reference's expressions (chemical_kinetics_solver.f90:323-335, 651-685).
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>

#include "chem_bdf.cuh"
#include "table.hpp"

namespace nrg {

// ------------------------------------------------------------ file format
// Fortran Ew.d output, w = 14, d = 7: blank or '-', "0.", seven significant
// digits, then E+xx (the letter dropped for three-digit exponents);
// non-finite values as the words Fortran prints, right-justified.
void format_e14_7(double x, char out[15]) {
  std::memset(out, ' ', 14);
  out[14] = '\0';
  std::string body;
  if (std::isnan(x)) {
    body = "NaN";
  } else if (std::isinf(x)) {
    body = x < 0 ? "-Infinity" : "Infinity";
  } else {
    int exp10 = 0;
    char digits[8] = "0000000";
    if (x != 0.0) {
      char sci[32];
      std::snprintf(sci, sizeof sci, "%.6e", std::fabs(x));  // d.dddddde+XX, correctly rounded
      digits[0] = sci[0];
      std::memcpy(digits + 1, sci + 2, 6);
      exp10 = std::atoi(std::strchr(sci, 'e') + 1) + 1;  // 0.ddddddd x 10^exp10
    }
    const int mag = std::abs(exp10);
    char ex[8];
    if (mag <= 99)
      std::snprintf(ex, sizeof ex, "E%c%02d", exp10 < 0 ? '-' : '+', mag);
    else
      std::snprintf(ex, sizeof ex, "%c%03d", exp10 < 0 ? '-' : '+', mag % 1000);
    body = std::string(std::signbit(x) ? "-" : "") + "0." + digits + ex;
  }
  std::memcpy(out + 14 - body.size(), body.data(), body.size());
}

namespace {

// Fortran Ew.d input, d = 7, on one 14-character field: blanks ignored, an
// empty field is zero, without a decimal point the last seven digits are
// the fraction; exponent E/D[sign]digits or sign digits.
bool parse_e14_7(const std::string& field, double* v) {
  std::string s;
  for (char ch : field)
    if (ch != ' ' && ch != '\t') s.push_back(ch);
  if (s.empty()) {
    *v = 0.0;
    return true;
  }
  size_t p = 0;
  bool neg = false;
  if (s[p] == '+' || s[p] == '-') neg = s[p++] == '-';
  std::string digits;
  long point = -1;
  for (; p < s.size() && (std::isdigit((unsigned char)s[p]) || s[p] == '.'); ++p) {
    if (s[p] == '.') {
      if (point >= 0) return false;
      point = (long)digits.size();
    } else {
      digits.push_back(s[p]);
    }
  }
  if (digits.empty()) return false;
  long ex = 0;
  const bool letter = p < s.size() && std::strchr("EeDd", s[p]) != nullptr;
  if (letter) ++p;
  if (p < s.size()) {
    bool eneg = false;
    if (s[p] == '+' || s[p] == '-') eneg = s[p++] == '-';
    else if (!letter) return false;
    if (p >= s.size()) return false;
    for (; p < s.size(); ++p) {
      if (!std::isdigit((unsigned char)s[p])) return false;
      ex = ex * 10 + (s[p] - '0');
      if (ex > 100000) return false;
    }
    if (eneg) ex = -ex;
  } else if (letter) {
    return false;
  }
  const long frac = point >= 0 ? (long)digits.size() - point : 7;
  const std::string text = std::string(neg ? "-" : "") + "0." + digits + "e" +
                           std::to_string(ex - frac + (long)digits.size());
  *v = std::strtod(text.c_str(), nullptr);
  return true;
}

bool blank(const std::string& r) {
  return std::all_of(r.begin(), r.end(), [](char c) { return std::isspace((unsigned char)c) != 0; });
}

}  // namespace

// read_chemical_kinetics_table (:608-650): the records a list-directed read
// accepts (every non-blank one) less the header give the row count; after
// the header that many records are read with (N+1)E14.7, short records
// padded with blanks.  Malformed fields are an error here (the reference's
// iostat would leave them unset).
std::string read_chem_table(const std::string& path, int n_species, ChemTable* out) {
  std::ifstream in(path);
  if (!in) return "cannot open " + path;
  std::vector<std::string> recs;
  for (std::string r; std::getline(in, r);) {
    if (!r.empty() && r.back() == '\r') r.pop_back();
    recs.push_back(r);
  }
  const long nonblank = (long)std::count_if(recs.begin(), recs.end(), [](const std::string& r) { return !blank(r); });
  const long rows = nonblank - 1;
  if (rows < 1) return "no table rows in " + path;
  size_t at = 0;
  while (blank(recs[at])) ++at;  // the header record
  out->rows = rows;
  out->T.assign((size_t)rows, 0.0);
  out->Y.assign((size_t)rows * (size_t)n_species, 0.0);
  for (long i = 0; i < rows; ++i) {
    const size_t ri = at + 1 + (size_t)i;
    std::string rec = ri < recs.size() ? recs[ri] : std::string();
    rec.resize((size_t)(n_species + 1) * 14, ' ');
    for (int q = 0; q <= n_species; ++q) {
      double v = 0.0;
      if (!parse_e14_7(rec.substr((size_t)q * 14, 14), &v))
        return "malformed value in row " + std::to_string(i + 1) + ", field " + std::to_string(q + 1) + " of " + path;
      if (q == 0) out->T[(size_t)i] = v;
      else out->Y[(size_t)(q - 1) * (size_t)rows + (size_t)i] = v;
    }
  }
  return std::string();
}

bool table_nodes_sorted(const std::vector<double>& T) {
  for (size_t i = 0; i < T.size(); ++i) {
    if (!std::isfinite(T[i])) return false;
    if (i + 1 < T.size() && !(T[i] <= T[i + 1])) return false;
  }
  return true;
}

bool build_table_index(const std::vector<double>& T, int n_buckets, TableIndex* out) {
  const size_t M = T.size();
  if (M < 2 || M > 2147483647u || n_buckets < 1 || !(T.front() < T.back())) return false;
  const double t0 = T.front(), span = T.back() - T.front();
  const double inv_w = (double)n_buckets / span;
  if (!std::isfinite(inv_w) || !std::isfinite(span)) return false;
  // The device's bucket (T - t0) * inv_w carries at most a few roundings
  // relative to its value (at most n_buckets); these bounds are wider by a
  // millionth of a bucket plus 2^-40 of the largest node.
  const double w = span / (double)n_buckets;
  const double margin = w * 1e-6 + std::ldexp(std::max(std::fabs(T.front()), std::fabs(T.back())), -40);
  out->lo.assign((size_t)n_buckets, 0);
  out->hi.assign((size_t)n_buckets, 0);
  out->t0 = t0;
  out->inv_w = inv_w;
  const auto count_le = [&](double x) { return (int)(std::upper_bound(T.begin(), T.end(), x) - T.begin()); };
  for (int j = 0; j < n_buckets; ++j) {
    out->lo[(size_t)j] = j == 0 ? 0 : count_le(t0 + (double)j * w - margin);
    out->hi[(size_t)j] = j == n_buckets - 1 ? (int)M : count_le(t0 + (double)(j + 1) * w + margin);
  }
  return true;
}

// --------------------------------------------------------------- device
void upload_mechanism_table(const DevMech& m, cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_mech, &m, sizeof(DevMech), 0, cudaMemcpyHostToDevice, s);
}

namespace {

// interpolate_chemical_kinetics (:651-685): the index of the last interval
// [T_t(i), T_t(i+1)] that holds T, or -1.  Sorted nodes: with u the number
// of nodes <= T (bisection), the last such interval starts at node u - 1,
// or at M - 2 when T equals the last node; otherwise the reference's scan.
__device__ __forceinline__ long table_interval(const TableArgs& t, double T) {
  const long M = t.rows;
  if (t.sorted) {
    long lo = 0, hi = M;
    if (t.idx) {  // the bucket's range of node counts (TableIndex); NaN falls in bucket 0
      const double x = (T - t.t0) * t.inv_w;
      const int j = x >= 0.0 ? (x < (double)t.nb ? (int)x : t.nb - 1) : 0;
      const int2 b = __ldg(t.idx + j);
      lo = b.x;
      hi = b.y;
    }
    while (lo < hi) {
      const long mid = (lo + hi) >> 1;
      if (__ldg(t.T + mid) <= T) lo = mid + 1;
      else hi = mid;
    }
    if (lo >= 1 && lo <= M - 1) return lo - 1;
    if (lo == M && M >= 2 && T == __ldg(t.T + M - 1)) return M - 2;
    return -1;
  }
  long iv = -1;
  for (long i = 0; i + 1 < M; ++i)
    if (T >= __ldg(t.T + i) && T <= __ldg(t.T + i + 1)) iv = i;
  return iv;
}

// TA: the temperature after the step is written (the energy closure's
// Newton iteration); without it the kernel is a lean streaming pass.  Six
// 128-thread blocks per SM (at most 85 registers): the kernel waits on HBM
// latency, and more warps keep more loads in flight.
template <int N, bool TA>
__global__ void __launch_bounds__(128, 6) k_table_step(StepArgs a, TableArgs t, unsigned long long* counters) {
  unsigned active = 0, bad = 0;
  const long M = t.rows;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < a.n; c += (long)gridDim.x * blockDim.x) {
    const double T = a.T[c];
    if (!reference_cell_active(T, a.bc, c)) {
      write_skipped_cell(a, c, N, T);
      continue;
    }
    ++active;
    double y[N], q[N];  // conc_in (mass fractions in this mode) and conc_out
#pragma unroll
    for (int k = 0; k < N; ++k) {
      y[k] = a.Y[k * a.ld + c];
      q[k] = y[k];
    }
    const long iv = table_interval(t, T);
    if (iv >= 0) {
      const double t0 = __ldg(t.T + iv), t1 = __ldg(t.T + iv + 1);
#pragma unroll
      for (int k = 0; k < N; ++k)
        q[k] = __ldg(t.Y + k * M + iv + 1) * (T - t0) / (t1 - t0) + __ldg(t.Y + k * M + iv) * (T - t1) / (t0 - t1);
    }
    if (T < __ldg(t.T)) {
#pragma unroll
      for (int k = 0; k < N; ++k) q[k] = 0.0;
    }
    if (T > __ldg(t.T + M - 1)) {
#pragma unroll
      for (int k = 0; k < N; ++k) q[k] = __ldg(t.Y + k * M + M - 1);
    }
    double E = 0.0, dYm[N];
    bool finite = true;
    const double rho = TA ? a.rho[c] : 1.0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double W = c_mech.W[k];
      double yp;
      if (W != 0.0) {
        yp = q[k] * W / a.dt;
        const double y2 = q[k] - y[k];
        a.Y_prod2[k * a.ld + c] = y2;
        finite = finite && isfinite(y2);
      } else {
        yp = q[k] - y[k];
      }
      a.Y_prod[k * a.ld + c] = yp;
      finite = finite && isfinite(yp);
      E = E - c_mech.h_ref[k] * q[k] / a.dt;
      dYm[k] = yp * a.dt / rho;
    }
    a.E_f_prod[c] = E;
    finite = finite && isfinite(E);
    if (TA) a.T_after[c] = temperature_after<N>(T, y, dYm, E * a.dt / rho);
    if (a.status) a.status[c] = finite ? (uint8_t)kCellOk : (uint8_t)kCellNonfinite;
    bad += finite ? 0u : 1u;
  }
  // one atomic per warp for each counter
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    active += __shfl_down_sync(0xffffffffu, active, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0 && counters) {
    if (active) atomicAdd(counters + 0, (unsigned long long)active);
    if (bad) atomicAdd(counters + 5, (unsigned long long)bad);
  }
}

}  // namespace

cudaError_t launch_table_step(int n_species, const StepArgs& a, const TableArgs& t, unsigned long long* counters,
                              cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  if (t.rows < 1 || !t.T || !t.Y) return cudaErrorInvalidValue;
  if (a.T_after && !a.rho) return cudaErrorInvalidValue;
  // a block per 128 cells: the block scheduler keeps every SM's six slots
  // busy to the end (measured faster than eight or sixteen blocks per SM
  // striding over the cells, than one resident wave, and than 256-thread
  // blocks)
  const unsigned grid = (unsigned)std::min<long>((a.n + 127) / 128, 2147483647L);
  const bool ta = a.T_after != nullptr;
#define NRG_TABLE_CASE(NS)                                                           \
  case NS:                                                                           \
    if (ta) k_table_step<NS, true><<<grid, 128, 0, s>>>(a, t, counters);             \
    else k_table_step<NS, false><<<grid, 128, 0, s>>>(a, t, counters);               \
    break;
  switch (n_species) {
    NRG_TABLE_CASE(9)
    NRG_TABLE_CASE(10)
    NRG_TABLE_CASE(13)
    NRG_TABLE_CASE(17)
    default: return cudaErrorNotSupported;
  }
#undef NRG_TABLE_CASE
  return cudaGetLastError();
}

}  // namespace nrg
