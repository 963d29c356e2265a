// Per-cell stiff integrator for the NRG chemistry step (device code).
//
// The integrator is the variable-order BDF (Gear) method with Nordsieck
// history, chord Newton, LU with partial pivoting and the step/order control
// of SLATEC DDRIV3 as the reference calls it (chemical_kinetics_solver.f90:
// 270-313: MINT=2, MITER=2, IMPL=0, IERROR=3, NTASK=1, EPS=1e-9, EWT=1e-4,
// HMAX=1.0E-7 (single-precision literal), MXORD=5, MXSTEP=10000).  Routine
// correspondences: ddriv3.f90:930-978,1292-1497 (driver), ddstp.f90:72-459
// (step), ddntl.f90:41-182 (first step), ddpst.f90:52-142 (Jacobian + LU),
// ddcor.f90:61-107 (corrector), ddscl/ddpsc/ddntp (rescale, predictor,
// interpolation), dgefa/dgesl (LINPACK LU), dnrm2 (scaled norm).
//
// The driver loop is split so that a thread can advance one accepted step at
// a time (cell_begin / cell_advance / cell_finish).  The persistent kernel uses
// this to refill a lane with a new cell as soon as its current cell reaches
// t = dt, which keeps lanes busy when substep counts differ by 100x.
//
// Jacobian modes: kJacFD reproduces the reference's finite-difference
// Jacobian with its adaptive increments (DDPST, MITER=2); kJacAnalytic forms
// dZdot/dZ from the mass-action rates directly, which removes N right-hand-side
// evaluations per Jacobian.  LU precision: double, or float factors with
// float64 residuals and iterative refinement (mixed mode).
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "chem_device.cuh"
#include "chem_kernels.hpp"
#include "gen_mechanisms.cuh"

namespace nrg {

// Each translation unit that includes this header holds its own copy of the
// tables and uploads it (upload_mechanism / surrogate set-up).
static __constant__ DevMech c_mech;

enum JacMode { kJacFD = 0, kJacAnalytic = 1 };

// ------------------------------------------------------------ storage
// Per-cell arrays live in shared memory in an [element][thread] layout: for
// element e, the BS threads of a block touch BS consecutive words, so every
// warp access is bank-conflict free.  Vectors that are only ever indexed by
// unrolled loops (y, YWT, SAVE1, SAVE2, FAC) stay in registers; the row
// permutation of the LU factors is packed into one or two 64-bit registers
// (RowPerm).
template <int N, int R, typename LUT, int BS>
struct SmemStore {
  static constexpr int kYH = 0;
  static constexpr int kKF = (kMaxOrd + 1) * N;
  static constexpr int kKR = kKF + R;
  static constexpr int kZ = kKR + R;
  static constexpr int kZD = kZ + N;
  static constexpr int kDoubles = kZD + N;
  static constexpr int kBytesPerThread = kDoubles * 8 + N * N * (int)sizeof(LUT);
  using lut_t = LUT;
  static constexpr int kBS = BS;
  static constexpr int kR = R;
  double* d;
  LUT* f;
  __device__ __forceinline__ void bind(char* smem, int tid) {
    d = reinterpret_cast<double*>(smem) + tid;
    f = reinterpret_cast<LUT*>(smem + (size_t)kDoubles * 8 * BS) + tid;
  }
  __device__ __forceinline__ double& yh(int j, int i) { return d[(kYH + j * N + i) * BS]; }
  __device__ __forceinline__ double& kf(int r) { return d[(kKF + r) * BS]; }
  __device__ __forceinline__ double& kr(int r) { return d[(kKR + r) * BS]; }
  __device__ __forceinline__ double& z(int k) { return d[(kZ + k) * BS]; }
  __device__ __forceinline__ double& zd(int k) { return d[(kZD + k) * BS]; }
  __device__ __forceinline__ LUT& a(int j, int i) { return f[(j * N + i) * BS]; }  // A(i+1, j+1)
};

template <int N, int R, typename LUT, int BS, int NF = N, int SPEC = 0>
struct CellState;

// Row permutation of the LU factors, packed in registers: row indices 0..N-1
// in 4-bit fields up to 16 rows, else in 5-bit fields (12 per 64-bit word).
template <int N>
struct RowPerm {
  static constexpr int kBits = N <= 16 ? 4 : 5;
  static constexpr int kPer = 64 / kBits;
  static constexpr int kWords = (N + kPer - 1) / kPer;
  static constexpr unsigned long long kMask = (1ull << kBits) - 1ull;
  unsigned long long w[kWords];
  __device__ __forceinline__ void identity() {
#pragma unroll
    for (int q = 0; q < kWords; ++q) w[q] = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) w[k / kPer] |= (unsigned long long)k << ((k % kPer) * kBits);
  }
  __device__ __forceinline__ int get(int k) const {
    const int q = k / kPer, r = (k - q * kPer) * kBits;
    unsigned long long x = w[0];
#pragma unroll
    for (int i = 1; i < kWords; ++i)
      if (q == i) x = w[i];
    return (int)((x >> r) & kMask);
  }
  __device__ __forceinline__ void set(int k, int v) {
    const int q = k / kPer, r = (k - q * kPer) * kBits;
#pragma unroll
    for (int i = 0; i < kWords; ++i)
      if (q == i) w[i] = (w[i] & ~(kMask << r)) | ((unsigned long long)v << r);
  }
};

// Out-of-line hot routines of the thread-per-cell integrator.  They touch only
// the cell's shared-memory arrays (passed as the two base pointers), so the
// register-resident vectors are never forced to local memory by the call.
template <int N, int R, typename LUT, int BS, int SPEC>
__device__ __noinline__ void nl_rhs(double* d, LUT* f);
template <int N, int R, typename LUT, int BS, int SPEC>
__device__ __noinline__ void nl_analytic_matrix(double* d, LUT* f, double factor);
template <int N, int R, typename LUT, int BS, bool RECIP>
__device__ __noinline__ RowPerm<N> nl_dgefa(double* d, LUT* f, int* info, int rolled);
template <int N, int R, typename LUT, int BS, bool FAST>
__device__ __noinline__ void nl_rate_constants(double* d, LUT* f, double T);

// N integrated species (vectors, Nordsieck rows, LU), NF mechanism species
// (inputs, outputs, norms' sqrt(NF)); NF - N inert species are not integrated.
// SPEC: 0 for the table-driven right-hand side and iteration matrix, else
// the number of the generated mechanism-specialised code (gen_mechanisms.cuh).
template <int N, int R, typename LUT, int BS, int NF, int SPEC>
struct CellState : SmemStore<N, R, LUT, BS> {
  static constexpr int kNF = NF;
  static constexpr int kSpec = SPEC;
  double y[N], ywt[N], s1[N], s2[N], fac[N];
  RowPerm<N> piv;  // row i of the factors is row piv.get(i) of the matrix
  double h, t, tout, rc, rmax, trend, eps;
  int nq, nwait, jtask, nstep, nfe, nje, nsolve, jstepl, nstepl, convrg, ier;
  int lu_rolled;  // LU factorisation as a loop (StepArgs::lu_rolled)
};

// Register-array element with a runtime index (select chain, no local memory).
template <int N>
__device__ __forceinline__ double sel(const double (&v)[N], int j) {
  double r = v[0];
#pragma unroll
  for (int i = 1; i < N; ++i)
    if (i == j) r = v[i];
  return r;
}
template <int N>
__device__ __forceinline__ void put(double (&v)[N], int j, double x) {
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (i == j) v[i] = x;
}

// Correctly rounded double division kept out of line: the integrator divides
// at dozens of sites inside unrolled species loops, and one shared copy keeps
// the kernel small enough for the instruction cache.
static __device__ __noinline__ double ddiv(double a, double b) { return a / b; }

#define NRG_FMAX(a, b) ((a) >= (b) ? (a) : (b))
#define NRG_FMIN(a, b) ((a) <= (b) ? (a) : (b))

// -------------------------------------------------------------- thermo
__device__ __forceinline__ int nasa_set(double t) { return t >= 1000.0 ? 1 : 0; }

// Single out-of-line copies of the thermo polynomials and of the libm calls
// used once per cell (rate constants, energy closure): the kernel image stays
// small enough for the instruction cache.
static __device__ __noinline__ double nexp(double x) { return exp(x); }
static __device__ __noinline__ double nlog(double x) { return log(x); }
static __device__ __noinline__ double nlog10(double x) { return log10(x); }

static __device__ __noinline__ double d_enthalpy(double T, int k) {
  double t = NRG_FMIN(T, 6000.0);
  const double* a = c_mech.a[k][nasa_set(t)];
  double h = a[4] / 5.0;
  h = h * t + a[3] / 4.0;
  h = h * t + a[2] / 3.0;
  h = h * t + a[1] / 2.0;
  h = h * t + a[0] / 1.0;
  h = h + a[5] / t;
  return h * t;
}

static __device__ __noinline__ double d_entropy(double T, int k, double logt) {
  double t = NRG_FMIN(T, 6000.0);
  const double* a = c_mech.a[k][nasa_set(t)];
  double s = a[4] / 4.0;
  s = s * t + a[3] / 3.0;
  s = s * t + a[2] / 2.0;
  s = s * t + a[1] / 1.0;
  return s * t + a[6] + a[0] * logt;
}

static __device__ __noinline__ double d_cp(double T, int k) {
  double t = NRG_FMIN(T, 6000.0);
  const double* a = c_mech.a[k][nasa_set(t)];
  double cp = a[4];
  cp = cp * t + a[3];
  cp = cp * t + a[2];
  cp = cp * t + a[1];
  cp = cp * t + a[0];
  return cp;
}

// One out-of-line copy of pow for the step-size control (called from many
// sites; inlining each copy bloats the kernel past the instruction cache).
static __device__ __noinline__ double npow(double x, double y) { return pow(x, y); }

// x ** dnu for the integer stoichiometric change of a reaction
__device__ __forceinline__ double int_pow(double x, double dnu) {
  if (dnu == 0.0) return 1.0;
  if (dnu == 1.0) return x;
  if (dnu == -1.0) return ddiv(1.0, x);
  if (dnu == 2.0) return x * x;
  if (dnu == -2.0) return ddiv(1.0, x * x);
  return npow(x, dnu);
}

// calculate_rate_constants (chemical_kinetics_solver.f90:360-493).  The
// frozen third-body concentration [M] of reactions written with M is folded
// into the rate constant here (k_f [M] and k_r [M]), so the right-hand side
// multiplies concentrations only.  Expects the third-body sums in c.kr(r).
template <int N, int R, class CS>
__device__ void rate_constants(CS& c, double Tin) {
  const double RG = 8.31446261815324, PATM = 101325.0;
  const double T = NRG_FMIN(Tin, 10000.0);
  const double logt = nlog(NRG_FMIN(T, 6000.0));
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    c.z(k) = d_entropy(T, c_mech.full_of[k], logt);
    c.zd(k) = d_enthalpy(T, c_mech.full_of[k]);
  }
  const double conc_ref = ddiv(ddiv(PATM, RG), T);
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    const double mc = c.kr(r);
    double d_s = 0.0, d_h = 0.0;
    bool m_left = false, m_right = false;
    for (int i = 0; i < c_mech.nr[r]; ++i) {
      int sp = c_mech.right[r][i];
      if (sp < 0) { m_right = true; continue; }
      d_s = d_s + c.z(sp);
      d_h = d_h + c.zd(sp);
    }
    for (int i = 0; i < c_mech.nl[r]; ++i) {
      int sp = c_mech.left[r][i];
      if (sp < 0) { m_left = true; continue; }
      d_s = d_s - c.z(sp);
      d_h = d_h - c.zd(sp);
    }
    const int type = c_mech.type[r];
    const double kinf = c_mech.A[r] * npow(T, c_mech.beta[r]) * nexp(-ddiv(ddiv(c_mech.E[r], RG), T));
    double k = kinf;
    if (type == 2 || type == 3 || type == 7) {
      const double k0 = c_mech.A_low[r] * npow(T, c_mech.beta_low[r]) * nexp(-ddiv(ddiv(c_mech.E_low[r], RG), T));
      const double rp = ddiv(k0 * mc, kinf);
      k = kinf * ddiv(rp, 1.0 + rp);
      if (type == 3) {
        const double al = c_mech.troe[r][0];
        const double Fc = (1.0 - al) * nexp(-ddiv(T, c_mech.troe[r][1])) + al * nexp(-ddiv(T, c_mech.troe[r][2])) +
                          nexp(-ddiv(c_mech.troe[r][3], T));
        const double lf = nlog10(Fc);
        const double cc = -0.4 - 0.67 * lf;
        const double nn = 0.75 - 1.27 * lf;
        double blend;
        if (rp != 0.0) {
          const double lr = nlog10(rp);
          const double x = ddiv(lr + cc, nn - 0.14 * (lr + cc));
          blend = npow(Fc, ddiv(1.0, 1.0 + x * x));
        } else {
          blend = npow(Fc, ddiv(-1.0, 0.14));
        }
        k = k * blend;
      }
    }
    double kr = 0.0;
    if (type < 5) {
      const double Kp = nexp(ddiv(d_s, RG) - ddiv(ddiv(d_h, RG), T));
      kr = ddiv(k, Kp * int_pow(conc_ref, c_mech.dnu[r]));
    }
    c.kf(r) = m_left ? k * mc : k;
    c.kr(r) = m_right ? kr * mc : kr;
  }
}

// calculate_rate_constants for the analytic-Jacobian and mixed modes, whose
// results agree with the reference's to its tolerance rather than bit for
// bit: each Arrhenius rate as one exponential, A exp(beta ln T - E / (R T)),
// the reverse rate as the forward one times one exponential of
// -dS/R + dH/(R T) - dnu ln(p_atm / (R T)), the Troe blending power as an
// exponential, and the reactions four at a time with the libm calls inline,
// so that their long-latency chains overlap.  The same temperature caps as
// the reference (1e4 K for the rates, 6000 K for the thermochemistry).
template <int N, int R, class CS>
__device__ void rate_constants_fast(CS& c, double Tin) {
  const double RG = 8.31446261815324, PATM = 101325.0;
  const double T = NRG_FMIN(Tin, 10000.0);
  const double tt = NRG_FMIN(T, 6000.0);
  const double logt = log(tt), lnT = log(T), rT = 1.0 / T, rRT = rT / RG;
  const int set = nasa_set(tt);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double* a = c_mech.a[c_mech.full_of[k]][set];
    // entropy and enthalpy as d_entropy / d_enthalpy
    const double sp = fma(fma(fma(a[4] * 0.25, tt, a[3] * (1.0 / 3.0)), tt, a[2] * 0.5), tt, a[1]);
    c.z(k) = fma(sp, tt, fma(a[0], logt, a[6]));
    const double hp = fma(fma(fma(fma(a[4] * 0.2, tt, a[3] * 0.25), tt, a[2] * (1.0 / 3.0)), tt, a[1] * 0.5), tt, a[0]);
    c.zd(k) = fma(hp, tt, a[5]);
  }
  const double ln_conc_ref = log(PATM / RG) - lnT;
#pragma unroll 4
  for (int r = 0; r < R; ++r) {
    const double mc = c.kr(r);
    double d_s = 0.0, d_h = 0.0;
    bool m_left = false, m_right = false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (i < c_mech.nr[r]) {
        const int sp = c_mech.right[r][i];
        if (sp < 0) m_right = true;
        else {
          d_s += c.z(sp);
          d_h += c.zd(sp);
        }
      }
      if (i < c_mech.nl[r]) {
        const int sp = c_mech.left[r][i];
        if (sp < 0) m_left = true;
        else {
          d_s -= c.z(sp);
          d_h -= c.zd(sp);
        }
      }
    }
    const int type = c_mech.type[r];
    const double kinf = c_mech.A[r] * exp(c_mech.beta[r] * lnT - c_mech.E[r] * rRT);
    double k = kinf;
    if (type == 2 || type == 3 || type == 7) {
      const double k0 = c_mech.A_low[r] * exp(c_mech.beta_low[r] * lnT - c_mech.E_low[r] * rRT);
      const double rp = k0 * mc / kinf;
      k = kinf * (rp / (1.0 + rp));
      if (type == 3) {
        const double al = c_mech.troe[r][0];
        const double Fc = (1.0 - al) * exp(-T / c_mech.troe[r][1]) + al * exp(-T / c_mech.troe[r][2]) +
                          exp(-c_mech.troe[r][3] * rT);
        const double lnFc = log(Fc), lf = lnFc * 0.43429448190325182765;
        const double cc = -0.4 - 0.67 * lf, nn = 0.75 - 1.27 * lf;
        double expo;
        if (rp != 0.0) {
          const double lr = log10(rp);
          const double x = (lr + cc) / (nn - 0.14 * (lr + cc));
          expo = 1.0 / (1.0 + x * x);
        } else {
          expo = -1.0 / 0.14;
        }
        k = k * exp(expo * lnFc);
      }
    }
    double kr = 0.0;
    if (type < 5) kr = k * exp(d_h * rRT - d_s / RG - c_mech.dnu[r] * ln_conc_ref);
    c.kf(r) = m_left ? k * mc : k;
    c.kr(r) = m_right ? kr * mc : kr;
  }
}

// fun (chemical_kinetics_solver.f90:495-540): zd = dC/dt at z (both in the
// cell's shared scratch), accumulated per reaction as the net rate f - b.
template <int N, int R, class CS>
__device__ __forceinline__ void rhs(CS& c) {
#pragma unroll
  for (int k = 0; k < N; ++k) c.zd(k) = 0.0;
// Fixed-trip inner loops (3 reactant and 3 product slots, unused and M
// slots hold -1 and multiply by 1.0, which leaves every product unchanged; 6
// update slots under a predicate): no data-dependent branches per reaction.
// Explicitly rounded operations (never fused into FMAs) make the result
// independent of how the compiler schedules this loop, so the generated
// straight-line version (gen_keromnes.cuh) gives the same bits.
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    double f = c.kf(r);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int sp = c_mech.left[r][i];
      f = __dmul_rn(f, sp >= 0 ? c.z(sp) : 1.0);
    }
    double b = c.kr(r);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int sp = c_mech.right[r][i];
      b = __dmul_rn(b, sp >= 0 ? c.z(sp) : 1.0);
    }
    const double q = __dsub_rn(f, b);
    const int nu = c_mech.nupd[r];
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      if (u < nu) {
        const int k = c_mech.upd_k[r][u];
        const double v = c.zd(k);
        c.zd(k) = c_mech.upd_prod[r][u] ? __dadd_rn(v, q) : __dsub_rn(v, q);
      }
    }
  }
}

// Right-hand side at the register vector v, result into the register vector out.
template <int N, int R, class CS>
__device__ __forceinline__ void rhs_at(CS& c, const double (&v)[N], double (&out)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) c.z(k) = v[k];
  nl_rhs<N, R, typename CS::lut_t, CS::kBS, CS::kSpec>(c.d, c.f);
#pragma unroll
  for (int k = 0; k < N; ++k) out[k] = c.zd(k);
}

// Iteration matrix I + factor * J with J = dZdot/dZ of the mass-action rates
// at z, written straight into the LU storage.
template <int N, int R, class CS>
__device__ void analytic_iteration_matrix(CS& c, double factor) {
  using LUT_T = typename CS::lut_t;
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int i = 0; i < N; ++i) c.a(j, i) = 0;
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    const int nu = c_mech.nupd[r];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const double k = side ? c.kr(r) : c.kf(r);
      const double sgn = side ? -factor : factor;  // d(f - b)
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const int sp = side ? c_mech.right[r][p] : c_mech.left[r][p];
        if (sp < 0) continue;
        double d = k;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q == p) continue;
          const int sq = side ? c_mech.right[r][q] : c_mech.left[r][q];
          d = __dmul_rn(d, sq >= 0 ? c.z(sq) : 1.0);
        }
        d = __dmul_rn(d, sgn);
#pragma unroll
        for (int u = 0; u < 6; ++u) {
          if (u < nu) {
            const int k2 = c_mech.upd_k[r][u];
            const double v = (double)c.a(sp, k2);
            c.a(sp, k2) = (LUT_T)(c_mech.upd_prod[r][u] ? __dadd_rn(v, d) : __dsub_rn(v, d));
          }
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) c.a(i, i) += 1;
}

// dnrm2.f90:75-162, Lawson-Hanson scaled two-norm, restated as a per-element
// state machine over an unrolled loop (phases 1-4 of the reference's
// ASSIGN/GO TO form: zero, small-scaled, mid-range, large-scaled).
template <int N>
__device__ __noinline__ double dnrm2_nl(const double* dx) {
  const double cutlo = 8.232e-11, cuthi = 1.304e19;
  const double hitest = cuthi / (double)N;
  enum { S30, S50, S70, S85, S110 };
  int st = S30;
  double sum = 0.0, xmax = 0.0;
#pragma unroll 1
  for (int i = 0; i < N; ++i) {
    const double x = dx[i], ax = fabs(x);
    if (st == S30) {
      if (ax > cutlo) st = S85;
      else { st = S50; xmax = 0.0; }
    }
    if (st == S50) {
      if (x == 0.0) continue;
      if (ax > cutlo) {
        st = S85;
      } else {
        st = S70;
        xmax = ax;
        const double q = ddiv(x, xmax);
        sum = sum + q * q;
        continue;
      }
    }
    if (st == S70) {
      if (ax > cutlo) {
        sum = (sum * xmax) * xmax;
        st = S85;
      }
    }
    if (st == S70 || st == S110) {
      if (ax <= xmax) {
        const double q = ddiv(x, xmax);
        sum = sum + q * q;
      } else {
        const double q = ddiv(xmax, x);
        sum = 1.0 + sum * (q * q);
        xmax = ax;
      }
      continue;
    }
    // S85: mid-range, unscaled
    if (ax >= hitest) {
      sum = ddiv(ddiv(sum, x), x);
      xmax = ax;
      const double q = ddiv(x, xmax);
      sum = sum + q * q;
      st = S110;
    } else {
      sum = sum + x * x;
    }
  }
  return st == S85 ? sqrt(sum) : xmax * sqrt(sum);
}

template <int N>
__device__ __forceinline__ double dnrm2(const double (&dx)[N]) {
  double t[N];
#pragma unroll
  for (int i = 0; i < N; ++i) t[i] = dx[i];
  return dnrm2_nl<N>(t);
}

// Power of an error ratio in the step-size and order choices (ddstp.f90).
// Reference mode: the reference's pow.  Analytic-Jacobian and mixed modes:
// 2^(p log2 x) in single precision, relative error about 1e-6, which only
// scales the next step size; outside [1e-30, 1e30] the double pow is used.
template <int JAC>
__device__ __forceinline__ double ratio_pow(double x, double p) {
  if constexpr (JAC != kJacFD) {
    if (x > 1e-30 && x < 1e30) return (double)exp2f((float)p * __log2f((float)x));
  }
  return npow(x, p);
}

// Division in the step-size and order control of DDSTP: the correctly
// rounded division (out of line) in every mode.  An inline quotient from the
// hardware reciprocal approximation (one Newton step and a correction) in
// the analytic-Jacobian and mixed modes measured no faster on the flame
// field and 7 % slower on the ignition and wide-range fields (larger code).
template <int JAC>
__device__ __forceinline__ double sdiv(double a, double b) {
  return ddiv(a, b);
}

// sqrt by Newton's iteration at compile time (constant scale factors).
__host__ __device__ constexpr double ct_sqrt(double x, double g = 1.0, int it = 0) {
  return it == 64 ? g : ct_sqrt(x, 0.5 * (g + x / g), it + 1);
}

// Weighted two-norm sqrt(sum_i (x_i / max(|y_i|, YWT_i))^2) of the corrector,
// error and order tests (ddcor.f90, ddstp.f90).  Reference mode: the
// reference's divisions and dnrm2.  Analytic-Jacobian and mixed modes: one
// pass over the species with the weights' reciprocals from the hardware
// approximation (rcp.approx.ftz.f64) refined by one Newton step
// r (1 + (1 - w r)), which squares its relative error to about 2^-44, and a
// plain sum of squares: it differs by rounding only, and these norms only
// steer step sizes, orders and the error test.  Weights are at least the
// error-weight floor; if one is not finite or the sum leaves the safe range,
// the reference form (out of line, so the fast path stays compact) is used.
template <int N>
__device__ __noinline__ double weighted_norm_ref(const double* x, const double* y, const double* ywt) {
  double q[N];
#pragma unroll
  for (int i = 0; i < N; ++i) q[i] = ddiv(x[i], NRG_FMAX(fabs(y[i]), ywt[i]));
  return dnrm2_nl<N>(q);
}

template <int N, int JAC, class CS>
__device__ __forceinline__ double weighted_norm(const CS& c, const double (&x)[N]) {
  if constexpr (JAC == kJacFD) {
    double q[N];
#pragma unroll
    for (int i = 0; i < N; ++i) q[i] = ddiv(x[i], NRG_FMAX(fabs(c.y[i]), c.ywt[i]));
    return dnrm2<N>(q);
  } else {
    double sum = 0.0;
    bool ok = true;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double w = NRG_FMAX(fabs(c.y[i]), c.ywt[i]);
      ok = ok && (w < 1e300);
      double r;
      asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(w));
      const double q = x[i] * fma(r, fma(-w, r, 1.0), r);
      sum = fma(q, q, sum);
    }
    if (ok && sum < 1e300) return sqrt(sum);
    double xs[N], ys[N], ws[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      xs[i] = x[i];
      ys[i] = c.y[i];
      ws[i] = c.ywt[i];
    }
    return weighted_norm_ref<N>(xs, ys, ws);
  }
}

// dgefa.f90:60-117 on the shared-memory matrix (column-major a(j, i) = A(i, j)):
// the same pivot choices, eliminations and roundings as LINPACK, with the
// row interchanges also applied to the multipliers of earlier columns (as
// LAPACK's getrf stores them), so that dgesl applies the whole permutation
// once instead of one interchange per column.  RECIP: each pivot is replaced
// by its reciprocal (the -1/pivot the elimination forms anyway, negated), so
// that dgesl<RECIP> multiplies where the reference divides; used by the
// analytic-Jacobian and mixed modes, whose results agree with the reference's
// to its tolerance, not bit for bit.
// x + t * y of the elimination.  The analytic-Jacobian modes (RECIP) with
// double factors fuse it into one FMA; the reference mode keeps the
// reference's separately rounded multiply and add.
template <typename LUT, bool RECIP>
__device__ __forceinline__ LUT lu_axpy(LUT x, LUT t, LUT y) {
  if constexpr (RECIP && std::is_same<LUT, double>::value) return fma(t, y, x);
  else return x + t * y;
}

// One elimination step k of dgefa (pivot search, interchange, scaling,
// column updates).
template <int N, bool RECIP, class CS, class LUT>
__device__ __forceinline__ void dgefa_step(CS& c, int k, RowPerm<N>& perm, int& info) {
  int l = k;
  LUT dmax = fabs(c.a(k, k));
  for (int i = k + 1; i < N; ++i) {
    const LUT xm = fabs(c.a(k, i));
    if (xm > dmax) { l = i; dmax = xm; }
  }
  if (c.a(k, l) == (LUT)0) {
    info = k + 1;
    return;
  }
  if (l != k) {
    const LUT t = c.a(k, l);
    c.a(k, l) = c.a(k, k);
    c.a(k, k) = t;
    for (int j = 0; j < k; ++j) {
      const LUT m = c.a(j, l);
      c.a(j, l) = c.a(j, k);
      c.a(j, k) = m;
    }
    const int pk = perm.get(k);
    perm.set(k, perm.get(l));
    perm.set(l, pk);
  }
  const LUT t = (LUT)-1 / c.a(k, k);
  if (RECIP) c.a(k, k) = -t;
  for (int i = k + 1; i < N; ++i) c.a(k, i) = t * c.a(k, i);
  for (int j = k + 1; j < N; ++j) {
    const LUT tj = c.a(j, l);
    if (l != k) {
      c.a(j, l) = c.a(j, k);
      c.a(j, k) = tj;
    }
    if (tj != (LUT)0)
      for (int i = k + 1; i < N; ++i) c.a(j, i) = lu_axpy<LUT, RECIP>(c.a(j, i), tj, c.a(k, i));
  }
}

// rolled: the elimination as a loop over k; otherwise, up to 9 integrated
// species, unrolled (every index but the pivot row a compile-time constant,
// the updates of the columns right of the pivot independent instructions).
// The two forms give the same bits; the unrolled one is faster where the
// cells' BDF paths are alike (the flame), the rolled one, a quarter of the
// code, where they vary (instruction cache): the autotuner picks.
template <int N, bool RECIP, class CS>
__device__ __forceinline__ int dgefa(CS& c, RowPerm<N>* perm_out, bool rolled) {
  using LUT = typename std::remove_reference<decltype(c.a(0, 0))>::type;
  int info = 0;
  RowPerm<N> perm;
  perm.identity();
  if (rolled) {
#pragma unroll 1
    for (int k = 0; k < N - 1; ++k) dgefa_step<N, RECIP, CS, LUT>(c, k, perm, info);
  } else {
#pragma unroll(N <= 9 ? N : 1)
    for (int k = 0; k < N - 1; ++k) dgefa_step<N, RECIP, CS, LUT>(c, k, perm, info);
  }
  *perm_out = perm;
  if (c.a(N - 1, N - 1) == (LUT)0) info = N;
  else if (RECIP) c.a(N - 1, N - 1) = (LUT)1 / c.a(N - 1, N - 1);
  return info;
}

// dgesl.f90:71-131, JOB = 0, on the register vector b.  The permutation is
// applied at once through the cell's shared scratch z (free during a solve),
// then the forward sweep runs without interchanges: each element receives
// the same updates in the same order as in LINPACK's interleaved form.
// RECIP: the factors hold the pivots' reciprocals (see dgefa).
template <int N, bool RECIP, class CS>
__device__ __forceinline__ void dgesl(CS& c, double (&b)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) c.z(i) = b[i];
#pragma unroll
  for (int i = 0; i < N; ++i) b[i] = c.z(c.piv.get(i));
#pragma unroll
  for (int k = 0; k < N - 1; ++k) {
    const double t = b[k];
    if (t != 0.0) {
#pragma unroll
      for (int i = k + 1; i < N; ++i) b[i] = b[i] + t * (double)c.a(k, i);
    }
  }
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    b[k] = RECIP ? b[k] * (double)c.a(k, k) : ddiv(b[k], (double)c.a(k, k));
    const double t = -b[k];
    if (t != 0.0) {
#pragma unroll
      for (int i = 0; i < k; ++i) b[i] = b[i] + t * (double)c.a(k, i);
    }
  }
}

template <int N, int R, typename LUT, int BS, int SPEC>
__device__ __noinline__ void nl_rhs(double* d, LUT* f) {
  SmemStore<N, R, LUT, BS> s;
  s.d = d;
  s.f = f;
  if constexpr (SPEC != 0) {
    static_assert(N == SpecOf<SPEC>::kN && R == SpecOf<SPEC>::kR, "specialised code is for another mechanism size");
    SpecOf<SPEC>::rhs(s);
  } else {
    rhs<N, R>(s);
  }
}

template <int N, int R, typename LUT, int BS, int SPEC>
__device__ __noinline__ void nl_analytic_matrix(double* d, LUT* f, double factor) {
  SmemStore<N, R, LUT, BS> s;
  s.d = d;
  s.f = f;
  if constexpr (SPEC != 0) {
    static_assert(N == SpecOf<SPEC>::kN && R == SpecOf<SPEC>::kR, "specialised code is for another mechanism size");
    SpecOf<SPEC>::template matrix<SmemStore<N, R, LUT, BS>, LUT>(s, factor);
  } else {
    analytic_iteration_matrix<N, R>(s, factor);
  }
}

template <int N, int R, typename LUT, int BS, bool RECIP>
__device__ __noinline__ RowPerm<N> nl_dgefa(double* d, LUT* f, int* info, int rolled) {
  SmemStore<N, R, LUT, BS> s;
  s.d = d;
  s.f = f;
  RowPerm<N> perm;
  *info = dgefa<N, RECIP>(s, &perm, rolled != 0);
  return perm;
}

template <int N, int R, typename LUT, int BS, bool FAST>
__device__ __noinline__ void nl_rate_constants(double* d, LUT* f, double T) {
  SmemStore<N, R, LUT, BS> s;
  s.d = d;
  s.f = f;
  if constexpr (FAST) rate_constants_fast<N, R>(s, T);
  else rate_constants<N, R>(s, T);
}

// --------------------------------------------------------- SLATEC pieces
// ddpsc.f90:22-40 on the Nordsieck array (shared memory only, so one
// out-of-line copy serves every call site).  Species do not mix, so each
// species' column of the array is loaded into registers once, takes the
// reference's additions in the reference's order, and is stored once.
template <int N, int Q, class S>
__device__ __forceinline__ void ddpsc_order(S& c, int ksgn) {
  // one species at a time (unrolling the species, so that their addition
  // chains overlap, measured slower: 73.2 against 70.0 ms per flame step,
  // 122 against 103 ms on the ignition field, from the larger code)
#pragma unroll 1
  for (int i = 0; i < N; ++i) {
    double v[Q + 1];
#pragma unroll
    for (int j = 0; j <= Q; ++j) v[j] = c.yh(j, i);
#pragma unroll
    for (int j1 = 1; j1 <= Q; ++j1)
#pragma unroll
      for (int j2 = j1; j2 <= Q; ++j2) {
        const int j = Q - j2 + j1;  // 1-based column
        v[j - 1] = ksgn > 0 ? v[j - 1] + v[j] : v[j - 1] - v[j];
      }
#pragma unroll
    for (int j = 0; j < Q; ++j) c.yh(j, i) = v[j];
  }
}

template <int N, int R, typename LUT, int BS>
__device__ __noinline__ void nl_ddpsc(double* d, LUT* f, int ksgn, int nq) {
  SmemStore<N, R, LUT, BS> c;
  c.d = d;
  c.f = f;
  static_assert(kMaxOrd == 5, "one unrolled predictor per order");
  switch (nq) {
    case 1: ddpsc_order<N, 1>(c, ksgn); break;
    case 2: ddpsc_order<N, 2>(c, ksgn); break;
    case 3: ddpsc_order<N, 3>(c, ksgn); break;
    case 4: ddpsc_order<N, 4>(c, ksgn); break;
    case 5: ddpsc_order<N, 5>(c, ksgn); break;
    default: break;
  }
}

template <int N, class CS>
__device__ __forceinline__ void ddpsc(int ksgn, CS& c) {
  nl_ddpsc<N, CS::kR, typename CS::lut_t, CS::kBS>(c.d, c.f, ksgn, c.nq);
}

// ddscl.f90:20-37: limits rh, rescales columns 1..nq of the Nordsieck array;
// returns the rh applied.
template <int N, int R, typename LUT, int BS, int JAC>
__device__ __noinline__ double nl_ddscl(double* d, LUT* f, int nq, double h, double rmax, double rh) {
  SmemStore<N, R, LUT, BS> c;
  c.d = d;
  c.f = f;
  const double hmax = c_mech.hmax;
  if (h < 1.0) {
    const double ah = fabs(h);
    rh = sdiv<JAC>(NRG_FMIN(NRG_FMIN(ah * rh, ah * rmax), hmax), ah);
  } else {
    rh = NRG_FMIN(NRG_FMIN(rh, rmax), sdiv<JAC>(hmax, fabs(h)));
  }
  double r1 = 1.0;
  for (int j = 1; j <= nq; ++j) {
    r1 = r1 * rh;
#pragma unroll
    for (int i = 0; i < N; ++i) c.yh(j, i) = c.yh(j, i) * r1;
  }
  return rh;
}

template <int N, int JAC, class CS>
__device__ __forceinline__ void ddscl(CS& c, double rh) {
  rh = nl_ddscl<N, CS::kR, typename CS::lut_t, CS::kBS, JAC>(c.d, c.f, c.nq, c.h, c.rmax, rh);
  c.h = c.h * rh;
  c.rc = c.rc * rh;
}

#define EL(i, j) c_mech.el[((j)-1) * 13 + ((i)-1)]
#define TQ(i, j) c_mech.tq[((j)-1) * 3 + ((i)-1)]

template <int N, int R, class CS>
__device__ void ddntl(CS& c) {
  c.ier = 0;
  if (c.jtask == 0) c.rmax = 10000.0;
  c.rc = 0.0;
  c.convrg = 0;
  c.trend = 1.0;
  c.nq = 1;
  c.nwait = 3;
  rhs_at<N, R>(c, c.y, c.s2);
  c.nfe += 1;
#pragma unroll
  for (int i = 0; i < N; ++i) c.s1[i] = ddiv(c.s2[i], NRG_FMAX(1.0, c.ywt[i]));
  const double sum = ddiv(dnrm2<N>(c.s1), sqrt((double)CS::kNF));
  if (sum > ddiv(c.eps, fabs(c.h))) c.h = copysign(ddiv(c.eps, sum), c.h);
#pragma unroll
  for (int i = 0; i < N; ++i) c.yh(1, i) = c.h * c.s2[i];
#pragma unroll
  for (int i = 0; i < N; ++i) c.fac[i] = c_mech.sqrt_uround;
}

// Iteration matrix I - h*l0*J and its LU (DDPST, ddpst.f90:52-142).
template <int N, int R, int JAC, class CS>
__device__ void ddpst(CS& c) {
  c.nje += 1;
  c.ier = 0;
  const double el1h = EL(1, c.nq) * c.h;
  if (JAC == kJacFD) {
    const double FACMAX = 0.5, BU = 0.5;
    const double br = c_mech.br, bl = c_mech.bl, bp = c_mech.bp, facmin = c_mech.facmin;
#pragma unroll
    for (int k = 0; k < N; ++k) c.z(k) = c.y[k];
#pragma unroll 1
    for (int j = 0; j < N; ++j) {
      const double yj = sel(c.y, j);
      const double ys = NRG_FMAX(fabs(sel(c.ywt, j)), fabs(yj));
      double fj = sel(c.fac, j);
      double dy;
      for (;;) {
        dy = fj * ys;
        if (dy == 0.0) {
          if (fj < FACMAX) {
            fj = NRG_FMIN(100.0 * fj, FACMAX);
            continue;
          }
          dy = ys;
        }
        break;
      }
      dy = (c.nq == 1) ? copysign(dy, sel(c.s2, j)) : copysign(dy, c.yh(2, j));
      dy = (yj + dy) - yj;
      c.z(j) = yj + dy;
      nl_rhs<N, R, typename CS::lut_t, CS::kBS, CS::kSpec>(c.d, c.f);
      c.z(j) = yj;
      const double factor = -ddiv(el1h, dy);
      double diff = -1.0, s2m = 0.0, s1m = 0.0;
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const double f1 = c.zd(i);
        c.a(j, i) = (f1 - c.s2[i]) * factor;
        const double di = fabs(c.s2[i] - f1);
        if (di > diff) { diff = di; s2m = fabs(c.s2[i]); s1m = fabs(f1); }
      }
      if (NRG_FMIN(s2m, s1m) > 0.0) {
        const double scale = NRG_FMAX(s2m, s1m);
        if (diff > BU * scale) fj = NRG_FMAX(facmin, fj * 0.5);
        else if (br * scale <= diff && diff <= bl * scale) fj = NRG_FMIN(fj * 2.0, FACMAX);
        else if (diff < br * scale) fj = NRG_FMIN(bp * fj, FACMAX);
      }
      put(c.fac, j, fj);
    }
    c.nfe += N;
#pragma unroll
    for (int i = 0; i < N; ++i) c.a(i, i) += 1;
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) c.z(k) = c.y[k];
    nl_analytic_matrix<N, R, typename CS::lut_t, CS::kBS, CS::kSpec>(c.d, c.f, -el1h);
  }
  int info = 0;
  c.piv = nl_dgefa<N, R, typename CS::lut_t, CS::kBS, JAC != kJacFD>(c.d, c.f, &info, c.lu_rolled);
  if (info != 0) c.ier = 1;
}

// Corrector solve (DDCOR MITER=2, IMPL=0, ddcor.f90:61-107).  The right-hand
// side (the corrector residual) is always formed in FP64 from FP64 state; with
// float LU factors (mixed mode) the chord iteration that calls this solve
// until the FP64 convergence test passes is itself the iterative refinement of
// the FP32 solution, so no further sweep is made per solve.
template <int N, int R, int JAC, typename LUT, class CS>
__device__ double ddcor(CS& c) {
  double b[N];
#pragma unroll
  for (int i = 0; i < N; ++i) b[i] = c.h * c.s2[i] - c.yh(1, i) - c.s1[i];
  double x[N];
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = b[i];
  dgesl<N, JAC != kJacFD>(c, x);
  c.nsolve += 1;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    c.s1[i] = c.s1[i] + x[i];
  }
  if constexpr (JAC == kJacFD) {
    return ddiv(weighted_norm<N, JAC>(c, x), sqrt((double)CS::kNF));
  } else {
    constexpr double kInvSqrtNF = 1.0 / ct_sqrt((double)CS::kNF);
    return weighted_norm<N, JAC>(c, x) * kInvSqrtNF;
  }
}

// One DDSTP call (ddstp.f90:72-459); returns JSTATE (1 ok, 2 h vanished,
// 3 MXTRY retries, 4 singular).
template <int N, int R, int JAC, typename LUT, class CS>
__device__ int ddstp(CS& c) {
  const double BIAS1 = 1.3, BIAS2 = 1.2, BIAS3 = 1.4, RCTEST = 0.3, RMFAIL = 2.0, RMNORM = 10.0,
               TRSHLD = 1.0;
  const int MXFAIL = 3, MXITER = 3, MXTRY = 50, NDJSTP = 10;
  const double uround = c_mech.uround;
  const double eps = c.eps;
  const double sqn = sqrt((double)CS::kNF);
  int ntry = 0, nfail = 0, iter = 0;
  bool evaljc;
  double told = c.t, ctest = 0.0, d = 0.0, d1 = 0.0, etest, rh;
  bool restart = false;  // ddntl after MXFAIL failures (then RMAX = RMNORM)
  if (c.jtask <= 0) goto L_NTL;
L100:
  ntry = ntry + 1;
  if (ntry > MXTRY) goto L410;
  c.t = c.t + c.h;
  ddpsc<N>(1, c);
  evaljc = (fabs(c.rc - 1.0) > RCTEST) || (c.nstep >= c.jstepl + NDJSTP);
L110:
  iter = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
  rhs_at<N, R>(c, c.y, c.s2);
  c.nfe += 1;
  if (evaljc || c.ier) {
    ddpst<N, R, JAC>(c);
    if (c.ier) goto L160;
    c.convrg = 0;
    c.rc = 1.0;
    c.jstepl = c.nstep;
  }
#pragma unroll
  for (int i = 0; i < N; ++i) c.s1[i] = 0.0;
L130:
  d = ddcor<N, R, JAC, LUT>(c);
  if (iter > 0) c.trend = NRG_FMAX(0.9 * c.trend, sdiv<JAC>(d, d1));
  d1 = d;
  ctest = NRG_FMIN(2.0 * c.trend, 1.0) * d;
  if (ctest <= eps) goto L170;
  iter = iter + 1;
  if (iter < MXITER) {
    const double el1 = EL(1, c.nq);
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i) + el1 * c.s1[i];
    rhs_at<N, R>(c, c.y, c.s2);
    c.nfe += 1;
    goto L130;
  }
  if (c.convrg) {
    evaljc = true;
    goto L110;
  }
L160:
  c.t = told;
  ddpsc<N>(-1, c);
  c.nwait = c.nq + 2;
  if (c.jtask != 0 && c.jtask != 2) c.rmax = RMFAIL;
  rh = (iter == 0) ? 0.3 : 0.9 * ratio_pow<JAC>(sdiv<JAC>(eps, ctest), 0.2);
  if (rh * c.h == 0.0) goto L400;
  ddscl<N, JAC>(c, rh);
  goto L100;
L170:
  c.convrg = 1;
  etest = sdiv<JAC>(weighted_norm<N, JAC>(c, c.s1), TQ(2, c.nq) * sqn);
  if (etest > eps) {
    c.t = told;
    ddpsc<N>(-1, c);
    nfail = nfail + 1;
    if (nfail < MXFAIL || c.nq == 1) {
      if (c.jtask != 0 && c.jtask != 2) c.rmax = RMFAIL;
      const double rh2 = sdiv<JAC>(1.0, BIAS2 * ratio_pow<JAC>(sdiv<JAC>(etest, eps), sdiv<JAC>(1.0, (double)(c.nq + 1))));
      if (c.nq > 1) {
        double v[N];
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = c.yh(c.nq, i);
        const double erdn = sdiv<JAC>(weighted_norm<N, JAC>(c, v), TQ(1, c.nq) * sqn);
        const double rh1 = sdiv<JAC>(1.0, NRG_FMAX(1.0, BIAS1 * ratio_pow<JAC>(sdiv<JAC>(erdn, eps), sdiv<JAC>(1.0, (double)c.nq))));
        if (rh2 < rh1) {
          c.nq = c.nq - 1;
          c.rc = sdiv<JAC>(c.rc * EL(1, c.nq), EL(1, c.nq + 1));
          rh = rh1;
        } else {
          rh = rh2;
        }
      } else {
        rh = rh2;
      }
      c.nwait = c.nq + 2;
      if (rh * c.h == 0.0) goto L400;
      ddscl<N, JAC>(c, rh);
      goto L100;
    }
    nfail = 0;
    c.jtask = 2;
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
    restart = true;
    goto L_NTL;
  }
  c.nstep += 1;
  for (int j = 0; j <= c.nq; ++j) {
    const double e = EL(j + 1, c.nq);
#pragma unroll
    for (int i = 0; i < N; ++i) c.yh(j, i) = c.yh(j, i) + e * c.s1[i];
  }
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
  if (c.jtask == 0 || c.jtask == 2) {
    rh = sdiv<JAC>(1.0, NRG_FMAX(uround, BIAS2 * ratio_pow<JAC>(sdiv<JAC>(etest, eps), sdiv<JAC>(1.0, (double)(c.nq + 1)))));
    if (rh > TRSHLD) ddscl<N, JAC>(c, rh);
  } else if (c.nwait > 1) {
    c.nwait = c.nwait - 1;
    if (c.nwait == 1 && c.nq < kMaxOrd) {
#pragma unroll
      for (int i = 0; i < N; ++i) c.yh(kMaxOrd, i) = c.s1[i];
    }
  } else {
    double rh1, rh2, rh3;
    if (c.nq == 1) {
      rh1 = 0.0;
    } else {
      double v[N];
#pragma unroll
      for (int i = 0; i < N; ++i) v[i] = c.yh(c.nq, i);
      const double erdn = sdiv<JAC>(weighted_norm<N, JAC>(c, v), TQ(1, c.nq) * sqn);
      rh1 = sdiv<JAC>(1.0, NRG_FMAX(uround, BIAS1 * ratio_pow<JAC>(sdiv<JAC>(erdn, eps), sdiv<JAC>(1.0, (double)c.nq))));
    }
    rh2 = sdiv<JAC>(1.0, NRG_FMAX(uround, BIAS2 * ratio_pow<JAC>(sdiv<JAC>(etest, eps), sdiv<JAC>(1.0, (double)(c.nq + 1)))));
    if (c.nq == kMaxOrd) {
      rh3 = 0.0;
    } else {
      double v[N];
#pragma unroll
      for (int i = 0; i < N; ++i) v[i] = c.s1[i] - c.yh(kMaxOrd, i);
      const double erup = sdiv<JAC>(weighted_norm<N, JAC>(c, v), TQ(3, c.nq) * sqn);
      rh3 = sdiv<JAC>(1.0, NRG_FMAX(uround, BIAS3 * ratio_pow<JAC>(sdiv<JAC>(erup, eps), sdiv<JAC>(1.0, (double)(c.nq + 2)))));
    }
    if (rh1 > rh2 && rh1 >= rh3) {
      rh = rh1;
      if (rh <= TRSHLD) goto L380;
      c.nq = c.nq - 1;
      c.rc = sdiv<JAC>(c.rc * EL(1, c.nq), EL(1, c.nq + 1));
    } else if (rh2 >= rh1 && rh2 >= rh3) {
      rh = rh2;
      if (rh <= TRSHLD) goto L380;
    } else {
      rh = rh3;
      if (rh <= TRSHLD) goto L380;
      const double e = EL(c.nq + 1, c.nq);
#pragma unroll
      for (int i = 0; i < N; ++i) c.yh(c.nq + 1, i) = sdiv<JAC>(c.s1[i] * e, (double)(c.nq + 1));
      c.nq = c.nq + 1;
      c.rc = sdiv<JAC>(c.rc * EL(1, c.nq), EL(1, c.nq - 1));
    }
    ddscl<N, JAC>(c, rh);
    c.rmax = RMNORM;
  L380:
    c.nwait = c.nq + 2;
  }
  return 1;
L_NTL:
  // the one inlined copy of DDNTL (first step and restart after failures)
  ddntl<N, R>(c);
  if (restart) c.rmax = RMNORM;
  if (c.h == 0.0) goto L400;
  if (c.ier) goto L420;
  goto L100;
L400:
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
  return 2;
L410:
  return 3;
L420:
  return 4;
}

// ----------------------------------------------------------- cell driver
// Cell set-up: skip rule (chemical_kinetics_solver.f90:228-231), third-body
// sums (:238-248), rate constants (:251), DDRIV3 init (ddriv3.f90:930-978).
// Returns false when the cell is passed through (outputs already written).
template <int N, int R, int JAC, class CS>
__device__ bool cell_begin(CS& c, const StepArgs& a, long cid) {
  constexpr int NF = CS::kNF;
  const double Tc = a.T[cid];
  if (!reference_cell_active(Tc, a.bc, cid)) {
    write_skipped_cell(a, cid, NF, Tc);
    return false;
  }
  const double rho = a.rho[cid];
  double yk[NF], conc[NF];
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    yk[k] = a.Y[k * a.ld + cid];
    conc[k] = yk[k] * rho / c_mech.W[k];  // the reference's Y*rho/W, formed once
  }
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NF; ++k) s = s + conc[k] * c_mech.eff_t[k][r];
    c.kr(r) = s;  // third-body sum, consumed by rate_constants
  }
  nl_rate_constants<N, R, typename CS::lut_t, CS::kBS, JAC != kJacFD>(c.d, c.f, Tc);
  if (NF == N) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double ci = yk[k] * rho / c_mech.W[k];
      c.yh(0, k) = ci;
      c.y[k] = ci;
    }
  } else {
    double ci[NF];
#pragma unroll
    for (int k = 0; k < NF; ++k) ci[k] = yk[k] * rho / c_mech.W[k];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double v = ci[c_mech.full_of[i]];
      c.yh(0, i) = v;
      c.y[i] = v;
    }
  }
  c.tout = a.dt_cells ? a.dt_cells[cid] : a.dt;
  c.t = 0.0;
  const double h = (c.tout - c.t) * (1.0 - 4.0 * c_mech.uround);
  c.h = copysign(NRG_FMIN(fabs(h), c_mech.hmax), h);
  c.eps = a.eps > 0.0 ? a.eps : c_mech.eps;
  c.jtask = 0;
  c.lu_rolled = a.lu_rolled;
  c.nstep = 0;
  c.nstepl = 0;
  c.jstepl = 0;
  c.nfe = 0;
  c.nje = 0;
  c.nsolve = 0;
  c.convrg = 0;
  c.ier = 0;
  c.nq = 1;
  c.rc = 0.0;
  c.rmax = 10000.0;
  c.trend = 1.0;
  c.nwait = 3;
  c.piv.identity();
  return true;
}

// One pass of the DDRIV3 loop (label 260, ddriv3.f90:1292-1448): error
// weights, accuracy and MXSTEP checks, one DDSTP step and, on reaching TOUT,
// the Nordsieck interpolation (DDNTP).  Returns 0 while running, else a
// CellStatus.
template <int N, int R, int JAC, typename LUT, class CS>
__device__ int cell_advance(CS& c, int mxstep) {
#pragma unroll
  for (int i = 0; i < N; ++i) c.ywt[i] = NRG_FMAX(c_mech.ewt, fabs(c.y[i]));
  // ddriv3.f90:1304-1316 tests EPS against SUM * UROUND with
  // SUM = max(1, rms_i(y_i / YWT_i)).  Here that SUM is exactly 1: YWT_i =
  // max(EWT, |y_i|) >= |y_i|, so every ratio is at most 1 in magnitude, their
  // sum of squares at most N and the rms at most 1, and rounding (monotone,
  // with N and sqrt(N) representable) cannot push it above 1; a NaN ratio
  // makes the test false in both forms.  The norm is therefore not formed.
  const double sum = 1.0;
  if (c.eps < sum * c_mech.uround) {
    c.eps = sum * c_mech.uround * (1.0 + 10.0 * c_mech.uround);
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
    return kCellOk;  // NSTATE = 4: the state at the current T is returned
  }
  if (c.nstep - c.nstepl == mxstep) {
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
    return kCellMxstep;
  }
  const int js = ddstp<N, R, JAC, LUT>(c);
  if (js != 1) {
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh(0, i);
    return kCellFatal;
  }
  c.jtask = 1;
  if (c.t < c.tout) return 0;
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh(c.nq, i);
  const double r = sdiv<JAC>(c.tout - c.t, c.h);
  for (int jj = 1; jj <= c.nq; ++jj) {
    const int j = c.nq - jj;
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh(j, i) + r * c.y[i];
  }
  return kCellOk;
}

// Energy closure at constant density: the temperature the reference EOS
// computes after the sources are added (cpm_solver.f90:517,549 ->
// table_approximated_real_gas.f90:404-440 -> calculate_temperature,
// thermophysical_properties_class.f90:409-452).  The reference starts the
// Newton iteration (frozen cp) at the temperature before the step; T_start
// lets a caller that already has an estimate of the result start there.
template <int N>
__device__ __noinline__ double temperature_after_nl(double T0, double T_start, const double* Y0, const double* dY,
                                                    double dE) {
  const double RG = 8.31446261815324;
  double X[N], avg = 0.0;
#pragma unroll 1
  for (int k = 0; k < N; ++k) avg = avg + ddiv(Y0[k], c_mech.W[k]);
  const double W0 = ddiv(1.0, avg);
  double e0 = 0.0, h0 = 0.0;
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    X[k] = ddiv(Y0[k], c_mech.W[k]) * W0;
    e0 = e0 + (d_enthalpy(T0, k) - RG * T0) * X[k];
  }
#pragma unroll 1
  for (int k = 0; k < N; ++k) h0 = h0 + c_mech.h_ref[k] * X[k];
  const double e1 = ddiv(e0 - h0, W0) + dE;
  avg = 0.0;
  double Y1[N];
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    Y1[k] = Y0[k] + dY[k];
    avg = avg + ddiv(Y1[k], c_mech.W[k]);
  }
  const double W1 = ddiv(1.0, avg);
  double hc = 0.0, cp = 0.0;
  double temp = NRG_FMIN(T_start, 6000.0);
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    X[k] = ddiv(Y1[k], c_mech.W[k]) * W1;
    hc = hc + c_mech.h_ref[k] * X[k];
    cp = cp + d_cp(temp, k) * X[k];
  }
  const double ei = e1 * W1;
  const double tol = (double)1e-08f;  // single-precision literal in the reference
  for (int it = 0; it < 1000; ++it) {
    double e = 0.0;
#pragma unroll 1
    for (int k = 0; k < N; ++k) e = e + (d_enthalpy(temp, k) - RG * temp) * X[k];
    const double res = ddiv(ei - (e - hc), cp);
    temp = temp + res;
    if (fabs(res) < tol) break;
  }
  return temp;
}

template <int N>
__device__ __forceinline__ double temperature_after(double T0, const double (&Y0)[N], const double (&dY)[N],
                                                    double dE, double T_start) {
  double a[N], b[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    a[k] = Y0[k];
    b[k] = dY[k];
  }
  return temperature_after_nl<N>(T0, T_start, a, b, dE);
}

template <int N>
__device__ __forceinline__ double temperature_after(double T0, const double (&Y0)[N], const double (&dY)[N],
                                                    double dE) {
  return temperature_after<N>(T0, Y0, dY, dE, T0);
}

// The same energy closure for the analytic-Jacobian and mixed modes, whose
// temperatures agree with the reference's to its tolerance rather than bit
// for bit: unrolled over the species in registers, with the reciprocal molar
// masses and one reciprocal of the frozen cp, inline (it runs once per cell,
// after the integration, when the integrator's registers are free).
__device__ __forceinline__ double nasa_enthalpy_fast(int k, double T) {
  const double t = NRG_FMIN(T, 6000.0);
  const double* a = c_mech.a[k][nasa_set(t)];
  const double hp = fma(fma(fma(fma(a[4] * 0.2, t, a[3] * 0.25), t, a[2] * (1.0 / 3.0)), t, a[1] * 0.5), t, a[0]);
  return fma(hp, t, a[5]);
}

template <int N>
__device__ __forceinline__ double temperature_after_fast(double T0, const double (&Y0)[N], const double (&dY)[N],
                                                         double dE) {
  const double RG = 8.31446261815324;
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) s0 += Y0[k] * c_mech.invW[k];
  const double W0 = 1.0 / s0;
  double e0 = 0.0, h0 = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double x = Y0[k] * c_mech.invW[k] * W0;
    e0 += nasa_enthalpy_fast(k, T0) * x;
    h0 += c_mech.h_ref[k] * x;
  }
  e0 -= RG * T0;
  const double e1 = (e0 - h0) / W0 + dE;
  double X[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    X[k] = Y0[k] + dY[k];
    s1 += X[k] * c_mech.invW[k];
  }
  const double W1 = 1.0 / s1;
  double hc = 0.0, cp = 0.0;
  double temp = NRG_FMIN(T0, 6000.0);
  const int set = nasa_set(temp);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    X[k] = X[k] * c_mech.invW[k] * W1;
    hc += c_mech.h_ref[k] * X[k];
    const double* a = c_mech.a[k][set];
    cp += fma(fma(fma(fma(a[4], temp, a[3]), temp, a[2]), temp, a[1]), temp, a[0]) * X[k];
  }
  const double ei = e1 * W1, rcp = 1.0 / cp;
  for (int it = 0; it < 1000; ++it) {
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) e += nasa_enthalpy_fast(k, temp) * X[k];
    e -= RG * temp;
    const double res = (ei - (e - hc)) * rcp;
    temp += res;
    if (fabs(res) < (double)1e-08f) break;
  }
  return temp;
}

// Outputs of a finished cell (chemical_kinetics_solver.f90:318-340); inert
// species keep their concentration, so their sources are exactly zero.
template <int N, int JAC, class CS>
__device__ void cell_finish(const CS& c, const StepArgs& a, long cid, int st) {
  constexpr int NF = CS::kNF;
  const double dt = c.tout;
  const double rho = a.rho[cid];
  double E = 0.0;
  bool finite = true;
  double Y0[NF], dYm[NF], dcs[NF];
#pragma unroll
  for (int k = 0; k < NF; ++k) Y0[k] = a.Y[k * a.ld + cid];
  if (NF == N) {
#pragma unroll
    for (int k = 0; k < NF; ++k) dcs[k] = c.y[k] - Y0[k] * rho / c_mech.W[k];
  } else {
#pragma unroll
    for (int k = 0; k < NF; ++k) dcs[k] = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const int k = c_mech.full_of[i];
      dcs[k] = c.y[i] - Y0[k] * rho / c_mech.W[k];
    }
  }
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    const double dc = dcs[k];
    finite = finite && isfinite(dc);
    const double yp = dc * c_mech.W[k] / dt;
    a.Y_prod[k * a.ld + cid] = yp;
    a.Y_prod2[k * a.ld + cid] = dc;
    E = E - c_mech.h_ref[k] * dc / dt;
    dYm[k] = yp * dt / rho;
  }
  a.E_f_prod[cid] = E;
  if (a.T_after) {
    if constexpr (JAC == kJacFD) a.T_after[cid] = temperature_after<NF>(a.T[cid], Y0, dYm, E * dt / rho);
    else a.T_after[cid] = temperature_after_fast<NF>(a.T[cid], Y0, dYm, E * dt / rho);
  }
  if (a.status) a.status[cid] = finite ? (uint8_t)st : (uint8_t)kCellNonfinite;
}

}  // namespace nrg
