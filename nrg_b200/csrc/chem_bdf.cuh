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

#include "chem_device.cuh"
#include "chem_kernels.hpp"

namespace nrg {

// Each translation unit that includes this header holds its own copy of the
// tables and uploads it (upload_mechanism / surrogate set-up).
static __constant__ DevMech c_mech;

enum JacMode { kJacFD = 0, kJacAnalytic = 1 };

template <int N, int R, typename LUT>
struct CellState {
  double yh[kMaxOrd + 1][N];
  LUT a[N][N];  // column-major: a[j][i] = A(i+1, j+1)
  double ywt[N], s1[N], s2[N], fac[N], y[N];
  double kf[R], kr[R], mc[R];
  double conc_in[N];
  int ipvt[N];
  double h, t, tout, rc, rmax, trend, eps;
  int nq, nwait, jtask, nstep, nfe, nje, nsolve, jstepl, nstepl, convrg, ier;
  int refine;  // iterative-refinement sweeps taken (mixed mode)
};

#define NRG_FMAX(a, b) ((a) >= (b) ? (a) : (b))
#define NRG_FMIN(a, b) ((a) <= (b) ? (a) : (b))

// -------------------------------------------------------------- thermo
__device__ __forceinline__ int nasa_set(double t) { return t >= 1000.0 ? 1 : 0; }

__device__ __forceinline__ double d_enthalpy(double T, int k) {
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

__device__ __forceinline__ double d_entropy(double T, int k, double logt) {
  double t = NRG_FMIN(T, 6000.0);
  const double* a = c_mech.a[k][nasa_set(t)];
  double s = a[4] / 4.0;
  s = s * t + a[3] / 3.0;
  s = s * t + a[2] / 2.0;
  s = s * t + a[1] / 1.0;
  return s * t + a[6] + a[0] * logt;
}

__device__ __forceinline__ double d_cp(double T, int k) {
  double t = NRG_FMIN(T, 6000.0);
  const double* a = c_mech.a[k][nasa_set(t)];
  double cp = a[4];
  cp = cp * t + a[3];
  cp = cp * t + a[2];
  cp = cp * t + a[1];
  cp = cp * t + a[0];
  return cp;
}

// x ** dnu for the integer stoichiometric change of a reaction
__device__ __forceinline__ double int_pow(double x, double dnu) {
  if (dnu == 0.0) return 1.0;
  if (dnu == 1.0) return x;
  if (dnu == -1.0) return 1.0 / x;
  if (dnu == 2.0) return x * x;
  if (dnu == -2.0) return 1.0 / (x * x);
  return pow(x, dnu);
}

// calculate_rate_constants (chemical_kinetics_solver.f90:360-493)
template <int N, int R>
__device__ void rate_constants(double Tin, const double* mc, double* kf, double* kr) {
  const double RG = 8.31446261815324, PATM = 101325.0;
  double T = NRG_FMIN(Tin, 10000.0);
  double tt = NRG_FMIN(T, 6000.0);
  double logt = log(tt);
  double s[N], h[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    s[k] = d_entropy(T, k, logt);
    h[k] = d_enthalpy(T, k);
  }
  const double inv_RT = 1.0 / RG / T;  // only used through the reference order below
  (void)inv_RT;
  const double conc_ref = PATM / RG / T;
  for (int r = 0; r < R; ++r) {
    double d_s = 0.0, d_h = 0.0;
    for (int i = 0; i < c_mech.nr[r]; ++i) {
      int sp = c_mech.right[r][i];
      if (sp < 0) continue;
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (k == sp) { d_s = d_s + s[k]; d_h = d_h + h[k]; }
    }
    for (int i = 0; i < c_mech.nl[r]; ++i) {
      int sp = c_mech.left[r][i];
      if (sp < 0) continue;
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (k == sp) { d_s = d_s - s[k]; d_h = d_h - h[k]; }
    }
    const int type = c_mech.type[r];
    double kinf = c_mech.A[r] * pow(T, c_mech.beta[r]) * exp(-(c_mech.E[r] / RG / T));
    double k = kinf;
    if (type == 2 || type == 3 || type == 7) {
      double k0 = c_mech.A_low[r] * pow(T, c_mech.beta_low[r]) * exp(-(c_mech.E_low[r] / RG / T));
      double rp = k0 * mc[r] / kinf;
      k = kinf * (rp / (1.0 + rp));
      if (type == 3) {
        const double al = c_mech.troe[r][0];
        double Fc = (1.0 - al) * exp(-(T / c_mech.troe[r][1])) + al * exp(-(T / c_mech.troe[r][2])) +
                    exp(-(c_mech.troe[r][3] / T));
        double lf = log10(Fc);
        double c = -0.4 - 0.67 * lf;
        double nn = 0.75 - 1.27 * lf;
        double blend;
        if (rp != 0.0) {
          double lr = log10(rp);
          double x = (lr + c) / (nn - 0.14 * (lr + c));
          blend = pow(Fc, 1.0 / (1.0 + x * x));
        } else {
          blend = pow(Fc, -1.0 / 0.14);
        }
        k = k * blend;
      }
    }
    kf[r] = k;
    if (type >= 5) {
      kr[r] = 0.0;
    } else {
      double Kp = exp(d_s / RG - d_h / RG / T);
      double Kc = Kp * int_pow(conc_ref, c_mech.dnu[r]);
      kr[r] = k / Kc;
    }
  }
}

// fun (chemical_kinetics_solver.f90:495-540); zd accumulated in the
// reference order (reaction-major, then the species-ordered update list).
template <int N, int R, typename CS>
__device__ __forceinline__ void rhs(const CS& c, const double* z, double* zd) {
#pragma unroll
  for (int k = 0; k < N; ++k) zd[k] = 0.0;
  for (int r = 0; r < R; ++r) {
    double f = c.kf[r];
    for (int i = 0; i < c_mech.nl[r]; ++i) {
      int sp = c_mech.left[r][i];
      f = f * (sp < 0 ? c.mc[r] : z[sp]);
    }
    double b = c.kr[r];
    for (int i = 0; i < c_mech.nr[r]; ++i) {
      int sp = c_mech.right[r][i];
      b = b * (sp < 0 ? c.mc[r] : z[sp]);
    }
    for (int u = 0; u < c_mech.nupd[r]; ++u) {
      int k = c_mech.upd_k[r][u];
      if (c_mech.upd_prod[r][u]) zd[k] = zd[k] - b + f;
      else zd[k] = zd[k] - f + b;
    }
  }
}

// dZdot/dZ of the mass-action RHS.  jac is column-major (jac[j][i] =
// dZdot_i/dZ_j) and is overwritten.
template <int N, int R, typename CS>
__device__ void analytic_jacobian(const CS& c, const double* z, double jac[N][N]) {
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int i = 0; i < N; ++i) jac[j][i] = 0.0;
  for (int r = 0; r < R; ++r) {
    const int nl = c_mech.nl[r], nr = c_mech.nr[r];
    double fac_l[3], fac_r[3];
    for (int i = 0; i < 3; ++i) {
      int sl = i < nl ? c_mech.left[r][i] : -2;
      int sr = i < nr ? c_mech.right[r][i] : -2;
      fac_l[i] = sl == -2 ? 1.0 : (sl < 0 ? c.mc[r] : z[sl]);
      fac_r[i] = sr == -2 ? 1.0 : (sr < 0 ? c.mc[r] : z[sr]);
    }
    const int nu = c_mech.nupd[r];
    // forward partials
    for (int p = 0; p < nl; ++p) {
      int sp = c_mech.left[r][p];
      if (sp < 0) continue;
      double d = c.kf[r];
      for (int q = 0; q < 3; ++q)
        if (q != p) d = d * fac_l[q];
      for (int u = 0; u < nu; ++u) {
        int k = c_mech.upd_k[r][u];
        if (c_mech.upd_prod[r][u]) jac[sp][k] += d;
        else jac[sp][k] -= d;
      }
    }
    // reverse partials
    for (int p = 0; p < nr; ++p) {
      int sp = c_mech.right[r][p];
      if (sp < 0) continue;
      double d = c.kr[r];
      for (int q = 0; q < 3; ++q)
        if (q != p) d = d * fac_r[q];
      for (int u = 0; u < nu; ++u) {
        int k = c_mech.upd_k[r][u];
        if (c_mech.upd_prod[r][u]) jac[sp][k] -= d;
        else jac[sp][k] += d;
      }
    }
  }
}

// dnrm2.f90:75-162 -- Lawson-Hanson scaled two-norm (sequential phases)
template <int N>
__device__ double dnrm2(const double* dx) {
  const double cutlo = 8.232e-11, cuthi = 1.304e19;
  double sum = 0.0, xmax = 0.0;
  int next = 30, i = 0, j = 0;
L20:
  if (next == 30) goto L30;
  if (next == 50) goto L50;
  if (next == 70) goto L70;
  goto L110;
L30:
  if (fabs(dx[i]) > cutlo) goto L85;
  next = 50;
  xmax = 0.0;
L50:
  if (dx[i] == 0.0) goto L200;
  if (fabs(dx[i]) > cutlo) goto L85;
  next = 70;
  goto L105;
L100:
  i = j;
  next = 110;
  sum = (sum / dx[i]) / dx[i];
L105:
  xmax = fabs(dx[i]);
  goto L115;
L70:
  if (fabs(dx[i]) > cutlo) goto L75;
L110:
  if (fabs(dx[i]) <= xmax) goto L115;
  {
    double q = xmax / dx[i];
    sum = 1.0 + sum * (q * q);
  }
  xmax = fabs(dx[i]);
  goto L200;
L115: {
  double q = dx[i] / xmax;
  sum = sum + q * q;
}
  goto L200;
L75:
  sum = (sum * xmax) * xmax;
L85: {
  const double hitest = cuthi / (double)N;
  for (j = i; j < N; ++j) {
    if (fabs(dx[j]) >= hitest) goto L100;
    sum = sum + dx[j] * dx[j];
  }
}
  return sqrt(sum);
L200:
  i = i + 1;
  if (i < N) goto L20;
  return xmax * sqrt(sum);
}

// dgefa.f90:60-117 on the column-major matrix a (element type LUT)
template <int N, typename LUT>
__device__ int dgefa(LUT a[N][N], int* ipvt) {
  int info = 0;
  for (int k = 0; k < N - 1; ++k) {
    // idamax over a[k][k..N-1]
    int l = k;
    LUT dmax = fabs(a[k][k]);
    for (int i = k + 1; i < N; ++i) {
      LUT xm = fabs(a[k][i]);
      if (xm > dmax) { l = i; dmax = xm; }
    }
    ipvt[k] = l;
    if (a[k][l] == (LUT)0) { info = k + 1; continue; }
    if (l != k) {
      LUT t = a[k][l];
      a[k][l] = a[k][k];
      a[k][k] = t;
    }
    LUT t = (LUT)-1 / a[k][k];
    for (int i = k + 1; i < N; ++i) a[k][i] = t * a[k][i];
    for (int j = k + 1; j < N; ++j) {
      LUT tj = a[j][l];
      if (l != k) {
        a[j][l] = a[j][k];
        a[j][k] = tj;
      }
      if (tj != (LUT)0)
        for (int i = k + 1; i < N; ++i) a[j][i] = a[j][i] + tj * a[k][i];
    }
  }
  ipvt[N - 1] = N - 1;
  if (a[N - 1][N - 1] == (LUT)0) info = N;
  return info;
}

// dgesl.f90:71-131, JOB = 0 (b overwritten with the solution)
template <int N, typename LUT, typename VT>
__device__ void dgesl(const LUT a[N][N], const int* ipvt, VT* b) {
  for (int k = 0; k < N - 1; ++k) {
    int l = ipvt[k];
    VT t = b[l];
    if (l != k) {
      b[l] = b[k];
      b[k] = t;
    }
    if (t != (VT)0)
      for (int i = k + 1; i < N; ++i) b[i] = b[i] + t * (VT)a[k][i];
  }
  for (int k = N - 1; k >= 0; --k) {
    b[k] = b[k] / (VT)a[k][k];
    VT t = -b[k];
    if (t != (VT)0)
      for (int i = 0; i < k; ++i) b[i] = b[i] + t * (VT)a[k][i];
  }
}

// --------------------------------------------------------- SLATEC pieces
template <int N, typename CS>
__device__ __forceinline__ void ddpsc(int ksgn, CS& c) {
  const int nq = c.nq;
  for (int j1 = 1; j1 <= nq; ++j1)
    for (int j2 = j1; j2 <= nq; ++j2) {
      int j = nq - j2 + j1;  // 1-based column
      if (ksgn > 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) c.yh[j - 1][i] = c.yh[j - 1][i] + c.yh[j][i];
      } else {
#pragma unroll
        for (int i = 0; i < N; ++i) c.yh[j - 1][i] = c.yh[j - 1][i] - c.yh[j][i];
      }
    }
}

template <int N, typename CS>
__device__ __forceinline__ void ddscl(CS& c, double rh) {
  const double hmax = c_mech.hmax;
  if (c.h < 1.0) {
    double ah = fabs(c.h);
    rh = NRG_FMIN(NRG_FMIN(ah * rh, ah * c.rmax), hmax) / ah;
  } else {
    rh = NRG_FMIN(NRG_FMIN(rh, c.rmax), hmax / fabs(c.h));
  }
  double r1 = 1.0;
  for (int j = 1; j <= c.nq; ++j) {
    r1 = r1 * rh;
#pragma unroll
    for (int i = 0; i < N; ++i) c.yh[j][i] = c.yh[j][i] * r1;
  }
  c.h = c.h * rh;
  c.rc = c.rc * rh;
}

#define EL(i, j) c_mech.el[((j)-1) * 13 + ((i)-1)]
#define TQ(i, j) c_mech.tq[((j)-1) * 3 + ((i)-1)]

template <int N, int R, typename CS>
__device__ void ddntl(CS& c) {
  c.ier = 0;
  if (c.jtask == 0) c.rmax = 10000.0;
  c.rc = 0.0;
  c.convrg = 0;
  c.trend = 1.0;
  c.nq = 1;
  c.nwait = 3;
  rhs<N, R>(c, c.y, c.s2);
  c.nfe += 1;
#pragma unroll
  for (int i = 0; i < N; ++i) c.s1[i] = c.s2[i] / NRG_FMAX(1.0, c.ywt[i]);
  double sum = dnrm2<N>(c.s1) / sqrt((double)N);
  if (sum > c.eps / fabs(c.h)) c.h = copysign(c.eps / sum, c.h);
#pragma unroll
  for (int i = 0; i < N; ++i) c.yh[1][i] = c.h * c.s2[i];
#pragma unroll
  for (int i = 0; i < N; ++i) c.fac[i] = c_mech.sqrt_uround;
}

// Iteration matrix I - h*l0*J and its LU (DDPST MITER=2 or analytic J).
template <int N, int R, int JAC, typename CS>
__device__ void ddpst(CS& c) {
  c.nje += 1;
  c.ier = 0;
  const double el1h = EL(1, c.nq) * c.h;
  if (JAC == kJacFD) {
    const double FACMAX = 0.5, BU = 0.5;
    const double br = c_mech.br, bl = c_mech.bl, bp = c_mech.bp, facmin = c_mech.facmin;
    for (int j = 0; j < N; ++j) {
      double ys = NRG_FMAX(fabs(c.ywt[j]), fabs(c.y[j]));
      double dy;
      for (;;) {
        dy = c.fac[j] * ys;
        if (dy == 0.0) {
          if (c.fac[j] < FACMAX) {
            c.fac[j] = NRG_FMIN(100.0 * c.fac[j], FACMAX);
            continue;
          }
          dy = ys;
        }
        break;
      }
      dy = (c.nq == 1) ? copysign(dy, c.s2[j]) : copysign(dy, c.yh[2][j]);
      dy = (c.y[j] + dy) - c.y[j];
      double yj = c.y[j];
      c.y[j] = c.y[j] + dy;
      rhs<N, R>(c, c.y, c.s1);
      c.y[j] = yj;
      double factor = -(el1h / dy);
#pragma unroll
      for (int i = 0; i < N; ++i) c.a[j][i] = (c.s1[i] - c.s2[i]) * factor;
      double diff = fabs(c.s2[0] - c.s1[0]);
      int imax = 0;
#pragma unroll
      for (int i = 1; i < N; ++i) {
        double di = fabs(c.s2[i] - c.s1[i]);
        if (di > diff) { imax = i; diff = di; }
      }
      double s2m = 0.0, s1m = 0.0;
#pragma unroll
      for (int i = 0; i < N; ++i)
        if (i == imax) { s2m = fabs(c.s2[i]); s1m = fabs(c.s1[i]); }
      if (NRG_FMIN(s2m, s1m) > 0.0) {
        double scale = NRG_FMAX(s2m, s1m);
        if (diff > BU * scale) c.fac[j] = NRG_FMAX(facmin, c.fac[j] * 0.5);
        else if (br * scale <= diff && diff <= bl * scale) c.fac[j] = NRG_FMIN(c.fac[j] * 2.0, FACMAX);
        else if (diff < br * scale) c.fac[j] = NRG_FMIN(bp * c.fac[j], FACMAX);
      }
    }
    c.nfe += N;
  } else {
    double jac[N][N];
    analytic_jacobian<N, R>(c, c.y, jac);
    const double factor = -el1h;
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
      for (int i = 0; i < N; ++i) c.a[j][i] = factor * jac[j][i];
  }
#pragma unroll
  for (int i = 0; i < N; ++i) c.a[i][i] = c.a[i][i] + 1.0;
  int info = dgefa<N>(c.a, c.ipvt);
  if (info != 0) c.ier = 1;
}

// Corrector solve (DDCOR MITER=2, IMPL=0).  With float LU factors the
// correction is refined: r = rhs - M x is formed in double with M rebuilt
// from its definition (I - h l0 J applied through a Jacobian-vector product
// would need J; instead the refinement uses the stored double residual of the
// Newton system, see mixed_solve).
template <int N, typename CS>
__device__ double ddcor(CS& c) {
#pragma unroll
  for (int i = 0; i < N; ++i) c.s2[i] = c.h * c.s2[i] - c.yh[1][i] - c.s1[i];
  dgesl<N>(c.a, c.ipvt, c.s2);
  c.nsolve += 1;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    c.s1[i] = c.s1[i] + c.s2[i];
    c.s2[i] = c.s2[i] / NRG_FMAX(fabs(c.y[i]), c.ywt[i]);
  }
  return dnrm2<N>(c.s2) / sqrt((double)N);
}

// One DDSTP call; returns JSTATE (1 ok, 2 h vanished, 3 MXTRY, 4 singular).
template <int N, int R, int JAC, typename CS>
__device__ int ddstp(CS& c) {
  const double BIAS1 = 1.3, BIAS2 = 1.2, BIAS3 = 1.4, RCTEST = 0.3, RMFAIL = 2.0, RMNORM = 10.0,
               TRSHLD = 1.0;
  const int MXFAIL = 3, MXITER = 3, MXTRY = 50, NDJSTP = 10;
  const double uround = c_mech.uround;
  const double eps = c.eps;
  const double sqn = sqrt((double)N);
  int ntry = 0, nfail = 0, iter = 0;
  bool evaljc;
  double told = c.t, ctest = 0.0, d = 0.0, d1 = 0.0, etest, rh;
  if (c.jtask <= 0) {
    ddntl<N, R>(c);
    if (c.h == 0.0) goto L400;
    if (c.ier) goto L420;
  }
L100:
  ntry = ntry + 1;
  if (ntry > MXTRY) goto L410;
  c.t = c.t + c.h;
  ddpsc<N>(1, c);
  evaljc = (fabs(c.rc - 1.0) > RCTEST) || (c.nstep >= c.jstepl + NDJSTP);
L110:
  iter = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
  rhs<N, R>(c, c.y, c.s2);
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
  d = ddcor<N>(c);
  if (iter > 0) c.trend = NRG_FMAX(0.9 * c.trend, d / d1);
  d1 = d;
  ctest = NRG_FMIN(2.0 * c.trend, 1.0) * d;
  if (ctest <= eps) goto L170;
  iter = iter + 1;
  if (iter < MXITER) {
    const double el1 = EL(1, c.nq);
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i] + el1 * c.s1[i];
    rhs<N, R>(c, c.y, c.s2);
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
  rh = (iter == 0) ? 0.3 : 0.9 * pow(eps / ctest, 0.2);
  if (rh * c.h == 0.0) goto L400;
  ddscl<N>(c, rh);
  goto L100;
L170:
  c.convrg = 1;
#pragma unroll
  for (int i = 0; i < N; ++i) c.s2[i] = c.s1[i] / NRG_FMAX(fabs(c.y[i]), c.ywt[i]);
  etest = dnrm2<N>(c.s2) / (TQ(2, c.nq) * sqn);
  if (etest > eps) {
    c.t = told;
    ddpsc<N>(-1, c);
    nfail = nfail + 1;
    if (nfail < MXFAIL || c.nq == 1) {
      if (c.jtask != 0 && c.jtask != 2) c.rmax = RMFAIL;
      double rh2 = 1.0 / (BIAS2 * pow(etest / eps, 1.0 / (double)(c.nq + 1)));
      if (c.nq > 1) {
#pragma unroll
        for (int i = 0; i < N; ++i) c.s2[i] = c.yh[c.nq][i] / NRG_FMAX(fabs(c.y[i]), c.ywt[i]);
        double erdn = dnrm2<N>(c.s2) / (TQ(1, c.nq) * sqn);
        double rh1 = 1.0 / NRG_FMAX(1.0, BIAS1 * pow(erdn / eps, 1.0 / (double)c.nq));
        if (rh2 < rh1) {
          c.nq = c.nq - 1;
          c.rc = c.rc * EL(1, c.nq) / EL(1, c.nq + 1);
          rh = rh1;
        } else {
          rh = rh2;
        }
      } else {
        rh = rh2;
      }
      c.nwait = c.nq + 2;
      if (rh * c.h == 0.0) goto L400;
      ddscl<N>(c, rh);
      goto L100;
    }
    nfail = 0;
    c.jtask = 2;
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
    ddntl<N, R>(c);
    c.rmax = RMNORM;
    if (c.h == 0.0) goto L400;
    if (c.ier) goto L420;
    goto L100;
  }
  c.nstep += 1;
  for (int j = 0; j <= c.nq; ++j) {
    const double e = EL(j + 1, c.nq);
#pragma unroll
    for (int i = 0; i < N; ++i) c.yh[j][i] = c.yh[j][i] + e * c.s1[i];
  }
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
  if (c.jtask == 0 || c.jtask == 2) {
    rh = 1.0 / NRG_FMAX(uround, BIAS2 * pow(etest / eps, 1.0 / (double)(c.nq + 1)));
    if (rh > TRSHLD) ddscl<N>(c, rh);
  } else if (c.nwait > 1) {
    c.nwait = c.nwait - 1;
    if (c.nwait == 1 && c.nq < kMaxOrd) {
#pragma unroll
      for (int i = 0; i < N; ++i) c.yh[kMaxOrd][i] = c.s1[i];
    }
  } else {
    double rh1, rh2, rh3;
    if (c.nq == 1) {
      rh1 = 0.0;
    } else {
#pragma unroll
      for (int i = 0; i < N; ++i) c.s2[i] = c.yh[c.nq][i] / NRG_FMAX(fabs(c.y[i]), c.ywt[i]);
      double erdn = dnrm2<N>(c.s2) / (TQ(1, c.nq) * sqn);
      rh1 = 1.0 / NRG_FMAX(uround, BIAS1 * pow(erdn / eps, 1.0 / (double)c.nq));
    }
    rh2 = 1.0 / NRG_FMAX(uround, BIAS2 * pow(etest / eps, 1.0 / (double)(c.nq + 1)));
    if (c.nq == kMaxOrd) {
      rh3 = 0.0;
    } else {
#pragma unroll
      for (int i = 0; i < N; ++i)
        c.s2[i] = (c.s1[i] - c.yh[kMaxOrd][i]) / NRG_FMAX(fabs(c.y[i]), c.ywt[i]);
      double erup = dnrm2<N>(c.s2) / (TQ(3, c.nq) * sqn);
      rh3 = 1.0 / NRG_FMAX(uround, BIAS3 * pow(erup / eps, 1.0 / (double)(c.nq + 2)));
    }
    if (rh1 > rh2 && rh1 >= rh3) {
      rh = rh1;
      if (rh <= TRSHLD) goto L380;
      c.nq = c.nq - 1;
      c.rc = c.rc * EL(1, c.nq) / EL(1, c.nq + 1);
    } else if (rh2 >= rh1 && rh2 >= rh3) {
      rh = rh2;
      if (rh <= TRSHLD) goto L380;
    } else {
      rh = rh3;
      if (rh <= TRSHLD) goto L380;
      const double e = EL(c.nq + 1, c.nq);
#pragma unroll
      for (int i = 0; i < N; ++i) c.yh[c.nq + 1][i] = c.s1[i] * e / (double)(c.nq + 1);
      c.nq = c.nq + 1;
      c.rc = c.rc * EL(1, c.nq) / EL(1, c.nq - 1);
    }
    ddscl<N>(c, rh);
    c.rmax = RMNORM;
  L380:
    c.nwait = c.nq + 2;
  }
  return 1;
L400:
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
  return 2;
L410:
  return 3;
L420:
  return 4;
}

// ----------------------------------------------------------- cell driver
enum CellPhase { kPhaseRunning = 0, kPhaseDone = 1 };

// Cell set-up: skip rule, third-body sums, rate constants, DDRIV3 init.
// Returns false when the cell is passed through (outputs already written).
template <int N, int R, typename CS>
__device__ bool cell_begin(CS& c, const StepArgs& a, long cid) {
  const double Tc = a.T[cid];
  const bool active = (Tc >= 305.0) && (a.bc == nullptr || a.bc[cid] == 0);
  if (!active) {
#pragma unroll
    for (int k = 0; k < N; ++k) a.Y_prod[k * a.ld + cid] = 0.0;
    a.E_f_prod[cid] = 0.0;
    if (a.status) a.status[cid] = kCellSkipped;
    return false;
  }
  const double rho = a.rho[cid];
  double yk[N];
#pragma unroll
  for (int k = 0; k < N; ++k) yk[k] = a.Y[k * a.ld + cid];
  for (int r = 0; r < R; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) s = s + yk[k] * rho / c_mech.W[k] * c_mech.eff[r][k];
    c.mc[r] = s;
  }
  rate_constants<N, R>(Tc, c.mc, c.kf, c.kr);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    c.conc_in[k] = yk[k] * rho / c_mech.W[k];
    c.yh[0][k] = c.conc_in[k];
    c.y[k] = c.conc_in[k];
  }
  // ddriv3.f90:930-978 (NSTATE = 1)
  c.tout = a.dt;
  c.t = 0.0;
  double h = (c.tout - c.t) * (1.0 - 4.0 * c_mech.uround);
  c.h = copysign(NRG_FMIN(fabs(h), c_mech.hmax), h);
  c.eps = c_mech.eps;
  c.jtask = 0;
  c.nstep = 0;
  c.nstepl = 0;
  c.jstepl = 0;
  c.nfe = 0;
  c.nje = 0;
  c.nsolve = 0;
  c.convrg = 0;
  c.ier = 0;
  c.refine = 0;
  c.nq = 1;
  return true;
}

// One pass of the DDRIV3 loop (label 260): error weights, accuracy and
// MXSTEP checks, one DDSTP step, and on reaching TOUT the interpolation.
// Returns 0 while running, else a CellStatus.
template <int N, int R, int JAC, typename CS>
__device__ int cell_advance(CS& c, int mxstep) {
#pragma unroll
  for (int i = 0; i < N; ++i) c.ywt[i] = NRG_FMAX(c_mech.ewt, fabs(c.y[i]));
#pragma unroll
  for (int i = 0; i < N; ++i) c.s2[i] = c.y[i] / c.ywt[i];
  double sum = NRG_FMAX(1.0, dnrm2<N>(c.s2) / sqrt((double)N));
  if (c.eps < sum * c_mech.uround) {
    c.eps = sum * c_mech.uround * (1.0 + 10.0 * c_mech.uround);
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
    return kCellOk;  // NSTATE = 4: state at current T returned
  }
  if (c.nstep - c.nstepl == mxstep) {
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
    return kCellMxstep;
  }
  int js = ddstp<N, R, JAC>(c);
  if (js != 1) {
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh[0][i];
    return kCellFatal;
  }
  c.jtask = 1;
  if (c.t < c.tout) return 0;
  // ddntp.f90 K = 0
#pragma unroll
  for (int i = 0; i < N; ++i) c.y[i] = c.yh[c.nq][i];
  const double r = (c.tout - c.t) / c.h;
  for (int jj = 1; jj <= c.nq; ++jj) {
    int j = c.nq - jj;  // 0-based column nq-jj
#pragma unroll
    for (int i = 0; i < N; ++i) c.y[i] = c.yh[j][i] + r * c.y[i];
  }
  return kCellOk;
}

// Energy closure at constant density (the temperature the reference EOS
// would compute after adding the sources: cpm_solver.f90:517,549 ->
// table_approximated_real_gas.f90:404-440 -> calculate_temperature
// thermophysical_properties_class.f90:409-452).
template <int N>
__device__ double temperature_after(double T0, double rho, const double* Y0, const double* dY,
                                    double dE /* E_f_prod*dt/rho */) {
  const double RG = 8.31446261815324;
  double X[N], avg = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) avg = avg + Y0[k] / c_mech.W[k];
  double W0 = 1.0 / avg;
  double e0 = 0.0, h0 = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    X[k] = Y0[k] / c_mech.W[k] * W0;
    e0 = e0 + (d_enthalpy(T0, k) - RG * T0) * X[k];
  }
#pragma unroll
  for (int k = 0; k < N; ++k) h0 = h0 + c_mech.h_ref[k] * X[k];
  double e1 = (e0 - h0) / W0 + dE;
  avg = 0.0;
  double Y1[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    Y1[k] = Y0[k] + dY[k];
    avg = avg + Y1[k] / c_mech.W[k];
  }
  double W1 = 1.0 / avg;
  double hc = 0.0, cp = 0.0;
  double temp = NRG_FMIN(T0, 6000.0);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    X[k] = Y1[k] / c_mech.W[k] * W1;
    hc = hc + c_mech.h_ref[k] * X[k];
    cp = cp + d_cp(temp, k) * X[k];
  }
  const double ei = e1 * W1;
  const double tol = (double)1e-08f;
  for (int it = 0; it < 1000; ++it) {
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) e = e + (d_enthalpy(temp, k) - RG * temp) * X[k];
    double res = (ei - (e - hc)) / cp;
    temp = temp + res;
    if (fabs(res) < tol) break;
  }
  return temp;
}

// Outputs for a finished cell (chemical_kinetics_solver.f90:318-340).
template <int N, typename CS>
__device__ void cell_finish(const CS& c, const StepArgs& a, long cid, int st) {
  const double dt = a.dt;
  double E = 0.0;
  bool finite = true;
  double dYm[N], Y0[N];
  const double rho = a.rho[cid];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double dc = c.y[k] - c.conc_in[k];
    finite = finite && isfinite(dc);
    a.Y_prod[k * a.ld + cid] = dc * c_mech.W[k] / dt;
    a.Y_prod2[k * a.ld + cid] = dc;
    E = E - c_mech.h_ref[k] * dc / dt;
    if (a.T_after) {
      Y0[k] = a.Y[k * a.ld + cid];
      dYm[k] = dc * c_mech.W[k] / dt * dt / rho;
    }
  }
  a.E_f_prod[cid] = E;
  if (a.T_after) a.T_after[cid] = temperature_after<N>(a.T[cid], rho, Y0, dYm, E * dt / rho);
  if (a.status) a.status[cid] = finite ? (uint8_t)st : (uint8_t)kCellNonfinite;
}

}  // namespace nrg
