// Warp-per-cell integrator for the NRG chemistry step (device code).
//
// One warp integrates one cell; the 32 lanes split the work so that control
// flow is identical on every lane (no divergence between cells, which is what
// limits a thread-per-cell integrator: its lanes sit in different branches of
// the step/order logic most of the time):
//   * species rows: lane i < N owns y_i, YWT_i, SAVE1_i, SAVE2_i, FAC_i and
//     row i of the Nordsieck array (registers) and row i of the iteration
//     matrix (shared memory, row-major);
//   * reactions: lane r (r < R, strided by 32) evaluates the rate constants
//     and the net rate of reaction r;
//   * scalars (h, order, error estimates, step decisions) are computed
//     redundantly and identically on all lanes from warp-gathered data.
// The arithmetic is the same SLATEC DDRIV3/DDSTP algorithm as the
// thread-per-cell code in chem_bdf.cuh (see the routine citations there).
#pragma once

#include "chem_bdf.cuh"

namespace nrg {

constexpr unsigned kFullMask = 0xffffffffu;

// Per-warp shared scratch.
template <int N, int R, typename LUT>
struct WarpSmem {
  double z[N];      // RHS input (gathered state)
  double w[N];      // Jacobian-vector input (mixed mode)
  double th_s[N];   // species entropies (cell set-up)
  double th_h[N];   // species enthalpies (cell set-up)
  double q[R];      // net rates
  double kf[R], kr[R];
  LUT a[N][N];      // iteration matrix, row-major: a[i][j] = A(i+1, j+1)
};

// What the out-of-line warp routines need: passed by value, so calling them
// never forces the register-resident cell state to local memory.
template <int N, int R, typename LUT>
struct WarpCtx {
  const DevMech* M;  // block-shared copy of the mechanism tables
  WarpSmem<N, R, LUT>* sm;
  int lane;
};

template <int N, int R, typename LUT>
struct WarpCell : WarpCtx<N, R, LUT> {
  double yh[kMaxOrd + 1];  // Nordsieck row `lane`
  double y, ywt, s1, s2, fac, conc_in;
  double h, t, tout, rc, rmax, trend, eps;  // warp-uniform
  int nq, nwait, jtask, nstep, nfe, nje, nsolve, jstepl, nstepl, convrg, ier;
  unsigned long long piv;
};

// ------------------------------------------------------------ helpers
template <int N>
__device__ __forceinline__ void wgather(double x, double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = __shfl_sync(kFullMask, x, i);
}

template <int N>
__device__ __forceinline__ double wnrm2(double x) {
  double v[N];
  wgather<N>(x, v);
  return dnrm2<N>(v);
}

__device__ __forceinline__ double yh_get(const double (&yh)[kMaxOrd + 1], int j) {
  double r = yh[0];
#pragma unroll
  for (int jj = 1; jj <= kMaxOrd; ++jj)
    if (jj == j) r = yh[jj];
  return r;
}

__device__ __forceinline__ void yh_set(double (&yh)[kMaxOrd + 1], int j, double v) {
#pragma unroll
  for (int jj = 0; jj <= kMaxOrd; ++jj)
    if (jj == j) yh[jj] = v;
}

// First index of the largest value over lanes (IDAMAX tie rule); lanes that
// do not take part pass v = -1.  A NaN ranks below every number of a lane
// that takes part, so (value, index) is a strict total order and every lane
// ends with the same participating index.
__device__ __forceinline__ int warp_argmax(double v, int idx, double* vmax) {
  if (v != v) v = -0.5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(kFullMask, v, o);
    const int i2 = __shfl_xor_sync(kFullMask, idx, o);
    if (v2 > v || (v2 == v && i2 < idx)) {
      v = v2;
      idx = i2;
    }
  }
  if (vmax) *vmax = v;
  return idx;
}

// ------------------------------------------------------ rates and RHS
// Rate constants of the reactions owned by this lane (calculate_rate_constants,
// chemical_kinetics_solver.f90:360-493); third-body concentration folded in.
template <int N, int R, typename LUT>
__device__ __noinline__ void warp_rate_constants(const WarpCtx<N, R, LUT> c, double Tin, double ci) {
  const double RG = 8.31446261815324, PATM = 101325.0;
  double yc[N];
  wgather<N>(ci, yc);
  const double T = NRG_FMIN(Tin, 10000.0);
  if (c.lane < N) {
    const double logt = log(NRG_FMIN(T, 6000.0));
    const double t = NRG_FMIN(T, 6000.0);
    const double* ak = c.M->a[c.lane][nasa_set(t)];
    double sv = ak[4] / 4.0;
    sv = sv * t + ak[3] / 3.0;
    sv = sv * t + ak[2] / 2.0;
    sv = sv * t + ak[1] / 1.0;
    c.sm->th_s[c.lane] = sv * t + ak[6] + ak[0] * logt;
    double hv = ak[4] / 5.0;
    hv = hv * t + ak[3] / 4.0;
    hv = hv * t + ak[2] / 3.0;
    hv = hv * t + ak[1] / 2.0;
    hv = hv * t + ak[0] / 1.0;
    hv = hv + ak[5] / t;
    c.sm->th_h[c.lane] = hv * t;
  }
  __syncwarp();
  const double conc_ref = PATM / RG / T;
  for (int r = c.lane; r < R; r += 32) {
    double mc = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) mc = mc + yc[k] * c.M->eff_t[k][r];
    double d_s = 0.0, d_h = 0.0;
    bool m_left = false, m_right = false;
    for (int i = 0; i < c.M->nr[r]; ++i) {
      const int sp = c.M->right[r][i];
      if (sp < 0) { m_right = true; continue; }
      d_s = d_s + c.sm->th_s[sp];
      d_h = d_h + c.sm->th_h[sp];
    }
    for (int i = 0; i < c.M->nl[r]; ++i) {
      const int sp = c.M->left[r][i];
      if (sp < 0) { m_left = true; continue; }
      d_s = d_s - c.sm->th_s[sp];
      d_h = d_h - c.sm->th_h[sp];
    }
    const int type = c.M->type[r];
    const double kinf = c.M->A[r] * pow(T, c.M->beta[r]) * exp(-(c.M->E[r] / RG / T));
    double k = kinf;
    if (type == 2 || type == 3 || type == 7) {
      const double k0 = c.M->A_low[r] * pow(T, c.M->beta_low[r]) * exp(-(c.M->E_low[r] / RG / T));
      const double rp = k0 * mc / kinf;
      k = kinf * (rp / (1.0 + rp));
      if (type == 3) {
        const double al = c.M->troe[r][0];
        const double Fc = (1.0 - al) * exp(-(T / c.M->troe[r][1])) + al * exp(-(T / c.M->troe[r][2])) +
                          exp(-(c.M->troe[r][3] / T));
        const double lf = log10(Fc);
        const double cc = -0.4 - 0.67 * lf;
        const double nn = 0.75 - 1.27 * lf;
        double blend;
        if (rp != 0.0) {
          const double lr = log10(rp);
          const double x = (lr + cc) / (nn - 0.14 * (lr + cc));
          blend = pow(Fc, 1.0 / (1.0 + x * x));
        } else {
          blend = pow(Fc, -1.0 / 0.14);
        }
        k = k * blend;
      }
    }
    double kr = 0.0;
    if (type < 5) {
      const double Kp = exp(d_s / RG - d_h / RG / T);
      kr = k / (Kp * int_pow(conc_ref, c.M->dnu[r]));
    }
    c.sm->kf[r] = m_left ? k * mc : k;
    c.sm->kr[r] = m_right ? kr * mc : kr;
  }
  __syncwarp();
}

// zd_lane = dC_lane/dt at the lane-distributed state x (fun,
// chemical_kinetics_solver.f90:495-540), summed per species in reaction
// order from the net rates.
template <int N, int R, typename LUT>
__device__ __noinline__ double warp_rhs(const WarpCtx<N, R, LUT> c, double x) {
  __syncwarp();
  if (c.lane < N) c.sm->z[c.lane] = x;
  __syncwarp();
  for (int r = c.lane; r < R; r += 32) {
    double f = c.sm->kf[r];
    for (int i = 0; i < c.M->nl[r]; ++i) {
      const int sp = c.M->left[r][i];
      if (sp >= 0) f = f * c.sm->z[sp];
    }
    double b = c.sm->kr[r];
    for (int i = 0; i < c.M->nr[r]; ++i) {
      const int sp = c.M->right[r][i];
      if (sp >= 0) b = b * c.sm->z[sp];
    }
    c.sm->q[r] = f - b;
  }
  __syncwarp();
  double acc = 0.0;
  if (c.lane < N) {
    const int n = c.M->sp_n[c.lane];
    for (int u = 0; u < n; ++u) {
      const int e = c.M->sp_list[u][c.lane];
      const double q = c.sm->q[e >> 1];
      acc = (e & 1) ? acc + q : acc - q;
    }
  }
  return acc;
}

// d(net rate of reaction r)/dz_sp for factor position p on one side, at z.
template <int N, int R, typename LUT>
__device__ __forceinline__ double rate_partial(const WarpCtx<N, R, LUT>& c, int r, int side, int p) {
  const int cnt = side ? c.M->nr[r] : c.M->nl[r];
  double d = side ? c.sm->kr[r] : c.sm->kf[r];
  for (int qq = 0; qq < cnt; ++qq) {
    if (qq == p) continue;
    const int sq = side ? c.M->right[r][qq] : c.M->left[r][qq];
    if (sq >= 0) d = d * c.sm->z[sq];
  }
  return side ? -d : d;
}

// Row `lane` of I + factor * J (J = dZdot/dZ, analytic) into the shared matrix.
template <int N, int R, typename LUT>
__device__ __noinline__ void warp_analytic_matrix(const WarpCtx<N, R, LUT> c, double y, double factor) {
  __syncwarp();
  if (c.lane < N) c.sm->z[c.lane] = y;
  __syncwarp();
  if (c.lane < N) {
    const int i = c.lane;
    double row[N];
#pragma unroll
    for (int j = 0; j < N; ++j) row[j] = 0.0;
    const int n = c.M->sp_n[i];
    for (int u = 0; u < n; ++u) {
      const int e = c.M->sp_list[u][i];
      const int r = e >> 1;
      const double sgn = (e & 1) ? factor : -factor;
      for (int side = 0; side < 2; ++side) {
        const int cnt = side ? c.M->nr[r] : c.M->nl[r];
        for (int p = 0; p < cnt; ++p) {
          const int sp = side ? c.M->right[r][p] : c.M->left[r][p];
          if (sp < 0) continue;
          const double d = sgn * rate_partial(c, r, side, p);
#pragma unroll
          for (int j = 0; j < N; ++j)
            if (j == sp) row[j] += d;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < N; ++j) c.sm->a[i][j] = (LUT)(row[j] + (j == i ? 1.0 : 0.0));
  }
  __syncwarp();
}

// (J v)_lane with v in sm->w and the state in sm->z (mixed-mode residual).
template <int N, int R, typename LUT>
__device__ __noinline__ double warp_jac_vec(const WarpCtx<N, R, LUT> c) {
  __syncwarp();
  for (int r = c.lane; r < R; r += 32) {
    double dq = 0.0;
    for (int side = 0; side < 2; ++side) {
      const int cnt = side ? c.M->nr[r] : c.M->nl[r];
      for (int p = 0; p < cnt; ++p) {
        const int sp = side ? c.M->right[r][p] : c.M->left[r][p];
        if (sp < 0) continue;
        dq = dq + rate_partial(c, r, side, p) * c.sm->w[sp];
      }
    }
    c.sm->q[r] = dq;
  }
  __syncwarp();
  double acc = 0.0;
  if (c.lane < N) {
    const int n = c.M->sp_n[c.lane];
    for (int u = 0; u < n; ++u) {
      const int e = c.M->sp_list[u][c.lane];
      const double q = c.sm->q[e >> 1];
      acc = (e & 1) ? acc + q : acc - q;
    }
  }
  return acc;
}

// dgefa.f90:60-117 on the shared row-major matrix, rows spread over lanes.
template <int N, int R, typename LUT>
__device__ __noinline__ unsigned long long warp_dgefa(const WarpCtx<N, R, LUT> c, int* info_out) {
  int info = 0;
  unsigned long long piv = 0;
  const int i = c.lane;
  LUT(*a)[N] = c.sm->a;
  __syncwarp();
#pragma unroll 1
  for (int k = 0; k < N - 1; ++k) {
    const double v = (i >= k && i < N) ? (double)fabs(a[i][k]) : -1.0;
    int l = warp_argmax(v, i, nullptr);
    l = l < k ? k : (l > N - 1 ? N - 1 : l);
    piv |= (unsigned long long)l << (4 * k);
    if (a[l][k] == (LUT)0) {
      info = k + 1;
      continue;
    }
    __syncwarp();
    if (l != k && i >= k && i < N) {  // lane = column for the row swap
      const LUT t = a[l][i];
      a[l][i] = a[k][i];
      a[k][i] = t;
    }
    __syncwarp();
    const LUT t = (LUT)-1 / a[k][k];
    if (i > k && i < N) a[i][k] = t * a[i][k];
    __syncwarp();
    if (i > k && i < N) {
      const LUT m = a[i][k];
      for (int j = k + 1; j < N; ++j) {
        const LUT tj = a[k][j];
        if (tj != (LUT)0) a[i][j] = a[i][j] + tj * m;
      }
    }
    __syncwarp();
  }
  piv |= (unsigned long long)(N - 1) << (4 * (N - 1));
  if (a[N - 1][N - 1] == (LUT)0) info = N;
  *info_out = info;
  return piv;
}

// dgesl.f90:71-131 (JOB = 0) on a lane-distributed right-hand side.
template <int N, int R, typename LUT>
__device__ __forceinline__ double warp_dgesl(const WarpCell<N, R, LUT>& c, double b) {
  const int i = c.lane;
  const LUT(*a)[N] = c.sm->a;
#pragma unroll
  for (int k = 0; k < N - 1; ++k) {
    const int l = (int)((c.piv >> (4 * k)) & 15ull);
    const double t = __shfl_sync(kFullMask, b, l);
    const double bk = __shfl_sync(kFullMask, b, k);
    if (i == l) b = bk;
    if (i == k) b = t;
    if (t != 0.0 && i > k && i < N) b = b + t * (double)a[i][k];
  }
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    if (i == k) b = b / (double)a[k][k];
    const double t = -__shfl_sync(kFullMask, b, k);
    if (t != 0.0 && i < k) b = b + t * (double)a[i][k];
  }
  return b;
}

// ------------------------------------------------------ SLATEC pieces
template <int N, int R, typename LUT>
__device__ __forceinline__ void warp_ddpsc(WarpCell<N, R, LUT>& c, int ksgn) {
  const int nq = c.nq;
#pragma unroll
  for (int j1 = 1; j1 <= kMaxOrd; ++j1) {
    if (j1 > nq) break;
#pragma unroll
    for (int j = kMaxOrd; j >= 1; --j)
      if (j <= nq && j >= j1) c.yh[j - 1] = ksgn > 0 ? c.yh[j - 1] + c.yh[j] : c.yh[j - 1] - c.yh[j];
  }
}

template <int N, int R, typename LUT>
__device__ __forceinline__ void warp_ddscl(WarpCell<N, R, LUT>& c, double rh) {
  const double hmax = c.M->hmax;
  if (c.h < 1.0) {
    const double ah = fabs(c.h);
    rh = NRG_FMIN(NRG_FMIN(ah * rh, ah * c.rmax), hmax) / ah;
  } else {
    rh = NRG_FMIN(NRG_FMIN(rh, c.rmax), hmax / fabs(c.h));
  }
  double r1 = 1.0;
#pragma unroll
  for (int j = 1; j <= kMaxOrd; ++j) {
    if (j <= c.nq) {
      r1 = r1 * rh;
      c.yh[j] = c.yh[j] * r1;
    }
  }
  c.h = c.h * rh;
  c.rc = c.rc * rh;
}

template <int N, int R, typename LUT>
__device__ void warp_ddntl(WarpCell<N, R, LUT>& c) {
  c.ier = 0;
  if (c.jtask == 0) c.rmax = 10000.0;
  c.rc = 0.0;
  c.convrg = 0;
  c.trend = 1.0;
  c.nq = 1;
  c.nwait = 3;
  c.s2 = warp_rhs<N, R, LUT>(c, c.y);
  c.nfe += 1;
  c.s1 = c.s2 / NRG_FMAX(1.0, c.ywt);
  const double sum = wnrm2<N>(c.s1) / sqrt((double)N);
  if (sum > c.eps / fabs(c.h)) c.h = copysign(c.eps / sum, c.h);
  c.yh[1] = c.h * c.s2;
  c.fac = c.M->sqrt_uround;
}

template <int N, int R, int JAC, typename LUT>
__device__ void warp_ddpst(WarpCell<N, R, LUT>& c) {
  c.nje += 1;
  c.ier = 0;
  const double el1h = EL(1, c.nq) * c.h;
  if (JAC == kJacFD) {
    const double FACMAX = 0.5, BU = 0.5;
    const double br = c.M->br, bl = c.M->bl, bp = c.M->bp, facmin = c.M->facmin;
#pragma unroll 1
    for (int j = 0; j < N; ++j) {
      const double yj = __shfl_sync(kFullMask, c.y, j);
      const double ys = NRG_FMAX(fabs(__shfl_sync(kFullMask, c.ywt, j)), fabs(yj));
      double fj = __shfl_sync(kFullMask, c.fac, j);
      const double sg = (c.nq == 1) ? __shfl_sync(kFullMask, c.s2, j) : __shfl_sync(kFullMask, c.yh[2], j);
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
      dy = copysign(dy, sg);
      dy = (yj + dy) - yj;
      const double f1 = warp_rhs<N, R, LUT>(c, c.lane == j ? yj + dy : c.y);
      const double factor = -(el1h / dy);
      if (c.lane < N) c.sm->a[c.lane][j] = (LUT)((f1 - c.s2) * factor);
      const double di = c.lane < N ? fabs(c.s2 - f1) : -1.0;
      double diff;
      int imax = warp_argmax(di, c.lane, &diff);
      imax = imax > N - 1 ? N - 1 : imax;
      const double s2m = fabs(__shfl_sync(kFullMask, c.s2, imax));
      const double s1m = fabs(__shfl_sync(kFullMask, f1, imax));
      if (NRG_FMIN(s2m, s1m) > 0.0) {
        const double scale = NRG_FMAX(s2m, s1m);
        if (diff > BU * scale) fj = NRG_FMAX(facmin, fj * 0.5);
        else if (br * scale <= diff && diff <= bl * scale) fj = NRG_FMIN(fj * 2.0, FACMAX);
        else if (diff < br * scale) fj = NRG_FMIN(bp * fj, FACMAX);
      }
      if (c.lane == j) c.fac = fj;
    }
    c.nfe += N;
    __syncwarp();
    if (c.lane < N) c.sm->a[c.lane][c.lane] += (LUT)1;
    __syncwarp();
  } else {
    warp_analytic_matrix<N, R, LUT>(c, c.y, -el1h);
  }
  int info = 0;
  c.piv = warp_dgefa<N, R, LUT>(c, &info);
  if (info != 0) c.ier = 1;
}

template <int N, int R, typename LUT>
__device__ double warp_ddcor(WarpCell<N, R, LUT>& c) {
  const double b = c.h * c.s2 - c.yh[1] - c.s1;
  double x = warp_dgesl(c, b);
  if (sizeof(LUT) == 4) {
    const double el1h = EL(1, c.nq) * c.h;
    __syncwarp();
    if (c.lane < N) {
      c.sm->z[c.lane] = c.y;
      c.sm->w[c.lane] = x;
    }
    const double jx = warp_jac_vec<N, R, LUT>(c);
    const double r = b - (x - el1h * jx);
    x = x + warp_dgesl(c, r);
    c.nsolve += 1;
  }
  c.nsolve += 1;
  c.s1 = c.s1 + x;
  c.s2 = x / NRG_FMAX(fabs(c.y), c.ywt);
  return wnrm2<N>(c.s2) / sqrt((double)N);
}

// Weighted norm of a lane vector v / max(|y|, YWT).
template <int N, int R, typename LUT>
__device__ __forceinline__ double wnorm(const WarpCell<N, R, LUT>& c, double v) {
  return wnrm2<N>(v / NRG_FMAX(fabs(c.y), c.ywt));
}

template <int N, int R, int JAC, typename LUT>
__device__ int warp_ddstp(WarpCell<N, R, LUT>& c) {
  const double BIAS1 = 1.3, BIAS2 = 1.2, BIAS3 = 1.4, RCTEST = 0.3, RMFAIL = 2.0, RMNORM = 10.0,
               TRSHLD = 1.0;
  const int MXFAIL = 3, MXITER = 3, MXTRY = 50, NDJSTP = 10;
  const double uround = c.M->uround;
  const double eps = c.eps;
  const double sqn = sqrt((double)N);
  int ntry = 0, nfail = 0, iter = 0;
  bool evaljc;
  double told = c.t, ctest = 0.0, d = 0.0, d1 = 0.0, etest, rh;
  if (c.jtask <= 0) {
    warp_ddntl(c);
    if (c.h == 0.0) goto L400;
    if (c.ier) goto L420;
  }
L100:
  ntry = ntry + 1;
  if (ntry > MXTRY) goto L410;
  c.t = c.t + c.h;
  warp_ddpsc(c, 1);
  evaljc = (fabs(c.rc - 1.0) > RCTEST) || (c.nstep >= c.jstepl + NDJSTP);
L110:
  iter = 0;
  c.y = c.yh[0];
  c.s2 = warp_rhs<N, R, LUT>(c, c.y);
  c.nfe += 1;
  if (evaljc || c.ier) {
    warp_ddpst<N, R, JAC>(c);
    if (c.ier) goto L160;
    c.convrg = 0;
    c.rc = 1.0;
    c.jstepl = c.nstep;
  }
  c.s1 = 0.0;
L130:
  d = warp_ddcor(c);
  if (iter > 0) c.trend = NRG_FMAX(0.9 * c.trend, d / d1);
  d1 = d;
  ctest = NRG_FMIN(2.0 * c.trend, 1.0) * d;
  if (ctest <= eps) goto L170;
  iter = iter + 1;
  if (iter < MXITER) {
    c.y = c.yh[0] + EL(1, c.nq) * c.s1;
    c.s2 = warp_rhs<N, R, LUT>(c, c.y);
    c.nfe += 1;
    goto L130;
  }
  if (c.convrg) {
    evaljc = true;
    goto L110;
  }
L160:
  c.t = told;
  warp_ddpsc(c, -1);
  c.nwait = c.nq + 2;
  if (c.jtask != 0 && c.jtask != 2) c.rmax = RMFAIL;
  rh = (iter == 0) ? 0.3 : 0.9 * npow(eps / ctest, 0.2);
  if (rh * c.h == 0.0) goto L400;
  warp_ddscl(c, rh);
  goto L100;
L170:
  c.convrg = 1;
  etest = wnorm(c, c.s1) / (TQ(2, c.nq) * sqn);
  if (etest > eps) {
    c.t = told;
    warp_ddpsc(c, -1);
    nfail = nfail + 1;
    if (nfail < MXFAIL || c.nq == 1) {
      if (c.jtask != 0 && c.jtask != 2) c.rmax = RMFAIL;
      const double rh2 = 1.0 / (BIAS2 * npow(etest / eps, 1.0 / (double)(c.nq + 1)));
      if (c.nq > 1) {
        const double erdn = wnorm(c, yh_get(c.yh, c.nq)) / (TQ(1, c.nq) * sqn);
        const double rh1 = 1.0 / NRG_FMAX(1.0, BIAS1 * npow(erdn / eps, 1.0 / (double)c.nq));
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
      warp_ddscl(c, rh);
      goto L100;
    }
    nfail = 0;
    c.jtask = 2;
    c.y = c.yh[0];
    warp_ddntl(c);
    c.rmax = RMNORM;
    if (c.h == 0.0) goto L400;
    if (c.ier) goto L420;
    goto L100;
  }
  c.nstep += 1;
#pragma unroll
  for (int j = 0; j <= kMaxOrd; ++j)
    if (j <= c.nq) c.yh[j] = c.yh[j] + EL(j + 1, c.nq) * c.s1;
  c.y = c.yh[0];
  if (c.jtask == 0 || c.jtask == 2) {
    rh = 1.0 / NRG_FMAX(uround, BIAS2 * npow(etest / eps, 1.0 / (double)(c.nq + 1)));
    if (rh > TRSHLD) warp_ddscl(c, rh);
  } else if (c.nwait > 1) {
    c.nwait = c.nwait - 1;
    if (c.nwait == 1 && c.nq < kMaxOrd) c.yh[kMaxOrd] = c.s1;
  } else {
    double rh1, rh2, rh3;
    if (c.nq == 1) {
      rh1 = 0.0;
    } else {
      const double erdn = wnorm(c, yh_get(c.yh, c.nq)) / (TQ(1, c.nq) * sqn);
      rh1 = 1.0 / NRG_FMAX(uround, BIAS1 * npow(erdn / eps, 1.0 / (double)c.nq));
    }
    rh2 = 1.0 / NRG_FMAX(uround, BIAS2 * npow(etest / eps, 1.0 / (double)(c.nq + 1)));
    if (c.nq == kMaxOrd) {
      rh3 = 0.0;
    } else {
      const double erup = wnorm(c, c.s1 - c.yh[kMaxOrd]) / (TQ(3, c.nq) * sqn);
      rh3 = 1.0 / NRG_FMAX(uround, BIAS3 * npow(erup / eps, 1.0 / (double)(c.nq + 2)));
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
      yh_set(c.yh, c.nq + 1, c.s1 * EL(c.nq + 1, c.nq) / (double)(c.nq + 1));
      c.nq = c.nq + 1;
      c.rc = c.rc * EL(1, c.nq) / EL(1, c.nq - 1);
    }
    warp_ddscl(c, rh);
    c.rmax = RMNORM;
  L380:
    c.nwait = c.nq + 2;
  }
  return 1;
L400:
  c.y = c.yh[0];
  return 2;
L410:
  return 3;
L420:
  return 4;
}

// ----------------------------------------------------------- cell driver
template <int N, int R, typename LUT>
__device__ bool warp_cell_begin(WarpCell<N, R, LUT>& c, const StepArgs& a, long cid) {
  const double Tc = a.T[cid];
  if (!reference_cell_active(Tc, a.bc, cid)) {
    if (c.lane == 0) write_skipped_cell(a, cid, N, Tc);
    return false;
  }
  const double rho = a.rho[cid];
  const double yk = c.lane < N ? a.Y[c.lane * a.ld + cid] : 0.0;
  const double ci = c.lane < N ? yk * rho / c.M->W[c.lane] : 0.0;
  warp_rate_constants<N, R, LUT>(c, Tc, ci);
  c.conc_in = ci;
  c.y = ci;
#pragma unroll
  for (int j = 0; j <= kMaxOrd; ++j) c.yh[j] = 0.0;
  c.yh[0] = ci;
  c.ywt = 0.0;
  c.s1 = 0.0;
  c.s2 = 0.0;
  c.fac = 0.0;
  c.tout = a.dt_cells ? a.dt_cells[cid] : a.dt;
  c.t = 0.0;
  const double h = (c.tout - c.t) * (1.0 - 4.0 * c.M->uround);
  c.h = copysign(NRG_FMIN(fabs(h), c.M->hmax), h);
  c.eps = a.eps > 0.0 ? a.eps : c.M->eps;
  c.jtask = 0;
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
  c.piv = 0;
  return true;
}

template <int N, int R, int JAC, typename LUT>
__device__ int warp_cell_advance(WarpCell<N, R, LUT>& c, int mxstep) {
  c.ywt = NRG_FMAX(c.M->ewt, fabs(c.y));
  const double sum = NRG_FMAX(1.0, wnrm2<N>(c.y / c.ywt) / sqrt((double)N));
  if (c.eps < sum * c.M->uround) {
    c.eps = sum * c.M->uround * (1.0 + 10.0 * c.M->uround);
    c.y = c.yh[0];
    return kCellOk;
  }
  if (c.nstep - c.nstepl == mxstep) {
    c.y = c.yh[0];
    return kCellMxstep;
  }
  const int js = warp_ddstp<N, R, JAC>(c);
  if (js != 1) {
    c.y = c.yh[0];
    return kCellFatal;
  }
  c.jtask = 1;
  if (c.t < c.tout) return 0;
  const double r = (c.tout - c.t) / c.h;
  double y = yh_get(c.yh, c.nq);
#pragma unroll
  for (int j = kMaxOrd - 1; j >= 0; --j)
    if (j < c.nq) y = c.yh[j] + r * y;
  c.y = y;
  return kCellOk;
}

template <int N, int R, typename LUT>
__device__ void warp_cell_finish(const WarpCell<N, R, LUT>& c, const StepArgs& a, long cid, int st) {
  const double dt = c.tout;
  const double rho = a.rho[cid];
  const double dc = c.y - c.conc_in;
  const double yp = c.lane < N ? dc * c.M->W[c.lane] / dt : 0.0;
  if (c.lane < N) {
    a.Y_prod[c.lane * a.ld + cid] = yp;
    a.Y_prod2[c.lane * a.ld + cid] = dc;
  }
  double dcv[N];
  wgather<N>(dc, dcv);
  double E = 0.0;
  bool finite = true;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    finite = finite && isfinite(dcv[k]);
    E = E - c.M->h_ref[k] * dcv[k] / dt;
  }
  if (a.T_after) {
    const double y0 = c.lane < N ? a.Y[c.lane * a.ld + cid] : 0.0;
    double Y0[N], dYm[N];
    wgather<N>(y0, Y0);
    wgather<N>(yp * dt / rho, dYm);
    const double Ta = temperature_after<N>(a.T[cid], Y0, dYm, E * dt / rho);
    if (c.lane == 0) a.T_after[cid] = Ta;
  }
  if (c.lane == 0) {
    a.E_f_prod[cid] = E;
    if (a.status) a.status[cid] = finite ? (uint8_t)st : (uint8_t)kCellNonfinite;
  }
}

}  // namespace nrg
