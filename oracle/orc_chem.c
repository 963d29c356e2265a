/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle.h; parity unpinned).
 *
 * Plain-C restatement of the reference chemistry step and of the SLATEC
 * DDRIV3 path it drives (MINT=2, MITER=2, IMPL=0, IERROR=3, NTASK=1,
 * NROOT=0, MXORD=5).  Every routine keeps the reference's operation order so
 * that the results are the reference's up to the system libm.  Fortran
 * 1-based indexing is kept through the YH/DFDY/EL/TQ macros.
 *
 * Compile WITHOUT -ffast-math and without FMA contraction (-ffp-contract=off).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

#define R_GASE_J 8.31446261815324    /* global_data.f90:36 */
#define T_REF 298.15                 /* global_data.f90:38 */
#define P_ATM 101325.0               /* global_data.f90:39 */
#define T_CEIL 6000.0                /* global_data.f90:44 (single literal 6000.0) */

#define FMAX2(a, b) ((a) >= (b) ? (a) : (b))
#define FMIN2(a, b) ((a) <= (b) ? (a) : (b))

/* ------------------------------------------------------------- thermo */
/* thermophysical_properties_class.f90:876-881 */
static double clip_temperature(double T) { return FMIN2(T, T_CEIL); }

/* thermophysical_properties_class.f90:225-242 */
double orc_specie_cp(const orc_mech *m, double T, int k) {
    double temp = clip_temperature(T);
    int s = temp >= 1000.0 ? 1 : 0;
    const double *a = m->a_coeffs[k][s];
    double cp = a[4];
    for (int i = 4; i >= 1; i--) cp = cp * temp + a[i - 1];
    return cp;
}

/* thermophysical_properties_class.f90:244-264 */
double orc_specie_enthalpy(const orc_mech *m, double T, int k) {
    double temp = clip_temperature(T);
    int s = temp >= 1000.0 ? 1 : 0;
    const double *a = m->a_coeffs[k][s];
    double h = a[4] / 5.0;
    for (int i = 4; i >= 1; i--) h = h * temp + a[i - 1] / (double)i;
    h = h + a[5] / temp;
    h = h * temp;
    return h;
}

/* thermophysical_properties_class.f90:266-286 */
double orc_specie_entropy(const orc_mech *m, double T, int k) {
    double temp = clip_temperature(T);
    int s = temp >= 1000.0 ? 1 : 0;
    const double *a = m->a_coeffs[k][s];
    double sm = a[4] / 4.0;
    for (int i = 4; i >= 2; i--) sm = sm * temp + a[i - 1] / (double)(i - 1);
    sm = sm * temp + a[6] + a[0] * log(temp);
    return sm;
}

/* thermophysical_properties_class.f90:288-300 */
static double specie_internal_energy(const orc_mech *m, double T, int k) {
    return orc_specie_enthalpy(m, T, k) - R_GASE_J * T;
}

/* thermophysical_properties_class.f90:303-359 */
static double mixture_cp(const orc_mech *m, double T, const double *X) {
    double cp = 0.0;
    for (int k = 0; k < m->n_species; k++) cp = cp + orc_specie_cp(m, T, k) * X[k];
    return cp;
}
static double mixture_enthalpy(const orc_mech *m, double T, const double *X) {
    double h = 0.0;
    for (int k = 0; k < m->n_species; k++) h = h + orc_specie_enthalpy(m, T, k) * X[k];
    return h;
}
static double mixture_internal_energy(const orc_mech *m, double T, const double *X) {
    double e = 0.0;
    for (int k = 0; k < m->n_species; k++) e = e + specie_internal_energy(m, T, k) * X[k];
    return e;
}

/* thermophysical_properties_class.f90:409-452 */
static double calculate_temperature(const orc_mech *m, double temperature, double e_i,
                                    const double *X) {
    double temp = clip_temperature(temperature);
    const int max_iter = 1000;
    const double eps = (double)1e-08f; /* single-precision literal */
    double h_const = mixture_enthalpy(m, T_REF, X);
    double cp = mixture_cp(m, temp, X);
    for (int iter = 1; iter <= max_iter; iter++) {
        double e_int = mixture_internal_energy(m, temp, X) - h_const;
        double residual = (e_i - e_int) / cp;
        temp = temp + residual;
        if (fabs(residual) < eps) break;
    }
    return temp;
}

/* ------------------------------------------------------ rate constants */
/* chemical_kinetics_solver.f90:360-493 */
void orc_rate_constants(const orc_mech *m, double Tin, const double *mix_conc,
                        double *kf, double *kr) {
    const int N = m->n_species;
    double s[ORC_NMAX], h[ORC_NMAX];
    double T = FMIN2(Tin, 10000.0);
    for (int k = 0; k < N; k++) {
        s[k] = orc_specie_entropy(m, T, k);
        h[k] = orc_specie_enthalpy(m, T, k);
    }
    for (int r = 0; r < m->n_reactions; r++) {
        double d_s = 0.0, d_h = 0.0, d_nu;
        for (int i = 2; i <= m->coeffs[1][r][0] + 1; i++) {
            int sp = m->coeffs[1][r][i - 1];
            if (sp == N + 1) continue;
            d_s = d_s + s[sp - 1];
            d_h = d_h + h[sp - 1];
        }
        for (int i = 2; i <= m->coeffs[0][r][0] + 1; i++) {
            int sp = m->coeffs[0][r][i - 1];
            if (sp == N + 1) continue;
            d_s = d_s - s[sp - 1];
            d_h = d_h - h[sp - 1];
        }
        d_nu = (double)(m->coeffs[1][r][0] - m->coeffs[0][r][0]);
        double Kp, Kc, k0, kinf, rp;
        switch (m->reaction_type[r]) {
        case 0:
        case 1:
            kf[r] = m->A[r] * pow(T, m->beta[r]) * exp(-(m->E_act[r] / R_GASE_J / T));
            Kp = exp(d_s / R_GASE_J - d_h / R_GASE_J / T);
            Kc = Kp * pow(P_ATM / R_GASE_J / T, d_nu);
            kr[r] = kf[r] / Kc;
            break;
        case 2:
            k0 = m->A_low[r] * pow(T, m->beta_low[r]) * exp(-(m->E_act_low[r] / R_GASE_J / T));
            kinf = m->A[r] * pow(T, m->beta[r]) * exp(-(m->E_act[r] / R_GASE_J / T));
            rp = k0 * mix_conc[r] / kinf;
            kf[r] = kinf * (rp / (1.0 + rp));
            Kp = exp(d_s / R_GASE_J - d_h / R_GASE_J / T);
            Kc = Kp * pow(P_ATM / R_GASE_J / T, d_nu);
            kr[r] = kf[r] / Kc;
            break;
        case 3: {
            k0 = exp(-(m->E_act_low[r] / R_GASE_J / T));
            kinf = exp(-(m->E_act[r] / R_GASE_J / T));
            k0 = m->A_low[r] * pow(T, m->beta_low[r]) * k0;
            kinf = m->A[r] * pow(T, m->beta[r]) * kinf;
            rp = k0 * mix_conc[r] / kinf;
            const double *tc = m->troe[r];
            double F_cent = (1.0 - tc[0]) * exp(-(T / tc[1])) + tc[0] * exp(-(T / tc[2])) +
                            exp(-(tc[3] / T));
            double c = -0.4 - 0.67 * log10(F_cent);
            double n = 0.75 - 1.27 * log10(F_cent);
            double d = 0.14;
            double blend;
            if (rp != 0.0) {
                double x = (log10(rp) + c) / (n - d * (log10(rp) + c));
                blend = pow(F_cent, 1.0 / (1.0 + x * x));
            } else {
                blend = pow(F_cent, -1.0 / d);
            }
            kf[r] = kinf * (rp / (1.0 + rp)) * blend;
            Kp = exp(d_s / R_GASE_J - d_h / R_GASE_J / T);
            Kc = Kp * pow(P_ATM / R_GASE_J / T, d_nu);
            kr[r] = kf[r] / Kc;
            break;
        }
        case 4:
            break; /* duplicate: the reference leaves the previous cell's value */
        case 5:
        case 6:
            kf[r] = m->A[r] * pow(T, m->beta[r]) * exp(-(m->E_act[r] / R_GASE_J / T));
            kr[r] = 0.0;
            break;
        case 7:
            k0 = m->A_low[r] * pow(T, m->beta_low[r]) * exp(-(m->E_act_low[r] / R_GASE_J / T));
            kinf = m->A[r] * pow(T, m->beta[r]) * exp(-(m->E_act[r] / R_GASE_J / T));
            rp = k0 * mix_conc[r] / kinf;
            kf[r] = kinf * (rp / (1.0 + rp));
            kr[r] = 0.0;
            break;
        }
    }
}

/* chemical_kinetics_solver.f90:495-540 */
void orc_rhs(const orc_mech *m, const double *kf, const double *kr,
             const double *mix_conc, const double *Z, double *Zdot) {
    const int N = m->n_species;
    for (int k = 0; k < N; k++) Zdot[k] = 0.0;
    for (int r = 0; r < m->n_reactions; r++) {
        const int *lc = m->coeffs[0][r], *rc = m->coeffs[1][r];
        double fwd = kf[r];
        for (int i = 2; i <= lc[0] + 1; i++) {
            if (lc[i - 1] == N + 1) fwd = fwd * mix_conc[r];
            else fwd = fwd * Z[lc[i - 1] - 1];
        }
        double rev = kr[r];
        for (int i = 2; i <= rc[0] + 1; i++) {
            if (rc[i - 1] == N + 1) rev = rev * mix_conc[r];
            else rev = rev * Z[rc[i - 1] - 1];
        }
        for (int k = 1; k <= N; k++) {
            for (int i = 2; i <= lc[0] + 1; i++)
                if (lc[i - 1] == k) Zdot[k - 1] = Zdot[k - 1] - fwd + rev;
            for (int i = 2; i <= rc[0] + 1; i++)
                if (rc[i - 1] == k) Zdot[k - 1] = Zdot[k - 1] - rev + fwd;
        }
    }
}

/* ------------------------------------------------------------- SLATEC */
#define NM ORC_NMAX
#define MAXORD 5

typedef struct {
    const orc_mech *m;
    const double *kf, *kr, *mc;
} rhs_ctx;

typedef struct {
    double yh[NM * (MAXORD + 1)];
    double dfdy[NM * NM];
    double ywt[NM], save1[NM], save2[NM], fac[NM];
    double el[13 * 12], tq[3 * 12];
    int ipvt[NM];
    double h, hmax, hold, rc, rmax, trend, t, avgh, avgord, hused, uround;
    int nq, nwait, jtask, nstep, nfe, nje, jstepl, nqused, convrg, ier;
} work_t;

#define YH(i, j) w->yh[((j)-1) * N + ((i)-1)]
#define DFDY(i, j) w->dfdy[((j)-1) * N + ((i)-1)]
#define EL(i, j) w->el[((j)-1) * 13 + ((i)-1)]
#define TQ(i, j) w->tq[((j)-1) * 3 + ((i)-1)]

static void F(const rhs_ctx *c, const double *y, double *ydot) {
    orc_rhs(c->m, c->kf, c->kr, c->mc, y, ydot);
}

/* dnrm2.f90:75-162 (Lawson-Hanson scaled 2-norm) */
double orc_dnrm2(int n, const double *dx, int incx) {
    const double cutlo = 8.232e-11, cuthi = 1.304e19;
    double sum = 0.0, xmax = 0.0, hitest;
    int next, i, j = 1, nn;
#define DX(k) dx[(k)-1]
    if (n <= 0) return 0.0;
    next = 30;
    sum = 0.0;
    nn = n * incx;
    i = 1;
L20:
    switch (next) {
    case 30: goto L30;
    case 50: goto L50;
    case 70: goto L70;
    default: goto L110;
    }
L30:
    if (fabs(DX(i)) > cutlo) goto L85;
    next = 50;
    xmax = 0.0;
L50:
    if (DX(i) == 0.0) goto L200;
    if (fabs(DX(i)) > cutlo) goto L85;
    next = 70;
    goto L105;
L100:
    i = j;
    next = 110;
    sum = (sum / DX(i)) / DX(i);
L105:
    xmax = fabs(DX(i));
    goto L115;
L70:
    if (fabs(DX(i)) > cutlo) goto L75;
L110:
    if (fabs(DX(i)) <= xmax) goto L115;
    {
        double q = xmax / DX(i);
        sum = 1.0 + sum * (q * q);
    }
    xmax = fabs(DX(i));
    goto L200;
L115:
    {
        double q = DX(i) / xmax;
        sum = sum + q * q;
    }
    goto L200;
L75:
    sum = (sum * xmax) * xmax;
L85:
    hitest = cuthi / (double)n;
    for (j = i; j <= nn; j += incx) {
        if (fabs(DX(j)) >= hitest) goto L100;
        sum = sum + DX(j) * DX(j);
    }
    return sqrt(sum);
L200:
    i = i + incx;
    if (i <= nn) goto L20;
    return xmax * sqrt(sum);
#undef DX
}

/* daxpy.f90 / dscal.f90 (element operations are independent) */
static void daxpy(int n, double da, const double *dx, double *dy) {
    if (n <= 0 || da == 0.0) return;
    for (int i = 0; i < n; i++) dy[i] = dy[i] + da * dx[i];
}
static void dscal(int n, double da, double *dx) {
    for (int i = 0; i < n; i++) dx[i] = da * dx[i];
}
static int idamax(int n, const double *dx) {
    if (n <= 0) return 0;
    int r = 1;
    if (n == 1) return 1;
    double dmax = fabs(dx[0]);
    for (int i = 2; i <= n; i++) {
        double xm = fabs(dx[i - 1]);
        if (xm > dmax) { r = i; dmax = xm; }
    }
    return r;
}

/* dgefa.f90:60-117 */
static void dgefa(double *a, int lda, int n, int *ipvt, int *info) {
#define A(i, j) a[((j)-1) * lda + ((i)-1)]
    *info = 0;
    int nm1 = n - 1;
    for (int k = 1; k <= nm1; k++) {
        int kp1 = k + 1;
        int l = idamax(n - k + 1, &A(k, k)) + k - 1;
        ipvt[k - 1] = l;
        if (A(l, k) == 0.0) { *info = k; continue; }
        if (l != k) {
            double t = A(l, k);
            A(l, k) = A(k, k);
            A(k, k) = t;
        }
        double t = -1.0 / A(k, k);
        dscal(n - k, t, &A(k + 1, k));
        for (int j = kp1; j <= n; j++) {
            t = A(l, j);
            if (l != k) {
                A(l, j) = A(k, j);
                A(k, j) = t;
            }
            daxpy(n - k, t, &A(k + 1, k), &A(k + 1, j));
        }
    }
    ipvt[n - 1] = n;
    if (A(n, n) == 0.0) *info = n;
#undef A
}

/* dgesl.f90:71-131, JOB = 0 */
static void dgesl(const double *a, int lda, int n, const int *ipvt, double *b) {
#define A(i, j) a[((j)-1) * lda + ((i)-1)]
    int nm1 = n - 1;
    for (int k = 1; k <= nm1; k++) {
        int l = ipvt[k - 1];
        double t = b[l - 1];
        if (l != k) {
            b[l - 1] = b[k - 1];
            b[k - 1] = t;
        }
        daxpy(n - k, t, &A(k + 1, k), &b[k]);
    }
    for (int kb = 1; kb <= n; kb++) {
        int k = n + 1 - kb;
        b[k - 1] = b[k - 1] / A(k, k);
        double t = -b[k - 1];
        daxpy(k - 1, t, &A(1, k), &b[0]);
    }
#undef A
}

/* ddcst.f90:35-106, MINT = 2 (Gear), ISWFLG /= 3 */
void orc_ddcst(int maxord, double *el, double *tq) {
    double factrl[12];
    factrl[0] = 1.0;
    for (int i = 2; i <= maxord; i++) factrl[i - 1] = (double)i * factrl[i - 2];
#define ELc(i, j) el[((j)-1) * 13 + ((i)-1)]
#define TQc(i, j) tq[((j)-1) * 3 + ((i)-1)]
    ELc(1, 1) = 1.0;
    ELc(2, 1) = 1.0;
    for (int j = 2; j <= maxord; j++) {
        ELc(1, j) = factrl[j - 1];
        for (int i = 2; i <= j; i++) ELc(i, j) = (double)j * ELc(i, j - 1) + ELc(i - 1, j - 1);
        ELc(j + 1, j) = 1.0;
    }
    double sum = 1.0;
    for (int j = 2; j <= maxord; j++) {
        sum = sum + 1.0 / (double)j;
        for (int i = 1; i <= j + 1; i++) ELc(i, j) = ELc(i, j) / (factrl[j - 1] * sum);
    }
    for (int j = 1; j <= maxord; j++) {
        if (j > 1) TQc(1, j) = 1.0 / factrl[j - 2];
        TQc(2, j) = (double)(j + 1) / ELc(1, j);
        TQc(3, j) = (double)(j + 2) / ELc(1, j);
    }
#undef ELc
#undef TQc
}

/* ddpsc.f90:22-40 */
static void ddpsc(int ksgn, int N, int nq, work_t *w) {
    for (int j1 = 1; j1 <= nq; j1++)
        for (int j2 = j1; j2 <= nq; j2++) {
            int j = nq - j2 + j1;
            if (ksgn > 0)
                for (int i = 1; i <= N; i++) YH(i, j) = YH(i, j) + YH(i, j + 1);
            else
                for (int i = 1; i <= N; i++) YH(i, j) = YH(i, j) - YH(i, j + 1);
        }
}

/* ddscl.f90:20-37 */
static void ddscl(double hmax, int N, int nq, double rmax, double *h, double *rc, double rh,
                  work_t *w) {
    if (*h < 1.0) {
        double ah = fabs(*h);
        rh = FMIN2(FMIN2(ah * rh, ah * rmax), hmax) / ah;
    } else {
        rh = FMIN2(FMIN2(rh, rmax), hmax / fabs(*h));
    }
    double r1 = 1.0;
    for (int j = 1; j <= nq; j++) {
        r1 = r1 * rh;
        for (int i = 1; i <= N; i++) YH(i, j + 1) = YH(i, j + 1) * r1;
    }
    *h = *h * rh;
    *rc = *rc * rh;
}

/* ddntp.f90:21-53, K = 0 */
static void ddntp(double h, int N, int nq, double t, double tout, const work_t *w, double *y) {
    for (int i = 1; i <= N; i++) y[i - 1] = YH(i, nq + 1);
    double r = (tout - t) / h;
    for (int jj = 1; jj <= nq; jj++) {
        int j = nq + 1 - jj;
        for (int i = 1; i <= N; i++) y[i - 1] = YH(i, j) + r * y[i - 1];
    }
}

/* ddntl.f90:41-182, JTASK >= 0 branch, IMPL = 0, MITER = 2 */
static void ddntl(const rhs_ctx *c, int N, double eps, double *y, work_t *w) {
    w->ier = 0;
    if (w->jtask == 0) {
        orc_ddcst(MAXORD, w->el, w->tq);
        w->rmax = 10000.0;
    }
    w->rc = 0.0;
    w->convrg = 0;
    w->trend = 1.0;
    w->nq = 1;
    w->nwait = 3;
    F(c, y, w->save2);
    w->nfe = w->nfe + 1;
    for (int i = 0; i < N; i++) w->save1[i] = w->save2[i] / FMAX2(1.0, w->ywt[i]);
    double sum = orc_dnrm2(N, w->save1, 1) / sqrt((double)N);
    if (sum > eps / fabs(w->h)) w->h = copysign(eps / sum, w->h);
    for (int i = 1; i <= N; i++) YH(i, 2) = w->h * w->save2[i - 1];
    for (int i = 0; i < N; i++) w->fac[i] = sqrt(w->uround);
}

/* ddpst.f90:28-287, MITER = 2, IMPL = 0 */
static void ddpst(const rhs_ctx *c, int N, double *y, work_t *w) {
    const double FACMAX = 0.5, BU = 0.5;
    w->nje = w->nje + 1;
    w->ier = 0;
    double br = pow(w->uround, 0.875);
    double bl = pow(w->uround, 0.75);
    double bp = pow(w->uround, -0.15);
    double facmin = pow(w->uround, 0.78);
    int nq = w->nq;
    for (int j = 1; j <= N; j++) {
        double ys = FMAX2(fabs(w->ywt[j - 1]), fabs(y[j - 1]));
        double dy;
        for (;;) {
            dy = w->fac[j - 1] * ys;
            if (dy == 0.0) {
                if (w->fac[j - 1] < FACMAX) {
                    w->fac[j - 1] = FMIN2(100.0 * w->fac[j - 1], FACMAX);
                    continue;
                } else {
                    dy = ys;
                }
            }
            break;
        }
        if (nq == 1) dy = copysign(dy, w->save2[j - 1]);
        else dy = copysign(dy, YH(j, 3));
        dy = (y[j - 1] + dy) - y[j - 1];
        double yj = y[j - 1];
        y[j - 1] = y[j - 1] + dy;
        F(c, y, w->save1);
        y[j - 1] = yj;
        double factor = -(w->el[(nq - 1) * 13] * w->h / dy);
        for (int i = 1; i <= N; i++) DFDY(i, j) = (w->save1[i - 1] - w->save2[i - 1]) * factor;
        double diff = fabs(w->save2[0] - w->save1[0]);
        int imax = 1;
        for (int i = 2; i <= N; i++) {
            if (fabs(w->save2[i - 1] - w->save1[i - 1]) > diff) {
                imax = i;
                diff = fabs(w->save2[i - 1] - w->save1[i - 1]);
            }
        }
        if (FMIN2(fabs(w->save2[imax - 1]), fabs(w->save1[imax - 1])) > 0.0) {
            double scale = FMAX2(fabs(w->save2[imax - 1]), fabs(w->save1[imax - 1]));
            if (diff > BU * scale) {
                w->fac[j - 1] = FMAX2(facmin, w->fac[j - 1] * 0.5);
            } else if (br * scale <= diff && diff <= bl * scale) {
                w->fac[j - 1] = FMIN2(w->fac[j - 1] * 2.0, FACMAX);
            } else if (diff < br * scale) {
                w->fac[j - 1] = FMIN2(bp * w->fac[j - 1], FACMAX);
            }
        }
    }
    w->nfe = w->nfe + N;
    for (int i = 1; i <= N; i++) DFDY(i, i) = DFDY(i, i) + 1.0;
    int info;
    dgefa(w->dfdy, N, N, w->ipvt, &info);
    if (info != 0) w->ier = 1;
}

/* ddcor.f90:30-193, MITER = 2, IMPL = 0, IERROR = 3 */
static double ddcor(int N, const double *y, work_t *w) {
    for (int i = 1; i <= N; i++)
        w->save2[i - 1] = w->h * w->save2[i - 1] - YH(i, 2) - w->save1[i - 1];
    dgesl(w->dfdy, N, N, w->ipvt, w->save2);
    for (int i = 0; i < N; i++) {
        w->save1[i] = w->save1[i] + w->save2[i];
        w->save2[i] = w->save2[i] / FMAX2(fabs(y[i]), w->ywt[i]);
    }
    return orc_dnrm2(N, w->save2, 1) / sqrt((double)N);
}

/* ddstp.f90:72-459 with MINT = 2, MITER = 2, IMPL = 0, IERROR = 3,
 * ISWFLG = 2.  Returns JSTATE. */
static int ddstp(const rhs_ctx *c, int N, double eps, double *y, work_t *w) {
    const double BIAS1 = 1.3, BIAS2 = 1.2, BIAS3 = 1.4, RCTEST = 0.3, RMFAIL = 2.0,
                 RMNORM = 10.0, TRSHLD = 1.0;
    const int MXFAIL = 3, MXITER = 3, MXTRY = 50, NDJSTP = 10;
    const double uround = w->uround;
    int ntry = 0, nfail = 0, iter = 0, evaljc;
    double told = w->t, ctest = 0.0, d = 0.0, d1 = 0.0, etest, erdn, erup, rh, rh1, rh2, rh3;
    if (w->jtask <= 0) {
        ddntl(c, N, eps, y, w);
        if (w->h == 0.0) goto L400;
        if (w->ier) goto L420;
    }
L100:
    ntry = ntry + 1;
    if (ntry > MXTRY) goto L410;
    w->t = w->t + w->h;
    ddpsc(1, N, w->nq, w);
    evaljc = (fabs(w->rc - 1.0) > RCTEST) || (w->nstep >= w->jstepl + NDJSTP);
L110:
    iter = 0;
    for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1);
    F(c, y, w->save2);
    w->nfe = w->nfe + 1;
    if (evaljc || w->ier) {
        ddpst(c, N, y, w);
        if (w->ier) goto L160;
        w->convrg = 0;
        w->rc = 1.0;
        w->jstepl = w->nstep;
    }
    for (int i = 0; i < N; i++) w->save1[i] = 0.0;
L130:
    d = ddcor(N, y, w);
    if (iter > 0) w->trend = FMAX2(0.9 * w->trend, d / d1);
    d1 = d;
    ctest = FMIN2(2.0 * w->trend, 1.0) * d;
    if (ctest <= eps) goto L170;
    iter = iter + 1;
    if (iter < MXITER) {
        double el1 = EL(1, w->nq);
        for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1) + el1 * w->save1[i - 1];
        F(c, y, w->save2);
        w->nfe = w->nfe + 1;
        goto L130;
    }
    if (w->convrg) {
        evaljc = 1;
        goto L110;
    }
L160:
    w->t = told;
    ddpsc(-1, N, w->nq, w);
    w->nwait = w->nq + 2;
    if (w->jtask != 0 && w->jtask != 2) w->rmax = RMFAIL;
    if (iter == 0) rh = 0.3;
    else rh = 0.9 * pow(eps / ctest, 0.2);
    if (rh * w->h == 0.0) goto L400;
    ddscl(w->hmax, N, w->nq, w->rmax, &w->h, &w->rc, rh, w);
    goto L100;
L170:
    w->convrg = 1;
    for (int i = 0; i < N; i++) w->save2[i] = w->save1[i] / FMAX2(fabs(y[i]), w->ywt[i]);
    etest = orc_dnrm2(N, w->save2, 1) / (TQ(2, w->nq) * sqrt((double)N));
    if (etest > eps) {
        w->t = told;
        ddpsc(-1, N, w->nq, w);
        nfail = nfail + 1;
        if (nfail < MXFAIL || w->nq == 1) {
            if (w->jtask != 0 && w->jtask != 2) w->rmax = RMFAIL;
            rh2 = 1.0 / (BIAS2 * pow(etest / eps, 1.0 / (double)(w->nq + 1)));
            if (w->nq > 1) {
                for (int i = 1; i <= N; i++)
                    w->save2[i - 1] = YH(i, w->nq + 1) / FMAX2(fabs(y[i - 1]), w->ywt[i - 1]);
                erdn = orc_dnrm2(N, w->save2, 1) / (TQ(1, w->nq) * sqrt((double)N));
                rh1 = 1.0 / FMAX2(1.0, BIAS1 * pow(erdn / eps, 1.0 / (double)w->nq));
                if (rh2 < rh1) {
                    w->nq = w->nq - 1;
                    w->rc = w->rc * EL(1, w->nq) / EL(1, w->nq + 1);
                    rh = rh1;
                } else {
                    rh = rh2;
                }
            } else {
                rh = rh2;
            }
            w->nwait = w->nq + 2;
            if (rh * w->h == 0.0) goto L400;
            ddscl(w->hmax, N, w->nq, w->rmax, &w->h, &w->rc, rh, w);
            goto L100;
        }
        nfail = 0;
        w->jtask = 2;
        for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1);
        ddntl(c, N, eps, y, w);
        w->rmax = RMNORM;
        if (w->h == 0.0) goto L400;
        if (w->ier) goto L420;
        goto L100;
    }
    w->nstep = w->nstep + 1;
    w->hused = w->h;
    w->nqused = w->nq;
    w->avgh = ((double)(w->nstep - 1) * w->avgh + w->h) / (double)w->nstep;
    w->avgord = ((double)(w->nstep - 1) * w->avgord + (double)w->nq) / (double)w->nstep;
    for (int j = 1; j <= w->nq + 1; j++) {
        double e = EL(j, w->nq);
        for (int i = 1; i <= N; i++) YH(i, j) = YH(i, j) + e * w->save1[i - 1];
    }
    for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1);
    if (w->jtask == 0 || w->jtask == 2) {
        rh = 1.0 / FMAX2(uround, BIAS2 * pow(etest / eps, 1.0 / (double)(w->nq + 1)));
        if (rh > TRSHLD) ddscl(w->hmax, N, w->nq, w->rmax, &w->h, &w->rc, rh, w);
    } else if (w->nwait > 1) {
        w->nwait = w->nwait - 1;
        if (w->nwait == 1 && w->nq < MAXORD)
            for (int i = 1; i <= N; i++) YH(i, MAXORD + 1) = w->save1[i - 1];
    } else {
        if (w->nq == 1) {
            rh1 = 0.0;
        } else {
            for (int i = 1; i <= N; i++)
                w->save2[i - 1] = YH(i, w->nq + 1) / FMAX2(fabs(y[i - 1]), w->ywt[i - 1]);
            erdn = orc_dnrm2(N, w->save2, 1) / (TQ(1, w->nq) * sqrt((double)N));
            rh1 = 1.0 / FMAX2(uround, BIAS1 * pow(erdn / eps, 1.0 / (double)w->nq));
        }
        rh2 = 1.0 / FMAX2(uround, BIAS2 * pow(etest / eps, 1.0 / (double)(w->nq + 1)));
        if (w->nq == MAXORD) {
            rh3 = 0.0;
        } else {
            for (int i = 1; i <= N; i++)
                w->save2[i - 1] = (w->save1[i - 1] - YH(i, MAXORD + 1)) /
                                  FMAX2(fabs(y[i - 1]), w->ywt[i - 1]);
            erup = orc_dnrm2(N, w->save2, 1) / (TQ(3, w->nq) * sqrt((double)N));
            rh3 = 1.0 / FMAX2(uround, BIAS3 * pow(erup / eps, 1.0 / (double)(w->nq + 2)));
        }
        if (rh1 > rh2 && rh1 >= rh3) {
            rh = rh1;
            if (rh <= TRSHLD) goto L380;
            w->nq = w->nq - 1;
            w->rc = w->rc * EL(1, w->nq) / EL(1, w->nq + 1);
        } else if (rh2 >= rh1 && rh2 >= rh3) {
            rh = rh2;
            if (rh <= TRSHLD) goto L380;
        } else {
            rh = rh3;
            if (rh <= TRSHLD) goto L380;
            double e = EL(w->nq + 1, w->nq);
            for (int i = 1; i <= N; i++)
                YH(i, w->nq + 2) = w->save1[i - 1] * e / (double)(w->nq + 1);
            w->nq = w->nq + 1;
            w->rc = w->rc * EL(1, w->nq) / EL(1, w->nq - 1);
        }
        ddscl(w->hmax, N, w->nq, w->rmax, &w->h, &w->rc, rh, w);
        w->rmax = RMNORM;
    L380:
        w->nwait = w->nq + 2;
    }
    w->hold = w->h;
    return 1;
L400:
    w->hold = w->h;
    for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1);
    return 2;
L410:
    w->hold = w->h;
    return 3;
L420:
    w->hold = w->h;
    return 4;
}

/* ddriv3.f90:723-1529 for NSTATE=1, NTASK=1, NROOT=0, IERROR=3.
 * Returns NSTATE (2 ok, 3 MXSTEP, 4 EPS raised, 12 fatal). */
static int ddriv3(const rhs_ctx *c, int N, double *y, double tout, double eps, double ewt,
                  double hmax, int mxstep, work_t *w, int *nstep, int *nfe, int *nje) {
    double t = 0.0;
    int nstate;
    w->hmax = hmax;
    w->uround = DBL_EPSILON; /* D1MACH(4) = epsilon(1.0D0) */
    double h = (tout - t) * (1.0 - 4.0 * w->uround);
    h = copysign(FMIN2(fabs(h), hmax), h);
    w->h = h;
    w->jtask = 0;
    w->avgh = 0.0;
    w->hused = 0.0;
    w->avgord = 0.0;
    w->nqused = 0;
    w->nstep = 0;
    w->jstepl = 0;
    w->nfe = 0;
    w->nje = 0;
    w->t = t;
    w->convrg = 0;
    w->ier = 0; /* DDSTP's saved IER; DDNTL clears it before first use */
    for (int i = 1; i <= N; i++) YH(i, 1) = y[i - 1];
    if (t == tout) { nstate = 2; goto done; }
    /* label 180 */
    int nstepl = w->nstep;
    for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1);
L260:
    for (int i = 0; i < N; i++) w->ywt[i] = FMAX2(ewt, fabs(y[i]));
    /* label 410 */
    for (int i = 0; i < N; i++) w->save2[i] = y[i] / w->ywt[i];
    {
        double sum = orc_dnrm2(N, w->save2, 1) / sqrt((double)N);
        sum = FMAX2(1.0, sum);
        if (eps < sum * w->uround) {
            eps = sum * w->uround * (1.0 + 10.0 * w->uround);
            nstate = 4;
            goto L560;
        }
    }
    if ((w->nstep - nstepl) == mxstep) {
        nstate = 3;
        goto L560;
    }
    {
        int jstate = ddstp(c, N, eps, y, w);
        t = w->t;
        if (jstate != 1) {
            /* 670/680/690: the reference reports a level-1 error and stops the
             * program; the restatement flags the cell and returns the state at
             * the start of the failed step. */
            nstate = 12;
            goto L560;
        }
    }
    w->jtask = 1;
    nstate = 2;
    if (t < tout) goto L260;
    ddntp(w->h, N, w->nq, t, tout, w, y);
    goto done;
L560:
    for (int i = 1; i <= N; i++) y[i - 1] = YH(i, 1);
done:
    *nstep = w->nstep;
    *nfe = w->nfe;
    *nje = w->nje;
    return nstate;
}

/* ------------------------------------------------------- cell driver */
/* chemical_kinetics_solver.f90:228-346 for one cell */
static void chem_cell(const orc_mech *m, long n, long cidx, double dt, const double *T,
                      const double *rho, const double *Y, const signed char *bc, double *Y_prod,
                      double *Y_prod2, double *E_f_prod, orc_counters *cnt, int mxstep,
                      work_t *w) {
    const int N = m->n_species, R = m->n_reactions;
    double Tc = T[cidx];
    if (!((Tc >= 305.0) && (bc == NULL || bc[cidx] == 0))) {
        for (int k = 0; k < N; k++) Y_prod[(long)k * n + cidx] = 0.0;
        E_f_prod[cidx] = 0.0;
        if (cnt) { cnt[cidx].nstate = 0; cnt[cidx].nstep = 0; cnt[cidx].nfe = 0; cnt[cidx].nje = 0; }
        return;
    }
    double rh = rho[cidx];
    double mc[ORC_RMAX], kf[ORC_RMAX], kr[ORC_RMAX];
    double conc_in[ORC_NMAX], conc_out[ORC_NMAX];
    double E = 0.0;
    for (int r = 0; r < R; r++) {
        mc[r] = 0.0;
        for (int k = 0; k < N; k++)
            if (m->molar_mass[k] != 0.0)
                mc[r] = mc[r] + Y[(long)k * n + cidx] * rh / m->molar_mass[k] * m->eff[r][k];
    }
    memset(kf, 0, sizeof(double) * R);
    memset(kr, 0, sizeof(double) * R);
    orc_rate_constants(m, Tc, mc, kf, kr);
    for (int k = 0; k < N; k++) {
        double yk = Y[(long)k * n + cidx];
        conc_in[k] = m->molar_mass[k] != 0.0 ? yk * rh / m->molar_mass[k] : yk;
        conc_out[k] = conc_in[k];
    }
    rhs_ctx ctx = {m, kf, kr, mc};
    const double EPS = 1.0e-9, EWT = 1.0e-4;
    const double HMAX = (double)1.0E-7f; /* single-precision literal */
    int nstep, nfe, nje;
    int nstate = ddriv3(&ctx, N, conc_out, dt, EPS, EWT, HMAX, mxstep, w, &nstep, &nfe, &nje);
    for (int k = 0; k < N; k++) {
        double W = m->molar_mass[k];
        double dc = conc_out[k] - conc_in[k];
        if (W != 0.0) {
            Y_prod[(long)k * n + cidx] = dc * W / dt;
            Y_prod2[(long)k * n + cidx] = dc;
        } else {
            Y_prod[(long)k * n + cidx] = dc;
        }
    }
    for (int k = 0; k < N; k++) {
        double hk = orc_specie_enthalpy(m, T_REF, k);
        E = E - hk * (conc_out[k] - conc_in[k]) / dt;
    }
    E_f_prod[cidx] = E;
    if (cnt) {
        cnt[cidx].nstate = nstate;
        cnt[cidx].nstep = nstep;
        cnt[cidx].nfe = nfe;
        cnt[cidx].nje = nje;
    }
}

int orc_chem_step_mx(const orc_mech *m, long n, double dt, const double *T,
                     const double *rho, const double *Y, const signed char *bc,
                     double *Y_prod, double *Y_prod2, double *E_f_prod,
                     orc_counters *counters, int n_threads, int mxstep) {
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
    {
        work_t *w = (work_t *)calloc(1, sizeof(work_t));
#pragma omp for schedule(dynamic)
        for (long c = 0; c < n; c++)
            chem_cell(m, n, c, dt, T, rho, Y, bc, Y_prod, Y_prod2, E_f_prod, counters, mxstep, w);
        free(w);
    }
#else
    (void)n_threads;
    work_t *w = (work_t *)calloc(1, sizeof(work_t));
    for (long c = 0; c < n; c++)
        chem_cell(m, n, c, dt, T, rho, Y, bc, Y_prod, Y_prod2, E_f_prod, counters, mxstep, w);
    free(w);
#endif
    return 0;
}

int orc_chem_step(const orc_mech *m, long n, double dt, const double *T,
                  const double *rho, const double *Y, const signed char *bc,
                  double *Y_prod, double *Y_prod2, double *E_f_prod,
                  orc_counters *counters, int n_threads) {
    return orc_chem_step_mx(m, n, dt, T, rho, Y, bc, Y_prod, Y_prod2, E_f_prod, counters,
                            n_threads, 10000);
}

/* Energy closure: cpm_solver.f90:517,549 then
 * table_approximated_real_gas.f90:404-440 and calculate_temperature. */
int orc_temperature_after(const orc_mech *m, long n, double dt,
                          const double *T, const double *rho, const double *Y,
                          const double *Y_prod, const double *E_f_prod,
                          double *T_out, int n_threads) {
    const int N = m->n_species;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
#else
    (void)n_threads;
#endif
    for (long c = 0; c < n; c++) {
        double X[ORC_NMAX], Y1[ORC_NMAX];
        double avg = 0.0;
        for (int k = 0; k < N; k++)
            if (m->molar_mass[k] != 0.0) avg = avg + Y[(long)k * n + c] / m->molar_mass[k];
        double W0 = 1.0 / avg;
        for (int k = 0; k < N; k++)
            X[k] = m->molar_mass[k] != 0.0 ? Y[(long)k * n + c] / m->molar_mass[k] * W0 : 0.0;
        double e0 = (mixture_internal_energy(m, T[c], X) - mixture_enthalpy(m, T_REF, X)) / W0;
        double e1 = e0 + E_f_prod[c] * dt / rho[c];
        for (int k = 0; k < N; k++) Y1[k] = Y[(long)k * n + c] + Y_prod[(long)k * n + c] * dt / rho[c];
        avg = 0.0;
        for (int k = 0; k < N; k++)
            if (m->molar_mass[k] != 0.0) avg = avg + Y1[k] / m->molar_mass[k];
        double W1 = 1.0 / avg;
        for (int k = 0; k < N; k++)
            X[k] = m->molar_mass[k] != 0.0 ? Y1[k] / m->molar_mass[k] * W1 : 0.0;
        T_out[c] = calculate_temperature(m, T[c], e1 * W1, X);
    }
    return 0;
}

/* ------------------------------------------------ sources + state equation */
/* The reactive terms of the source integration in cpm_solver.f90:513-560
 * (E_f_int = E_f + E_f_prod * dt / rho, Y_int = Y + Y_prod * dt / rho; the
 * renormalisation there is commented out) followed by apply_state_equation,
 * table_approximated_real_gas.f90:368-470, for cells with bc == 0. */
int orc_apply_state(const orc_mech *m, long n, int dims, double dt, const double *rho,
                    const double *Y_prod, const double *E_f_prod, const signed char *bc,
                    double *Y, double *E_f, const double *v, double *T, double *p,
                    double *gamma, double *cp_mass, double *h_s, double *h_full, double *v_s,
                    double *mix_mol_mass, unsigned char *status, int n_threads) {
    const int N = m->n_species;
#ifdef _OPENMP
    int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
#else
    (void)n_threads;
#endif
    for (long c = 0; c < n; c++) {
        if (bc && bc[c] != 0) {
            if (status) status[c] = 0;
            continue;
        }
        if (E_f_prod) E_f[c] = E_f[c] + E_f_prod[c] * dt / rho[c];
        if (Y_prod)
            for (int k = 0; k < N; k++)
                Y[(long)k * n + c] = Y[(long)k * n + c] + Y_prod[(long)k * n + c] * dt / rho[c];
        double e_i = E_f[c];
        for (int d = 0; d < dims; d++) e_i = e_i - 0.5 * (v[(long)d * n + c] * v[(long)d * n + c]);
        double avg = 0.0;
        for (int k = 0; k < N; k++)
            if (m->molar_mass[k] != 0.0) avg = avg + Y[(long)k * n + c] / m->molar_mass[k];
        avg = 1.0 / avg;
        mix_mol_mass[c] = avg;
        double X[ORC_NMAX];
        for (int k = 0; k < N; k++)
            X[k] = m->molar_mass[k] != 0.0 ? Y[(long)k * n + c] / m->molar_mass[k] * avg : 0.0;
        e_i = e_i * avg;
        const double h_s_tref = mixture_enthalpy(m, T_REF, X);
        const double t = calculate_temperature(m, T[c], e_i, X);
        T[c] = t;
        p[c] = t * rho[c] * R_GASE_J / avg;
        const double cp = mixture_cp(m, t, X);
        const double cv = cp - R_GASE_J;
        gamma[c] = cp / cv;
        const double h = mixture_enthalpy(m, t, X);
        h_s[c] = (h - h_s_tref) / avg;
        h_full[c] = h / avg;
        cp_mass[c] = cp / avg;
        const int bad = (gamma[c] < 0.0) || (p[c] < 0.0) || (rho[c] < 0.0);
        if (status) status[c] = bad ? 2 : 1;
        v_s[c] = sqrt(gamma[c] * p[c] / rho[c]);
    }
    return 0;
}
