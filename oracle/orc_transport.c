/* CPU oracle (test infrastructure only): the species predictor of the
 * low-Mach solver, the explicit convective update of rho*Y_k that brackets
 * the chemistry step in the operator split.  Restates
 *   fds_low_mach_solver.f90:785-954   calculate_interm_Y_predictor
 *   fds_low_mach_solver.f90:4979-5009 charm_face_value
 *   fds_low_mach_solver.f90:5011-5070 eos_corrected_species_face_vector
 * in the reference's operation order (built with -ffp-contract=off).
 *
 * Layout (0-based, ghost layer included, as the reference's cell fields
 * cells(0:n+1, ...) for active directions and cells(1:1) for inactive ones):
 * extents e[d] = n[d] + 2 (active) or 1; cell (i,j,k) at i + e0*(j + e1*k);
 * species k of a cell field at [k*ld + cell].  Face field of velocity
 * component d (the reference's v_f%pr(d)%cells(dims, 0:n+2, ...)): extents
 * f[d] = e[d] + 1 (active) or 1, element (c, i, j, k) at
 * c + dims*(i + f0*(j + f1*k)); face i is the low face of cell i.
 * The second half restates the mixture-averaged diffusion coefficients.
 * Parity with the reference is unpinned: it ships no known-answer test for
 * these routines. */
#include <float.h>
#include <math.h>
#include <stddef.h>

#include "oracle.h"

/* fds_low_mach_solver.f90:4979-5009 */
static double charm_face_value(const double a[4], double velocity) {
    double phi_up = 0.0, B_r = 0.0, r, s;
    const double phi_loc = a[2] - a[1];
    if (velocity > 0.0)
        phi_up = a[1] - a[0];
    else
        phi_up = a[3] - a[2];
    if (phi_loc != 0.0)
        r = phi_up / phi_loc;
    else
        r = 0.0;
    if (r > 1.0e-10) {
        s = 1.0 / r;
        B_r = s * (3.0 * s + 1.0) / (s + 1.0) / (s + 1.0);
    } else {
        B_r = 0.0;
    }
    if (velocity > 0.0)
        return a[1] + B_r * 0.5 * phi_up;
    return a[2] - B_r * 0.5 * phi_up;
}

typedef struct {
    int dims, N;
    long e[3], f[3], ld;
    const double *rho, *Y, *W;
} grid_t;

static long cell_at(const grid_t *g, long i, long j, long k) { return i + g->e[0] * (j + g->e[1] * k); }

/* fds_low_mach_solver.f90:5011-5070: CHARM face values of rho*Y_k over the
 * four cells around the face, with the most abundant species of the upwind
 * cell corrected so that sum_k phi_k / W_k equals the CHARM face value of
 * rho / W. face_side +1: high face of cell (i,j,k), -1: low face. */
static void eos_face_vector(const grid_t *g, int dim, long i, long j, long k, int face_side, double velocity,
                            double *phi) {
    const long I[3] = {dim == 0, dim == 1, dim == 2};
    const int offset0 = face_side > 0 ? -1 : -2;
    const int gamma_offset = velocity > 0.0 ? offset0 + 1 : offset0 + 2;
    int gamma = 0;
    double rhoY_max = -DBL_MAX;
    long c = cell_at(g, i + gamma_offset * I[0], j + gamma_offset * I[1], k + gamma_offset * I[2]);
    for (int s = 0; s < g->N; s++) {
        const double rhoY_loc = g->rho[c] * g->Y[(long)s * g->ld + c];
        if (rhoY_loc > rhoY_max) {
            rhoY_max = rhoY_loc;
            gamma = s;
        }
    }
    double row[4] = {0.0, 0.0, 0.0, 0.0}, a[4];
    for (int s = 0; s < g->N; s++) {
        for (int n = 0; n < 4; n++) {
            const int off = offset0 + n;
            c = cell_at(g, i + off * I[0], j + off * I[1], k + off * I[2]);
            a[n] = g->rho[c] * g->Y[(long)s * g->ld + c];
            row[n] = row[n] + a[n] / g->W[s];
        }
        phi[s] = charm_face_value(a, velocity);
    }
    const double row_face = charm_face_value(row, velocity);
    double sum_not_gamma = 0.0;
    for (int s = 0; s < g->N; s++)
        if (s != gamma) sum_not_gamma = sum_not_gamma + phi[s] / g->W[s];
    phi[gamma] = g->W[gamma] * (row_face - sum_not_gamma);
}

int orc_species_predictor(int N, const double *W, int dims, const int n_cells[3], long ld, int coord, double dx,
                          double dt, const double *const v_f[3], const double *x_center, const signed char *bc,
                          const double *Y_prod_diff, const double *Y_prod_chem, int n_part,
                          const double *const *Y_prod_part, double *rho, double *Y, double *rho_old,
                          double *Y_old, double *rho_int, double *Y_int) {
    if (N < 1 || N > ORC_NMAX || dims < 1 || dims > 3) return 1;
    grid_t g;
    g.dims = dims;
    g.N = N;
    g.ld = ld;
    g.rho = rho;
    g.Y = Y;
    g.W = W;
    long lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        const int act = d < dims;
        g.e[d] = act ? n_cells[d] + 2 : 1;
        g.f[d] = act ? g.e[d] + 1 : 1;
        lo[d] = act ? 1 : 0;
        hi[d] = act ? n_cells[d] : 0;
    }
    if (ld < g.e[0] * g.e[1] * g.e[2]) return 1;
    const double inv_dx = 1.0 / dx;
    /* calculate_interm_Y_predictor:850-920, all cells from the old rho, Y */
#pragma omp parallel for collapse(3) schedule(static)
    for (long k = lo[2]; k <= hi[2]; k++)
        for (long j = lo[1]; j <= hi[1]; j++)
            for (long i = lo[0]; i <= hi[0]; i++) {
                const long c = cell_at(&g, i, j, k);
                if (bc && bc[c] != 0) continue;
                double lame[3][3];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) lame[a][b] = 1.0;
                if (coord == 1) {
                    lame[0][0] = x_center[i] - 0.5 * dx;
                    lame[0][1] = x_center[i];
                    lame[0][2] = x_center[i] + 0.5 * dx;
                } else if (coord == 2) {
                    const double l = x_center[i] - 0.5 * dx, m = x_center[i], r = x_center[i] + 0.5 * dx;
                    lame[0][0] = l * l;
                    lame[0][1] = m * m;
                    lame[0][2] = r * r;
                }
                double rhs[ORC_NMAX], fr[ORC_NMAX], fl[ORC_NMAX], rhoY_new[ORC_NMAX];
                for (int s = 0; s < N; s++) rhs[s] = 0.0;
                for (int dim = 0; dim < dims; dim++) {
                    const long I[3] = {dim == 0, dim == 1, dim == 2};
                    const long pos = dim == 0 ? i : dim == 1 ? j : k;
                    const double v_r =
                        v_f[dim][dim + dims * ((i + I[0]) + g.f[0] * ((j + I[1]) + g.f[1] * (k + I[2])))];
                    const double v_l = v_f[dim][dim + dims * (i + g.f[0] * (j + g.f[1] * k))];
                    if (pos < hi[dim]) {
                        eos_face_vector(&g, dim, i, j, k, 1, v_r, fr);
                    } else {
                        const long cu = v_r > 0.0 ? c : cell_at(&g, i + I[0], j + I[1], k + I[2]);
                        for (int s = 0; s < N; s++) fr[s] = rho[cu] * Y[(long)s * ld + cu];
                    }
                    if (pos > lo[dim]) {
                        eos_face_vector(&g, dim, i, j, k, -1, v_l, fl);
                    } else {
                        const long cu = v_l > 0.0 ? cell_at(&g, i - I[0], j - I[1], k - I[2]) : c;
                        for (int s = 0; s < N; s++) fl[s] = rho[cu] * Y[(long)s * ld + cu];
                    }
                    for (int s = 0; s < N; s++)
                        rhs[s] = rhs[s] - (fr[s] * v_r * lame[dim][2] - fl[s] * v_l * lame[dim][0]) * inv_dx /
                                              lame[dim][1];
                }
                for (int s = 0; s < N; s++) {
                    const long o = (long)s * ld + c;
                    rhoY_new[s] = rho[c] * Y[o] + rhs[s] * dt;
                    if (Y_prod_diff) rhoY_new[s] = rhoY_new[s] + Y_prod_diff[o] * dt;
                    if (Y_prod_chem) rhoY_new[s] = rhoY_new[s] + Y_prod_chem[o] * dt;
                    for (int p = 0; p < n_part; p++) rhoY_new[s] = rhoY_new[s] + Y_prod_part[p][o] * dt;
                }
                /* :922-933 boundedness and reconstruction */
                double summ = 0.0;
                for (int s = 0; s < N; s++) {
                    rhoY_new[s] = rhoY_new[s] > 0.0 ? rhoY_new[s] : 0.0;
                    summ = summ + rhoY_new[s];
                }
                if (summ > DBL_MIN) {
                    rho_int[c] = summ;
                    for (int s = 0; s < N; s++) Y_int[(long)s * ld + c] = rhoY_new[s] / rho_int[c];
                }
            }
    /* :940-953 the copy, after every cell's fluxes saw the old values */
#pragma omp parallel for collapse(3) schedule(static)
    for (long k = lo[2]; k <= hi[2]; k++)
        for (long j = lo[1]; j <= hi[1]; j++)
            for (long i = lo[0]; i <= hi[0]; i++) {
                const long c = cell_at(&g, i, j, k);
                if (bc && bc[c] != 0) continue;
                rho_old[c] = rho[c];
                rho[c] = rho_int[c];
                for (int s = 0; s < N; s++) {
                    Y_old[(long)s * ld + c] = Y[(long)s * ld + c];
                    Y[(long)s * ld + c] = Y_int[(long)s * ld + c];
                }
            }
    return 0;
}

/* ------------------------------------------------------------------------
 * Mixture-averaged diffusion coefficients (thermophysical_properties_class
 * .f90:560-577, 737-814) with the Neufeld, Janzen and Aziz (1972) collision
 * integral fits the reference sets in set_properties (:173-207).
 * ---------------------------------------------------------------------- */
static const double OMEGA_C[3][8] = {
    /* (1,1) */ {1.06036, 0.15610, 0.19300, 0.47635, 1.03587, 1.52996, 1.76474, 3.89411},
    /* (1,2) */ {1.00220, 0.15530, 0.16105, 0.72751, 0.86125, 2.06848, 1.95162, 4.84492},
    /* (2,2) */ {1.16145, 0.14874, 0.52487, 0.77320, 2.16178, 2.43787, 0.0, 0.0}};

double orc_omega(double T_red, int l, int s) {
    const double *c = OMEGA_C[l == 2 ? 2 : (s == 2 ? 1 : 0)];
    if (T_red < 70.0)
        return c[0] / pow(T_red, c[1]) + c[2] / exp(c[3] * T_red) + c[4] / exp(c[5] * T_red) +
               c[6] / exp(c[7] * T_red);
    return c[0] / pow(T_red, c[1]);
}

double orc_binary_diffusion(const orc_mech *m, const orc_transport *t, double T, double p, int i, int j) {
    (void)m;
    if (T <= 0.0 || p <= 0.0) return 0.0;
    if (i == j) return 0.0;
    const int i1 = i < j ? i : j, i2 = i < j ? j : i;
    if (t->bdc[i1][i2] <= 0.0) return 0.0;
    if (t->well_depth[i1] <= 0.0 || t->well_depth[i2] <= 0.0) return 0.0;
    const double T_red = T / sqrt(t->well_depth[i1] * t->well_depth[i2]);
    const double omega = orc_omega(T_red, 1, 1);
    if (omega <= 0.0) return 0.0;
    return t->bdc[i1][i2] * pow(T, 1.5) / (p * omega);
}

static void mixture_cell(const orc_mech *m, const orc_transport *t, double T, double p, const double *Y,
                         double m_mix, double *D) {
    const int N = m->n_species;
    const double *W = m->molar_mass;
    for (int i = 0; i < N; i++) D[i] = 0.0;
    if (N <= 0 || T <= 0.0 || p <= 0.0 || m_mix <= 0.0) return;
    double Db[ORC_NMAX][ORC_NMAX];
    for (int i = 0; i < N - 1; i++)
        for (int j = i + 1; j < N; j++) Db[i][j] = orc_binary_diffusion(m, t, T, p, i, j);
    for (int i = 0; i < N; i++) {
        if (W[i] <= 0.0) continue;
        double acc = 0.0;
        for (int j = 0; j < N; j++) {
            if (j == i) continue;
            if (W[j] <= 0.0) continue;
            const double Dij = j > i ? Db[i][j] : Db[j][i];
            if (Dij <= 0.0) continue;
            acc = acc + (1.0 - Y[i]) * W[i] * Y[j] / (Dij * W[j]);
            acc = acc + Y[i] * Y[j] / Dij;
        }
        if (acc > 1.0e-10) D[i] = (1.0 - Y[i]) * W[i] / (acc * m_mix);
    }
}

void orc_mixture_diffusivity(const orc_mech *m, const orc_transport *t, long n, const double *T, const double *p,
                             const double *Y, const double *m_mix, const signed char *bc, double *D, int n_threads) {
    const int N = m->n_species;
    (void)n_threads;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; c++) {
        double y[ORC_NMAX], d[ORC_NMAX];
        for (int k = 0; k < N; k++) d[k] = 0.0;
        if (!bc || bc[c] == 0) {
            for (int k = 0; k < N; k++) y[k] = Y[(long)k * n + c];
            mixture_cell(m, t, T[c], p[c], y, m_mix[c], d);
        }
        for (int k = 0; k < N; k++) D[(long)k * n + c] = d[k];
    }
}
