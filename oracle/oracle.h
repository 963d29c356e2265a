/*
 * CPU ORACLE for the NRG per-cell chemistry step -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference Fortran path, used by the
 * test-suite, the smoke check and the benchmark's CPU baseline as the checker.
 * The product (nrg_b200/) never links, loads or calls it.
 *
 * Parity status: UNPINNED. The reference is Fortran and no Fortran compiler is
 * available, and the reference ships no golden vectors or known-answer tests
 * for this path. The restatement is cross-checked against an independent
 * integrator (scipy BDF at tight tolerance), element conservation and
 * hand-checked parser values instead.
 *
 * Reference files restated (paths inside yakovenko-ivan/NRG):
 *   computing_module/src/current_build/chemical_kinetics_solver.f90:175-685
 *   package_library/src/chemical_properties_class.f90:117-181,289-768
 *   package_library/src/thermophysical_properties_class.f90:225-452,876-881,1226-1341
 *   package_library/src/global_data.f90:35-44
 *   computing_module/src/third_party/slatec/{ddriv3,ddstp,ddntl,ddpst,ddcor,
 *       ddscl,ddpsc,ddcst,ddntp,dgefa,dgesl,dnrm2,idamax,daxpy,dscal,d1mach}.f90
 */
#ifndef NRG_ORACLE_H
#define NRG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NMAX 64   /* species */
#define ORC_RMAX 512  /* reactions */

typedef struct {
    int n_species;
    int n_reactions;
    char species_names[ORC_NMAX + 1][21]; /* index n_species holds "M" */
    int reaction_type[ORC_RMAX];
    /* coeffs[side][r][0] = count, [1..3] = 1-based species index (n+1 = M) */
    int coeffs[2][ORC_RMAX][4];
    double A[ORC_RMAX], beta[ORC_RMAX], E_act[ORC_RMAX];
    double A_low[ORC_RMAX], beta_low[ORC_RMAX], E_act_low[ORC_RMAX];
    double troe[ORC_RMAX][4];
    double eff[ORC_RMAX][ORC_NMAX];
    double a_coeffs[ORC_NMAX][2][7]; /* [k][set 0:T<1000, 1:T>=1000][i], times R */
    double molar_mass[ORC_NMAX];
} orc_mech;

/* Transport data of the mechanism's species (thermophysical_properties_class
 * .f90:137-210, 1343-1414): Lennard-Jones well depth eps/k_B [K], collision
 * diameter [nm], binary diffusivity constants (symmetric, 0 on the diagonal). */
typedef struct {
    int n_species;
    double well_depth[ORC_NMAX];
    double collision_diameter[ORC_NMAX];
    double bdc[ORC_NMAX][ORC_NMAX];
} orc_transport;

/* per-cell DDRIV3 counters */
typedef struct {
    int nstate; /* DDRIV3 NSTATE on return (2 = ok, 3 = MXSTEP, 12 = fatal) */
    int nstep;
    int nfe;
    int nje;
} orc_counters;

/* Parse mechanism + thermo + molar masses.  eact_units is one of
 * "J.mol", "kJ.mol", "cal.mol", "kcal.mol".  Returns 0 on success. */
int orc_load_mechanism(const char *mech_path, const char *thermo_path,
                       const char *molar_path, double eff_default,
                       const char *eact_units, orc_mech *out);

/* One chemistry step over n cells (SoA: Y[k*n + c]).  Mirrors
 * solve_chemical_kinetics including the skip rule (T >= 305 and bc == 0).
 * Y_prod2 is not written for skipped cells.  counters may be NULL.
 * n_threads <= 0 uses all OpenMP threads.  Returns 0. */
int orc_chem_step(const orc_mech *m, long n, double dt, const double *T,
                  const double *rho, const double *Y, const signed char *bc,
                  double *Y_prod, double *Y_prod2, double *E_f_prod,
                  orc_counters *counters, int n_threads);

/* Same step with an explicit mxstep (reference value: 10000). */
int orc_chem_step_mx(const orc_mech *m, long n, double dt, const double *T,
                     const double *rho, const double *Y, const signed char *bc,
                     double *Y_prod, double *Y_prod2, double *E_f_prod,
                     orc_counters *counters, int n_threads, int mxstep);

/* Energy closure used to define the temperature after the step (constant
 * density): e0 from (T0, Y0), e1 = e0 + E_f_prod*dt/rho,
 * Y1 = Y0 + Y_prod*dt/rho, T1 = calculate_temperature(T0, e1*W1, X1). */
int orc_temperature_after(const orc_mech *m, long n, double dt,
                          const double *T, const double *rho, const double *Y,
                          const double *Y_prod, const double *E_f_prod,
                          double *T_out, int n_threads);

/* Building blocks exposed for unit tests. */
void orc_rate_constants(const orc_mech *m, double T, const double *mix_conc,
                        double *kf, double *kr);
void orc_rhs(const orc_mech *m, const double *kf, const double *kr,
             const double *mix_conc, const double *Z, double *Zdot);
double orc_specie_enthalpy(const orc_mech *m, double T, int k);
double orc_specie_entropy(const orc_mech *m, double T, int k);
double orc_specie_cp(const orc_mech *m, double T, int k);
double orc_dnrm2(int n, const double *dx, int incx);
/* Gear (MINT=2) coefficient tables, EL(13,12) and TQ(3,12) column-major */
void orc_ddcst(int maxord, double *el, double *tq);

/* The chemistry sources applied to the state (the reactive terms of
 * cpm_solver.f90:513-560: E_f += E_f_prod*dt/rho, Y += Y_prod*dt/rho) and the
 * state equation (apply_state_equation, table_approximated_real_gas.f90:
 * 368-470) for cells with bc == 0 (bc may be NULL).  Y_prod / E_f_prod may be
 * NULL (state equation only).  v holds dims velocity components (v[d*n+c]).
 * T is read as the Newton start and overwritten.  Per-cell status: 0 skipped
 * (bc), 1 ok, 2 negative gamma, p or rho (the reference stops there). */
int orc_apply_state(const orc_mech *m, long n, int dims, double dt, const double *rho,
                    const double *Y_prod, const double *E_f_prod, const signed char *bc,
                    double *Y, double *E_f, const double *v, double *T, double *p,
                    double *gamma, double *cp_mass, double *h_s, double *h_full, double *v_s,
                    double *mix_mol_mass, unsigned char *status, int n_threads);

/* Reads the transport deck for the mechanism's species.  Returns 0 on success. */
int orc_load_transport(const orc_mech *m, const char *transport_path, orc_transport *out);

/* Neufeld collision integral (calculate_omega, :560-577), binary diffusion
 * coefficient (:737-762) and the mixture-averaged coefficients of every cell
 * (mixture_averaged_diffusion_coefficients :768-814 as called by
 * calculate_diffusivity_coeff, fickean_diffusion_solver.f90:358-395: zero in
 * cells with bc /= 0).  Y and D: species-major, stride n. */
double orc_omega(double T_red, int l, int s);
double orc_binary_diffusion(const orc_mech *m, const orc_transport *t, double T, double p, int i, int j);
void orc_mixture_diffusivity(const orc_mech *m, const orc_transport *t, long n, const double *T, const double *p,
                             const double *Y, const double *m_mix, const signed char *bc, double *D, int n_threads);

/* Species predictor of the low-Mach solver (orc_transport.c; layout there). */
int orc_species_predictor(int N, const double *W, int dims, const int n_cells[3], long ld, int coord, double dx,
                          double dt, const double *const v_f[3], const double *x_center, const signed char *bc,
                          const double *Y_prod_diff, const double *Y_prod_chem, int n_part,
                          const double *const *Y_prod_part, double *rho, double *Y, double *rho_old,
                          double *Y_old, double *rho_int, double *Y_int);

/* table_approximated mode (orc_table.c; chemical_kinetics_solver.f90:542-685
 * and the mode's branches of :228-346).  Table rows: T_t[i], Y_t[k*M + i]. */
void orc_format_e14_7(double x, char out[15]);
int orc_parse_e14_7(const char *field, int len, double *value);
int orc_table_read(const char *path, int n_species, long capacity, double *T_t, double *Y_t, long *rows);
int orc_table_write(const char *path, int n_species, const char (*names)[21], int lb, int ub, int lo, int hi,
                    const double *T_row, const double *Y_prod2_row);
int orc_table_step(const orc_mech *m, long M, const double *T_t, const double *Y_t, long n, double dt,
                   const double *T, const double *Y, const signed char *bc, double *Y_prod, double *Y_prod2,
                   double *E_f_prod, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
