/*
 * nrg_chem.h -- C ABI of the B200 chemistry step for NRG.
 *
 * Drop-in boundary for the operator-split chemistry source term of NRG
 * (module chemical_kinetics_solver_class,
 *  computing_module/src/current_build/chemical_kinetics_solver.f90).
 * Plain pointers and sizes only; every function returns an int status
 * (NRG_OK = 0, negative = error, see nrg_chem_last_error) and never exits the
 * process.  One handle owns one CUDA stream on the device that was current at
 * creation; a handle is not re-entrant across host threads.
 */
#ifndef NRG_CHEM_H
#define NRG_CHEM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NRG_MAX_SPECIES 24

#if defined(__GNUC__)
#define NRG_API __attribute__((visibility("default")))
#else
#define NRG_API
#endif

enum nrg_status {
  NRG_OK = 0,
  NRG_ERR_ARG = -1,         /* bad argument (null pointer, bad size, bad bounds) */
  NRG_ERR_IO = -2,          /* mechanism / thermo / molar-mass deck unreadable */
  NRG_ERR_CUDA = -3,        /* CUDA runtime error (message in nrg_chem_last_error) */
  NRG_ERR_UNSUPPORTED = -4, /* mechanism size without a compiled kernel */
  NRG_ERR_STATE = -5        /* call not valid in the current state */
};

/* Activation-energy units of the deck (reference E_act_units,
 * chemical_properties_class.f90:165-174). */
enum nrg_eact_units { NRG_EACT_J_MOL = 0, NRG_EACT_KJ_MOL = 1, NRG_EACT_CAL_MOL = 2, NRG_EACT_KCAL_MOL = 3 };

/* Integration modes. */
enum nrg_mode {
  NRG_MODE_REFERENCE = 0, /* FP64, finite-difference Jacobian exactly as the reference (DDPST MITER=2) */
  NRG_MODE_FAST = 1,      /* FP64, analytic Jacobian */
  NRG_MODE_MIXED = 2,     /* analytic Jacobian, FP32 LU + FP64 residual and refinement */
  NRG_MODE_SURROGATE = 3, /* gated BF16 MLP surrogate with FP64 fallback (needs a trained model) */
  NRG_MODE_TABLE = 4      /* ODE_solver = 'table_approximated': Y_prod2 interpolated in T from a table
                             (needs nrg_chem_load_table or nrg_chem_set_table) */
};

/* Per-cell status byte (nrg_chem_step_device status output). */
enum nrg_cell_status {
  NRG_CELL_SKIPPED = 0,   /* T < 305 K or bc_markers /= 0: zero sources, Y_prod2 untouched */
  NRG_CELL_OK = 1,
  NRG_CELL_MXSTEP = 2,    /* MXSTEP steps without reaching dt (reference NSTATE = 3) */
  NRG_CELL_FATAL = 3,     /* step size vanished or 50 retries (reference stops the program) */
  NRG_CELL_NONFINITE = 4,
  NRG_CELL_SURROGATE = 5  /* surrogate prediction accepted by the gate */
};

typedef struct nrg_chem nrg_chem;

/* Host field block in the reference layout: every array is a Fortran
 * column-major 3-D array cells(lb(1):ub(1), lb(2):ub(2), lb(3):ub(3)) with the
 * ghost layer included (field_scalar_class.f90:68-73); Y, Y_prod and Y_prod2
 * hold one array per species (field_vector_class.f90:61-80).  lo/hi are the
 * interior bounds the reference loops over (get_local_inner_cells_bounds,
 * computational_domain_class.f90:492-503). */
typedef struct {
  int lb[3], ub[3];
  int lo[3], hi[3];
  const double* T;
  const double* p; /* read by the reference, unused by its arithmetic; may be NULL */
  const double* rho;
  const double* Y[NRG_MAX_SPECIES];
  double* Y_prod[NRG_MAX_SPECIES];
  double* Y_prod2[NRG_MAX_SPECIES];
  double* E_f_prod;
  const signed char* bc_markers; /* int8 markers; NULL = all interior */
} nrg_field_desc;

typedef struct {
  long long cells;           /* cells in the call */
  long long cells_active;    /* cells integrated (not skipped) */
  long long cells_bad;       /* MXSTEP / fatal / non-finite cells */
  long long cells_surrogate; /* cells answered by the surrogate */
  long long cells_fallback;  /* active cells sent to the FP64 integrator by the gate */
  long long steps, rhs_evals, jacobians, solves;
  double device_ms;          /* device time of the step (CUDA events) */
  /* per-phase device time when phase timing is on (nrg_chem_set_timing):
   * [0] surrogate inference (features + MLP, then the FP64 gate), [1] the
   * rejected cells' list (temperature order, or compaction in cell order), [2] FP64
   * integrator (with the plain step's temperature order), [3] unused.
   * nrg_chem_step (host arrays) reports host wall times instead: [0] the
   * gather of the inputs into pinned staging, [1] the chunks' scatter with
   * its waits for their copies, [2] unused, [3] the whole call */
  double phase_ms[4];
} nrg_chem_stats;

/* Replaces chemical_kinetics_solver_c(manager) (chemical_kinetics_solver.f90:
 * 111-173) together with the mechanism set-up it relies on
 * (chemical_properties%set_properties, chemical_properties_class.f90:117-181;
 * thermophysical_properties%set_properties, thermophysical_properties_class.f90:
 * 137-210).  Paths name the three input decks. */
NRG_API int nrg_chem_create(const char* mechanism_path, const char* thermo_path, const char* molar_masses_path,
                    double default_enhanced_efficiencies, int eact_units, nrg_chem** out);

/* Releases the handle and its device memory (never the caller's arrays). */
NRG_API int nrg_chem_destroy(nrg_chem* h);

/* Replaces call this%solve_chemical_kinetics(time_step)
 * (chemical_kinetics_solver.f90:175-358) on host arrays in the reference
 * layout: gathers the interior, runs the step on the GPU and scatters
 * Y_prod / Y_prod2 / E_f_prod back.  stats may be NULL. */
NRG_API int nrg_chem_step(nrg_chem* h, double time_step, const nrg_field_desc* fields, nrg_chem_stats* stats);

/* Same step on device-resident species-major arrays: element (k, c) at
 * [k*ld + c], ld >= n.  T_after (temperature after the energy closure),
 * status and bc may be NULL.  stream is the caller's cudaStream_t (NULL: the
 * legacy default stream): the step is ordered after work already queued there
 * and the call returns when the step has finished. */
NRG_API int nrg_chem_step_device(nrg_chem* h, double time_step, long n, long ld, const double* T,
                         const double* rho, const double* Y, const signed char* bc, double* Y_prod,
                         double* Y_prod2, double* E_f_prod, double* T_after, unsigned char* status,
                         void* stream, nrg_chem_stats* stats);

/* No counterpart in the reference.  The same FP64 step as
 * nrg_chem_step_device for callers that must not allocate device memory while
 * stepping (for example a host code whose device memory is owned by its own
 * pool, or that steps from a context where cudaMalloc is not allowed): this
 * call allocates nothing.  Its scratch (cell flags, scan, the list of active
 * cells, queue head, counters) is one fixed device array inside the library,
 * about 5.3 MB, which every GPU that loads the library keeps until exit; n is
 * limited to 1,048,576 cells per call and larger n is rejected with
 * NRG_ERR_ARG.  The first call on each device looks up the array's address
 * (set-up), so make that first call before any stream capture.  All calls on
 * a device share the array: calls that overlap on the GPU (several streams or
 * host threads at once) race on it.  The array's address is looked up once
 * per device and kept for the life of the process; a device reset
 * (cudaDeviceReset) invalidates it, so do not call this entry point again on
 * a device after resetting it in the same process.  The surrogate and table
 * modes are not available here. */
/* Relative tolerance EPS of the FP64 integrator (DDRIV3's EPS; the
 * reference fixes it at 1e-9, chemical_kinetics_solver.f90:282).  0 restores
 * 1e-9; any other value departs from the reference's results. */
NRG_API int nrg_chem_set_eps(nrg_chem* h, double eps);

NRG_API int nrg_chem_step_device_noalloc(nrg_chem* h, double time_step, long n, long ld, const double* T,
                                         const double* rho, const double* Y, const signed char* bc,
                                         double* Y_prod, double* Y_prod2, double* E_f_prod, double* T_after,
                                         unsigned char* status, void* stream, nrg_chem_stats* stats);

/* The table_approximated mode (ODE_solver = 'table_approximated',
 * chemical_kinetics_solver.f90:91,168-170).  A table holds, per row, a
 * temperature and the N per-step concentration changes Y_prod2 of a
 * tabulated 1-D flame.  In NRG_MODE_TABLE every active cell takes its values
 * from the table by linear interpolation in T (the last row interval
 * holding T; 0 below the first row, the last row above it;
 * interpolate_chemical_kinetics, :651-685), and the step writes
 * Y_prod = value * W / dt, Y_prod2 = value - Y and
 * E_f_prod = -sum h_k(T_ref) * value / dt (:256-262, :314-315, :318-340).
 * Table arrays: T_t[i], Y_t[k * stride + i] (stride = rows, or capacity in
 * nrg_table_read). */

/* Replaces read_chemical_kinetics_table (:608-650): reads a table file of
 * n_species species -- one header record, then one record per row in the
 * Fortran edit format (n_species+1)E14.7.  Host only (no GPU, no handle).
 * With T_t == NULL only *rows is set; otherwise capacity >= *rows. */
NRG_API int nrg_table_read(const char* path, int n_species, long capacity, double* T_t, double* Y_t, long* rows);

/* Replaces write_chemical_kinetics_table (:542-607): writes the table of
 * the row j = 1, k = 1 of the host arrays f->T and f->Y_prod2 (reference
 * layout), from the first interior cell between 300.5 and 310 K to the first
 * cell of the largest temperature.  Host only. */
NRG_API int nrg_table_write(const char* path, int n_species, const char* const* species_names,
                            const nrg_field_desc* f);

/* The handle's table for NRG_MODE_TABLE (copied to the device). */
NRG_API int nrg_chem_set_table(nrg_chem* h, long rows, const double* T_t, const double* Y_t);

/* nrg_table_read + nrg_chem_set_table: the constructor's
 * read_chemical_kinetics_table call (:168-170). */
NRG_API int nrg_chem_load_table(nrg_chem* h, const char* path);

/* The chemistry sources applied to the flow state and the state equation,
 * on device arrays (same layout as nrg_chem_step_device), for cells with
 * bc == 0 (bc may be NULL).  Replaces the reactive terms of the source
 * integration (cpm_solver.f90:513-560: E_f += E_f_prod * dt / rho,
 * Y += Y_prod * dt / rho) followed by apply_state_equation
 * (table_approximated_real_gas.f90:368-470), so the chemistry step's outputs
 * update Y, E_f, T and p without leaving the GPU.  Y_prod and E_f_prod may be
 * NULL (state equation only; time_step is then ignored).  v: dims (0..3)
 * velocity components, v[d * ld + c].  T is read as the Newton start of the
 * temperature solve and overwritten.  cp_mass, h_s, h_full, v_s,
 * mix_mol_mass and status may be NULL; status: 0 skipped, 1 ok, 2 negative
 * gamma, p or rho (the reference stops the run there). */
NRG_API int nrg_chem_apply_state_device(nrg_chem* h, double time_step, long n, long ld, int dims,
                                        const double* rho, const double* Y_prod, const double* E_f_prod,
                                        const signed char* bc, double* Y, double* E_f, const double* v, double* T,
                                        double* p, double* gamma, double* cp_mass, double* h_s, double* h_full,
                                        double* v_s, double* mix_mol_mass, unsigned char* status, void* stream);

/* Block of the low-Mach solver's cell fields on the device, for
 * nrg_species_predictor_device.  Cell arrays include the ghost layer: extents
 * e[d] = n[d] + 2 for the dims active directions and 1 for the others, cell
 * (i, j, k) (0-based, interior 1..n[d] in active directions) at
 * i + e0 * (j + e1 * k), species s at [s * ld + cell] -- the reference's
 * cells(0:n+1, 0:n+1, 1:1) arrays (get_local_utter_cells_bounds,
 * computational_domain_class.f90:497-504) stacked by species. */
typedef struct {
  int dims;      /* 1..3 */
  int n[3];      /* interior cells per active direction */
  long long ld;  /* species stride of the cell arrays, >= e0 * e1 * e2 */
  int coord;     /* 0 cartesian, 1 cylindrical (x = r), 2 spherical (x = r) */
  double dx;     /* cell_size(1): the reference divides every direction's fluxes by it */
} nrg_grid_desc;

/* Replaces calculate_interm_Y_predictor (fds_low_mach_solver.f90:785-954) on
 * device arrays: the explicit convective update of rho*Y_k with CHARM-limited
 * face values and the equation-of-state correction of the most abundant
 * species (eos_corrected_species_face_vector, :5011-5070), plus dt times the
 * diffusion, chemistry and particle sources, clipped at zero and
 * renormalised; for interior cells with bc == 0: rho_old, Y_old = the old
 * rho, Y; rho_int, Y_int = the new ones (left unchanged where all rho*Y_k
 * clip to zero, as the reference does); then rho, Y = rho_int, Y_int.  The
 * mechanism of h supplies the species count and molar masses.  v_f: dims
 * pointers, v_f[d] the reference's face field of velocity component d,
 * v_f%pr(d)%cells(1:dims, 0:n+2, ...) in Fortran order (element (c, i, j, k)
 * at c + dims * (i + f0 * (j + f1 * k)), f[d] = e[d] + 1 for active
 * directions; face i is the low face of cell i).  x_center: e0 cell-centre x
 * coordinates (mesh%mesh(1, i, j, k)), needed for coord 1 and 2, else NULL.
 * bc, Y_prod_diff (diffusion_flag off), Y_prod_chem (reactive_flag off) may
 * be NULL; n_particle_phases <= 4 source arrays.  Same stream rules as
 * nrg_chem_step_device. */
NRG_API int nrg_species_predictor_device(nrg_chem* h, double time_step, const nrg_grid_desc* grid,
                                         const double* const* v_f, const double* x_center, const signed char* bc,
                                         const double* Y_prod_diff, const double* Y_prod_chem,
                                         int n_particle_phases, const double* const* Y_prod_particles, double* rho,
                                         double* Y, double* rho_old, double* Y_old, double* rho_int, double* Y_int,
                                         void* stream);

/* Reads the transport deck (thermophysical_properties%set_properties
 * transport part, thermophysical_properties_class.f90:163-171, 1343-1414):
 * Lennard-Jones well depth and collision diameter of every mechanism species
 * (e.g. KEROMNES_TRANSDATA.txt) and the binary diffusivity constants.
 * NRG_ERR_IO when a species is missing (the reference stops the program). */
NRG_API int nrg_chem_load_transport(nrg_chem* h, const char* transport_path);

/* Host-only parse (no CUDA call) of the three decks plus the transport deck:
 * n_species well depths [K], collision diameters [nm] and the n_species x
 * n_species binary diffusivity constants (row-major, symmetric), as
 * nrg_chem_load_transport builds them.  Any output pointer may be NULL.  No
 * counterpart in the reference. */
NRG_API int nrg_mech_transport_tables(const char* mechanism_path, const char* thermo_path,
                                      const char* molar_masses_path, const char* transport_path,
                                      double* well_depth, double* collision_diameter, double* binary_diffusivity);

/* Replaces calculate_diffusivity_coeff (fickean_diffusion_solver.f90:358-395)
 * on device arrays: the mixture-averaged diffusion coefficient of every
 * species (mixture_averaged_diffusion_coefficients,
 * thermophysical_properties_class.f90:768-814, with the Chapman-Enskog binary
 * coefficients of :737-762 and the Neufeld collision integral of :560-577) in
 * each of n cells; D = 0 where bc /= 0 (bc may be NULL).  Y and D
 * species-major at [k * ld + c]; mix_mol_mass as written by
 * nrg_chem_apply_state_device.  Needs nrg_chem_load_transport. */
NRG_API int nrg_mixture_diffusivity_device(nrg_chem* h, long n, long ld, const double* T, const double* p,
                                           const double* Y, const double* mix_mol_mass, const signed char* bc,
                                           double* D, void* stream);

/* Mode (enum nrg_mode).  The reference's ODE_solver selector
 * (chemical_kinetics_solver.f90:91,309-316) has no GPU counterpart for
 * 'table_approximated'. */
NRG_API int nrg_chem_set_mode(nrg_chem* h, int mode);

/* Launch shape.  kernel: 0 = one thread per cell over a grid covering the
 * cells (default), 1 = one thread per cell pulling cells from a device work
 * queue, 2 = one warp per cell pulling cells from the work queue.  block: 32
 * (default) or 64 for kernels 0/1 (each cell keeps ~1.6 KB in shared memory),
 * 128 or 256 for kernel 2.  grid: persistent grid size (0 = fill the GPU).
 * chunk: cells reserved per queue fetch (1..64). */
NRG_API int nrg_chem_set_launch(nrg_chem* h, int kernel, int block, int grid, int chunk);
NRG_API int nrg_chem_get_launch(nrg_chem* h, int* kernel, int* block, int* grid, int* chunk);
/* Form of the LU factorisation in the thread-per-cell kernels: 0 (default)
 * unrolled over the integrated species, 1 a loop.  Same results; the
 * unrolled form is faster where neighbouring cells take alike BDF paths
 * (the flame field), the loop, with a quarter of the code, where they vary
 * (ignition and wide-range fields).  nrg_chem_autotune tries both. */
NRG_API int nrg_chem_set_lu_form(nrg_chem* h, int rolled);
NRG_API int nrg_chem_get_lu_form(nrg_chem* h, int* rolled);

/* Times candidate launch shapes on the given device-resident inputs (outputs
 * are scratch) and keeps the fastest for this handle.  ms_best may be NULL. */
NRG_API int nrg_chem_autotune(nrg_chem* h, double time_step, long n, long ld, const double* T,
                      const double* rho, const double* Y, const signed char* bc, double* Y_prod,
                      double* Y_prod2, double* E_f_prod, double* ms_best);

/* Right-hand side and analytic iteration matrix of the thread-per-cell
 * analytic-Jacobian kernels: 1 = straight-line code generated for the reaction
 * structure of one of the four reference mechanisms (KEROMNES, ZHANG, TEREZA,
 * KONNOV; nrg_b200/gen_mech.py; registers instead of table walks through
 * shared memory), used by default when the parsed mechanism has exactly that
 * structure; 0 = the table-driven loops.  Both give the same bits.  No
 * counterpart in the reference. */
NRG_API int nrg_chem_set_specialised(nrg_chem* h, int enable);

/* Capture the step in a CUDA graph (1) or launch directly (0). */
NRG_API int nrg_chem_set_graph(nrg_chem* h, int enable);

/* Order in which the FP64 integrator takes the cells of a step (the plain
 * step and the surrogate's fallback cells): 1 (default) = sorted by
 * temperature (stable radix sort on a 1/1024 K key, cells the step skips
 * first), so that the lanes of a warp take similar BDF paths; 0 = cell order.  Cells are independent, so both give the same results.  No
 * counterpart in the reference (its OpenMP loop takes cells one by one,
 * chemical_kinetics_solver.f90:222). */
NRG_API int nrg_chem_set_cell_order(nrg_chem* h, int enable);

/* Per-phase CUDA-event timing of the step (stats.phase_ms); launches the step
 * without a graph while enabled. */
NRG_API int nrg_chem_set_timing(nrg_chem* h, int enable);

/* Mechanism size and parsed tables (for checks against the reference decks).
 * Arrays may be NULL; sizes follow n_species (N) and n_reactions (R):
 * reaction_type[R], coeffs[2*R*4] ([side][r][count,i1,i2,i3], 1-based, N+1 = M),
 * arrhenius[R*9] (A, beta, E, A_low, beta_low, E_low, troe0..2), troe3[R],
 * eff[R*N], a_coeffs[N*2*7] (times R), molar_mass[N]. */
NRG_API int nrg_chem_info(nrg_chem* h, int* n_species, int* n_reactions);
NRG_API int nrg_chem_tables(nrg_chem* h, int* reaction_type, int* coeffs, double* arrhenius, double* troe3,
                    double* eff, double* a_coeffs, double* molar_mass);
NRG_API int nrg_chem_species_name(nrg_chem* h, int k, char* buf, int buflen);

/* Host-only parse of the three decks (no CUDA call): fills n_species /
 * n_reactions and, when non-NULL, the tables in the nrg_chem_tables layout.
 * Call once with NULL arrays to size them. */
NRG_API int nrg_mech_tables(const char* mechanism_path, const char* thermo_path,
                            const char* molar_masses_path, double default_enhanced_efficiencies,
                            int eact_units, int* n_species, int* n_reactions, int* reaction_type,
                            int* coeffs, double* arrhenius, double* troe3, double* eff,
                            double* a_coeffs, double* molar_mass);

/* Failure-handling self test (no counterpart in the reference): one warp
 * waits, with the bounded mbarrier wait that every wait of the tensor-core
 * kernel uses, on a barrier that nothing arrives at; the wait gives up after
 * limit_ns (at most 2 s), *timed_out is set to 1 and waited_ms (may be NULL)
 * to the time waited, and the context stays usable. */
NRG_API int nrg_selftest_bounded_wait(long long limit_ns, int* timed_out, double* waited_ms);

/* Message of the last failing call on this handle (or of the last failing
 * nrg_chem_create when h is NULL). */
NRG_API const char* nrg_chem_last_error(nrg_chem* h);

/* ---- Gated surrogate (no counterpart in the reference: NRG has no learned
 * chemistry).  A BF16 MLP predicts the per-cell increment (dY_1..dY_9, dT)
 * from (T, log p, Y_1..Y_9, log10 dt); cells outside the training hull, or
 * whose prediction fails the element-conservation or temperature check, are
 * integrated by the FP64 kernel.  x_bf16 arrays hold n x 16 bf16 standardised
 * features, y arrays n x 10 fp32 standardised targets (device memory). */
NRG_API int nrg_surrogate_param_count(void);
NRG_API int nrg_surrogate_norm_count(void);
/* A handle holds up to eight networks: 0, the main one, and 1..7 for
 * narrower temperature bands (the committed models: 1 a flame's preheat
 * band, 305-800 K, 2 the low-temperature part of its front, 800-1500 K) or
 * serving as another network's committee partner.  A
 * surrogate step needs network 0; each active cell goes to the enabled
 * network of highest index whose training hull's temperature range holds it
 * (network 0 also takes the cells above its hull, which its hull test then
 * rejects), and to the FP64 integrator when there is none; each network has
 * its own standardisation and gate settings.  The set-up calls below (init,
 * parameters, norm, training, gate, enable, save, load, inference) act on
 * the network selected here (0 by default). */
NRG_API int nrg_surrogate_select(nrg_chem* h, int net);
NRG_API int nrg_surrogate_init(nrg_chem* h, unsigned long long seed);
NRG_API int nrg_surrogate_get_params(nrg_chem* h, float* params);
NRG_API int nrg_surrogate_set_params(nrg_chem* h, const float* params);
NRG_API int nrg_surrogate_get_norm(nrg_chem* h, float* norm);
NRG_API int nrg_surrogate_set_norm(nrg_chem* h, const float* norm);
/* Choices made when training arrays are prepared. */
typedef struct nrg_surrogate_opts {
  float hull_margin;    /* fraction of each raw feature's range added on both sides of the hull */
  float dt_pow;         /* targets are divided by (dt / 1e-6)^dt_pow */
  unsigned log_mask;    /* bit k: Y_k enters the network as log10(Y_k + log_eps) (k < 9) */
  float log_eps;        /* > 0 */
  int common_dY_scale;  /* 1: one scale for all dY_k (absolute-error loss); 0: per species */
} nrg_surrogate_opts;
/* Training arrays from integrated states (Y_prod, T_after from
 * nrg_chem_integrate with the same dt / dt_cells); also fits the feature and
 * target scaling and the training hull (on the raw features). */
NRG_API int nrg_surrogate_prepare(nrg_chem* h, long n, long ld, double dt, const double* dt_cells,
                                  const double* T, const double* rho, const double* Y, const double* Y_prod,
                                  const double* T_after, const nrg_surrogate_opts* opts, void* x_bf16,
                                  float* y);
NRG_API int nrg_surrogate_features(nrg_chem* h, long n, long ld, double dt, const double* dt_cells,
                                   const double* T, const double* rho, const double* Y, float* xraw,
                                   void* x_bf16);
NRG_API int nrg_surrogate_forward(nrg_chem* h, long n, const void* x_bf16, float* out);
/* Mean-squared-error gradient over n rows into host memory (no update). */
NRG_API int nrg_surrogate_grad(nrg_chem* h, long n, const void* x_bf16, const float* y, float* grads_host,
                               double* loss_host);
NRG_API int nrg_surrogate_train(nrg_chem* h, long n, const void* x_bf16, const float* y, int epochs, int batch,
                                float lr, unsigned long long seed, float* loss_per_epoch);
/* Gate: element residual (element mass fraction, H/O/N) of the dY that is
 * written, after its orthogonal projection onto the element-conserving
 * increments; residual of the network's own dY before that projection; bound
 * on the gap between the network's dT and the FP64 energy closure of the
 * written dY (K); |dT| bound (K). */
NRG_API int nrg_surrogate_set_gate(nrg_chem* h, double elem_tol, double raw_elem_tol, double dT_tol,
                                   double dT_max);
/* Longest step (s) whose cells the gate may accept; cells with a longer step
 * go to the FP64 integrator.  Default 1e-6 s: the gate bounds above were
 * calibrated on 1e-6 s steps, and on 1e-5 s steps of the wide-range
 * distribution they let cells through with errors of many kelvin.  No
 * counterpart in the reference. */
NRG_API int nrg_surrogate_set_gate_dt(nrg_chem* h, double dt_max);
/* Committee check of the selected network: a cell it answers is accepted
 * only if network `partner` (-1: no check), evaluated on the same cell,
 * predicts every dY_k within agree_Y (mass fraction) and dT within agree_T
 * (K) of it -- two networks trained on different temperature ranges rarely
 * share an error, so their agreement marks reliable predictions.  No
 * counterpart in the reference. */
NRG_API int nrg_surrogate_set_partner(nrg_chem* h, int partner, double agree_Y, double agree_T);
/* Routing band [T_lo, T_hi) of the selected network instead of its training
 * hull's temperature range (0, 0: back to the hull's; T_lo >= T_hi: no cells
 * are routed to it, it only answers as a committee partner).  No
 * counterpart in the reference. */
NRG_API int nrg_surrogate_set_band(nrg_chem* h, double T_lo, double T_hi);
/* Step band (dt_lo, dt_hi] of the selected network (default (0, 1e300]):
 * only cells whose step lies in it are routed to the network, so a network
 * trained on long steps answers those alone.  No counterpart in the
 * reference. */
NRG_API int nrg_surrogate_set_dt_band(nrg_chem* h, double dt_lo, double dt_hi);
/* Relative tolerance EPS of the FP64 integration of the cells the gate
 * rejects (0, the default: the handle's EPS, nrg_chem_set_eps).  The
 * surrogate mode is an approximation to |dT| <= 1 K, |dY_k| <= 1e-4; an EPS
 * of 1e-5 keeps the fallback cells' error below 1e-6 in Y on the flame
 * field while taking about 40% fewer BDF steps than 1e-9.  Per handle, for
 * every network.  No counterpart in the reference. */
NRG_API int nrg_surrogate_set_fallback_eps(nrg_chem* h, double eps);
/* Gate bounds of the selected network for longer steps: band 1..3 applies to
 * steps in (the previous band's dt_max, dt_max], band 0 being
 * nrg_surrogate_set_gate with nrg_surrogate_set_gate_dt's bound; the bounds
 * mean what they mean in nrg_surrogate_set_gate.  dt_max 0 leaves the band
 * unused.  Steps above every band go to FP64.  No counterpart in the
 * reference. */
NRG_API int nrg_surrogate_set_gate_band(nrg_chem* h, int band, double dt_max, double elem_tol,
                                        double raw_elem_tol, double dT_tol, double dT_max);
/* Inference path of the surrogate step: 1 (default) the tensor-core kernel
 * (features and the five layers on tcgen05 with TMEM accumulators) followed
 * by the wide FP64 gate kernel; 0 the GEMM chain (features, one tcgen05
 * GEMM per layer) followed by the same gate kernel. */
NRG_API int nrg_surrogate_set_inference(nrg_chem* h, int fused);
/* Network outputs (n x 16 fp32, normalised units) of the fused kernel for
 * every cell, no gate (device arrays, same layout as nrg_chem_step_device). */
NRG_API int nrg_surrogate_infer(nrg_chem* h, long n, long ld, double dt, const double* dt_cells, const double* T,
                                const double* rho, const double* Y, float* out);
NRG_API int nrg_surrogate_enable(nrg_chem* h, int enable);
NRG_API int nrg_surrogate_save(nrg_chem* h, const char* path);
NRG_API int nrg_surrogate_load(nrg_chem* h, const char* path);

/* FP64 integration with an optional per-cell step dt_cells (device, n
 * entries); never uses the surrogate.  Same layout as nrg_chem_step_device. */
NRG_API int nrg_chem_integrate(nrg_chem* h, long n, long ld, double dt, const double* dt_cells,
                               const double* T, const double* rho, const double* Y, const signed char* bc,
                               double* Y_prod, double* Y_prod2, double* E_f_prod, double* T_after,
                               unsigned char* status, void* stream, nrg_chem_stats* stats);

/* Measured dependent-FMA FP64 throughput of the current device, TFLOP/s. */
NRG_API int nrg_fp64_peak_tflops(double* tflops);

#ifdef __cplusplus
}
#endif
#endif
