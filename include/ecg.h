/*
 * ecg.h -- C ABI of the B200 (sm_100a) euler_compare hot path.
 *
 * The reference keeps its hot path as internal C++ functions inside one
 * translation unit (amrex/apps/euler_compare/src/euler_compare_app.cpp:41-62);
 * each entry point below replaces one of those calls so that the AMReX driver
 * (amrex/apps/euler_compare/src/euler_compare/app/driver_main.hpp) can keep its
 * call sites, ParmParse selectors and MultiFab layout.  Plain C types only: no
 * CUDA or torch types cross this boundary.
 *
 * Ownership: a context owns every device buffer (state, scratch, Krylov basis).
 * The host MultiFab is copied only by ecg_upload_state / ecg_download_state.
 * Threading: one context per host thread; a context is not internally
 * thread-safe.  Errors: every call returns an ecg_status; nothing throws
 * across the ABI.  IMEX solver outcomes (the reference's solver_status
 * strings) are reported in ecg_imex_diag.solver_status, as the reference
 * reports them in ImexStepDiagnostics, and do not make the call fail.
 */
#ifndef ECG_H
#define ECG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ECG_ABI_VERSION 1

typedef enum ecg_status {
  ECG_OK = 0,
  ECG_ERR_BAD_ARG = 1,      /* invalid pointer, size or option */
  ECG_ERR_CUDA = 2,         /* a CUDA runtime call failed; see ecg_last_error */
  ECG_ERR_TIMEOUT = 3,      /* a bounded device-side wait gave up */
  ECG_ERR_NO_DEVICE = 4,    /* no usable sm_100 device */
  ECG_ERR_UNSUPPORTED = 5,  /* configuration outside the rebuilt hot path */
  ECG_ERR_NOT_READY = 6,    /* state not uploaded yet */
  ECG_ERR_IO = 7            /* an output file could not be written */
} ecg_status;

/* Mirrors ProblemKind (core/solver_types.hpp:2-10), same order. */
typedef enum ecg_problem {
  ECG_PROBLEM_ADVECTION_BLOB = 0,
  ECG_PROBLEM_TORO1 = 1,
  ECG_PROBLEM_GRESHO_VORTEX = 2,
  ECG_PROBLEM_RIEMANN_QUADRANT = 3,
  ECG_PROBLEM_ISENTROPIC_VORTEX = 4,
  ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D = 5,
  ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL = 6,
  /* No counterpart in ProblemKind: a Mach 1.22 planar shock at x = 0.5 running
   * into (rho, p) = (1, 1) and a circular bubble (r = 0.25 at (1, 0.5),
   * rho = 0.138, p = 1) on [0,4] x [0,1], post-shock inflow on the left,
   * outflow on the right, reflecting walls at y = 0 and y = 1, gamma = 1.4.
   * The reference's config reader rejects this geometry for
   * shock_density_bubble_2d (config_reader.hpp:288-298).  Both the explicit
   * and the IMEX method run it; the IMEX step uses the bubble's source-map
   * boundary policy with a reflecting wall at both y ends. */
  ECG_PROBLEM_SHOCK_BUBBLE_MACH122 = 7
} ecg_problem;

/* Mirrors RiemannKind (core/solver_types.hpp:11). */
typedef enum ecg_riemann {
  ECG_RIEMANN_RUSANOV = 0,
  ECG_RIEMANN_HLLC = 1,
  ECG_RIEMANN_LOWMACH_HLLC = 2,
  ECG_RIEMANN_XIE_AM_HLLC_P = 3
} ecg_riemann;

/* Mirrors MethodKind (core/solver_types.hpp:12). */
typedef enum ecg_method { ECG_METHOD_EXPLICIT = 0, ECG_METHOD_IMEX = 1 } ecg_method;

/* Mirrors SlopeLimiterKind (core/solver_types.hpp:14). */
typedef enum ecg_limiter {
  ECG_LIMITER_MINMOD = 0,
  ECG_LIMITER_MC = 1,
  ECG_LIMITER_VANLEER = 2
} ecg_limiter;

/* RunConfig::field_boundary string (core/run_config.hpp:48). */
typedef enum ecg_field_boundary {
  ECG_FIELD_BOUNDARY_OUTFLOW = 0,
  ECG_FIELD_BOUNDARY_EXACT_DIRICHLET = 1
} ecg_field_boundary;

/*
 * Numeric mirror of RunConfig (core/run_config.hpp:2-55).  String selectors
 * become the enums above.  ecg_default_run_config fills RunConfig's defaults.
 */
typedef struct ecg_run_config {
  int32_t n_cell[2];
  int32_t is_periodic[2];
  double prob_lo[2];
  double prob_hi[2];
  int32_t max_step;
  int32_t spatial_order;
  int32_t toro_test;
  int32_t problem;         /* ecg_problem */
  int32_t riemann;         /* ecg_riemann */
  int32_t method;          /* ecg_method */
  int32_t slope_limiter;   /* ecg_limiter */
  int32_t field_boundary;  /* ecg_field_boundary */
  double stop_time;
  double gamma;
  double cfl;
  double imex_cfl;
  double imex_acoustic_cfl_cap;
  double imex_solver_tol;
  double velocity_x;
  double velocity_y;
  double density_inner;
  double density_outer;
  double pressure;
  double mach;
  double blob_cx;
  double blob_cy;
  double blob_radius;
  double vortex_cx;
  double vortex_cy;
  double isentropic_vortex_strength;
  double riemann_interface_x;
  double riemann_interface_y;
  int32_t imex_solver_max_iter;
  int32_t imex_acoustic_startup;
  int32_t imex_picard_iterations;
  int32_t imex_picard_extra_iterations;
} ecg_run_config;

/* Arithmetic contract of the FP64 stencil kernels. */
typedef enum ecg_arith {
  /* Default: nvcc contracts a*b+c into FMA.  Per step within 1e-12 relative
   * of the reference CPU build. */
  ECG_ARITH_FAST = 0,
  /* No contraction, IEEE division and square root, the reference's operation
   * order: bit-identical to the reference CPU build (gcc, x86-64, no FMA). */
  ECG_ARITH_EXACT = 1
} ecg_arith;

/* Precision of the IMEX pressure solve. */
typedef enum ecg_imex_precision {
  ECG_IMEX_FP64 = 0,   /* all-FP64 GMRES */
  ECG_IMEX_MIXED = 1   /* FP32-stored Krylov basis, FP64 arithmetic, restarts from the true FP64 residual */
} ecg_imex_precision;

typedef struct ecg_gpu_options {
  int32_t device;           /* CUDA device ordinal */
  int32_t arith;            /* ecg_arith */
  int32_t imex_precision;   /* ecg_imex_precision */
  int32_t mixed_inner_max_iter;  /* mixed: iterations per FP32-basis cycle (0: no limit) */
  double mixed_inner_rtol;       /* mixed: restart once the recurrence residual fell by this factor, after at
                                    least 16 iterations of the cycle (0: never; negative, the default: 1e-4
                                    when the solve keeps its basis in shared memory, an L2-resident system,
                                    1e-3 otherwise, where shorter cycles keep the streamed basis short) */
  int32_t mixed_max_refinements; /* mixed: cycles, each opened with the true FP64 residual */
  int32_t tile_x;           /* column-strip kernel: rows each warp marches (0: sized so the grid fills one wave) */
  int32_t tile_y;           /* explicit kernel: 0 default (column strips, x- and y-faces
                               evaluated together, rows staged through shared memory by
                               cp.async), 3 the same with rows loaded into registers, 2
                               column strips with faces one at a time, 1 square 16x16
                               tiles, 8 or 16 the 32 x tile_y tiles */
  int32_t mixed_reorth;     /* mixed: Gram-Schmidt second pass (DGKS) of the FP32-basis cycles:
                               1 when ||w'|| < ||w||/sqrt(2), as the FP64 solve; 0 (default) only
                               when ||w'|| < 1e-3 ||w||, where the Pythagorean norm would lose digits */
  void* stream;             /* cudaStream_t to run on, NULL = context-owned stream */
  int32_t deterministic;    /* 1: the GMRES grid sums run in a fixed block order, so repeated IMEX steps on
                               the same inputs give the same bits (a little slower); 0 (default): atomic
                               accumulation, whose order can change the last bits from run to run */
  int32_t mixed_min_iterations; /* mixed: a step whose previous step's pressure solves took fewer iterations
                                   than this on average solves on the FP64 basis (short solves stay in L2,
                                   where the FP32 basis saves nothing and its restart cycle costs
                                   iterations); 0: always the FP32 basis.  Default 8. */
} ecg_gpu_options;

/* Diagnostics (core/basic_diagnostics.hpp:3-7). */
typedef struct ecg_diagnostics {
  double rho_min;
  double pressure_min;
  int32_t nonfinite_count;
} ecg_diagnostics;

/* AdmissibilityDiagnostics (core/basic_diagnostics.hpp:9-17). */
typedef struct ecg_admissibility {
  double rho_min;
  double pressure_min;
  double internal_energy_min;
  int32_t nonfinite_count;
  int32_t density_failure_count;
  int32_t pressure_failure_count;
  int32_t internal_energy_failure_count;
} ecg_admissibility;

/* ImexTimeStepDiagnostics (core/problem_metrics.hpp:14-19). */
typedef struct ecg_imex_timestep_diag {
  double material_rate_max;
  double acoustic_rate_max;
  int32_t acoustic_startup_used;
  int32_t acoustic_cap_used;
} ecg_imex_timestep_diag;

/* ImexStepDiagnostics solver_status strings (imex/imex_source_map_step.hpp:398-567). */
typedef enum ecg_solver_status {
  ECG_SOLVER_NOT_RUN = 0,
  ECG_SOLVER_CONVERGED_ABSOLUTE = 1,
  ECG_SOLVER_CONVERGED_RELATIVE = 2,
  ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED = 3,
  ECG_SOLVER_GMRES_BREAKDOWN_NOT_CONVERGED = 4,
  ECG_SOLVER_LINEAR_RESIDUAL_NONFINITE = 5,
  ECG_SOLVER_SOURCE_MAP_PRESSURE_ROW_NONFINITE = 6,
  ECG_SOLVER_SOURCE_MAP_LAGGED_MOMENTUM_NONFINITE = 7,
  ECG_SOLVER_DENSITY_DENOMINATOR_FLOOR_USED = 8,
  ECG_SOLVER_UNSUPPORTED_MPI = 9
} ecg_solver_status;

/*
 * Numeric fields of ImexStepDiagnostics (core/imex_diagnostics.hpp:5-171)
 * that euler_imex_bdltv20_o1_source_map_picard_one_step fills
 * (imex/imex_source_map_step.hpp:300-616).  The label strings of that record
 * are constants of the method and are not repeated here.
 */
typedef struct ecg_imex_diag {
  int32_t solver_status;              /* ecg_solver_status */
  int32_t linear_solver_status_last;  /* ecg_solver_status */
  int32_t solver_iterations;          /* summed over Picard solves */
  int32_t picard_pressure_solves_used;
  int32_t source_picard_iterations_used;
  int32_t kinetic_lag_update_count;
  int32_t kinetic_lag_nonfinite_count;
  int32_t pressure_matrix_rows;
  int32_t pressure_matrix_nonzeros;
  int32_t pressure_matrix_max_row_width;
  int32_t density_denominator_floor_count;
  int32_t nonfinite_count;
  int32_t positivity_failure_count;
  int32_t face_enthalpy_denominator_guard_count;
  int32_t face_enthalpy_nonfinite_count;
  int32_t energy_flux_nonfinite_count;
  int32_t gmres_inner_iterations;     /* mixed precision: iterations over the FP32 basis, all cycles (not in the reference) */
  int32_t gmres_refinements;          /* mixed precision: cycles, each opened with the true FP64 residual (not in the reference) */
  double solver_initial_residual;
  double solver_initial_rhs_norm;
  double solver_residual;
  double solver_relative_residual;
  double pressure_linear_residual_linf;
  double pressure_linear_residual_relative_linf;
  double kinetic_jacobian_abs_max;
  double pressure_matrix_symmetry_linf;
  double pressure_picard_delta_linf;
  double source_picard_delta_l2_relative_to_pmax;
  double pressure_energy_residual_before_linf;
  double coupled_residual_l1_final;
  double coupled_residual_linf_final;
  double coupled_residual_relative_linf_final;
  double pressure_energy_residual_l1;
  double pressure_energy_residual_linf;
  double pressure_energy_residual_relative_linf;
  double rho_min;
  double pressure_min;
  double internal_energy_min;
  double trial_density_min;
  double solved_pressure_min;
  double solved_pressure_max;
  double eos_pressure_min;
  double eos_pressure_max;
  double internal_energy_max;
  double momentum_correction_linf;
  double energy_correction_linf;
  double energy_flux_linf;
  double energy_flux_divergence_linf;
  double eq78_divergence_linf;
  double eq78_divergence_scaled_linf;
  double energy_closeout_delta_l1;
  double energy_closeout_delta_linf;
  double gmres_vector_bytes;          /* bytes the step's GMRES sweeps read and write, counted from the iterations
                                         run: every sweep over a vector of n rows counts n entries of its width
                                         (not in the reference) */
  int32_t gmres_fp64_fallbacks;       /* mixed precision: Picard solves the FP32-basis cycles left above the
                                         tolerance and the FP64 solve finished from their iterate (not in the
                                         reference) */
  int32_t gmres_fp32_basis;           /* mixed precision: 1 when the step's solves ran on the FP32 basis, 0 when
                                         mixed_min_iterations sent them to the FP64 solve (not in the reference) */
} ecg_imex_diag;

/* Result of a device-resident time loop (driver_main.hpp:224-333). */
typedef struct ecg_run_result {
  int32_t steps;
  int32_t failed;               /* 0 = ok */
  int32_t failure_code;         /* ecg_failure_* below */
  int32_t hllc_degenerate_star_count;
  int32_t imex_solver_iterations_max;
  double time;
  double dt_min;
  double dt_max;
  double dt_sum;
  ecg_diagnostics diagnostics;  /* after the last step */
} ecg_run_result;

/* Direct BDLTV20 T1/S2 driver (imex/imex_bdltv20_direct_driver.hpp:44-779):
 * the euler.bdltv20_paper_t1_s2 settings of RunConfig (core/run_config.hpp:33-52). */
typedef enum ecg_paper_mode {
  ECG_PAPER_OFF = 0,
  ECG_PAPER_TORO_X_EXACT_DIRICHLET_Y_PERIODIC = 1, /* "toro_x_exact_dirichlet_y_periodic_2d" */
  ECG_PAPER_TORO_XY_EXACT_DIRICHLET = 2,           /* "toro_xy_exact_dirichlet_2d" */
  ECG_PAPER_GRESHO_EXACT_DIRICHLET = 3,            /* "gresho_exact_dirichlet_2d" */
  ECG_PAPER_ISENTROPIC_VORTEX_PERIODIC = 4,        /* "isentropic_vortex_periodic_2d" */
  ECG_PAPER_ADVECTION_BLOB_PERIODIC = 5            /* "advection_blob_periodic_2d" */
} ecg_paper_mode;

typedef struct ecg_paper_options {
  int32_t mode;        /* ecg_paper_mode */
  int32_t max_steps;   /* bdltv20_paper_t1_s2_max_steps */
  double epsilon;      /* bdltv20_paper_epsilon */
  double fixed_dt;     /* bdltv20_paper_t1_s2_dt: > 0 fixed, < 0 eq79 CFL mode */
} ecg_paper_options;

/* The key=value report of run_bdltv20_paper_t1_s2 (:686-777), numeric fields. */
typedef struct ecg_paper_result {
  int32_t steps;
  int32_t solver_failure_count;
  int32_t gmres_iterations_max;
  int32_t enthalpy_guard_count;
  int32_t nonfinite_count;
  int32_t nonpositive_count;
  int32_t passed;                 /* bdltv20_paper_t1_s2_status == passed */
  int32_t pad;
  double final_time;
  double pressure_residual_linf_max;
  double pressure_relative_residual_linf_max;
  double rho_min;
  double pressure_min;
  double density_l1_error;
  double velocity_l1_error;
  double pressure_l1_error;
  double density_l2_error;
  double velocity_l2_error;
  double pressure_l2_error;
  double density_linf_error;
  double pressure_linf_error;
} ecg_paper_result;

/* Failure categories of the driver loop (driver_main.hpp:216-340). */
enum {
  ECG_FAILURE_NONE = 0,
  ECG_FAILURE_NONFINITE_STATE = 1,
  ECG_FAILURE_NONPOSITIVE_DENSITY = 2,
  ECG_FAILURE_NONPOSITIVE_PRESSURE = 3,
  ECG_FAILURE_INVALID_TIME_STEP = 4,
  ECG_FAILURE_IMEX_SOLVER = 5,
  ECG_FAILURE_MAX_STEP_BEFORE_STOP_TIME = 6
};

typedef struct ecg_ctx ecg_ctx;

/* ---- library ---------------------------------------------------------- */
int32_t ecg_abi_version(void);
const char* ecg_status_str(ecg_status s);
/* The reference's exact solver_status string for an ecg_solver_status. */
const char* ecg_solver_status_str(int32_t solver_status);
/* RunConfig defaults (core/run_config.hpp:2-55). */
void ecg_default_run_config(ecg_run_config* cfg);
void ecg_default_gpu_options(ecg_gpu_options* opt);

/* ---- context ---------------------------------------------------------- */
/* Validates cfg as read_config does for the rebuilt path
 * (core/config_reader.hpp:123-324) and allocates the device state. */
ecg_status ecg_create(ecg_ctx** out, const ecg_run_config* cfg, const ecg_gpu_options* opt);
void ecg_destroy(ecg_ctx* ctx);
const char* ecg_last_error(const ecg_ctx* ctx);

/*
 * State exchange with one AMReX FArrayBox / Array4 covering the domain.
 * Element (i, j, comp) lives at base[(i - lo_x) + (j - lo_y) * jstride + comp * nstride]
 * (AMReX_Array4.H), comp in {Rho, Mx, My, E} (euler_compare_app.cpp:47).
 * Only the valid cells [0, nx) x [0, ny) are copied; ghost cells are derived
 * on the device from the boundary conditions.  A box in pinned (page-locked)
 * memory is copied directly; a pageable one (an FArrayBox as AMReX allocates
 * it) crosses through the context's own pinned staging copy of the state,
 * which host threads fill or drain band by band while the previous band
 * crosses (allocated on the first pageable call: 2 x 32 bytes a cell).
 */
ecg_status ecg_upload_state(ecg_ctx* ctx, const double* base, int32_t lo_x, int32_t lo_y,
                            int64_t jstride, int64_t nstride);
ecg_status ecg_download_state(ecg_ctx* ctx, double* base, int32_t lo_x, int32_t lo_y,
                              int64_t jstride, int64_t nstride);
/* Same with base in device memory (e.g. a torch CUDA tensor). */
ecg_status ecg_upload_state_device(ecg_ctx* ctx, const double* base, int32_t lo_x, int32_t lo_y,
                                   int64_t jstride, int64_t nstride);
ecg_status ecg_download_state_device(ecg_ctx* ctx, double* base, int32_t lo_x, int32_t lo_y,
                                     int64_t jstride, int64_t nstride);
/* initialize_state (problems/problem_initialization.hpp:420-435): writes the
 * problem's initial condition into the context's state on the device (one
 * kernel; no host data).  Transcendental profiles (Gresho, isentropic vortex)
 * agree with the reference to rounding of log/exp/pow; the others exactly in
 * ECG_ARITH_EXACT. */
ecg_status ecg_initialize_state(ecg_ctx* ctx);
/* Fills the whole ghosted box [-2, nx+2) x [-2, ny+2) (4 planes, jstride
 * nx+4, nstride (nx+4)(ny+4)) as fill_problem_ghosts does
 * (problems/boundary_conditions.hpp:202-219). */
ecg_status ecg_fill_problem_ghosts(ecg_ctx* ctx, double time, double* ghosted_host);

/* Synchronises the context's stream. */
ecg_status ecg_synchronize(ecg_ctx* ctx);

/* ---- hot path --------------------------------------------------------- */
/* euler_fv_one_step (numerics/explicit_update.hpp:58-102): one forward-Euler
 * MUSCL + Riemann-flux update of the device state.  Returns the
 * count_hllc_degenerate_star_states value (explicit_update.hpp:2-56) through
 * hllc_degenerate_count when non-NULL. */
ecg_status ecg_euler_fv_one_step(ecg_ctx* ctx, double dt, double time, int32_t* hllc_degenerate_count);
/* euler_fv_one_step on a HOST box (the Array4 description of
 * ecg_upload_state for `in` and `out`, which may be the same array): the
 * upload, the step and the download in one call, pipelined over bands of
 * rows: each upload chunk carries the rows its band's step reads that no
 * earlier chunk held (under periodic y the grid's last two rows, the first
 * band's ghosts, cross first), later chunks cross while a band is stepped,
 * and finished bands cross back.  The result depends only on `in`, never on
 * what the context's device state held before the call.  Pinned host memory lets the copies overlap;
 * pageable boxes go through the staging copy described above.
 * The context's state becomes the new state, and its fused CFL / diagnostic
 * reductions are those of `out`.  No counterpart in the reference (a drop-in
 * for its host-MultiFab call sequence upload -> euler_fv_one_step ->
 * download). */
ecg_status ecg_euler_fv_one_step_host(ecg_ctx* ctx, const double* in, double* out, int32_t lo_x, int32_t lo_y,
                                      int64_t jstride, int64_t nstride, double dt, double time, int32_t* degenerate);
/* compute_euler_dt (numerics/diagnostic_metrics_timestep.hpp:227-260). */
ecg_status ecg_compute_euler_dt(ecg_ctx* ctx, double time, double* dt);
/* compute_imex_dt (numerics/diagnostic_metrics_timestep.hpp:272-326). */
ecg_status ecg_compute_imex_dt(ecg_ctx* ctx, double time, double* dt, ecg_imex_timestep_diag* diag);
/* compute_diagnostics (numerics/diagnostic_metrics_timestep.hpp:18-47). */
ecg_status ecg_compute_diagnostics(ecg_ctx* ctx, ecg_diagnostics* out);
/* compute_admissibility_diagnostics (numerics/diagnostic_metrics_timestep.hpp:49-111). */
ecg_status ecg_compute_admissibility_diagnostics(ecg_ctx* ctx, ecg_admissibility* out);
/* euler_imex_bdltv20_o1_source_map_picard_one_step
 * (imex/imex_source_map_step.hpp:300-616): the IMEX T1/S2 BDLTV20 step with
 * the GMRES pressure solve.  The state is updated only when the step
 * succeeds, as in the reference. */
ecg_status ecg_imex_step(ecg_ctx* ctx, double dt, ecg_imex_diag* out);
/* The driver's time loop (app/driver_main.hpp:224-333) kept on the device:
 * dt, step and fail-fast diagnostics per step, no host round trip for the
 * explicit method. */
ecg_status ecg_run(ecg_ctx* ctx, int32_t max_step, double stop_time, ecg_run_result* out);
/* run_bdltv20_paper_t1_s2 (imex/imex_bdltv20_direct_driver.hpp:44-779): the
 * direct T1/S2 driver of the report rows, on the device.  It initialises the
 * context's state from the configured problem (ε-scaled energy), steps to
 * stop_time or opts->max_steps, and leaves the final (ε-scaled) state in the
 * context.  The configuration must satisfy the reference's checks for the
 * mode (core/config_reader.hpp:133-258), else ECG_ERR_BAD_ARG. */
ecg_status ecg_paper_t1s2_run(ecg_ctx* ctx, const ecg_paper_options* opts, ecg_paper_result* out);

/* ---- output writers (io/output_cases.hpp) -------------------------------- */
/* The run's files in the reference's formats: columns computed on the device
 * in the reference's arithmetic, rows printed with %.17g (its
 * std::setprecision(17)) by all host threads. */
typedef struct ecg_output_info {
  int32_t step;
  int32_t pad;
  double time;
  /* Gresho file only: the IMEX admissibility run minima (NaN for explicit runs,
   * as the driver passes them, app/driver_main.hpp:350-358) */
  double trial_density_min, trial_pressure_min, trial_internal_energy_min;
} ecg_output_info;

typedef struct ecg_bubble_metrics {  /* ShockDensityBubbleMetrics, io/output_cases.hpp:253-265 */
  double rho_min, rho_max, pressure_min, pressure_max, internal_energy_min;
  double density_bubble_centroid_x, density_bubble_centroid_y, density_bubble_area;
  double density_bubble_area_threshold, schlieren_max;
  int32_t nonfinite_count;
  int32_t pad;
} ecg_bubble_metrics;

typedef struct ecg_bubble_run {  /* run-level fields of the bubble summary, from the driver */
  int32_t steps_accepted, steps_rejected;
  double time, wall_time_sec, dt_min, dt_max, dt_mean;
  const char* status;
  const char* failure_category;
  const char* snapshot_status;
  const char* snapshot_dir;
  const char* snapshot_times;
} ecg_bubble_run;

/* write_gresho_final_csv / write_toro_final_csv / write_riemann_quadrant_final_csv
 * / write_advection_blob_final_csv (io/output_cases.hpp:16-216), chosen by the
 * configured problem; ECG_ERR_UNSUPPORTED for other problems. */
ecg_status ecg_write_final_csv(ecg_ctx* ctx, const char* path, const ecg_output_info* info);
/* compute_shock_density_bubble_metrics (io/output_cases.hpp:329-403) of the
 * current state: one device reduction (the area and centroid sums are
 * summed in a different order than the reference's loop). */
ecg_status ecg_shock_bubble_metrics(ecg_ctx* ctx, double time, ecg_bubble_metrics* out);
/* write_shock_density_bubble_snapshot (io/output_cases.hpp:405-487) of the
 * current state into dir.  async != 0: the columns are copied on a side
 * stream and a host thread writes the file while the caller keeps stepping
 * (two in flight; ecg_output_wait joins them). */
ecg_status ecg_write_bubble_snapshot(ecg_ctx* ctx, const char* dir, int32_t index, int32_t step, double time,
                                     int32_t async);
/* Waits for the asynchronous snapshots; *failed = files not written. */
ecg_status ecg_output_wait(ecg_ctx* ctx, int32_t* failed);
/* write_shock_density_bubble_summary_csv (io/output_cases.hpp:489-588) with
 * the metrics of the current state. */
ecg_status ecg_write_bubble_summary_csv(ecg_ctx* ctx, const char* path, const ecg_bubble_run* run);

/* ---- slabs of a grid split along x (several GPUs) ------------------------ */
/* No counterpart in the reference (it runs one box on one process).  A slab
 * context holds columns [x0, x1) of the grid `cfg` describes, with the whole
 * grid's dx bit for bit and the whole grid's problem definition; halo_lo /
 * halo_hi mark the x sides whose two ghost columns are a neighbour slab's edge
 * columns (periodic x: every side).  Explicit method only, and no
 * exact-state Dirichlet rings (ECG_ERR_UNSUPPORTED).  Halo blocks are device
 * buffers of 8 ny doubles: 4 planes (rho, mx, my, E) of ny rows x 2 columns,
 * columns in increasing x.  A step reads the blocks bound last; y ghosts of
 * the halo columns follow the y policy, as in the undivided grid. */
ecg_status ecg_create_slab(ecg_ctx** out, const ecg_run_config* cfg, const ecg_gpu_options* opt, int32_t x0,
                           int32_t x1, int32_t halo_lo, int32_t halo_hi);
/* Binds the halo blocks the steps read: lo = columns -2, -1; hi = nx, nx+1. */
ecg_status ecg_slab_bind_halo(ecg_ctx* ctx, const double* lo, const double* hi);
/* Writes the slab's edge columns of the current state, on the context's
 * stream: lo <- columns 0, 1 (the left neighbour's hi halo), hi <- columns
 * nx-2, nx-1 (the right neighbour's lo halo).  Either may be NULL. */
ecg_status ecg_slab_pack(ecg_ctx* ctx, double* lo, double* hi);

/* ---- measurement -------------------------------------------------------- */
/* No counterpart in the reference: the FP64 FMA throughput of `device` in
 * TFLOP/s (independent fma chains at full occupancy, best of five timed
 * launches), the denominator of the explicit step's FP64 roofline. */
ecg_status ecg_measure_fp64_peak(int32_t device, double* tflops);

/* No counterpart in the reference: the bounded wait of the GMRES grid barrier
 * (the only device-side wait here), checked on its own.  4 blocks pass one
 * barrier; then block 0 leaves without arriving at the next, and the other 3
 * give up after spin_limit polls (1 .. 2^25) instead of hanging.  Reports how
 * many blocks passed the first barrier (4) and how many timed out at the
 * second (3); the device stays usable. */
ecg_status ecg_check_grid_barrier_timeout(int32_t device, int64_t spin_limit, int32_t* passed_first,
                                          int32_t* timed_out);

/* ---- adjoint of the explicit step --------------------------------------- */
/* Vector-Jacobian product of U1 = euler_fv_one_step(U0; dt) with dt held
 * fixed: gU0 = (dU1/dU0)^T gU1.  All arrays are device memory holding 4
 * planes of nx*ny doubles (component-major, i fastest).  Boundary conditions
 * are the context's.  No counterpart in the reference (its code has no
 * adjoint). */
ecg_status ecg_explicit_step_vjp_device(ecg_ctx* ctx, const double* u0, double dt,
                                        const double* g_u1, double* g_u0);
/* Forward step on caller-provided device planes (same layout), used by the
 * checkpointed adjoint: u1 = euler_fv_one_step(u0; dt). */
ecg_status ecg_explicit_step_device(ecg_ctx* ctx, const double* u0, double dt, double* u1);

/* ---- allocation-free explicit step -------------------------------------- */
/* No counterpart in the reference: euler_fv_one_step
 * (numerics/explicit_update.hpp:58-102) on caller-owned DEVICE arrays with no
 * context and no device or host allocation, for callers that cannot allocate
 * inside their time loop (an AMReX GPU build whose arena reserves most of HBM
 * at start-up and whose stream pipeline a cudaFree would synchronise).
 * state_in/state_out: device arrays in the Array4 layout of ecg_upload_state
 * (same lo, jstride, nstride for both) that share no byte (4 planes of nstride
 * doubles from each base; overlap is ECG_ERR_BAD_ARG); ghost cells come from
 * the boundary conditions of cfg.  opt may be NULL (defaults; opt->stream is
 * the stream the work is queued on, opt->device the device).  Scratch lives
 * in one static device array of ECG_NOALLOC_SCRATCH_BYTES per device: the
 * exact-Dirichlet problems need 32*(nx+4)*(ny+4) bytes of it for their ghost
 * ring and are rejected with ECG_ERR_BAD_ARG beyond that; the others have no
 * size limit.  Calls that overlap in time on one device race on that scratch.
 * The first call on a device looks the scratch up (make it before any stream
 * capture) and keeps its address until exit: after a cudaDeviceReset of that
 * device the entry point must not be called on it again.  hllc_degenerate_count (may be NULL) synchronises the stream.  On
 * failure a message is written to err (err_len bytes, may be NULL). */
#define ECG_NOALLOC_SCRATCH_BYTES (8u << 20)
ecg_status ecg_euler_fv_one_step_noalloc(const ecg_run_config* cfg, const ecg_gpu_options* opt,
                                         const double* state_in, double* state_out, int32_t lo_x, int32_t lo_y,
                                         int64_t jstride, int64_t nstride, double dt, double time,
                                         int32_t* hllc_degenerate_count, char* err, int32_t err_len);

/* ---- batched independent solves ----------------------------------------- */
/* Many explicit O2 solves of uneven grid sizes advanced together by one
 * persistent launch per step (captured in a CUDA graph).  Each solve keeps
 * its own dt (compute_euler_dt per solve).  No counterpart in the reference,
 * which runs one solve per process. */
typedef struct ecg_batch ecg_batch;
typedef struct ecg_batch_result {
  int32_t steps;
  int32_t failed;
  int32_t hllc_degenerate_star_count;
  int32_t pad;
  double time;
  ecg_diagnostics diagnostics;
} ecg_batch_result;
ecg_status ecg_batch_create(ecg_batch** out, int32_t nsolve, const ecg_run_config* cfgs,
                            const ecg_gpu_options* opt);
void ecg_batch_destroy(ecg_batch* b);
ecg_status ecg_batch_upload(ecg_batch* b, int32_t solve, const double* base, int32_t lo_x, int32_t lo_y,
                            int64_t jstride, int64_t nstride);
ecg_status ecg_batch_download(ecg_batch* b, int32_t solve, double* base, int32_t lo_x, int32_t lo_y,
                              int64_t jstride, int64_t nstride);
/* Advances every solve by `steps` steps (each solve stops at its stop_time). */
ecg_status ecg_batch_run(ecg_batch* b, int32_t steps, ecg_batch_result* per_solve);
const char* ecg_batch_last_error(const ecg_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* ECG_H */
