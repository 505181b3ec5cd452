/*
 * ecg_bridge.hpp: the euler_compare driver's hot-path calls over libecg.so.
 *
 * A maintainer adds one line to amrex/apps/euler_compare/src/euler_compare_app.cpp,
 * after the numerics headers and before "euler_compare/app/driver_main.hpp":
 *
 *     #include "ecg_bridge.hpp"
 *
 * and links the executable with -lecg.  The functions below live in namespace
 * ecg_bridge, and the macros at the end of this header send the driver's calls
 * of the six names to them (an overload next to the originals would tie with
 * them: argument-dependent lookup finds the originals through RunConfig).  The
 * originals stay compiled and serve every call not listed here
 * (configuration, initialisation, ghost fills of the host box, writers); the
 * macros apply only to code after this header, i.e. driver_main.hpp.
 *
 * Replaced (paths under src/euler_compare/):
 *   euler_fv_one_step                          numerics/explicit_update.hpp:58-102
 *   compute_euler_dt                           numerics/diagnostic_metrics_timestep.hpp:227-260
 *   compute_imex_dt                            numerics/diagnostic_metrics_timestep.hpp:272-326
 *   compute_diagnostics                        numerics/diagnostic_metrics_timestep.hpp:18-47
 *   compute_admissibility_diagnostics          numerics/diagnostic_metrics_timestep.hpp:49-111
 *   euler_imex_bdltv20_o1_source_map_picard_one_step
 *                                              imex/imex_source_map_step.hpp:300-616
 *
 * State.  One device context per run, created by the first bridged call from
 * the RunConfig, which uploads the MultiFab's valid box.  After every step the
 * new valid box is copied back into the MultiFab, because the driver reads it
 * between steps (mass and energy sums, snapshots, plot files, the final CSV),
 * so the MultiFab and the device agree after every bridged call.  The bridge
 * assumes the valid cells change only through bridged calls after the first
 * one, as in run_application; code that changes them otherwise calls
 * ecg_bridge::invalidate(), and the next bridged call uploads again.  The
 * copies use the FArrayBox memory as AMReX allocated it: the bridge does not
 * page-lock memory it does not own.
 *
 * Device path, from ParmParse (all optional):
 *   ecg.arith          = fast (default: FMA contraction, 1e-12 per step) | exact
 *                        (no contraction, IEEE division: the reference's bits)
 *   ecg.imex_precision = fp64 (default) | mixed (FP32-stored Krylov basis)
 *   ecg.device         = CUDA device ordinal (default 0)
 *   ecg.deterministic  = 0 (default) | 1 (GMRES sums in a fixed order)
 *   ecg.mixed_min_iterations = 8 (default): with mixed, a step after solves
 *                        that averaged fewer iterations solves on the FP64
 *                        basis; 0 keeps the FP32 basis on every step
 *
 * Errors from the library end the run through amrex::Abort with its message.
 */
#pragma once

#include <cstdint>
#include <string>

#include "ecg.h"

namespace ecg_bridge {

struct Session {
  ecg_ctx* ctx = nullptr;
  bool resident = false;  // the device holds the MultiFab's current valid cells
  ~Session()
  {
    if (ctx) ecg_destroy(ctx);
  }
};

inline Session& session()
{
  static Session s;
  return s;
}

// The next bridged call uploads the MultiFab again.
inline void invalidate() { session().resident = false; }

inline void check(ecg_status st, const char* what)
{
  if (st == ECG_OK) return;
  std::string msg = std::string("ecg_bridge: ") + what + ": " + ecg_status_str(st);
  if (session().ctx) msg += std::string(" (") + ecg_last_error(session().ctx) + ")";
  amrex::Abort(msg);
}

namespace detail {

// RunConfig (core/run_config.hpp:2-55) -> ecg_run_config.  The enums keep the
// reference's orders (ProblemKind, RiemannKind, MethodKind, SlopeLimiterKind),
// so they convert by value.
inline ecg_run_config to_abi(const RunConfig& c)
{
  ecg_run_config r;
  ecg_default_run_config(&r);
  for (int d = 0; d < 2; ++d) {
    r.n_cell[d] = c.n_cell[d];
    r.is_periodic[d] = c.is_periodic[d];
    r.prob_lo[d] = c.prob_lo[d];
    r.prob_hi[d] = c.prob_hi[d];
  }
  r.max_step = c.max_step;
  r.spatial_order = c.spatial_order;
  r.toro_test = c.toro_test;
  r.problem = static_cast<int32_t>(c.problem);
  r.riemann = static_cast<int32_t>(c.riemann);
  r.method = static_cast<int32_t>(c.method);
  r.slope_limiter = static_cast<int32_t>(c.slope_limiter);
  r.field_boundary = c.field_boundary == "exact_dirichlet" ? ECG_FIELD_BOUNDARY_EXACT_DIRICHLET
                                                           : ECG_FIELD_BOUNDARY_OUTFLOW;
  r.stop_time = c.stop_time;
  r.gamma = c.gamma;
  r.cfl = c.cfl;
  r.imex_cfl = c.imex_cfl;
  r.imex_acoustic_cfl_cap = c.imex_acoustic_cfl_cap;
  r.imex_solver_tol = c.imex_solver_tol;
  r.velocity_x = c.velocity_x;
  r.velocity_y = c.velocity_y;
  r.density_inner = c.density_inner;
  r.density_outer = c.density_outer;
  r.pressure = c.pressure;
  r.mach = c.mach;
  r.blob_cx = c.blob_cx;
  r.blob_cy = c.blob_cy;
  r.blob_radius = c.blob_radius;
  r.vortex_cx = c.vortex_cx;
  r.vortex_cy = c.vortex_cy;
  r.isentropic_vortex_strength = c.isentropic_vortex_strength;
  r.riemann_interface_x = c.riemann_interface_x;
  r.riemann_interface_y = c.riemann_interface_y;
  r.imex_solver_max_iter = c.imex_solver_max_iter;
  r.imex_acoustic_startup = c.imex_acoustic_startup;
  r.imex_picard_iterations = c.imex_picard_iterations;
  r.imex_picard_extra_iterations = c.imex_picard_extra_iterations;
  return r;
}

inline ecg_gpu_options gpu_options()
{
  ecg_gpu_options o;
  ecg_default_gpu_options(&o);
  amrex::ParmParse pp("ecg");
  std::string s;
  if (pp.query("arith", s)) o.arith = s == "exact" ? ECG_ARITH_EXACT : ECG_ARITH_FAST;
  if (pp.query("imex_precision", s)) o.imex_precision = s == "mixed" ? ECG_IMEX_MIXED : ECG_IMEX_FP64;
  int v = 0;
  if (pp.query("device", v)) o.device = v;
  if (pp.query("deterministic", v)) o.deterministic = v;
  if (pp.query("mixed_min_iterations", v)) o.mixed_min_iterations = v;
  return o;
}

// Array4 of the MultiFab's single box: base, lower corner, strides
// (AMReX_Array4.H: p[(i - lo.x) + (j - lo.y) jstride + n nstride]).
template <class MF, class F>
inline void with_box(MF& mf, F&& f)
{
  int boxes = 0;
  for (amrex::MFIter mfi(mf); mfi.isValid(); ++mfi) {
    const auto a = mf.array(mfi);
    f(a.p, static_cast<int32_t>(a.begin.x), static_cast<int32_t>(a.begin.y), static_cast<int64_t>(a.jstride),
      static_cast<int64_t>(a.nstride));
    ++boxes;
  }
  if (boxes != 1) amrex::Abort("ecg_bridge: the state must be one box (amr.max_grid_size >= the domain)");
}

// The context of the run, with the MultiFab's valid cells on the device.
inline ecg_ctx* ready(const amrex::MultiFab& state, const RunConfig& c)
{
  Session& s = session();
  if (!s.ctx) {
    const ecg_run_config r = to_abi(c);
    const ecg_gpu_options o = gpu_options();
    check(ecg_create(&s.ctx, &r, &o), "ecg_create");
    s.resident = false;
  }
  if (!s.resident) {
    with_box(const_cast<amrex::MultiFab&>(state), [&](double* p, int32_t lx, int32_t ly, int64_t js, int64_t ns) {
      check(ecg_upload_state(s.ctx, p, lx, ly, js, ns), "ecg_upload_state");
    });
    s.resident = true;
  }
  return s.ctx;
}

// The device state after a step back into the MultiFab's valid cells.
inline void store(amrex::MultiFab& state, ecg_ctx* ctx)
{
  with_box(state, [&](double* p, int32_t lx, int32_t ly, int64_t js, int64_t ns) {
    check(ecg_download_state(ctx, p, lx, ly, js, ns), "ecg_download_state");
  });
}

}  // namespace detail

inline int euler_fv_one_step(amrex::MultiFab& state, const amrex::Geometry&, const RunConfig& cfg, amrex::Real dt,
                             amrex::Real time = 0)
{
  ecg_ctx* ctx = detail::ready(state, cfg);
  int32_t degenerate = 0;
  check(ecg_euler_fv_one_step(ctx, dt, time, &degenerate), "ecg_euler_fv_one_step");
  detail::store(state, ctx);
  return degenerate;
}

inline amrex::Real compute_euler_dt(const amrex::MultiFab& state, const amrex::Geometry&, const RunConfig& cfg,
                                    amrex::Real time)
{
  ecg_ctx* ctx = detail::ready(state, cfg);
  double dt = 0.0;
  check(ecg_compute_euler_dt(ctx, time, &dt), "ecg_compute_euler_dt");
  return dt;
}

inline amrex::Real compute_imex_dt(const amrex::MultiFab& state, const amrex::Geometry&, const RunConfig& cfg,
                                   amrex::Real time, ImexTimeStepDiagnostics& diagnostics)
{
  ecg_ctx* ctx = detail::ready(state, cfg);
  double dt = 0.0;
  ecg_imex_timestep_diag d;
  check(ecg_compute_imex_dt(ctx, time, &dt, &d), "ecg_compute_imex_dt");
  diagnostics.material_rate_max = d.material_rate_max;
  diagnostics.acoustic_rate_max = d.acoustic_rate_max;
  diagnostics.acoustic_startup_used = d.acoustic_startup_used;
  diagnostics.acoustic_cap_used = d.acoustic_cap_used;
  return dt;
}

inline Diagnostics compute_diagnostics(const amrex::MultiFab& state, const RunConfig& cfg)
{
  ecg_ctx* ctx = detail::ready(state, cfg);
  ecg_diagnostics d;
  check(ecg_compute_diagnostics(ctx, &d), "ecg_compute_diagnostics");
  Diagnostics out;
  out.rho_min = d.rho_min;
  out.pressure_min = d.pressure_min;
  out.nonfinite_count = d.nonfinite_count;
  return out;
}

inline AdmissibilityDiagnostics compute_admissibility_diagnostics(const amrex::MultiFab& state, const RunConfig& cfg)
{
  ecg_ctx* ctx = detail::ready(state, cfg);
  ecg_admissibility a;
  check(ecg_compute_admissibility_diagnostics(ctx, &a), "ecg_compute_admissibility_diagnostics");
  AdmissibilityDiagnostics out;
  out.rho_min = a.rho_min;
  out.pressure_min = a.pressure_min;
  out.internal_energy_min = a.internal_energy_min;
  out.nonfinite_count = a.nonfinite_count;
  out.density_failure_count = a.density_failure_count;
  out.pressure_failure_count = a.pressure_failure_count;
  out.internal_energy_failure_count = a.internal_energy_failure_count;
  return out;
}

// The IMEX T1/S2 source-map step.  Numbers come from the device step; the
// labels that name the scheme (operator, row stencil, equation set, orders,
// enthalpy and momentum policies) are the reference's, since the step is the
// same scheme, and the two that name the solver describe this one.  The
// solved-pressure check MultiFab of the original is not produced.
inline ImexStepDiagnostics euler_imex_bdltv20_o1_source_map_picard_one_step(amrex::MultiFab& state,
                                                                            const amrex::Geometry&,
                                                                            const RunConfig& cfg, amrex::Real dt,
                                                                            amrex::MultiFab* = nullptr)
{
  ecg_ctx* ctx = detail::ready(state, cfg);
  ecg_imex_diag d;
  check(ecg_imex_step(ctx, dt, &d), "ecg_imex_step");
  const bool committed = d.solver_status == ECG_SOLVER_CONVERGED_ABSOLUTE ||
                         d.solver_status == ECG_SOLVER_CONVERGED_RELATIVE;
  if (committed) detail::store(state, ctx);

  ImexStepDiagnostics o;
  const bool t1s2 = is_bdltv20_t1_s2_source_map_form(cfg.imex_form);
  o.solver = "b200_cooperative_gmres_source_map_pressure_row_matrix_free";
  o.pressure_solver_path = "device_single_grid_gmres";
  o.solver_status = ecg_solver_status_str(d.solver_status);
  o.linear_solver_status_last =
      d.linear_solver_status_last >= 0 ? ecg_solver_status_str(d.linear_solver_status_last) : "unset";
  o.pressure_operator_label = "bdltv20_o1_source_picard_eq49_50_52_eq76_77_zdrop_2d_pressure_row_no_eq51_claim";
  o.pressure_row_stencil =
      "eq49_76_lhs_enthalpy_eq50_77_rhs_star_energy_lagged_kinetic_star_momentum_eq52_host_sparse_zdrop_2d_no_eq51_"
      "claim";
  o.pressure_energy_form = to_string(cfg.imex_form);
  o.face_enthalpy_policy = "bdltv20_eq46_corrected_momentum_weighted_face_enthalpy_with_tolerance_guard";
  o.face_momentum_policy = "centered_eq54_eq71_72_corrected_normal_momentum";
  o.source_primary_paper = "bdltv20_2020_jcp_415_109486";
  o.source_equation_set =
      t1s2 ? "eq25_28_split_eq43_55_source_map_eq69_79_zdrop_2d_plus_eq87_89_conserved_minmod_explicit_advection"
           : "eq25_28_split_eq43_55_source_map_eq69_79_zdrop_2d";
  o.source_time_order = "first_order_time_t1";
  o.source_space_order = t1s2 ? "second_order_space_s2" : "first_order_space_s1";
  o.source_advection_reconstruction =
      t1s2 ? "bdltv20_eq87_89_conserved_variable_minmod_explicit_toro_vazquez_star_update"
           : "piecewise_constant_first_order_source_map_star_update";
  o.source_picard_iterations_config = cfg.imex_picard_iterations;
  o.picard_extra_iterations_requested = cfg.imex_picard_extra_iterations;
  o.solver_requested_relative_tol = cfg.imex_solver_tol;
  o.solver_requested_absolute_tol = cfg.imex_solver_tol;
  o.density_denominator_floor_value = 1.0e-14;

  o.solver_iterations = d.solver_iterations;
  o.picard_pressure_solves_used = d.picard_pressure_solves_used;
  o.source_picard_iterations_used = d.source_picard_iterations_used;
  o.kinetic_lag_update_count = d.kinetic_lag_update_count;
  o.kinetic_lag_nonfinite_count = d.kinetic_lag_nonfinite_count;
  o.pressure_matrix_rows = d.pressure_matrix_rows;
  o.pressure_matrix_nonzeros = d.pressure_matrix_nonzeros;
  o.pressure_matrix_max_row_width = d.pressure_matrix_max_row_width;
  o.density_denominator_floor_count = d.density_denominator_floor_count;
  o.nonfinite_count = d.nonfinite_count;
  o.positivity_failure_count = d.positivity_failure_count;
  o.face_enthalpy_denominator_guard_count = d.face_enthalpy_denominator_guard_count;
  o.face_enthalpy_nonfinite_count = d.face_enthalpy_nonfinite_count;
  o.energy_flux_nonfinite_count = d.energy_flux_nonfinite_count;
  o.solver_initial_residual = d.solver_initial_residual;
  o.solver_initial_rhs_norm = d.solver_initial_rhs_norm;
  o.solver_residual = d.solver_residual;
  o.solver_relative_residual = d.solver_relative_residual;
  o.pressure_linear_residual_linf = d.pressure_linear_residual_linf;
  o.pressure_linear_residual_relative_linf = d.pressure_linear_residual_relative_linf;
  o.kinetic_jacobian_abs_max = d.kinetic_jacobian_abs_max;
  o.pressure_matrix_symmetry_linf = d.pressure_matrix_symmetry_linf;
  o.pressure_picard_delta_linf = d.pressure_picard_delta_linf;
  o.source_picard_delta_l2_relative_to_pmax = d.source_picard_delta_l2_relative_to_pmax;
  o.pressure_energy_residual_before_linf = d.pressure_energy_residual_before_linf;
  o.coupled_residual_l1_final = d.coupled_residual_l1_final;
  o.coupled_residual_linf_final = d.coupled_residual_linf_final;
  o.coupled_residual_relative_linf_final = d.coupled_residual_relative_linf_final;
  o.pressure_energy_residual_l1 = d.pressure_energy_residual_l1;
  o.pressure_energy_residual_linf = d.pressure_energy_residual_linf;
  o.pressure_energy_residual_relative_linf = d.pressure_energy_residual_relative_linf;
  o.rho_min = d.rho_min;
  o.pressure_min = d.pressure_min;
  o.internal_energy_min = d.internal_energy_min;
  o.trial_density_min = d.trial_density_min;
  o.trial_pressure_min = d.eos_pressure_min;
  o.trial_internal_energy_min = d.internal_energy_min;
  o.trial_nonfinite_count = d.nonfinite_count;
  o.trial_positivity_count = d.positivity_failure_count;
  o.solved_pressure_min = d.solved_pressure_min;
  o.solved_pressure_max = d.solved_pressure_max;
  o.eos_pressure_min = d.eos_pressure_min;
  o.eos_pressure_max = d.eos_pressure_max;
  o.internal_energy_max = d.internal_energy_max;
  o.momentum_correction_linf = d.momentum_correction_linf;
  o.energy_correction_linf = d.energy_correction_linf;
  o.energy_flux_linf = d.energy_flux_linf;
  o.energy_flux_divergence_linf = d.energy_flux_divergence_linf;
  o.eq78_divergence_linf = d.eq78_divergence_linf;
  o.eq78_divergence_scaled_linf = d.eq78_divergence_scaled_linf;
  o.energy_closeout_delta_l1 = d.energy_closeout_delta_l1;
  o.energy_closeout_delta_linf = d.energy_closeout_delta_linf;
  return o;
}

}  // namespace ecg_bridge

#define euler_fv_one_step ::ecg_bridge::euler_fv_one_step
#define compute_euler_dt ::ecg_bridge::compute_euler_dt
#define compute_imex_dt ::ecg_bridge::compute_imex_dt
#define compute_diagnostics ::ecg_bridge::compute_diagnostics
#define compute_admissibility_diagnostics ::ecg_bridge::compute_admissibility_diagnostics
#define euler_imex_bdltv20_o1_source_map_picard_one_step ::ecg_bridge::euler_imex_bdltv20_o1_source_map_picard_one_step
