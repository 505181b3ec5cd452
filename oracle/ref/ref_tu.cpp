// Reference oracle translation unit.  TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own euler_compare numerics and output headers, in
// the include order of amrex/apps/euler_compare/src/euler_compare_app.cpp:41-62
// (minus the app driver; plotfiles are a no-op), against the single-box AMReX
// shim in amrex_shim.hpp and the reference's vendored Eigen.  The extern "C"
// wrappers below run one reference call on host arrays so tests can compare
// the CUDA path with the reference's exact arithmetic.
//
// Host array layout used by every wrapper: 4 component planes of nx*ny
// doubles, i fastest (the valid cells of an Array4 box).
#include "amrex_shim.hpp"

#include <Eigen/Dense>
#include <Eigen/IterativeLinearSolvers>
#include <Eigen/Sparse>
#include <Eigen/SparseLU>

#include <chrono>
#include <cctype>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>

#include "ecg.h"

namespace ecref {

enum ConservedComponent { Rho = 0, Mx = 1, My = 2, E = 3, NCons = 4 };

#include "euler_compare/core/solver_types.hpp"
#include "euler_compare/core/diagnostics.hpp"
#include "euler_compare/core/run_config.hpp"
#include "euler_compare/core/config_reader.hpp"
#include "euler_compare/problems/problem_setup_boundary.hpp"
#include "euler_compare/numerics/explicit_update.hpp"
#include "euler_compare/imex/imex_source_map_helpers.hpp"
#include "euler_compare/imex/imex_pressure_helpers.hpp"
#include "euler_compare/imex/imex_bdltv20_updates.hpp"
#include "euler_compare/io/output_cases.hpp"

}  // namespace ecref

using namespace ecref;

namespace {

std::string g_error;
RunConfig g_cfg;
bool g_have_cfg = false;

struct Fabs {
  amrex::Geometry geom;
  amrex::BoxArray ba;
  amrex::DistributionMapping dm;
  explicit Fabs(const RunConfig& cfg) : geom(make_geometry(cfg)), ba(geom.Domain()), dm(ba) {}
};

void load_interior(amrex::MultiFab& mf, const double* u, int nx, int ny)
{
  auto a = mf.arr();
  for (int n = 0; n < NCons; ++n) {
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        a(i, j, 0, n) = u[static_cast<std::size_t>(n) * nx * ny + static_cast<std::size_t>(j) * nx + i];
      }
    }
  }
}

void store_interior(const amrex::MultiFab& mf, double* u, int nx, int ny)
{
  auto a = mf.const_array_impl();
  for (int n = 0; n < NCons; ++n) {
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        u[static_cast<std::size_t>(n) * nx * ny + static_cast<std::size_t>(j) * nx + i] = a(i, j, 0, n);
      }
    }
  }
}

int solver_status_code(const std::string& s)
{
  if (s == "not_run") return ECG_SOLVER_NOT_RUN;
  if (s == "converged_absolute") return ECG_SOLVER_CONVERGED_ABSOLUTE;
  if (s == "converged_relative") return ECG_SOLVER_CONVERGED_RELATIVE;
  if (s == "linear_solve_not_converged") return ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED;
  if (s == "gmres_breakdown_not_converged") return ECG_SOLVER_GMRES_BREAKDOWN_NOT_CONVERGED;
  if (s == "linear_residual_nonfinite") return ECG_SOLVER_LINEAR_RESIDUAL_NONFINITE;
  if (s == "source_map_pressure_row_nonfinite") return ECG_SOLVER_SOURCE_MAP_PRESSURE_ROW_NONFINITE;
  if (s == "source_map_lagged_momentum_nonfinite") return ECG_SOLVER_SOURCE_MAP_LAGGED_MOMENTUM_NONFINITE;
  if (s == "density_denominator_floor_used") return ECG_SOLVER_DENSITY_DENOMINATOR_FLOOR_USED;
  if (s == "unsupported_mpi_for_host_single_level_gmres") return ECG_SOLVER_UNSUPPORTED_MPI;
  return -1;
}

}  // namespace

extern "C" {

const char* ecref_last_error() { return g_error.c_str(); }

// Parses whitespace/newline separated "key=value ..." tokens the way AMReX
// parses argv overrides, then runs the reference's read_config().
int ecref_configure(const char* kv)
{
  try {
    auto& table = amrex::parmparse_table();
    table.clear();
    // Lines of "key = v1 v2 ...": split without iostreams.
    auto split_ws = [](const std::string& t) {
      std::vector<std::string> out;
      std::size_t k = 0;
      while (k < t.size()) {
        while (k < t.size() && std::isspace(static_cast<unsigned char>(t[k]))) ++k;
        std::size_t e = k;
        while (e < t.size() && !std::isspace(static_cast<unsigned char>(t[e]))) ++e;
        if (e > k) out.push_back(t.substr(k, e - k));
        k = e;
      }
      return out;
    };
    const std::string text(kv);
    std::size_t pos = 0;
    while (pos <= text.size()) {
      std::size_t nl = text.find('\n', pos);
      if (nl == std::string::npos) nl = text.size();
      const std::string line = text.substr(pos, nl - pos);
      pos = nl + 1;
      const auto eq = line.find('=');
      if (eq == std::string::npos) continue;
      const auto key_tokens = split_ws(line.substr(0, eq));
      if (key_tokens.size() != 1) continue;
      table[key_tokens[0]] = split_ws(line.substr(eq + 1));
    }
    g_cfg = read_config();
    g_have_cfg = true;
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    g_have_cfg = false;
    return -1;
  }
}

// The parsed RunConfig as the C-ABI mirror struct.
int ecref_get_config(ecg_run_config* out)
{
  if (!g_have_cfg) return -1;
  const RunConfig& c = g_cfg;
  std::memset(out, 0, sizeof(*out));
  out->n_cell[0] = c.n_cell[0];
  out->n_cell[1] = c.n_cell[1];
  out->is_periodic[0] = c.is_periodic[0];
  out->is_periodic[1] = c.is_periodic[1];
  out->prob_lo[0] = c.prob_lo[0];
  out->prob_lo[1] = c.prob_lo[1];
  out->prob_hi[0] = c.prob_hi[0];
  out->prob_hi[1] = c.prob_hi[1];
  out->max_step = c.max_step;
  out->spatial_order = c.spatial_order;
  out->toro_test = c.toro_test;
  out->problem = static_cast<int>(c.problem);
  out->riemann = static_cast<int>(c.riemann);
  out->method = static_cast<int>(c.method);
  out->slope_limiter = static_cast<int>(c.slope_limiter);
  out->field_boundary = c.field_boundary == "exact_dirichlet" ? 1 : 0;
  out->stop_time = c.stop_time;
  out->gamma = c.gamma;
  out->cfl = c.cfl;
  out->imex_cfl = c.imex_cfl;
  out->imex_acoustic_cfl_cap = c.imex_acoustic_cfl_cap;
  out->imex_solver_tol = c.imex_solver_tol;
  out->velocity_x = c.velocity_x;
  out->velocity_y = c.velocity_y;
  out->density_inner = c.density_inner;
  out->density_outer = c.density_outer;
  out->pressure = c.pressure;
  out->mach = c.mach;
  out->blob_cx = c.blob_cx;
  out->blob_cy = c.blob_cy;
  out->blob_radius = c.blob_radius;
  out->vortex_cx = c.vortex_cx;
  out->vortex_cy = c.vortex_cy;
  out->isentropic_vortex_strength = c.isentropic_vortex_strength;
  out->riemann_interface_x = c.riemann_interface_x;
  out->riemann_interface_y = c.riemann_interface_y;
  out->imex_solver_max_iter = c.imex_solver_max_iter;
  out->imex_acoustic_startup = c.imex_acoustic_startup;
  out->imex_picard_iterations = c.imex_picard_iterations;
  out->imex_picard_extra_iterations = c.imex_picard_extra_iterations;
  return 0;
}

int ecref_initialize_state(double* u)
{
  try {
    Fabs f(g_cfg);
    amrex::MultiFab s(f.ba, f.dm, NCons, 2);
    initialize_state(s, f.geom, g_cfg);
    store_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
    return 0;
  } catch (const std::exception& e) { g_error = e.what(); return -1; }
}

// euler_fv_one_step on the valid cells in u (updated in place); returns the
// degenerate-star count.
int ecref_euler_fv_one_step(double* u, double dt, double time)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  const int count = euler_fv_one_step(s, f.geom, g_cfg, dt, time);
  store_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  return count;
}

double ecref_compute_euler_dt(const double* u, double time)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  return compute_euler_dt(s, f.geom, g_cfg, time);
}

double ecref_compute_imex_dt(const double* u, double time, ecg_imex_timestep_diag* d)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  ImexTimeStepDiagnostics td;
  const double dt = compute_imex_dt(s, f.geom, g_cfg, time, td);
  if (d) {
    d->material_rate_max = td.material_rate_max;
    d->acoustic_rate_max = td.acoustic_rate_max;
    d->acoustic_startup_used = td.acoustic_startup_used;
    d->acoustic_cap_used = td.acoustic_cap_used;
  }
  return dt;
}

void ecref_compute_diagnostics(const double* u, ecg_diagnostics* out)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  const Diagnostics d = compute_diagnostics(s, g_cfg);
  out->rho_min = d.rho_min;
  out->pressure_min = d.pressure_min;
  out->nonfinite_count = d.nonfinite_count;
}

void ecref_compute_admissibility(const double* u, ecg_admissibility* out)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  const AdmissibilityDiagnostics d = compute_admissibility_diagnostics(s, g_cfg);
  out->rho_min = d.rho_min;
  out->pressure_min = d.pressure_min;
  out->internal_energy_min = d.internal_energy_min;
  out->nonfinite_count = d.nonfinite_count;
  out->density_failure_count = d.density_failure_count;
  out->pressure_failure_count = d.pressure_failure_count;
  out->internal_energy_failure_count = d.internal_energy_failure_count;
}

// fill_problem_ghosts; writes the whole ghosted box (4 planes of (nx+4)(ny+4)).
void ecref_fill_problem_ghosts(const double* u, double time, double* ghosted)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  fill_problem_ghosts(s, f.geom, g_cfg, time);
  std::memcpy(ghosted, s.data.data(), s.data.size() * sizeof(double));
}

// euler_imex_bdltv20_o1_source_map_picard_one_step; u updated in place.
int ecref_imex_step(double* u, double dt, ecg_imex_diag* o)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  const ImexStepDiagnostics d = euler_imex_bdltv20_o1_source_map_picard_one_step(s, f.geom, g_cfg, dt, nullptr);
  store_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  std::memset(o, 0, sizeof(*o));
  o->solver_status = solver_status_code(d.solver_status);
  o->linear_solver_status_last = solver_status_code(d.linear_solver_status_last);
  o->solver_iterations = d.solver_iterations;
  o->picard_pressure_solves_used = d.picard_pressure_solves_used;
  o->source_picard_iterations_used = d.source_picard_iterations_used;
  o->kinetic_lag_update_count = d.kinetic_lag_update_count;
  o->kinetic_lag_nonfinite_count = d.kinetic_lag_nonfinite_count;
  o->pressure_matrix_rows = d.pressure_matrix_rows;
  o->pressure_matrix_nonzeros = d.pressure_matrix_nonzeros;
  o->pressure_matrix_max_row_width = d.pressure_matrix_max_row_width;
  o->density_denominator_floor_count = d.density_denominator_floor_count;
  o->nonfinite_count = d.nonfinite_count;
  o->positivity_failure_count = d.positivity_failure_count;
  o->face_enthalpy_denominator_guard_count = d.face_enthalpy_denominator_guard_count;
  o->face_enthalpy_nonfinite_count = d.face_enthalpy_nonfinite_count;
  o->energy_flux_nonfinite_count = d.energy_flux_nonfinite_count;
  o->solver_initial_residual = d.solver_initial_residual;
  o->solver_initial_rhs_norm = d.solver_initial_rhs_norm;
  o->solver_residual = d.solver_residual;
  o->solver_relative_residual = d.solver_relative_residual;
  o->pressure_linear_residual_linf = d.pressure_linear_residual_linf;
  o->pressure_linear_residual_relative_linf = d.pressure_linear_residual_relative_linf;
  o->kinetic_jacobian_abs_max = d.kinetic_jacobian_abs_max;
  o->pressure_matrix_symmetry_linf = d.pressure_matrix_symmetry_linf;
  o->pressure_picard_delta_linf = d.pressure_picard_delta_linf;
  o->source_picard_delta_l2_relative_to_pmax = d.source_picard_delta_l2_relative_to_pmax;
  o->pressure_energy_residual_before_linf = d.pressure_energy_residual_before_linf;
  o->coupled_residual_l1_final = d.coupled_residual_l1_final;
  o->coupled_residual_linf_final = d.coupled_residual_linf_final;
  o->coupled_residual_relative_linf_final = d.coupled_residual_relative_linf_final;
  o->pressure_energy_residual_l1 = d.pressure_energy_residual_l1;
  o->pressure_energy_residual_linf = d.pressure_energy_residual_linf;
  o->pressure_energy_residual_relative_linf = d.pressure_energy_residual_relative_linf;
  o->rho_min = d.rho_min;
  o->pressure_min = d.pressure_min;
  o->internal_energy_min = d.internal_energy_min;
  o->trial_density_min = d.trial_density_min;
  o->solved_pressure_min = d.solved_pressure_min;
  o->solved_pressure_max = d.solved_pressure_max;
  o->eos_pressure_min = d.eos_pressure_min;
  o->eos_pressure_max = d.eos_pressure_max;
  o->internal_energy_max = d.internal_energy_max;
  o->momentum_correction_linf = d.momentum_correction_linf;
  o->energy_correction_linf = d.energy_correction_linf;
  o->energy_flux_linf = d.energy_flux_linf;
  o->energy_flux_divergence_linf = d.energy_flux_divergence_linf;
  o->eq78_divergence_linf = d.eq78_divergence_linf;
  o->eq78_divergence_scaled_linf = d.eq78_divergence_scaled_linf;
  o->energy_closeout_delta_l1 = d.energy_closeout_delta_l1;
  o->energy_closeout_delta_linf = d.energy_closeout_delta_linf;
  return o->solver_status;
}

// compute_bdltv20_pressure_split_star on u (the IMEX step's ghost policy is
// applied first, imex_source_map_step.hpp:405-411); writes the star valid cells.
void ecref_imex_star(const double* u, double dt, double* star_out)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  if (g_cfg.problem == ProblemKind::ShockDensityBubble2D) {
    fill_problem_ghosts(s, f.geom, g_cfg);
  } else {
    fill_physical_outflow_ghosts(s, f.geom);
  }
  amrex::MultiFab star(f.ba, f.dm, NCons, 2);
  compute_bdltv20_pressure_split_star(s, star, f.geom, g_cfg, dt);
  store_interior(star, star_out, g_cfg.n_cell[0], g_cfg.n_cell[1]);
}

static CoupledHostGrid grid_from(const double* star, const Fabs& f)
{
  const int nx = g_cfg.n_cell[0], ny = g_cfg.n_cell[1];
  CoupledHostGrid grid;
  grid.nx = nx;
  grid.ny = ny;
  grid.periodic_x = f.geom.isPeriodic(0);
  grid.periodic_y = f.geom.isPeriodic(1);
  grid.cell.resize(static_cast<std::size_t>(nx) * ny);
  const std::size_t plane = static_cast<std::size_t>(nx) * ny;
  for (std::size_t r = 0; r < plane; ++r) {
    grid.cell[r] = ConservedState{star[r], star[plane + r], star[2 * plane + r], star[3 * plane + r]};
  }
  return grid;
}

// source_map_build_pressure_system for the star state, Picard pressure p and
// lagged momentum K (2 planes).  Writes CSR (row_ptr n+1, col/val up to cap)
// and rhs; returns nnz, -1 if cap is too small.
int ecref_imex_build_system(const double* star, const double* p, const double* k, double dt,
                            int* row_ptr, int* col, double* val, double* rhs, int cap,
                            int* nonfinite_count)
{
  Fabs f(g_cfg);
  const CoupledHostGrid grid = grid_from(star, f);
  const int n = grid.nx * grid.ny;
  std::vector<double> pv(p, p + n);
  std::vector<SourceMapMomentum> km(static_cast<std::size_t>(n));
  for (int r = 0; r < n; ++r) km[r] = SourceMapMomentum{k[r], k[n + r]};
  const SourceMapPressureSystem sys = source_map_build_pressure_system(grid, pv, km, g_cfg, f.geom, dt);
  if (nonfinite_count) *nonfinite_count = sys.nonfinite_count;
  if (sys.matrix.nonZeros() > cap) return -1;
  int nnz = 0;
  for (int r = 0; r < n; ++r) {
    row_ptr[r] = nnz;
    for (HostSparseMatrix::InnerIterator it(sys.matrix, r); it; ++it) {
      col[nnz] = static_cast<int>(it.col());
      val[nnz] = it.value();
      ++nnz;
    }
    rhs[r] = sys.rhs(r);
  }
  row_ptr[n] = nnz;
  return nnz;
}

// solve_host_sparse_gmres on a CSR matrix.
int ecref_gmres(int n, const int* row_ptr, const int* col, const double* val, const double* rhs,
                const double* x0, int max_iter, double tol, double* x, int* iterations,
                int* converged, int* breakdown, int* nonfinite, double* residual_linf,
                double* relative_residual_linf)
{
  std::vector<Eigen::Triplet<double>> t;
  for (int r = 0; r < n; ++r) {
    for (int q = row_ptr[r]; q < row_ptr[r + 1]; ++q) t.emplace_back(r, col[q], val[q]);
  }
  HostSparseMatrix a(n, n);
  a.setFromTriplets(t.begin(), t.end());
  a.makeCompressed();
  Eigen::VectorXd b(n), g(n);
  for (int r = 0; r < n; ++r) { b(r) = rhs[r]; g(r) = x0[r]; }
  const HostGmresResult res = solve_host_sparse_gmres(a, b, g, max_iter, tol);
  for (int r = 0; r < n; ++r) x[r] = res.solution(r);
  *iterations = res.iterations;
  *converged = res.converged ? 1 : 0;
  *breakdown = res.breakdown ? 1 : 0;
  *nonfinite = res.nonfinite ? 1 : 0;
  *residual_linf = res.residual_linf;
  *relative_residual_linf = res.relative_residual_linf;
  return 0;
}

// source_map_eq54_corrected_momentum_field with the physical-boundary
// pressure map (cfg != nullptr), as the Picard refresh uses it.
void ecref_corrected_momentum(const double* star, const double* p, double dt, double* k)
{
  Fabs f(g_cfg);
  const CoupledHostGrid grid = grid_from(star, f);
  const int n = grid.nx * grid.ny;
  std::vector<double> pv(p, p + n);
  const auto dx = f.geom.CellSizeArray();
  const auto m = source_map_eq54_corrected_momentum_field(grid, pv, dt, 1.0 / dx[0], 1.0 / dx[1], &g_cfg);
  for (int r = 0; r < n; ++r) { k[r] = m[r][0]; k[n + r] = m[r][1]; }
}

// exact_riemann_sample (problems/exact_riemann.hpp:113-205) for Sod-type L1.
void ecref_exact_riemann_sample(double x, double time, const double* left, const double* right,
                                double gamma, double interface_x, double* out)
{
  const PrimitiveState l{left[0], left[1], left[2], left[3]};
  const PrimitiveState r{right[0], right[1], right[2], right[3]};
  const PrimitiveState q = exact_riemann_sample(x, time, l, r, gamma, interface_x);
  out[0] = q.rho; out[1] = q.u; out[2] = q.v; out[3] = q.p;
}

// gresho_state (problems/problem_state_functions.hpp:2-30).
void ecref_gresho_state(double x, double y, double* out)
{
  const PrimitiveState q = gresho_state(x, y, g_cfg);
  out[0] = q.rho; out[1] = q.u; out[2] = q.v; out[3] = q.p;
}

// compute_gresho_metrics density_l1_error (diagnostic_metrics_timestep.hpp:150-225).
double ecref_gresho_density_l1(const double* u)
{
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  return compute_gresho_metrics(s, f.geom, g_cfg).density_l1_error;
}

// run_bdltv20_paper_t1_s2 (imex/imex_bdltv20_direct_driver.hpp:44-779), the
// reference's direct T1/S2 driver, on the configured run: returns its exit
// code and writes its key=value report (at most len bytes) into out.
int ecref_paper_run(char* out, int len)
{
  if (!g_have_cfg) return -1;
  std::string text;
  amrex::print_sink() = &text;
  const int rc = run_bdltv20_paper_t1_s2(g_cfg);
  amrex::print_sink() = nullptr;
  if (out && len > 0) std::snprintf(out, static_cast<size_t>(len), "%s", text.c_str());
  return rc;
}

// The reference's final CSV writers (io/output_cases.hpp:16-216) on a host
// state: Gresho, Toro, Riemann quadrant or advection blob by the configured
// problem.  trial_* are the IMEX admissibility run minima of the Gresho file.
int ecref_write_final_csv(const double* u, int step, double time, const char* path, double trial_rho,
                          double trial_p, double trial_ie)
{
  if (!g_have_cfg) return -1;
  RunConfig cfg = g_cfg;
  cfg.final_csv = path;
  Fabs f(cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, cfg.n_cell[0], cfg.n_cell[1]);
  HighTrialRunDiagnostics h;
  h.rho_min = trial_rho;
  h.pressure_min = trial_p;
  h.internal_energy_min = trial_ie;
  write_gresho_final_csv(s, f.geom, cfg, step, time, h);
  write_toro_final_csv(s, f.geom, cfg);
  write_riemann_quadrant_final_csv(s, f.geom, cfg, step, time);
  write_advection_blob_final_csv(s, f.geom, cfg, step, time);
  return 0;
}

// compute_shock_density_bubble_metrics (io/output_cases.hpp:329-403) after
// fill_problem_ghosts at `time`: out = rho_min, rho_max, pressure_min,
// pressure_max, internal_energy_min, centroid_x, centroid_y, area,
// schlieren_max; returns the nonfinite count.
int ecref_bubble_metrics(const double* u, double time, double* out)
{
  if (!g_have_cfg) return -1;
  Fabs f(g_cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, g_cfg.n_cell[0], g_cfg.n_cell[1]);
  fill_problem_ghosts(s, f.geom, g_cfg, time);
  const ShockDensityBubbleMetrics m = compute_shock_density_bubble_metrics(s, f.geom, g_cfg);
  const double v[9] = {m.rho_min, m.rho_max, m.pressure_min, m.pressure_max, m.internal_energy_min,
                       m.density_bubble_centroid_x, m.density_bubble_centroid_y, m.density_bubble_area,
                       m.schlieren_max};
  for (int k = 0; k < 9; ++k) out[k] = v[k];
  return m.nonfinite_count;
}

// write_shock_density_bubble_snapshot (io/output_cases.hpp:422-487) after
// fill_problem_ghosts at `time`, into `dir`; 0 on success.
int ecref_bubble_snapshot(const double* u, int step, double time, int index, const char* dir)
{
  if (!g_have_cfg) return -1;
  RunConfig cfg = g_cfg;
  cfg.shock_density_bubble_snapshot_dir = dir;
  Fabs f(cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, cfg.n_cell[0], cfg.n_cell[1]);
  fill_problem_ghosts(s, f.geom, cfg, time);
  return write_shock_density_bubble_snapshot(s, f.geom, cfg, step, time, index) ? 0 : 1;
}

// write_shock_density_bubble_summary_csv (io/output_cases.hpp:489-588) with
// the metrics of the state (after fill_problem_ghosts at `time`) and the
// run-level fields the driver passes.
int ecref_bubble_summary(const double* u, const char* path, int step, double time, const char* status,
                         const char* failure, int rejected, double wall, double dt_min, double dt_max,
                         double dt_mean, const char* snapshot_status, const char* snapshot_dir,
                         const char* snapshot_times)
{
  if (!g_have_cfg) return -1;
  RunConfig cfg = g_cfg;
  cfg.final_csv = path;
  cfg.shock_density_bubble_snapshot_dir = snapshot_dir;
  cfg.shock_density_bubble_snapshot_times = snapshot_times;
  Fabs f(cfg);
  amrex::MultiFab s(f.ba, f.dm, NCons, 2);
  load_interior(s, u, cfg.n_cell[0], cfg.n_cell[1]);
  fill_problem_ghosts(s, f.geom, cfg, time);
  const ShockDensityBubbleMetrics m = compute_shock_density_bubble_metrics(s, f.geom, cfg);
  write_shock_density_bubble_summary_csv(s, f.geom, cfg, step, time, status, failure, rejected, wall, dt_min, dt_max,
                                         dt_mean, snapshot_status, m);
  return 0;
}

}  // extern "C"
