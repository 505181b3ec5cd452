// euler_imex_bdltv20_o1_source_map_picard_one_step on the device
// (imex/imex_source_map_step.hpp:300-616): star update -> Picard iterations
// {face enthalpies, pressure-row rhs, GMRES, gate, p <- x, eq54 momentum} ->
// conservative closeout.  The state stays on the device.
//
// The whole step is queued at once and the host waits once, at its end.
// Each phase writes its reductions to a slot of its own; the reference's
// early-return tests run on the device (a one-thread gate kernel after the
// star update, each assembly and each refresh; the GMRES kernel on its own
// result), and once one fails every later phase is a no-op launch.  The host
// then reads all slots and results (a few KB) and takes the reference's
// decisions in the reference's order, so the diagnostics and the state are
// those of the step that stopped where the first failing test stopped it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <limits>

#include "ctx.h"
#include "imex_internal.h"

struct EcgImexState {
  long long n = 0;
  int max_iter = 0;
  bool mixed = false;
  double* S = nullptr;   // star state, 4 compact planes
  double* p = nullptr;   // Picard pressure
  double* K = nullptr;   // lagged momentum, 2 planes
  double* hx = nullptr;  // x-face enthalpy / energy flux, (nx+1) x ny
  double* hy = nullptr;  // y-face, nx x (ny+1)
  double* fx = nullptr;
  double* fy = nullptr;
  unsigned char* fxf = nullptr;
  unsigned char* fyf = nullptr;
  double* rhs = nullptr;
  double* x = nullptr;
  // reduction slots of one step: the star update, per Picard pass the
  // assembly and the refresh, the matrix diagnostics, the closeout
  int passes = -1;                   // Picard passes the slots were made for
  EcgImexStats* d_st = nullptr;
  EcgImexStats* h_st = nullptr;      // pinned
  EcgImexStats* h_init = nullptr;    // pinned: the reset template in every slot
  EcgGmresResult* d_res = nullptr;   // per pass: the solve, then its FP64 fallback
  EcgGmresResult* h_res = nullptr;   // pinned
  int* d_gate = nullptr;             // {a phase failed, a mixed solve needs the fallback}
  EcgGmresWork* gw = nullptr;
  EcgGmresWork* gw64 = nullptr;      // mixed precision: FP64 workspace of the fallback (and of short) solves
  double last_its = -1.0;            // iterations per solve of the previous step (-1: none yet)
};

namespace {
constexpr int kSlotStar = 0;
int slot_assemble(int k) { return 1 + 2 * k; }
int slot_refresh(int k) { return 2 + 2 * k; }
int slot_matrix(int passes) { return 1 + 2 * passes; }
int slot_close(int passes) { return 2 + 2 * passes; }
int slot_count(int passes) { return 3 + 2 * passes; }

// The reference's early-return tests on a phase's reductions
// (imex_source_map_step.hpp:405-454 after the star update, :464-497 after an
// assembly, :536-564 after a refresh): gate[0] is set when the test fails.
enum GateKind { kGateStar = 0, kGateAssemble = 1, kGateRefresh = 2 };

__device__ bool key_is_finite(unsigned long long k)
{
  const unsigned long long b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  return isfinite(__longlong_as_double(static_cast<long long>(b)));
}

__global__ void imex_gate_kernel(const EcgImexStats* st, int kind, int* gate)
{
  bool fail;
  if (kind == kGateStar) fail = st->floor_count > 0;
  else if (kind == kGateAssemble) fail = st->row_nonfinite > 0 || !key_is_finite(st->rhs_linf_key);
  else fail = st->k_nonfinite > 0;
  if (fail) gate[0] = 1;
}
}  // namespace

namespace {

unsigned long long key_of(double x)
{
  unsigned long long b;
  std::memcpy(&b, &x, sizeof(b));
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}

EcgImexStats stats_template()
{
  const double inf = std::numeric_limits<double>::infinity();
  EcgImexStats s;
  std::memset(&s, 0, sizeof(s));
  s.trial_rho_min_key = key_of(inf);
  s.mismatch_before_key = key_of(0.0);
  s.abs_max_key = key_of(0.0);
  s.sym_key = key_of(0.0);
  s.rhs_linf_key = key_of(0.0);
  s.delta_linf_key = key_of(0.0);
  s.pmax_key = key_of(1.0);
  s.flux_linf_key = key_of(0.0);
  s.density_min_key = key_of(inf);
  s.solved_p_min_key = key_of(inf);
  s.solved_p_max_key = key_of(-inf);
  s.eos_p_min_key = key_of(inf);
  s.eos_p_max_key = key_of(-inf);
  s.ie_min_key = key_of(inf);
  s.ie_max_key = key_of(-inf);
  s.momentum_corr_key = key_of(0.0);
  s.energy_corr_key = key_of(0.0);
  s.flux_div_key = key_of(0.0);
  s.res_linf_key = key_of(0.0);
  s.res_rel_key = key_of(0.0);
  s.mis_linf_key = key_of(0.0);
  s.mis_rel_key = key_of(0.0);
  s.eq78_key = key_of(0.0);
  s.eq78_scaled_key = key_of(0.0);
  return s;
}

bool ensure_state(ecg_ctx* c)
{
  const bool mixed = c->opt.imex_precision == ECG_IMEX_MIXED;
  const int max_iter = c->cfg.imex_solver_max_iter;
  EcgImexState* im = c->imex;
  if (im && im->max_iter >= max_iter && (!mixed || im->mixed)) return true;
  imex_free(c);
  im = new EcgImexState();
  c->imex = im;
  const int nx = c->grid.nx, ny = c->grid.ny;
  const long long n = static_cast<long long>(nx) * ny;
  im->n = n;
  im->max_iter = max_iter;
  im->mixed = mixed;
  const long long nfx = static_cast<long long>(nx + 1) * ny, nfy = static_cast<long long>(nx) * (ny + 1);
  bool ok = true;
  auto alloc = [&](void** p, size_t bytes) {
    if (ok) ok = ecgi::cuda_ok(c, cudaMalloc(p, bytes), "imex alloc");
  };
  alloc(reinterpret_cast<void**>(&im->S), sizeof(double) * 4 * n);
  alloc(reinterpret_cast<void**>(&im->p), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&im->K), sizeof(double) * 2 * n);
  alloc(reinterpret_cast<void**>(&im->hx), sizeof(double) * nfx);
  alloc(reinterpret_cast<void**>(&im->hy), sizeof(double) * nfy);
  alloc(reinterpret_cast<void**>(&im->fx), sizeof(double) * nfx);
  alloc(reinterpret_cast<void**>(&im->fy), sizeof(double) * nfy);
  alloc(reinterpret_cast<void**>(&im->fxf), nfx);
  alloc(reinterpret_cast<void**>(&im->fyf), nfy);
  alloc(reinterpret_cast<void**>(&im->rhs), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&im->x), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&im->d_gate), sizeof(int) * 2);
  if (ok) {
    std::string err;
    im->gw = gmres_work_create(n, max_iter < 1 ? 1 : max_iter, c->num_sms, c->device, mixed, &err);
    if (!im->gw) {
      c->err = err;
      ok = false;
    }
    // the fallback solve is queued (gated) with every mixed solve, so its
    // workspace exists from the start
    if (ok && mixed) {
      im->gw64 = gmres_work_create(n, max_iter < 1 ? 1 : max_iter, c->num_sms, c->device, false, &err);
      if (!im->gw64) {
        c->err = err;
        ok = false;
      }
    }
  }
  return ok;
}

// Stats slots and result records for a step of `passes` Picard passes.
bool ensure_slots(ecg_ctx* c, int passes)
{
  EcgImexState* im = c->imex;
  if (im->passes >= passes) return true;
  cudaFree(im->d_st);
  cudaFreeHost(im->h_st);
  cudaFreeHost(im->h_init);
  cudaFree(im->d_res);
  cudaFreeHost(im->h_res);
  im->d_st = im->h_st = im->h_init = nullptr;
  im->d_res = im->h_res = nullptr;
  im->passes = -1;
  const int ns = slot_count(passes), nr = 2 * (passes > 0 ? passes : 1);
  const bool ok = ecgi::cuda_ok(c, cudaMalloc(&im->d_st, sizeof(EcgImexStats) * ns), "imex alloc") &&
                  ecgi::cuda_ok(c, cudaMallocHost(&im->h_st, sizeof(EcgImexStats) * ns), "imex host alloc") &&
                  ecgi::cuda_ok(c, cudaMallocHost(&im->h_init, sizeof(EcgImexStats) * ns), "imex host alloc") &&
                  ecgi::cuda_ok(c, cudaMalloc(&im->d_res, sizeof(EcgGmresResult) * nr), "imex alloc") &&
                  ecgi::cuda_ok(c, cudaMallocHost(&im->h_res, sizeof(EcgGmresResult) * nr), "imex host alloc");
  if (!ok) return false;
  const EcgImexStats t = stats_template();
  for (int k = 0; k < ns; ++k) im->h_init[k] = t;
  im->passes = passes;
  return true;
}

double kd(unsigned long long k) { return ecgi::okey_to_double(k); }
double finite_or_nan(double v) { return std::isfinite(v) ? v : std::numeric_limits<double>::quiet_NaN(); }

EcgImexMap imex_map(ecg_ctx* c)
{
  EcgImexMap m;
  std::memset(&m, 0, sizeof(m));
  m.nx = c->grid.nx;
  m.ny = c->grid.ny;
  m.px = c->cfg.is_periodic[0] != 0;
  m.py = c->cfg.is_periodic[1] != 0;
  const bool mach122 = c->cfg.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122;
  m.bubble = c->cfg.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D || mach122;
  m.top_wall = mach122 ? 1 : 0;
  m.gamma = c->cfg.gamma;
  // shock_density_bubble_post_shock_state, problem_initialization.hpp:51-58;
  // the Mach 1.22 variant (no reference counterpart) has its own inflow state
  // and the bubble's boundary policy with a wall at the top too
  double q[4] = {2.8181818181818183, 1.6064386578049976, 0.0, 5.0};
  if (mach122) mach122_post_shock(c->cfg.gamma, q);
  const double kin = 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
  m.cst[0] = q[0];
  m.cst[1] = q[0] * q[1];
  m.cst[2] = q[0] * q[2];
  m.cst[3] = q[3] / (c->cfg.gamma - 1.0) + kin;
  m.p_fixed = q[3];
  return m;
}

}  // namespace

void imex_free(ecg_ctx* c)
{
  EcgImexState* im = c->imex;
  if (!im) return;
  cudaFree(im->S);
  cudaFree(im->p);
  cudaFree(im->K);
  cudaFree(im->hx);
  cudaFree(im->hy);
  cudaFree(im->fx);
  cudaFree(im->fy);
  cudaFree(im->fxf);
  cudaFree(im->fyf);
  cudaFree(im->rhs);
  cudaFree(im->x);
  if (im->gw64) gmres_work_destroy(im->gw64);
  cudaFree(im->d_st);
  cudaFreeHost(im->h_st);
  cudaFreeHost(im->h_init);
  cudaFree(im->d_res);
  cudaFreeHost(im->h_res);
  cudaFree(im->d_gate);
  gmres_work_destroy(im->gw);
  delete im;
  c->imex = nullptr;
}

extern "C" ecg_status ecg_imex_step(ecg_ctx* c, double dt, ecg_imex_diag* out)
{
  if (!c || !out) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (c->cfg.spatial_order != 2) return ECG_ERR_UNSUPPORTED;
  if (c->slab()) {
    c->err = "the IMEX pressure system couples the whole grid: no slab contexts";
    return ECG_ERR_UNSUPPORTED;
  }
  if (!ensure_state(c)) return ECG_ERR_CUDA;
  const int passes = c->cfg.imex_picard_iterations > 0 ? c->cfg.imex_picard_iterations : 0;
  if (!ensure_slots(c, passes)) return ECG_ERR_CUDA;
  EcgImexState* im = c->imex;
  const EcgImexOps* ops = c->opt.arith == ECG_ARITH_EXACT ? &ecg_imex_exact_ops : &ecg_imex_fast_ops;
  // Mixed precision puts a step's solves on the FP32 basis unless the
  // previous step's solves were short (mixed_min_iterations): their basis
  // stays in L2, and the restart cycle the FP32 basis needs to reach the
  // tolerance costs more iterations than the halved bytes save.
  const bool mixed = c->opt.imex_precision == ECG_IMEX_MIXED &&
                     !(c->opt.mixed_min_iterations > 0 && im->last_its >= 0.0 &&
                       im->last_its < static_cast<double>(c->opt.mixed_min_iterations));
  EcgGmresWork* const gw = mixed || !im->gw64 ? im->gw : im->gw64;
  // the mixed cycles' restart factor: measured best at 1e-4 where the basis
  // sits in shared memory and L2 (Gresho 256^2: 1.76x against 1.69x FP64), at
  // 1e-3 where it streams from HBM (768^2: 3.88x against 3.45x)
  const double inner_rtol =
      c->opt.mixed_inner_rtol >= 0.0 ? c->opt.mixed_inner_rtol : (gmres_work_resident(im->gw) ? 1.0e-4 : 1.0e-3);
  const bool det = c->opt.deterministic != 0;
  ecg_imex_diag& d = *out;
  std::memset(&d, 0, sizeof(d));
  d.solver_status = ECG_SOLVER_NOT_RUN;
  d.linear_solver_status_last = -1;
  d.gmres_fp32_basis = mixed ? 1 : 0;
  const double inf = std::numeric_limits<double>::infinity();
  const EcgFvParams P = ecgi::fv_params(c, true);
  const EcgImexMap m = imex_map(c);  // ungated: the matrix diagnostics always run
  EcgImexMap mg = m;                 // the phases that stop after a failed test
  mg.abort = im->d_gate;
  const long long n = im->n;
  const double idx = c->grid.inv_dx, idy = c->grid.inv_dy;
  const double tol = c->cfg.imex_solver_tol;
  cudaStream_t s = c->stream;

  EcgPressureOp op;
  std::memset(&op, 0, sizeof(op));
  op.nx = m.nx;
  op.ny = m.ny;
  op.px = m.px;
  op.py = m.py;
  op.bubble = m.bubble;
  op.diag0 = 1.0 / (c->cfg.gamma - 1.0);
  op.xc = 0.25 * dt * dt * idx * idx;
  op.yc = 0.25 * dt * dt * idy * idy;
  op.hx = im->hx;
  op.hy = im->hy;

  // ---- queue the step ----------------------------------------------------------------
  auto ok = [&](cudaError_t e, const char* what) { return ecgi::cuda_ok(c, e, what); };
  auto gate = [&](int slot, int kind) {
    imex_gate_kernel<<<1, 1, 0, s>>>(im->d_st + slot, kind, im->d_gate);
    return ok(cudaGetLastError(), "gate");
  };
  if (!ok(cudaMemcpyAsync(im->d_st, im->h_init, sizeof(EcgImexStats) * slot_count(passes), cudaMemcpyHostToDevice, s),
          "reset stats") ||
      !ok(cudaMemsetAsync(im->d_gate, 0, sizeof(int) * 2, s), "reset gate"))
    return ECG_ERR_CUDA;
  // star update and step initialisation (imex_source_map_step.hpp:405-454)
  if (!ok(ops->star(P, c->cur_state(), dt, im->S, im->p, im->K, im->d_st + kSlotStar, s), "star") ||
      !gate(kSlotStar, kGateStar))
    return ECG_ERR_CUDA;
  for (int pic = 0; pic < passes; ++pic) {
    // pressure system (source_map_build_pressure_system, imex_source_map_step.hpp:8-38,464-497)
    if (!ok(ops->assemble(mg, im->S, im->p, im->K, im->hx, im->hy, dt, idx, idy, im->rhs, im->d_st + slot_assemble(pic),
                          s),
            "assemble") ||
        !gate(slot_assemble(pic), kGateAssemble))
      return ECG_ERR_CUDA;
    // The solve reports the true residuals before and after (||A p - b||inf,
    // ||A x - b||inf and ||b||inf, pressure_residual's values) with its
    // result.  A mixed solve that ends with a finite true residual above the
    // rule (its iteration budget ran out, or its FP32 basis stalled) is
    // finished by the FP64 solve from the iterate it reached, so the mixed
    // step fails only where the FP64 step would.
    if (!ok(gmres_enqueue(gw, op, im->rhs, im->p, im->x, c->cfg.imex_solver_max_iter, tol, mixed,
                          c->opt.mixed_inner_max_iter, inner_rtol, c->opt.mixed_max_refinements,
                          c->opt.mixed_reorth, det, im->d_res + 2 * pic, im->d_gate, 1, s),
            "gmres"))
      return ECG_ERR_CUDA;
    if (mixed && !ok(gmres_enqueue(im->gw64, op, im->rhs, im->x, im->x, c->cfg.imex_solver_max_iter, tol, false, 0,
                                   0.0, 0, 1, det, im->d_res + 2 * pic + 1, im->d_gate, 2, s),
                     "gmres fallback"))
      return ECG_ERR_CUDA;
    // p <- x, eq54 momentum refresh (imex_source_map_step.hpp:536-564), in one
    // sweep: K from x, then x becomes the pressure buffer (no copy).  The
    // buffers are renamed as queued: a step that stops early reaches no
    // closeout, and the next step's star update rewrites p.
    if (!ok(ops->refresh(mg, im->p, im->x, im->S, dt, idx, idy, im->K, im->d_st + slot_refresh(pic), s), "refresh") ||
        !gate(slot_refresh(pic), kGateRefresh))
      return ECG_ERR_CUDA;
    std::swap(im->p, im->x);
  }
  // Matrix diagnostics (imex_source_map_step.hpp:466-489) of the pressure
  // system of the last assembled pass: the pass that ended the step, whether
  // it stopped early or not (the later passes' assemblies did nothing).
  if (passes > 0 && !ok(ops->matrix(m, im->hx, im->hy, dt, idx, idy, im->d_st + slot_matrix(passes), s), "matrix"))
    return ECG_ERR_CUDA;
  // conservative closeout (evaluate_source_map_final, imex_source_map_step.hpp:75-258)
  double* out_state = c->next_state();
  if (!ok(ops->faces(mg, im->S, im->p, im->K, im->fx, im->fy, im->fxf, im->fyf, 1, s), "faces") ||
      !ok(ops->closeout(mg, c->grid, im->S, im->p, im->K, im->fx, im->fy, im->fxf, im->fyf, dt, out_state,
                        im->d_st + slot_close(passes), s),
          "closeout") ||
      !ok(ops->eq78(mg, c->grid, im->S, im->K, im->d_st + slot_close(passes), s), "eq78"))
    return ECG_ERR_CUDA;
  if (!ok(cudaMemcpyAsync(im->h_st, im->d_st, sizeof(EcgImexStats) * slot_count(passes), cudaMemcpyDeviceToHost, s),
          "fetch stats") ||
      (passes > 0 &&
       !ok(cudaMemcpyAsync(im->h_res, im->d_res, sizeof(EcgGmresResult) * 2 * passes, cudaMemcpyDeviceToHost, s),
           "fetch results")) ||
      !ok(cudaStreamSynchronize(s), "sync"))
    return ECG_ERR_CUDA;

  // ---- the reference's decisions, in its order, on what the phases reported ----
  // (the iterations per solve of the passes that ran pick the next step's basis)
  struct SolveCount {
    EcgImexState* im;
    int solves = 0;
    double its = 0.0;
    ~SolveCount()
    {
      if (solves > 0) im->last_its = its / solves;
    }
  } count{im};
  const EcgImexStats* stp = &im->h_st[kSlotStar];
  auto matrix_report = [&]() {
    const EcgImexStats& ms = im->h_st[slot_matrix(passes)];
    d.pressure_matrix_nonzeros = static_cast<int>(ms.nnz);
    d.pressure_matrix_max_row_width = static_cast<int>(ms.max_row_width);
    d.kinetic_jacobian_abs_max = kd(ms.abs_max_key);
    d.pressure_matrix_symmetry_linf = kd(ms.sym_key);
    return ECG_OK;
  };
  d.kinetic_lag_nonfinite_count = static_cast<int>(stp->k_nonfinite);
  d.trial_density_min = kd(stp->trial_rho_min_key);
  d.density_denominator_floor_count = static_cast<int>(stp->floor_count);
  if (stp->floor_count > 0) {
    d.solver_status = ECG_SOLVER_DENSITY_DENOMINATOR_FLOOR_USED;
    d.positivity_failure_count = static_cast<int>(stp->floor_count);
    return ECG_OK;
  }
  d.pressure_energy_residual_before_linf = stp->mismatch_before_nonfinite ? inf : kd(stp->mismatch_before_key);

  for (int pic = 0; pic < passes; ++pic) {
    const EcgImexStats& sa = im->h_st[slot_assemble(pic)];
    d.pressure_matrix_rows = static_cast<int>(n);
    if (sa.row_nonfinite > 0 || !std::isfinite(kd(sa.rhs_linf_key))) {
      d.solver_status = ECG_SOLVER_SOURCE_MAP_PRESSURE_ROW_NONFINITE;
      d.kinetic_lag_nonfinite_count = static_cast<int>(sa.row_nonfinite);
      d.nonfinite_count = static_cast<int>(sa.row_nonfinite);
      return matrix_report();
    }
    EcgGmresResult g = im->h_res[2 * pic];
    count.solves += 1;
    count.its += g.inner_iterations;
    if (g.timeout) {
      c->err = "gmres grid barrier timed out";
      return ECG_ERR_TIMEOUT;
    }
    if (mixed && !g.nonfinite && std::isfinite(g.final_linf) && std::isfinite(g.final_b_linf) &&
        !(g.final_linf <= tol || g.final_linf / std::max(g.final_b_linf, 1.0) <= tol)) {
      // the FP64 fallback ran from the mixed iterate
      const double r0 = g.initial_linf, b0 = g.b_linf;
      const int its = g.iterations, inner = g.inner_iterations, cyc = g.refinements;
      const double bytes = static_cast<double>(n) * (8.0 * g.vec_access64 + 4.0 * g.vec_access32);
      g = im->h_res[2 * pic + 1];
      count.its += g.inner_iterations;
      if (g.timeout) {
        c->err = "gmres grid barrier timed out";
        return ECG_ERR_TIMEOUT;
      }
      ++d.gmres_fp64_fallbacks;
      g.initial_linf = r0;
      g.b_linf = b0;
      g.iterations += its;
      g.inner_iterations += inner;
      g.refinements += cyc;
      d.gmres_vector_bytes += bytes;
    }
    const double nan = std::numeric_limits<double>::quiet_NaN();
    // b is finite here (a nonfinite row returned above); a nonfinite residual
    // reads as NaN, as pressure_residual reports it
    d.solver_initial_residual = std::isfinite(g.initial_linf) ? g.initial_linf : nan;
    d.solver_initial_rhs_norm = g.b_linf > 1.0 ? g.b_linf : 1.0;
    d.solver_iterations += g.iterations;
    d.gmres_inner_iterations += g.inner_iterations;
    d.gmres_refinements += g.refinements;
    d.gmres_vector_bytes += static_cast<double>(n) * (8.0 * g.vec_access64 + 4.0 * g.vec_access32);
    const int nf = std::isfinite(g.final_linf) && std::isfinite(g.final_b_linf) ? 0 : 1;
    const double lr = nf ? nan : g.final_linf;
    d.pressure_linear_residual_linf = lr;
    d.pressure_linear_residual_relative_linf = lr / d.solver_initial_rhs_norm;
    d.solver_residual = d.pressure_linear_residual_linf;
    d.solver_relative_residual = d.pressure_linear_residual_relative_linf;
    const bool abs_ok = lr <= tol;
    const bool rel_ok = d.pressure_linear_residual_relative_linf <= tol;
    d.linear_solver_status_last = abs_ok ? ECG_SOLVER_CONVERGED_ABSOLUTE
                                         : (rel_ok ? ECG_SOLVER_CONVERGED_RELATIVE : ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED);
    if (!std::isfinite(lr) || nf) {
      d.solver_status = ECG_SOLVER_LINEAR_RESIDUAL_NONFINITE;
      d.nonfinite_count = 1;
      return matrix_report();
    }
    if (!abs_ok && !rel_ok) {
      d.solver_status = g.breakdown ? ECG_SOLVER_GMRES_BREAKDOWN_NOT_CONVERGED : ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED;
      return matrix_report();
    }
    const EcgImexStats& sr = im->h_st[slot_refresh(pic)];
    d.kinetic_lag_nonfinite_count = static_cast<int>(sr.k_nonfinite);
    if (sr.k_nonfinite > 0) {
      d.solver_status = ECG_SOLVER_SOURCE_MAP_LAGGED_MOMENTUM_NONFINITE;
      d.nonfinite_count = d.kinetic_lag_nonfinite_count;
      return matrix_report();
    }
    ++d.kinetic_lag_update_count;
    d.pressure_picard_delta_linf = kd(sr.delta_linf_key);
    d.source_picard_delta_l2_relative_to_pmax = std::sqrt(sr.delta_l2_sum / static_cast<double>(n)) / kd(sr.pmax_key);
    ++d.source_picard_iterations_used;
    ++d.picard_pressure_solves_used;
  }
  d.solver_status = d.linear_solver_status_last;
  if (passes > 0) matrix_report();

  const EcgImexStats& st = im->h_st[slot_close(passes)];
  const int rcount = static_cast<int>(st.residual_count);
  const int nfc = static_cast<int>(st.final_nonfinite);
  double rl1 = 0.0, ml1 = 0.0, el1 = 0.0;
  double rlinf = kd(st.res_linf_key), rrel = kd(st.res_rel_key), mlinf = kd(st.mis_linf_key), mrel = kd(st.mis_rel_key);
  double e78 = kd(st.eq78_key), e78s = kd(st.eq78_scaled_key);
  if (nfc > 0 || rcount == 0) {
    rl1 = rlinf = rrel = ml1 = mlinf = mrel = el1 = e78 = e78s = inf;
  } else if (st.eq78_count == 0) {
    e78 = e78s = inf;
  } else {
    const double ic = 1.0 / static_cast<double>(rcount);
    rl1 = st.res_sum * ic;
    ml1 = st.mis_sum * ic;
    el1 = st.energy_sum * ic;
  }
  d.coupled_residual_l1_final = rl1;
  d.coupled_residual_linf_final = rlinf;
  d.coupled_residual_relative_linf_final = rrel;
  d.pressure_energy_residual_l1 = ml1;
  d.pressure_energy_residual_linf = mlinf;
  d.pressure_energy_residual_relative_linf = mrel;
  d.rho_min = finite_or_nan(kd(st.density_min_key));
  d.pressure_min = finite_or_nan(kd(st.eos_p_min_key));
  d.internal_energy_min = finite_or_nan(kd(st.ie_min_key));
  d.trial_density_min = d.rho_min;
  d.solved_pressure_min = finite_or_nan(kd(st.solved_p_min_key));
  d.solved_pressure_max = finite_or_nan(kd(st.solved_p_max_key));
  d.eos_pressure_min = finite_or_nan(kd(st.eos_p_min_key));
  d.eos_pressure_max = finite_or_nan(kd(st.eos_p_max_key));
  d.internal_energy_max = finite_or_nan(kd(st.ie_max_key));
  d.nonfinite_count = nfc;
  d.positivity_failure_count = static_cast<int>(st.density_fail + st.pressure_fail + st.ie_fail);
  d.momentum_correction_linf = kd(st.momentum_corr_key);
  d.energy_correction_linf = kd(st.energy_corr_key);
  d.energy_closeout_delta_linf = kd(st.energy_corr_key);
  d.energy_flux_linf = kd(st.flux_linf_key);
  d.energy_flux_divergence_linf = kd(st.flux_div_key);
  d.eq78_divergence_linf = e78;
  d.eq78_divergence_scaled_linf = e78s;
  d.energy_closeout_delta_l1 = el1;
  d.face_enthalpy_denominator_guard_count = static_cast<int>(st.guard);
  d.face_enthalpy_nonfinite_count = static_cast<int>(st.h_nonfinite);
  d.energy_flux_nonfinite_count = static_cast<int>(st.flux_nonfinite);
  // copy_source_map_eval_to_state: the step reached its end, commit U^{n+1}
  c->cur ^= 1;
  c->invalidate();
  return ECG_OK;
}

// The driver loop for the IMEX method (app/driver_main.hpp:224-310).
ecg_status imex_run(ecg_ctx* c, int32_t max_step, double stop_time, ecg_run_result* out)
{
  std::memset(out, 0, sizeof(*out));
  out->dt_min = std::numeric_limits<double>::infinity();
  const double saved_stop = c->cfg.stop_time;
  c->cfg.stop_time = stop_time;
  double t = 0.0;
  int steps = 0;
  ecg_diagnostics dg;
  ecg_status e = ecg_compute_diagnostics(c, &dg);
  if (e != ECG_OK) {
    c->cfg.stop_time = saved_stop;
    return e;
  }
  if (dg.nonfinite_count > 0 || dg.rho_min <= 0.0 || dg.pressure_min <= 0.0) {
    out->failed = 1;
    out->failure_code = ECG_FAILURE_NONFINITE_STATE;
  }
  while (!out->failed && steps < max_step && t < stop_time - 1.0e-14) {
    double dt = 0.0;
    e = ecg_compute_imex_dt(c, t, &dt, nullptr);
    if (e != ECG_OK) break;
    if (!std::isfinite(dt) || dt <= 0.0) {
      out->failed = 1;
      out->failure_code = ECG_FAILURE_INVALID_TIME_STEP;
      break;
    }
    ecg_imex_diag d;
    e = ecg_imex_step(c, dt, &d);
    if (e != ECG_OK) break;
    out->imex_solver_iterations_max = std::max(out->imex_solver_iterations_max, d.solver_iterations);
    if (d.solver_status != ECG_SOLVER_CONVERGED_ABSOLUTE && d.solver_status != ECG_SOLVER_CONVERGED_RELATIVE) {
      out->failed = 1;
      out->failure_code = ECG_FAILURE_IMEX_SOLVER;
      break;
    }
    out->dt_min = std::min(out->dt_min, dt);
    out->dt_max = std::max(out->dt_max, dt);
    out->dt_sum += dt;
    t += dt;
    ++steps;
    e = ecg_compute_diagnostics(c, &dg);
    if (e != ECG_OK) break;
    if (dg.nonfinite_count > 0) out->failure_code = ECG_FAILURE_NONFINITE_STATE;
    else if (dg.rho_min <= 0.0) out->failure_code = ECG_FAILURE_NONPOSITIVE_DENSITY;
    else if (dg.pressure_min <= 0.0) out->failure_code = ECG_FAILURE_NONPOSITIVE_PRESSURE;
    out->failed = out->failure_code != 0;
  }
  if (!out->failed && steps >= max_step && t < stop_time - 1.0e-14) out->failure_code = ECG_FAILURE_MAX_STEP_BEFORE_STOP_TIME;
  out->steps = steps;
  out->time = t;
  out->diagnostics = dg;
  c->cfg.stop_time = saved_stop;
  return e;
}
