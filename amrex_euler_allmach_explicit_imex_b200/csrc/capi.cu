// C ABI of libecg (include/ecg.h): context management, Array4 state
// transfers and the explicit hot-path entry points.  The IMEX step lives in
// imex.cu, the batched driver in batched.cu, the adjoint in adjoint.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "ctx.h"
#include "ecg.h"

// ---- helpers ---------------------------------------------------------------------

namespace ecgi {

double okey_to_double(unsigned long long k)
{
  const unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  double d;
  std::memcpy(&d, &b, sizeof(d));
  return d;
}

bool cuda_ok(ecg_ctx* c, cudaError_t e, const char* what)
{
  if (e == cudaSuccess) return true;
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

// Post-shock state of the shock-density bubble,
// problems/problem_initialization.hpp:51-58 (primitive rho, u, v, p).
static const double kBubblePostShock[4] = {2.8181818181818183, 1.6064386578049976, 0.0, 5.0};

static bool toro_states(int id, double l[4], double r[4])
{
  // toro_state, problems/exact_riemann.hpp:2-35 as {rho, u, v, p}
  struct T { int id; double v[8]; };
  static const T tab[] = {
      {1, {1.0, 0.0, 0.0, 1.0, 0.125, 0.0, 0.0, 0.1}},
      {2, {1.0, -2.0, 0.0, 0.4, 1.0, 2.0, 0.0, 0.4}},
      {3, {1.0, 0.0, 0.0, 1000.0, 1.0, 0.0, 0.0, 0.01}},
      {4, {1.0, 0.0, 0.0, 0.01, 1.0, 0.0, 0.0, 100.0}},
      {5, {5.99924, 19.5975, 0.0, 460.894, 5.99242, -6.19633, 0.0, 46.0950}},
      {93, {0.445, 1.698, 0.0, 3.528, 0.5, 0.0, 0.0, 0.571}},
      {94, {1000.0, 1.0, 0.0, 1.0e5, 0.01, 1.0, 0.0, 1.0e5}},
      {95, {1.0, 0.0, 0.0, 1.01, 1.0, 0.0, 0.0, 1.0}},
      {96, {1.0, 0.0, 0.0, 1.0001, 1.0, 0.0, 0.0, 1.0}},
      {97, {1.0, 2.0, 0.0, 0.1, 1.0, -2.0, 0.0, 0.1}},
      {90, {1.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 1.0}},
      {91, {2.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 1.0}},
      {92, {2.0, 0.1, 0.0, 1.0, 1.0, 0.1, 0.0, 1.0}},
  };
  for (const T& t : tab) {
    if (t.id == id) {
      for (int q = 0; q < 4; ++q) { l[q] = t.v[q]; r[q] = t.v[4 + q]; }
      return true;
    }
  }
  return false;
}

bool is_bubble(const ecg_run_config& c)
{
  return c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D || c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL;
}

// Ghost policy of fill_problem_ghosts (problems/boundary_conditions.hpp:165-219)
// as an EcgBc + EcgProblem pair.  `outflow_only` gives the
// fill_physical_outflow_ghosts policy the IMEX step uses for non-bubble
// problems (imex/imex_source_map_step.hpp:405-409).
void make_bc(const ecg_run_config& c, bool outflow_only, EcgBc& bc, EcgProblem& pr)
{
  std::memset(&bc, 0, sizeof(bc));
  std::memset(&pr, 0, sizeof(pr));
  pr.periodic_x = c.is_periodic[0] != 0;
  pr.periodic_y = c.is_periodic[1] != 0;
  pr.problem = c.problem;
  pr.gamma = c.gamma;
  pr.interface_x = c.riemann_interface_x;
  pr.interface_y = c.riemann_interface_y;
  pr.vortex_cx = c.vortex_cx;
  pr.vortex_cy = c.vortex_cy;
  pr.density_outer = c.density_outer;
  pr.density_inner = c.density_inner;
  pr.pressure = c.pressure;
  pr.mach = c.mach;
  pr.blob_cx = c.blob_cx;
  pr.blob_cy = c.blob_cy;
  pr.blob_radius = c.blob_radius;
  pr.velocity_x = c.velocity_x;
  pr.velocity_y = c.velocity_y;
  pr.isentropic_vortex_strength = c.isentropic_vortex_strength;
  pr.prob_hi_x = c.prob_hi[0];
  pr.prob_hi_y = c.prob_hi[1];
  if (c.problem == ECG_PROBLEM_TORO1) toro_states(c.toro_test, pr.toro_l, pr.toro_r);
  const int px = pr.periodic_x ? BC_PERIODIC : BC_CLAMP;
  const int py = pr.periodic_y ? BC_PERIODIC : BC_CLAMP;
  bc.x_lo = bc.x_hi = px;
  bc.y_lo = bc.y_hi = py;
  pr.ring_kind = RING_NONE;
  if (is_bubble(c)) {
    // fill_shock_density_bubble_ghosts, boundary_conditions.hpp:27-73
    const double* q = kBubblePostShock;
    const double g = c.gamma;
    const double kin = 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
    bc.x_lo = BC_CONST;
    bc.cst[0] = q[0];
    bc.cst[1] = q[0] * q[1];
    bc.cst[2] = q[0] * q[2];
    bc.cst[3] = q[3] / (g - 1.0) + kin;
    bc.x_hi = BC_CLAMP;
    bc.y_lo = BC_REFLECT;
    bc.y_hi = BC_CLAMP;
    return;
  }
  if (c.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122) {
    // post-shock inflow on the left, outflow on the right, walls at y = 0 and y = 1
    mach122_post_shock(c.gamma, pr.post_shock);
    const double* q = pr.post_shock;
    bc.x_lo = BC_CONST;
    bc.cst[0] = q[0];
    bc.cst[1] = q[0] * q[1];
    bc.cst[2] = q[0] * q[2];
    bc.cst[3] = q[3] / (c.gamma - 1.0) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
    bc.x_hi = BC_CLAMP;
    bc.y_lo = BC_REFLECT;
    bc.y_hi = BC_REFLECT;
    return;
  }
  if (outflow_only) return;
  const bool exact = c.field_boundary == ECG_FIELD_BOUNDARY_EXACT_DIRICHLET && (!pr.periodic_x || !pr.periodic_y);
  if (!exact) return;
  switch (c.problem) {
    case ECG_PROBLEM_GRESHO_VORTEX: pr.ring_kind = RING_GRESHO; break;
    case ECG_PROBLEM_TORO1: pr.ring_kind = RING_TORO; break;
    case ECG_PROBLEM_RIEMANN_QUADRANT: pr.ring_kind = RING_QUADRANT; break;
    case ECG_PROBLEM_ADVECTION_BLOB: pr.ring_kind = RING_BLOB; break;
    default: break;
  }
  bc.ring = pr.ring_kind != RING_NONE;
}

EcgFvParams fv_params(ecg_ctx* c, bool imex_policy)
{
  EcgFvParams p;
  std::memset(&p, 0, sizeof(p));
  p.g = c->grid;
  EcgProblem pr;
  make_bc(c->cfg, imex_policy, p.bc, pr);
  p.ring = c->d_ring;
  p.ring_pitch = c->grid.nx + 4;
  p.ring_plane = static_cast<long long>(c->grid.nx + 4) * (c->grid.ny + 4);
  p.gamma = c->cfg.gamma;
  p.order = c->cfg.spatial_order;
  p.limiter = c->cfg.slope_limiter;
  p.riemann = c->cfg.riemann;
  p.march_rows = c->opt.tile_x;
  p.sm_count = c->num_sms;
  if (c->halo_lo) p.bc.x_lo = BC_HALO;
  if (c->halo_hi) p.bc.x_hi = BC_HALO;
  p.halo_lo = c->d_halo_lo;
  p.halo_hi = c->d_halo_hi;
  return p;
}

EcgProblem problem_of(ecg_ctx* c, bool imex_policy)
{
  EcgBc bc;
  EcgProblem pr;
  make_bc(c->cfg, imex_policy, bc, pr);
  return pr;
}

// Whole-state reductions of the current state into c->h_state_stats.
bool reduce_state(ecg_ctx* c)
{
  if (c->state_stats_valid) return true;
  const EcgFvParams p = fv_params(c, false);
  const int eq79 = c->cfg.method == ECG_METHOD_IMEX && c->cfg.imex_acoustic_startup == 0 &&
                   c->cfg.imex_acoustic_cfl_cap == 0.0;
  if (!cuda_ok(c, c->ops->init_state_stats(c->d_state_stats, c->stream), "init_state_stats")) return false;
  if (!cuda_ok(c, c->ops->state_reduce(p, c->cur_state(), eq79, c->d_state_stats, c->stream), "state_reduce"))
    return false;
  if (!cuda_ok(c, cudaMemcpyAsync(c->h_state_stats, c->d_state_stats, sizeof(EcgStateStats), cudaMemcpyDeviceToHost,
                                  c->stream), "copy state stats"))
    return false;
  if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "sync")) return false;
  c->state_stats_valid = true;
  return true;
}

// Copies the fused reductions of the last explicit step to the host.
bool fetch_fused(ecg_ctx* c)
{
  if (!c->fused_pending) return true;
  if (!cuda_ok(c, cudaMemcpyAsync(c->h_stats, c->d_stats + c->fused_slot, sizeof(EcgStepStats),
                                  cudaMemcpyDeviceToHost, c->stream),
               "copy stats"))
    return false;
  if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "sync")) return false;
  const EcgStepStats& s = c->h_stats[0];
  c->fused_max_rate = okey_to_double(s.max_rate_key);
  c->fused_rho_min = okey_to_double(s.rho_min_key);
  c->fused_p_min = okey_to_double(s.p_min_key);
  c->fused_nonfinite = s.nonfinite;
  c->fused_degenerate = s.degenerate;
  c->fused_pending = false;
  c->fused_valid = true;
  return true;
}

// Ghost ring for exact-state Dirichlet policies at `time` (host) or at the
// time recorded in stats[k] (device loop).
bool fill_ring(ecg_ctx* c, const double* u, double time, const EcgStepStats* stats, int k)
{
  const EcgFvParams p = fv_params(c, false);
  if (!p.bc.ring) return true;
  const EcgProblem pr = problem_of(c, false);
  return cuda_ok(c, c->ops->ghost_box(p, pr, u, time, stats, k, c->d_ring, p.ring_pitch, p.ring_plane, 1, c->stream),
                 "ghost ring");
}

}  // namespace ecgi

using namespace ecgi;

// ---- context ---------------------------------------------------------------------

ecg_ctx::~ecg_ctx()
{
  if (device >= 0) cudaSetDevice(device);
  for (auto& g : graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
  }
  imex_free(this);
  output_destroy(out);
  cudaFree(d_state[0]);
  cudaFree(d_state[1]);
  cudaFree(d_ring);
  cudaFree(d_stats);
  cudaFree(d_state_stats);
  cudaFree(adj_gq);
  cudaFree(adj_stats);
  cudaFreeHost(h_stats);
  cudaFreeHost(h_state_stats);
  for (cudaEvent_t e : band_up) cudaEventDestroy(e);
  for (cudaEvent_t e : band_done) cudaEventDestroy(e);
  for (cudaEvent_t e : band_dl) cudaEventDestroy(e);
  host_stage_destroy(stage);
  if (up_stream) cudaStreamDestroy(up_stream);
  if (down_stream) cudaStreamDestroy(down_stream);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

extern "C" {

int32_t ecg_abi_version(void) { return ECG_ABI_VERSION; }

const char* ecg_status_str(ecg_status s)
{
  switch (s) {
    case ECG_OK: return "ok";
    case ECG_ERR_BAD_ARG: return "bad argument";
    case ECG_ERR_CUDA: return "CUDA error";
    case ECG_ERR_TIMEOUT: return "device wait timed out";
    case ECG_ERR_NO_DEVICE: return "no usable sm_100 device";
    case ECG_ERR_UNSUPPORTED: return "unsupported configuration";
    case ECG_ERR_NOT_READY: return "state not uploaded";
    case ECG_ERR_IO: return "output file not written";
  }
  return "unknown status";
}

const char* ecg_solver_status_str(int32_t s)
{
  // ImexStepDiagnostics::solver_status strings (imex/imex_source_map_step.hpp:398-567)
  switch (s) {
    case ECG_SOLVER_NOT_RUN: return "not_run";
    case ECG_SOLVER_CONVERGED_ABSOLUTE: return "converged_absolute";
    case ECG_SOLVER_CONVERGED_RELATIVE: return "converged_relative";
    case ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED: return "linear_solve_not_converged";
    case ECG_SOLVER_GMRES_BREAKDOWN_NOT_CONVERGED: return "gmres_breakdown_not_converged";
    case ECG_SOLVER_LINEAR_RESIDUAL_NONFINITE: return "linear_residual_nonfinite";
    case ECG_SOLVER_SOURCE_MAP_PRESSURE_ROW_NONFINITE: return "source_map_pressure_row_nonfinite";
    case ECG_SOLVER_SOURCE_MAP_LAGGED_MOMENTUM_NONFINITE: return "source_map_lagged_momentum_nonfinite";
    case ECG_SOLVER_DENSITY_DENOMINATOR_FLOOR_USED: return "density_denominator_floor_used";
    case ECG_SOLVER_UNSUPPORTED_MPI: return "unsupported_mpi_for_host_single_level_gmres";
  }
  return "unset";
}

void ecg_default_run_config(ecg_run_config* c)
{
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  // RunConfig defaults, core/run_config.hpp:2-55
  c->n_cell[0] = 64;
  c->n_cell[1] = 64;
  c->is_periodic[0] = 1;
  c->is_periodic[1] = 1;
  c->prob_hi[0] = 1.0;
  c->prob_hi[1] = 1.0;
  c->max_step = 8;
  c->spatial_order = 1;
  c->toro_test = 1;
  c->problem = ECG_PROBLEM_ADVECTION_BLOB;
  c->riemann = ECG_RIEMANN_HLLC;
  c->method = ECG_METHOD_EXPLICIT;
  c->slope_limiter = ECG_LIMITER_MINMOD;
  c->field_boundary = ECG_FIELD_BOUNDARY_OUTFLOW;
  c->stop_time = 0.05;
  c->gamma = 1.4;
  c->cfl = 0.4;
  c->imex_cfl = 0.8;
  c->imex_solver_tol = 1.0e-10;
  c->velocity_x = 1.0;
  c->velocity_y = 0.5;
  c->density_inner = 2.0;
  c->density_outer = 1.0;
  c->pressure = 1.0;
  c->mach = 0.1;
  c->blob_cx = 0.35;
  c->blob_cy = 0.35;
  c->blob_radius = 0.15;
  c->isentropic_vortex_strength = 5.0;
  c->riemann_interface_x = 0.5;
  c->riemann_interface_y = 0.5;
  c->imex_solver_max_iter = 100;
  c->imex_acoustic_startup = 1;
  c->imex_picard_extra_iterations = 1;
  c->imex_picard_iterations = 2;
}

void ecg_default_gpu_options(ecg_gpu_options* o)
{
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->arith = ECG_ARITH_FAST;
  o->imex_precision = ECG_IMEX_FP64;
  o->mixed_inner_max_iter = 0;
  o->mixed_inner_rtol = -1.0;  // chosen per system (ecg.h)
  o->mixed_max_refinements = 12;
  o->mixed_reorth = 0;
  o->mixed_min_iterations = 8;
  o->tile_x = 0;
  o->tile_y = 0;
  o->stream = nullptr;
}

ecg_status ecg_create(ecg_ctx** out, const ecg_run_config* cfg, const ecg_gpu_options* opt)
{
  if (!out || !cfg) return ECG_ERR_BAD_ARG;
  *out = nullptr;
  const int nx = cfg->n_cell[0], ny = cfg->n_cell[1];
  if (nx < 1 || ny < 1 || static_cast<long long>(nx) * ny > (1LL << 31)) return ECG_ERR_BAD_ARG;
  if (cfg->spatial_order != 1 && cfg->spatial_order != 2) return ECG_ERR_BAD_ARG;
  if (cfg->riemann < 0 || cfg->riemann > 3 || cfg->slope_limiter < 0 || cfg->slope_limiter > 2) return ECG_ERR_BAD_ARG;
  if (!(cfg->gamma > 1.0) || !(cfg->prob_hi[0] > cfg->prob_lo[0]) || !(cfg->prob_hi[1] > cfg->prob_lo[1]))
    return ECG_ERR_BAD_ARG;
  if (cfg->problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL) return ECG_ERR_UNSUPPORTED;
  ecg_gpu_options o;
  if (opt) o = *opt;
  else ecg_default_gpu_options(&o);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) return ECG_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major != 10) return ECG_ERR_NO_DEVICE;
  if (cudaSetDevice(o.device) != cudaSuccess) return ECG_ERR_NO_DEVICE;

  ecg_ctx* c = new ecg_ctx();
  c->cfg = *cfg;
  c->opt = o;
  c->device = o.device;
  c->num_sms = prop.multiProcessorCount;
  c->ops = o.arith == ECG_ARITH_EXACT ? &ecg_exact_ops : &ecg_fast_ops;
  c->grid.nx = nx;
  c->grid.ny = ny;
  c->grid.pitch = (nx + 31) / 32 * 32;  // 256-byte aligned rows
  c->grid.plane = c->grid.pitch * ny;
  // AMReX Geometry cell size: (hi - lo) / n  (AMReX_Geometry.cpp:527)
  c->grid.dx = (cfg->prob_hi[0] - cfg->prob_lo[0]) / static_cast<double>(nx);
  c->grid.dy = (cfg->prob_hi[1] - cfg->prob_lo[1]) / static_cast<double>(ny);
  // explicit_update.hpp:69-70
  c->grid.inv_dx = 1.0 / c->grid.dx;
  c->grid.inv_dy = 1.0 / c->grid.dy;
  c->grid.plo_x = cfg->prob_lo[0];
  c->grid.plo_y = cfg->prob_lo[1];
  // kernel choice: 0 default (fast build: column-strip kernel with paired
  // faces; exact build: 32x16 tile), 2 column strips with faces one at a time,
  // 1 square 16x16 tile (fast build), 8 or 16: 32xTY tile
  c->tile_y = (o.tile_y == 1 || o.tile_y == 2 || o.tile_y == 3 || o.tile_y == 8 || o.tile_y == 16) ? o.tile_y : 0;
  const size_t sbytes = sizeof(double) * 4 * c->grid.plane;
  bool ok = true;
  if (o.stream) {
    c->stream = static_cast<cudaStream_t>(o.stream);
    c->own_stream = false;
  } else {
    ok = ok && cuda_ok(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
    c->own_stream = true;
  }
  ok = ok && cuda_ok(c, cudaMalloc(&c->d_state[0], sbytes), "alloc state");
  ok = ok && cuda_ok(c, cudaMalloc(&c->d_state[1], sbytes), "alloc state");
  ok = ok && cuda_ok(c, cudaMemsetAsync(c->d_state[0], 0, sbytes, c->stream), "memset");
  ok = ok && cuda_ok(c, cudaMemsetAsync(c->d_state[1], 0, sbytes, c->stream), "memset");
  const size_t rbytes = sizeof(double) * 4 * static_cast<size_t>(nx + 4) * (ny + 4);
  ok = ok && cuda_ok(c, cudaMalloc(&c->d_ring, rbytes), "alloc ring");
  ok = ok && cuda_ok(c, cudaMemsetAsync(c->d_ring, 0, rbytes, c->stream), "memset");
  c->stats_cap = ecg_ctx::kChunk + 1;  // >= 3 host-mode slots
  ok = ok && cuda_ok(c, cudaMalloc(&c->d_stats, sizeof(EcgStepStats) * c->stats_cap), "alloc stats");
  ok = ok && cuda_ok(c, cudaMallocHost(&c->h_stats, sizeof(EcgStepStats) * c->stats_cap), "alloc host stats");
  ok = ok && cuda_ok(c, cudaMalloc(&c->d_state_stats, sizeof(EcgStateStats)), "alloc state stats");
  ok = ok && cuda_ok(c, cudaMallocHost(&c->h_state_stats, sizeof(EcgStateStats)), "alloc host state stats");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(c->stream), "sync");
  if (!ok) {
    std::fprintf(stderr, "ecg_create: %s\n", c->err.c_str());
    delete c;
    return ECG_ERR_CUDA;
  }
  *out = c;
  return ECG_OK;
}

void ecg_destroy(ecg_ctx* ctx) { delete ctx; }

const char* ecg_last_error(const ecg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

ecg_status ecg_synchronize(ecg_ctx* c)
{
  if (!c) return ECG_ERR_BAD_ARG;
  return cuda_ok(c, cudaStreamSynchronize(c->stream), "sync") ? ECG_OK : ECG_ERR_CUDA;
}

// ---- state exchange ----------------------------------------------------------

// One event per band of rows in `ev` (created on first use).
static bool band_events(ecg_ctx* c, std::vector<cudaEvent_t>& ev, int nb)
{
  while (static_cast<int>(ev.size()) < nb) {
    cudaEvent_t e = nullptr;
    if (!cuda_ok(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event")) return false;
    ev.push_back(e);
  }
  return true;
}

// Rows [r0, r1) of the 4 planes between the compact stage (pitch nx) and the
// device state (the context's pitch and plane).
static cudaError_t stage_rows(ecg_ctx* c, double* stage, double* dev, int r0, int r1, bool upload, cudaStream_t st)
{
  const int nx = c->grid.nx;
  const size_t splane = static_cast<size_t>(nx) * static_cast<size_t>(c->grid.ny);
  for (int n = 0; n < 4; ++n) {
    double* s = stage + n * splane + static_cast<size_t>(r0) * nx;
    double* d = dev + n * c->grid.plane + static_cast<long long>(r0) * c->grid.pitch;
    const cudaError_t e =
        upload ? cudaMemcpy2DAsync(d, sizeof(double) * c->grid.pitch, s, sizeof(double) * nx, sizeof(double) * nx,
                                   r1 - r0, cudaMemcpyHostToDevice, st)
               : cudaMemcpy2DAsync(s, sizeof(double) * nx, d, sizeof(double) * c->grid.pitch, sizeof(double) * nx,
                                   r1 - r0, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The state to or from a pageable host box (host: offset to cell (0, 0))
// through the pinned stage in bands of rows: the host threads copy band b+1
// while band b crosses.
static ecg_status transfer_staged(ecg_ctx* c, double* host, int64_t jstride, int64_t nstride, bool upload)
{
  const int nx = c->grid.nx, ny = c->grid.ny;
  HostStage* hs = host_stage(c);
  if (!hs) return ECG_ERR_CUDA;
  const int nb = ny < 64 ? 1 : std::min(8, ny / 32);
  auto row0 = [&](int b) { return static_cast<int>(static_cast<long long>(ny) * b / nb); };
  double* dev = c->cur_state_mut();
  if (upload) {
    double* stage = host_stage_in(hs);
    for (int b = 0; b < nb; ++b) {
      host_stage_copy(hs, stage, host, jstride, nstride, nx, ny, row0(b), row0(b + 1), true);
      if (!cuda_ok(c, stage_rows(c, stage, dev, row0(b), row0(b + 1), true, c->stream), "upload")) return ECG_ERR_CUDA;
    }
    c->uploaded = true;
    c->invalidate();
    return cuda_ok(c, cudaStreamSynchronize(c->stream), "sync") ? ECG_OK : ECG_ERR_CUDA;
  }
  double* stage = host_stage_out(hs);
  if (!band_events(c, c->band_dl, nb)) return ECG_ERR_CUDA;
  for (int b = 0; b < nb; ++b) {
    if (!cuda_ok(c, stage_rows(c, stage, dev, row0(b), row0(b + 1), false, c->stream), "download") ||
        !cuda_ok(c, cudaEventRecord(c->band_dl[b], c->stream), "event"))
      return ECG_ERR_CUDA;
  }
  for (int b = 0; b < nb; ++b) {
    if (!cuda_ok(c, cudaEventSynchronize(c->band_dl[b]), "sync")) return ECG_ERR_CUDA;
    host_stage_copy(hs, stage, host, jstride, nstride, nx, ny, row0(b), row0(b + 1), false);
  }
  return ECG_OK;
}

static ecg_status transfer(ecg_ctx* c, double* host, const double* hostc, int32_t lo_x, int32_t lo_y, int64_t jstride,
                           int64_t nstride, bool upload, bool device_side)
{
  if (!c || (!host && !hostc)) return ECG_ERR_BAD_ARG;
  const int nx = c->grid.nx, ny = c->grid.ny;
  if (lo_x > 0 || lo_y > 0 || jstride < nx - lo_x || nstride < jstride * (ny - lo_y)) return ECG_ERR_BAD_ARG;
  const int64_t off = static_cast<int64_t>(-lo_x) + static_cast<int64_t>(-lo_y) * jstride;
  const cudaMemcpyKind kind = device_side ? cudaMemcpyDeviceToDevice
                                          : (upload ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost);
  double* dev = upload ? c->cur_state_mut() : c->cur_state_mut();
  if (!device_side && host_pageable(upload ? static_cast<const void*>(hostc) : static_cast<const void*>(host)))
    return transfer_staged(c, upload ? const_cast<double*>(hostc) + off : host + off, jstride, nstride, upload);
  for (int n = 0; n < 4; ++n) {
    double* d = dev + n * c->grid.plane;
    cudaError_t e;
    if (upload) {
      e = cudaMemcpy2DAsync(d, sizeof(double) * c->grid.pitch, hostc + off + n * nstride, sizeof(double) * jstride,
                            sizeof(double) * nx, ny, kind, c->stream);
    } else {
      e = cudaMemcpy2DAsync(host + off + n * nstride, sizeof(double) * jstride, d, sizeof(double) * c->grid.pitch,
                            sizeof(double) * nx, ny, kind, c->stream);
    }
    if (!cuda_ok(c, e, upload ? "upload" : "download")) return ECG_ERR_CUDA;
  }
  if (upload) {
    c->uploaded = true;
    c->invalidate();
  }
  // Host memory may be pageable and is reused by the caller on return.
  if (!device_side && !cuda_ok(c, cudaStreamSynchronize(c->stream), "sync")) return ECG_ERR_CUDA;
  return ECG_OK;
}

ecg_status ecg_upload_state(ecg_ctx* c, const double* base, int32_t lo_x, int32_t lo_y, int64_t jstride, int64_t nstride)
{
  return transfer(c, nullptr, base, lo_x, lo_y, jstride, nstride, true, false);
}

ecg_status ecg_download_state(ecg_ctx* c, double* base, int32_t lo_x, int32_t lo_y, int64_t jstride, int64_t nstride)
{
  if (c && !c->uploaded) return ECG_ERR_NOT_READY;
  return transfer(c, base, nullptr, lo_x, lo_y, jstride, nstride, false, false);
}

ecg_status ecg_upload_state_device(ecg_ctx* c, const double* base, int32_t lo_x, int32_t lo_y, int64_t jstride,
                                   int64_t nstride)
{
  return transfer(c, nullptr, base, lo_x, lo_y, jstride, nstride, true, true);
}

ecg_status ecg_download_state_device(ecg_ctx* c, double* base, int32_t lo_x, int32_t lo_y, int64_t jstride,
                                     int64_t nstride)
{
  if (c && !c->uploaded) return ECG_ERR_NOT_READY;
  return transfer(c, base, nullptr, lo_x, lo_y, jstride, nstride, false, true);
}

ecg_status ecg_initialize_state(ecg_ctx* c)
{
  if (!c) return ECG_ERR_BAD_ARG;
  const EcgFvParams p = fv_params(c, false);
  const EcgProblem pr = problem_of(c, false);
  if (!cuda_ok(c, c->ops->init_state(p, pr, c->cur_state_mut(), c->stream), "initialize state")) return ECG_ERR_CUDA;
  c->uploaded = true;
  c->invalidate();
  return ECG_OK;
}

ecg_status ecg_fill_problem_ghosts(ecg_ctx* c, double time, double* ghosted_host)
{
  if (!c || !ghosted_host) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  const EcgFvParams p = fv_params(c, false);
  const EcgProblem pr = problem_of(c, false);
  const long long gp = c->grid.nx + 4, gpl = gp * (c->grid.ny + 4);
  double* d = nullptr;
  if (!cuda_ok(c, cudaMallocAsync(&d, sizeof(double) * 4 * gpl, c->stream), "alloc")) return ECG_ERR_CUDA;
  bool ok = cuda_ok(c, c->ops->ghost_box(p, pr, c->cur_state(), time, nullptr, 0, d, gp, gpl, 0, c->stream), "ghost box");
  ok = ok && cuda_ok(c, cudaMemcpyAsync(ghosted_host, d, sizeof(double) * 4 * gpl, cudaMemcpyDeviceToHost, c->stream),
                     "copy");
  cudaFreeAsync(d, c->stream);
  ok = ok && cuda_ok(c, cudaStreamSynchronize(c->stream), "sync");
  return ok ? ECG_OK : ECG_ERR_CUDA;
}

// ---- explicit hot path ------------------------------------------------------

ecg_status ecg_euler_fv_one_step(ecg_ctx* c, double dt, double time, int32_t* degenerate)
{
  if (!c) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  const EcgFvParams p = fv_params(c, false);
  // Host-dt launches rotate over three stats records: launch n accumulates
  // into (n+1)%3 and re-initialises (n+2)%3 for launch n+1, so one launch is
  // the whole step.
  if (!c->host_slots_ready) {
    if (!cuda_ok(c, c->ops->init_stats(c->d_stats, 3, time, c->stream), "init stats")) return ECG_ERR_CUDA;
    c->host_slots_ready = true;
    c->host_step = 0;
  }
  EcgDtCtl ctl;
  std::memset(&ctl, 0, sizeof(ctl));
  ctl.device_dt = 0;
  ctl.dt = dt;
  ctl.time = time;
  ctl.count_degenerate = c->cfg.riemann != ECG_RIEMANN_RUSANOV;
  ctl.read_slot = static_cast<int>(c->host_step % 3);
  ctl.acc_slot = static_cast<int>((c->host_step + 1) % 3);
  ctl.reset_slot = static_cast<int>((c->host_step + 2) % 3);
  if (!fill_ring(c, c->cur_state(), time, nullptr, 0)) return ECG_ERR_CUDA;
  if (!cuda_ok(c, c->ops->fv_step(p, c->cur_state(), c->next_state(), c->d_stats, ctl, c->tile_y, c->stream),
               "fv_step"))
    return ECG_ERR_CUDA;
  c->cur ^= 1;
  ++c->host_step;
  // The fused epilogue reduced compute_euler_dt / compute_diagnostics over the
  // new state into d_stats[acc_slot]: those calls read it instead of a second pass.
  c->state_stats_valid = false;
  c->fused_valid = false;
  c->fused_pending = true;
  c->fused_slot = ctl.acc_slot;
  if (degenerate) {
    if (!fetch_fused(c)) return ECG_ERR_CUDA;
    *degenerate = c->fused_degenerate;
  }
  return ECG_OK;
}

// euler_fv_one_step on a host-resident box, pipelined over bands of rows:
// band b+1 is copied to the device on one stream while band b is stepped on
// the context's stream and the finished bands are copied back on a third,
// so the two copy directions and the step overlap.  Falls back to upload,
// step, download in sequence where the step is not the column-strip kernel
// (exact arithmetic, HLLC-P off the staged strips, exact-Dirichlet rings).
ecg_status ecg_euler_fv_one_step_host(ecg_ctx* c, const double* in, double* out, int32_t lo_x, int32_t lo_y,
                                      int64_t jstride, int64_t nstride, double dt, double time, int32_t* degenerate)
{
  if (!c || !in || !out) return ECG_ERR_BAD_ARG;
  const int nx = c->grid.nx, ny = c->grid.ny;
  if (lo_x > 0 || lo_y > 0 || jstride < nx - lo_x || nstride < jstride * (ny - lo_y)) return ECG_ERR_BAD_ARG;
  EcgFvParams p = fv_params(c, false);
  // HLLC-P takes bands on the staged strips only (tile_y 0)
  const bool banded = c->opt.arith == ECG_ARITH_FAST && (c->tile_y == 0 || c->tile_y == 2 || c->tile_y == 3) && !c->slab() &&
                      (c->cfg.riemann != ECG_RIEMANN_XIE_AM_HLLC_P || c->tile_y == 0) && !p.bc.ring && ny >= 32;
  if (!banded) {
    ecg_status st = ecg_upload_state(c, in, lo_x, lo_y, jstride, nstride);
    if (st == ECG_OK) st = ecg_euler_fv_one_step(c, dt, time, degenerate);
    if (st == ECG_OK) st = ecg_download_state(c, out, lo_x, lo_y, jstride, nstride);
    return st;
  }
  // bands of at least 16 rows, at most 8 of them
  const int nb = ny / 16 < 8 ? ny / 16 : 8;
  if (!c->up_stream && !cuda_ok(c, cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking), "stream"))
    return ECG_ERR_CUDA;
  if (!c->down_stream && !cuda_ok(c, cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking), "stream"))
    return ECG_ERR_CUDA;
  while (static_cast<int>(c->band_up.size()) < nb) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (!cuda_ok(c, cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "event") ||
        !cuda_ok(c, cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "event"))
      return ECG_ERR_CUDA;
    c->band_up.push_back(a);
    c->band_done.push_back(b);
  }
  auto row0 = [&](int b) { return static_cast<int>(static_cast<long long>(ny) * b / nb); };
  const int64_t off = static_cast<int64_t>(-lo_x) + static_cast<int64_t>(-lo_y) * jstride;
  double* cur = c->cur_state_mut();
  double* nxt = c->next_state();
  // the previous call's work on the context's stream (and its read of this
  // context's state) is ordered before the uploads
  if (!cuda_ok(c, cudaEventRecord(c->band_done[0], c->stream), "event") ||
      !cuda_ok(c, cudaStreamWaitEvent(c->up_stream, c->band_done[0], 0), "event"))
    return ECG_ERR_CUDA;
  // Pageable boxes cross through the context's pinned stage (compact, pitch
  // nx): the host threads copy band b+1 into it while band b crosses, and the
  // downloaded bands are copied out of it as each one lands.
  const bool stage_in = host_pageable(in), stage_out = host_pageable(out);
  HostStage* hs = nullptr;
  if ((stage_in || stage_out) && !(hs = host_stage(c))) return ECG_ERR_CUDA;
  if (stage_out && !band_events(c, c->band_dl, nb)) return ECG_ERR_CUDA;
  const long long splane = static_cast<long long>(nx) * ny;
  // The four field planes of a band move in one 3D copy (planes at a fixed
  // stride on both sides); per-plane 2D copies otherwise.  Fewer, larger copy
  // commands let the two directions share the link better.
  auto copy_band = [&](double* dst, long long dpitch, long long dslice, const double* src, long long spitch,
                       long long sslice, int rows, cudaMemcpyKind kind, cudaStream_t st) -> cudaError_t {
    if (sslice % spitch == 0 && dslice % dpitch == 0) {
      cudaMemcpy3DParms m;
      std::memset(&m, 0, sizeof(m));
      m.srcPtr = make_cudaPitchedPtr(const_cast<double*>(src), sizeof(double) * spitch, sizeof(double) * nx,
                                     static_cast<size_t>(sslice / spitch));
      m.dstPtr = make_cudaPitchedPtr(dst, sizeof(double) * dpitch, sizeof(double) * nx,
                                     static_cast<size_t>(dslice / dpitch));
      m.extent = make_cudaExtent(sizeof(double) * nx, static_cast<size_t>(rows), 4);
      m.kind = kind;
      return cudaMemcpy3DAsync(&m, st);
    }
    for (int n = 0; n < 4; ++n) {
      const cudaError_t e = cudaMemcpy2DAsync(dst + n * dslice, sizeof(double) * dpitch, src + n * sslice,
                                              sizeof(double) * spitch, sizeof(double) * nx, rows, kind, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  auto upload_rows = [&](int r0, int r1) -> cudaError_t {
    if (stage_in) {
      double* stage = host_stage_in(hs);
      host_stage_copy(hs, stage, const_cast<double*>(in) + off, jstride, nstride, nx, ny, r0, r1, true);
      return copy_band(cur + static_cast<long long>(r0) * c->grid.pitch, c->grid.pitch, c->grid.plane,
                       stage + static_cast<long long>(r0) * nx, nx, splane, r1 - r0, cudaMemcpyHostToDevice,
                       c->up_stream);
    }
    return copy_band(cur + static_cast<long long>(r0) * c->grid.pitch, c->grid.pitch, c->grid.plane,
                     in + off + static_cast<int64_t>(r0) * jstride, jstride, nstride, r1 - r0, cudaMemcpyHostToDevice,
                     c->up_stream);
  };
  // Band b's step reads rows row0(b) - 2 .. row0(b + 1) + 1, so upload chunk
  // b carries its band's rows shifted by two, [row0(b) + 2, row0(b + 1) + 2)
  // (the first from row 0, the last to row ny), and band b waits for chunk b
  // alone: the downloads start one band earlier than if band b also waited
  // for the next band's upload.  Under periodic y the first band's ghost rows
  // are rows ny - 2 and ny - 1; they cross ahead of chunk 0 (bands are at
  // least 16 rows, so every chunk is non-empty).
  const bool wrap_y = p.bc.y_lo == BC_PERIODIC;
  if (wrap_y && !cuda_ok(c, upload_rows(ny - 2, ny), "upload rows")) return ECG_ERR_CUDA;
  for (int b = 0; b < nb; ++b) {
    const int lo = b == 0 ? 0 : row0(b) + 2;
    const int hi = b + 1 < nb ? row0(b + 1) + 2 : (wrap_y ? ny - 2 : ny);
    if (!cuda_ok(c, upload_rows(lo, hi), "upload band")) return ECG_ERR_CUDA;
    if (!cuda_ok(c, cudaEventRecord(c->band_up[b], c->up_stream), "event")) return ECG_ERR_CUDA;
  }
  c->uploaded = true;
  c->invalidate();
  if (!c->host_slots_ready) {
    if (!cuda_ok(c, c->ops->init_stats(c->d_stats, 3, time, c->stream), "init stats")) return ECG_ERR_CUDA;
    c->host_slots_ready = true;
    c->host_step = 0;
  }
  EcgDtCtl ctl;
  std::memset(&ctl, 0, sizeof(ctl));
  ctl.dt = dt;
  ctl.time = time;
  ctl.count_degenerate = c->cfg.riemann != ECG_RIEMANN_RUSANOV;
  ctl.read_slot = static_cast<int>(c->host_step % 3);
  ctl.acc_slot = static_cast<int>((c->host_step + 1) % 3);
  ctl.reset_slot = static_cast<int>((c->host_step + 2) % 3);
  for (int b = 0; b < nb; ++b) {
    // rows r0-2 .. r1+1 are read: chunk b holds those not in earlier chunks
    if (!cuda_ok(c, cudaStreamWaitEvent(c->stream, c->band_up[b], 0), "event")) return ECG_ERR_CUDA;
    p.row_lo = row0(b);
    p.row_hi = row0(b + 1);
    if (!cuda_ok(c, c->ops->fv_step(p, cur, nxt, c->d_stats, ctl, c->tile_y, c->stream), "fv_step band"))
      return ECG_ERR_CUDA;
    if (!cuda_ok(c, cudaEventRecord(c->band_done[b], c->stream), "event") ||
        !cuda_ok(c, cudaStreamWaitEvent(c->down_stream, c->band_done[b], 0), "event"))
      return ECG_ERR_CUDA;
    const int r0 = row0(b), r1 = row0(b + 1);
    if (stage_out) {
      if (!cuda_ok(c, copy_band(host_stage_out(hs) + static_cast<long long>(r0) * nx, nx, splane,
                                nxt + static_cast<long long>(r0) * c->grid.pitch, c->grid.pitch, c->grid.plane,
                                r1 - r0, cudaMemcpyDeviceToHost, c->down_stream),
                   "download band") ||
          !cuda_ok(c, cudaEventRecord(c->band_dl[b], c->down_stream), "event"))
        return ECG_ERR_CUDA;
    } else if (!cuda_ok(c, copy_band(out + off + static_cast<int64_t>(r0) * jstride, jstride, nstride,
                                     nxt + static_cast<long long>(r0) * c->grid.pitch, c->grid.pitch, c->grid.plane,
                                     r1 - r0, cudaMemcpyDeviceToHost, c->down_stream),
                        "download band")) {
      return ECG_ERR_CUDA;
    }
  }
  if (stage_out) {
    for (int b = 0; b < nb; ++b) {
      if (!cuda_ok(c, cudaEventSynchronize(c->band_dl[b]), "sync")) return ECG_ERR_CUDA;
      host_stage_copy(hs, host_stage_out(hs), out + off, jstride, nstride, nx, ny, row0(b), row0(b + 1), false);
    }
  }
  c->cur ^= 1;
  ++c->host_step;
  c->state_stats_valid = false;
  c->fused_valid = false;
  c->fused_pending = true;
  c->fused_slot = ctl.acc_slot;
  // the caller owns `out` on return; the context's stream waits for the
  // copies before it touches the state again
  if (!cuda_ok(c, cudaEventRecord(c->band_up[0], c->down_stream), "event") ||
      !cuda_ok(c, cudaStreamWaitEvent(c->stream, c->band_up[0], 0), "event") ||
      !cuda_ok(c, cudaStreamSynchronize(c->down_stream), "sync"))
    return ECG_ERR_CUDA;
  if (degenerate) {
    if (!fetch_fused(c)) return ECG_ERR_CUDA;
    *degenerate = c->fused_degenerate;
  }
  return ECG_OK;
}

ecg_status ecg_compute_euler_dt(ecg_ctx* c, double time, double* dt)
{
  if (!c || !dt) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  double rate;
  if (!fetch_fused(c)) return ECG_ERR_CUDA;
  if (c->fused_valid) {
    rate = c->fused_max_rate;
  } else {
    if (!reduce_state(c)) return ECG_ERR_CUDA;
    rate = okey_to_double(c->h_state_stats->max_rate_key);
  }
  // diagnostic_metrics_timestep.hpp:252-259
  double d = c->cfg.stop_time - time;
  if (rate > 0.0) d = c->cfg.cfl / rate;
  if (!std::isfinite(d) || d <= 0.0) d = c->cfg.stop_time - time;
  *dt = std::min(d, c->cfg.stop_time - time);
  return ECG_OK;
}

ecg_status ecg_compute_imex_dt(ecg_ctx* c, double time, double* dt, ecg_imex_timestep_diag* diag)
{
  if (!c || !dt) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (!reduce_state(c)) return ECG_ERR_CUDA;
  // diagnostic_metrics_timestep.hpp:301-325
  ecg_imex_timestep_diag td;
  td.material_rate_max = okey_to_double(c->h_state_stats->material_rate_key);
  td.acoustic_rate_max = okey_to_double(c->h_state_stats->acoustic_rate_key);
  td.acoustic_startup_used = 0;
  td.acoustic_cap_used = 0;
  double rate = td.material_rate_max;
  if (c->cfg.imex_acoustic_startup != 0 && td.material_rate_max <= 1.0e-12 && td.acoustic_rate_max > 0.0) {
    rate = td.acoustic_rate_max;
    td.acoustic_startup_used = 1;
  }
  double d = c->cfg.stop_time - time;
  if (rate > 0.0) d = c->cfg.imex_cfl / rate;
  if (c->cfg.imex_acoustic_cfl_cap > 0.0 && td.acoustic_rate_max > 0.0) {
    const double lim = c->cfg.imex_acoustic_cfl_cap / td.acoustic_rate_max;
    if (lim < d) {
      d = lim;
      td.acoustic_cap_used = 1;
    }
  }
  if (!std::isfinite(d) || d <= 0.0) d = c->cfg.stop_time - time;
  *dt = std::min(d, c->cfg.stop_time - time);
  if (diag) *diag = td;
  return ECG_OK;
}

ecg_status ecg_compute_diagnostics(ecg_ctx* c, ecg_diagnostics* out)
{
  if (!c || !out) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (!fetch_fused(c)) return ECG_ERR_CUDA;
  if (c->fused_valid) {
    out->rho_min = c->fused_rho_min;
    out->pressure_min = c->fused_p_min;
    out->nonfinite_count = c->fused_nonfinite;
    return ECG_OK;
  }
  if (!reduce_state(c)) return ECG_ERR_CUDA;
  out->rho_min = okey_to_double(c->h_state_stats->diag_rho_min_key);
  out->pressure_min = okey_to_double(c->h_state_stats->diag_p_min_key);
  out->nonfinite_count = c->h_state_stats->diag_nonfinite;
  return ECG_OK;
}

ecg_status ecg_compute_admissibility_diagnostics(ecg_ctx* c, ecg_admissibility* out)
{
  if (!c || !out) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (!reduce_state(c)) return ECG_ERR_CUDA;
  const EcgStateStats& s = *c->h_state_stats;
  out->rho_min = okey_to_double(s.adm_rho_min_key);
  out->pressure_min = okey_to_double(s.adm_p_min_key);
  out->internal_energy_min = okey_to_double(s.adm_ie_min_key);
  out->nonfinite_count = s.adm_nonfinite;
  out->density_failure_count = s.adm_density_fail;
  out->pressure_failure_count = s.adm_pressure_fail;
  out->internal_energy_failure_count = s.adm_ie_fail;
  return ECG_OK;
}

// The driver loop (app/driver_main.hpp:216-340) for the explicit method,
// kept on the device: chunks of kChunk launches captured once in a CUDA
// graph; dt, time, the stop test and the fail-fast checks travel between
// launches through the stats records.  One host sync per chunk.
static ecg_status run_explicit(ecg_ctx* c, int32_t max_step, double stop_time, ecg_run_result* out)
{
  std::memset(out, 0, sizeof(*out));
  out->dt_min = std::numeric_limits<double>::infinity();
  const EcgFvParams p = fv_params(c, false);
  const int K = ecg_ctx::kChunk;
  c->host_slots_ready = false;
  double t = 0.0;
  int steps = 0;
  // stats[0] <- reductions of the initial state (compute_diagnostics before
  // the loop, driver_main.hpp:216-222)
  c->state_stats_valid = false;
  if (!cuda_ok(c, c->ops->init_stats(c->d_stats, K + 1, t, c->stream), "init stats")) return ECG_ERR_CUDA;
  if (!cuda_ok(c, c->ops->init_state_stats(c->d_state_stats, c->stream), "init")) return ECG_ERR_CUDA;
  const int eq79 = 0;
  if (!cuda_ok(c, c->ops->state_reduce(p, c->cur_state(), eq79, c->d_state_stats, c->stream), "reduce"))
    return ECG_ERR_CUDA;
  if (!cuda_ok(c, c->ops->seed_stats(c->d_stats, c->d_state_stats, c->stream), "seed")) return ECG_ERR_CUDA;
  for (;;) {
    EcgDtCtl ctl;
    std::memset(&ctl, 0, sizeof(ctl));
    ctl.device_dt = 1;
    ctl.max_step = max_step;
    ctl.count_degenerate = c->cfg.riemann != ECG_RIEMANN_RUSANOV;
    ctl.reset_slot = -1;
    ctl.cfl = c->cfg.cfl;
    ctl.stop_time = stop_time;
    // capture (or reuse) the chunk graph for this buffer parity and step base
    ecg_ctx::Graph* gr = nullptr;
    for (auto& g : c->graphs) {
      if (g.cur == c->cur && g.max_step == max_step && g.stop_time == stop_time) gr = &g;
    }
    if (!gr) {
      c->graphs.push_back(ecg_ctx::Graph());
      gr = &c->graphs.back();
      gr->cur = c->cur;
      gr->max_step = max_step;
      gr->stop_time = stop_time;
      cudaGraph_t graph;
      if (!cuda_ok(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "capture")) return ECG_ERR_CUDA;
      for (int k = 0; k < K; ++k) {
        const double* in = c->d_state[(c->cur + k) & 1];
        double* o = c->d_state[(c->cur + k + 1) & 1];
        fill_ring(c, in, 0.0, c->d_stats, k);
        EcgDtCtl kc = ctl;
        kc.read_slot = k;
        kc.acc_slot = k + 1;
        c->ops->fv_step(p, in, o, c->d_stats, kc, c->tile_y, c->stream);
      }
      const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
      if (!cuda_ok(c, ce, "end capture")) return ECG_ERR_CUDA;
      const cudaError_t ie = cudaGraphInstantiate(&gr->exec, graph, 0);
      cudaGraphDestroy(graph);
      if (!cuda_ok(c, ie, "instantiate")) return ECG_ERR_CUDA;
    }
    if (!cuda_ok(c, cudaGraphLaunch(gr->exec, c->stream), "graph launch")) return ECG_ERR_CUDA;
    if (!cuda_ok(c, cudaMemcpyAsync(c->h_stats, c->d_stats, sizeof(EcgStepStats) * (K + 1), cudaMemcpyDeviceToHost,
                                    c->stream), "copy stats"))
      return ECG_ERR_CUDA;
    if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "sync")) return ECG_ERR_CUDA;
    int ran = 0;
    for (int k = 0; k < K; ++k) {
      const EcgStepStats& s = c->h_stats[k];
      if (!s.ran) break;
      ++ran;
      out->dt_min = std::min(out->dt_min, s.dt);
      out->dt_max = std::max(out->dt_max, s.dt);
      out->dt_sum += s.dt;
      out->hllc_degenerate_star_count += c->h_stats[k + 1].degenerate;
    }
    steps += ran;
    const EcgStepStats& last = c->h_stats[ran];
    t = last.t;
    c->cur = (c->cur + ran) & 1;
    out->diagnostics.rho_min = okey_to_double(last.rho_min_key);
    out->diagnostics.pressure_min = okey_to_double(last.p_min_key);
    out->diagnostics.nonfinite_count = last.nonfinite;
    if (ran < K) {
      out->failure_code = last.failure;
      out->failed = last.failure != 0;
      break;
    }
    // the next chunk starts from the record of its first state; slots 1..K reset
    if (!cuda_ok(c, cudaMemcpyAsync(c->d_stats, c->d_stats + K, sizeof(EcgStepStats), cudaMemcpyDeviceToDevice,
                                    c->stream), "carry"))
      return ECG_ERR_CUDA;
    if (!cuda_ok(c, c->ops->init_stats(c->d_stats + 1, K, 0.0, c->stream), "init stats")) return ECG_ERR_CUDA;
  }
  // the final diagnostics check of the last step (driver_main.hpp:300-310)
  if (!out->failed) {
    const ecg_diagnostics& d = out->diagnostics;
    if (d.nonfinite_count > 0) out->failure_code = ECG_FAILURE_NONFINITE_STATE;
    else if (d.rho_min <= 0.0) out->failure_code = ECG_FAILURE_NONPOSITIVE_DENSITY;
    else if (d.pressure_min <= 0.0) out->failure_code = ECG_FAILURE_NONPOSITIVE_PRESSURE;
    out->failed = out->failure_code != 0;
  }
  if (!out->failed && steps >= max_step && t < stop_time - 1.0e-14) out->failure_code = ECG_FAILURE_MAX_STEP_BEFORE_STOP_TIME;
  out->steps = steps;
  out->time = t;
  c->invalidate();
  return ECG_OK;
}

ecg_status ecg_run(ecg_ctx* c, int32_t max_step, double stop_time, ecg_run_result* out)
{
  if (!c || !out) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  if (c->slab()) {
    c->err = "a slab needs its halo exchanged every step: step it with ecg_euler_fv_one_step";
    return ECG_ERR_UNSUPPORTED;
  }
  if (c->cfg.method == ECG_METHOD_IMEX) return imex_run(c, max_step, stop_time, out);
  return run_explicit(c, max_step, stop_time, out);
}

// ---- slabs of a grid split along x ------------------------------------------

namespace {
// Edge columns of a slab into the halo layout (4 planes x ny rows x 2):
// lo <- columns 0, 1; hi <- columns nx-2, nx-1.
__global__ void slab_pack_kernel(const double* __restrict__ u, long long pitch, long long plane, int nx, int ny,
                                 double* __restrict__ lo, double* __restrict__ hi)
{
  const long long n = 4LL * ny * 2;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(t & 1);
    const long long fj = t >> 1;  // field * ny + row
    const int f = static_cast<int>(fj / ny), j = static_cast<int>(fj - static_cast<long long>(f) * ny);
    const double* row = u + f * plane + j * pitch;
    if (lo) lo[t] = row[k];
    if (hi) hi[t] = row[nx - 2 + k];
  }
}
}  // namespace

ecg_status ecg_create_slab(ecg_ctx** out, const ecg_run_config* cfg, const ecg_gpu_options* opt, int32_t x0,
                           int32_t x1, int32_t halo_lo, int32_t halo_hi)
{
  if (!out || !cfg) return ECG_ERR_BAD_ARG;
  *out = nullptr;
  const int nx = cfg->n_cell[0];
  if (x0 < 0 || x1 > nx || x1 - x0 < 2 || !(cfg->prob_hi[0] > cfg->prob_lo[0])) return ECG_ERR_BAD_ARG;
  if (halo_lo || halo_hi) {
    if (cfg->method == ECG_METHOD_IMEX) return ECG_ERR_UNSUPPORTED;
    EcgBc bc;
    EcgProblem pr;
    std::memset(&bc, 0, sizeof(bc));
    make_bc(*cfg, false, bc, pr);
    if (bc.ring) return ECG_ERR_UNSUPPORTED;  // exact-state Dirichlet rings cover the whole grid
  }
  // the global cell size (AMReX Geometry: (hi - lo) / n) and the slab's origin
  const double dx = (cfg->prob_hi[0] - cfg->prob_lo[0]) / static_cast<double>(nx);
  ecg_run_config local = *cfg;
  local.n_cell[0] = x1 - x0;
  local.prob_lo[0] = cfg->prob_lo[0] + static_cast<double>(x0) * dx;
  local.prob_hi[0] = cfg->prob_lo[0] + static_cast<double>(x1) * dx;
  const ecg_status st = ecg_create(out, &local, opt);
  if (st != ECG_OK) return st;
  ecg_ctx* c = *out;
  // the problem keeps the whole grid's extent (periodic wraps, exact states);
  // the slab's cells keep the whole grid's dx bit for bit
  c->cfg.prob_lo[0] = cfg->prob_lo[0];
  c->cfg.prob_hi[0] = cfg->prob_hi[0];
  c->grid.dx = dx;
  c->grid.inv_dx = 1.0 / dx;
  c->grid.plo_x = local.prob_lo[0];
  c->halo_lo = halo_lo != 0;
  c->halo_hi = halo_hi != 0;
  c->slab_x0 = x0;
  return ECG_OK;
}

ecg_status ecg_slab_bind_halo(ecg_ctx* c, const double* lo, const double* hi)
{
  if (!c) return ECG_ERR_BAD_ARG;
  if ((c->halo_lo && !lo) || (c->halo_hi && !hi)) return ECG_ERR_BAD_ARG;
  c->d_halo_lo = lo;
  c->d_halo_hi = hi;
  c->invalidate();
  return ECG_OK;
}

ecg_status ecg_slab_pack(ecg_ctx* c, double* lo, double* hi)
{
  if (!c || (!lo && !hi)) return ECG_ERR_BAD_ARG;
  if (!c->uploaded) return ECG_ERR_NOT_READY;
  const long long n = 8LL * c->grid.ny;
  const int blocks = static_cast<int>((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184);
  slab_pack_kernel<<<blocks, 256, 0, c->stream>>>(c->cur_state(), c->grid.pitch, c->grid.plane, c->grid.nx,
                                                  c->grid.ny, lo, hi);
  return cuda_ok(c, cudaGetLastError(), "slab pack") ? ECG_OK : ECG_ERR_CUDA;
}

}  // extern "C"
