// Batched independent explicit solves (include/ecg.h, ecg_batch_*).
//
// All solves live in one device arena; every step of the whole batch is one
// launch of the persistent batch kernel (fv_batch.cuh), and runs of steps are
// replayed from CUDA graphs of kChunk launches.  dt is computed per solve on
// the device from that solve's own reductions, so nothing returns to the
// host between steps.  The tile shape (rows per warp, warps per block) is
// chosen by timing every candidate shape on a scratch copy of the batch the
// first time the batch runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"
#include "ecg.h"

namespace ecgi {
void make_bc(const ecg_run_config& c, bool outflow_only, EcgBc& bc, EcgProblem& pr);
double okey_to_double(unsigned long long k);
}

namespace {
constexpr int kChunk = 24;  // launches per graph (a multiple of the 3-record rotation)
}

struct ecg_batch {
  std::string err;
  int device = 0, num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int nsolve = 0;
  int riemann = ECG_RIEMANN_HLLC, limiter = ECG_LIMITER_MINMOD;
  std::vector<ecg_run_config> cfg;
  std::vector<EcgBatchSolve> solves;   // host copy of d_solves
  std::vector<int> steps;              // steps taken per solve (host view after the last run)
  std::vector<char> fresh;             // uploaded since the last run: reductions must be seeded
  double* arena = nullptr;
  size_t arena_doubles = 0;
  EcgBatchSolve* d_solves = nullptr;
  EcgStepStats* d_stats = nullptr;
  EcgStepStats* h_stats = nullptr;     // pinned
  unsigned long long* d_deg = nullptr;
  unsigned long long* h_deg = nullptr; // pinned
  int* d_max_step = nullptr;
  int* h_max_step = nullptr;           // pinned
  EcgStateStats* d_state_stats = nullptr;
  int shape = -1;                      // autotuned tile shape
  int ntiles = 0, grid = 0;
  long long launches = 0;              // launches so far (multiple of 3 between runs)
  cudaGraphExec_t graph = nullptr;

  bool ok(cudaError_t e, const char* what)
  {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  }
  ~ecg_batch()
  {
    if (graph) cudaGraphExecDestroy(graph);
    cudaFree(arena);
    cudaFree(d_solves);
    cudaFree(d_stats);
    cudaFreeHost(h_stats);
    cudaFree(d_deg);
    cudaFreeHost(h_deg);
    cudaFree(d_max_step);
    cudaFreeHost(h_max_step);
    cudaFree(d_state_stats);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

// Tile geometry of every solve for `shape`, written into `sv`; returns the tile count.
int layout_tiles(std::vector<EcgBatchSolve>& sv, int shape)
{
  int t = 0;
  for (auto& s : sv) {
    ecg_fast::batch_tiles(s.p.g.nx, s.p.g.ny, shape, s.strip_blocks, s.row_blocks);
    s.tile0 = t;
    t += s.strip_blocks * s.row_blocks;
  }
  return t;
}

cudaError_t launch_step(ecg_batch* b, const EcgBatchSolve* d_solves, EcgStepStats* stats, unsigned long long* deg,
                        const int* max_step, int shape, int ntiles, int grid, long long k)
{
  EcgBatchCtl ctl;
  ctl.nsolve = b->nsolve;
  ctl.ntiles = ntiles;
  ctl.read_slot = static_cast<int>(k % 3);
  ctl.acc_slot = static_cast<int>((k + 1) % 3);
  ctl.reset_slot = static_cast<int>((k + 2) % 3);
  ctl.count_degenerate = b->riemann != ECG_RIEMANN_RUSANOV;
  return ecg_fast::launch_batch_step(b->riemann, b->limiter, shape, d_solves, stats, deg, max_step, ctl, grid,
                                     b->stream);
}

int grid_for(ecg_batch* b, int shape, int ntiles)
{
  const int per_sm = ecg_fast::batch_blocks_per_sm(b->riemann, b->limiter, shape);
  return std::max(1, std::min(ntiles, per_sm * b->num_sms));
}

// Re-initialises the three records of solve s and seeds record 0 with the
// reductions of its uploaded state (what compute_euler_dt / compute_diagnostics
// see before the first step).
bool seed_solve(ecg_batch* b, int s)
{
  const EcgBatchSolve& S = b->solves[s];
  EcgStepStats* st = b->d_stats + 3 * s;
  return b->ok(ecg_fast_ops.init_stats(st, 3, 0.0, b->stream), "init stats") &&
         b->ok(ecg_fast_ops.init_state_stats(b->d_state_stats, b->stream), "init state stats") &&
         b->ok(ecg_fast_ops.state_reduce(S.p, S.u[0], 0, b->d_state_stats, b->stream), "reduce") &&
         b->ok(ecg_fast_ops.seed_stats(st, b->d_state_stats, b->stream), "seed");
}

// Times every tile shape for a few launches on a scratch copy of the batch
// (states and records), keeps the fastest.
bool autotune(ecg_batch* b)
{
  const size_t abytes = sizeof(double) * b->arena_doubles;
  const size_t sbytes = sizeof(EcgStepStats) * 3 * b->nsolve;
  double* arena = nullptr;
  EcgStepStats* stats = nullptr;
  EcgBatchSolve* d_solves = nullptr;
  unsigned long long* deg = nullptr;  // scratch totals
  int* limit = nullptr;               // scratch step limit: no solve stops on it
  bool good = b->ok(cudaMalloc(&arena, abytes), "autotune alloc") &&
              b->ok(cudaMalloc(&stats, sbytes), "autotune alloc") &&
              b->ok(cudaMalloc(&d_solves, sizeof(EcgBatchSolve) * b->nsolve), "autotune alloc") &&
              b->ok(cudaMalloc(&deg, sizeof(unsigned long long) * b->nsolve), "autotune alloc") &&
              b->ok(cudaMalloc(&limit, sizeof(int)), "autotune alloc");
  good = good && b->ok(cudaMemcpyAsync(arena, b->arena, abytes, cudaMemcpyDeviceToDevice, b->stream), "copy") &&
         b->ok(cudaMemcpyAsync(stats, b->d_stats, sbytes, cudaMemcpyDeviceToDevice, b->stream), "copy") &&
         b->ok(cudaMemsetAsync(deg, 0, sizeof(unsigned long long) * b->nsolve, b->stream), "memset") &&
         b->ok(cudaMemsetAsync(limit, 0x7f, sizeof(int), b->stream), "memset");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  good = good && b->ok(cudaEventCreate(&e0), "event") && b->ok(cudaEventCreate(&e1), "event");
  float best = 1e30f;
  int best_shape = 1;
  long long k = b->launches;
  for (int shape = 0; good && shape < ecg_fast::kBatchShapes; ++shape) {
    std::vector<EcgBatchSolve> sv = b->solves;
    for (auto& s : sv) {
      s.u[0] = arena + (s.u[0] - b->arena);
      s.u[1] = arena + (s.u[1] - b->arena);
    }
    const int nt = layout_tiles(sv, shape);
    const int grid = grid_for(b, shape, nt);
    good = b->ok(cudaMemcpyAsync(d_solves, sv.data(), sizeof(EcgBatchSolve) * b->nsolve, cudaMemcpyHostToDevice,
                                 b->stream),
                 "upload tiles");
    // one warm-up launch, then three timed
    for (int r = 0; good && r < 4; ++r) {
      if (r == 1) good = b->ok(cudaEventRecord(e0, b->stream), "event");
      good = good && b->ok(launch_step(b, d_solves, stats, deg, limit, shape, nt, grid, k++), "batch step");
    }
    good = good && b->ok(cudaEventRecord(e1, b->stream), "event") && b->ok(cudaEventSynchronize(e1), "sync");
    float ms = 0.0f;
    if (good && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best) {
      best = ms;
      best_shape = shape;
    }
  }
  good = good && b->ok(cudaStreamSynchronize(b->stream), "sync");
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(arena);
  cudaFree(stats);
  cudaFree(d_solves);
  cudaFree(deg);
  cudaFree(limit);
  if (!good) return false;
  b->shape = best_shape;
  b->ntiles = layout_tiles(b->solves, b->shape);
  b->grid = grid_for(b, b->shape, b->ntiles);
  return b->ok(cudaMemcpyAsync(b->d_solves, b->solves.data(), sizeof(EcgBatchSolve) * b->nsolve,
                               cudaMemcpyHostToDevice, b->stream),
               "upload tiles");
}

bool capture_graph(ecg_batch* b)
{
  cudaGraph_t g = nullptr;
  if (!b->ok(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return false;
  bool good = true;
  // launches start at a multiple of 3, so relative slots k % 3 are absolute
  for (int k = 0; k < kChunk && good; ++k)
    good = b->ok(launch_step(b, b->d_solves, b->d_stats, b->d_deg, b->d_max_step, b->shape, b->ntiles, b->grid, k),
                 "batch step");
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (!good) {
    if (g) cudaGraphDestroy(g);
    return false;
  }
  if (!b->ok(e, "end capture")) return false;
  const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  return b->ok(ie, "instantiate");
}

ecg_status transfer(ecg_batch* b, int s, double* host, const double* hostc, int32_t lo_x, int32_t lo_y,
                    int64_t jstride, int64_t nstride, bool upload)
{
  if (!b || s < 0 || s >= b->nsolve || (!host && !hostc)) return ECG_ERR_BAD_ARG;
  const EcgBatchSolve& S = b->solves[s];
  const int nx = S.p.g.nx, ny = S.p.g.ny;
  if (lo_x > 0 || lo_y > 0 || jstride < nx - lo_x || nstride < jstride * (ny - lo_y)) return ECG_ERR_BAD_ARG;
  const int64_t off = static_cast<int64_t>(-lo_x) + static_cast<int64_t>(-lo_y) * jstride;
  double* dev = upload ? S.u[0] : S.u[b->steps[s] & 1];
  for (int n = 0; n < 4; ++n) {
    double* d = dev + n * S.p.g.plane;
    cudaError_t e;
    if (upload) {
      e = cudaMemcpy2DAsync(d, sizeof(double) * S.p.g.pitch, hostc + off + n * nstride, sizeof(double) * jstride,
                            sizeof(double) * nx, ny, cudaMemcpyHostToDevice, b->stream);
    } else {
      e = cudaMemcpy2DAsync(host + off + n * nstride, sizeof(double) * jstride, d, sizeof(double) * S.p.g.pitch,
                            sizeof(double) * nx, ny, cudaMemcpyDeviceToHost, b->stream);
    }
    if (!b->ok(e, upload ? "upload" : "download")) return ECG_ERR_CUDA;
  }
  if (upload) {
    b->steps[s] = 0;
    b->fresh[s] = 1;
  }
  return b->ok(cudaStreamSynchronize(b->stream), "sync") ? ECG_OK : ECG_ERR_CUDA;
}

}  // namespace

extern "C" {

ecg_status ecg_batch_create(ecg_batch** out, int32_t nsolve, const ecg_run_config* cfgs, const ecg_gpu_options* opt)
{
  if (!out || !cfgs || nsolve < 1) return ECG_ERR_BAD_ARG;
  *out = nullptr;
  ecg_gpu_options o;
  if (opt) o = *opt;
  else ecg_default_gpu_options(&o);
  // one Riemann solver and limiter per batch (one kernel instantiation);
  // ghost policies without an exact-state ring
  for (int s = 0; s < nsolve; ++s) {
    const ecg_run_config& c = cfgs[s];
    if (c.n_cell[0] < 1 || c.n_cell[1] < 1 || static_cast<long long>(c.n_cell[0]) * c.n_cell[1] > (1LL << 31) ||
        (c.spatial_order != 1 && c.spatial_order != 2) || c.slope_limiter < 0 || c.slope_limiter > 2 ||
        !(c.gamma > 1.0) || !(c.prob_hi[0] > c.prob_lo[0]) || !(c.prob_hi[1] > c.prob_lo[1]))
      return ECG_ERR_BAD_ARG;
    if (c.method != ECG_METHOD_EXPLICIT || c.riemann != cfgs[0].riemann || c.slope_limiter != cfgs[0].slope_limiter ||
        c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL)
      return ECG_ERR_UNSUPPORTED;
    EcgBc bc;
    EcgProblem pr;
    ecgi::make_bc(c, false, bc, pr);
    if (bc.ring) return ECG_ERR_UNSUPPORTED;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) return ECG_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major != 10) return ECG_ERR_NO_DEVICE;
  if (cudaSetDevice(o.device) != cudaSuccess) return ECG_ERR_NO_DEVICE;

  ecg_batch* b = new ecg_batch();
  b->device = o.device;
  b->num_sms = prop.multiProcessorCount;
  b->nsolve = nsolve;
  b->riemann = cfgs[0].riemann;
  b->limiter = cfgs[0].slope_limiter;
  b->cfg.assign(cfgs, cfgs + nsolve);
  b->steps.assign(nsolve, 0);
  b->fresh.assign(nsolve, 1);
  b->solves.resize(nsolve);
  // arena layout: per solve two state buffers, rows padded to 32 doubles
  size_t total = 0;
  std::vector<size_t> offs(nsolve);
  for (int s = 0; s < nsolve; ++s) {
    const int nx = cfgs[s].n_cell[0], ny = cfgs[s].n_cell[1];
    const long long pitch = (nx + 31) / 32 * 32;
    offs[s] = total;
    total += 2 * 4 * static_cast<size_t>(pitch) * ny;
  }
  b->arena_doubles = total;
  bool good = true;
  if (o.stream) {
    b->stream = static_cast<cudaStream_t>(o.stream);
  } else {
    good = b->ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
    b->own_stream = good;
  }
  good = good && b->ok(cudaMalloc(&b->arena, sizeof(double) * total), "alloc arena") &&
         b->ok(cudaMemsetAsync(b->arena, 0, sizeof(double) * total, b->stream), "memset") &&
         b->ok(cudaMalloc(&b->d_solves, sizeof(EcgBatchSolve) * nsolve), "alloc solves") &&
         b->ok(cudaMalloc(&b->d_stats, sizeof(EcgStepStats) * 3 * nsolve), "alloc stats") &&
         b->ok(cudaMallocHost(&b->h_stats, sizeof(EcgStepStats) * 3 * nsolve), "alloc host stats") &&
         b->ok(cudaMalloc(&b->d_deg, sizeof(unsigned long long) * nsolve), "alloc deg") &&
         b->ok(cudaMemsetAsync(b->d_deg, 0, sizeof(unsigned long long) * nsolve, b->stream), "memset") &&
         b->ok(cudaMallocHost(&b->h_deg, sizeof(unsigned long long) * nsolve), "alloc host deg") &&
         b->ok(cudaMalloc(&b->d_max_step, sizeof(int)), "alloc") &&
         b->ok(cudaMallocHost(&b->h_max_step, sizeof(int)), "alloc") &&
         b->ok(cudaMalloc(&b->d_state_stats, sizeof(EcgStateStats)), "alloc");
  if (good) {
    for (int s = 0; s < nsolve; ++s) {
      const ecg_run_config& c = cfgs[s];
      EcgBatchSolve& S = b->solves[s];
      std::memset(&S, 0, sizeof(S));
      EcgProblem pr;
      ecgi::make_bc(c, false, S.p.bc, pr);
      const int nx = c.n_cell[0], ny = c.n_cell[1];
      S.p.g.nx = nx;
      S.p.g.ny = ny;
      S.p.g.pitch = (nx + 31) / 32 * 32;
      S.p.g.plane = S.p.g.pitch * ny;
      // AMReX Geometry cell size (hi - lo) / n and explicit_update.hpp:69-70
      S.p.g.dx = (c.prob_hi[0] - c.prob_lo[0]) / static_cast<double>(nx);
      S.p.g.dy = (c.prob_hi[1] - c.prob_lo[1]) / static_cast<double>(ny);
      S.p.g.inv_dx = 1.0 / S.p.g.dx;
      S.p.g.inv_dy = 1.0 / S.p.g.dy;
      S.p.g.plo_x = c.prob_lo[0];
      S.p.g.plo_y = c.prob_lo[1];
      S.p.gamma = c.gamma;
      S.p.order = c.spatial_order;
      S.p.limiter = c.slope_limiter;
      S.p.riemann = c.riemann;
      S.u[0] = b->arena + offs[s];
      S.u[1] = S.u[0] + 4 * S.p.g.plane;
      S.cfl = c.cfl;
      S.stop_time = c.stop_time;
    }
    b->ntiles = layout_tiles(b->solves, 1);
    good = b->ok(cudaMemcpyAsync(b->d_solves, b->solves.data(), sizeof(EcgBatchSolve) * nsolve,
                                 cudaMemcpyHostToDevice, b->stream),
                 "upload solves") &&
           b->ok(cudaStreamSynchronize(b->stream), "sync");
  }
  if (!good) {
    delete b;
    return ECG_ERR_CUDA;
  }
  *out = b;
  return ECG_OK;
}

void ecg_batch_destroy(ecg_batch* b) { delete b; }

ecg_status ecg_batch_upload(ecg_batch* b, int32_t solve, const double* base, int32_t lo_x, int32_t lo_y,
                            int64_t jstride, int64_t nstride)
{
  return transfer(b, solve, nullptr, base, lo_x, lo_y, jstride, nstride, true);
}

ecg_status ecg_batch_download(ecg_batch* b, int32_t solve, double* base, int32_t lo_x, int32_t lo_y,
                              int64_t jstride, int64_t nstride)
{
  return transfer(b, solve, base, nullptr, lo_x, lo_y, jstride, nstride, false);
}

ecg_status ecg_batch_run(ecg_batch* b, int32_t steps, ecg_batch_result* per_solve)
{
  if (!b || steps < 0) return ECG_ERR_BAD_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return ECG_ERR_NO_DEVICE;
  // Records: launches so far are a multiple of 3, so this run reads slot 0.
  for (int s = 0; s < b->nsolve; ++s) {
    if (b->fresh[s]) {
      if (!seed_solve(b, s)) return ECG_ERR_CUDA;
      if (!b->ok(cudaMemsetAsync(b->d_deg + s, 0, sizeof(unsigned long long), b->stream), "memset")) return ECG_ERR_CUDA;
      b->fresh[s] = 0;
    }
  }
  if (!b->ok(ecg_fast::launch_batch_rearm(b->d_stats, b->nsolve, 0, b->stream), "rearm")) return ECG_ERR_CUDA;
  // step limit of this run: `steps` more than the solve furthest along
  int base = 0;
  for (int s = 0; s < b->nsolve; ++s) base = std::max(base, b->steps[s]);
  *b->h_max_step = base + steps;
  if (!b->ok(cudaMemcpyAsync(b->d_max_step, b->h_max_step, sizeof(int), cudaMemcpyHostToDevice, b->stream), "limit"))
    return ECG_ERR_CUDA;
  if (b->shape < 0) {
    if (!autotune(b)) return ECG_ERR_CUDA;
  }
  if (!b->graph && !capture_graph(b)) return ECG_ERR_CUDA;
  const int chunks = (steps + kChunk - 1) / kChunk;
  for (int c = 0; c < chunks; ++c) {
    if (!b->ok(cudaGraphLaunch(b->graph, b->stream), "graph launch")) return ECG_ERR_CUDA;
  }
  b->launches += static_cast<long long>(chunks) * kChunk;
  if (!b->ok(cudaMemcpyAsync(b->h_stats, b->d_stats, sizeof(EcgStepStats) * 3 * b->nsolve, cudaMemcpyDeviceToHost,
                             b->stream),
             "read stats") ||
      !b->ok(cudaMemcpyAsync(b->h_deg, b->d_deg, sizeof(unsigned long long) * b->nsolve, cudaMemcpyDeviceToHost,
                             b->stream),
             "read deg") ||
      !b->ok(cudaStreamSynchronize(b->stream), "sync"))
    return ECG_ERR_CUDA;
  for (int s = 0; s < b->nsolve; ++s) {
    const EcgStepStats& r = b->h_stats[3 * s];  // read slot of the next launch
    b->steps[s] = r.step;
    if (per_solve) {
      ecg_batch_result& o = per_solve[s];
      std::memset(&o, 0, sizeof(o));
      o.steps = r.step;
      o.failed = r.failure;
      o.hllc_degenerate_star_count = static_cast<int32_t>(b->h_deg[s]);
      o.time = r.t;
      o.diagnostics.rho_min = ecgi::okey_to_double(r.rho_min_key);
      o.diagnostics.pressure_min = ecgi::okey_to_double(r.p_min_key);
      o.diagnostics.nonfinite_count = r.nonfinite;
    }
  }
  return ECG_OK;
}

const char* ecg_batch_last_error(const ecg_batch* b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
