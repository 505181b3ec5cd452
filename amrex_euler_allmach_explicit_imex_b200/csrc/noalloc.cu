// ecg_euler_fv_one_step_noalloc: one explicit step on caller-owned device
// memory that allocates nothing (include/ecg.h).
//
// Who needs it: a GPU build of the AMReX driver owns device memory through
// its arena, which reserves most of HBM when AMReX starts, and keeps its
// per-step work asynchronous on its own stream.  A plugin step that calls
// cudaMalloc/cudaFree there may fail for want of memory the arena holds, and
// cudaFree synchronises the whole device in the middle of the caller's
// pipeline.  This entry point therefore takes the state as the caller's own
// device arrays and keeps its scratch in a fixed, module-scope device array.
//
// Scratch (ECG_NOALLOC_SCRATCH_BYTES, 8 MiB):
//   [0, 256)   the EcgStepStats record the step kernel reduces into
//              (re-initialised by a kernel before every step);
//   [256, ...) the exact-state ghost ring, 4 planes of (nx+4)(ny+4) doubles,
//              for the exact-Dirichlet policies only (Toro, Gresho,
//              quadrant, blob); other policies need no ring and no limit.
// Ring problems whose ring does not fit are rejected with ECG_ERR_BAD_ARG and
// a message.  Every call on one device shares the one scratch array, so calls
// that overlap in time (other streams or host threads) race and corrupt each
// other's statistics and ring.
//
// The first call on each device looks up the array's address with
// cudaGetSymbolAddress (with that device current), reads the device's SM count
// and checks that the device is a compute-capability 10 part; the first call
// should therefore come before any stream capture.  The address is kept until
// the process exits: a cudaDeviceReset (or any teardown of the device's primary
// context) leaves it pointing into a context that no longer exists, so callers
// that reset a device must not call this entry point on it afterwards.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ctx.h"
#include "ecg.h"

namespace ecgi {
void make_bc(const ecg_run_config& c, bool outflow_only, EcgBc& bc, EcgProblem& pr);
}

namespace {

constexpr size_t kScratchBytes = ECG_NOALLOC_SCRATCH_BYTES;
constexpr size_t kRingOffset = 256;
static_assert(sizeof(EcgStepStats) <= kRingOffset, "stats record must fit before the ring");

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};  // SM count of each device, read with its address

void set_err(char* err, int32_t len, const char* msg)
{
  if (!err || len <= 0) return;
  std::snprintf(err, static_cast<size_t>(len), "%s", msg);
}

// Address of g_scratch on `dev` (current) and the device's SM count; looked
// up once per device.
ecg_status scratch_on(int dev, unsigned char** out, int* sms, char* err, int32_t len)
{
  if (dev < 0 || dev >= kMaxDevices) {
    set_err(err, len, "device ordinal out of range");
    return ECG_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10) {
      set_err(err, len, "device is not a compute-capability 10 (B200-class) GPU");
      return ECG_ERR_NO_DEVICE;
    }
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) {
      set_err(err, len, "device SM count unavailable");
      return ECG_ERR_CUDA;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      char msg[256];
      std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
      set_err(err, len, msg);
      return ECG_ERR_CUDA;
    }
    g_addr[dev] = static_cast<unsigned char*>(p);
    g_sms[dev] = nsm;
  }
  *out = g_addr[dev];
  *sms = g_sms[dev];
  return ECG_OK;
}

// Restores the caller's current device on every exit path.
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  cudaError_t enter(int dev)
  {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    if (prev == dev) return cudaSuccess;
    e = cudaSetDevice(dev);
    switched = e == cudaSuccess;
    return e;
  }
  ~DeviceGuard()
  {
    if (switched) cudaSetDevice(prev);
  }
};

ecg_status fail(char* err, int32_t len, ecg_status st, const char* what, cudaError_t e)
{
  char msg[256];
  std::snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  set_err(err, len, msg);
  return st;
}

}  // namespace

ecg_status ecg_euler_fv_one_step_noalloc(const ecg_run_config* cfg, const ecg_gpu_options* opt,
                                         const double* state_in, double* state_out, int32_t lo_x, int32_t lo_y,
                                         int64_t jstride, int64_t nstride, double dt, double time,
                                         int32_t* hllc_degenerate_count, char* err, int32_t err_len)
{
  if (!cfg || !state_in || !state_out || state_in == state_out) {
    set_err(err, err_len, "null configuration or state, or state_in == state_out");
    return ECG_ERR_BAD_ARG;
  }
  const int nx = cfg->n_cell[0], ny = cfg->n_cell[1];
  // same validation as ecg_create
  if (nx < 1 || ny < 1 || static_cast<long long>(nx) * ny > (1LL << 31) ||
      (cfg->spatial_order != 1 && cfg->spatial_order != 2) || cfg->riemann < 0 || cfg->riemann > 3 ||
      cfg->slope_limiter < 0 || cfg->slope_limiter > 2 || !(cfg->gamma > 1.0) ||
      !(cfg->prob_hi[0] > cfg->prob_lo[0]) || !(cfg->prob_hi[1] > cfg->prob_lo[1])) {
    set_err(err, err_len, "invalid run configuration");
    return ECG_ERR_BAD_ARG;
  }
  if (cfg->problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL) {
    set_err(err, err_len, "cylindrical bubble is not supported");
    return ECG_ERR_UNSUPPORTED;
  }
  // Array4 layout shared by state_in and state_out, as in ecg_upload_state_device
  if (lo_x > 0 || lo_y > 0 || jstride < nx - lo_x || nstride < jstride * (ny - lo_y)) {
    set_err(err, err_len, "layout does not cover [0, nx) x [0, ny)");
    return ECG_ERR_BAD_ARG;
  }
  ecg_gpu_options o;
  if (opt) o = *opt;
  else ecg_default_gpu_options(&o);

  EcgFvParams p;
  std::memset(&p, 0, sizeof(p));
  EcgProblem pr;
  ecgi::make_bc(*cfg, false, p.bc, pr);
  const size_t ring_bytes = sizeof(double) * 4 * static_cast<size_t>(nx + 4) * static_cast<size_t>(ny + 4);
  if (p.bc.ring && ring_bytes > kScratchBytes - kRingOffset) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "exact-Dirichlet ghost ring of %zu bytes for %d x %d cells exceeds the %zu-byte static scratch "
                  "((nx+4)*(ny+4) must be <= %zu)",
                  ring_bytes, nx, ny, kScratchBytes - kRingOffset, (kScratchBytes - kRingOffset) / 32);
    set_err(err, err_len, msg);
    return ECG_ERR_BAD_ARG;
  }

  // The step reads neighbour cells of state_in while it writes state_out, so
  // the two arrays (4 planes of nstride doubles from their Array4 bases) must
  // not share a byte.
  {
    const auto a0 = reinterpret_cast<uintptr_t>(state_in), b0 = reinterpret_cast<uintptr_t>(state_out);
    const uintptr_t len = sizeof(double) * 4 * static_cast<uintptr_t>(nstride);
    if (a0 < b0 + len && b0 < a0 + len) {
      set_err(err, err_len, "state_in and state_out overlap");
      return ECG_ERR_BAD_ARG;
    }
  }
  DeviceGuard guard;
  cudaError_t e = guard.enter(o.device);
  if (e != cudaSuccess) return fail(err, err_len, ECG_ERR_NO_DEVICE, "select device", e);
  unsigned char* scratch = nullptr;
  int sms = 0;
  const ecg_status st = scratch_on(o.device, &scratch, &sms, err, err_len);
  if (st != ECG_OK) return st;

  const EcgStencilOps* ops = o.arith == ECG_ARITH_EXACT ? &ecg_exact_ops : &ecg_fast_ops;
  const int tile_y = (o.tile_y == 1 || o.tile_y == 2 || o.tile_y == 3 || o.tile_y == 8 || o.tile_y == 16) ? o.tile_y : 0;
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);

  // grid of ecg_create with the caller's strides
  p.g.nx = nx;
  p.g.ny = ny;
  p.g.pitch = jstride;
  p.g.plane = nstride;
  p.g.dx = (cfg->prob_hi[0] - cfg->prob_lo[0]) / static_cast<double>(nx);
  p.g.dy = (cfg->prob_hi[1] - cfg->prob_lo[1]) / static_cast<double>(ny);
  p.g.inv_dx = 1.0 / p.g.dx;
  p.g.inv_dy = 1.0 / p.g.dy;
  p.g.plo_x = cfg->prob_lo[0];
  p.g.plo_y = cfg->prob_lo[1];
  p.gamma = cfg->gamma;
  p.order = cfg->spatial_order;
  p.limiter = cfg->slope_limiter;
  p.riemann = cfg->riemann;
  p.march_rows = o.tile_x;
  p.sm_count = sms;
  const int64_t off = static_cast<int64_t>(-lo_x) + static_cast<int64_t>(-lo_y) * jstride;
  const double* u = state_in + off;
  double* v = state_out + off;

  EcgStepStats* stats = reinterpret_cast<EcgStepStats*>(scratch);
  if (p.bc.ring) {
    double* ring = reinterpret_cast<double*>(scratch + kRingOffset);
    p.ring = ring;
    p.ring_pitch = nx + 4;
    p.ring_plane = static_cast<long long>(nx + 4) * (ny + 4);
    e = ops->ghost_box(p, pr, u, time, nullptr, 0, ring, p.ring_pitch, p.ring_plane, 1, s);
    if (e != cudaSuccess) return fail(err, err_len, ECG_ERR_CUDA, "ghost ring", e);
  }
  // the reduction record starts at its identity values
  e = ops->init_stats(stats, 1, time, s);
  if (e != cudaSuccess) return fail(err, err_len, ECG_ERR_CUDA, "init stats", e);
  EcgDtCtl ctl;
  std::memset(&ctl, 0, sizeof(ctl));
  ctl.device_dt = 0;
  ctl.dt = dt;
  ctl.time = time;
  ctl.count_degenerate = cfg->riemann != ECG_RIEMANN_RUSANOV;
  ctl.read_slot = 0;
  ctl.acc_slot = 0;
  ctl.reset_slot = -1;
  e = ops->fv_step(p, u, v, stats, ctl, tile_y, s);
  if (e != cudaSuccess) return fail(err, err_len, ECG_ERR_CUDA, "fv_step", e);
  if (hllc_degenerate_count) {
    EcgStepStats h;
    e = cudaMemcpyAsync(&h, stats, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(err, err_len, ECG_ERR_CUDA, "read stats", e);
    *hllc_degenerate_count = h.degenerate;
  }
  return ECG_OK;
}
