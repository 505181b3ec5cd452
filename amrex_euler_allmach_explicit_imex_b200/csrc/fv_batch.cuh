// Batched explicit step: many independent solves of uneven grid sizes
// advanced by one persistent launch per step.  Included inside the ecg_fast
// namespace of stencil.cuh after fv_march.cuh (it reuses march_strip_staged:
// the rows of each warp strip come through the warp's shared-memory ring, as
// in the single-grid default; 20.3 against 17.4 G cell-updates/s with the
// rows in registers on the 64-solve bench batch).
//
// The solves' work is cut into tiles of WPB warp strips x H rows; tile
// indices run over all solves (EcgBatchSolve::tile0 is the prefix sum).  A
// grid of resident blocks walks the tile list.  Every solve keeps three
// rotating EcgStepStats records, like the single-solve device loop: launch k
// reads record k%3 (the reductions of the solve's current state), reduces
// the new state into (k+1)%3 and re-initialises (k+2)%3.  The state buffer a
// solve reads is chosen by the parity of its own step count, so solves that
// stop early keep their final state where the host expects it.
namespace batch {

// dt of solve `S` for this launch from its read record: the driver loop's
// checks and compute_euler_dt (driver_main.hpp:224-247).  On a stop the
// leading block copies the whole read record (reductions included) into the
// acc record so the record chain keeps describing the final state.
__device__ __forceinline__ bool solve_control(EcgStepStats* __restrict__ st, const EcgBatchSolve& S,
                                              const EcgBatchCtl& ctl, int max_step, bool lead, double& dt)
{
  const EcgStepStats& r = st[ctl.read_slot];
  if (lead) reset_record(st[ctl.reset_slot]);
  const double t = r.t;
  int failure = r.halt ? r.failure : 0;
  bool halt = r.halt != 0;
  if (!halt) {
    if (r.nonfinite > 0) failure = ECG_FAILURE_NONFINITE_STATE;
    else if (okey_inv(r.rho_min_key) <= 0.0) failure = ECG_FAILURE_NONPOSITIVE_DENSITY;
    else if (okey_inv(r.p_min_key) <= 0.0) failure = ECG_FAILURE_NONPOSITIVE_PRESSURE;
    halt = failure != 0 || r.step >= max_step || !(t < S.stop_time - 1.0e-14);
  }
  dt = 0.0;
  if (!halt) {
    dt = euler_dt_from_rate(okey_inv(r.max_rate_key), S.cfl, S.stop_time, t);
    if (!isfinite(dt) || dt <= 0.0) {
      halt = true;
      failure = ECG_FAILURE_INVALID_TIME_STEP;
    }
  }
  if (lead) {
    EcgStepStats& a = st[ctl.acc_slot];
    if (halt) {
      a = r;
      a.halt = 1;
      a.failure = failure;
      a.ran = 0;
      a.dt = 0.0;
    } else {
      st[ctl.read_slot].dt = dt;
      st[ctl.read_slot].ran = 1;
      a.t = t + dt;
      a.step = r.step + 1;
    }
  }
  return !halt;
}

template <int RK, int LIM, int H, int WPB>
__global__ void __launch_bounds__(WPB * 32, 12 / WPB)
fv_batch_kernel(const EcgBatchSolve* __restrict__ solves, EcgStepStats* __restrict__ stats,
                unsigned long long* __restrict__ degenerate_total, const int* __restrict__ max_step,
                const EcgBatchCtl ctl)
{
  __shared__ BlockRed<WPB * 32> red;
  __shared__ march::StageRing ring[WPB];
  __shared__ EcgBatchSolve S;
  __shared__ double s_dt;
  __shared__ int s_go;
  const int warp = threadIdx.x >> 5;
  const int limit = *max_step;
  int s = 0;
  for (int tile = blockIdx.x; tile < ctl.ntiles; tile += gridDim.x) {
    // solve of this tile (tiles are ordered by solve; blocks move forward)
    while (s + 1 < ctl.nsolve && solves[s + 1].tile0 <= tile) ++s;
    __syncthreads();  // previous tile done with the shared copies
    if (threadIdx.x == 0) {
      S = solves[s];
      const bool lead = tile == S.tile0;
      double dt;
      s_go = solve_control(stats + 3 * s, S, ctl, limit, lead, dt) ? 1 : 0;
      s_dt = dt;
    }
    __syncthreads();
    if (!s_go) continue;
    const int local = tile - S.tile0;
    const int sblk = local % S.strip_blocks, rblk = local / S.strip_blocks;
    const int strip = sblk * WPB + warp;
    const int c0 = strip * march::kCells, j0 = rblk * H;
    const EcgStepStats& r = stats[3 * s + ctl.read_slot];
    const int par = r.step & 1;
    march::MarchAcc acc;
    acc.init();
    if (c0 < S.p.g.nx)
      march::march_strip_staged<RK, LIM, true>(S.p, S.u[par], S.u[par ^ 1], c0, j0, H, s_dt,
                                               ctl.count_degenerate != 0, acc, ring[warp]);
    const int deg = block_commit<WPB * 32>(red, acc.kmax, acc.krho, acc.kp, acc.nonfinite, acc.degenerate,
                                           &stats[3 * s + ctl.acc_slot]);
    if (threadIdx.x == 0 && deg != 0) atomicAdd(&degenerate_total[s], static_cast<unsigned long long>(deg));
  }
}

// Clears the stop of solves that stopped only at the previous run's step
// limit, so the next run continues them; failures and stop_time stay.
__global__ void batch_rearm_kernel(EcgStepStats* stats, int nsolve, int read_slot)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsolve) return;
  EcgStepStats& r = stats[3 * s + read_slot];
  if (r.halt && r.failure == 0) r.halt = 0;
}

// Shapes the autotuner picks from: (rows per warp, warps per block).
constexpr int kShapes = 3;
__host__ __device__ constexpr int shape_h(int k) { return k == 0 ? 16 : 32; }
__host__ __device__ constexpr int shape_wpb(int k) { return k == 2 ? 2 : 4; }

template <int RK, int LIM, int K>
cudaError_t launch_shape(const EcgBatchSolve* solves, EcgStepStats* stats, unsigned long long* deg, const int* max_step,
                         const EcgBatchCtl& ctl, int grid, cudaStream_t st)
{
  constexpr int H = shape_h(K), WPB = shape_wpb(K);
  fv_batch_kernel<RK, LIM, H, WPB><<<grid, WPB * 32, 0, st>>>(solves, stats, deg, max_step, ctl);
  return cudaGetLastError();
}

template <int RK, int LIM, int K>
int occupancy_shape()
{
  constexpr int H = shape_h(K), WPB = shape_wpb(K);
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fv_batch_kernel<RK, LIM, H, WPB>, WPB * 32, 0) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

template <int RK, int LIM>
int occupancy_lim(int shape)
{
  return shape == 0 ? occupancy_shape<RK, LIM, 0>() : (shape == 2 ? occupancy_shape<RK, LIM, 2>()
                                                                  : occupancy_shape<RK, LIM, 1>());
}

template <int RK>
int occupancy_rk(int limiter, int shape)
{
  return limiter == ECG_LIMITER_MC        ? occupancy_lim<RK, ECG_LIMITER_MC>(shape)
         : limiter == ECG_LIMITER_VANLEER ? occupancy_lim<RK, ECG_LIMITER_VANLEER>(shape)
                                          : occupancy_lim<RK, ECG_LIMITER_MINMOD>(shape);
}

template <int RK, int LIM>
cudaError_t launch_lim(int shape, const EcgBatchSolve* solves, EcgStepStats* stats, unsigned long long* deg,
                       const int* max_step, const EcgBatchCtl& ctl, int grid, cudaStream_t st)
{
  switch (shape) {
    case 0: return launch_shape<RK, LIM, 0>(solves, stats, deg, max_step, ctl, grid, st);
    case 2: return launch_shape<RK, LIM, 2>(solves, stats, deg, max_step, ctl, grid, st);
    default: return launch_shape<RK, LIM, 1>(solves, stats, deg, max_step, ctl, grid, st);
  }
}

template <int RK>
cudaError_t launch_rk(int limiter, int shape, const EcgBatchSolve* solves, EcgStepStats* stats,
                      unsigned long long* deg, const int* max_step, const EcgBatchCtl& ctl, int grid, cudaStream_t st)
{
  switch (limiter) {
    case ECG_LIMITER_MC: return launch_lim<RK, ECG_LIMITER_MC>(shape, solves, stats, deg, max_step, ctl, grid, st);
    case ECG_LIMITER_VANLEER:
      return launch_lim<RK, ECG_LIMITER_VANLEER>(shape, solves, stats, deg, max_step, ctl, grid, st);
    default: return launch_lim<RK, ECG_LIMITER_MINMOD>(shape, solves, stats, deg, max_step, ctl, grid, st);
  }
}

}  // namespace batch

// Tile geometry of one solve for autotuner shape `shape`.
void batch_tiles(int nx, int ny, int shape, int& strip_blocks, int& row_blocks)
{
  const int strips = (nx + march::kCells - 1) / march::kCells;
  const int wpb = batch::shape_wpb(shape), h = batch::shape_h(shape);
  strip_blocks = (strips + wpb - 1) / wpb;
  row_blocks = (ny + h - 1) / h;
}

int batch_block_threads(int shape) { return batch::shape_wpb(shape) * 32; }

cudaError_t launch_batch_step(int riemann, int limiter, int shape, const EcgBatchSolve* solves, EcgStepStats* stats,
                              unsigned long long* degenerate_total, const int* max_step, const EcgBatchCtl& ctl,
                              int grid, cudaStream_t st)
{
  switch (riemann) {
    case ECG_RIEMANN_RUSANOV:
      return batch::launch_rk<ECG_RIEMANN_RUSANOV>(limiter, shape, solves, stats, degenerate_total, max_step, ctl,
                                                   grid, st);
    case ECG_RIEMANN_LOWMACH_HLLC:
      return batch::launch_rk<ECG_RIEMANN_LOWMACH_HLLC>(limiter, shape, solves, stats, degenerate_total, max_step,
                                                        ctl, grid, st);
    case ECG_RIEMANN_XIE_AM_HLLC_P:
      // the staged strip body carries the 5-face sensor along
      return batch::launch_rk<ECG_RIEMANN_XIE_AM_HLLC_P>(limiter, shape, solves, stats, degenerate_total, max_step,
                                                         ctl, grid, st);
    default:
      return batch::launch_rk<ECG_RIEMANN_HLLC>(limiter, shape, solves, stats, degenerate_total, max_step, ctl, grid,
                                                st);
  }
}

int batch_blocks_per_sm(int riemann, int limiter, int shape)
{
  switch (riemann) {
    case ECG_RIEMANN_RUSANOV: return batch::occupancy_rk<ECG_RIEMANN_RUSANOV>(limiter, shape);
    case ECG_RIEMANN_LOWMACH_HLLC: return batch::occupancy_rk<ECG_RIEMANN_LOWMACH_HLLC>(limiter, shape);
    case ECG_RIEMANN_XIE_AM_HLLC_P: return batch::occupancy_rk<ECG_RIEMANN_XIE_AM_HLLC_P>(limiter, shape);
    default: return batch::occupancy_rk<ECG_RIEMANN_HLLC>(limiter, shape);
  }
}

cudaError_t launch_batch_rearm(EcgStepStats* stats, int nsolve, int read_slot, cudaStream_t st)
{
  batch::batch_rearm_kernel<<<(nsolve + 127) / 128, 128, 0, st>>>(stats, nsolve, read_slot);
  return cudaGetLastError();
}
