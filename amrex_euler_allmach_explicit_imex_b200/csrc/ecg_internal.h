// Host/device structures shared by the CUDA translation units of libecg.
// Not part of the public ABI (include/ecg.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Boundary kind of one side of the domain, derived from the reference's
// fill_problem_ghosts policies (problems/boundary_conditions.hpp:2-219).
enum EcgBcKind : int {
  BC_PERIODIC = 0,  // FillBoundary(periodicity): wrap
  BC_CLAMP = 1,     // outflow: nearest valid cell
  BC_REFLECT = 2,   // shock-bubble bottom wall: mirror row, negate my
  BC_CONST = 3,     // shock-bubble inflow: fixed post-shock conserved state
  BC_HALO = 4       // x side of a slab: ghost columns from the neighbour slab (EcgFvParams::halo)
};

struct EcgBc {
  int x_lo, x_hi, y_lo, y_hi;  // EcgBcKind
  int ring;                    // 1: out-of-domain cells come from the ghost ring buffer
  int pad;
  double cst[4];               // BC_CONST conserved state
};

// Geometry and layout of one device state: 4 planes (rho, mx, my, E) of ny
// rows with row pitch `pitch` doubles; plane stride `plane` doubles.
struct EcgGrid {
  int nx, ny;
  long long pitch, plane;
  double dx, dy, inv_dx, inv_dy;
  double plo_x, plo_y;
};

// Exact-state ghost fill selectors (ring mode).
enum EcgRingKind : int { RING_NONE = 0, RING_TORO = 1, RING_GRESHO = 2, RING_QUADRANT = 3, RING_BLOB = 4 };

struct EcgProblem {
  int ring_kind;
  int periodic_x, periodic_y;
  int problem;
  double gamma;
  double toro_l[4], toro_r[4];  // primitive rho,u,v,p
  double interface_x, interface_y;
  double vortex_cx, vortex_cy, density_outer, density_inner, pressure, mach;
  double blob_cx, blob_cy, blob_radius, velocity_x, velocity_y;
  double isentropic_vortex_strength;
  double prob_hi_x, prob_hi_y;
  double post_shock[4];  // primitive post-shock state of ECG_PROBLEM_SHOCK_BUBBLE_MACH122
};

// Mach 1.22 shock / bubble configuration (ECG_PROBLEM_SHOCK_BUBBLE_MACH122).
constexpr double kM122Mach = 1.22;
constexpr double kM122ShockX = 0.5;
constexpr double kM122BubbleX = 1.0, kM122BubbleY = 0.5, kM122BubbleR = 0.25, kM122BubbleRho = 0.138;

// Rankine-Hugoniot state behind a shock of Mach number m running into
// (rho, u, p) = (1, 0, 1) at rest: {rho, u, v, p}.
inline void mach122_post_shock(double gamma, double q[4])
{
  const double m2 = kM122Mach * kM122Mach;
  const double rho2 = (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0);
  const double p2 = 1.0 + 2.0 * gamma * (m2 - 1.0) / (gamma + 1.0);
  const double s = kM122Mach * __builtin_sqrt(gamma);
  q[0] = rho2;
  q[1] = s * (1.0 - 1.0 / rho2);
  q[2] = 0.0;
  q[3] = p2;
}

struct EcgFvParams {
  EcgGrid g;
  EcgBc bc;
  const double* ring;        // ghosted box (nx+4) x (ny+4), 4 planes, when bc.ring
  long long ring_pitch, ring_plane;
  double gamma;
  int order, limiter, riemann;
  int march_rows;            // rows per warp of the column-strip kernel (0: sized to fill one wave)
  int sm_count;              // SMs of the device (0: 148)
  int row_lo, row_hi;        // column-strip kernel: update rows [row_lo, row_hi) only (row_hi 0: all rows)
  int pad;
  // BC_HALO sides: columns -2, -1 (halo_lo) and nx, nx+1 (halo_hi), each
  // block 4 planes of ny rows x 2 columns
  const double* halo_lo;
  const double* halo_hi;
};

// Per-step reduction record.  Keys are order-preserving integer images of
// doubles (okey in ecg_device.cuh) so atomics give exact min/max.
struct EcgStepStats {
  unsigned long long max_rate_key;   // max spectral rate (compute_euler_dt)
  unsigned long long rho_min_key;    // compute_diagnostics rho_min
  unsigned long long p_min_key;      // compute_diagnostics pressure_min
  int nonfinite;
  int degenerate;                    // hllc degenerate-star count of the step that produced this state
  double t;                          // time at the start of the step reading this record
  double dt;                         // dt taken by the step reading this record
  int ran;                           // the step reading this record executed
  int halt;                          // loop stopped before this step
  int failure;                       // ECG_FAILURE_* that stopped the loop
  int step;                          // steps taken before the step reading this record
};

// dt control of one explicit launch.
struct EcgDtCtl {
  int device_dt;      // 0: use dt/time below; 1: compute dt from stats[read_slot] like compute_euler_dt
  int max_step;       // device mode: loop step limit
  int count_degenerate;
  int read_slot;      // device mode: record of the state this launch advances
  int acc_slot;       // record receiving the reductions of the new state
  int reset_slot;     // record this launch re-initialises for the next one (-1: none)
  double dt, time;    // host mode
  double cfl, stop_time;
};

// One solve of a batch (batched.cu).  u[k & 1] holds the state after k
// steps of this solve.
struct EcgBatchSolve {
  EcgFvParams p;         // grid, boundary policy and physics of the solve
  double* u[2];          // state double buffer (pitch p.g.pitch, plane p.g.plane)
  double cfl, stop_time;
  int tile0;             // first tile of this solve in the batch's tile list
  int strip_blocks;      // tiles across x
  int row_blocks;        // tiles along y
  int pad;
};

// Per-launch control of a batched step.
struct EcgBatchCtl {
  int nsolve, ntiles;
  int read_slot, acc_slot, reset_slot;  // rotation over each solve's three records
  int count_degenerate;
};

// Whole-state reductions (one pass).
struct EcgStateStats {
  unsigned long long max_rate_key;        // compute_euler_dt
  unsigned long long diag_rho_min_key;    // compute_diagnostics
  unsigned long long diag_p_min_key;
  unsigned long long material_rate_key;   // compute_imex_dt
  unsigned long long acoustic_rate_key;
  unsigned long long adm_rho_min_key;     // compute_admissibility_diagnostics
  unsigned long long adm_p_min_key;
  unsigned long long adm_ie_min_key;
  int diag_nonfinite;
  int adm_nonfinite, adm_density_fail, adm_pressure_fail, adm_ie_fail;
  int pad[3];
};

// Function table of one arithmetic build of the stencil kernels.
struct EcgStencilOps {
  cudaError_t (*fv_step)(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats,
                         const EcgDtCtl& ctl, int tile_y, cudaStream_t s);
  cudaError_t (*state_reduce)(const EcgFvParams& p, const double* u, int eq79, EcgStateStats* out, cudaStream_t s);
  cudaError_t (*ghost_box)(const EcgFvParams& p, const EcgProblem& pr, const double* u, double time,
                           const EcgStepStats* stats, int k, double* out, long long opitch, long long oplane,
                           int only_ring, cudaStream_t s);
  cudaError_t (*init_stats)(EcgStepStats* stats, int n, double t0, cudaStream_t s);
  cudaError_t (*init_state_stats)(EcgStateStats* st, cudaStream_t s);
  cudaError_t (*seed_stats)(EcgStepStats* stats, const EcgStateStats* st, cudaStream_t s);
  cudaError_t (*init_state)(const EcgFvParams& p, const EcgProblem& pr, double* u, cudaStream_t s);
};

namespace ecg_fast {
// Batched step launcher and tile geometry (fv_batch.cuh, fast build).
cudaError_t launch_batch_step(int riemann, int limiter, int shape, const EcgBatchSolve* solves, EcgStepStats* stats,
                              unsigned long long* degenerate_total, const int* max_step, const EcgBatchCtl& ctl,
                              int grid, cudaStream_t st);
void batch_tiles(int nx, int ny, int shape, int& strip_blocks, int& row_blocks);
int batch_block_threads(int shape);
int batch_blocks_per_sm(int riemann, int limiter, int shape);
cudaError_t launch_batch_rearm(EcgStepStats* stats, int nsolve, int read_slot, cudaStream_t st);
constexpr int kBatchShapes = 3;
}  // namespace ecg_fast

extern const EcgStencilOps ecg_exact_ops;
extern const EcgStencilOps ecg_fast_ops;

#define ECG_MAX_TILE_Y 16
