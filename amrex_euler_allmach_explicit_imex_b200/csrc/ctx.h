// The context behind the opaque ecg_ctx handle of include/ecg.h.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ecg.h"
#include "ecg_internal.h"

struct EcgImexState;  // imex.cu
struct EcgOutput;     // output.cu
struct HostStage;     // hoststage.cu

struct ecg_ctx {
  static constexpr int kChunk = 32;  // explicit steps per captured graph

  ecg_run_config cfg{};
  ecg_gpu_options opt{};
  int device = -1;
  int num_sms = 0;
  const EcgStencilOps* ops = nullptr;
  EcgGrid grid{};
  int tile_y = 16;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // pipelined host step (ecg_euler_fv_one_step_host): copy streams and one
  // event per band for the upload and for the step
  cudaStream_t up_stream = nullptr, down_stream = nullptr;
  std::vector<cudaEvent_t> band_up, band_done, band_dl;
  // pageable host boxes: pinned staging copies of the state and the host
  // threads that fill and drain them (hoststage.cu), made on first use
  HostStage* stage = nullptr;

  double* d_state[2] = {nullptr, nullptr};  // double buffer, 4 planes each
  int cur = 0;
  bool uploaded = false;
  double* d_ring = nullptr;                 // ghosted box for exact-state Dirichlet fills

  EcgStepStats* d_stats = nullptr;
  EcgStepStats* h_stats = nullptr;          // pinned
  int stats_cap = 0;
  EcgStateStats* d_state_stats = nullptr;
  EcgStateStats* h_state_stats = nullptr;   // pinned
  bool state_stats_valid = false;

  // compute_euler_dt / compute_diagnostics of the current state, reduced by
  // the fused epilogue of the last explicit step
  bool fused_valid = false;    // fused_* hold the reductions of the current state
  bool fused_pending = false;  // they are still in d_stats[1] on the device
  double fused_max_rate = 0.0, fused_rho_min = 0.0, fused_p_min = 0.0;
  int fused_nonfinite = 0, fused_degenerate = 0;
  int fused_slot = 1;
  // host-dt launches: rotating stats records (see ecg_euler_fv_one_step)
  bool host_slots_ready = false;
  long long host_step = 0;

  struct Graph {
    int cur = 0;
    int max_step = 0;
    double stop_time = 0.0;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<Graph> graphs;

  // slab of a grid split along x (ecg_create_slab): x sides whose ghost
  // columns come from the neighbour slabs, and the caller's halo blocks
  bool halo_lo = false, halo_hi = false;
  int slab_x0 = 0;
  const double* d_halo_lo = nullptr;
  const double* d_halo_hi = nullptr;
  bool slab() const { return halo_lo || halo_hi; }
  EcgImexState* imex = nullptr;
  EcgOutput* out = nullptr;  // output writers' buffers (output.cu)
  // adjoint workspace (adjoint.cu): primitive gradients, one stats record
  double* adj_gq = nullptr;
  EcgStepStats* adj_stats = nullptr;
  std::string err;

  const double* cur_state() const { return d_state[cur]; }
  double* cur_state_mut() { return d_state[cur]; }
  double* next_state() { return d_state[cur ^ 1]; }
  void invalidate()
  {
    fused_valid = false;
    fused_pending = false;
    state_stats_valid = false;
  }
  ~ecg_ctx();
};

namespace ecgi {
bool cuda_ok(ecg_ctx* c, cudaError_t e, const char* what);
double okey_to_double(unsigned long long k);
EcgFvParams fv_params(ecg_ctx* c, bool imex_policy);
EcgProblem problem_of(ecg_ctx* c, bool imex_policy);
bool is_bubble(const ecg_run_config& c);
bool reduce_state(ecg_ctx* c);
bool fetch_fused(ecg_ctx* c);
}  // namespace ecgi

// hoststage.cu: copies between pageable host boxes and the device through
// the context's pinned staging buffers
bool host_pageable(const void* p);
HostStage* host_stage(ecg_ctx* c);  // null when the pinned buffers cannot be allocated (c->err set)
void host_stage_destroy(HostStage* s);
double* host_stage_in(HostStage* s);
double* host_stage_out(HostStage* s);
// rows [r0, r1) of the 4 planes between the caller's box (offset to cell (0, 0))
// and the compact stage, on the staging threads
void host_stage_copy(HostStage* s, double* stage, double* host, int64_t jstride, int64_t nstride, int nx, int ny,
                     int r0, int r1, bool to_stage);

// imex.cu
void imex_free(ecg_ctx* c);
// output.cu
void output_destroy(EcgOutput* o);
ecg_status imex_run(ecg_ctx* c, int32_t max_step, double stop_time, ecg_run_result* out);
