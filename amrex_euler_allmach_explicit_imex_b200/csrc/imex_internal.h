// Structures of the IMEX path shared by its translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "ecg_internal.h"

// Index maps and physical-boundary states of the IMEX host grid
// (imex/imex_source_map_helpers.hpp:70-245).
struct EcgImexMap {
  int nx, ny, px, py, bubble;
  int top_wall;     // the Mach 1.22 variant: a reflecting wall above the last row as well
  double gamma;
  double cst[4];    // bubble post-shock conserved state
  double p_fixed;   // bubble fixed post-shock pressure
  // The step's phases are queued without host waits: once a phase has failed
  // (*abort nonzero) the kernels given this map do nothing.  Null: always run.
  const int* abort;
};

// Reductions of the IMEX kernels (min/max as ordered keys, counts, sums).
struct EcgImexStats {
  // star + initialisation
  unsigned long long floor_count;
  unsigned long long k_nonfinite;
  unsigned long long trial_rho_min_key;
  unsigned long long mismatch_before_key;
  unsigned long long mismatch_before_nonfinite;
  // pressure system
  unsigned long long row_nonfinite;
  unsigned long long nnz;
  unsigned long long max_row_width;
  unsigned long long abs_max_key;
  unsigned long long sym_key;
  unsigned long long rhs_linf_key;
  // Picard update
  unsigned long long delta_linf_key;
  unsigned long long pmax_key;
  double delta_l2_sum;
  // closeout
  unsigned long long guard, h_nonfinite, flux_nonfinite, final_nonfinite;
  unsigned long long density_fail, pressure_fail, ie_fail, residual_count;
  unsigned long long flux_linf_key, density_min_key, solved_p_min_key, solved_p_max_key;
  unsigned long long eos_p_min_key, eos_p_max_key, ie_min_key, ie_max_key;
  unsigned long long momentum_corr_key, energy_corr_key, flux_div_key;
  unsigned long long res_linf_key, res_rel_key, mis_linf_key, mis_rel_key;
  double res_sum, mis_sum, energy_sum;
  unsigned long long eq78_count, eq78_key, eq78_scaled_key;
};

// Function table of one arithmetic build of the IMEX stencil kernels.
struct EcgImexOps {
  cudaError_t (*star)(const EcgFvParams& P, const double* u, double dt, double* S, double* p, double* K,
                      EcgImexStats* st, cudaStream_t s);
  cudaError_t (*faces)(const EcgImexMap& m, const double* S, const double* p, const double* K, double* fx, double* fy,
                       unsigned char* fxf, unsigned char* fyf, int mode, cudaStream_t s);
  cudaError_t (*matrix)(const EcgImexMap& m, const double* hx, const double* hy, double dt, double idx, double idy,
                        EcgImexStats* st, cudaStream_t s);
  cudaError_t (*closeout)(const EcgImexMap& m, const EcgGrid& G, const double* S, const double* p, const double* K,
                          const double* fx, const double* fy, const unsigned char* fxf, const unsigned char* fyf,
                          double dt, double* out, EcgImexStats* st, cudaStream_t s);
  cudaError_t (*eq78)(const EcgImexMap& m, const EcgGrid& G, const double* S, const double* K, EcgImexStats* st,
                      cudaStream_t s);
  // faces (mode 0) and rhs in one launch
  cudaError_t (*assemble)(const EcgImexMap& m, const double* S, const double* p, const double* K, double* hx,
                          double* hy, double dt, double idx, double idy, double* rhs, EcgImexStats* st,
                          cudaStream_t s);
  // p_update and momentum in one sweep, K from x; the caller swaps p and x
  cudaError_t (*refresh)(const EcgImexMap& m, const double* p_old, const double* x, const double* S, double dt,
                         double idx, double idy, double* K, EcgImexStats* st, cudaStream_t s);
};

extern const EcgImexOps ecg_imex_exact_ops;
extern const EcgImexOps ecg_imex_fast_ops;

// ---- GMRES (gmres.cu) -------------------------------------------------------------------

// Matrix-free pressure operator of source_map_pressure_row_data
// (imex_source_map_helpers.hpp:533-543) from the face enthalpies.
struct EcgPressureOp {
  int nx, ny, px, py, bubble;
  int drop;          // columns outside a non-periodic axis are not in A (their terms are in the rhs)
  double diag0;      // 1 / (gamma - 1)
  double xc, yc;     // dt^2 / (4 dx^2), dt^2 / (4 dy^2)
  const double* hx;  // (nx+1) x ny
  const double* hy;  // nx x (ny+1)
  const float* hx32; // FP32 copies for the mixed-precision inner solve
  const float* hy32;
};

struct EcgGmresResult {
  int iterations;      // index of the returned iterate
  int converged;
  int breakdown;
  int nonfinite;
  int timeout;         // a bounded grid barrier gave up
  int inner_iterations;
  int refinements;
  int stalled_cycles;  // mixed: cycles after which the DGKS second pass was turned on (0 or 1)
  double residual_linf;
  double relative_residual_linf;
  // true residuals, as pressure_residual computes them: ||A x0 - b||inf and
  // ||b||inf at the start, ||A x - b||inf and ||b||inf of the returned x
  // (NaN when nonfinite; the final pair is NaN after a timeout)
  double initial_linf, b_linf, final_linf, final_b_linf;
  // algorithmic traffic: vector-element accesses per row of the whole solve
  // (one sweep over one vector counts 1), to FP64 vectors and to FP32 basis
  // vectors; bytes = n (8 vec_access64 + 4 vec_access32)
  double vec_access64, vec_access32;
};

struct EcgGmresWork;  // gmres.cu

EcgGmresWork* gmres_work_create(long long n, int max_iter, int num_sms, int device, bool mixed, std::string* err);
void gmres_work_destroy(EcgGmresWork* w);
// whether the solve keeps (the first of) its basis vectors in shared memory
bool gmres_work_resident(const EcgGmresWork* w);
// Solves A x = b from x0 (device vectors of n doubles) with the reference's
// semantics (solve_host_sparse_gmres, imex/imex_pressure_helpers.hpp:92-217).
// mixed: cycles on an FP32-stored Krylov basis, each opened with the true
// FP64 residual.  det: grid sums in a fixed block order, so repeated solves of
// the same system give the same bits.
cudaError_t gmres_solve(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x0, double* x,
                        int max_iter, double tol, bool mixed, int inner_max_iter, double inner_rtol, int max_refine,
                        int reorth, bool det, EcgGmresResult* out, cudaStream_t s);
// gmres_solve without waiting: the result lands in d_res (device memory).
// gate (device int[2], may be null) chains the solve into a sequence of
// launches the host does not wait between: gate[0] nonzero means an earlier
// phase failed, gate[1] that a mixed solve left its system to the FP64
// fallback.  role 1: skipped when gate[0] is set; sets gate[0] when the
// returned iterate fails the acceptance rule (||A x - b||inf <= tol or
// relative to max(||b||inf, 1)), or, for a mixed solve ending finite above
// it, gate[1] instead.  role 2 (the FP64 fallback, from x): runs only when
// gate[1] is set and gate[0] is not; clears gate[1], sets gate[0] on failure.
cudaError_t gmres_enqueue(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x0, double* x,
                          int max_iter, double tol, bool mixed, int inner_max_iter, double inner_rtol, int max_refine,
                          int reorth, bool det, EcgGmresResult* d_res, int* gate, int role, cudaStream_t s);
// r = A x - b: infinity norm, rhs infinity norm (max(|b|inf, 1)) and nonfinite flag.
cudaError_t pressure_residual(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x,
                              double* res_linf, double* rhs_norm, int* nonfinite, cudaStream_t s);
