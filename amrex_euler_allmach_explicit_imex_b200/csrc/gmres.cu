// GMRES pressure solve of the IMEX step: one persistent cooperative launch
// per solve, matrix-free operator, deterministic grid reductions.
//
// Reference semantics (solve_host_sparse_gmres, imex/imex_pressure_helpers.hpp:92-217):
// unrestarted GMRES from x0 with iterations_limit = min(max_iter, n); the
// infinity norm of the true residual of every iterate decides convergence
// (||r||inf <= tol or ||r||inf / max(||b||inf, 1) <= tol); the best iterate
// (smallest ||r||inf) is returned when the limit is reached; breakdown when
// h_{j+1,j} <= 100 eps max(beta, 1).
//
// B200 formulation of the same algorithm:
//  * the Hessenberg least-squares problem is reduced with Givens rotations
//    (the reference re-solves it by QR every iteration; same y in exact
//    arithmetic);
//  * the residual vector of every iterate is carried by the recurrence
//      r_j = s_j^2 r_{j-1} - s_j c_j g_j v_{j+1}
//    (r_j = g_{j+1} Q_j^T e_{j+1} in the Krylov basis), so its infinity norm
//    costs one fused pass instead of forming x_j and an extra SpMV;
//  * orthogonalisation is classical Gram-Schmidt with the DGKS test (a second
//    pass only when ||w'|| < ||w|| / sqrt(2)), with all dot products of a pass
//    fused into one sweep and one grid reduction;
//  * the iterate is formed once, at the end.
// Mixed precision: FP32 basis, FP32 operator, FP64-accumulated dot products
// inside FP64 iterative refinement on the true FP64 residual; the stopping
// test stays the reference's on the FP64 residual.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "ecg.h"
#include "imex_internal.h"

namespace {

// 512 threads per block (one block per SM): 16 warps in flight for the
// latency-bound dot products and basis updates, within 128 registers a thread.
constexpr int NT = 512;
constexpr int kResidualBlocks = 148 * 2;  // grid of residual_kernel
constexpr double kEps = 2.220446049250313e-16;

struct GridBar {
  unsigned int arrive;
  unsigned int gen;
  int timeout;
  int pad;
};

struct GmresArgs {
  EcgPressureOp op;
  long long n;
  const double* b;
  const double* x0;
  double* x;
  double* V;     // (m+1) x n
  double* w;     // n
  double* r;     // n
  float* V32;    // (m+1) x n (mixed)
  float* w32;
  float* r32;    // inner right-hand side
  double* part;  // nblocks x ld
  double* red;   // ld reduced values
  double* R;     // column-major (m+1) x m
  double* yv;    // m
  GridBar* bar;
  EcgGmresResult* res;
  int ld;
  int m;          // basis capacity
  int max_iter;
  double tol;
  int mixed;
  int inner_max;
  double inner_rtol;
  int max_refine;
  long long spin_limit;
};

__device__ __forceinline__ unsigned int ld_volatile(const unsigned int* p) { return *reinterpret_cast<const volatile unsigned int*>(p); }
__device__ __forceinline__ int ld_volatile_i(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Grid-wide barrier over co-resident blocks (cooperative launch), with a
// bounded spin: a block that waits longer than spin_limit polls sets the
// timeout flag and leaves; every block then exits at its next check.
__device__ __forceinline__ bool grid_sync(GridBar* bar, unsigned int& gen, long long spin_limit)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int g = gen;
    __threadfence();
    const unsigned int t = atomicAdd(&bar->arrive, 1u);
    if (t == gridDim.x - 1) {
      atomicExch(&bar->arrive, 0u);
      __threadfence();
      atomicExch(&bar->gen, g + 1u);
    } else {
      long long spins = 0;
      while (ld_volatile(&bar->gen) == g) {
        if (++spins > spin_limit) {
          atomicExch(&bar->timeout, 1);
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
  }
  ++gen;
  __syncthreads();
  return ld_volatile_i(&bar->timeout) == 0;
}

__device__ __forceinline__ int wrapi(int i, int n)
{
  int r = i % n;
  return r < 0 ? r + n : r;
}
// source_map_index: wrap or even reflection (imex_source_map_helpers.hpp:169-188)
__device__ __forceinline__ int pmap(int k, int n, int per)
{
  if (per) return wrapi(k, n);
  if (k < 0) {
    const int r = -k - 1;
    return r < n - 1 ? r : n - 1;
  }
  if (k >= n) {
    const int r = n - (k - n + 1);
    return r > 0 ? r : 0;
  }
  return k;
}

// Row r of A v with A the source-map pressure operator
// (imex_source_map_helpers.hpp:533-543); columns at a fixed Dirichlet
// pressure are not part of A (their terms are in the right-hand side): the
// bubble's left boundary, and with op.drop every column outside a
// non-periodic axis (the direct T1/S2 driver, imex_bdltv20_direct_driver.hpp:455-466).
template <typename T>
__device__ __forceinline__ T apply_row(const EcgPressureOp& op, const T* __restrict__ v, int i, int j, long long r)
{
  const int nx = op.nx, ny = op.ny;
  const T he = static_cast<T>(op.hx[static_cast<long long>(j) * (nx + 1) + i + 1]);
  const T hw = static_cast<T>(op.hx[static_cast<long long>(j) * (nx + 1) + i]);
  const T hn = static_cast<T>(op.hy[static_cast<long long>(j + 1) * nx + i]);
  const T hs = static_cast<T>(op.hy[static_cast<long long>(j) * nx + i]);
  const T xc = static_cast<T>(op.xc), yc = static_cast<T>(op.yc);
  const long long row = static_cast<long long>(j) * nx;
  T acc = (static_cast<T>(op.diag0) + xc * (he + hw) + yc * (hn + hs)) * __ldcg(v + r);
  const bool fix = op.bubble && !op.px;
  const bool dropx = op.drop && !op.px, dropy = op.drop && !op.py;
  auto vx = [&](int ci) -> T {
    if (fix && ci < 0) return T(0);
    if (dropx && (ci < 0 || ci >= nx)) return T(0);
    return __ldcg(v + row + pmap(ci, nx, op.px));
  };
  auto vy = [&](int cj) -> T {
    if (dropy && (cj < 0 || cj >= ny)) return T(0);
    return __ldcg(v + static_cast<long long>(pmap(cj, ny, op.py)) * nx + i);
  };
  acc += -xc * he * vx(i + 2) - xc * (he - hw) * vx(i + 1) + xc * (he - hw) * vx(i - 1) - xc * hw * vx(i - 2);
  acc += -yc * hn * vy(j + 2) - yc * (hn - hs) * vy(j + 1) + yc * (hn - hs) * vy(j - 1) - yc * hs * vy(j - 2);
  return acc;
}

struct Rows {
  long long r0, r1;
};
__device__ __forceinline__ Rows own_rows(long long n)
{
  const long long per = (n + gridDim.x - 1) / gridDim.x;
  Rows o;
  o.r0 = per * blockIdx.x;
  o.r1 = o.r0 + per < n ? o.r0 + per : n;
  if (o.r0 > n) o.r0 = n;
  return o;
}

// Shared-memory layout of one block (doubles): six vectors of m+8 (Givens
// cosines/sines, rotated rhs g, current Hessenberg column, reduced values,
// update coefficients), per-warp partials of one sum (NW), and NT + m + 8
// scratch (grid reductions stage at most max(NT, m + 8) values).
constexpr int NW = NT / 32;
struct Smem {
  double* cs;
  double* sn;
  double* g;
  double* hcol;
  double* red;
  double* coef;
  double* wpart;
  double* scratch;
};
__device__ __forceinline__ Smem carve(double* base, int m)
{
  const int L = m + 8;
  Smem s;
  s.cs = base;
  s.sn = s.cs + L;
  s.g = s.sn + L;
  s.hcol = s.g + L;
  s.red = s.hcol + L;
  s.coef = s.red + L;
  s.wpart = s.coef + L;
  s.scratch = s.wpart + NW;
  return s;
}
inline size_t smem_bytes(int m) { return sizeof(double) * (static_cast<size_t>(7) * (m + 8) + NW + NT); }

// Per-thread value v of one sum -> per-warp partial (lane 0 stores).
__device__ __forceinline__ void warp_partial(double v, double* wpart)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) wpart[threadIdx.x >> 5] = v;
}

// *dst = sum of the warp partials in warp order.
__device__ __forceinline__ void commit_partial(const double* wpart, double* dst)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < NW; ++w) s += wpart[w];
    *dst = s;
  }
  __syncthreads();
}

// out[q] = sum over blocks of part[b][q] (q < cnt), blocks in fixed groups,
// groups in order: every block computes identical values.
__device__ __forceinline__ void grid_reduce_redundant(const double* part, int ld, int cnt, double* out, double* scratch)
{
  const int nb = gridDim.x;
  int groups = NT / cnt;
  if (groups < 1) groups = 1;
  const int per = (nb + groups - 1) / groups;
  for (int t = threadIdx.x; t < cnt * groups; t += NT) {
    const int q = t % cnt, gi = t / cnt;
    const int b0 = gi * per, b1 = b0 + per < nb ? b0 + per : nb;
    double s = 0.0;
    for (int b = b0; b < b1; ++b) s += __ldcg(part + static_cast<long long>(b) * ld + q);
    if (cnt * groups <= NT) scratch[gi * cnt + q] = s;
    else scratch[q] = s;  // cnt > NT: one group
  }
  __syncthreads();
  for (int q = threadIdx.x; q < cnt; q += NT) {
    double s = 0.0;
    if (cnt * groups <= NT)
      for (int gi = 0; gi < groups; ++gi) s += scratch[gi * cnt + q];
    else
      s = scratch[q];
    out[q] = s;
  }
  __syncthreads();
}

__device__ __forceinline__ double nanmax(double m, double v) { return (m < v || v != v) ? v : m; }

__device__ __forceinline__ double warp_max(double m)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = nanmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

// Block max (NaN propagates, marking nonfinite) -> part_row[q].
__device__ __forceinline__ void block_max_partial(double v, double* part_row, int q, double* scratch)
{
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = scratch[0];
    for (int w = 1; w < NW; ++w) m = nanmax(m, scratch[w]);
    part_row[q] = m;
  }
  __syncthreads();
}

__device__ __forceinline__ double grid_max_redundant(const double* part, int ld, int q, double* scratch)
{
  double m = 0.0;
  for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += NT)
    m = nanmax(m, __ldcg(part + static_cast<long long>(b) * ld + q));
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = m;
  __syncthreads();
  double r = scratch[0];
  for (int w = 1; w < NW; ++w) r = nanmax(r, scratch[w]);
  __syncthreads();
  return r;
}

struct SolveState {
  int it;          // iterations completed
  int best_it;     // index of the iterate returned
  double best_linf;
  int converged, breakdown, nonfinite, timeout;
};

// Back substitution R y = g (k x k; R column-major, leading dimension ldr) by
// warp 0; y in shared memory.
__device__ void back_substitute(const double* R, int ldr, const double* g, int k, double* y)
{
  if (threadIdx.x < 32) {
    for (int i = k - 1; i >= 0; --i) {
      double s = 0.0;
      for (int c = i + 1 + threadIdx.x; c < k; c += 32) s += __ldcg(R + static_cast<long long>(c) * ldr + i) * y[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) y[i] = (g[i] - s) / __ldcg(R + static_cast<long long>(i) * ldr + i);
      __syncwarp();
    }
  }
  __syncthreads();
}

// Dot products of the block's rows: part_row[i] = v_i . w for i < nvec, by
// warps (warp k takes i = k, k + NW, ...), lanes striding the rows: every
// load of a warp is coalesced and independent.  Also ||w||^2 -> part_row[nvec]
// and a nonfinite flag of w -> part_row[nvec + 1] (when with_norm).
template <typename T>
__device__ __forceinline__ void block_dots(const T* __restrict__ V, long long n, const T* __restrict__ w, Rows rw,
                                           int nvec, bool with_norm, double* part_row)
{
  __syncthreads();  // w of the block's rows is complete
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tot = nvec + (with_norm ? 2 : 0);
  for (int i = warp; i < tot; i += NW) {
    double s = 0.0;
    if (i < nvec) {
      // 8 rows a lane per pass, all loads issued before the first use
      const T* vi = V + static_cast<long long>(i) * n;
      for (long long base = rw.r0 + lane; base < rw.r1; base += 32 * 8) {
        T a[8], b[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const long long q = base + 32LL * k;
          const bool ok = q < rw.r1;
          a[k] = ok ? __ldcg(vi + q) : T(0);
          b[k] = ok ? w[q] : T(0);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) s += static_cast<double>(a[k]) * static_cast<double>(b[k]);
      }
    } else if (i == nvec) {
#pragma unroll 4
      for (long long q = rw.r0 + lane; q < rw.r1; q += 32) {
        const double wd = static_cast<double>(__ldcg(w + q));
        s += wd * wd;
      }
    } else {
      for (long long q = rw.r0 + lane; q < rw.r1; q += 32)
        if (!isfinite(static_cast<double>(__ldcg(w + q)))) s = 1.0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) part_row[i] = s;
  }
  __syncthreads();
}

// One GMRES solve A x = b from x0 in precision T on this block's rows.
//  reference_rule (FP64): stop at ||r_j||inf <= tol or ||r_j||inf/max(||b||inf,1)
//    <= tol with r_j carried by the residual recurrence in rres; return the
//    iterate with the smallest ||r||inf otherwise.  The infinity norm of r_j
//    is reduced after the barrier that opens iteration j+1 (the barrier is
//    needed there anyway for the SpMV of v_{j+1}).
//  otherwise (FP32 inner solve): stop at |g_{j+1}| <= rtol * beta.
template <typename T>
__device__ SolveState krylov(const GmresArgs& a, const T* __restrict__ bvec, const T* __restrict__ x0vec,
                             T* __restrict__ xvec, T* __restrict__ V, T* __restrict__ w, double* __restrict__ rres,
                             int kmax, double tol, double rtol, bool reference_rule, unsigned int& gen, double* shbase)
{
  const long long n = a.n;
  const int nx = a.op.nx;
  const Rows rw = own_rows(n);
  const int ld = a.ld;
  const int XSLOT = ld - 1;  // block max of |r_j|, read after the next barrier
  double* part_row = a.part + static_cast<long long>(blockIdx.x) * ld;
  const Smem S = carve(shbase, a.m);
  SolveState st;
  st.it = 0;
  st.best_it = 0;
  st.best_linf = __builtin_huge_val();
  st.converged = st.breakdown = st.nonfinite = st.timeout = 0;
  double beta = 0.0;

  // ---- r0 = b - A x0: ||b||inf, ||r0||inf, ||r0||2 ----
  {
    double bmax = 0.0, rmax = 0.0, r2 = 0.0;
    for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
      const int i = static_cast<int>(q % nx), j = static_cast<int>(q / nx);
      const double bq = static_cast<double>(bvec[q]);
      const double rq = bq - static_cast<double>(apply_row<T>(a.op, x0vec, i, j, q));
      bmax = nanmax(bmax, fabs(bq));
      rmax = nanmax(rmax, fabs(rq));
      r2 += rq * rq;
      w[q] = static_cast<T>(rq);
      if (rres) rres[q] = rq;
    }
    block_max_partial(bmax, part_row, 0, S.scratch);
    block_max_partial(rmax, part_row, 1, S.scratch);
    warp_partial(r2, S.wpart);
    commit_partial(S.wpart, part_row + 2);
  }
  if (!grid_sync(a.bar, gen, a.spin_limit)) {
    st.timeout = 1;
    return st;
  }
  const double bn_raw = grid_max_redundant(a.part, ld, 0, S.scratch);
  const double r0inf = grid_max_redundant(a.part, ld, 1, S.scratch);
  grid_reduce_redundant(a.part + 2, ld, 1, S.red, S.scratch);
  beta = sqrt(S.red[0]);
  const double bn = bn_raw > 1.0 ? bn_raw : 1.0;
  bool stop = false;
  if (!isfinite(bn_raw) || !isfinite(r0inf)) {
    st.nonfinite = 1;
    stop = true;
  } else {
    st.best_linf = r0inf;  // update_best(initial_guess, 0)
    if (reference_rule && (r0inf <= tol || r0inf / bn <= tol)) {
      st.converged = 1;
      stop = true;
    } else if (kmax <= 0) {
      stop = true;
    } else if (!isfinite(beta)) {
      st.nonfinite = 1;
      stop = true;
    } else if (beta == 0.0) {
      st.converged = 1;
      st.best_linf = 0.0;
      stop = true;
    }
  }
  const double btol = kEps * 100.0 * (beta > 1.0 ? beta : 1.0);
  if (!stop) {
    for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) V[q] = static_cast<T>(static_cast<double>(w[q]) / beta);
    if (threadIdx.x == 0) S.g[0] = beta;
    __syncthreads();
  }
  bool broke = false;
  for (int j = 0; !stop; ++j) {
    if (!grid_sync(a.bar, gen, a.spin_limit)) {
      st.timeout = 1;
      return st;
    }
    if (j > 0 && reference_rule) {
      // update_best / convergence test of iterate j (residual r_{j-1})
      const double linf = grid_max_redundant(a.part, ld, XSLOT, S.scratch);
      if (!isfinite(linf)) {
        st.nonfinite = 1;
        break;
      }
      if (linf < st.best_linf) {
        st.best_linf = linf;
        st.best_it = j;
      }
      if (linf <= tol || linf / bn <= tol) {
        st.converged = 1;
        st.best_it = j;
        st.best_linf = linf;
        break;
      }
    }
    if (broke) {
      st.breakdown = 1;
      break;
    }
    if (j >= kmax) break;
    const T* vj = V + static_cast<long long>(j) * n;
    // ---- sweep A: w = A v_j; d_i = v_i . w (i <= j); ||w||^2; nonfinite ----
    for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
      const int i = static_cast<int>(q % nx), jj = static_cast<int>(q / nx);
      w[q] = apply_row<T>(a.op, vj, i, jj, q);
    }
    block_dots<T>(V, n, w, rw, j + 1, true, part_row);
    if (!grid_sync(a.bar, gen, a.spin_limit)) {
      st.timeout = 1;
      return st;
    }
    grid_reduce_redundant(a.part, ld, j + 3, S.red, S.scratch);
    if (S.red[j + 2] != 0.0) {
      st.nonfinite = 1;
      break;
    }
    double sw = S.red[j + 1];
    double dsum = 0.0;
    for (int q = 0; q <= j; ++q) dsum += S.red[q] * S.red[q];
    for (int q = threadIdx.x; q <= j; q += NT) {
      S.hcol[q] = S.red[q];
      S.coef[q] = S.red[q];
    }
    __syncthreads();
    double nn2 = sw - dsum;
    if (!(nn2 >= 0.5 * sw)) {
      // ---- DGKS second pass: w <- w - V d; d2_i = v_i . w; ||w||^2 ----
      for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
        double wv = static_cast<double>(w[q]);
#pragma unroll 8
        for (int i = 0; i <= j; ++i) wv -= S.coef[i] * static_cast<double>(V[static_cast<long long>(i) * n + q]);
        w[q] = static_cast<T>(wv);
      }
      block_dots<T>(V, n, w, rw, j + 1, true, part_row);
      if (!grid_sync(a.bar, gen, a.spin_limit)) {
        st.timeout = 1;
        return st;
      }
      grid_reduce_redundant(a.part, ld, j + 2, S.red, S.scratch);
      sw = S.red[j + 1];
      double dd = 0.0;
      for (int q = 0; q <= j; ++q) dd += S.red[q] * S.red[q];
      nn2 = sw - dd;
      for (int q = threadIdx.x; q <= j; q += NT) {
        S.hcol[q] += S.red[q];
        S.coef[q] = S.red[q];
      }
      __syncthreads();
    }
    const double nn = sqrt(nn2 > 0.0 ? nn2 : 0.0);
    if (!isfinite(nn)) {
      st.nonfinite = 1;
      break;
    }
    // ---- Givens rotation of the new column (identical in every block) ----
    if (threadIdx.x == 0) {
      S.hcol[j + 1] = nn;
      for (int i = 0; i < j; ++i) {
        const double h0 = S.hcol[i], h1 = S.hcol[i + 1];
        S.hcol[i] = S.cs[i] * h0 + S.sn[i] * h1;
        S.hcol[i + 1] = -S.sn[i] * h0 + S.cs[i] * h1;
      }
      const double h0 = S.hcol[j], h1 = S.hcol[j + 1];
      const double rho = hypot(h0, h1);
      S.cs[j] = rho == 0.0 ? 1.0 : h0 / rho;
      S.sn[j] = rho == 0.0 ? 0.0 : h1 / rho;
      S.hcol[j] = rho;
      S.hcol[j + 1] = 0.0;
      S.scratch[NT - 1] = S.g[j];  // g_j before the rotation
      S.g[j + 1] = -S.sn[j] * S.g[j];
      S.g[j] = S.cs[j] * S.g[j];
    }
    __syncthreads();
    const double c = S.cs[j], s = S.sn[j], gam = S.scratch[NT - 1];
    if (blockIdx.x == 0)
      for (int q = threadIdx.x; q <= j; q += NT) a.R[static_cast<long long>(j) * (a.m + 1) + q] = S.hcol[q];
    if (!isfinite(S.g[j]) || !isfinite(S.hcol[j])) {
      st.nonfinite = 1;
      break;
    }
    broke = !(nn > btol);
    // ---- sweep C: w <- w - V coef; v_{j+1} = w / nn; r_j recurrence ----
    T* vn = V + static_cast<long long>(j + 1) * n;
    const double inv_nn = broke ? 0.0 : 1.0 / nn;
    const double cr1 = s * s, cr2 = -s * c * gam;
    double rmx = 0.0;
    for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
      double wv = static_cast<double>(w[q]);
#pragma unroll 8
      for (int i = 0; i <= j; ++i) wv -= S.coef[i] * static_cast<double>(V[static_cast<long long>(i) * n + q]);
      const T vq = static_cast<T>(wv * inv_nn);
      vn[q] = vq;
      if (rres) {
        const double rq = cr1 * rres[q] + cr2 * static_cast<double>(vq);
        rres[q] = rq;
        rmx = nanmax(rmx, fabs(rq));
      }
    }
    st.it = j + 1;
    if (reference_rule) {
      block_max_partial(rmx, part_row, XSLOT, S.scratch);
    } else {
      const double est = fabs(S.g[j + 1]);
      st.best_it = j + 1;
      st.best_linf = est;
      if (est <= rtol * beta) {
        st.converged = 1;
        break;
      }
      if (broke) {
        st.breakdown = 1;
        break;
      }
      if (j + 1 >= kmax) break;
    }
  }
  // ---- x = x0 + V_k y_k for the returned iterate k ----
  if (!grid_sync(a.bar, gen, a.spin_limit)) {
    st.timeout = 1;
    return st;
  }
  const int k = st.best_it;
  double* y = S.red;
  back_substitute(a.R, a.m + 1, S.g, k, y);
  // For k below the last rotated column, g[0..k) and R's leading k x k block
  // are unchanged by the later rotations, so y is that iterate's.
  bool ynf = false;
  for (int q = 0; q < k; ++q) ynf |= !isfinite(y[q]);
  if (ynf) st.nonfinite = 1;
  for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
    double xv = static_cast<double>(x0vec[q]);
    if (!ynf) {
#pragma unroll 8
      for (int i = 0; i < k; ++i) xv += y[i] * static_cast<double>(V[static_cast<long long>(i) * n + q]);
    }
    xvec[q] = static_cast<T>(xv);
  }
  return st;
}

__global__ void __launch_bounds__(NT) gmres_kernel(GmresArgs a)
{
  extern __shared__ double sh[];
  unsigned int gen = 0;
  gen = ld_volatile(&a.bar->gen);  // reset to 0 by the host before the launch
  const Rows rw = own_rows(a.n);
  EcgGmresResult out;
  std::memset(&out, 0, sizeof(out));
  const int limit = a.max_iter < a.n ? a.max_iter : static_cast<int>(a.n);
  if (!a.mixed) {
    const SolveState st = krylov<double>(a, a.b, a.x0, a.x, a.V, a.w, a.r, limit > 0 ? limit : 0, a.tol, 0.0, true,
                                         gen, sh);
    out.iterations = st.best_it;
    out.converged = st.converged;
    out.breakdown = st.breakdown;
    out.nonfinite = st.nonfinite;
    out.timeout = st.timeout;
    out.residual_linf = st.best_linf;
    out.inner_iterations = st.it;
  } else {
    // FP64 iterative refinement around FP32 GMRES.
    // x <- x0; repeat: r = b - A x (FP64); stop on the reference rule;
    // solve A d = r in FP32 to inner_rtol; x <- x + d.
    for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) a.x[q] = a.x0[q];
    int total_inner = 0, sweeps = 0;
    double bn = 1.0;
    double linf = __builtin_huge_val();
    int conv = 0, nf = 0, to = 0;
    const Smem S = carve(sh, a.m);
    double* tmp = S.scratch;
    double* part_row = a.part + static_cast<long long>(blockIdx.x) * a.ld;
    for (;;) {
      if (!grid_sync(a.bar, gen, a.spin_limit)) {
        to = 1;
        break;
      }
      double bmax = 0.0, rmax = 0.0;
      for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
        const int i = static_cast<int>(q % a.op.nx), j = static_cast<int>(q / a.op.nx);
        const double rq = a.b[q] - apply_row<double>(a.op, a.x, i, j, q);
        bmax = nanmax(bmax, fabs(a.b[q]));
        rmax = nanmax(rmax, fabs(rq));
        a.r32[q] = static_cast<float>(rq);
        a.r[q] = rq;
      }
      block_max_partial(bmax, part_row, 0, tmp);
      block_max_partial(rmax, part_row, 1, tmp);
      if (!grid_sync(a.bar, gen, a.spin_limit)) {
        to = 1;
        break;
      }
      const double braw = grid_max_redundant(a.part, a.ld, 0, tmp);
      linf = grid_max_redundant(a.part, a.ld, 1, tmp);
      bn = braw > 1.0 ? braw : 1.0;
      if (!isfinite(linf) || !isfinite(braw)) {
        nf = 1;
        break;
      }
      if (linf <= a.tol || linf / bn <= a.tol) {
        conv = 1;
        break;
      }
      if (sweeps >= a.max_refine || total_inner >= limit) break;
      // inner solve from d0 = 0 (w32 holds zeros for x0)
      for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) a.w32[q] = 0.0f;
      float* d32 = a.w32 + a.n;  // correction
      for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) d32[q] = 0.0f;
      if (!grid_sync(a.bar, gen, a.spin_limit)) {
        to = 1;
        break;
      }
      const int kin = a.inner_max < limit - total_inner ? a.inner_max : limit - total_inner;
      const SolveState st = krylov<float>(a, a.r32, a.w32, d32, a.V32, a.w32 + 2 * a.n, nullptr, kin, 0.0,
                                          a.inner_rtol, false, gen, sh);
      total_inner += st.it;
      ++sweeps;
      if (st.timeout) {
        to = 1;
        break;
      }
      if (st.nonfinite) {
        nf = 1;
        break;
      }
      for (long long q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) a.x[q] += static_cast<double>(d32[q]);
    }
    out.iterations = total_inner;
    out.inner_iterations = total_inner;
    out.refinements = sweeps;
    out.converged = conv;
    out.nonfinite = nf;
    out.timeout = to;
    out.residual_linf = linf;
  }
  out.relative_residual_linf = 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.res = out;
}

// ---- residual A x - b (FP64), ||.||inf, max(||b||inf, 1), nonfinite -------------------

__global__ void __launch_bounds__(NT) residual_kernel(EcgPressureOp op, long long n, const double* __restrict__ b,
                                                      const double* __restrict__ x, double* __restrict__ part)
{
  __shared__ double sh[NW];
  double rmax = 0.0, bmax = 0.0;
  for (long long q = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * NT) {
    const int i = static_cast<int>(q % op.nx), j = static_cast<int>(q / op.nx);
    const double rq = apply_row<double>(op, x, i, j, q) - b[q];
    rmax = nanmax(rmax, fabs(rq));
    bmax = nanmax(bmax, fabs(b[q]));
  }
  block_max_partial(rmax, part + blockIdx.x * 2, 0, sh);
  block_max_partial(bmax, part + blockIdx.x * 2, 1, sh);
}

}  // namespace

struct EcgGmresWork {
  long long n = 0;
  int m = 0;
  int nblocks = 0;
  int device = 0;
  bool mixed_ready = false;
  double* V = nullptr;
  double* w = nullptr;
  double* r = nullptr;
  float* V32 = nullptr;
  float* w32 = nullptr;
  float* r32 = nullptr;
  double* part = nullptr;
  int ld = 0;
  double* R = nullptr;
  double* yv = nullptr;
  GridBar* bar = nullptr;
  EcgGmresResult* d_res = nullptr;
  EcgGmresResult* h_res = nullptr;
  double* h_part = nullptr;
  size_t smem = 0;
};

EcgGmresWork* gmres_work_create(long long n, int max_iter, int num_sms, int device, bool mixed, std::string* err)
{
  EcgGmresWork* w = new EcgGmresWork();
  w->n = n;
  w->m = max_iter < 1 ? 1 : max_iter;
  if (w->m > n) w->m = static_cast<int>(n);
  w->device = device;
  w->smem = smem_bytes(w->m);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gmres_kernel, NT, w->smem);
  if (per_sm < 1) per_sm = 1;
  // one block per SM (every SM's share of bandwidth), fewer for tiny systems
  long long want = (n + 63) / 64;
  long long cap = static_cast<long long>(num_sms) * (per_sm < 1 ? 1 : 1);
  w->nblocks = static_cast<int>(want < cap ? (want < 1 ? 1 : want) : cap);
  w->ld = w->m + 8;
  bool ok = true;
  auto alloc = [&](void** p, size_t bytes) {
    if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  alloc(reinterpret_cast<void**>(&w->V), sizeof(double) * (w->m + 1) * n);
  alloc(reinterpret_cast<void**>(&w->w), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&w->r), sizeof(double) * n);
  const long long part_len = static_cast<long long>(w->ld) * w->nblocks;
  alloc(reinterpret_cast<void**>(&w->part),
        sizeof(double) * (part_len > 2LL * kResidualBlocks ? part_len : 2LL * kResidualBlocks));
  alloc(reinterpret_cast<void**>(&w->R), sizeof(double) * (w->m + 1) * (w->m + 1));
  alloc(reinterpret_cast<void**>(&w->yv), sizeof(double) * (w->m + 1));
  alloc(reinterpret_cast<void**>(&w->bar), sizeof(GridBar));
  alloc(reinterpret_cast<void**>(&w->d_res), sizeof(EcgGmresResult));
  if (mixed) {
    alloc(reinterpret_cast<void**>(&w->V32), sizeof(float) * (w->m + 1) * n);
    alloc(reinterpret_cast<void**>(&w->w32), sizeof(float) * 3 * n);
    alloc(reinterpret_cast<void**>(&w->r32), sizeof(float) * n);
    w->mixed_ready = true;
  }
  if (ok && cudaMallocHost(&w->h_res, sizeof(EcgGmresResult)) != cudaSuccess) ok = false;
  if (ok && cudaMallocHost(&w->h_part, sizeof(double) * 2 * kResidualBlocks) != cudaSuccess) ok = false;
  if (ok && cudaMemset(w->bar, 0, sizeof(GridBar)) != cudaSuccess) ok = false;
  if (ok && cudaFuncSetAttribute(gmres_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(w->smem)) !=
                cudaSuccess)
    ok = false;
  if (!ok) {
    if (err) *err = "gmres workspace allocation failed";
    gmres_work_destroy(w);
    return nullptr;
  }
  return w;
}

void gmres_work_destroy(EcgGmresWork* w)
{
  if (!w) return;
  cudaFree(w->V);
  cudaFree(w->w);
  cudaFree(w->r);
  cudaFree(w->V32);
  cudaFree(w->w32);
  cudaFree(w->r32);
  cudaFree(w->part);
  cudaFree(w->R);
  cudaFree(w->yv);
  cudaFree(w->bar);
  cudaFree(w->d_res);
  cudaFreeHost(w->h_res);
  cudaFreeHost(w->h_part);
  delete w;
}

cudaError_t gmres_solve(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x0, double* x,
                        int max_iter, double tol, bool mixed, int inner_max_iter, double inner_rtol, int max_refine,
                        EcgGmresResult* out, cudaStream_t s)
{
  if (mixed && !w->mixed_ready) return cudaErrorInvalidValue;
  GmresArgs a;
  std::memset(&a, 0, sizeof(a));
  a.op = op;
  a.n = w->n;
  a.b = b;
  a.x0 = x0;
  a.x = x;
  a.V = w->V;
  a.w = w->w;
  a.r = w->r;
  a.V32 = w->V32;
  a.w32 = w->w32;
  a.r32 = w->r32;
  a.part = w->part;
  a.R = w->R;
  a.yv = w->yv;
  a.bar = w->bar;
  a.res = w->d_res;
  a.ld = w->ld;
  a.m = w->m;
  a.max_iter = max_iter < w->m ? max_iter : w->m;
  a.tol = tol;
  a.mixed = mixed ? 1 : 0;
  a.inner_max = inner_max_iter < a.max_iter ? inner_max_iter : a.max_iter;
  a.inner_rtol = inner_rtol;
  a.max_refine = max_refine;
  a.spin_limit = 1LL << 25;  // ~2 s of polling before a barrier gives up
  cudaError_t e = cudaMemsetAsync(w->bar, 0, sizeof(GridBar), s);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(gmres_kernel), dim3(w->nblocks), dim3(NT), args, w->smem, s);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(w->h_res, w->d_res, sizeof(EcgGmresResult), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  *out = *w->h_res;
  return cudaSuccess;
}

cudaError_t pressure_residual(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x,
                              double* res_linf, double* rhs_norm, int* nonfinite, cudaStream_t s)
{
  const int nb = kResidualBlocks;
  residual_kernel<<<nb, NT, 0, s>>>(op, w->n, b, x, w->part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(w->h_part, w->part, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  double rm = 0.0, bm = 0.0;
  bool nf = false;
  for (int q = 0; q < nb; ++q) {
    const double rv = w->h_part[2 * q], bv = w->h_part[2 * q + 1];
    if (!std::isfinite(rv) || !std::isfinite(bv)) nf = true;
    rm = rm < rv ? rv : rm;
    bm = bm < bv ? bv : bm;
  }
  *res_linf = nf ? std::numeric_limits<double>::quiet_NaN() : rm;
  *rhs_norm = bm > 1.0 ? bm : 1.0;
  *nonfinite = nf ? 1 : 0;
  return cudaSuccess;
}
