// GMRES pressure solve of the IMEX step: one persistent cooperative launch
// per solve, matrix-free operator, grid reductions through accumulator rows
// that every block reads after a barrier.
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
// Mixed precision: the Krylov basis is stored in FP32 (half the bytes of
// every sweep over it); the operator, w, the dot products, the Hessenberg
// column, the rotations and the residual recurrence stay FP64, so the basis
// rounding is the only FP32 error (a compressed-basis GMRES).  The solve
// restarts from the current iterate whenever the recurrence says the cycle
// converged, or its residual fell by inner_rtol after at least kMinCycle
// iterations, and every cycle opens with the true FP64 residual b - A x: the
// reference's stopping rule is applied to it.  These cycles take the DGKS
// second pass only under severe cancellation (option reorth).
// Small systems keep the first basis vectors resident in shared memory on
// each block's rows (the RES instantiation of the kernel).
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
constexpr int kMinCycle = 16;  // mixed: shortest cycle a restart may end

struct GridBar {
  unsigned int arrive;  // arrivals; the top bit is the timeout flag
  unsigned int settle;  // deterministic mode: blocks that have written their partial sums
  unsigned int pad[2];
};

struct GmresArgs {
  EcgPressureOp op;
  long long n;
  const double* b;
  const double* x0;
  double* x;
  double* V;     // (m+1) x n (FP64 solve)
  double* w;     // n
  double* r;     // n: residual recurrence
  float* V32;    // (m+1) x n (mixed)
  double* part;  // residual_kernel: 2 x its blocks
  double* acc;   // three accumulator rows of ld doubles, zeroed by the host before the launch
  double* dpt;   // deterministic mode: three tables of per-block partial sums (nblocks x ld each)
  double* R;     // column-major (m+1) x m
  GridBar* bar;
  EcgGmresResult* res;
  int ld;
  int m;          // basis capacity
  int max_iter;
  double tol;
  int mixed;
  int inner_max;      // mixed: iterations per cycle
  double inner_rtol;  // mixed: restart when the recurrence residual fell by this factor
  int max_refine;     // mixed: cycles
  int reorth;         // mixed: DGKS test of the FP32-basis cycles, 1 as the FP64 solve, 0 severe cancellation only
  int kres;           // basis vectors resident in shared memory on each block's rows
  int prow;           // rows of a block (the last may have fewer)
  int det;            // grid sums in a fixed order (bit-reproducible solves)
  long long spin_limit;
  // Chained solves (gmres_enqueue): gate[0] is set once a phase of the chain
  // failed, gate[1] when a mixed solve left its system to the FP64 fallback.
  // role 1: a chain's solve; role 2: its FP64 fallback.
  int* gate;
  int role;
};

// Grid-wide barrier over co-resident blocks (cooperative launch): one
// arrival counter that only grows (zeroed by the host before the launch), so
// barrier number g is passed once it reaches (g + 1) x blocks; one release
// atomic per block and no reset on the critical path.  The counter's top bit
// is the timeout flag: a block that waits longer than spin_limit polls sets
// it and leaves, every block polling sees it in the value it reads, and the
// flag costs no load of its own after the barrier.
constexpr unsigned int kBarTimeout = 0x80000000u;

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p)
{
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned int atom_add_release(unsigned int* p, unsigned int x)
{
  unsigned int v;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "r"(x) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_sync(GridBar* bar, unsigned int& gen, long long spin_limit)
{
  __shared__ int passed;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int target = (gen + 1u) * gridDim.x;
    unsigned int v = atom_add_release(&bar->arrive, 1u) + 1u;
    long long spins = 0;
    while (!(v & kBarTimeout) && static_cast<int>(v - target) < 0) {
      if (++spins > spin_limit) {
        atomicOr(&bar->arrive, kBarTimeout);
        v |= kBarTimeout;
        break;
      }
      __nanosleep(32);
      v = ld_acquire(&bar->arrive);
    }
    passed = (v & kBarTimeout) ? 0 : 1;
  }
  ++gen;
  __syncthreads();
  return passed != 0;
}

// source_map_index: wrap or even reflection (imex_source_map_helpers.hpp:169-188),
// for k within two cells of [0, n)
__device__ __forceinline__ int pmap(int k, int n, int per)
{
  if (per) {
    if (n >= 2) return k < 0 ? k + n : (k >= n ? k - n : k);
    return 0;
  }
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

template <typename TV>
__device__ __forceinline__ double ldv(const TV* p)
{
  return static_cast<double>(__ldcg(p));
}

// The Krylov basis: V in global memory ((m+1) x n, the copy other blocks'
// operator rows read), and its first K vectors on the block's own rows
// r0 .. r0+P-1 also resident in shared memory (vector i, row q at
// s[i P + q - r0]), where the block's dot products and combinations read
// them without an L2 round trip.
template <typename TV>
struct Basis {
  TV* V;
  long long n;
  TV* s;
  int K, P, r0;
  __device__ __forceinline__ TV* vec(int i) const { return V + static_cast<long long>(i) * n; }
  __device__ __forceinline__ void store(int i, int q, TV v) const
  {
    V[static_cast<long long>(i) * n + q] = v;
    if (i < K) s[i * P + q - r0] = v;
  }
};

// acc[r] + sgn sum_{i<cnt} c[i] V_i[q_r] for R rows q_r of the block at once,
// i ascending (the rounding of the plain loop): the resident vectors from
// shared memory, then the rest with 32 (FP64) or 16 (FP32) loads in flight
// before the first FMA (the stores that follow a call would otherwise keep
// the compiler from starting the next row's loads: the new basis vector
// aliases V).
template <typename TV, bool SUB, int R>
__device__ __forceinline__ void basis_combine(double (&acc)[R], const Basis<TV>& bs, const int (&q)[R], const double* c,
                                              int cnt)
{
  constexpr int B = (sizeof(TV) == 8 ? 32 : 16) / R;
  constexpr int BS = 8 / R;  // shared-memory loads in flight: their latency is short
  const int ks = cnt < bs.K ? cnt : bs.K;
  for (int i0 = 0; i0 < ks; i0 += BS) {
    TV a[R][BS];
#pragma unroll
    for (int k = 0; k < BS; ++k)
#pragma unroll
      for (int r = 0; r < R; ++r) a[r][k] = bs.s[(i0 + k < ks ? i0 + k : ks - 1) * bs.P + q[r] - bs.r0];
#pragma unroll
    for (int k = 0; k < BS; ++k)
      if (i0 + k < ks) {
        const double ck = c[i0 + k];
#pragma unroll
        for (int r = 0; r < R; ++r)
          acc[r] = SUB ? acc[r] - ck * static_cast<double>(a[r][k]) : acc[r] + ck * static_cast<double>(a[r][k]);
      }
  }
  const TV* __restrict__ V = bs.V;
  const long long n = bs.n;
  for (int i0 = ks; i0 < cnt; i0 += B) {
    TV a[R][B];
#pragma unroll
    for (int k = 0; k < B; ++k)
#pragma unroll
      for (int r = 0; r < R; ++r) a[r][k] = i0 + k < cnt ? __ldcg(V + static_cast<long long>(i0 + k) * n + q[r]) : TV(0);
#pragma unroll
    for (int k = 0; k < B; ++k)
      if (i0 + k < cnt) {
        const double ck = c[i0 + k];
#pragma unroll
        for (int r = 0; r < R; ++r)
          acc[r] = SUB ? acc[r] - ck * static_cast<double>(a[r][k]) : acc[r] + ck * static_cast<double>(a[r][k]);
      }
  }
}

// basis_combine for the FP32 basis of an even-sized system on the row pair
// q, q+1 (q even): one 8-byte load per vector and pair, so twice the bytes
// in flight for the same loads.  Resident vectors come from shared memory.
template <bool SUB>
__device__ __forceinline__ void basis_combine_pair(double (&acc)[2], const Basis<float>& bs, int q, const double* c,
                                                   int cnt)
{
  constexpr int B = 16;
  const int ks = cnt < bs.K ? cnt : bs.K;
  for (int i = 0; i < ks; ++i) {
    const double ck = c[i];
    const float* sv = bs.s + i * bs.P + q - bs.r0;
    acc[0] = SUB ? acc[0] - ck * static_cast<double>(sv[0]) : acc[0] + ck * static_cast<double>(sv[0]);
    acc[1] = SUB ? acc[1] - ck * static_cast<double>(sv[1]) : acc[1] + ck * static_cast<double>(sv[1]);
  }
  const float* __restrict__ V = bs.V;
  const long long n = bs.n;
  for (int i0 = ks; i0 < cnt; i0 += B) {
    float2 a[B];
#pragma unroll
    for (int k = 0; k < B; ++k)
      a[k] = __ldcg(reinterpret_cast<const float2*>(V + static_cast<long long>(i0 + k < cnt ? i0 + k : cnt - 1) * n + q));
#pragma unroll
    for (int k = 0; k < B; ++k)
      if (i0 + k < cnt) {
        const double ck = c[i0 + k];
        acc[0] = SUB ? acc[0] - ck * static_cast<double>(a[k].x) : acc[0] + ck * static_cast<double>(a[k].x);
        acc[1] = SUB ? acc[1] - ck * static_cast<double>(a[k].y) : acc[1] + ck * static_cast<double>(a[k].y);
      }
  }
}

// Rows q_r = j nx + i of A v with A the source-map pressure operator
// (imex_source_map_helpers.hpp:533-543), in FP64 whatever the storage of v,
// R rows with every load issued before the arithmetic (indices are always in
// range; left-out terms are selected away after the load).  Columns at a
// fixed Dirichlet pressure are not part of A (their terms are in the
// right-hand side): the bubble's left boundary, and with op.drop every column
// outside a non-periodic axis (the direct T1/S2 driver,
// imex_bdltv20_direct_driver.hpp:455-466).
template <typename TV, int R>
__device__ __forceinline__ void apply_rows(const EcgPressureOp& op, const TV* __restrict__ v, const int (&q)[R],
                                           double (&out)[R])
{
  const int nx = op.nx, ny = op.ny;
  const double* __restrict__ hx = op.hx;
  const double* __restrict__ hy = op.hy;
  const bool fix = op.bubble && !op.px;
  const bool dropx = op.drop && !op.px, dropy = op.drop && !op.py;
  double h[R][4], c[R][9];
  bool keep[R][8];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = q[r] / nx, i = q[r] - j * nx;
    h[r][0] = hx[j * (nx + 1) + i + 1];
    h[r][1] = hx[j * (nx + 1) + i];
    h[r][2] = hy[(j + 1) * nx + i];
    h[r][3] = hy[j * nx + i];
    c[r][0] = ldv(v + q[r]);
    const int row = j * nx;
    const int dx[4] = {2, 1, -1, -2};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int ci = i + dx[k], cj = j + dx[k];
      keep[r][k] = !((fix && ci < 0) || (dropx && (ci < 0 || ci >= nx)));
      keep[r][4 + k] = !(dropy && (cj < 0 || cj >= ny));
      c[r][1 + k] = ldv(v + row + pmap(ci, nx, op.px));
      c[r][5 + k] = ldv(v + pmap(cj, ny, op.py) * nx + i);
    }
  }
  const double xc = op.xc, yc = op.yc;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double he = h[r][0], hw = h[r][1], hn = h[r][2], hs = h[r][3];
    double e[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) e[k] = keep[r][k] ? c[r][1 + k] : 0.0;
    double acc = (op.diag0 + xc * (he + hw) + yc * (hn + hs)) * c[r][0];
    acc += -xc * he * e[0] - xc * (he - hw) * e[1] + xc * (he - hw) * e[2] - xc * hw * e[3];
    acc += -yc * hn * e[4] - yc * (hn - hs) * e[5] + yc * (hn - hs) * e[6] - yc * hs * e[7];
    out[r] = acc;
  }
}

struct Rows {
  int r0, r1;
};
// Rows of a block: an even count (so row pairs of an even-sized system stay
// 8-byte aligned in an FP32 basis), the last block taking what is left.
__host__ __device__ constexpr long long rows_per_block(long long n, int nblocks)
{
  return ((n + nblocks - 1) / nblocks + 1) / 2 * 2;
}
__device__ __forceinline__ Rows own_rows(long long n)
{
  const long long per = rows_per_block(n, gridDim.x);
  long long r0 = per * blockIdx.x, r1 = r0 + per;
  if (r1 > n) r1 = n;
  if (r0 > n) r0 = n;
  return Rows{static_cast<int>(r0), static_cast<int>(r1)};
}

// Shared-memory layout of one block (doubles): six vectors of m+8 (Givens
// cosines/sines, rotated rhs g, current Hessenberg column, reduced values,
// update coefficients), per-warp partials of one sum (NW), NT + m + 8 scratch
// (grid reductions stage at most max(NT, m + 8) values), and the per-warp
// partials of every dot product of a sweep (NW x LW).
constexpr int NW = NT / 32;
// dot products a thread accumulates per pass over its rows (16 spills under
// the 128-register cap of 512-thread blocks)
constexpr int DG_ROWS = 8;
__host__ __device__ constexpr int dots_ld(int m) { return ((m + 3 + DG_ROWS - 1) / DG_ROWS) * DG_ROWS; }
struct Smem {
  double* cs;
  double* sn;
  double* g;
  double* hcol;
  double* red;
  double* coef;
  double* wpart;
  double* scratch;
  double* vs;  // resident basis vectors (TV)
  double* dpart;
  double* cnt;  // block 0: vector accesses per row of the solve, [0] FP64 vectors, [1] basis vectors stored as FP32
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
  s.cnt = s.scratch + NT + L;
  s.dpart = s.cnt + 2;
  s.vs = s.dpart + NW * dots_ld(m);
  return s;
}
// bytes of the fixed part; the resident basis vectors follow it
inline size_t smem_bytes(int m)
{
  return sizeof(double) * (static_cast<size_t>(7) * (m + 8) + NW + NT + 2 + static_cast<size_t>(NW) * dots_ld(m));
}

// Algorithmic traffic of the solve, counted by block 0's thread 0 in
// vector-element accesses per row: a sweep that reads or writes one vector of
// n entries counts 1 (the operator's 9-point stencil reads its input vector
// once, and the two face-enthalpy arrays as one vector each).  nb: accesses to
// basis vectors (FP64 or FP32, the TV of the solve), n64: to FP64 vectors.
template <typename TV>
__device__ __forceinline__ void count(const Smem& S, double n64, double nb)
{
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S.cnt[0] += n64 + (sizeof(TV) == 8 ? nb : 0.0);
    S.cnt[1] += sizeof(TV) == 8 ? 0.0 : nb;
  }
}

// Per-thread value v of one sum -> per-warp partial (lane 0 stores).
__device__ __forceinline__ void warp_partial(double v, double* wpart)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) wpart[threadIdx.x >> 5] = v;
}

// Grid sums and maxima go through accumulator rows: every block adds its
// partial sums (or raises its partial maxima) into entry q of one row, a grid
// barrier follows, and every block reads the row.  All blocks read the same
// final values; the order of the additions is the memory system's, so a sum
// may differ from launch to launch in its last bits.  Three rows rotate:
// after reading row k, block 0 clears row k + 2, which no block reads or
// writes again before the barrier that precedes the producers of reduction
// k + 2.
//
// Deterministic mode (dpt set): a block writes its partial sums of reduction
// k into its own slot of partial table k % 3 instead, and the block that
// writes its partials last adds them up in block order into the row before
// the grid barrier (acc_settle), so every launch on the same inputs gives the
// same bits.  Maxima are exact in any order and stay atomic.
struct Acc {
  double* rows;
  int ld;
  double* dpt;  // per-block partial tables (deterministic mode), else null
  __device__ __forceinline__ double* row(unsigned int k) const { return rows + (k % 3) * ld; }
};

// Destination of one block's partial sums of one reduction.
struct SumSink {
  double* p;
  bool det;
};
__device__ __forceinline__ SumSink sink(const Acc& A, unsigned int k)
{
  if (A.dpt) return SumSink{A.dpt + (static_cast<size_t>(k % 3) * gridDim.x + blockIdx.x) * A.ld, true};
  return SumSink{A.row(k), false};
}

__device__ __forceinline__ void acc_add(const SumSink& s, int q, double v)
{
  if (s.det) s.p[q] = v;
  else atomicAdd(s.p + q, v);
}

// Maxima are nonnegative or NaN (with the sign bit clear), which order as
// their bit patterns, NaN above every number.
__device__ __forceinline__ void acc_max(double* row, int q, double v)
{
  atomicMax(reinterpret_cast<unsigned long long*>(row + q), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// Deterministic mode, after every block has written its partial sums of
// reduction k (entries [0, ns)) and before the grid barrier that precedes
// their readers: the block that arrives last sums the partial table in block
// order (lane l takes blocks l, l + 32, ..., then a fixed shuffle tree) into
// row k.  The arrival count only grows; nset counts the settles passed.
__device__ __forceinline__ void acc_settle(const Acc& A, GridBar* bar, unsigned int k, int ns, unsigned int& nset)
{
  if (!A.dpt) return;
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int v = atomicAdd(&bar->settle, 1u);
    last = v + 1u == (nset + 1u) * gridDim.x ? 1 : 0;
  }
  ++nset;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* tab = A.dpt + static_cast<size_t>(k % 3) * gridDim.x * A.ld;
  double* row = A.row(k);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = warp; q < ns; q += NW) {
    double s = 0.0;
    for (int b = lane; b < static_cast<int>(gridDim.x); b += 32) s += __ldcg(tab + static_cast<size_t>(b) * A.ld + q);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) __stcg(row + q, s);
  }
  __syncthreads();
}

// After the grid barrier that follows the producers of reduction k: out[q] =
// entry q of row k (q < ne) in every block; k advances.
__device__ __forceinline__ void acc_read(const Acc& A, unsigned int& k, int ne, double* out)
{
  const double* r = A.row(k);
  for (int q = threadIdx.x; q < ne; q += NT) out[q] = __ldcg(r + q);
  if (blockIdx.x == 0) {
    double* z = A.row(k + 2);
    for (int q = threadIdx.x; q < A.ld; q += NT) z[q] = 0.0;
  }
  ++k;
  __syncthreads();
}

// Adds the sum of the warp partials, in warp order, to entry q of an
// accumulator row (or writes it to the block's partial slot).
__device__ __forceinline__ void commit_sum(const double* wpart, const SumSink& row, int q)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < NW; ++w) s += wpart[w];
    acc_add(row, q, s);
  }
  __syncthreads();
}

__device__ __forceinline__ double nanmax(double m, double v) { return (m < v || v != v) ? v : m; }

// sum_{q<k} red[q]^2 by every warp (lanes stride, fixed shuffle tree): the
// same value in every thread of every block.
__device__ __forceinline__ double sum_squares(const double* red, int k)
{
  double s = 0.0;
  for (int q = threadIdx.x & 31; q < k; q += 32) s += red[q] * red[q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

__device__ __forceinline__ double warp_max(double m)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = nanmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

// Block max (NaN propagates, marking nonfinite), returned in thread 0.
__device__ __forceinline__ double block_max(double v, double* scratch)
{
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = scratch[0];
  if (threadIdx.x == 0)
    for (int w = 1; w < NW; ++w) m = nanmax(m, scratch[w]);
  __syncthreads();
  return m;
}

struct SolveState {
  int it;          // iterations completed
  int best_it;     // index of the iterate returned
  double best_linf;
  double r0_linf;  // infinity norm of b - A x0
  double b_linf;   // infinity norm of b
  int converged, breakdown, nonfinite, timeout;
  int restart;     // mixed: the recurrence residual fell by inner_rtol
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

// Warp sums of DG values by a reduce-scatter butterfly: after it, lane
// (32 / DG) k holds the warp's sum of s[k] (DG - 1 + log2(32 / DG) shuffles in
// place of 5 DG).  Fixed pairing: the same result in every warp and launch.
template <int DG>
__device__ __forceinline__ double warp_reduce_scatter(double (&s)[DG], int lane)
{
#pragma unroll
  for (int h = DG / 2, off = 16; h >= 1; h >>= 1, off >>= 1) {
    const bool up = (lane & off) != 0;
#pragma unroll
    for (int k = 0; k < h; ++k) {
      const double send = up ? s[k] : s[k + h];
      const double keep = up ? s[k + h] : s[k];
      s[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  double v = s[0];
#pragma unroll
  for (int off = 16 / DG; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Dot products of the block's rows, added to an accumulator row: entry i
// += v_i . w for i < nvec, and with_norm: ||w||^2 to entry nvec, a nonfinite
// count of w to entry nvec + 1.  Every thread takes part: DG sums a pass over its rows
// (w read once a pass), a reduce-scatter of the DG sums in each warp, then
// the warps' partials summed in warp order.
template <typename TV>
__device__ __forceinline__ void block_dots(const Basis<TV>& bs, const double* __restrict__ w, Rows rw, int nvec,
                                           bool with_norm, const SumSink& row, double* dpart, bool pair)
{
  const TV* __restrict__ V = bs.V;
  const long long n = bs.n;
  constexpr int DG = DG_ROWS;
  constexpr int SMALL = 16;  // rows a lane holds in the small-block layout
  __syncthreads();  // w of the block's rows is complete
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tot = nvec + (with_norm ? 2 : 0);
  if (rw.r1 - rw.r0 <= 32 * SMALL) {
    // Few rows (an L2-resident system): warp k takes vectors k, k + NW, ...
    // over all the block's rows, lanes striding the rows with w in registers;
    // one round trip a vector and no block-wide step between vectors.
    double wr[SMALL];
#pragma unroll
    for (int k = 0; k < SMALL; ++k) {
      const int q = rw.r0 + lane + 32 * k;
      wr[k] = q < rw.r1 ? w[q] : 0.0;
    }
    for (int i = warp; i < tot; i += NW) {
      double sm = 0.0;
      if (i < nvec) {
        TV av[SMALL];
        if (i < bs.K) {
          const TV* pv = bs.s + i * bs.P + lane;
#pragma unroll
          for (int k = 0; k < SMALL; ++k) av[k] = rw.r0 + lane + 32 * k < rw.r1 ? pv[32 * k] : TV(0);
        } else {
          const TV* pv = V + static_cast<long long>(i) * n + rw.r0 + lane;  // rows at immediate offsets
#pragma unroll
          for (int k = 0; k < SMALL; ++k) av[k] = rw.r0 + lane + 32 * k < rw.r1 ? __ldcg(pv + 32 * k) : TV(0);
        }
#pragma unroll
        for (int k = 0; k < SMALL; ++k) sm += static_cast<double>(av[k]) * wr[k];
      } else if (i == nvec) {
#pragma unroll
        for (int k = 0; k < SMALL; ++k) sm += wr[k] * wr[k];
      } else {
#pragma unroll
        for (int k = 0; k < SMALL; ++k)
          if (!isfinite(wr[k])) sm = 1.0;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sm += __shfl_xor_sync(0xffffffffu, sm, o);
      if (lane == 0) acc_add(row, i, sm);
    }
    __syncthreads();
    return;
  }
  for (int g0 = 0; g0 < tot; g0 += DG) {
    double s[DG];
#pragma unroll
    for (int k = 0; k < DG; ++k) s[k] = 0.0;
    // FP64 basis: two rows a pass (2 DG loads in flight); FP32: one, or with
    // pair (an even-sized system) the adjacent rows q, q+1 in one 8-byte load
    constexpr int RS = sizeof(TV) == 8 ? 2 : 1;
    const bool pr = sizeof(TV) == 4 && pair;
    const int qstep = pr ? 2 * NT : RS * NT;
    for (int q = rw.r0 + (pr ? 2 : 1) * static_cast<int>(threadIdx.x); q < rw.r1; q += qstep) {
      const bool hb = pr || (RS == 2 && q + NT < rw.r1);
      const int qb = pr ? q + 1 : (hb ? q + NT : q);
      const double wq[2] = {w[q], hb ? w[qb] : 0.0};
      TV a[2][DG];
      if (g0 + DG <= bs.K) {  // a group of resident vectors
#pragma unroll
        for (int k = 0; k < DG; ++k) {
          a[0][k] = bs.s[(g0 + k) * bs.P + q - rw.r0];
          a[1][k] = hb ? bs.s[(g0 + k) * bs.P + qb - rw.r0] : TV(0);
        }
      } else if (pr) {
        if constexpr (sizeof(TV) == 4) {
#pragma unroll
          for (int k = 0; k < DG; ++k) {
            const float2 v = __ldcg(reinterpret_cast<const float2*>(
                V + static_cast<long long>(g0 + k < nvec ? g0 + k : nvec - 1) * n + q));
            a[0][k] = v.x;
            a[1][k] = v.y;
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < DG; ++k) {
          a[0][k] = g0 + k < nvec ? __ldcg(V + static_cast<long long>(g0 + k) * n + q) : TV(0);
          a[1][k] = g0 + k < nvec && hb ? __ldcg(V + static_cast<long long>(g0 + k) * n + qb) : TV(0);
        }
      }
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        if (r == 1 && !hb) break;
#pragma unroll
        for (int k = 0; k < DG; ++k) {
          const int i = g0 + k;
          if (i < nvec) s[k] += static_cast<double>(a[r][k]) * wq[r];
          else if (i == nvec && with_norm) s[k] += wq[r] * wq[r];
          else if (i == nvec + 1 && with_norm && !isfinite(wq[r])) s[k] = 1.0;
        }
      }
    }
    const double v = warp_reduce_scatter<DG>(s, lane);
    if ((lane & (32 / DG - 1)) == 0) dpart[(g0 + lane / (32 / DG)) * NW + warp] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < tot; i += NT) {
    double t = 0.0;
    for (int wv = 0; wv < NW; ++wv) t += dpart[i * NW + wv];
    acc_add(row, i, t);
  }
  __syncthreads();
}

// Short FP64 bases (nvec + 2 <= DG_ROWS) on blocks of more rows than
// threads: the operator (COMB false: w = A v) or the Gram-Schmidt update
// (COMB true: w <- w - V c, c of length nvec) and then the dot products
// v_i . w (i < nvec), ||w||^2 and w's nonfinite flag, in ONE pass over the
// block's rows: w is not read back, and the update's basis values serve the
// dot products too.  Rows q and q + NT a pass and the sums in block_dots'
// order, so the results are those of the two separate sweeps.
template <bool COMB>
__device__ __forceinline__ void fused_sweep_dots(const EcgPressureOp& op, Rows rw, const double* __restrict__ v,
                                                 const Basis<double>& bs, const double* c, double* __restrict__ w,
                                                 int nvec, const SumSink& row, double* dpart)
{
  constexpr int DG = DG_ROWS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tot = nvec + 2;
  const double* __restrict__ V = bs.V;
  const long long n = bs.n;
  double s[DG];
#pragma unroll
  for (int k = 0; k < DG; ++k) s[k] = 0.0;
  for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += 2 * NT) {
    const bool hb = q + NT < rw.r1;
    const int qq[2] = {q, hb ? q + NT : q};
    double val[2];
    double a[2][DG];
    if (!COMB) apply_rows<double, 2>(op, v, qq, val);
#pragma unroll
    for (int k = 0; k < DG; ++k)
#pragma unroll
      for (int r = 0; r < 2; ++r)
        a[r][k] = k < nvec ? (k < bs.K ? bs.s[k * bs.P + qq[r] - bs.r0] : __ldcg(V + static_cast<long long>(k) * n + qq[r]))
                           : 0.0;
    if (COMB) {
#pragma unroll
      for (int r = 0; r < 2; ++r) val[r] = w[qq[r]];
#pragma unroll
      for (int k = 0; k < DG; ++k)
        if (k < nvec) {
          const double ck = c[k];
#pragma unroll
          for (int r = 0; r < 2; ++r) val[r] = val[r] - ck * a[r][k];
        }
    }
    w[qq[0]] = val[0];
    if (hb) w[qq[1]] = val[1];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (r == 1 && !hb) break;
#pragma unroll
      for (int k = 0; k < DG; ++k) {
        if (k < nvec) s[k] += a[r][k] * val[r];
        else if (k == nvec) s[k] += val[r] * val[r];
        else if (k == nvec + 1 && !isfinite(val[r])) s[k] = 1.0;
      }
    }
  }
  const double vs = warp_reduce_scatter<DG>(s, lane);
  if ((lane & (32 / DG - 1)) == 0) dpart[(lane / (32 / DG)) * NW + warp] = vs;
  __syncthreads();
  for (int i = threadIdx.x; i < tot; i += NT) {
    double t = 0.0;
    for (int wv = 0; wv < NW; ++wv) t += dpart[i * NW + wv];
    acc_add(row, i, t);
  }
  __syncthreads();
}

// The row sweeps of a cycle, R rows of the block at a time (R = 2 when the
// block has more rows than threads, else 1: no duplicate loads).

// w = b - A x0 and rres = w on the block's rows; running max |b|, max |r|, sum r^2.
template <int R>
__device__ __forceinline__ void sweep_r0(const EcgPressureOp& op, Rows rw, const double* __restrict__ b,
                                         const double* __restrict__ x0, double* __restrict__ w, double* __restrict__ rres,
                                         double& bmax, double& rmax, double& r2)
{
  for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += R * NT) {
    int qq[R];
#pragma unroll
    for (int r = 0; r < R; ++r) qq[r] = q + r * NT < rw.r1 ? q + r * NT : q;
    double ax[R];
    apply_rows<double, R>(op, x0, qq, ax);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (q + r * NT >= rw.r1) break;
      const double bq = b[qq[r]];
      const double rq = bq - ax[r];
      bmax = nanmax(bmax, fabs(bq));
      rmax = nanmax(rmax, fabs(rq));
      r2 += rq * rq;
      w[qq[r]] = rq;
      rres[qq[r]] = rq;
    }
  }
}

// w = A v on the block's rows.
template <typename TV, int R>
__device__ __forceinline__ void sweep_spmv(const EcgPressureOp& op, Rows rw, const TV* __restrict__ v,
                                           double* __restrict__ w)
{
  for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += R * NT) {
    int qq[R];
#pragma unroll
    for (int r = 0; r < R; ++r) qq[r] = q + r * NT < rw.r1 ? q + r * NT : q;
    double av[R];
    apply_rows<TV, R>(op, v, qq, av);
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (q + r * NT < rw.r1) w[qq[r]] = av[r];
  }
}

// out = in + sgn V c (cnt basis vectors) on the block's rows.
template <typename TV, bool SUB, int R>
__device__ __forceinline__ void sweep_combine(Rows rw, const Basis<TV>& bs, const double* c, int cnt, const double* in,
                                              double* out)
{
  for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += R * NT) {
    int qq[R];
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      qq[r] = q + r * NT < rw.r1 ? q + r * NT : q;
      acc[r] = in[qq[r]];
    }
    basis_combine<TV, SUB, R>(acc, bs, qq, c, cnt);
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (q + r * NT < rw.r1) out[qq[r]] = acc[r];
  }
}

// sweep_next on row pairs (FP32 basis, even-sized system): thread t takes
// rows r0 + 2t, r0 + 2t + 1, then 2 NT rows further.
__device__ __forceinline__ double sweep_next_pair(Rows rw, const Basis<float>& bs, const double* c, int cnt,
                                                  const double* __restrict__ w, double inv_nn, double cr1, double cr2,
                                                  double* __restrict__ rres)
{
  double rmx = 0.0;
  for (int q = rw.r0 + 2 * static_cast<int>(threadIdx.x); q < rw.r1; q += 2 * NT) {
    double acc[2] = {w[q], w[q + 1]};
    const double rp[2] = {rres[q], rres[q + 1]};
    basis_combine_pair<true>(acc, bs, q, c, cnt);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const float vq = static_cast<float>(acc[r] * inv_nn);
      bs.store(cnt, q + r, vq);
      const double rq = cr1 * rp[r] + cr2 * static_cast<double>(vq);
      rres[q + r] = rq;
      rmx = nanmax(rmx, fabs(rq));
    }
  }
  return rmx;
}

// w - V c -> v_cnt = (w - V c) inv_nn (stored as TV), and the residual
// recurrence rres <- cr1 rres + cr2 v_cnt; returns the block-local max |rres|.
template <typename TV, int R>
__device__ __forceinline__ double sweep_next(Rows rw, const Basis<TV>& bs, const double* c, int cnt,
                                             const double* __restrict__ w, double inv_nn, double cr1, double cr2,
                                             double* __restrict__ rres)
{
  double rmx = 0.0;
  for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += R * NT) {
    int qq[R];
    double acc[R], rp[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      qq[r] = q + r * NT < rw.r1 ? q + r * NT : q;
      acc[r] = w[qq[r]];
      rp[r] = rres[qq[r]];
    }
    basis_combine<TV, true, R>(acc, bs, qq, c, cnt);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (q + r * NT >= rw.r1) break;
      const TV vq = static_cast<TV>(acc[r] * inv_nn);
      bs.store(cnt, qq[r], vq);
      const double rq = cr1 * rp[r] + cr2 * static_cast<double>(vq);
      rres[qq[r]] = rq;
      rmx = nanmax(rmx, fabs(rq));
    }
  }
  return rmx;
}

// One GMRES cycle A x = b from x0, basis stored as TV, arithmetic FP64.
// Stops at ||r_j||inf <= tol or ||r_j||inf/max(||b||inf,1) <= tol (the
// reference's rule) with r_0 = b - A x0 computed and r_j carried by the
// residual recurrence in rres; returns the iterate with the smallest
// ||r||inf otherwise.  The infinity norm of r_j is reduced after the barrier
// that opens iteration j+1 (needed there anyway for the SpMV of v_{j+1}).
// restart_rtol > 0 (mixed): also stop, with restart set, once ||r_j||inf <=
// restart_rtol ||r_0||inf.  x0vec and xvec may be the same array (a restart):
// each row of x is read and then written by one thread, after the last read
// of x0 by any other row.
template <typename TV, bool RES>
__device__ SolveState krylov(const GmresArgs& a, const double* __restrict__ bvec, const double* x0vec, double* xvec,
                             TV* __restrict__ V, double* __restrict__ w,
                             double* __restrict__ rres, int kmax, double tol, double restart_rtol, int reorth,
                             unsigned int& gen, unsigned int& nred, unsigned int& nset, double* shbase)
{
  const long long n = a.n;
  const Rows rw = own_rows(n);
  const bool wide = rw.r1 - rw.r0 > NT;  // two rows a thread per pass
  // FP32 basis of an even-sized system: adjacent row pairs, 8-byte loads
  const bool pair = sizeof(TV) == 4 && wide && (n & 1) == 0;
  const Smem S = carve(shbase, a.m);
  // RES = false: no resident vectors (K a constant 0, the shared-memory
  // paths compiled out, the register budget of the plain solve)
  const Basis<TV> bs{V, n, reinterpret_cast<TV*>(S.vs), RES ? a.kres : 0, a.prow, rw.r0};
  const Acc A{a.acc, a.ld, a.det ? a.dpt : nullptr};
  SolveState st;
  st.it = 0;
  st.best_it = 0;
  st.best_linf = __builtin_huge_val();
  st.r0_linf = __builtin_huge_val();
  st.b_linf = 0.0;
  st.converged = st.breakdown = st.nonfinite = st.timeout = st.restart = 0;
  double beta = 0.0;

  // ---- r0 = b - A x0: ||r0||2, ||b||inf, ||r0||inf ----
  {
    double bmax = 0.0, rmax = 0.0, r2 = 0.0;
    if (wide) sweep_r0<2>(a.op, rw, bvec, x0vec, w, rres, bmax, rmax, r2);
    else sweep_r0<1>(a.op, rw, bvec, x0vec, w, rres, bmax, rmax, r2);
    warp_partial(r2, S.wpart);
    commit_sum(S.wpart, sink(A, nred), 0);
    bmax = block_max(bmax, S.scratch);
    rmax = block_max(rmax, S.scratch);
    if (threadIdx.x == 0) {
      acc_max(A.row(nred), 1, bmax);
      acc_max(A.row(nred), 2, rmax);
    }
    acc_settle(A, a.bar, nred, 1, nset);
  }
  if (!grid_sync(a.bar, gen, a.spin_limit)) {
    st.timeout = 1;
    return st;
  }
  acc_read(A, nred, 3, S.red);
  count<TV>(S, 6.0, 0.0);  // r0 = b - A x0: x0, hx, hy, b read; w, rres written
  beta = sqrt(S.red[0]);
  const double bn_raw = S.red[1];
  const double r0inf = S.red[2];
  st.r0_linf = r0inf;
  st.b_linf = bn_raw;
  const double bn = bn_raw > 1.0 ? bn_raw : 1.0;
  const double rtarget = restart_rtol > 0.0 ? restart_rtol * r0inf : -1.0;
  bool stop = false;
  if (!isfinite(bn_raw) || !isfinite(r0inf)) {
    st.nonfinite = 1;
    stop = true;
  } else {
    st.best_linf = r0inf;  // update_best(initial_guess, 0)
    if (r0inf <= tol || r0inf / bn <= tol) {
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
    for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) bs.store(0, q, static_cast<TV>(w[q] / beta));
    if (threadIdx.x == 0) S.g[0] = beta;
    __syncthreads();
  }
  bool broke = false;
  // update_best / convergence test of iterate j (residual r_{j-1}, whose
  // block maxima sweep C of iteration j-1 left in slot j+3); true: stop
  auto check = [&](int j, double linf) {
    if (!isfinite(linf)) {
      st.nonfinite = 1;
      return true;
    }
    if (linf < st.best_linf) {
      st.best_linf = linf;
      st.best_it = j;
    }
    if (linf <= tol || linf / bn <= tol) {
      st.converged = 1;
      st.best_it = j;
      st.best_linf = linf;
      return true;
    }
    // a cycle restarts only once its basis holds kMinCycle vectors: shorter
    // cycles would pay the restart (a true residual and the iterate's update)
    // for the few sweeps they save
    if (linf <= rtarget && j >= kMinCycle) {
      st.restart = 1;
      st.best_it = j;
      st.best_linf = linf;
      return true;
    }
    return false;
  };
  for (int j = 0; !stop; ++j) {
    if (!grid_sync(a.bar, gen, a.spin_limit)) {
      st.timeout = 1;
      return st;
    }
    if (broke || j >= kmax) {
      // no further column: the test of iterate j on its own
      if (j > 0) {
        acc_read(A, nred, j + 4, S.red);
        if (check(j, S.red[j + 3])) break;
      }
      if (broke) st.breakdown = 1;
      break;
    }
    const TV* vj = V + static_cast<long long>(j) * n;
    // ---- sweep A: w = A v_j; d_i = v_i . w (i <= j); ||w||^2; nonfinite ----
    // (a short FP64 basis: one pass, w not read back)
    bool fused = false;
    if constexpr (sizeof(TV) == 8) {
      if (wide && j + 3 <= DG_ROWS) {
        fused_sweep_dots<false>(a.op, rw, vj, bs, nullptr, w, j + 1, sink(A, nred), S.dpart);
        count<TV>(S, 4.0, j + 1.0);  // v_j, hx, hy, w written; j + 1 vectors
        fused = true;
      }
    }
    if (!fused) {
      if (wide) sweep_spmv<TV, 2>(a.op, rw, vj, w);
      else sweep_spmv<TV, 1>(a.op, rw, vj, w);
      block_dots<TV>(bs, w, rw, j + 1, true, sink(A, nred), S.dpart, pair);
      count<TV>(S, 4.0, j + 2.0);  // w = A v_j (v_j, hx, hy, w); v_i . w (j + 1 vectors, w)
    }
    acc_settle(A, a.bar, nred, j + 3, nset);
    if (!grid_sync(a.bar, gen, a.spin_limit)) {
      st.timeout = 1;
      return st;
    }
    // the dot products and, in the same read, the residual maximum of iterate
    // j: the test runs here, one sweep A later than its data, so it costs no
    // reduction of its own (a stopping iterate discards this w)
    acc_read(A, nred, j > 0 ? j + 4 : j + 3, S.red);
    if (j > 0 && check(j, S.red[j + 3])) break;
    if (S.red[j + 2] != 0.0) {
      st.nonfinite = 1;
      break;
    }
    double sw = S.red[j + 1];
    const double dsum = sum_squares(S.red, j + 1);
    for (int q = threadIdx.x; q <= j; q += NT) {
      S.hcol[q] = S.red[q];
      S.coef[q] = S.red[q];
    }
    __syncthreads();
    double nn2 = sw - dsum;
    // DGKS: a second pass when ||w'||^2 < eta ||w||^2.  The FP32-basis cycles
    // may take it only under severe cancellation: their basis rounding
    // (2^-24) already bounds orthogonality far above what the second pass
    // restores, and a cycle only has to reduce its residual by inner_rtol.
    const double eta = (sizeof(TV) == 8 || reorth) ? 0.5 : 1.0e-6;
    if (!(nn2 >= eta * sw)) {
      // ---- DGKS second pass: w <- w - V d; d2_i = v_i . w; ||w||^2 ----
      // (a short FP64 basis: one pass, the basis read once)
      bool fused2 = false;
      if constexpr (sizeof(TV) == 8) {
        if (wide && j + 3 <= DG_ROWS) {
          fused_sweep_dots<true>(a.op, rw, nullptr, bs, S.coef, w, j + 1, sink(A, nred), S.dpart);
          count<TV>(S, 2.0, j + 1.0);  // w read and written; j + 1 vectors
          fused2 = true;
        }
      }
      if (!fused2) {
        if (wide) sweep_combine<TV, true, 2>(rw, bs, S.coef, j + 1, w, w);
        else sweep_combine<TV, true, 1>(rw, bs, S.coef, j + 1, w, w);
        block_dots<TV>(bs, w, rw, j + 1, true, sink(A, nred), S.dpart, pair);
        count<TV>(S, 3.0, 2.0 * (j + 1));  // w -= V d (j + 1 vectors, w twice); v_i . w again
      }
      acc_settle(A, a.bar, nred, j + 3, nset);
      if (!grid_sync(a.bar, gen, a.spin_limit)) {
        st.timeout = 1;
        return st;
      }
      acc_read(A, nred, j + 2, S.red);
      sw = S.red[j + 1];
      nn2 = sw - sum_squares(S.red, j + 1);
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
    broke = !(nn > btol);
    const double inv_nn = broke ? 0.0 : 1.0 / nn;
    // ---- sweep C, first half, on few-row blocks (one row a thread of warps
    // 1-15): w <- w - V coef, v_{j+1} = w / nn, while thread 0 rotates; the
    // recurrence, which needs the rotation, follows from registers ----
    const bool overlap = rw.r1 - rw.r0 <= NT - 32;
    int qv = -1;
    double vqd = 0.0, rp = 0.0;
    if (overlap && threadIdx.x >= 32) {
      const int q = rw.r0 + static_cast<int>(threadIdx.x) - 32;
      if (q < rw.r1) {
        const int qq[1] = {q};
        double acc[1] = {w[q]};
        rp = rres[q];
        basis_combine<TV, true, 1>(acc, bs, qq, S.coef, j + 1);
        const TV vq = static_cast<TV>(acc[0] * inv_nn);
        bs.store(j + 1, q, vq);
        vqd = static_cast<double>(vq);
        qv = q;
      }
    }
    // ---- Givens rotation of the new column (identical in every block) ----
    if (threadIdx.x == 0) {
      // the running entry stays in a register; the rotations and the column
      // are read 8 at a time ahead of the dependent chain
      double hr = S.hcol[0];
      for (int i0 = 0; i0 < j; i0 += 8) {
        double cc[8], ss[8], hh[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int i = i0 + k < j ? i0 + k : j - 1;
          cc[k] = S.cs[i];
          ss[k] = S.sn[i];
          hh[k] = S.hcol[i + 1];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if (i0 + k < j) {
            S.hcol[i0 + k] = cc[k] * hr + ss[k] * hh[k];
            hr = -ss[k] * hr + cc[k] * hh[k];
          }
        }
      }
      const double h0 = hr, h1 = nn;
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
    // ---- sweep C: w <- w - V coef; v_{j+1} = w / nn; r_j recurrence ----
    const double cr1 = s * s, cr2 = -s * c * gam;
    double rmx = 0.0;
    if (overlap) {
      if (qv >= 0) {
        const double rq = cr1 * rp + cr2 * vqd;
        rres[qv] = rq;
        rmx = nanmax(rmx, fabs(rq));
      }
    } else {
      if constexpr (sizeof(TV) == 4) {
        if (pair) rmx = sweep_next_pair(rw, bs, S.coef, j + 1, w, inv_nn, cr1, cr2, rres);
        else
          rmx = wide ? sweep_next<TV, 2>(rw, bs, S.coef, j + 1, w, inv_nn, cr1, cr2, rres)
                     : sweep_next<TV, 1>(rw, bs, S.coef, j + 1, w, inv_nn, cr1, cr2, rres);
      } else {
        rmx = wide ? sweep_next<TV, 2>(rw, bs, S.coef, j + 1, w, inv_nn, cr1, cr2, rres)
                   : sweep_next<TV, 1>(rw, bs, S.coef, j + 1, w, inv_nn, cr1, cr2, rres);
      }
    }
    st.it = j + 1;
    count<TV>(S, 3.0, j + 2.0);  // v_{j+1} = (w - V coef) / nn: j + 1 vectors, w, v_{j+1}; rres read and written
    rmx = block_max(rmx, S.scratch);
    if (threadIdx.x == 0) acc_max(A.row(nred), j + 4, rmx);  // entry (j+1)+3, read after the next sweep A
  }
  // ---- x = x0 + V_k y_k for the returned iterate k ----
  if (!grid_sync(a.bar, gen, a.spin_limit)) {
    st.timeout = 1;
    return st;
  }
  int k = st.best_it;
  double* y = S.red;
  back_substitute(a.R, a.m + 1, S.g, k, y);
  // For k below the last rotated column, g[0..k) and R's leading k x k block
  // are unchanged by the later rotations, so y is that iterate's.
  bool ynf = false;
  for (int q = 0; q < k; ++q) ynf |= !isfinite(y[q]);
  if (ynf) st.nonfinite = 1;
  if (ynf) k = 0;  // x = x0
  if (wide) sweep_combine<TV, false, 2>(rw, bs, y, k, x0vec, xvec);
  else sweep_combine<TV, false, 1>(rw, bs, y, k, x0vec, xvec);
  count<TV>(S, 2.0, k);  // x = x0 + V_k y: x0, x, k vectors
  return st;
}

// One instantiation per (resident basis, basis precision): the FP64 and the
// FP32-basis solves each get the registers of their own path.
template <bool RES, bool MIXED>
__global__ void __launch_bounds__(NT) gmres_kernel(GmresArgs a)
{
  extern __shared__ double sh[];
  // A gated solve whose chain already failed, or a fallback nobody needs,
  // does nothing (every block reads the same flags, written before the launch).
  if (a.gate && (__ldcg(a.gate) != 0 || (a.role == 2 && __ldcg(a.gate + 1) == 0))) return;
  unsigned int gen = 0;   // barriers passed; the counter is zeroed by the host before the launch
  unsigned int nred = 0;  // accumulator reductions completed
  unsigned int nset = 0;  // deterministic mode: partial-sum settles passed
  EcgGmresResult out;
  std::memset(&out, 0, sizeof(out));
  const int limit = a.max_iter < a.n ? a.max_iter : static_cast<int>(a.n);
  bool final_known = false;  // mixed: the final true residual is already known
  double known_r = 0.0, known_b = 0.0;
  {
    const Smem S0 = carve(sh, a.m);
    if (threadIdx.x == 0) S0.cnt[0] = S0.cnt[1] = 0.0;
  }
  if constexpr (!MIXED) {
    const SolveState st =
        krylov<double, RES>(a, a.b, a.x0, a.x, a.V, a.w, a.r, limit > 0 ? limit : 0, a.tol, 0.0, 1, gen, nred, nset, sh);
    out.iterations = st.best_it;
    out.converged = st.converged;
    out.breakdown = st.breakdown;
    out.nonfinite = st.nonfinite;
    out.timeout = st.timeout;
    out.residual_linf = st.best_linf;
    out.inner_iterations = st.it;
    out.initial_linf = st.r0_linf;
    out.b_linf = st.b_linf;
  } else {
    // Cycles of the FP32-basis solve; each opens with the true FP64 residual
    // of the current iterate (x0, then x) and the reference's stopping rule.
    // A cycle that cut the true residual by less than kStall (its recurrence
    // believed an FP32 basis that had lost its orthogonality) turns the DGKS
    // second pass on for the cycles that follow.
    constexpr double kStall = 0.1;
    int total = 0, cycles = 0;
    int reorth = a.reorth;
    double prev_r0 = __builtin_huge_val();
    const double* xin = a.x0;
    SolveState st;
    std::memset(&st, 0, sizeof(st));
    const int per_cycle = a.inner_max > 0 ? a.inner_max : limit;
    for (;;) {
      const int left = limit - total;
      const bool last = cycles + 1 >= a.max_refine;
      const int kin = per_cycle < left ? per_cycle : left;
      st = krylov<float, RES>(a, a.b, xin, a.x, a.V32, a.w, a.r, kin > 0 ? kin : 0, a.tol, last ? 0.0 : a.inner_rtol,
                              reorth, gen, nred, nset, sh);
      if (cycles == 0) {
        out.initial_linf = st.r0_linf;
        out.b_linf = st.b_linf;
      }
      if (cycles > 0 && !(st.r0_linf <= kStall * prev_r0) && !reorth) {
        reorth = 1;
        out.stalled_cycles += 1;
      }
      prev_r0 = st.r0_linf;
      ++cycles;
      out.iterations = total + st.best_it;
      total += st.it;
      if (st.timeout || st.nonfinite || st.breakdown) break;
      if (st.converged && st.it == 0) {
        // the true residual of x, computed as this cycle opened, meets the
        // rule: it is the returned iterate's final residual as well
        final_known = true;
        known_r = st.r0_linf;
        known_b = st.b_linf;
        break;
      }
      if (total >= limit || last) break;
      xin = a.x;
      if (!grid_sync(a.bar, gen, a.spin_limit)) {  // x complete before the next residual
        st.timeout = 1;
        break;
      }
    }
    out.converged = st.converged;
    out.breakdown = st.breakdown;
    out.nonfinite = st.nonfinite;
    out.timeout = st.timeout;
    out.residual_linf = st.best_linf;
    out.inner_iterations = total;
    out.refinements = cycles;
  }
  out.relative_residual_linf = 0.0;
  // ---- the returned iterate's true residual ||A x - b||inf, ||b||inf (one
  // sweep after x is complete; the host reads them with the result) ----
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  out.final_linf = out.final_b_linf = nan;
  if (final_known) {
    out.final_linf = known_r;
    out.final_b_linf = known_b;
  } else if (!out.timeout && grid_sync(a.bar, gen, a.spin_limit)) {
    const Rows rw = own_rows(a.n);
    const Smem S = carve(sh, a.m);
    const Acc A{a.acc, a.ld, nullptr};  // maxima only
    double rmax = 0.0, bmax = 0.0;
    for (int q = rw.r0 + threadIdx.x; q < rw.r1; q += NT) {
      const int qq[1] = {q};
      double ax[1];
      apply_rows<double, 1>(a.op, a.x, qq, ax);
      rmax = nanmax(rmax, fabs(ax[0] - a.b[q]));
      bmax = nanmax(bmax, fabs(a.b[q]));
    }
    rmax = block_max(rmax, S.scratch);
    bmax = block_max(bmax, S.scratch);
    if (threadIdx.x == 0) {
      acc_max(A.row(nred), 0, rmax);
      acc_max(A.row(nred), 1, bmax);
    }
    if (grid_sync(a.bar, gen, a.spin_limit)) {
      if (blockIdx.x == 0) {
        acc_read(A, nred, 2, S.red);
        out.final_linf = S.red[0];
        out.final_b_linf = S.red[1];
      }
    } else {
      out.timeout = 1;
    }
  } else {
    out.timeout = 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const Smem S = carve(sh, a.m);
    out.vec_access64 = S.cnt[0] + (final_known ? 0.0 : 4.0);  // the final residual: x, hx, hy, b
    out.vec_access32 = S.cnt[1];
    *a.res = out;
    if (a.gate) {
      // the caller's tests on the returned iterate's true residual, as the
      // IMEX step takes them: a mixed solve ending finite above the rule is
      // handed to the fallback, any other solve failing it stops the chain
      const bool fin = isfinite(out.final_linf) && isfinite(out.final_b_linf);
      if (a.role == 2) a.gate[1] = 0;
      bool hand_over = false;
      if (MIXED && a.role == 1 && !out.timeout && !out.nonfinite && fin) {
        const double fb = out.final_b_linf < 1.0 ? 1.0 : out.final_b_linf;
        hand_over = !(out.final_linf <= a.tol || out.final_linf / fb <= a.tol);
      }
      if (hand_over) {
        a.gate[1] = 1;
      } else {
        const double bn = out.b_linf > 1.0 ? out.b_linf : 1.0;
        const bool conv = fin && (out.final_linf <= a.tol || out.final_linf / bn <= a.tol);
        if (out.timeout || !conv) a.gate[0] = 1;
      }
    }
  }
}

// ---- residual A x - b (FP64), ||.||inf, max(||b||inf, 1), nonfinite -------------------

__global__ void __launch_bounds__(NT) residual_kernel(EcgPressureOp op, long long n, const double* __restrict__ b,
                                                      const double* __restrict__ x, double* __restrict__ part)
{
  __shared__ double sh[NW];
  double rmax = 0.0, bmax = 0.0;
  for (int q = blockIdx.x * NT + threadIdx.x; q < n; q += gridDim.x * NT) {
    const int qq[1] = {q};
    double ax[1];
    apply_rows<double, 1>(op, x, qq, ax);
    const double rq = ax[0] - b[q];
    rmax = nanmax(rmax, fabs(rq));
    bmax = nanmax(bmax, fabs(b[q]));
  }
  rmax = block_max(rmax, sh);
  bmax = block_max(bmax, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = rmax;
    part[blockIdx.x * 2 + 1] = bmax;
  }
}

// The grid barrier's bounded wait, exercised on its own: every block passes
// barrier 0, then block 0 leaves without arriving at barrier 1, so the
// others' wait runs out after spin_limit polls.  passed[b] = 1 + (barrier 1
// passed), 0 if barrier 0 already gave up.
__global__ void barrier_probe_kernel(GridBar* bar, long long spin_limit, int* passed)
{
  unsigned int gen = 0;
  if (!grid_sync(bar, gen, spin_limit)) {
    if (threadIdx.x == 0) passed[blockIdx.x] = 0;
    return;
  }
  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) passed[0] = 1;
    return;
  }
  const bool second = grid_sync(bar, gen, spin_limit);
  if (threadIdx.x == 0) passed[blockIdx.x] = second ? 2 : 1;
}

// The kernel instantiation for a workspace: with or without the resident
// basis, FP64 or FP32 basis.
const void* gmres_entry(bool res, bool mixed)
{
  if (res) return mixed ? reinterpret_cast<const void*>(gmres_kernel<true, true>)
                        : reinterpret_cast<const void*>(gmres_kernel<true, false>);
  return mixed ? reinterpret_cast<const void*>(gmres_kernel<false, true>)
               : reinterpret_cast<const void*>(gmres_kernel<false, false>);
}

}  // namespace

struct EcgGmresWork {
  long long n = 0;
  int m = 0;
  int nblocks = 0;
  int device = 0;
  bool mixed = false;
  double* V = nullptr;
  double* w = nullptr;
  double* r = nullptr;
  float* V32 = nullptr;
  double* part = nullptr;  // residual_kernel's block maxima
  double* acc = nullptr;   // three accumulator rows of ld doubles
  double* dpt = nullptr;   // deterministic mode: three per-block partial tables (nblocks x ld)
  int ld = 0;
  double* R = nullptr;
  GridBar* bar = nullptr;
  EcgGmresResult* d_res = nullptr;
  EcgGmresResult* h_res = nullptr;
  double* h_part = nullptr;
  size_t smem = 0;
  int kres = 0;  // basis vectors resident in shared memory
  int prow = 0;  // rows of a block
};

EcgGmresWork* gmres_work_create(long long n, int max_iter, int num_sms, int device, bool mixed, std::string* err)
{
  // rows are indexed with 32-bit integers on the device
  if (n < 1 || n > (1LL << 31) - (1LL << 24)) {
    if (err) *err = "pressure system too large for the GMRES workspace (rows >= 2^31 - 2^24)";
    return nullptr;
  }
  EcgGmresWork* w = new EcgGmresWork();
  w->n = n;
  w->m = max_iter < 1 ? 1 : max_iter;
  if (w->m > n) w->m = static_cast<int>(n);
  w->device = device;
  w->mixed = mixed;
  // one block per SM (every SM's share of bandwidth), fewer for tiny systems
  const long long want = (n + 63) / 64;
  const long long cap = num_sms;
  w->nblocks = static_cast<int>(want < cap ? (want < 1 ? 1 : want) : cap);
  w->ld = w->m + 8;
  // The shared memory left over by the fixed part holds the first basis
  // vectors on the block's rows (one block per SM, so the whole opt-in
  // budget is the block's).
  w->prow = static_cast<int>(rows_per_block(n, w->nblocks));
  int optin = 0;
  cudaFuncAttributes fa;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, gmres_entry(true, mixed)) != cudaSuccess) {
    if (err) *err = "gmres kernel attributes unavailable";
    delete w;
    return nullptr;
  }
  const size_t budget = static_cast<size_t>(optin) - fa.sharedSizeBytes;
  const size_t fixed = smem_bytes(w->m);
  const size_t vbytes = static_cast<size_t>(w->prow) * (mixed ? sizeof(float) : sizeof(double));
  long long kres = budget > fixed ? static_cast<long long>((budget - fixed) / vbytes) : 0;
  if (kres > w->m + 1) kres = w->m + 1;
  // A few resident vectors save less than the L1 cache they displace costs
  // the operator's loads (measured at 768^2: 5 FP64 / 11 FP32 vectors, 16-20 %
  // slower), so residency needs 32 vectors or the whole basis.
  if (kres < 32 && kres < w->m + 1) kres = 0;
  w->kres = static_cast<int>(kres);
  w->smem = fixed + static_cast<size_t>(kres) * vbytes;
  bool ok = true;
  auto alloc = [&](void** p, size_t bytes) {
    if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  // the basis in the precision the context solves in
  if (mixed) alloc(reinterpret_cast<void**>(&w->V32), sizeof(float) * (w->m + 1) * n);
  else alloc(reinterpret_cast<void**>(&w->V), sizeof(double) * (w->m + 1) * n);
  alloc(reinterpret_cast<void**>(&w->w), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&w->r), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&w->part), sizeof(double) * 2 * kResidualBlocks);
  alloc(reinterpret_cast<void**>(&w->acc), sizeof(double) * 3 * w->ld);
  alloc(reinterpret_cast<void**>(&w->dpt), sizeof(double) * 3 * static_cast<size_t>(w->nblocks) * w->ld);
  alloc(reinterpret_cast<void**>(&w->R), sizeof(double) * (w->m + 1) * (w->m + 1));
  alloc(reinterpret_cast<void**>(&w->bar), sizeof(GridBar));
  alloc(reinterpret_cast<void**>(&w->d_res), sizeof(EcgGmresResult));
  if (ok && cudaMallocHost(&w->h_res, sizeof(EcgGmresResult)) != cudaSuccess) ok = false;
  if (ok && cudaMallocHost(&w->h_part, sizeof(double) * 2 * kResidualBlocks) != cudaSuccess) ok = false;
  if (ok && cudaMemset(w->bar, 0, sizeof(GridBar)) != cudaSuccess) ok = false;
  // the whole budget, so workspaces of any size can launch
  for (int v = 0; v < 4 && ok; ++v)
    if (cudaFuncSetAttribute(gmres_entry(v & 1, v & 2), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(budget)) != cudaSuccess)
      ok = false;
  int per_sm = 0;
  if (ok && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gmres_entry(w->kres > 0, mixed), NT, w->smem) !=
                 cudaSuccess ||
             per_sm < 1)) {
    if (err) *err = "gmres kernel does not fit on one SM with its shared memory";
    gmres_work_destroy(w);
    return nullptr;
  }
  if (!ok) {
    if (err) *err = "gmres workspace allocation failed";
    gmres_work_destroy(w);
    return nullptr;
  }
  return w;
}

bool gmres_work_resident(const EcgGmresWork* w) { return w && w->kres > 0; }

void gmres_work_destroy(EcgGmresWork* w)
{
  if (!w) return;
  cudaFree(w->V);
  cudaFree(w->w);
  cudaFree(w->r);
  cudaFree(w->V32);
  cudaFree(w->part);
  cudaFree(w->acc);
  cudaFree(w->dpt);
  cudaFree(w->R);
  cudaFree(w->bar);
  cudaFree(w->d_res);
  cudaFreeHost(w->h_res);
  cudaFreeHost(w->h_part);
  delete w;
}

cudaError_t gmres_enqueue(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x0, double* x,
                          int max_iter, double tol, bool mixed, int inner_max_iter, double inner_rtol, int max_refine,
                          int reorth, bool det, EcgGmresResult* d_res, int* gate, int role, cudaStream_t s)
{
  if (mixed != w->mixed) return cudaErrorInvalidValue;  // the basis is allocated for one precision
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
  a.part = w->part;
  a.acc = w->acc;
  a.dpt = w->dpt;
  a.det = det ? 1 : 0;
  a.R = w->R;
  a.bar = w->bar;
  a.res = d_res ? d_res : w->d_res;
  a.gate = gate;
  a.role = gate ? role : 0;
  a.ld = w->ld;
  a.m = w->m;
  a.max_iter = max_iter < w->m ? max_iter : w->m;
  a.tol = tol;
  a.mixed = mixed ? 1 : 0;
  a.inner_max = inner_max_iter < a.max_iter ? inner_max_iter : a.max_iter;  // <= 0: no per-cycle limit
  a.inner_rtol = inner_rtol;
  a.max_refine = max_refine;
  a.reorth = reorth;
  a.kres = w->kres;
  a.prow = w->prow;
  a.spin_limit = 1LL << 25;  // ~2 s of polling before a barrier gives up
  cudaError_t e = cudaMemsetAsync(w->bar, 0, sizeof(GridBar), s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(w->acc, 0, sizeof(double) * 3 * w->ld, s);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel(gmres_entry(w->kres > 0, w->mixed), dim3(w->nblocks), dim3(NT), args, w->smem, s);
}

cudaError_t gmres_solve(EcgGmresWork* w, const EcgPressureOp& op, const double* b, const double* x0, double* x,
                        int max_iter, double tol, bool mixed, int inner_max_iter, double inner_rtol, int max_refine,
                        int reorth, bool det, EcgGmresResult* out, cudaStream_t s)
{
  cudaError_t e = gmres_enqueue(w, op, b, x0, x, max_iter, tol, mixed, inner_max_iter, inner_rtol, max_refine, reorth,
                                det, nullptr, nullptr, 0, s);
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

// No counterpart in the reference: the timeout path of the GMRES grid
// barrier, on 4 blocks of 32 threads (see barrier_probe_kernel).
extern "C" ecg_status ecg_check_grid_barrier_timeout(int32_t device, int64_t spin_limit, int32_t* passed_first,
                                                     int32_t* timed_out)
{
  if (!passed_first || !timed_out || spin_limit < 1 || spin_limit > (1LL << 25)) return ECG_ERR_BAD_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return ECG_ERR_NO_DEVICE;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return ECG_ERR_CUDA;
  constexpr int kBlocks = 4;
  GridBar* bar = nullptr;
  int* d = nullptr;
  cudaStream_t s = nullptr;
  int h[kBlocks] = {};
  bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&bar, sizeof(GridBar)) == cudaSuccess && cudaMalloc(&d, sizeof(h)) == cudaSuccess &&
            cudaMemsetAsync(bar, 0, sizeof(GridBar), s) == cudaSuccess &&
            cudaMemsetAsync(d, 0xff, sizeof(h), s) == cudaSuccess;
  if (ok) {
    barrier_probe_kernel<<<kBlocks, 32, 0, s>>>(bar, spin_limit, d);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
  }
  cudaFree(bar);
  cudaFree(d);
  if (s) cudaStreamDestroy(s);
  cudaSetDevice(prev);
  if (!ok) return ECG_ERR_CUDA;
  int first = 0, out = 0;
  for (int b = 0; b < kBlocks; ++b) {
    first += h[b] >= 1 ? 1 : 0;
    out += b > 0 && h[b] == 1 ? 1 : 0;
  }
  *passed_first = first;
  *timed_out = out;
  return ECG_OK;
}
