// Stencil kernels of the explicit path: the fused MUSCL + Riemann-flux
// update with its CFL / admissibility / degenerate-star reductions, the
// whole-state reductions, and ghost fills.
//
// Included by stencil_exact.cu (compiled with -fmad=false) and
// stencil_fast.cu (-fmad=true) with ECG_NS naming the namespace.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "ecg.h"
#include "ecg_internal.h"

namespace ECG_NS {

#include "ecg_device.cuh"

constexpr double kInf = __builtin_huge_val();
constexpr double kLowest = -1.7976931348623157e308;
constexpr double kMax = 1.7976931348623157e308;

// ---- boundary-aware cell loads ---------------------------------------------

__device__ __forceinline__ int wrapi(int i, int n)
{
  int r = i % n;
  return r < 0 ? r + n : r;
}

// Where the conserved state of cell (i, j) comes from, i or j possibly
// outside the domain: the four component planes at p, p + pl, p + 2 pl,
// p + 3 pl (with my negated when flip), or the constant state bc.cst when p is
// null.  The index map reproduces the ghost values that fill_problem_ghosts
// writes (boundary_conditions.hpp:2-73): periodic wrap, outflow clamp, bubble
// wall mirror (row -j-1, my negated) and bubble inflow state; exact-state
// Dirichlet kinds read the precomputed ghost ring.
struct CellSrc {
  const double* p;
  long long pl;
  bool flip;
};

__device__ __forceinline__ CellSrc cell_src(const EcgFvParams& P, const double* __restrict__ u, int i, int j)
{
  const int nx = P.g.nx, ny = P.g.ny;
  if (static_cast<unsigned>(i) < static_cast<unsigned>(nx) && static_cast<unsigned>(j) < static_cast<unsigned>(ny))
    return CellSrc{u + static_cast<long long>(j) * P.g.pitch + i, P.g.plane, false};
  if (P.bc.ring) {
    // Tiles and warp strips that overhang the domain load cells past the
    // two-cell ring; their values feed no in-domain face, so clamp them onto
    // the ring to keep every read inside it.
    i = i < -2 ? -2 : (i > nx + 1 ? nx + 1 : i);
    j = j < -2 ? -2 : (j > ny + 1 ? ny + 1 : j);
    return CellSrc{P.ring + static_cast<long long>(j + 2) * P.ring_pitch + (i + 2), P.ring_plane, false};
  }
  int hs = -1;  // halo column of a slab side: 0, 1 left (x = -2, -1), 2, 3 right (x = nx, nx + 1)
  if (i < 0) {
    if (P.bc.x_lo == BC_HALO) hs = i < -2 ? 0 : i + 2;
    else if (P.bc.x_lo == BC_CONST) return CellSrc{nullptr, 0, false};
    else i = P.bc.x_lo == BC_PERIODIC ? wrapi(i, nx) : 0;
  } else if (i >= nx) {
    // strips past the last column read cells beyond the halo; they feed no face of the slab
    if (P.bc.x_hi == BC_HALO) hs = i - nx > 1 ? 3 : 2 + (i - nx);
    else if (P.bc.x_hi == BC_CONST) return CellSrc{nullptr, 0, false};
    else i = P.bc.x_hi == BC_PERIODIC ? wrapi(i, nx) : nx - 1;
  }
  bool flip = false;
  if (j < 0) {
    if (P.bc.y_lo == BC_CONST) return CellSrc{nullptr, 0, false};
    if (P.bc.y_lo == BC_PERIODIC) {
      j = wrapi(j, ny);
    } else if (P.bc.y_lo == BC_REFLECT) {
      j = -j - 1;
      j = j > ny - 1 ? ny - 1 : j;
      flip = true;
    } else {
      j = 0;
    }
  } else if (j >= ny) {
    if (P.bc.y_hi == BC_CONST) return CellSrc{nullptr, 0, false};
    if (P.bc.y_hi == BC_PERIODIC) {
      j = wrapi(j, ny);
    } else if (P.bc.y_hi == BC_REFLECT) {
      j = 2 * ny - 1 - j;  // row ny + k mirrors row ny - 1 - k
      j = j < 0 ? 0 : j;
      flip = true;
    } else {
      j = ny - 1;
    }
  }
  if (hs >= 0) {
    // the neighbour slab's cell, after the y policy (a corner ghost is the
    // y-mapped row of the halo column, as in the undivided grid)
    const long long fs = 2LL * ny;
    return CellSrc{(hs < 2 ? P.halo_lo : P.halo_hi) + static_cast<long long>(j) * 2 + (hs & 1), fs, flip};
  }
  return CellSrc{u + static_cast<long long>(j) * P.g.pitch + i, P.g.plane, flip};
}

// Conserved state of cell (i, j), i or j possibly outside the domain
// (cell_src's ghost policy).
__device__ __forceinline__ Cons load_cell(const EcgFvParams& P, const double* __restrict__ u, int i, int j)
{
  const CellSrc c = cell_src(P, u, i, j);
  if (!c.p) return Cons{P.bc.cst[0], P.bc.cst[1], P.bc.cst[2], P.bc.cst[3]};
  Cons r{__ldg(c.p), __ldg(c.p + c.pl), __ldg(c.p + 2 * c.pl), __ldg(c.p + 3 * c.pl)};
  if (c.flip) r.my = -r.my;
  return r;
}

// ---- block reductions --------------------------------------------------------

template <int NT>
struct BlockRed {
  unsigned long long k[3][NT / 32];
  int n[2][NT / 32];
};

__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) { return a > b ? a : b; }
__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) { return a < b ? a : b; }

// Reduces (max key, min key, min key, count, count) over the block and
// commits one atomic per quantity into `dst`.  Thread 0 gets the block's
// second count back.
template <int NT>
__device__ __forceinline__ int block_commit(BlockRed<NT>& red, unsigned long long kmax, unsigned long long kmin1,
                                             unsigned long long kmin2, int c1, int c2, EcgStepStats* dst)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    kmax = umax64(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    kmin1 = umin64(kmin1, __shfl_xor_sync(0xffffffffu, kmin1, o));
    kmin2 = umin64(kmin2, __shfl_xor_sync(0xffffffffu, kmin2, o));
    c1 += __shfl_xor_sync(0xffffffffu, c1, o);
    c2 += __shfl_xor_sync(0xffffffffu, c2, o);
  }
  if (lane == 0) {
    red.k[0][warp] = kmax;
    red.k[1][warp] = kmin1;
    red.k[2][warp] = kmin2;
    red.n[0][warp] = c1;
    red.n[1][warp] = c2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NT / 32; ++w) {
      kmax = umax64(kmax, red.k[0][w]);
      kmin1 = umin64(kmin1, red.k[1][w]);
      kmin2 = umin64(kmin2, red.k[2][w]);
      c1 += red.n[0][w];
      c2 += red.n[1][w];
    }
    atomicMax(&dst->max_rate_key, kmax);
    atomicMin(&dst->rho_min_key, kmin1);
    atomicMin(&dst->p_min_key, kmin2);
    if (c1) atomicAdd(&dst->nonfinite, c1);
    if (c2) atomicAdd(&dst->degenerate, c2);
  }
  return c2;
}

// ---- dt control --------------------------------------------------------------

// compute_euler_dt's clamp (diagnostic_metrics_timestep.hpp:252-259) on a
// reduced rate.
__device__ __host__ __forceinline__ double euler_dt_from_rate(double max_rate, double cfl, double stop, double time)
{
  double dt = stop - time;
  if (max_rate > 0.0) dt = cfl / max_rate;
  if (!isfinite(dt) || dt <= 0.0) dt = stop - time;
  const double rem = stop - time;
  return (rem < dt) ? rem : dt;
}

__device__ __forceinline__ void reset_record(EcgStepStats& s)
{
  s.max_rate_key = okey(kLowest);
  s.rho_min_key = okey(kMax);
  s.p_min_key = okey(kMax);
  s.nonfinite = 0;
  s.degenerate = 0;
  s.t = 0.0;
  s.dt = 0.0;
  s.ran = 0;
  s.halt = 0;
  s.failure = 0;
  s.step = 0;
}

// dt of this launch.  Host mode: ctl.dt.  Device mode: the driver loop's
// checks and compute_euler_dt on the reductions of the previous launch
// (driver_main.hpp:224-247, 300-310).  Returns false when the loop stops here
// (block 0 then records the stop in stats[acc_slot]).
__device__ __forceinline__ bool step_control(EcgStepStats* __restrict__ stats, const EcgDtCtl& ctl, double& dt)
{
  const bool lead = blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0;
  if (lead && ctl.reset_slot >= 0) reset_record(stats[ctl.reset_slot]);
  dt = ctl.dt;
  if (!ctl.device_dt) return true;
  const EcgStepStats& s = stats[ctl.read_slot];
  const double t = s.t;
  int failure = s.halt ? s.failure : 0;
  bool halt = s.halt != 0;
  if (!halt) {
    if (s.nonfinite > 0) failure = ECG_FAILURE_NONFINITE_STATE;
    else if (okey_inv(s.rho_min_key) <= 0.0) failure = ECG_FAILURE_NONPOSITIVE_DENSITY;
    else if (okey_inv(s.p_min_key) <= 0.0) failure = ECG_FAILURE_NONPOSITIVE_PRESSURE;
    halt = failure != 0 || s.step >= ctl.max_step || !(t < ctl.stop_time - 1.0e-14);
  }
  if (!halt) {
    dt = euler_dt_from_rate(okey_inv(s.max_rate_key), ctl.cfl, ctl.stop_time, t);
    if (!isfinite(dt) || dt <= 0.0) {
      halt = true;
      failure = ECG_FAILURE_INVALID_TIME_STEP;
    }
  }
  if (halt) {
    if (lead) {
      stats[ctl.acc_slot].halt = 1;
      stats[ctl.acc_slot].failure = failure;
      stats[ctl.acc_slot].t = t;
      stats[ctl.acc_slot].step = s.step;
    }
    return false;
  }
  if (lead) {
    stats[ctl.read_slot].dt = dt;
    stats[ctl.read_slot].ran = 1;
    stats[ctl.acc_slot].t = t + dt;
    stats[ctl.acc_slot].step = s.step + 1;
  }
  return true;
}

// ---- the fused explicit step ---------------------------------------------------

template <int TX, int TY, bool XIE>
struct FvSmem {
  static constexpr int RW = TX + 4, RH = TY + 4, RN = RW * RH;
  static constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
  static constexpr int NXR = XIE ? (TX + 1) * (TY + 2) : 0;
  static constexpr int NYR = XIE ? (TX + 2) * (TY + 1) : 0;
  static constexpr int doubles = 4 * RN + 4 * NFX + 4 * NFY + NXR + NYR;
  static constexpr size_t bytes = sizeof(double) * doubles;
};

// Face flux from the four cells (m2, m1 | c0, p1) along the face normal:
// left state = cell m1 reconstructed to its +side face, right state = cell c0
// reconstructed to its -side face (reconstructed_interface_flux,
// reconstruction_fluxes.hpp:442-460), then interface_flux (:373-388).
template <int RK>
__device__ __forceinline__ Cons face_flux(const double* __restrict__ sr, const double* __restrict__ su,
                                          const double* __restrict__ sv, const double* __restrict__ sp, int m2, int m1,
                                          int c0, int p1, int axis, const EcgFvParams& P, double sensor, bool& deg)
{
  Prim l, r;
  if (P.order <= 1) {
    l = Prim{sr[m1], su[m1], sv[m1], sp[m1]};
    r = Prim{sr[c0], su[c0], sv[c0], sp[c0]};
  } else {
    const int lim = P.limiter;
    l = Prim{recon1(sr[m2], sr[m1], sr[c0], 0.5, lim), recon1(su[m2], su[m1], su[c0], 0.5, lim),
             recon1(sv[m2], sv[m1], sv[c0], 0.5, lim), recon1(sp[m2], sp[m1], sp[c0], 0.5, lim)};
    r = Prim{recon1(sr[m1], sr[c0], sr[p1], -0.5, lim), recon1(su[m1], su[c0], su[p1], -0.5, lim),
             recon1(sv[m1], sv[c0], sv[p1], -0.5, lim), recon1(sp[m1], sp[c0], sp[p1], -0.5, lim)};
  }
  const double g = P.gamma;
  deg = false;
  if (RK == ECG_RIEMANN_RUSANOV) return rusanov_flux(l, r, axis, g);
  if (RK == ECG_RIEMANN_LOWMACH_HLLC) lowmach_correct(l, r, g);
  if (RK == ECG_RIEMANN_XIE_AM_HLLC_P) return xie_flux(l, r, axis, g, sensor, deg);
  return hllc_flux(l, r, axis, g, deg);
}

// Face pressure of cell c reconstructed to side h (= +-0.5) along one axis.
__device__ __forceinline__ double face_pressure(const double* sp, int m, int c, int p, double h, const EcgFvParams& P)
{
  return P.order <= 1 ? sp[c] : recon1(sp[m], sp[c], sp[p], h, P.limiter);
}

// One launch = one euler_fv_one_step (numerics/explicit_update.hpp:58-102)
// over a TX x TY tile per CTA: the (TX+4) x (TY+4) halo region is loaded once
// (boundary conditions folded into the load) and converted to primitives in
// shared memory, every face flux of the tile is evaluated once, and each cell
// is updated from its four face fluxes.  The epilogue reduces, over the new
// state, the spectral rate of compute_euler_dt and the minima/counts of
// compute_diagnostics, plus the degenerate-star count of this step, into
// stats[k+1].  With ctl.device_dt the kernel takes dt and time from stats[k]
// (the previous launch's reductions) so consecutive launches need no host.
template <int RK, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 2)
fv_step_kernel(const EcgFvParams P, const double* __restrict__ u, double* __restrict__ out,
               EcgStepStats* __restrict__ stats, const EcgDtCtl ctl)
{
  constexpr bool XIE = RK == ECG_RIEMANN_XIE_AM_HLLC_P;
  using S = FvSmem<TX, TY, XIE>;
  extern __shared__ double smem[];
  __shared__ BlockRed<NT> red;
  double* s_r = smem;
  double* s_u = s_r + S::RN;
  double* s_v = s_u + S::RN;
  double* s_p = s_v + S::RN;
  double* s_fx = s_p + S::RN;
  double* s_fy = s_fx + 4 * S::NFX;
  double* s_xr = s_fy + 4 * S::NFY;
  double* s_yr = s_xr + S::NXR;

  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int nx = P.g.nx, ny = P.g.ny;

  double dt;
  if (!step_control(stats, ctl, dt)) return;

  // ---- phase A: halo region -> primitives in shared memory ----
  for (int e = tid; e < S::RN; e += NT) {
    const int li = e % S::RW, lj = e / S::RW;
    const Prim q = to_prim(load_cell(P, u, i0 - 2 + li, j0 - 2 + lj), P.gamma);
    s_r[e] = q.rho;
    s_u[e] = q.u;
    s_v[e] = q.v;
    s_p[e] = q.p;
  }
  __syncthreads();

  // region index of tile-local cell (x, y), x in [-2, TX+1], y in [-2, TY+1]
  auto R = [](int x, int y) { return (y + 2) * S::RW + (x + 2); };

  // ---- phase A2 (HLLC-P): face pressure ratios of the multiface sensor ----
  if (XIE) {
    // x-faces fx in [0, TX] on rows y in [-1, TY]
    for (int e = tid; e < S::NXR; e += NT) {
      const int fx = e % (TX + 1), y = e / (TX + 1) - 1;
      const double pl = face_pressure(s_p, R(fx - 2, y), R(fx - 1, y), R(fx, y), 0.5, P);
      const double pr = face_pressure(s_p, R(fx - 1, y), R(fx, y), R(fx + 1, y), -0.5, P);
      s_xr[e] = pressure_ratio(pl, pr);
    }
    // y-faces fy in [0, TY] on columns x in [-1, TX]
    for (int e = tid; e < S::NYR; e += NT) {
      const int x = e % (TX + 2) - 1, fy = e / (TX + 2);
      const double pl = face_pressure(s_p, R(x, fy - 2), R(x, fy - 1), R(x, fy), 0.5, P);
      const double pr = face_pressure(s_p, R(x, fy - 1), R(x, fy), R(x, fy + 1), -0.5, P);
      s_yr[e] = pressure_ratio(pl, pr);
    }
    __syncthreads();
  }
  auto XR = [&](int fx, int y) { return s_xr[(y + 1) * (TX + 1) + fx]; };
  auto YR = [&](int x, int fy) { return s_yr[fy * (TX + 2) + (x + 1)]; };

  // ---- phase B: every face of the tile once ----
  int degenerate = 0;
  for (int f = tid; f < S::NFX + S::NFY; f += NT) {
    if (f < S::NFX) {
      const int fx = f % (TX + 1), y = f / (TX + 1);
      const int gj = j0 + y;
      const int wl = (fx >= 1 && i0 + fx - 1 < nx) ? 1 : 0;
      const int wr = (fx < TX && i0 + fx < nx) ? 1 : 0;
      if (gj >= ny || (wl + wr) == 0) continue;
      double sensor = 1.0;
      if (XIE) {
        // xie_multiface_pressure_sensor, axis 0 (reconstruction_fluxes.hpp:426-431)
        double m = XR(fx, y);
        m = smin(m, YR(fx - 1, y));
        m = smin(m, YR(fx - 1, y + 1));
        m = smin(m, YR(fx, y));
        m = smin(m, YR(fx, y + 1));
        const double h = clamp01(m);
        sensor = h * h * h;
      }
      bool deg;
      const Cons fl = face_flux<RK>(s_r, s_u, s_v, s_p, R(fx - 2, y), R(fx - 1, y), R(fx, y), R(fx + 1, y), 0, P,
                                    sensor, deg);
      if (ctl.count_degenerate && deg) degenerate += wl + wr;
      s_fx[f] = fl.rho;
      s_fx[S::NFX + f] = fl.mx;
      s_fx[2 * S::NFX + f] = fl.my;
      s_fx[3 * S::NFX + f] = fl.E;
    } else {
      const int g = f - S::NFX;
      const int x = g % TX, fy = g / TX;
      const int gi = i0 + x;
      const int wb = (fy >= 1 && j0 + fy - 1 < ny) ? 1 : 0;
      const int wt = (fy < TY && j0 + fy < ny) ? 1 : 0;
      if (gi >= nx || (wb + wt) == 0) continue;
      double sensor = 1.0;
      if (XIE) {
        // xie_multiface_pressure_sensor, axis 1 (reconstruction_fluxes.hpp:433-437)
        double m = YR(x, fy);
        m = smin(m, XR(x, fy - 1));
        m = smin(m, XR(x + 1, fy - 1));
        m = smin(m, XR(x, fy));
        m = smin(m, XR(x + 1, fy));
        const double h = clamp01(m);
        sensor = h * h * h;
      }
      bool deg;
      const Cons fl = face_flux<RK>(s_r, s_u, s_v, s_p, R(x, fy - 2), R(x, fy - 1), R(x, fy), R(x, fy + 1), 1, P,
                                    sensor, deg);
      if (ctl.count_degenerate && deg) degenerate += wb + wt;
      s_fy[g] = fl.rho;
      s_fy[S::NFY + g] = fl.mx;
      s_fy[2 * S::NFY + g] = fl.my;
      s_fy[3 * S::NFY + g] = fl.E;
    }
  }
  __syncthreads();

  // ---- phase C: conservative update + fused reductions ----
  unsigned long long kmax = okey(kLowest), krho = okey(kMax), kp = okey(kMax);
  int nonfinite = 0;
  const double inv_dx = P.g.inv_dx, inv_dy = P.g.inv_dy, g = P.gamma;
  for (int c = tid; c < TX * TY; c += NT) {
    const int x = c % TX, y = c / TX;
    const int gi = i0 + x, gj = j0 + y;
    if (gi >= nx || gj >= ny) continue;
    const long long o = static_cast<long long>(gj) * P.g.pitch + gi;
    const long long pl = P.g.plane;
    const int xl = y * (TX + 1) + x, yb = y * TX + x;
    Cons n;
    {
      const double* F = s_fx;
      const double* G = s_fy;
      const double o0 = __ldg(u + o);
      n.rho = o0 - dt * ((F[xl + 1] - F[xl]) * inv_dx + (G[yb + TX] - G[yb]) * inv_dy);
      F += S::NFX;
      G += S::NFY;
      const double o1 = __ldg(u + o + pl);
      n.mx = o1 - dt * ((F[xl + 1] - F[xl]) * inv_dx + (G[yb + TX] - G[yb]) * inv_dy);
      F += S::NFX;
      G += S::NFY;
      const double o2 = __ldg(u + o + 2 * pl);
      n.my = o2 - dt * ((F[xl + 1] - F[xl]) * inv_dx + (G[yb + TX] - G[yb]) * inv_dy);
      F += S::NFX;
      G += S::NFY;
      const double o3 = __ldg(u + o + 3 * pl);
      n.E = o3 - dt * ((F[xl + 1] - F[xl]) * inv_dx + (G[yb + TX] - G[yb]) * inv_dy);
    }
    out[o] = n.rho;
    out[o + pl] = n.mx;
    out[o + 2 * pl] = n.my;
    out[o + 3 * pl] = n.E;
    // compute_euler_dt (diagnostic_metrics_timestep.hpp:240-245) and
    // compute_diagnostics (:163-169) on the new state
    const Prim q = to_prim(n, g);
    const double cs = csound(q, g);
    const double rate = (fabs(q.u) + cs) / P.g.dx + (fabs(q.v) + cs) / P.g.dy;
    if (!isnan(rate)) kmax = umax64(kmax, okey(rate));
    const bool bad = !isfinite(q.rho) || !isfinite(q.u) || !isfinite(q.v) || !isfinite(q.p) || !isfinite(n.E);
    krho = umin64(krho, okey(bad ? -kInf : q.rho));
    kp = umin64(kp, okey(bad ? -kInf : q.p));
    nonfinite += bad ? 1 : 0;
  }
  block_commit<NT>(red, kmax, krho, kp, nonfinite, degenerate, &stats[ctl.acc_slot]);
}

template <int RK, int TY>
cudaError_t launch_fv_t(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats,
                        const EcgDtCtl& ctl, cudaStream_t s)
{
  constexpr int TX = 32, NT = 256;
  using S = FvSmem<TX, TY, RK == ECG_RIEMANN_XIE_AM_HLLC_P>;
  auto kern = fv_step_kernel<RK, TX, TY, NT>;
  const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::bytes));
  if (e != cudaSuccess) return e;
  const dim3 grid((p.g.nx + TX - 1) / TX, (p.g.ny + TY - 1) / TY);
  kern<<<grid, NT, S::bytes, s>>>(p, in, out, stats, ctl);
  return cudaGetLastError();
}

template <int RK>
cudaError_t launch_fv_rk(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats,
                         const EcgDtCtl& ctl, int tile_y, cudaStream_t s)
{
  if (tile_y == 8) return launch_fv_t<RK, 8>(p, in, out, stats, ctl, s);
  // 0 (default) in the exact build, 16: the 32x16 tile
  return launch_fv_t<RK, 16>(p, in, out, stats, ctl, s);
}

#ifdef ECG_FAST_KERNEL
#include "fv_fast.cuh"
#include "fv_march.cuh"
#include "fv_batch.cuh"
#endif

cudaError_t launch_fv_step(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats,
                           const EcgDtCtl& ctl, int tile_y, cudaStream_t s)
{
#ifdef ECG_FAST_KERNEL
  // 0: column-strip kernel, x- and y-faces evaluated together, rows staged
  // through shared memory by cp.async, 168 registers (default: 75.8 us at
  // 2560x640); 3: the same with rows loaded into registers, 128 registers
  // (77.8 us); 2: column-strip kernel, faces one after the other; 1:
  // square-tile kernel
  if (tile_y == 0) return march::launch(p, in, out, stats, ctl, s, true, true);
  if (tile_y == 3) return march::launch(p, in, out, stats, ctl, s, true, false);
  if (tile_y == 2) return march::launch(p, in, out, stats, ctl, s, false, false);
  if (tile_y == 1) return fast::launch(p, in, out, stats, ctl, s);
#endif
  switch (p.riemann) {
    case ECG_RIEMANN_RUSANOV: return launch_fv_rk<ECG_RIEMANN_RUSANOV>(p, in, out, stats, ctl, tile_y, s);
    case ECG_RIEMANN_LOWMACH_HLLC: return launch_fv_rk<ECG_RIEMANN_LOWMACH_HLLC>(p, in, out, stats, ctl, tile_y, s);
    case ECG_RIEMANN_XIE_AM_HLLC_P: return launch_fv_rk<ECG_RIEMANN_XIE_AM_HLLC_P>(p, in, out, stats, ctl, tile_y, s);
    default: return launch_fv_rk<ECG_RIEMANN_HLLC>(p, in, out, stats, ctl, tile_y, s);
  }
}

// ---- whole-state reductions ---------------------------------------------------

// One pass over the state for compute_euler_dt (diagnostic_metrics_timestep.hpp:227-260),
// compute_imex_dt (:272-326), compute_diagnostics (:18-47) and
// compute_admissibility_diagnostics (:49-111).
template <int NT>
__global__ void __launch_bounds__(NT) state_reduce_kernel(const EcgFvParams P, const double* __restrict__ u,
                                                          const int eq79, EcgStateStats* __restrict__ out)
{
  __shared__ unsigned long long sk[8][NT / 32];
  __shared__ int sn[5][NT / 32];
  unsigned long long k[8];
  k[0] = okey(kLowest);  // max spectral rate
  k[1] = okey(kMax);     // diag rho min
  k[2] = okey(kMax);     // diag p min
  k[3] = okey(kLowest);  // material rate
  k[4] = okey(kLowest);  // acoustic rate
  k[5] = okey(kMax);     // adm rho min
  k[6] = okey(kMax);     // adm p min
  k[7] = okey(kMax);     // adm ie min
  int n[5] = {0, 0, 0, 0, 0};
  const double g = P.gamma;
  const double mdx = smin(P.g.dx, P.g.dy);
  const long long total = static_cast<long long>(P.g.nx) * P.g.ny;
  for (long long c = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; c < total;
       c += static_cast<long long>(gridDim.x) * NT) {
    const int i = static_cast<int>(c % P.g.nx), j = static_cast<int>(c / P.g.nx);
    const long long o = static_cast<long long>(j) * P.g.pitch + i;
    const long long pl = P.g.plane;
    const Cons s{__ldg(u + o), __ldg(u + o + pl), __ldg(u + o + 2 * pl), __ldg(u + o + 3 * pl)};
    const Prim q = to_prim(s, g);
    const double cs = csound(q, g);
    const double rate = (fabs(q.u) + cs) / P.g.dx + (fabs(q.v) + cs) / P.g.dy;
    if (!isnan(rate)) {
      k[0] = umax64(k[0], okey(rate));
      k[4] = umax64(k[4], okey(rate));
    }
    const double sp = sqrt(q.u * q.u + q.v * q.v);
    const double mat = eq79 ? (2.0 * sp / mdx) : (fabs(q.u) / P.g.dx + fabs(q.v) / P.g.dy);
    if (!isnan(mat)) k[3] = umax64(k[3], okey(mat));
    const bool bad = !isfinite(q.rho) || !isfinite(q.u) || !isfinite(q.v) || !isfinite(q.p) || !isfinite(s.E);
    k[1] = umin64(k[1], okey(bad ? -kInf : q.rho));
    k[2] = umin64(k[2], okey(bad ? -kInf : q.p));
    n[0] += bad ? 1 : 0;
    // admissibility (diagnostic_metrics_timestep.hpp:64-92)
    const bool cnf = !isfinite(s.rho) || !isfinite(s.mx) || !isfinite(s.my) || !isfinite(s.E);
    const bool dbad = !cnf && s.rho <= 0.0;
    double ie = -kInf, pr = -kInf;
    bool tnf = false;
    if (!cnf && !dbad) {
      const double kin = 0.5 * (s.mx * s.mx + s.my * s.my) / s.rho;
      ie = s.E - kin;
      pr = (g - 1.0) * ie;
      tnf = !isfinite(kin) || !isfinite(ie) || !isfinite(pr);
    }
    const bool nf = cnf || tnf;
    k[5] = umin64(k[5], okey(nf ? -kInf : s.rho));
    k[6] = umin64(k[6], okey((nf || dbad) ? -kInf : pr));
    k[7] = umin64(k[7], okey((nf || dbad) ? -kInf : ie));
    n[1] += nf ? 1 : 0;
    n[2] += dbad ? 1 : 0;
    n[3] += (!nf && !dbad && pr <= 0.0) ? 1 : 0;
    n[4] += (!nf && !dbad && ie <= 0.0) ? 1 : 0;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    k[0] = umax64(k[0], __shfl_xor_sync(0xffffffffu, k[0], o));
    k[3] = umax64(k[3], __shfl_xor_sync(0xffffffffu, k[3], o));
    k[4] = umax64(k[4], __shfl_xor_sync(0xffffffffu, k[4], o));
    k[1] = umin64(k[1], __shfl_xor_sync(0xffffffffu, k[1], o));
    k[2] = umin64(k[2], __shfl_xor_sync(0xffffffffu, k[2], o));
    k[5] = umin64(k[5], __shfl_xor_sync(0xffffffffu, k[5], o));
    k[6] = umin64(k[6], __shfl_xor_sync(0xffffffffu, k[6], o));
    k[7] = umin64(k[7], __shfl_xor_sync(0xffffffffu, k[7], o));
#pragma unroll
    for (int m = 0; m < 5; ++m) n[m] += __shfl_xor_sync(0xffffffffu, n[m], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < 8; ++m) sk[m][warp] = k[m];
#pragma unroll
    for (int m = 0; m < 5; ++m) sn[m][warp] = n[m];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NT / 32; ++w) {
      k[0] = umax64(k[0], sk[0][w]);
      k[3] = umax64(k[3], sk[3][w]);
      k[4] = umax64(k[4], sk[4][w]);
      k[1] = umin64(k[1], sk[1][w]);
      k[2] = umin64(k[2], sk[2][w]);
      k[5] = umin64(k[5], sk[5][w]);
      k[6] = umin64(k[6], sk[6][w]);
      k[7] = umin64(k[7], sk[7][w]);
      for (int m = 0; m < 5; ++m) n[m] += sn[m][w];
    }
    atomicMax(&out->max_rate_key, k[0]);
    atomicMin(&out->diag_rho_min_key, k[1]);
    atomicMin(&out->diag_p_min_key, k[2]);
    atomicMax(&out->material_rate_key, k[3]);
    atomicMax(&out->acoustic_rate_key, k[4]);
    atomicMin(&out->adm_rho_min_key, k[5]);
    atomicMin(&out->adm_p_min_key, k[6]);
    atomicMin(&out->adm_ie_min_key, k[7]);
    atomicAdd(&out->diag_nonfinite, n[0]);
    atomicAdd(&out->adm_nonfinite, n[1]);
    atomicAdd(&out->adm_density_fail, n[2]);
    atomicAdd(&out->adm_pressure_fail, n[3]);
    atomicAdd(&out->adm_ie_fail, n[4]);
  }
}

__global__ void init_state_stats_kernel(EcgStateStats* st)
{
  st->max_rate_key = okey(kLowest);
  st->diag_rho_min_key = okey(kMax);
  st->diag_p_min_key = okey(kMax);
  st->material_rate_key = okey(kLowest);
  st->acoustic_rate_key = okey(kLowest);
  st->adm_rho_min_key = okey(kMax);
  st->adm_p_min_key = okey(kMax);
  st->adm_ie_min_key = okey(kMax);
  st->diag_nonfinite = 0;
  st->adm_nonfinite = st->adm_density_fail = st->adm_pressure_fail = st->adm_ie_fail = 0;
}

__global__ void init_stats_kernel(EcgStepStats* stats, int n, double t0)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    EcgStepStats s;
    s.max_rate_key = okey(kLowest);
    s.rho_min_key = okey(kMax);
    s.p_min_key = okey(kMax);
    s.nonfinite = 0;
    s.degenerate = 0;
    s.t = q == 0 ? t0 : 0.0;
    s.dt = 0.0;
    s.ran = 0;
    s.halt = 0;
    s.failure = 0;
    s.step = 0;
    stats[q] = s;
  }
}

// stats[0] <- the whole-state reductions of the initial state.
__global__ void seed_stats_kernel(EcgStepStats* stats, const EcgStateStats* st)
{
  stats[0].max_rate_key = st->max_rate_key;
  stats[0].rho_min_key = st->diag_rho_min_key;
  stats[0].p_min_key = st->diag_p_min_key;
  stats[0].nonfinite = st->diag_nonfinite;
}

#include "exact_states.cuh"

// Ghost value of cell (i, j) outside the domain under an exact-state
// Dirichlet policy (boundary_conditions.hpp:133-163,
// problem_initialization.hpp:209-263,308-375), including the periodic images
// that FillBoundary writes first.
__device__ Cons exact_ghost(const EcgFvParams& P, const EcgProblem& pr, const double* __restrict__ u, int i, int j,
                            double time)
{
  const int nx = P.g.nx, ny = P.g.ny;
  const bool xp = !pr.periodic_x && (i < 0 || i >= nx);
  const bool yp = !pr.periodic_y && (j < 0 || j >= ny);
  const double x = P.g.plo_x + (static_cast<double>(i) + 0.5) * P.g.dx;
  const double y = P.g.plo_y + (static_cast<double>(j) + 0.5) * P.g.dy;
  bool exact;
  if (pr.ring_kind == RING_TORO) exact = (i < 0 || i >= nx || yp);
  else exact = xp || yp;
  if (!exact) {
    // FillBoundary image (only periodic dimensions are out of range here)
    const int ii = pr.periodic_x ? wrapi(i, nx) : i;
    const int jj = pr.periodic_y ? wrapi(j, ny) : j;
    const long long o = static_cast<long long>(jj) * P.g.pitch + ii;
    const long long pl = P.g.plane;
    return Cons{u[o], u[o + pl], u[o + 2 * pl], u[o + 3 * pl]};
  }
  Prim q;
  if (pr.ring_kind == RING_TORO) {
    q = riemann_sample(x, time, Prim{pr.toro_l[0], pr.toro_l[1], pr.toro_l[2], pr.toro_l[3]},
                       Prim{pr.toro_r[0], pr.toro_r[1], pr.toro_r[2], pr.toro_r[3]}, pr.gamma, pr.interface_x);
  } else if (pr.ring_kind == RING_GRESHO) {
    q = gresho_state(x, y, pr);
  } else if (pr.ring_kind == RING_QUADRANT) {
    q = quadrant_state(x, y, pr);
  } else {
    const int ii = pr.periodic_x ? wrapi(i, nx) : i;
    const int jj = pr.periodic_y ? wrapi(j, ny) : j;
    const double xx = P.g.plo_x + (static_cast<double>(ii) + 0.5) * P.g.dx;
    const double yy = P.g.plo_y + (static_cast<double>(jj) + 0.5) * P.g.dy;
    const double cx = pr.blob_cx + pr.velocity_x * time, cy = pr.blob_cy + pr.velocity_y * time;
    const double r2 = (xx - cx) * (xx - cx) + (yy - cy) * (yy - cy);
    const double rho = r2 <= pr.blob_radius * pr.blob_radius ? pr.density_inner : pr.density_outer;
    q = Prim{rho, pr.velocity_x, pr.velocity_y, pr.pressure};
  }
  return to_cons(q, pr.gamma);
}

// ---- initial states (initialize_state, problems/problem_initialization.hpp:420-435) ----

// shock_density_bubble_fraction / _cell_state, problem_initialization.hpp:51-102:
// post-shock state left of x = 0.2, else ambient p = 1 with the density mixed
// by the 4 x 4 sub-cell fraction inside the r = 0.2 bubble at (0.5, 0).
__device__ Prim bubble_cell_state(double x, double y, double dx, double dy)
{
  if (x < 0.2) return Prim{2.8181818181818183, 1.6064386578049976, 0.0, 5.0};
  double inside = 0.0;
  for (int sy = 0; sy < 4; ++sy) {
    for (int sx = 0; sx < 4; ++sx) {
      const double xs = x + ((static_cast<double>(sx) + 0.5) / 4.0 - 0.5) * dx;
      const double ys = y + ((static_cast<double>(sy) + 0.5) / 4.0 - 0.5) * dy;
      const double rx = xs - 0.5, ry = ys - 0.0;
      if (xs >= 0.2 && rx * rx + ry * ry <= 0.2 * 0.2) inside += 1.0;
    }
  }
  const double f = inside / 16.0;
  return Prim{f * 0.1 + (1.0 - f) * 1.0, 0.0, 0.0, 1.0};
}

// Mach 1.22 shock / bubble cell: post-shock state left of the shock, else
// ambient (1, 0, 0, 1) with the bubble density mixed by its 4 x 4 sub-cell
// area fraction (the sampling of shock_density_bubble_fraction).
__device__ Prim mach122_cell_state(double x, double y, double dx, double dy, const double* post_shock)
{
  if (x < kM122ShockX) return Prim{post_shock[0], post_shock[1], post_shock[2], post_shock[3]};
  double inside = 0.0;
  for (int sy = 0; sy < 4; ++sy) {
    for (int sx = 0; sx < 4; ++sx) {
      const double xs = x + ((static_cast<double>(sx) + 0.5) / 4.0 - 0.5) * dx;
      const double ys = y + ((static_cast<double>(sy) + 0.5) / 4.0 - 0.5) * dy;
      const double rx = xs - kM122BubbleX, ry = ys - kM122BubbleY;
      if (xs >= kM122ShockX && rx * rx + ry * ry <= kM122BubbleR * kM122BubbleR) inside += 1.0;
    }
  }
  const double f = inside / 16.0;
  return Prim{f * kM122BubbleRho + (1.0 - f) * 1.0, 0.0, 0.0, 1.0};
}

// One thread per cell: the dispatch of initialize_state over the problems.
__global__ void init_state_kernel(const EcgFvParams P, const EcgProblem pr, double* __restrict__ u)
{
  const long long n = static_cast<long long>(P.g.nx) * P.g.ny;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % P.g.nx), j = static_cast<int>(e / P.g.nx);
    const double x = P.g.plo_x + (static_cast<double>(i) + 0.5) * P.g.dx;
    const double y = P.g.plo_y + (static_cast<double>(j) + 0.5) * P.g.dy;
    Cons c;
    if (pr.problem == ECG_PROBLEM_TORO1) {
      // initialize_toro (problem_initialization.hpp:265-289): the two states of the test
      const double* q = x < pr.interface_x ? pr.toro_l : pr.toro_r;
      c = to_cons(Prim{q[0], q[1], q[2], q[3]}, pr.gamma);
    } else if (pr.problem == ECG_PROBLEM_GRESHO_VORTEX) {
      c = to_cons(gresho_state(x, y, pr), pr.gamma);
    } else if (pr.problem == ECG_PROBLEM_ISENTROPIC_VORTEX) {
      c = to_cons(isentropic_vortex_state(x, y, pr, P.g.plo_x, P.g.plo_y, 0.0), pr.gamma);
    } else if (pr.problem == ECG_PROBLEM_RIEMANN_QUADRANT) {
      c = to_cons(quadrant_state(x, y, pr), pr.gamma);
    } else if (pr.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122) {
      c = to_cons(mach122_cell_state(x, y, P.g.dx, P.g.dy, pr.post_shock), pr.gamma);
    } else if (pr.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D ||
               pr.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL) {
      c = to_cons(bubble_cell_state(x, y, P.g.dx, P.g.dy), pr.gamma);
    } else {
      // initialize_blob (problem_initialization.hpp:127-155): top hat, stored directly
      const double r2 = (x - pr.blob_cx) * (x - pr.blob_cx) + (y - pr.blob_cy) * (y - pr.blob_cy);
      const double rho = r2 <= pr.blob_radius * pr.blob_radius ? pr.density_inner : pr.density_outer;
      const double vu = pr.velocity_x, vv = pr.velocity_y;
      c = Cons{rho, rho * vu, rho * vv, pr.pressure / (pr.gamma - 1.0) + 0.5 * rho * (vu * vu + vv * vv)};
    }
    const long long o = static_cast<long long>(j) * P.g.pitch + i;
    u[o] = c.rho;
    u[o + P.g.plane] = c.mx;
    u[o + 2 * P.g.plane] = c.my;
    u[o + 3 * P.g.plane] = c.E;
  }
}

// Writes the ghosted box [-2, nx+2) x [-2, ny+2) as fill_problem_ghosts
// leaves it.  only_ring: write the out-of-domain cells only (the ghost ring
// read by the stencil kernels under exact-state Dirichlet policies).
__global__ void ghost_box_kernel(const EcgFvParams P, const EcgProblem pr, const double* __restrict__ u, double time,
                                 const EcgStepStats* __restrict__ stats, int k, double* __restrict__ out,
                                 long long opitch, long long oplane, int only_ring)
{
  if (stats != nullptr) time = stats[k].t;
  const int W = P.g.nx + 4, H = P.g.ny + 4;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < W * H; e += gridDim.x * blockDim.x) {
    const int i = e % W - 2, j = e / W - 2;
    const bool inside = i >= 0 && i < P.g.nx && j >= 0 && j < P.g.ny;
    if (only_ring && inside) continue;
    Cons c;
    if (inside || pr.ring_kind == RING_NONE) c = load_cell(P, u, i, j);
    else c = exact_ghost(P, pr, u, i, j, time);
    const long long o = static_cast<long long>(j + 2) * opitch + (i + 2);
    out[o] = c.rho;
    out[o + oplane] = c.mx;
    out[o + 2 * oplane] = c.my;
    out[o + 3 * oplane] = c.E;
  }
}

// ---- host launchers ----------------------------------------------------------

inline int reduce_blocks(long long n, int nt)
{
  long long b = (n + nt - 1) / nt;
  if (b > 148 * 8) b = 148 * 8;
  return static_cast<int>(b < 1 ? 1 : b);
}

cudaError_t launch_state_reduce(const EcgFvParams& p, const double* u, int eq79, EcgStateStats* out, cudaStream_t s)
{
  constexpr int NT = 256;
  state_reduce_kernel<NT><<<reduce_blocks(static_cast<long long>(p.g.nx) * p.g.ny, NT), NT, 0, s>>>(p, u, eq79, out);
  return cudaGetLastError();
}

cudaError_t launch_ghost_box(const EcgFvParams& p, const EcgProblem& pr, const double* u, double time,
                             const EcgStepStats* stats, int k, double* out, long long opitch, long long oplane,
                             int only_ring, cudaStream_t s)
{
  const long long n = static_cast<long long>(p.g.nx + 4) * (p.g.ny + 4);
  ghost_box_kernel<<<reduce_blocks(n, 256), 256, 0, s>>>(p, pr, u, time, stats, k, out, opitch, oplane, only_ring);
  return cudaGetLastError();
}

cudaError_t launch_init_state(const EcgFvParams& p, const EcgProblem& pr, double* u, cudaStream_t s)
{
  const long long n = static_cast<long long>(p.g.nx) * p.g.ny;
  init_state_kernel<<<reduce_blocks(n, 256), 256, 0, s>>>(p, pr, u);
  return cudaGetLastError();
}

cudaError_t launch_init_stats(EcgStepStats* stats, int n, double t0, cudaStream_t s)
{
  init_stats_kernel<<<(n + 127) / 128, 128, 0, s>>>(stats, n, t0);
  return cudaGetLastError();
}

cudaError_t launch_init_state_stats(EcgStateStats* st, cudaStream_t s)
{
  init_state_stats_kernel<<<1, 1, 0, s>>>(st);
  return cudaGetLastError();
}

cudaError_t launch_seed_stats(EcgStepStats* stats, const EcgStateStats* st, cudaStream_t s)
{
  seed_stats_kernel<<<1, 1, 0, s>>>(stats, st);
  return cudaGetLastError();
}

}  // namespace ECG_NS
