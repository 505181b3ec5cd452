// Kernels of the IMEX T1/S2 BDLTV20 source-map step
// (imex/imex_source_map_step.hpp:300-616 and imex/imex_source_map_helpers.hpp):
// star update, face enthalpies, pressure-row right-hand side and matrix
// diagnostics, the matrix-free pressure operator, the Picard refresh and the
// conservative closeout.  Vectors are compact row-major (row = j*nx + i).
//
// Included by imex_exact.cu (-fmad=false) and imex_fast.cu (-fmad=true).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "ecg.h"
#include "ecg_internal.h"
#include "imex_internal.h"

namespace ECG_NS {

#include "ecg_device.cuh"

namespace imexk {

// Cell indices r = j * nx + i fit 32 bits in every kernel here: the step
// allocates the GMRES workspace, which rejects n >= 2^31 - 2^24 rows, before
// it launches any of them.  Cell coordinates therefore come from a 32-bit
// unsigned division.

constexpr double kInf = __builtin_huge_val();
constexpr double kLowest = -1.7976931348623157e308;
constexpr double kMax = 1.7976931348623157e308;

// Division in the state-update arithmetic: IEEE in the exact build; in the
// fast build (ECG_IMEX_FAST_DIV) the hardware reciprocal refined by one
// third-order step y (1 + e + e^2), e = 1 - b y (a few units in the last
// place), for divisors of magnitude in (1e-300, 1e300); IEEE otherwise.
__device__ __forceinline__ double qdiv(double a, double b)
{
#ifdef ECG_IMEX_FAST_DIV
  const double ab = fabs(b);
  if (ab < 1.0e300 && ab > 1.0e-300) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    const double e = fma(-b, y, 1.0);
    return a * fma(y, fma(e, e, e), y);
  }
#endif
  return a / b;
}

// to_primitive (core/state_primitives.hpp:103-111) with qdiv
__device__ __forceinline__ Prim to_prim_q(const Cons& c, double g)
{
  const double inv_rho = qdiv(1.0, c.rho);
  const double u = c.mx * inv_rho;
  const double v = c.my * inv_rho;
  const double kin = 0.5 * c.rho * (u * u + v * v);
  return Prim{c.rho, u, v, (g - 1.0) * (c.E - kin)};
}

__device__ __forceinline__ int wrapi(int i, int n)
{
  int r = i % n;
  return r < 0 ? r + n : r;
}
__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); }

// CoupledHostGrid::map_i / map_j (imex_source_map_helpers.hpp:79-93)
__device__ __forceinline__ int mi(const EcgImexMap& m, int i) { return m.px ? wrapi(i, m.nx) : clampi(i, m.nx); }
__device__ __forceinline__ int mj(const EcgImexMap& m, int j) { return m.py ? wrapi(j, m.ny) : clampi(j, m.ny); }

// source_map_index (imex_source_map_helpers.hpp:169-188): wrap or even reflection
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
__device__ __forceinline__ int prow(const EcgImexMap& m, int i, int j)
{
  return pmap(j, m.ny, m.py) * m.nx + pmap(i, m.nx, m.px);
}

__device__ __forceinline__ Cons star_at(const EcgImexMap& m, const double* __restrict__ S, int i, int j)
{
  const long long r = static_cast<long long>(mj(m, j)) * m.nx + mi(m, i);
  const long long n = static_cast<long long>(m.nx) * m.ny;
  return Cons{S[r], S[r + n], S[r + 2 * n], S[r + 3 * n]};
}

// source_map_state_at_physical_boundary (imex_source_map_helpers.hpp:98-115)
__device__ __forceinline__ Cons state_b(const EcgImexMap& m, const double* __restrict__ S, int i, int j)
{
  if (m.bubble) {
    if (!m.px && i < 0) return Cons{m.cst[0], m.cst[1], m.cst[2], m.cst[3]};
    const int ii = mi(m, i);
    if (!m.py && j < 0) {
      Cons c = star_at(m, S, ii, 0);
      c.my = -c.my;
      return c;
    }
    if (m.top_wall && !m.py && j >= m.ny) {
      Cons c = star_at(m, S, ii, m.ny - 1);
      c.my = -c.my;
      return c;
    }
    return star_at(m, S, ii, j);
  }
  return star_at(m, S, i, j);
}

// source_map_pressure_at_physical_boundary (imex_source_map_helpers.hpp:222-245)
__device__ __forceinline__ double p_b(const EcgImexMap& m, const double* __restrict__ p, int i, int j)
{
  if (m.bubble && !m.px && i < 0) return m.p_fixed;
  return p[prow(m, i, j)];
}

// source_map_lagged_momentum_at(_physical_boundary) (imex_source_map_helpers.hpp:293-320)
__device__ __forceinline__ void m_at(const EcgImexMap& m, const double* __restrict__ K, int i, int j, double& m0,
                                     double& m1)
{
  const long long r = static_cast<long long>(mj(m, j)) * m.nx + mi(m, i);
  m0 = K[r];
  m1 = K[r + static_cast<long long>(m.nx) * m.ny];
}
__device__ __forceinline__ void m_b(const EcgImexMap& m, const double* __restrict__ K, int i, int j, double& m0,
                                    double& m1)
{
  if (m.bubble) {
    if (!m.px && i < 0) {
      m0 = m.cst[1];
      m1 = m.cst[2];
      return;
    }
    const int ii = mi(m, i);
    if (!m.py && j < 0) {
      m_at(m, K, ii, 0, m0, m1);
      m1 = -m1;
      return;
    }
    if (m.top_wall && !m.py && j >= m.ny) {
      m_at(m, K, ii, m.ny - 1, m0, m1);
      m1 = -m1;
      return;
    }
  }
  m_at(m, K, i, j, m0, m1);
}

struct FaceOut {
  double h_hat, flux;
  int flags;  // bit0 guard, bit1 enthalpy inputs nonfinite, bit2 flux nonfinite
};

// source_map_face_flux_detail (imex_source_map_helpers.hpp:359-402) from the
// face's two boundary-mapped densities, pressures and normal lagged momenta
__device__ __forceinline__ FaceOut face_math(double gamma, double rho_l, double rho_r, double pl, double pr,
                                             double ql, double qr)
{
  const double gm1 = gamma - 1.0;
  const double hl = qdiv(gamma * pl, gm1 * rho_l);
  const double hr = qdiv(gamma * pr, gm1 * rho_r);
  const double den = ql + qr;
  const double scale = smax(smax(fabs(ql), fabs(qr)), 1.0);
  const int guard = fabs(den) <= 1.0e-14 * scale ? 1 : 0;
  const double h = guard ? 0.5 * (hl + hr) : qdiv(hl * ql + hr * qr, den);
  const double mh = 0.5 * (ql + qr);
  FaceOut o;
  o.h_hat = h;
  o.flux = h * mh;
  o.flags = guard | ((!isfinite(hl) || !isfinite(hr) || !isfinite(h) || !isfinite(ql) || !isfinite(qr)) ? 2 : 0) |
            (isfinite(o.flux) ? 0 : 4);
  return o;
}

// source_map_face_flux_detail of the face between cells (il, jl) and (ir, jr)
__device__ __forceinline__ FaceOut face_detail(const EcgImexMap& m, const double* __restrict__ S,
                                               const double* __restrict__ p, const double* __restrict__ K, int il,
                                               int jl, int ir, int jr, int axis)
{
  const Cons L = state_b(m, S, il, jl), R = state_b(m, S, ir, jr);
  double ml0, ml1, mr0, mr1;
  m_b(m, K, il, jl, ml0, ml1);
  m_b(m, K, ir, jr, mr0, mr1);
  const double pl = p_b(m, p, il, jl), pr = p_b(m, p, ir, jr);
  return face_math(m.gamma, L.rho, R.rho, pl, pr, axis == 0 ? ml0 : ml1, axis == 0 ? mr0 : mr1);
}

// ---- block reduction helpers ------------------------------------------------------

__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) { return a > b ? a : b; }
__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) { return a < b ? a : b; }

template <int NT>
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* sh)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = umax64(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < NT / 32; ++w) v = umax64(v, sh[w]);
  __syncthreads();
  return v;
}
template <int NT>
__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long* sh)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = umin64(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < NT / 32; ++w) v = umin64(v, sh[w]);
  __syncthreads();
  return v;
}
template <int NT>
__device__ __forceinline__ long long block_sum_i64(long long v, long long* sh)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < NT / 32; ++w) v += sh[w];
  __syncthreads();
  return v;
}
template <int NT>
__device__ __forceinline__ double block_sum_f64(double v, double* sh)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < NT / 32; ++w) v += sh[w];
  __syncthreads();
  return v;
}

struct Shared {
  unsigned long long u[32];
  long long l[32];
  double d[32];
};

#define ECG_RED_MAX(field, val)                                              \
  {                                                                          \
    const unsigned long long _v = block_max_u64<NT>((val), sh.u);            \
    if (threadIdx.x == 0) atomicMax(&(field), _v);                           \
  }
#define ECG_RED_MIN(field, val)                                              \
  {                                                                          \
    const unsigned long long _v = block_min_u64<NT>((val), sh.u);            \
    if (threadIdx.x == 0) atomicMin(&(field), _v);                           \
  }
#define ECG_RED_ADD_I(field, val)                                            \
  {                                                                          \
    const long long _v = block_sum_i64<NT>((val), sh.l);                     \
    if (threadIdx.x == 0 && _v) atomicAdd(&(field), static_cast<unsigned long long>(_v)); \
  }
#define ECG_RED_ADD_D(field, val)                                            \
  {                                                                          \
    const double _v = block_sum_f64<NT>((val), sh.d);                        \
    if (threadIdx.x == 0) atomicAdd(&(field), _v);                           \
  }

// ---- star update -----------------------------------------------------------------

// Conserved-minmod reconstruction of cell c0 to side h (BDLTV20 eq 87-89),
// reconstruction_fluxes.hpp:26-52.
__device__ __forceinline__ Prim recon_cmm(const Cons& um, const Cons& u, const Cons& up, double h, double g)
{
  const Cons s{minmod(u.rho - um.rho, up.rho - u.rho), minmod(u.mx - um.mx, up.mx - u.mx),
               minmod(u.my - um.my, up.my - u.my), minmod(u.E - um.E, up.E - u.E)};
  return to_prim_q(Cons{u.rho + h * s.rho, u.mx + h * s.mx, u.my + h * s.my, u.E + h * s.E}, g);
}

// bdltv20_pressure_split_lf_flux with material speed, reconstruction_fluxes.hpp:462-484,504-515
__device__ __forceinline__ Cons split_lf(const Prim& l, const Prim& r, int axis, double g)
{
  const Cons ul = to_cons(l, g), ur = to_cons(r, g);
  const double lmx = l.rho * l.u, lmy = l.rho * l.v, lk = 0.5 * l.rho * (l.u * l.u + l.v * l.v);
  const double rmx = r.rho * r.u, rmy = r.rho * r.v, rk = 0.5 * r.rho * (r.u * r.u + r.v * r.v);
  Cons fl, fr;
  if (axis == 0) {
    fl = Cons{lmx, lmx * l.u, lmy * l.u, lk * l.u};
    fr = Cons{rmx, rmx * r.u, rmy * r.u, rk * r.u};
  } else {
    fl = Cons{lmy, lmx * l.v, lmy * l.v, lk * l.v};
    fr = Cons{rmy, rmx * r.v, rmy * r.v, rk * r.v};
  }
  const double sm = smax(fabs(normal_vel(l, axis)), fabs(normal_vel(r, axis)));
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
              0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// Ghost-aware conserved state of the old state (IMEX ghost policy).
__device__ __forceinline__ Cons old_cell(const EcgFvParams& P, const double* __restrict__ u, int i, int j);

// compute_bdltv20_pressure_split_star (imex_source_map_helpers.hpp:2-68) with
// the step's initialisation fused in: p0 = pressure of U^n
// (imex_source_map_step.hpp:422-434), K0 = star momentum (:418), the density
// floor check (:436-451) and the star pressure mismatch (:278-298,453-454).
constexpr int SX = 32, SY = 8;              // cells of a star tile
constexpr int SHX = SX + 4, SHY = SY + 4;   // staged old state: columns c0-2 .. c0+SX+1, rows j0-2 .. j0+SY+1
template <int NT>
__global__ void __launch_bounds__(NT) imex_star_kernel(const EcgFvParams P, const double* __restrict__ u,
                                                       const double dt, double* __restrict__ S, double* __restrict__ p,
                                                       double* __restrict__ K, EcgImexStats* __restrict__ st)
{
  static_assert(NT == SX * SY, "one thread per cell of the tile");
  __shared__ Shared sh;
  // A block takes a tile of SX x SY cells: the old state of the tile and a
  // two-cell ring (the IMEX ghost policy applied once per cell), then each
  // x- and y-face flux of the tile once (the per-cell form evaluates every
  // face twice), then the update of its cells.
  __shared__ double us[4][SHY][SHX];
  __shared__ double fxs[4][SY][SX + 1];
  __shared__ double fys[4][SY + 1][SX];
  const int nx = P.g.nx, ny = P.g.ny;
  const long long n = static_cast<long long>(nx) * ny;
  const double g = P.gamma, idx = P.g.inv_dx, idy = P.g.inv_dy;
  const int c0 = blockIdx.x * SX, j0 = blockIdx.y * SY;
  for (int e = threadIdx.x; e < SHX * SHY; e += NT) {
    const int ex = e % SHX, ey = e / SHX;
    const Cons c = old_cell(P, u, c0 - 2 + ex, j0 - 2 + ey);
    us[0][ey][ex] = c.rho;
    us[1][ey][ex] = c.mx;
    us[2][ey][ex] = c.my;
    us[3][ey][ex] = c.E;
  }
  __syncthreads();
  auto cell = [&](int ex, int ey) { return Cons{us[0][ey][ex], us[1][ey][ex], us[2][ey][ex], us[3][ey][ex]}; };
  // x-face f of row y lies between staged cells (f + 1, y + 2) and (f + 2, y + 2)
  for (int e = threadIdx.x; e < SY * (SX + 1); e += NT) {
    const int f = e % (SX + 1), y = e / (SX + 1);
    const int ey = y + 2;
    const Cons a = cell(f, ey), b = cell(f + 1, ey), c = cell(f + 2, ey), d = cell(f + 3, ey);
    const Cons fl = split_lf(recon_cmm(a, b, c, 0.5, g), recon_cmm(b, c, d, -0.5, g), 0, g);
    fxs[0][y][f] = fl.rho;
    fxs[1][y][f] = fl.mx;
    fxs[2][y][f] = fl.my;
    fxs[3][y][f] = fl.E;
  }
  // y-face f of column x lies between staged cells (x + 2, f + 1) and (x + 2, f + 2)
  for (int e = threadIdx.x; e < (SY + 1) * SX; e += NT) {
    const int x = e % SX, f = e / SX;
    const int ex = x + 2;
    const Cons a = cell(ex, f), b = cell(ex, f + 1), c = cell(ex, f + 2), d = cell(ex, f + 3);
    const Cons fl = split_lf(recon_cmm(a, b, c, 0.5, g), recon_cmm(b, c, d, -0.5, g), 1, g);
    fys[0][f][x] = fl.rho;
    fys[1][f][x] = fl.mx;
    fys[2][f][x] = fl.my;
    fys[3][f][x] = fl.E;
  }
  __syncthreads();
  long long floor_count = 0, knf = 0;
  unsigned long long rho_min = okey(kInf), mis = okey(0.0);
  long long mis_nf = 0;
  const int tx = threadIdx.x % SX, ty = threadIdx.x / SX;
  const int i = c0 + tx, j = j0 + ty;
  if (i < nx && j < ny) {
    const long long r = static_cast<long long>(j) * nx + i;
    const Cons c = cell(tx + 2, ty + 2);
    const Cons up{c.rho - dt * ((fxs[0][ty][tx + 1] - fxs[0][ty][tx]) * idx + (fys[0][ty + 1][tx] - fys[0][ty][tx]) * idy),
                  c.mx - dt * ((fxs[1][ty][tx + 1] - fxs[1][ty][tx]) * idx + (fys[1][ty + 1][tx] - fys[1][ty][tx]) * idy),
                  c.my - dt * ((fxs[2][ty][tx + 1] - fxs[2][ty][tx]) * idx + (fys[2][ty + 1][tx] - fys[2][ty][tx]) * idy),
                  c.E - dt * ((fxs[3][ty][tx + 1] - fxs[3][ty][tx]) * idx + (fys[3][ty + 1][tx] - fys[3][ty][tx]) * idy)};
    S[r] = up.rho;
    S[r + n] = up.mx;
    S[r + 2 * n] = up.my;
    S[r + 3 * n] = up.E;
    K[r] = up.mx;
    K[r + n] = up.my;
    const double p0 = to_prim_q(c, g).p;
    p[r] = p0;
    if (!isfinite(up.mx) || !isfinite(up.my)) ++knf;
    if (!isfinite(up.rho) || up.rho <= 1.0e-14) ++floor_count;
    if (isfinite(up.rho)) rho_min = umin64(rho_min, okey(up.rho));
    const double kin = qdiv(0.5 * (up.mx * up.mx + up.my * up.my), up.rho);
    const double pe = (g - 1.0) * (up.E - kin);
    if (!isfinite(pe) || !isfinite(p0)) ++mis_nf;
    else mis = umax64(mis, okey(fabs(p0 - pe)));
  }
  ECG_RED_ADD_I(st->floor_count, floor_count);
  ECG_RED_ADD_I(st->k_nonfinite, knf);
  ECG_RED_MIN(st->trial_rho_min_key, rho_min);
  ECG_RED_MAX(st->mismatch_before_key, mis);
  ECG_RED_ADD_I(st->mismatch_before_nonfinite, mis_nf);
}

// ---- faces ------------------------------------------------------------------------

// Face enthalpies h_hat (mode 0) or energy fluxes h_hat * m_hat (mode 1) of
// every x-face (nx+1 per row) and y-face (ny+1 per column).  Thread c of row
// j takes x-face (c, j) and y-face (c, j), which share the cell (c, j); rows
// stride over grid.y, so no face index is divided.
// A queued phase of a step whose earlier phase failed does nothing (the
// flag was written before the launch, so every thread reads the same value).
__device__ __forceinline__ bool gated_off(const EcgImexMap& m) { return m.abort && __ldcg(m.abort) != 0; }

template <int NT>
__global__ void __launch_bounds__(NT) imex_face_kernel(const EcgImexMap m, const double* __restrict__ S,
                                                       const double* __restrict__ p, const double* __restrict__ K,
                                                       double* __restrict__ fxv, double* __restrict__ fyv,
                                                       unsigned char* __restrict__ fxf, unsigned char* __restrict__ fyf,
                                                       const int mode)
{
  if (gated_off(m)) return;
  const int c = blockIdx.x * NT + threadIdx.x;
  if (c > m.nx) return;
  for (int j = blockIdx.y; j <= m.ny; j += gridDim.y) {
    if (j < m.ny) {
      const long long f = static_cast<long long>(j) * (m.nx + 1) + c;
      const FaceOut o = face_detail(m, S, p, K, c - 1, j, c, j, 0);
      fxv[f] = mode ? o.flux : o.h_hat;
      if (fxf) fxf[f] = static_cast<unsigned char>(o.flags);
    }
    if (c < m.nx) {
      const long long g = static_cast<long long>(j) * m.nx + c;
      const FaceOut o = face_detail(m, S, p, K, c, j - 1, c, j, 1);
      fyv[g] = mode ? o.flux : o.h_hat;
      if (fyf) fyf[g] = static_cast<unsigned char>(o.flags);
    }
  }
}

// ---- pressure rows -------------------------------------------------------------------

struct RowTerms {
  int n;
  int col[11];
  double val[11];
};

// The eleven lhs terms of source_map_pressure_row_data
// (imex_source_map_helpers.hpp:533-543) with boundary-mapped columns; terms
// whose column is a fixed (Dirichlet) pressure are left out (they go to the
// rhs).  Then zero terms are dropped, duplicate columns summed in insertion
// order and the entries sorted by column, as setFromTriplets stores the row
// (imex_source_map_step.hpp:20-36).
__device__ __forceinline__ void row_terms(const EcgImexMap& m, const double* __restrict__ hx,
                                          const double* __restrict__ hy, double xc, double yc, int i, int j,
                                          RowTerms& t)
{
  const double he = hx[static_cast<long long>(j) * (m.nx + 1) + i + 1];
  const double hw = hx[static_cast<long long>(j) * (m.nx + 1) + i];
  const double hn = hy[static_cast<long long>(j + 1) * m.nx + i];
  const double hs = hy[static_cast<long long>(j) * m.nx + i];
  const int ci[11] = {i, i + 2, i + 1, i, i - 1, i - 2, i, i, i, i, i};
  const int cj[11] = {j, j, j, j, j, j, j + 2, j + 1, j, j - 1, j - 2};
  const double cv[11] = {1.0 / (m.gamma - 1.0), -xc * he, -xc * (he - hw), xc * (he + hw), xc * (he - hw),
                         -xc * hw, -yc * hn, -yc * (hn - hs), yc * (hn + hs), yc * (hn - hs), -yc * hs};
  t.n = 0;
  for (int q = 0; q < 11; ++q) {
    if (m.bubble && !m.px && ci[q] < 0) continue;
    if (cv[q] == 0.0) continue;
    const int c = prow(m, ci[q], cj[q]);
    int found = -1;
    for (int s = 0; s < t.n; ++s)
      if (t.col[s] == c) found = s;
    if (found >= 0) {
      t.val[found] = t.val[found] + cv[q];
    } else {
      t.col[t.n] = c;
      t.val[t.n] = cv[q];
      ++t.n;
    }
  }
  for (int a = 1; a < t.n; ++a) {  // insertion sort by column
    const int c = t.col[a];
    const double v = t.val[a];
    int b = a - 1;
    while (b >= 0 && t.col[b] > c) {
      t.col[b + 1] = t.col[b];
      t.val[b + 1] = t.val[b];
      --b;
    }
    t.col[b + 1] = c;
    t.val[b + 1] = v;
  }
}

// The cell values a pressure row reads (boundary-mapped as
// source_map_state_at_physical_boundary and the lagged-momentum lookup map
// them): its star state and lagged momentum, the x-momentum of its east and
// west neighbours and the y-momentum of its north and south neighbours.
struct RowData {
  double rho, mx, my, E, k0, k1, mx_e, mx_w, my_n, my_s;
};

// Right-hand side of row (i, j) of source_map_pressure_row_data
// (imex_source_map_helpers.hpp:488-570) from the row's four face enthalpies;
// rnf counts its nonfinite terms.
__device__ __forceinline__ double rhs_math(const EcgImexMap& m, const RowData& d, double he, double hw, double hn,
                                           double hs, int i, double dt, double idx, double idy, double xc, double yc,
                                           int& rnf)
{
  const double gm1 = m.gamma - 1.0;
  rnf = 0;
  double b = 0.0;
  if (!isfinite(he) || !isfinite(hw) || !isfinite(hn) || !isfinite(hs)) ++rnf;
  {
    const int ci[11] = {i, i + 2, i + 1, i, i - 1, i - 2, i, i, i, i, i};
    const double cv[11] = {1.0 / gm1, -xc * he, -xc * (he - hw), xc * (he + hw), xc * (he - hw),
                           -xc * hw, -yc * hn, -yc * (hn - hs), yc * (hn + hs), yc * (hn - hs), -yc * hs};
#pragma unroll
    for (int q = 0; q < 11; ++q) {
      if (m.bubble && !m.px && ci[q] < 0) {
        const double c = -cv[q] * m.p_fixed;
        b += c;
        if (!isfinite(c)) ++rnf;
      } else if (!isfinite(cv[q])) {
        ++rnf;
      }
    }
  }
  const double kin = qdiv(0.5 * (d.k0 * d.k0 + d.k1 * d.k1), d.rho);
  double v;
  v = d.E;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = -kin;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = -0.5 * dt * idx * he * d.mx_e;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = -0.5 * dt * idx * (he - hw) * d.mx;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = 0.5 * dt * idx * hw * d.mx_w;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = -0.5 * dt * idy * hn * d.my_n;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = -0.5 * dt * idy * (hn - hs) * d.my;
  if (!isfinite(v)) ++rnf;
  b += v;
  v = 0.5 * dt * idy * hs * d.my_s;
  if (!isfinite(v)) ++rnf;
  b += v;
  if (!isfinite(b)) ++rnf;
  return b;
}

// The assembly of one Picard pass in one kernel: the eq46 face enthalpies
// (imex_face_kernel, mode 0) and the right-hand side of
// source_map_pressure_row_data (imex_source_map_helpers.hpp:488-570) with its
// nonfinite count.  A block takes a tile of AX columns x AY rows of cells.
// It first stages, for the tile and a one-cell ring around it, every value
// its faces and rows read, boundary-mapped once per cell (star density,
// momenta and energy, pressure, lagged momentum): coalesced loads, the maps
// evaluated once.  Every thread then evaluates the x-face on its cell's left
// and the y-face below it from shared memory; the tile's right x-faces and
// top y-faces are evaluated once more by 40 threads (they belong to the
// neighbour tiles, which store them), and the rows' right-hand sides read all
// four faces from shared memory.  Tiles run over the face columns 0 .. nx
// and rows 0 .. ny.
constexpr int AX = 32, AY = 8;
constexpr int HX = AX + 2, HY = AY + 2;  // staged cells: columns c0-1 .. c0+AX, rows j0-1 .. j0+AY
template <int NT>
__global__ void __launch_bounds__(NT) imex_assemble_kernel(const EcgImexMap m, const double* __restrict__ S,
                                                           const double* __restrict__ p, const double* __restrict__ K,
                                                           double* __restrict__ hx, double* __restrict__ hy,
                                                           const double dt, const double idx, const double idy,
                                                           double* __restrict__ rhs, EcgImexStats* __restrict__ st)
{
  static_assert(NT == AX * AY, "one thread per cell of the tile");
  if (gated_off(m)) return;
  __shared__ Shared sh;
  __shared__ double fx[AY][AX + 1];
  __shared__ double fy[AY + 1][AX];
  __shared__ double t_rho[HY][HX], t_mx[HY][HX], t_my[HY][HX], t_e[HY][HX], t_p[HY][HX], t_k0[HY][HX],
      t_k1[HY][HX];
  const int tx = threadIdx.x % AX, ty = threadIdx.x / AX;
  const int c0 = blockIdx.x * AX, j0 = blockIdx.y * AY;
  const int i = c0 + tx, j = j0 + ty;
  const int nx = m.nx, ny = m.ny;
  for (int e = threadIdx.x; e < HX * HY; e += NT) {
    const int ex = e % HX, ey = e / HX;
    const int ci = c0 - 1 + ex, cj = j0 - 1 + ey;
    const Cons c = state_b(m, S, ci, cj);
    double k0, k1;
    m_b(m, K, ci, cj, k0, k1);
    t_rho[ey][ex] = c.rho;
    t_mx[ey][ex] = c.mx;
    t_my[ey][ex] = c.my;
    t_e[ey][ex] = c.E;
    t_p[ey][ex] = p_b(m, p, ci, cj);
    t_k0[ey][ex] = k0;
    t_k1[ey][ex] = k1;
  }
  __syncthreads();
  // the face between staged cells (ax, ay) and (bx, by)
  auto face = [&](int ax, int ay, int bx, int by, int axis) {
    const double ql = axis == 0 ? t_k0[ay][ax] : t_k1[ay][ax];
    const double qr = axis == 0 ? t_k0[by][bx] : t_k1[by][bx];
    return face_math(m.gamma, t_rho[ay][ax], t_rho[by][bx], t_p[ay][ax], t_p[by][bx], ql, qr).h_hat;
  };
  // the faces of the tile's own cells (and the domain's last face column/row)
  if (j < ny && i <= nx) {
    const double h = face(tx, ty + 1, tx + 1, ty + 1, 0);
    hx[static_cast<long long>(j) * (nx + 1) + i] = h;
    fx[ty][tx] = h;
  }
  if (i < nx && j <= ny) {
    const double h = face(tx + 1, ty, tx + 1, ty + 1, 1);
    hy[static_cast<long long>(j) * nx + i] = h;
    fy[ty][tx] = h;
  }
  // the neighbour tiles' faces the tile's rows also need: column c0 + AX of
  // x-faces (threads 0 .. AY-1), row j0 + AY of y-faces (threads 32 .. 63)
  if (threadIdx.x < AY) {
    const int jj = j0 + threadIdx.x, ii = c0 + AX;
    if (jj < ny && ii <= nx) fx[threadIdx.x][AX] = face(AX, threadIdx.x + 1, AX + 1, threadIdx.x + 1, 0);
  } else if (threadIdx.x >= 32 && threadIdx.x < 32 + AX) {
    const int xx = threadIdx.x - 32;
    const int ii = c0 + xx, jj = j0 + AY;
    if (ii < nx && jj <= ny) fy[AY][xx] = face(xx + 1, AY, xx + 1, AY + 1, 1);
  }
  __syncthreads();
  long long nonfinite = 0;
  unsigned long long bmax = okey(0.0);
  if (i < nx && j < ny) {
    const double xc = 0.25 * dt * dt * idx * idx, yc = 0.25 * dt * dt * idy * idy;
    const int sx = tx + 1, sy = ty + 1;
    const RowData d{t_rho[sy][sx], t_mx[sy][sx],     t_my[sy][sx],     t_e[sy][sx],      t_k0[sy][sx],
                    t_k1[sy][sx],  t_mx[sy][sx + 1], t_mx[sy][sx - 1], t_my[sy + 1][sx], t_my[sy - 1][sx]};
    int rnf;
    const double b = rhs_math(m, d, fx[ty][tx + 1], fx[ty][tx], fy[ty + 1][tx], fy[ty][tx], i, dt, idx, idy, xc, yc,
                              rnf);
    rhs[static_cast<long long>(j) * nx + i] = b;
    nonfinite = rnf;
    bmax = isfinite(b) ? okey(fabs(b)) : okey(kInf);
  }
  ECG_RED_ADD_I(st->row_nonfinite, nonfinite);
  ECG_RED_MAX(st->rhs_linf_key, bmax);
}

// ---- matrix diagnostics of the Picard loop (imex_source_map_step.hpp:466-489) ----------------
// Stored entries, widest row, largest |a_ij| and max |A - A^T| of the pressure
// matrix as setFromTriplets stores it (row_terms).  They are reported for the
// Picard pass that ends the step, so the step computes them once, there.

__device__ __forceinline__ bool interior_row(const EcgImexMap& m, int i, int j)
{
  return (m.px ? m.nx >= 5 : (i >= 2 && i <= m.nx - 3)) && (m.py ? m.ny >= 5 : (j >= 2 && j <= m.ny - 3));
}

__device__ __forceinline__ double nanmax_d(double a, double v) { return (a < v || v != v) ? v : a; }

// Rows away from the walls: no two columns of the row coincide and column r
// appears once in each neighbour row (the reflection and the fixed bubble
// columns only touch rows within two cells of a wall), so the stored entries
// are the raw terms and the transposed entry of each is the neighbour's raw
// term.  Maxima are kept in FP64 (NaN wins) and keyed once per thread.
template <int NT>
__global__ void __launch_bounds__(NT) imex_matrix_interior_kernel(const EcgImexMap m, const double* __restrict__ hx,
                                                                  const double* __restrict__ hy, const double xc,
                                                                  const double yc, EcgImexStats* __restrict__ st)
{
  __shared__ Shared sh;
  const int nx = m.nx, n = m.nx * m.ny;
  const double gi = 1.0 / (m.gamma - 1.0);
  long long nnz = 0;
  unsigned long long width = 0;
  double amax = 0.0, sym = 0.0;
  for (int r = blockIdx.x * NT + threadIdx.x; r < n; r += gridDim.x * NT) {
    const int j = r / nx, i = r - j * nx;
    if (!interior_row(m, i, j)) continue;
    const int hr = j * (nx + 1);
    const double he = hx[hr + i + 1], hw = hx[hr + i];
    const double hn = hy[(j + 1) * nx + i], hs = hy[j * nx + i];
    const int ie2 = pmap(i + 2, nx, m.px), ie1 = pmap(i + 1, nx, m.px);
    const int iw1 = pmap(i - 1, nx, m.px), iw2 = pmap(i - 2, nx, m.px);
    const int jn2 = pmap(j + 2, m.ny, m.py), jn1 = pmap(j + 1, m.ny, m.py);
    const int js1 = pmap(j - 1, m.ny, m.py), js2 = pmap(j - 2, m.ny, m.py);
    const double d = (gi + xc * (he + hw)) + yc * (hn + hs);
    const double a[8] = {-xc * he, -xc * (he - hw), xc * (he - hw), -xc * hw,
                         -yc * hn, -yc * (hn - hs), yc * (hn - hs), -yc * hs};
    const double tr[8] = {-xc * hx[hr + ie2],
                          xc * (hx[hr + ie1 + 1] - hx[hr + ie1]),
                          -xc * (hx[hr + iw1 + 1] - hx[hr + iw1]),
                          -xc * hx[hr + iw2 + 1],
                          -yc * hy[jn2 * nx + i],
                          yc * (hy[(jn1 + 1) * nx + i] - hy[jn1 * nx + i]),
                          -yc * (hy[(js1 + 1) * nx + i] - hy[js1 * nx + i]),
                          -yc * hy[(js2 + 1) * nx + i]};
    int cnt = d != 0.0 ? 1 : 0;
    amax = nanmax_d(amax, fabs(d));
    sym = nanmax_d(sym, fabs(d - d));
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      cnt += a[q] != 0.0 ? 1 : 0;
      amax = nanmax_d(amax, fabs(a[q]));
      sym = nanmax_d(sym, fabs(a[q] - tr[q]));
    }
    nnz += cnt;
    width = umax64(width, static_cast<unsigned long long>(cnt));
  }
  ECG_RED_ADD_I(st->nnz, nnz);
  ECG_RED_MAX(st->max_row_width, width);
  ECG_RED_MAX(st->abs_max_key, okey(amax));
  ECG_RED_MAX(st->sym_key, okey(sym));
}

// The eleven lhs terms of row (i, j) in insertion order (row_terms before the
// merge): column and value, and whether the term is left out (a fixed bubble
// column, or a zero value).
struct RowRaw {
  int col[11];
  double val[11];
  bool out[11];
};
__device__ __forceinline__ void row_raw(const EcgImexMap& m, const double* __restrict__ hx, const double* __restrict__ hy,
                                        double xc, double yc, int i, int j, RowRaw& t)
{
  const double he = hx[j * (m.nx + 1) + i + 1], hw = hx[j * (m.nx + 1) + i];
  const double hn = hy[(j + 1) * m.nx + i], hs = hy[j * m.nx + i];
  const int ci[11] = {i, i + 2, i + 1, i, i - 1, i - 2, i, i, i, i, i};
  const int cj[11] = {j, j, j, j, j, j, j + 2, j + 1, j, j - 1, j - 2};
  const double cv[11] = {1.0 / (m.gamma - 1.0), -xc * he, -xc * (he - hw), xc * (he + hw), xc * (he - hw),
                         -xc * hw, -yc * hn, -yc * (hn - hs), yc * (hn + hs), yc * (hn - hs), -yc * hs};
#pragma unroll
  for (int q = 0; q < 11; ++q) {
    t.out[q] = (m.bubble && !m.px && ci[q] < 0) || cv[q] == 0.0;
    t.col[q] = prow(m, ci[q], cj[q]);
    t.val[q] = cv[q];
  }
}

// Stored value of row (i, j) at column c (duplicates summed in insertion
// order, as setFromTriplets does); false when the row stores nothing there.
__device__ __forceinline__ bool row_entry(const EcgImexMap& m, const double* __restrict__ hx,
                                          const double* __restrict__ hy, double xc, double yc, int i, int j, int c,
                                          double& v)
{
  RowRaw t;
  row_raw(m, hx, hy, xc, yc, i, j, t);
  bool found = false;
  v = 0.0;
#pragma unroll
  for (int q = 0; q < 11; ++q)
    if (!t.out[q] && t.col[q] == c) {
      v = found ? v + t.val[q] : t.val[q];
      found = true;
    }
  return found;
}

// Rows within two cells of a wall (every row when a periodic axis has fewer
// than five cells): the merged row and, for each stored entry, the stored
// entry of the transposed row; all in registers.  Threads walk the ring of
// such rows only: x-edge columns of every row, then the y-edge rows' other
// columns.
template <int NT>
__global__ void __launch_bounds__(NT) imex_matrix_edge_kernel(const EcgImexMap m, const double* __restrict__ hx,
                                                              const double* __restrict__ hy, const double xc,
                                                              const double yc, EcgImexStats* __restrict__ st)
{
  __shared__ Shared sh;
  const int nx = m.nx, ny = m.ny;
  const bool all = (m.px && nx < 5) || (m.py && ny < 5);
  const int xcnt = m.px ? 0 : (nx >= 5 ? 4 : nx), ycnt = m.py ? 0 : (ny >= 5 ? 4 : ny);
  const int inner = nx - xcnt;  // columns outside the x ring
  const int slots = all ? nx * ny : xcnt * ny + inner * ycnt;
  long long nnz = 0;
  unsigned long long width = 0;
  double amax = 0.0, sym = 0.0;
  for (int t = blockIdx.x * NT + threadIdx.x; t < slots; t += gridDim.x * NT) {
    int i, j;
    if (all) {
      j = t / nx;
      i = t - j * nx;
    } else if (t < xcnt * ny) {
      j = t / xcnt;
      const int k = t - j * xcnt;
      i = xcnt == nx ? k : (k < 2 ? k : nx - 4 + k);
    } else {
      const int u = t - xcnt * ny;
      const int kr = inner > 0 ? u / inner : 0;
      i = (xcnt == 0 ? 0 : 2) + (u - kr * inner);
      j = ycnt == ny ? kr : (kr < 2 ? kr : ny - 4 + kr);
    }
    const int r = j * nx + i;
    RowRaw a;
    row_raw(m, hx, hy, xc, yc, i, j, a);
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < 11; ++q) {
      if (a.out[q]) continue;
      bool first = true;
#pragma unroll
      for (int p = 0; p < q; ++p)
        if (!a.out[p] && a.col[p] == a.col[q]) first = false;
      if (!first) continue;
      ++cnt;
      double v = a.val[q];  // merged value: the later duplicates, in order
#pragma unroll
      for (int p = q + 1; p < 11; ++p)
        if (!a.out[p] && a.col[p] == a.col[q]) v = v + a.val[p];
      amax = nanmax_d(amax, fabs(v));
      const int c = a.col[q];
      double tv;
      if (!row_entry(m, hx, hy, xc, yc, c % nx, c / nx, r, tv)) tv = 0.0;
      sym = nanmax_d(sym, fabs(v - tv));
    }
    nnz += cnt;
    width = umax64(width, static_cast<unsigned long long>(cnt));
  }
  ECG_RED_ADD_I(st->nnz, nnz);
  ECG_RED_MAX(st->max_row_width, width);
  ECG_RED_MAX(st->abs_max_key, okey(amax));
  ECG_RED_MAX(st->sym_key, okey(sym));
}

// ---- p update and eq54 momentum -----------------------------------------------------------

// The end of a Picard pass in one sweep: p <- x with the Picard delta
// statistics (imex_source_map_step.hpp:536-547), and the
// source_map_eq54_corrected_momentum_field with the physical-boundary
// pressure (imex_source_map_helpers.hpp:249-268,334-346) and its nonfinite
// count (:348-357), taken from x.  x is not copied into p: the caller swaps
// the two buffers, so x becomes the pass's pressure.
template <int NT>
__global__ void __launch_bounds__(NT) imex_refresh_kernel(const EcgImexMap m, const double* __restrict__ p_old,
                                                          const double* __restrict__ x, const double* __restrict__ S,
                                                          const double dt, const double idx, const double idy,
                                                          double* __restrict__ K, EcgImexStats* __restrict__ st)
{
  if (gated_off(m)) return;
  __shared__ Shared sh;
  const long long n = static_cast<long long>(m.nx) * m.ny;
  unsigned long long dl = okey(0.0), pm = okey(1.0);
  double d2 = 0.0;
  long long nf = 0;
  for (long long r = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; r < n;
       r += static_cast<long long>(gridDim.x) * NT) {
    const double o = p_old[r], nv = x[r];
    const double d = nv - o;
    dl = umax64(dl, okey(fabs(d)));
    d2 += d * d;
    pm = umax64(pm, umax64(okey(fabs(o)), okey(fabs(nv))));
    const int j = static_cast<int>(static_cast<unsigned>(r) / static_cast<unsigned>(m.nx)), i = static_cast<int>(r) - j * m.nx;
    const double gx = 0.5 * (p_b(m, x, i + 1, j) - p_b(m, x, i - 1, j)) * idx;
    const double gy = 0.5 * (p_b(m, x, i, j + 1) - p_b(m, x, i, j - 1)) * idy;
    const double k0 = S[r + n] - dt * gx, k1 = S[r + 2 * n] - dt * gy;
    K[r] = k0;
    K[r + n] = k1;
    if (!isfinite(k0) || !isfinite(k1)) ++nf;
  }
  ECG_RED_MAX(st->delta_linf_key, dl);
  ECG_RED_ADD_D(st->delta_l2_sum, d2);
  ECG_RED_MAX(st->pmax_key, pm);
  ECG_RED_ADD_I(st->k_nonfinite, nf);
}

// ---- closeout ------------------------------------------------------------------------

// evaluate_source_map_final (imex_source_map_step.hpp:75-188): the
// conservative enthalpy-flux energy closeout and its statistics.  Writes the
// candidate state U^{n+1} = (rho*, K, E) into `out` (pitched state layout).
template <int NT>
__global__ void __launch_bounds__(NT) imex_closeout_kernel(const EcgImexMap m, const EcgGrid G,
                                                           const double* __restrict__ S, const double* __restrict__ p,
                                                           const double* __restrict__ K, const double* __restrict__ fx,
                                                           const double* __restrict__ fy,
                                                           const unsigned char* __restrict__ fxf,
                                                           const unsigned char* __restrict__ fyf, const double dt,
                                                           double* __restrict__ out, EcgImexStats* __restrict__ st)
{
  if (gated_off(m)) return;
  __shared__ Shared sh;
  const long long n = static_cast<long long>(m.nx) * m.ny;
  const double gm1 = m.gamma - 1.0, idx = G.inv_dx, idy = G.inv_dy;
  long long guard = 0, hnf = 0, fnf = 0, nfc = 0, dfail = 0, pfail = 0, ifail = 0, rcount = 0;
  unsigned long long flinf = okey(0.0);
  unsigned long long dmin = okey(kInf), spmin = okey(kInf), spmax = okey(-kInf), epmin = okey(kInf),
                     epmax = okey(-kInf), iemin = okey(kInf), iemax = okey(-kInf);
  unsigned long long mcl = okey(0.0), ecl = okey(0.0), fdl = okey(0.0), rl = okey(0.0), rrel = okey(0.0),
                     ml = okey(0.0), mrel = okey(0.0);
  double rsum = 0.0, msum = 0.0, esum = 0.0;
  for (long long r = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; r < n;
       r += static_cast<long long>(gridDim.x) * NT) {
    const int j = static_cast<int>(static_cast<unsigned>(r) / static_cast<unsigned>(m.nx)), i = static_cast<int>(r) - j * m.nx;
    const long long xe = static_cast<long long>(j) * (m.nx + 1) + i + 1, xw = xe - 1;
    const long long yn = static_cast<long long>(j + 1) * m.nx + i, ys = static_cast<long long>(j) * m.nx + i;
    const double fe = fx[xe], fw = fx[xw], fn = fy[yn], fs = fy[ys];
    const int fl[4] = {fxf[xe], fxf[xw], fyf[yn], fyf[ys]};
    const double fv[4] = {fe, fw, fn, fs};
    unsigned long long cfl = okey(0.0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      guard += fl[q] & 1;
      hnf += (fl[q] >> 1) & 1;
      if (fl[q] & 4) ++fnf;
      else cfl = umax64(cfl, okey(fabs(fv[q])));
    }
    flinf = umax64(flinf, cfl);
    const Cons s{S[r], S[r + n], S[r + 2 * n], S[r + 3 * n]};
    const double m0 = K[r], m1 = K[r + n];
    const double pr = p[r];
    const double div = (fe - fw) * idx + (fn - fs) * idy;
    const double en = s.E - dt * div;
    const double kin = qdiv(0.5 * (m0 * m0 + m1 * m1), s.rho);
    const double ie = en - kin;
    const double pe = gm1 * ie;
    const double res = pr / gm1 - en + kin;
    const double mis = pr - pe;
    const double rs = smax(smax(smax(fabs(pr) / gm1, fabs(en)), fabs(kin)), 1.0);
    const double ms = smax(smax(smax(fabs(pr), fabs(pe)), fabs(kin)), 1.0);
    const long long o = static_cast<long long>(j) * G.pitch + i;
    out[o] = s.rho;
    out[o + G.plane] = m0;
    out[o + 2 * G.plane] = m1;
    out[o + 3 * G.plane] = en;
    const bool nfb = !isfinite(s.rho) || !isfinite(m0) || !isfinite(m1) || !isfinite(en) || !isfinite(pr) ||
                     !isfinite(kin) || !isfinite(ie) || !isfinite(pe) || !isfinite(res) || !isfinite(div);
    if (nfb) {
      ++nfc;
      continue;
    }
    dmin = umin64(dmin, okey(s.rho));
    spmin = umin64(spmin, okey(pr));
    spmax = umax64(spmax, okey(pr));
    epmin = umin64(epmin, okey(pe));
    epmax = umax64(epmax, okey(pe));
    iemin = umin64(iemin, okey(ie));
    iemax = umax64(iemax, okey(ie));
    mcl = umax64(mcl, okey(sqrt((m0 - s.mx) * (m0 - s.mx) + (m1 - s.my) * (m1 - s.my))));
    const double ed = fabs(en - s.E);
    ecl = umax64(ecl, okey(ed));
    fdl = umax64(fdl, okey(fabs(div)));
    if (s.rho <= 0.0) ++dfail;
    if (pr <= 0.0 || pe <= 0.0) ++pfail;
    if (ie <= 0.0) ++ifail;
    rsum += fabs(res);
    msum += fabs(mis);
    esum += ed;
    rl = umax64(rl, okey(fabs(res)));
    rrel = umax64(rrel, okey(fabs(res) / rs));
    ml = umax64(ml, okey(fabs(mis)));
    mrel = umax64(mrel, okey(fabs(mis) / ms));
    ++rcount;
  }
  ECG_RED_ADD_I(st->guard, guard);
  ECG_RED_ADD_I(st->h_nonfinite, hnf);
  ECG_RED_ADD_I(st->flux_nonfinite, fnf);
  ECG_RED_ADD_I(st->final_nonfinite, nfc);
  ECG_RED_ADD_I(st->density_fail, dfail);
  ECG_RED_ADD_I(st->pressure_fail, pfail);
  ECG_RED_ADD_I(st->ie_fail, ifail);
  ECG_RED_ADD_I(st->residual_count, rcount);
  ECG_RED_MAX(st->flux_linf_key, flinf);
  ECG_RED_MIN(st->density_min_key, dmin);
  ECG_RED_MIN(st->solved_p_min_key, spmin);
  ECG_RED_MAX(st->solved_p_max_key, spmax);
  ECG_RED_MIN(st->eos_p_min_key, epmin);
  ECG_RED_MAX(st->eos_p_max_key, epmax);
  ECG_RED_MIN(st->ie_min_key, iemin);
  ECG_RED_MAX(st->ie_max_key, iemax);
  ECG_RED_MAX(st->momentum_corr_key, mcl);
  ECG_RED_MAX(st->energy_corr_key, ecl);
  ECG_RED_MAX(st->flux_div_key, fdl);
  ECG_RED_MAX(st->res_linf_key, rl);
  ECG_RED_MAX(st->res_rel_key, rrel);
  ECG_RED_MAX(st->mis_linf_key, ml);
  ECG_RED_MAX(st->mis_rel_key, mrel);
  ECG_RED_ADD_D(st->res_sum, rsum);
  ECG_RED_ADD_D(st->mis_sum, msum);
  ECG_RED_ADD_D(st->energy_sum, esum);
}

// eq 78 divergence of the final velocity (imex_source_map_step.hpp:190-224),
// velocities looked up through the pressure index map.
template <int NT>
__global__ void __launch_bounds__(NT) imex_eq78_kernel(const EcgImexMap m, const EcgGrid G,
                                                       const double* __restrict__ S, const double* __restrict__ K,
                                                       EcgImexStats* __restrict__ st)
{
  if (gated_off(m)) return;
  __shared__ Shared sh;
  const long long n = static_cast<long long>(m.nx) * m.ny;
  const double idx = G.inv_dx, idy = G.inv_dy;
  long long cnt = 0;
  unsigned long long dl = okey(0.0), ds = okey(0.0);
  auto vel = [&](int i, int j, int axis) {
    const long long r = prow(m, i, j);
    const double rho = S[r];
    const double mm = axis == 0 ? K[r] : K[r + n];
    if (!isfinite(rho) || rho == 0.0 || !isfinite(mm)) return __longlong_as_double(0x7ff8000000000000LL);
    return qdiv(mm, rho);
  };
  for (long long r = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; r < n;
       r += static_cast<long long>(gridDim.x) * NT) {
    const int j = static_cast<int>(static_cast<unsigned>(r) / static_cast<unsigned>(m.nx)), i = static_cast<int>(r) - j * m.nx;
    const double ue = vel(i + 1, j, 0), uw = vel(i - 1, j, 0), vn = vel(i, j + 1, 1), vs = vel(i, j - 1, 1);
    const double dv = 0.5 * (ue - uw) * idx + 0.5 * (vn - vs) * idy;
    // std::max({...}) keeps the first of equal maxima and skips NaN only in
    // the positions compare() allows; the values here are finite or NaN-free.
    double sc = fabs(ue);
    sc = (sc < fabs(uw)) ? fabs(uw) : sc;
    sc = (sc < fabs(vn)) ? fabs(vn) : sc;
    sc = (sc < fabs(vs)) ? fabs(vs) : sc;
    sc = (sc < 1.0) ? 1.0 : sc;
    const double den = sc * smax(idx, idy);
    if (!isfinite(dv) || !isfinite(den) || den <= 0.0) continue;
    dl = umax64(dl, okey(fabs(dv)));
    ds = umax64(ds, okey(fabs(dv) / den));
    ++cnt;
  }
  ECG_RED_ADD_I(st->eq78_count, cnt);
  ECG_RED_MAX(st->eq78_key, dl);
  ECG_RED_MAX(st->eq78_scaled_key, ds);
}

// Old-state loads with the IMEX step's ghost policy.
__device__ __forceinline__ Cons old_cell(const EcgFvParams& P, const double* __restrict__ u, int i, int j)
{
  const int nx = P.g.nx, ny = P.g.ny;
  if (static_cast<unsigned>(i) >= static_cast<unsigned>(nx) || static_cast<unsigned>(j) >= static_cast<unsigned>(ny)) {
    if (i < 0) {
      if (P.bc.x_lo == BC_CONST) return Cons{P.bc.cst[0], P.bc.cst[1], P.bc.cst[2], P.bc.cst[3]};
      i = P.bc.x_lo == BC_PERIODIC ? wrapi(i, nx) : 0;
    } else if (i >= nx) {
      i = P.bc.x_hi == BC_PERIODIC ? wrapi(i, nx) : nx - 1;
    }
    bool flip = false;
    if (j < 0) {
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
      if (P.bc.y_hi == BC_PERIODIC) {
        j = wrapi(j, ny);
      } else if (P.bc.y_hi == BC_REFLECT) {  // the Mach 1.22 variant's top wall
        j = 2 * ny - 1 - j;
        j = j < 0 ? 0 : j;
        flip = true;
      } else {
        j = ny - 1;
      }
    }
    const long long o = static_cast<long long>(j) * P.g.pitch + i;
    Cons c{u[o], u[o + P.g.plane], u[o + 2 * P.g.plane], u[o + 3 * P.g.plane]};
    if (flip) c.my = -c.my;
    return c;
  }
  const long long o = static_cast<long long>(j) * P.g.pitch + i;
  return Cons{u[o], u[o + P.g.plane], u[o + 2 * P.g.plane], u[o + 3 * P.g.plane]};
}

#undef ECG_RED_MAX
#undef ECG_RED_MIN
#undef ECG_RED_ADD_I
#undef ECG_RED_ADD_D

inline int blocks_for(long long n, int nt)
{
  long long b = (n + nt - 1) / nt;
  if (b > 148 * 8) b = 148 * 8;
  return static_cast<int>(b < 1 ? 1 : b);
}

}  // namespace imexk

// ---- launchers ---------------------------------------------------------------------------

inline cudaError_t imex_star(const EcgFvParams& P, const double* u, double dt, double* S, double* p, double* K,
                             EcgImexStats* st, cudaStream_t s)
{
  const dim3 grid((P.g.nx + imexk::SX - 1) / imexk::SX, (P.g.ny + imexk::SY - 1) / imexk::SY);
  imexk::imex_star_kernel<imexk::SX * imexk::SY><<<grid, imexk::SX * imexk::SY, 0, s>>>(P, u, dt, S, p, K, st);
  return cudaGetLastError();
}

inline cudaError_t imex_faces(const EcgImexMap& m, const double* S, const double* p, const double* K, double* fx,
                              double* fy, unsigned char* fxf, unsigned char* fyf, int mode, cudaStream_t s)
{
  const dim3 grid((m.nx + 256) / 256, m.ny + 1 < 65535 ? m.ny + 1 : 65535);
  imexk::imex_face_kernel<256><<<grid, 256, 0, s>>>(m, S, p, K, fx, fy, fxf, fyf, mode);
  return cudaGetLastError();
}

// faces (mode 0) and right-hand side of a Picard pass in one launch
inline cudaError_t imex_assemble(const EcgImexMap& m, const double* S, const double* p, const double* K, double* hx,
                                 double* hy, double dt, double idx, double idy, double* rhs, EcgImexStats* st,
                                 cudaStream_t s)
{
  const dim3 grid((m.nx + 1 + imexk::AX - 1) / imexk::AX, (m.ny + 1 + imexk::AY - 1) / imexk::AY);
  imexk::imex_assemble_kernel<imexk::AX * imexk::AY><<<grid, imexk::AX * imexk::AY, 0, s>>>(m, S, p, K, hx, hy, dt, idx,
                                                                                            idy, rhs, st);
  return cudaGetLastError();
}

// nnz, widest row, largest |a_ij| and max |A - A^T| into st (zeroed by the caller)
inline cudaError_t imex_matrix(const EcgImexMap& m, const double* hx, const double* hy, double dt, double idx,
                               double idy, EcgImexStats* st, cudaStream_t s)
{
  const long long n = static_cast<long long>(m.nx) * m.ny;
  const double xc = 0.25 * dt * dt * idx * idx, yc = 0.25 * dt * dt * idy * idy;
  imexk::imex_matrix_interior_kernel<256><<<imexk::blocks_for(n, 256), 256, 0, s>>>(m, hx, hy, xc, yc, st);
  const long long ring = 4LL * (m.nx + m.ny);
  imexk::imex_matrix_edge_kernel<128><<<imexk::blocks_for(n < 2 * ring ? n : ring, 128), 128, 0, s>>>(m, hx, hy, xc,
                                                                                                       yc, st);
  return cudaGetLastError();
}

inline cudaError_t imex_refresh(const EcgImexMap& m, const double* p_old, const double* x, const double* S, double dt,
                                double idx, double idy, double* K, EcgImexStats* st, cudaStream_t s)
{
  const long long n = static_cast<long long>(m.nx) * m.ny;
  imexk::imex_refresh_kernel<256><<<imexk::blocks_for(n, 256), 256, 0, s>>>(m, p_old, x, S, dt, idx, idy, K, st);
  return cudaGetLastError();
}

inline cudaError_t imex_closeout(const EcgImexMap& m, const EcgGrid& G, const double* S, const double* p,
                                 const double* K, const double* fx, const double* fy, const unsigned char* fxf,
                                 const unsigned char* fyf, double dt, double* out, EcgImexStats* st, cudaStream_t s)
{
  const long long n = static_cast<long long>(m.nx) * m.ny;
  imexk::imex_closeout_kernel<256><<<imexk::blocks_for(n, 256), 256, 0, s>>>(m, G, S, p, K, fx, fy, fxf, fyf, dt, out,
                                                                              st);
  return cudaGetLastError();
}

inline cudaError_t imex_eq78(const EcgImexMap& m, const EcgGrid& G, const double* S, const double* K, EcgImexStats* st,
                             cudaStream_t s)
{
  const long long n = static_cast<long long>(m.nx) * m.ny;
  imexk::imex_eq78_kernel<256><<<imexk::blocks_for(n, 256), 256, 0, s>>>(m, G, S, K, st);
  return cudaGetLastError();
}

}  // namespace ECG_NS
