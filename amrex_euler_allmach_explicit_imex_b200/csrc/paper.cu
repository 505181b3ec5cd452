// Direct BDLTV20 T1/S2 driver on the device: ecg_paper_t1s2_run (include/ecg.h),
// the report rows' IMEX driver run_bdltv20_paper_t1_s2
// (imex/imex_bdltv20_direct_driver.hpp:44-779).
//
// Differences from the main-loop IMEX step (imex.cu) that this driver keeps:
//  * the epsilon-scaled energy E = p/(gamma-1) + eps K (core/state_primitives.hpp:119-139);
//  * neighbours outside a non-periodic axis are the exact solution sampled on
//    the boundary (x = prob_lo or prob_hi), at t for the explicit star update
//    and at t + dt for the pressure system, whose out-of-domain columns move
//    to the right-hand side;
//  * the material Lax-Friedrichs star flux carries eps K u in its energy row;
//  * the Toro modes drop the y-terms of the pressure row (cy = 0, :428-431);
//  * the face-enthalpy guard is 1e-12 max(1, |q_L| + |q_R|)
//    (problems/problem_state_functions.hpp:112-127);
//  * the closeout is E = p/(gamma-1) + eps K (:582-584).
// Per step: one star kernel, then per Picard iteration the corrected cells,
// the face enthalpies, the pressure rows and one cooperative GMRES solve with
// the reference's stopping rule (gmres.cu); then the closeout.  Built without
// FMA contraction, in the reference's operation order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "ctx.h"
#include "ecg.h"
#include "imex_internal.h"

namespace ecg_paper {

#include "ecg_device.cuh"
#include "exact_states.cuh"

constexpr int NT = 256;
constexpr double kMax = 1.7976931348623157e308;

struct Ctl {
  int mode, nx, ny, px, py, toro;
  long long pitch, plane;  // padded layout of the context state
  double gamma, eps, dx, dy, plo_x, plo_y, phi_x, phi_y;
  EcgProblem pr;
  Prim toro_l, toro_r;
  double x0;
};

// Counters and reductions on the device.
struct Acc {
  unsigned long long rate_key;  // material rate (okey)
  int guard;                    // face-enthalpy guards
  int nonfinite;
  int nonpositive;
  int pad;
  unsigned long long rho_min_key, p_min_key, drho_max_key, dp_max_key;
};

__device__ __forceinline__ int wrapi(int i, int n)
{
  int r = i % n;
  return r < 0 ? r + n : r;
}

// bdltv20_paper_to_primitive / _to_conserved (core/state_primitives.hpp:119-139)
__device__ __forceinline__ Prim paper_prim(const Cons& u, double g, double eps)
{
  const double inv_rho = 1.0 / u.rho;
  const double ux = u.mx * inv_rho;
  const double uy = u.my * inv_rho;
  const double kinetic = 0.5 * u.rho * (ux * ux + uy * uy);
  return Prim{u.rho, ux, uy, (g - 1.0) * (u.E - eps * kinetic)};
}
__device__ __forceinline__ Cons paper_cons(const Prim& q, double g, double eps)
{
  const double kinetic = 0.5 * q.rho * (q.u * q.u + q.v * q.v);
  return Cons{q.rho, q.rho * q.u, q.rho * q.v, q.p / (g - 1.0) + eps * kinetic};
}

// The exact solution of the mode at (x, y, t).
__device__ Prim exact_state(const Ctl& C, double x, double y, double t)
{
  if (C.toro) return riemann_sample(x, t, C.toro_l, C.toro_r, C.gamma, C.x0);
  if (C.mode == ECG_PAPER_ISENTROPIC_VORTEX_PERIODIC) return isentropic_vortex_state(x, y, C.pr, C.plo_x, C.plo_y, t);
  if (C.mode == ECG_PAPER_ADVECTION_BLOB_PERIODIC) return exact_blob_state(x, y, C.pr, C.plo_x, C.plo_y, t);
  return gresho_state(x, y, C.pr);
}

// exact_boundary_state (:100-130): the exact state sampled at the boundary
// coordinate of an out-of-domain index (cell centre along the other axis).
__device__ Cons exact_boundary_state(const Ctl& C, int i, int j, double t)
{
  const int ic = i < 0 ? 0 : (i > C.nx - 1 ? C.nx - 1 : i);
  const int jc = j < 0 ? 0 : (j > C.ny - 1 ? C.ny - 1 : j);
  double x = C.plo_x + (static_cast<double>(ic) + 0.5) * C.dx;
  double y = C.plo_y + (static_cast<double>(jc) + 0.5) * C.dy;
  if (i < 0) x = C.plo_x;
  else if (i >= C.nx) x = C.phi_x;
  if (j < 0) y = C.plo_y;
  else if (j >= C.ny) y = C.phi_y;
  return paper_cons(exact_state(C, x, y, t), C.gamma, C.eps);
}

// A cell of a compact 4-plane array (or of the padded state), wrapped on
// periodic axes, else the exact boundary state at t.
__device__ __forceinline__ Cons cell_from(const Ctl& C, const double* __restrict__ a, long long pitch, long long plane,
                                          int i, int j, double t)
{
  if (C.px) i = wrapi(i, C.nx);
  if (C.py) j = wrapi(j, C.ny);
  if (i >= 0 && i < C.nx && j >= 0 && j < C.ny) {
    const long long o = static_cast<long long>(j) * pitch + i;
    return Cons{a[o], a[o + plane], a[o + 2 * plane], a[o + 3 * plane]};
  }
  return exact_boundary_state(C, i, j, t);
}

// pressure_from (:294-307): the pressure vector inside, the exact boundary
// pressure outside.
__device__ __forceinline__ double pressure_from(const Ctl& C, const double* __restrict__ p, int i, int j, double t)
{
  if (C.px) i = wrapi(i, C.nx);
  if (C.py) j = wrapi(j, C.ny);
  if (i >= 0 && i < C.nx && j >= 0 && j < C.ny) return p[static_cast<long long>(j) * C.nx + i];
  return paper_prim(exact_boundary_state(C, i, j, t), C.gamma, C.eps).p;
}

__device__ __forceinline__ void store(double* a, long long o, long long plane, const Cons& c)
{
  a[o] = c.rho;
  a[o + plane] = c.mx;
  a[o + 2 * plane] = c.my;
  a[o + 3 * plane] = c.E;
}

template <class T>
__device__ __forceinline__ T grid_stride_begin()
{
  return static_cast<T>(blockIdx.x) * blockDim.x + threadIdx.x;
}

// ---- kernels --------------------------------------------------------------------

// State from initialize_state -> epsilon-scaled conserved (:74-84).
__global__ void convert_kernel(const Ctl C, double* __restrict__ u)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    const long long o = static_cast<long long>(j) * C.pitch + i;
    const Cons c{u[o], u[o + C.plane], u[o + 2 * C.plane], u[o + 3 * C.plane]};
    store(u, o, C.plane, paper_cons(to_prim(c, C.gamma), C.gamma, C.eps));
  }
}

// compute_bdltv20_paper_t1_s2_dt (:8-41): max of 2 |u| / min(dx, dy).
__global__ void rate_kernel(const Ctl C, const double* __restrict__ u, Acc* acc)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  const double min_dx = C.dx < C.dy ? C.dx : C.dy;
  unsigned long long k = okey(0.0);
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    const long long o = static_cast<long long>(j) * C.pitch + i;
    const Prim q = paper_prim(Cons{u[o], u[o + C.plane], u[o + 2 * C.plane], u[o + 3 * C.plane]}, C.gamma, C.eps);
    if (isfinite(q.u) && isfinite(q.v)) {
      const double speed = sqrt(q.u * q.u + q.v * q.v);
      const unsigned long long kk = okey(2.0 * speed / min_dx);
      k = kk > k ? kk : k;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, k, o);
    k = v > k ? v : k;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(&acc->rate_key, k);
}

// Conserved minmod reconstruction of the old state (:179-196).
__device__ __forceinline__ Cons recon_old(const Ctl& C, const double* __restrict__ u, int i, int j, int axis, int side,
                                          double t)
{
  const Cons um = axis == 0 ? cell_from(C, u, C.pitch, C.plane, i - 1, j, t) : cell_from(C, u, C.pitch, C.plane, i, j - 1, t);
  const Cons uc = cell_from(C, u, C.pitch, C.plane, i, j, t);
  const Cons up = axis == 0 ? cell_from(C, u, C.pitch, C.plane, i + 1, j, t) : cell_from(C, u, C.pitch, C.plane, i, j + 1, t);
  const double h = 0.5 * side;
  return Cons{uc.rho + h * minmod(uc.rho - um.rho, up.rho - uc.rho), uc.mx + h * minmod(uc.mx - um.mx, up.mx - uc.mx),
              uc.my + h * minmod(uc.my - um.my, up.my - uc.my), uc.E + h * minmod(uc.E - um.E, up.E - uc.E)};
}

// explicit_flux (:197-225): material Lax-Friedrichs flux, eps K u in the energy row.
__device__ __forceinline__ Cons lf_flux(const Ctl& C, const Cons& lu, const Cons& ru, int axis)
{
  const Prim l = paper_prim(lu, C.gamma, C.eps), r = paper_prim(ru, C.gamma, C.eps);
  const double mxl = l.rho * l.u, myl = l.rho * l.v, mxr = r.rho * r.u, myr = r.rho * r.v;
  const double kl = C.eps * 0.5 * l.rho * (l.u * l.u + l.v * l.v);
  const double kr = C.eps * 0.5 * r.rho * (r.u * r.u + r.v * r.v);
  Cons fl, fr;
  if (axis == 0) {
    fl = Cons{mxl, mxl * l.u, myl * l.u, kl * l.u};
    fr = Cons{mxr, mxr * r.u, myr * r.u, kr * r.u};
  } else {
    fl = Cons{myl, mxl * l.v, myl * l.v, kl * l.v};
    fr = Cons{myr, mxr * r.v, myr * r.v, kr * r.v};
  }
  const double sm = smax(fabs(axis == 0 ? l.u : l.v), fabs(axis == 0 ? r.u : r.v));
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ru.rho - lu.rho), 0.5 * (fl.mx + fr.mx) - hs * (ru.mx - lu.mx),
              0.5 * (fl.my + fr.my) - hs * (ru.my - lu.my), 0.5 * (fl.E + fr.E) - hs * (ru.E - lu.E)};
}

// Star update (:226-250), the old pressure and the first Picard guess.
__global__ void star_kernel(const Ctl C, const double* __restrict__ u, double t, double dt, double* __restrict__ star,
                            double* __restrict__ p_old, double* __restrict__ p)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    const Cons fxl = lf_flux(C, recon_old(C, u, i - 1, j, 0, 1, t), recon_old(C, u, i, j, 0, -1, t), 0);
    const Cons fxr = lf_flux(C, recon_old(C, u, i, j, 0, 1, t), recon_old(C, u, i + 1, j, 0, -1, t), 0);
    const Cons fyb = lf_flux(C, recon_old(C, u, i, j - 1, 1, 1, t), recon_old(C, u, i, j, 1, -1, t), 1);
    const Cons fyt = lf_flux(C, recon_old(C, u, i, j, 1, 1, t), recon_old(C, u, i, j + 1, 1, -1, t), 1);
    const long long o = static_cast<long long>(j) * C.pitch + i;
    const Cons old{u[o], u[o + C.plane], u[o + 2 * C.plane], u[o + 3 * C.plane]};
    Cons s;
    s.rho = old.rho - dt * ((fxr.rho - fxl.rho) / C.dx + (fyt.rho - fyb.rho) / C.dy);
    s.mx = old.mx - dt * ((fxr.mx - fxl.mx) / C.dx + (fyt.mx - fyb.mx) / C.dy);
    s.my = old.my - dt * ((fxr.my - fxl.my) / C.dx + (fyt.my - fyb.my) / C.dy);
    s.E = old.E - dt * ((fxr.E - fxl.E) / C.dx + (fyt.E - fyb.E) / C.dy);
    store(star, e, n, s);
    const double po = paper_prim(old, C.gamma, C.eps).p;
    p_old[e] = po;
    p[e] = po;
  }
}

// refresh_corrected_cells_and_faces, cells (:320-336): star momentum minus
// dt grad p / eps (central), the y-part dropped in the Toro modes.
__global__ void correct_kernel(const Ctl C, const double* __restrict__ star, const double* __restrict__ p, int use_p,
                               double dt, double t1, double* __restrict__ corr)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    Cons u{star[e], star[e + n], star[e + 2 * n], star[e + 3 * n]};
    if (use_p) {
      const double pe = pressure_from(C, p, i + 1, j, t1), pw = pressure_from(C, p, i - 1, j, t1);
      const double pn = pressure_from(C, p, i, j + 1, t1), ps = pressure_from(C, p, i, j - 1, t1);
      u.mx -= dt * (pe - pw) / (2.0 * C.eps * C.dx);
      if (!C.toro) u.my -= dt * (pn - ps) / (2.0 * C.eps * C.dy);
    }
    store(corr, e, n, u);
  }
}

// bdltv20_eq46_face_enthalpy (problems/problem_state_functions.hpp:112-127)
__device__ __forceinline__ double eq46(double rl, double pl, double ql, double rr, double pr, double qr, double g,
                                       int& guard)
{
  const double hl = g * pl / ((g - 1.0) * rl);
  const double hr = g * pr / ((g - 1.0) * rr);
  const double denom = ql + qr;
  const double scale = smax(1.0, fabs(ql) + fabs(qr));
  if (fabs(denom) <= 1.0e-12 * scale) {
    ++guard;
    return 0.5 * (hl + hr);
  }
  return (hl * ql + hr * qr) / denom;
}

// refresh_corrected_cells_and_faces, faces (:337-380).  x-faces are stored
// (nx + 1) per row, face f between cells f - 1 and f; on a periodic axis face
// 0 repeats face nx and is not counted twice.
__global__ void face_kernel(const Ctl C, const double* __restrict__ corr, const double* __restrict__ p, double t1,
                            double* __restrict__ hx, double* __restrict__ hy, Acc* acc)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  const long long nfx = static_cast<long long>(C.nx + 1) * C.ny;
  const long long nfy = static_cast<long long>(C.nx) * (C.ny + 1);
  int guard = 0, nonfinite = 0;
  for (long long e = grid_stride_begin<long long>(); e < nfx + nfy; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    int g = 0;
    bool counted;
    double h, m;
    if (e < nfx) {
      const int f = static_cast<int>(e % (C.nx + 1)), j = static_cast<int>(e / (C.nx + 1));
      const Cons l = cell_from(C, corr, C.nx, n, f - 1, j, t1), r = cell_from(C, corr, C.nx, n, f, j, t1);
      const double pl = pressure_from(C, p, f - 1, j, t1), pr = pressure_from(C, p, f, j, t1);
      h = eq46(l.rho, pl, l.mx, r.rho, pr, r.mx, C.gamma, g);
      m = 0.5 * (l.mx + r.mx);
      hx[e] = h;
      counted = !(C.px && f == 0);
    } else {
      const long long k = e - nfx;
      const int i = static_cast<int>(k % C.nx), f = static_cast<int>(k / C.nx);
      const Cons b = cell_from(C, corr, C.nx, n, i, f - 1, t1), tp = cell_from(C, corr, C.nx, n, i, f, t1);
      const double pb = pressure_from(C, p, i, f - 1, t1), pt = pressure_from(C, p, i, f, t1);
      h = eq46(b.rho, pb, b.my, tp.rho, pt, tp.my, C.gamma, g);
      m = 0.5 * (b.my + tp.my);
      hy[k] = h;
      counted = !(C.py && f == 0);
    }
    if (counted) {
      guard += g;
      if (!isfinite(h) || !isfinite(m)) ++nonfinite;
    }
  }
  if (guard) atomicAdd(&acc->guard, guard);
  if (nonfinite) atomicAdd(&acc->nonfinite, nonfinite);
}

// Pressure rows (:412-485): eps (E* - K - dt div(h m*)) with the out-of-domain
// columns moved to the right-hand side at t + dt; the matrix itself is applied
// matrix-free by the GMRES operator (boundary columns dropped).
__global__ void rhs_kernel(const Ctl C, const double* __restrict__ star, const double* __restrict__ corr,
                           const double* __restrict__ hx, const double* __restrict__ hy, double dt, double t1,
                           double cx, double cy, double* __restrict__ rhs, Acc* acc)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  int nonfinite = 0;
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    const Cons s{star[e], star[e + n], star[e + 2 * n], star[e + 3 * n]};
    const double lmx = corr[e + n], lmy = corr[e + 2 * n];
    const double he = hx[static_cast<long long>(j) * (C.nx + 1) + i + 1], hw = hx[static_cast<long long>(j) * (C.nx + 1) + i];
    const double hn = hy[static_cast<long long>(j + 1) * C.nx + i], hs = hy[static_cast<long long>(j) * C.nx + i];
    const double kinetic = C.eps * 0.5 * (lmx * lmx + lmy * lmy) / s.rho;
    const Cons se = cell_from(C, star, C.nx, n, i + 1, j, t1), sw = cell_from(C, star, C.nx, n, i - 1, j, t1);
    const Cons sn = cell_from(C, star, C.nx, n, i, j + 1, t1), ss = cell_from(C, star, C.nx, n, i, j - 1, t1);
    const double div = (he * se.mx + (he - hw) * s.mx - hw * sw.mx) / (2.0 * C.dx) +
                       (hn * sn.my + (hn - hs) * s.my - hs * ss.my) / (2.0 * C.dy);
    double b = C.eps * (s.E - kinetic - dt * div);
    // add_lhs order: i+2, i+1, (diagonal, always inside), i-1, i-2, j+2, j+1, j-1, j-2
    const int ci[8] = {i + 2, i + 1, i - 1, i - 2, i, i, i, i};
    const int cj[8] = {j, j, j, j, j + 2, j + 1, j - 1, j - 2};
    const double cv[8] = {-cx * he, -cx * (he - hw), cx * (he - hw), -cx * hw,
                          -cy * hn, -cy * (hn - hs), cy * (hn - hs), -cy * hs};
    for (int q = 0; q < 8; ++q) {
      if (cv[q] == 0.0) continue;
      int a = ci[q], c = cj[q];
      if (C.px) a = wrapi(a, C.nx);
      if (C.py) c = wrapi(c, C.ny);
      if (a >= 0 && a < C.nx && c >= 0 && c < C.ny) continue;
      b -= cv[q] * paper_prim(exact_boundary_state(C, ci[q], cj[q], t1), C.gamma, C.eps).p;
    }
    rhs[e] = b;
    if (!isfinite(b) || !(s.rho > 0.0)) ++nonfinite;
  }
  if (nonfinite) atomicAdd(&acc->nonfinite, nonfinite);
}

// Closeout (:569-600): the corrected cells with E = p/(gamma-1) + eps K.
__global__ void closeout_kernel(const Ctl C, const double* __restrict__ corr, const double* __restrict__ p,
                                double* __restrict__ u, Acc* acc)
{
  const long long n = static_cast<long long>(C.nx) * C.ny;
  int nonfinite = 0, nonpositive = 0;
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    Cons c{corr[e], corr[e + n], corr[e + 2 * n], corr[e + 3 * n]};
    const double kinetic = C.eps * 0.5 * (c.mx * c.mx + c.my * c.my) / c.rho;
    c.E = p[e] / (C.gamma - 1.0) + kinetic;
    const Prim q = paper_prim(c, C.gamma, C.eps);
    if (!isfinite(q.rho) || !isfinite(q.u) || !isfinite(q.v) || !isfinite(q.p)) ++nonfinite;
    if (!(q.rho > 0.0) || !(q.p > 0.0)) ++nonpositive;
    store(u, static_cast<long long>(j) * C.pitch + i, C.plane, c);
  }
  if (nonfinite) atomicAdd(&acc->nonfinite, nonfinite);
  if (nonpositive) atomicAdd(&acc->nonpositive, nonpositive);
}

// Error norms against the exact solution (:604-660): per-block partial sums
// (summed on the host in block order), maxima and minima by ordered keys.
__global__ void metrics_kernel(const Ctl C, const double* __restrict__ u, double t, double* __restrict__ part, Acc* acc)
{
  __shared__ double sh[6][NT / 32];
  const long long n = static_cast<long long>(C.nx) * C.ny;
  double s[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long kr = okey(kMax), kp = okey(kMax), kdr = okey(0.0), kdp = okey(0.0);
  for (long long e = grid_stride_begin<long long>(); e < n; e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % C.nx), j = static_cast<int>(e / C.nx);
    const double x = C.plo_x + (static_cast<double>(i) + 0.5) * C.dx;
    const double y = C.plo_y + (static_cast<double>(j) + 0.5) * C.dy;
    const long long o = static_cast<long long>(j) * C.pitch + i;
    const Prim q = paper_prim(Cons{u[o], u[o + C.plane], u[o + 2 * C.plane], u[o + 3 * C.plane]}, C.gamma, C.eps);
    const Prim ex = exact_state(C, x, y, t);
    const double du = sqrt((q.u - ex.u) * (q.u - ex.u) + (q.v - ex.v) * (q.v - ex.v));
    const double dr = fabs(q.rho - ex.rho), dp = fabs(q.p - ex.p);
    s[0] += dr;
    s[1] += du;
    s[2] += dp;
    s[3] += dr * dr;
    s[4] += du * du;
    s[5] += dp * dp;
    const unsigned long long a = okey(dr), b = okey(dp), c = okey(q.rho), d = okey(q.p);
    kdr = a > kdr ? a : kdr;
    kdp = b > kdp ? b : kdp;
    kr = c < kr ? c : kr;
    kp = d < kp ? d : kp;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = 0; q < 6; ++q) {
    double v = s[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[q][warp] = v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long v = __shfl_xor_sync(0xffffffffu, kdr, o);
    kdr = v > kdr ? v : kdr;
    v = __shfl_xor_sync(0xffffffffu, kdp, o);
    kdp = v > kdp ? v : kdp;
    v = __shfl_xor_sync(0xffffffffu, kr, o);
    kr = v < kr ? v : kr;
    v = __shfl_xor_sync(0xffffffffu, kp, o);
    kp = v < kp ? v : kp;
  }
  if (lane == 0) {
    atomicMax(&acc->drho_max_key, kdr);
    atomicMax(&acc->dp_max_key, kdp);
    atomicMin(&acc->rho_min_key, kr);
    atomicMin(&acc->p_min_key, kp);
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0.0;
    for (int w = 0; w < NT / 32; ++w) v += sh[threadIdx.x][w];
    part[blockIdx.x * 6 + threadIdx.x] = v;
  }
}

__global__ void acc_init_kernel(Acc* acc)
{
  acc->rate_key = okey(0.0);
  acc->guard = acc->nonfinite = acc->nonpositive = 0;
  acc->rho_min_key = okey(kMax);
  acc->p_min_key = okey(kMax);
  acc->drho_max_key = okey(0.0);
  acc->dp_max_key = okey(0.0);
}

__global__ void rate_reset_kernel(Acc* acc) { acc->rate_key = okey(0.0); }

}  // namespace ecg_paper

namespace {

using ecg_paper::Acc;
using ecg_paper::Ctl;
using ecg_paper::NT;

int blocks(long long n)
{
  long long b = (n + NT - 1) / NT;
  if (b > 148 * 8) b = 148 * 8;
  return static_cast<int>(b < 1 ? 1 : b);
}

double key_to_double(unsigned long long k) { return ecgi::okey_to_double(k); }

// core/config_reader.hpp:133-258 for the direct driver's modes.
bool mode_ok(const ecg_run_config& c, const ecg_paper_options& o, std::string& why)
{
  const bool exact = c.field_boundary == ECG_FIELD_BOUNDARY_EXACT_DIRICHLET;
  why.clear();
  if (c.method != ECG_METHOD_IMEX) why = "euler.bdltv20_paper_t1_s2 requires euler.method=imex.";
  else if (c.spatial_order != 2) why = "euler.bdltv20_paper_t1_s2 requires euler.spatial_order=2.";
  else if (c.slope_limiter != ECG_LIMITER_MINMOD) why = "euler.bdltv20_paper_t1_s2 requires euler.slope_limiter=minmod.";
  else if (!(c.gamma > 1.0) || !std::isfinite(c.gamma)) why = "euler.bdltv20_paper_t1_s2 requires finite gamma > 1.";
  else if (!(c.imex_solver_tol > 0.0) || !std::isfinite(c.imex_solver_tol) || c.imex_solver_max_iter < 0)
    why = "euler.bdltv20_paper_t1_s2 requires positive finite GMRES tolerance and nonnegative max_iter.";
  else if (!(o.fixed_dt < 0.0) && (!(o.fixed_dt > 0.0) || !std::isfinite(o.fixed_dt)))
    why = "euler.bdltv20_paper_t1_s2_dt must be negative for CFL mode or finite positive.";
  else if (!(o.epsilon > 0.0) || !std::isfinite(o.epsilon)) why = "euler.bdltv20_paper_epsilon must be finite and positive.";
  else if (o.max_steps < 1) why = "euler.bdltv20_paper_t1_s2_max_steps must be at least one.";
  else if (o.mode == ECG_PAPER_TORO_X_EXACT_DIRICHLET_Y_PERIODIC) {
    if (c.problem != ECG_PROBLEM_TORO1 || c.is_periodic[0] != 0 || c.is_periodic[1] != 1 || !exact ||
        c.n_cell[0] < 16 || c.n_cell[1] < 2)
      why = "BDLTV20 Toro x-exact mode requires problem=toro1, periodicity=0 1, exact Dirichlet, and at least 16x2 cells.";
  } else if (o.mode == ECG_PAPER_TORO_XY_EXACT_DIRICHLET) {
    if (c.problem != ECG_PROBLEM_TORO1 || c.is_periodic[0] != 0 || c.is_periodic[1] != 0 || !exact ||
        c.n_cell[0] < 16 || c.n_cell[1] < 2)
      why = "BDLTV20 Toro xy-exact mode requires problem=toro1, periodicity=0 0, exact Dirichlet, and at least 16x2 cells.";
  } else if (o.mode == ECG_PAPER_GRESHO_EXACT_DIRICHLET) {
    if (c.problem != ECG_PROBLEM_GRESHO_VORTEX || c.is_periodic[0] != 0 || c.is_periodic[1] != 0 || !exact ||
        c.n_cell[0] < 8 || c.n_cell[1] < 8)
      why = "BDLTV20 Gresho mode requires problem=gresho_vortex, periodicity=0 0, exact Dirichlet, and at least 8x8 cells.";
  } else if (o.mode == ECG_PAPER_ISENTROPIC_VORTEX_PERIODIC) {
    if (c.problem != ECG_PROBLEM_ISENTROPIC_VORTEX || c.is_periodic[0] != 1 || c.is_periodic[1] != 1 ||
        c.n_cell[0] < 8 || c.n_cell[1] < 8)
      why = "BDLTV20 isentropic-vortex mode requires problem=isentropic_vortex, periodicity=1 1, and at least 8x8 cells.";
  } else if (o.mode == ECG_PAPER_ADVECTION_BLOB_PERIODIC) {
    if (c.problem != ECG_PROBLEM_ADVECTION_BLOB || c.is_periodic[0] != 1 || c.is_periodic[1] != 1 ||
        c.n_cell[0] < 8 || c.n_cell[1] < 8)
      why = "BDLTV20 advection-blob mode requires problem=advection_blob, periodicity=1 1, and at least 8x8 cells.";
  } else {
    why = "Unsupported euler.bdltv20_paper_t1_s2 setting.";
  }
  return why.empty();
}

struct Buffers {
  double* star = nullptr;
  double* corr = nullptr;
  double* p_old = nullptr;
  double* p = nullptr;
  double* x = nullptr;
  double* hx = nullptr;
  double* hy = nullptr;
  double* rhs = nullptr;
  double* part = nullptr;
  Acc* acc = nullptr;
  Acc* h_acc = nullptr;
  EcgGmresWork* gw = nullptr;
  ~Buffers()
  {
    cudaFree(star);
    cudaFree(corr);
    cudaFree(p_old);
    cudaFree(p);
    cudaFree(x);
    cudaFree(hx);
    cudaFree(hy);
    cudaFree(rhs);
    cudaFree(part);
    cudaFree(acc);
    cudaFreeHost(h_acc);
    gmres_work_destroy(gw);
  }
};

}  // namespace

extern "C" ecg_status ecg_paper_t1s2_run(ecg_ctx* c, const ecg_paper_options* opts, ecg_paper_result* out)
{
  if (!c || !opts || !out) return ECG_ERR_BAD_ARG;
  std::memset(out, 0, sizeof(*out));
  if (c->slab()) {
    c->err = "the direct T1/S2 driver runs on the whole grid: no slab contexts";
    return ECG_ERR_UNSUPPORTED;
  }
  const ecg_run_config& cfg = c->cfg;
  std::string why;
  if (!mode_ok(cfg, *opts, why)) {
    c->err = why;
    return ECG_ERR_BAD_ARG;
  }
  const int nx = c->grid.nx, ny = c->grid.ny;
  const long long n = static_cast<long long>(nx) * ny;
  cudaStream_t s = c->stream;

  Ctl C;
  std::memset(&C, 0, sizeof(C));
  C.mode = opts->mode;
  C.nx = nx;
  C.ny = ny;
  C.px = cfg.is_periodic[0] != 0;
  C.py = cfg.is_periodic[1] != 0;
  C.toro = opts->mode == ECG_PAPER_TORO_X_EXACT_DIRICHLET_Y_PERIODIC || opts->mode == ECG_PAPER_TORO_XY_EXACT_DIRICHLET;
  C.pitch = c->grid.pitch;
  C.plane = c->grid.plane;
  C.gamma = cfg.gamma;
  C.eps = opts->epsilon;
  C.dx = c->grid.dx;
  C.dy = c->grid.dy;
  C.plo_x = cfg.prob_lo[0];
  C.plo_y = cfg.prob_lo[1];
  C.phi_x = cfg.prob_hi[0];
  C.phi_y = cfg.prob_hi[1];
  C.pr = ecgi::problem_of(c, false);
  C.toro_l = ecg_paper::Prim{C.pr.toro_l[0], C.pr.toro_l[1], C.pr.toro_l[2], C.pr.toro_l[3]};
  C.toro_r = ecg_paper::Prim{C.pr.toro_r[0], C.pr.toro_r[1], C.pr.toro_r[2], C.pr.toro_r[3]};
  C.x0 = cfg.riemann_interface_x;

  Buffers B;
  bool ok = true;
  auto alloc = [&](double** ptr, long long count) {
    ok = ok && ecgi::cuda_ok(c, cudaMalloc(ptr, sizeof(double) * static_cast<size_t>(count)), "alloc");
  };
  alloc(&B.star, 4 * n);
  alloc(&B.corr, 4 * n);
  alloc(&B.p_old, n);
  alloc(&B.p, n);
  alloc(&B.x, n);
  alloc(&B.hx, static_cast<long long>(nx + 1) * ny);
  alloc(&B.hy, static_cast<long long>(nx) * (ny + 1));
  alloc(&B.rhs, n);
  alloc(&B.part, 6LL * blocks(n));
  ok = ok && ecgi::cuda_ok(c, cudaMalloc(&B.acc, sizeof(Acc)), "alloc") &&
       ecgi::cuda_ok(c, cudaMallocHost(&B.h_acc, sizeof(Acc)), "alloc");
  if (!ok) return ECG_ERR_CUDA;
  const int max_iter = cfg.imex_solver_max_iter;
  std::string gerr;
  B.gw = gmres_work_create(n, max_iter < 1 ? 1 : max_iter, c->num_sms, c->device, false, &gerr);
  if (!B.gw) {
    c->err = gerr;
    return ECG_ERR_CUDA;
  }

  // initial state: initialize_state, then the epsilon-scaled energy
  if (ecg_initialize_state(c) != ECG_OK) return ECG_ERR_CUDA;
  double* u = c->cur_state_mut();
  ecg_paper::acc_init_kernel<<<1, 1, 0, s>>>(B.acc);
  ecg_paper::convert_kernel<<<blocks(n), NT, 0, s>>>(C, u);
  if (!ecgi::cuda_ok(c, cudaGetLastError(), "paper init")) return ECG_ERR_CUDA;

  EcgPressureOp op;
  std::memset(&op, 0, sizeof(op));
  op.nx = nx;
  op.ny = ny;
  op.px = C.px;
  op.py = C.py;
  op.drop = 1;
  op.diag0 = C.eps / (cfg.gamma - 1.0);
  op.hx = B.hx;
  op.hy = B.hy;

  int steps = 0, failures = 0, it_max = 0, dt_nonfinite = 0;
  double time = 0.0, res_max = 0.0, rel_max = 0.0;
  const double dx = c->grid.dx, dy = c->grid.dy;
  while (time < cfg.stop_time - 1.0e-14 && steps < opts->max_steps) {
    // compute_bdltv20_paper_t1_s2_dt (:8-41)
    double dt;
    if (opts->fixed_dt > 0.0) {
      dt = std::min(opts->fixed_dt, cfg.stop_time - time);
    } else {
      ecg_paper::rate_reset_kernel<<<1, 1, 0, s>>>(B.acc);
      ecg_paper::rate_kernel<<<blocks(n), NT, 0, s>>>(C, u, B.acc);
      if (!ecgi::cuda_ok(c, cudaMemcpyAsync(B.h_acc, B.acc, sizeof(Acc), cudaMemcpyDeviceToHost, s), "rate") ||
          !ecgi::cuda_ok(c, cudaStreamSynchronize(s), "sync"))
        return ECG_ERR_CUDA;
      const double rate = key_to_double(B.h_acc->rate_key);
      const double remaining = cfg.stop_time - time;
      dt = !(rate > 0.0) ? remaining : std::min(cfg.imex_cfl / rate, remaining);
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) {
      ++dt_nonfinite;
      break;
    }
    const double t1 = time + dt;
    ecg_paper::star_kernel<<<blocks(n), NT, 0, s>>>(C, u, time, dt, B.star, B.p_old, B.p);
    const double cx = 0.25 * dt * dt / (dx * dx);
    const double cy = C.toro ? 0.0 : 0.25 * dt * dt / (dy * dy);
    op.xc = cx;
    op.yc = cy;
    for (int picard = 0; picard < cfg.imex_picard_iterations; ++picard) {
      ecg_paper::correct_kernel<<<blocks(n), NT, 0, s>>>(C, B.star, B.p, picard == 0 ? 0 : 1, dt, t1, B.corr);
      ecg_paper::face_kernel<<<blocks(static_cast<long long>(nx + 1) * ny + static_cast<long long>(nx) * (ny + 1)), NT,
                               0, s>>>(C, B.corr, picard == 0 ? B.p_old : B.p, t1, B.hx, B.hy, B.acc);
      ecg_paper::rhs_kernel<<<blocks(n), NT, 0, s>>>(C, B.star, B.corr, B.hx, B.hy, dt, t1, cx, cy, B.rhs, B.acc);
      if (!ecgi::cuda_ok(c, cudaGetLastError(), "paper rows")) return ECG_ERR_CUDA;
      EcgGmresResult g;
      if (!ecgi::cuda_ok(c, gmres_solve(B.gw, op, B.rhs, B.p, B.x, max_iter, cfg.imex_solver_tol, false, 0, 0.0, 0, 1,
                                            c->opt.deterministic != 0, &g, s),
                         "gmres"))
        return ECG_ERR_CUDA;
      if (g.timeout) {
        c->err = "gmres grid barrier timed out";
        return ECG_ERR_TIMEOUT;
      }
      if (!g.converged || g.nonfinite || g.breakdown) ++failures;
      it_max = std::max(it_max, g.iterations);
      double lr = 0.0, bn = 1.0;
      int nf = 0;
      if (!ecgi::cuda_ok(c, pressure_residual(B.gw, op, B.rhs, B.x, &lr, &bn, &nf, s), "residual")) return ECG_ERR_CUDA;
      res_max = std::max(res_max, lr);
      rel_max = std::max(rel_max, lr / bn);
      std::swap(B.p, B.x);
    }
    ecg_paper::correct_kernel<<<blocks(n), NT, 0, s>>>(C, B.star, B.p, 1, dt, t1, B.corr);
    ecg_paper::face_kernel<<<blocks(static_cast<long long>(nx + 1) * ny + static_cast<long long>(nx) * (ny + 1)), NT, 0,
                             s>>>(C, B.corr, B.p, t1, B.hx, B.hy, B.acc);
    ecg_paper::closeout_kernel<<<blocks(n), NT, 0, s>>>(C, B.corr, B.p, u, B.acc);
    if (!ecgi::cuda_ok(c, cudaGetLastError(), "paper closeout")) return ECG_ERR_CUDA;
    time += dt;
    ++steps;
  }
  c->uploaded = true;
  c->invalidate();

  // report (:604-777)
  const int nb = blocks(n);
  ecg_paper::metrics_kernel<<<nb, NT, 0, s>>>(C, u, time, B.part, B.acc);
  std::vector<double> part(6 * static_cast<size_t>(nb));
  if (!ecgi::cuda_ok(c, cudaGetLastError(), "metrics") ||
      !ecgi::cuda_ok(c, cudaMemcpyAsync(part.data(), B.part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s),
                     "metrics") ||
      !ecgi::cuda_ok(c, cudaMemcpyAsync(B.h_acc, B.acc, sizeof(Acc), cudaMemcpyDeviceToHost, s), "metrics") ||
      !ecgi::cuda_ok(c, cudaStreamSynchronize(s), "sync"))
    return ECG_ERR_CUDA;
  double sums[6] = {0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nb; ++b)
    for (int q = 0; q < 6; ++q) sums[q] += part[6 * static_cast<size_t>(b) + q];
  const double denom = static_cast<double>(std::max<long long>(n, 1));
  const Acc& a = *B.h_acc;
  out->steps = steps;
  out->solver_failure_count = failures;
  out->gmres_iterations_max = it_max;
  out->enthalpy_guard_count = a.guard;
  out->nonfinite_count = a.nonfinite + dt_nonfinite;
  out->nonpositive_count = a.nonpositive;
  out->final_time = time;
  out->pressure_residual_linf_max = res_max;
  out->pressure_relative_residual_linf_max = rel_max;
  out->rho_min = key_to_double(a.rho_min_key);
  out->pressure_min = key_to_double(a.p_min_key);
  out->density_l1_error = sums[0] / denom;
  out->velocity_l1_error = sums[1] / denom;
  out->pressure_l1_error = sums[2] / denom;
  out->density_l2_error = std::sqrt(sums[3] / denom);
  out->velocity_l2_error = std::sqrt(sums[4] / denom);
  out->pressure_l2_error = std::sqrt(sums[5] / denom);
  out->density_linf_error = key_to_double(a.drho_max_key);
  out->pressure_linf_error = key_to_double(a.dp_max_key);
  const bool finished = time >= cfg.stop_time - 1.0e-12;
  out->passed = finished && failures == 0 && out->nonfinite_count == 0 && out->nonpositive_count == 0;
  return ECG_OK;
}
