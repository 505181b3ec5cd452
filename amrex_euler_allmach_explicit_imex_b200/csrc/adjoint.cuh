// Local Jacobians of the explicit step for its adjoint (adjoint.cu).
//
// The face flux of euler_fv_one_step is restated over a generic number type
// T: `double` gives the forward value, `Dual` (value + one directional
// derivative) gives one column of the face Jacobian per evaluation.  Branches
// (limiter cases, Riemann fallbacks, upwind side, std::min/max) are taken on
// values, so each column is the derivative of the branch the forward step
// takes.  Formulas and branch order follow the reference lines cited at each
// function (paths relative to amrex/apps/euler_compare/src/euler_compare/).
#pragma once

#include <math.h>

namespace ecg_adj {

struct Dual {
  double v, d;
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual{-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
  const double q = a.v / b.v;
  return Dual{q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual{a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return Dual{a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator+(Dual a, double b) { return Dual{a.v + b, a.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return Dual{a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return Dual{a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return Dual{a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b)
{
  const double q = a / b.v;
  return Dual{q, -q * b.d / b.v};
}

__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Dual a) { return a.v; }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ Dual dsqrt(Dual a)
{
  const double s = sqrt(a.v);
  return Dual{s, s > 0.0 ? 0.5 * a.d / s : 0.0};
}
__device__ __forceinline__ double dabs(double a) { return fabs(a); }
__device__ __forceinline__ Dual dabs(Dual a) { return a.v < 0.0 ? -a : a; }
// std::min / std::max semantics (first argument unless the second is strictly smaller / larger)
template <class T> __device__ __forceinline__ T tmin(T a, T b) { return val(b) < val(a) ? b : a; }
template <class T> __device__ __forceinline__ T tmax(T a, T b) { return val(a) < val(b) ? b : a; }
template <class T> __device__ __forceinline__ T lit(double x) { return T(x); }
template <> __device__ __forceinline__ Dual lit<Dual>(double x) { return Dual{x, 0.0}; }

template <class T> struct P4 { T rho, u, v, p; };
template <class T> struct C4 { T rho, mx, my, E; };

// minmod / limited_slope, core/state_primitives.hpp:57-91
template <class T> __device__ __forceinline__ T t_minmod(T a, T b)
{
  if (val(a) * val(b) <= 0.0) return lit<T>(0.0);
  return fabs(val(a)) < fabs(val(b)) ? a : b;
}
template <class T> __device__ __forceinline__ T t_slope(T bk, T fw, int lim)
{
  if (val(bk) * val(fw) <= 0.0) return lit<T>(0.0);
  if (lim == 1) return t_minmod(t_minmod(2.0 * bk, 0.5 * (bk + fw)), 2.0 * fw);
  if (lim == 2) {
    const T d = bk + fw;
    if (fabs(val(d)) <= 1.0e-14) return lit<T>(0.0);
    return 2.0 * bk * fw / d;
  }
  return t_minmod(bk, fw);
}

template <class T> __device__ __forceinline__ C4<T> t_cons(const P4<T>& q, double g)
{
  const T kin = 0.5 * q.rho * (q.u * q.u + q.v * q.v);
  return C4<T>{q.rho, q.rho * q.u, q.rho * q.v, q.p / (g - 1.0) + kin};
}
template <class T> __device__ __forceinline__ T t_sound(const P4<T>& q, double g) { return dsqrt(g * q.p / q.rho); }
template <class T> __device__ __forceinline__ T t_un(const P4<T>& q, int axis) { return axis == 0 ? q.u : q.v; }

// physical_flux, reconstruction_fluxes.hpp:66-74
template <class T> __device__ __forceinline__ C4<T> t_pflux(const P4<T>& q, const C4<T>& u, int axis)
{
  if (axis == 0) return C4<T>{u.mx, u.mx * q.u + q.p, u.my * q.u, (u.E + q.p) * q.u};
  return C4<T>{u.my, u.mx * q.v, u.my * q.v + q.p, (u.E + q.p) * q.v};
}

// rusanov_flux, reconstruction_fluxes.hpp:82-92
template <class T> __device__ C4<T> t_rusanov(const P4<T>& l, const P4<T>& r, int axis, double g)
{
  const C4<T> ul = t_cons(l, g), ur = t_cons(r, g);
  const C4<T> fl = t_pflux(l, ul, axis), fr = t_pflux(r, ur, axis);
  const T sm = tmax(dabs(t_un(l, axis)) + t_sound(l, g), dabs(t_un(r, axis)) + t_sound(r, g));
  const T hs = 0.5 * sm;
  return C4<T>{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
               0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// hllc_flux, reconstruction_fluxes.hpp:151-210
template <class T> __device__ C4<T> t_hllc(const P4<T>& l, const P4<T>& r, int axis, double g)
{
  const T unl = t_un(l, axis), unr = t_un(r, axis);
  const T cl = t_sound(l, g), cr = t_sound(r, g);
  const T sl = tmin(unl - cl, unr - cr), sr = tmax(unl + cl, unr + cr);
  if (!(val(sl) < val(sr))) return t_rusanov(l, r, axis, g);
  const bool left_super = val(sl) >= 0.0, right_super = val(sr) <= 0.0;
  if (left_super || right_super) {
    const P4<T>& q = left_super ? l : r;
    return t_pflux(q, t_cons(q, g), axis);
  }
  const T den = l.rho * (sl - unl) - r.rho * (sr - unr);
  if (fabs(val(den)) <= 1.0e-12) return t_rusanov(l, r, axis, g);
  const T sm = (r.p - l.p + l.rho * unl * (sl - unl) - r.rho * unr * (sr - unr)) / den;
  const T lsd = sl - sm, rsd = sr - sm;
  if (fabs(val(lsd)) <= 1.0e-12 || fabs(val(rsd)) <= 1.0e-12) return t_rusanov(l, r, axis, g);
  const T psl = l.p + l.rho * (sl - unl) * (sm - unl);
  const T psr = r.p + r.rho * (sr - unr) * (sm - unr);
  const T ps = 0.5 * (psl + psr);
  const bool use_left = val(sm) >= 0.0;
  const P4<T> q = use_left ? l : r;
  const T s = use_left ? sl : sr, un = use_left ? unl : unr, sd = use_left ? lsd : rsd;
  const C4<T> u = t_cons(q, g);
  const C4<T> f = t_pflux(q, u, axis);
  const T rs = q.rho * (s - un) / sd;
  const T es = ((s - un) * u.E - q.p * un + ps * sm) / sd;
  const T tang = axis == 0 ? q.v : q.u;
  const T smx = axis == 0 ? rs * sm : rs * tang;
  const T smy = axis == 0 ? rs * tang : rs * sm;
  return C4<T>{f.rho + s * (rs - u.rho), f.mx + s * (smx - u.mx), f.my + s * (smy - u.my), f.E + s * (es - u.E)};
}

// low_mach_correct_velocity_states, reconstruction_fluxes.hpp:212-232
template <class T> __device__ void t_lowmach(P4<T>& l, P4<T>& r, double g)
{
  const T al = t_sound(l, g), ar = t_sound(r, g);
  const T spl = dsqrt(l.u * l.u + l.v * l.v), spr = dsqrt(r.u * r.u + r.v * r.v);
  const T ml = spl / tmax(al, lit<T>(1.0e-12)), mr = spr / tmax(ar, lit<T>(1.0e-12));
  const T z = tmin(tmax(tmax(ml, mr), lit<T>(0.0)), lit<T>(1.0));
  const T ua = 0.5 * (l.u + r.u), va = 0.5 * (l.v + r.v);
  const T lu = ua + 0.5 * z * (l.u - r.u);
  const T ru = ua + 0.5 * z * (r.u - l.u);
  const T lv = va + 0.5 * z * (l.v - r.v);
  const T rv = va + 0.5 * z * (r.v - l.v);
  l.u = lu;
  r.u = ru;
  l.v = lv;
  r.v = rv;
}

// reconstructed_interface_flux (reconstruction_fluxes.hpp:442-460) of the face
// between cells b = c[1] and c = c[2] of the 4-cell line c[0..3] along `axis`.
template <class T>
__device__ C4<T> t_face_flux(const P4<T> c[4], int axis, double g, int riemann, int order, int lim)
{
  P4<T> l = c[1], r = c[2];
  if (order > 1) {
    // reconstruct_state (:2-24): right face of c[1], left face of c[2]
    l.rho = c[1].rho + 0.5 * t_slope(c[1].rho - c[0].rho, c[2].rho - c[1].rho, lim);
    l.u = c[1].u + 0.5 * t_slope(c[1].u - c[0].u, c[2].u - c[1].u, lim);
    l.v = c[1].v + 0.5 * t_slope(c[1].v - c[0].v, c[2].v - c[1].v, lim);
    l.p = c[1].p + 0.5 * t_slope(c[1].p - c[0].p, c[2].p - c[1].p, lim);
    r.rho = c[2].rho + -0.5 * t_slope(c[2].rho - c[1].rho, c[3].rho - c[2].rho, lim);
    r.u = c[2].u + -0.5 * t_slope(c[2].u - c[1].u, c[3].u - c[2].u, lim);
    r.v = c[2].v + -0.5 * t_slope(c[2].v - c[1].v, c[3].v - c[2].v, lim);
    r.p = c[2].p + -0.5 * t_slope(c[2].p - c[1].p, c[3].p - c[2].p, lim);
  }
  if (riemann == ECG_RIEMANN_RUSANOV) return t_rusanov(l, r, axis, g);
  if (riemann == ECG_RIEMANN_LOWMACH_HLLC) t_lowmach(l, r, g);
  return t_hllc(l, r, axis, g);
}

}  // namespace ecg_adj
