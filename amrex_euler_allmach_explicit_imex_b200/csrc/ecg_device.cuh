// Device numerics of the euler_compare hot path (FP64).
//
// Every expression keeps the operand order of the reference line it cites so
// that the translation unit compiled with -fmad=false (ECG_ARITH_EXACT) is
// bit-identical to the reference CPU build; the -fmad=true build
// (ECG_ARITH_FAST) differs only by FMA contraction.  Paths are relative to
// amrex/apps/euler_compare/src/euler_compare/.
//
// This header is included inside a per-arithmetic namespace (ECG_NS) by
// stencil.cuh, so both builds can live in one library.
#pragma once

struct Cons { double rho, mx, my, E; };
struct Prim { double rho, u, v, p; };

// amrex::min / amrex::max are std::min / std::max (AMReX_Algorithm.H:20-56):
// they return the first argument unless the second compares strictly smaller
// (larger).  fmin/fmax differ for NaN and signed zero, so they are not used.
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// to_primitive, core/state_primitives.hpp:103-111
__device__ __forceinline__ Prim to_prim(const Cons& c, double g)
{
  const double inv_rho = 1.0 / c.rho;
  const double u = c.mx * inv_rho;
  const double v = c.my * inv_rho;
  const double kin = 0.5 * c.rho * (u * u + v * v);
  return Prim{c.rho, u, v, (g - 1.0) * (c.E - kin)};
}

// to_conserved, state_primitives.hpp:113-117
__device__ __forceinline__ Cons to_cons(const Prim& q, double g)
{
  const double kin = 0.5 * q.rho * (q.u * q.u + q.v * q.v);
  return Cons{q.rho, q.rho * q.u, q.rho * q.v, q.p / (g - 1.0) + kin};
}

// sound_speed, state_primitives.hpp:202-205
__device__ __forceinline__ double csound(const Prim& q, double g) { return sqrt(g * q.p / q.rho); }

// minmod, state_primitives.hpp:57-63
__device__ __forceinline__ double minmod(double a, double b)
{
  if (a * b <= 0.0) return 0.0;
  return fabs(a) < fabs(b) ? a : b;
}

// limited_slope, state_primitives.hpp:71-91 (0 minmod, 1 MC, 2 van Leer)
__device__ __forceinline__ double limited_slope(double bk, double fw, int lim)
{
  if (bk * fw <= 0.0) return 0.0;
  if (lim == 1) return minmod(minmod(2.0 * bk, 0.5 * (bk + fw)), 2.0 * fw);
  if (lim == 2) {
    const double d = bk + fw;
    if (fabs(d) <= 1.0e-14) return 0.0;
    return 2.0 * bk * fw / d;
  }
  return minmod(bk, fw);
}

// One component of reconstruct_state, reconstruction_fluxes.hpp:2-24:
// q + (0.5*side) * limited_slope(q - qm, qp - q).
__device__ __forceinline__ double recon1(double qm, double q, double qp, double half_side, int lim)
{
  return q + half_side * limited_slope(q - qm, qp - q, lim);
}

__device__ __forceinline__ double normal_vel(const Prim& q, int axis) { return axis == 0 ? q.u : q.v; }

// physical_flux, reconstruction_fluxes.hpp:66-74
__device__ __forceinline__ Cons pflux(const Prim& q, const Cons& u, int axis)
{
  if (axis == 0) return Cons{u.mx, u.mx * q.u + q.p, u.my * q.u, (u.E + q.p) * q.u};
  return Cons{u.my, u.mx * q.v, u.my * q.v + q.p, (u.E + q.p) * q.v};
}

// rusanov_flux, reconstruction_fluxes.hpp:82-92
static __device__ __noinline__ Cons rusanov_flux(const Prim& l, const Prim& r, int axis, double g)
{
  const Cons ul = to_cons(l, g), ur = to_cons(r, g);
  const Cons fl = pflux(l, ul, axis), fr = pflux(r, ur, axis);
  const double sm = smax(fabs(normal_vel(l, axis)) + csound(l, g), fabs(normal_vel(r, axis)) + csound(r, g));
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
              0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// hllc_flux, reconstruction_fluxes.hpp:151-210.  `degenerate` reports whether
// hllc_star_state_is_degenerate (:117-149) holds for these states: the same
// three conditions that send hllc_flux to its Rusanov fallback.
__device__ __forceinline__ Cons hllc_flux(const Prim& l, const Prim& r, int axis, double g, bool& degenerate)
{
  const double unl = normal_vel(l, axis), unr = normal_vel(r, axis);
  const double cl = csound(l, g), cr = csound(r, g);
  const double sl = smin(unl - cl, unr - cr), sr = smax(unl + cl, unr + cr);
  degenerate = false;
  if (!(sl < sr)) {
    degenerate = true;
    return rusanov_flux(l, r, axis, g);
  }
  const bool left_super = sl >= 0.0, right_super = sr <= 0.0;
  if (left_super || right_super) {
    const Prim& q = left_super ? l : r;
    return pflux(q, to_cons(q, g), axis);
  }
  const double den = l.rho * (sl - unl) - r.rho * (sr - unr);
  if (fabs(den) <= 1.0e-12) {
    degenerate = true;
    return rusanov_flux(l, r, axis, g);
  }
  const double sm = (r.p - l.p + l.rho * unl * (sl - unl) - r.rho * unr * (sr - unr)) / den;
  const double lsd = sl - sm, rsd = sr - sm;
  if (fabs(lsd) <= 1.0e-12 || fabs(rsd) <= 1.0e-12) {
    degenerate = true;
    return rusanov_flux(l, r, axis, g);
  }
  const double psl = l.p + l.rho * (sl - unl) * (sm - unl);
  const double psr = r.p + r.rho * (sr - unr) * (sm - unr);
  const double ps = 0.5 * (psl + psr);
  // Only the upwind star state enters the flux (reconstruction_fluxes.hpp:206-209).
  const bool use_left = sm >= 0.0;
  const Prim q = use_left ? l : r;
  const double s = use_left ? sl : sr, un = use_left ? unl : unr, sd = use_left ? lsd : rsd;
  const Cons u = to_cons(q, g);
  const Cons f = pflux(q, u, axis);
  const double rs = q.rho * (s - un) / sd;
  const double es = ((s - un) * u.E - q.p * un + ps * sm) / sd;
  const double tang = axis == 0 ? q.v : q.u;
  const double smx = axis == 0 ? rs * sm : rs * tang;
  const double smy = axis == 0 ? rs * tang : rs * sm;
  return Cons{f.rho + s * (rs - u.rho), f.mx + s * (smx - u.mx), f.my + s * (smy - u.my), f.E + s * (es - u.E)};
}

// low_mach_correct_velocity_states, reconstruction_fluxes.hpp:212-232
__device__ __forceinline__ void lowmach_correct(Prim& l, Prim& r, double g)
{
  const double al = csound(l, g), ar = csound(r, g);
  const double spl = sqrt(l.u * l.u + l.v * l.v), spr = sqrt(r.u * r.u + r.v * r.v);
  const double ml = spl / smax(al, 1.0e-12), mr = spr / smax(ar, 1.0e-12);
  const double z = smin(smax(smax(ml, mr), 0.0), 1.0);
  const double ua = 0.5 * (l.u + r.u), va = 0.5 * (l.v + r.v);
  const double lu = ua + 0.5 * z * (l.u - r.u);
  const double ru = ua + 0.5 * z * (r.u - l.u);
  const double lv = va + 0.5 * z * (l.v - r.v);
  const double rv = va + 0.5 * z * (r.v - l.v);
  l.u = lu;
  r.u = ru;
  l.v = lv;
  r.v = rv;
}

__device__ __forceinline__ double clamp01(double v) { return smin(smax(v, 0.0), 1.0); }

// xie_am_hllc_p_flux, reconstruction_fluxes.hpp:254-371.  `degenerate` is the
// HLLC degeneracy of the same (uncorrected) states, as
// count_hllc_degenerate_star_states evaluates it (explicit_update.hpp:17-50).
static __device__ __noinline__ Cons xie_flux(const Prim& l, const Prim& r, int axis, double g, double sensor, bool& degenerate)
{
  const double ql = normal_vel(l, axis), qr = normal_vel(r, axis);
  const double pl = l.p, pr = r.p;
  const double cl = csound(l, g), cr = csound(r, g);
  const double sl = smin(ql - cl, qr - cr), sr = smax(ql + cl, qr + cr);
  degenerate = false;
  if (!(sl < sr)) return hllc_flux(l, r, axis, g, degenerate);
  if (sl >= 0.0) return pflux(l, to_cons(l, g), axis);
  if (sr <= 0.0) return pflux(r, to_cons(r, g), axis);
  {
    // degeneracy test of hllc_star_state_is_degenerate on these states
    const double den = l.rho * (sl - ql) - r.rho * (sr - qr);
    if (fabs(den) <= 1.0e-12) {
      degenerate = true;
    } else {
      const double sm = (r.p - l.p + l.rho * ql * (sl - ql) - r.rho * qr * (sr - qr)) / den;
      degenerate = fabs(sl - sm) <= 1.0e-12 || fabs(sr - sm) <= 1.0e-12;
    }
  }
  bool dummy;
  const double al = l.rho * (sl - ql), ar = r.rho * (sr - qr);
  const double ad = ar - al;
  if (fabs(ad) <= 1.0e-12) return hllc_flux(l, r, axis, g, dummy);
  const double ss = (ar * qr - al * ql + pl - pr) / ad;
  const double dl = sl - ss, dr = sr - ss;
  if (fabs(dl) <= 1.0e-12 || fabs(dr) <= 1.0e-12 || fabs(al) <= 1.0e-12 || fabs(ar) <= 1.0e-12)
    return hllc_flux(l, r, axis, g, dummy);
  const Cons ul = to_cons(l, g), ur = to_cons(r, g);
  const double ps = (ar * pl - al * pr - al * ar * (ql - qr)) / ad;
  const double srl = sqrt(l.rho), srr = sqrt(r.rho);
  const double rd = srl + srr;
  if (!(rd > 0.0)) return hllc_flux(l, r, axis, g, dummy);
  const double uh = (srl * l.u + srr * r.u) / rd;
  const double vh = (srl * l.v + srr * r.v) / rd;
  const double qh = axis == 0 ? uh : vh;
  const double hl = (ul.E + pl) / l.rho, hr = (ur.E + pr) / r.rho;
  const double hh = (srl * hl + srr * hr) / rd;
  const double c2 = (g - 1.0) * (hh - 0.5 * (uh * uh + vh * vh));
  if (!(c2 > 0.0) || !isfinite(c2)) return hllc_flux(l, r, axis, g, dummy);
  const double ch = sqrt(c2);
  const double mh = qh / smax(ch, 1.0e-12);
  const double spl = sqrt(l.u * l.u + l.v * l.v), spr = sqrt(r.u * r.u + r.v * r.v);
  const double th = clamp01(smax(spl / smax(cl, 1.0e-12), spr / smax(cr, 1.0e-12)));
  const double f = clamp01(sensor);
  const double pss = th * ps + (1.0 - th) * 0.5 * (pl + pr);
  const double psss = f * pss + (1.0 - f) * ps;
  const double bp = (f - 1.0) * sl * sr / (sr - sl) * (pr - pl) / (c2 * (1.0 + fabs(mh)));
  const double nxv = axis == 0 ? 1.0 : 0.0, nyv = axis == 1 ? 1.0 : 0.0;
  const bool use_left = ss >= 0.0;
  const Prim q = use_left ? l : r;
  const double qn = use_left ? ql : qr;
  const double rs = use_left ? al / dl : ar / dr;
  const double e = use_left ? ul.E / l.rho : ur.E / r.rho;
  const double es = e + (ss - qn) * (ss + (use_left ? pl / al : pr / ar));
  const Cons out{rs * ss + bp,
                 rs * ss * (q.u + nxv * (ss - qn)) + nxv * psss + bp * uh,
                 rs * ss * (q.v + nyv * (ss - qn)) + nyv * psss + bp * vh,
                 ss * (rs * es + ps) + 0.5 * bp * (uh * uh + vh * vh)};
  if (!isfinite(out.rho) || !isfinite(out.mx) || !isfinite(out.my) || !isfinite(out.E))
    return hllc_flux(l, r, axis, g, dummy);
  return out;
}

// xie_pressure_ratio_from_states on face pressures, reconstruction_fluxes.hpp:390-397
__device__ __forceinline__ double pressure_ratio(double pl_in, double pr_in)
{
  const double floor = 1.0e-14;
  const double pl = isfinite(pl_in) ? smax(pl_in, floor) : floor;
  const double pr = isfinite(pr_in) ? smax(pr_in, floor) : floor;
  return clamp01(smin(pl / pr, pr / pl));
}

// Ordered 64-bit keys for IEEE doubles: key(a) < key(b) iff a < b (with
// -0 < +0), so unsigned integer atomics implement exact min/max reductions.
__device__ __forceinline__ unsigned long long okey(double x)
{
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double okey_inv(unsigned long long k)
{
  const unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  return __longlong_as_double(static_cast<long long>(b));
}
