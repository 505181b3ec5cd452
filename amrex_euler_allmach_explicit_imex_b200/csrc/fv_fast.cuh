// Fast (default) explicit step: the same numerics as fv_step_kernel in a
// formulation that trades IEEE-rounded division and square root for
// Newton-refined hardware approximations and removes redundant work.
// Included inside the ecg_fast namespace of stencil.cuh.
//
//  * Division and square root: the PTX approximations rcp.approx.ftz.f64 and
//    rsqrt.approx.ftz.f64 (about 2^-20 relative, measured on B200) refined by
//    one third-order Householder step each, which takes the error to a few
//    units in the last place; a quotient is a * (1/b).
//  * Sound speed sqrt(g p / rho) = (g p) * rsqrt(g p rho): no division.
//  * HLLC star state: one reciprocal of (s_K - s_M) for density and energy.
//  * MUSCL: the limited slope of every cell and axis is computed once per
//    tile (the reference recomputes it for each face a cell touches).
//  * Square T x T tiles with T(T+1) threads: each thread evaluates exactly one
//    x-face and one y-face, so no thread idles at the face barrier.
namespace fast {

// 1/b: the hardware approximation (about 2^-20 relative) refined by one
// third-order step y (1 + e + e^2), e = 1 - b y (error about e^3).
__device__ __forceinline__ double frcp(double b)
{
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  const double e = fma(-b, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

__device__ __forceinline__ double fdiv(double a, double b) { return a * frcp(b); }

// 1/sqrt(x): the hardware approximation refined by one third-order step
// y (1 + e/2 + 3e^2/8), e = 1 - x y^2.
__device__ __forceinline__ double frsqrt(double x)
{
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}

// sqrt(x) for x > 0 via x * rsqrt(x); IEEE sqrt for 0, negative, inf, NaN.
__device__ __forceinline__ double fsqrt(double x)
{
  if (!(x > 0.0) || !(x < 1.0e300)) return sqrt(x);
  return x * frsqrt(x);
}

// sound_speed sqrt(g p / rho) without a division.
__device__ __forceinline__ double fsound(double rho, double p, double g)
{
  const double t = g * p;
  const double q = t * rho;
  if (!(q > 0.0) || !(q < 1.0e300)) return sqrt(t / rho);
  return t * frsqrt(q);
}

__device__ __forceinline__ Prim to_prim_f(const Cons& c, double g)
{
  const double inv_rho = frcp(c.rho);
  const double u = c.mx * inv_rho;
  const double v = c.my * inv_rho;
  const double kin = 0.5 * c.rho * (u * u + v * v);
  return Prim{c.rho, u, v, (g - 1.0) * (c.E - kin)};
}

__device__ __forceinline__ Cons to_cons_f(const Prim& q, double inv_gm1)
{
  const double kin = 0.5 * q.rho * (q.u * q.u + q.v * q.v);
  return Cons{q.rho, q.rho * q.u, q.rho * q.v, fma(q.p, inv_gm1, kin)};
}

__device__ __forceinline__ Cons rusanov_i(const Prim& l, const Prim& r, int axis, double g, double inv_gm1)
{
  const Cons ul = to_cons_f(l, inv_gm1), ur = to_cons_f(r, inv_gm1);
  const Cons fl = pflux(l, ul, axis), fr = pflux(r, ur, axis);
  const double sm = smax(fabs(normal_vel(l, axis)) + fsound(l.rho, l.p, g),
                         fabs(normal_vel(r, axis)) + fsound(r.rho, r.p, g));
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
              0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// Out-of-line copy for the rarely taken fallbacks; arguments by value so
// they travel in registers rather than through the stack.
static __device__ __noinline__ Cons rusanov_f(Prim l, Prim r, int axis, double g, double inv_gm1)
{
  return rusanov_i(l, r, axis, g, inv_gm1);
}

// hllc_flux (reconstruction_fluxes.hpp:151-210), fast arithmetic.  deg: the
// star-state degeneracy test (:117-149) of these states.
__device__ __forceinline__ Cons hllc_f(const Prim& l, const Prim& r, int axis, double g, double inv_gm1, bool& deg)
{
  const double unl = normal_vel(l, axis), unr = normal_vel(r, axis);
  const double cl = fsound(l.rho, l.p, g), cr = fsound(r.rho, r.p, g);
  const double sl = smin(unl - cl, unr - cr), sr = smax(unl + cl, unr + cr);
  deg = true;
  // The three degenerate exits share one inline Rusanov evaluation at the end.
  if (sl < sr) {
    if (sl >= 0.0 || sr <= 0.0) {
      deg = false;
      const Prim& q = sl >= 0.0 ? l : r;
      return pflux(q, to_cons_f(q, inv_gm1), axis);
    }
    const double al = l.rho * (sl - unl), ar = r.rho * (sr - unr);
    const double den = al - ar;
    if (!(fabs(den) <= 1.0e-12)) {
      const double sm = fdiv(r.p - l.p + al * unl - ar * unr, den);
      const double lsd = sl - sm, rsd = sr - sm;
      if (!(fabs(lsd) <= 1.0e-12 || fabs(rsd) <= 1.0e-12)) {
        deg = false;
        const double ps = 0.5 * (l.p + al * (sm - unl) + r.p + ar * (sm - unr));
        const bool left = sm >= 0.0;
        const Prim q = left ? l : r;
        const double s = left ? sl : sr, un = left ? unl : unr, a = left ? al : ar;
        const double inv_sd = frcp(left ? lsd : rsd);
        const Cons u = to_cons_f(q, inv_gm1);
        const Cons f = pflux(q, u, axis);
        const double rs = a * inv_sd;
        const double es = ((s - un) * u.E - q.p * un + ps * sm) * inv_sd;
        const double tang = axis == 0 ? q.v : q.u;
        const double smx = axis == 0 ? rs * sm : rs * tang;
        const double smy = axis == 0 ? rs * tang : rs * sm;
        return Cons{fma(s, rs - u.rho, f.rho), fma(s, smx - u.mx, f.mx), fma(s, smy - u.my, f.my),
                    fma(s, es - u.E, f.E)};
      }
    }
  }
  return rusanov_i(l, r, axis, g, inv_gm1);
}

// 0 < x < 1e300 by one unsigned integer compare of the bit pattern (positive
// doubles order like their bits; zero, negatives, NaN and huge values fail).
__device__ __forceinline__ bool pos_normal_range(double x)
{
  constexpr unsigned long long kHi = 0x7E37E43C8800759CULL;  // bits of 1.0e300
  return static_cast<unsigned long long>(__double_as_longlong(x)) - 1ULL < kHi - 1ULL;
}

// fsound for whole warps: the rsqrt path, and the IEEE formula only when some
// lane of the warp has a state outside (0, 1e300) (a uniform branch).
__device__ __forceinline__ double fsound_w(double rho, double p, double g)
{
  const double t = g * p;
  const double q = t * rho;
  double c = t * frsqrt(q);
  const bool ok = pos_normal_range(q);
  if (__any_sync(0xffffffffu, !ok)) {
    if (!ok) c = sqrt(t / rho);
  }
  return c;
}

// hllc_flux of hllc_f without divergent branches: every lane evaluates the
// star-state flux of its upwind side, supersonic faces select the plain
// physical flux, and the Rusanov fallback (the three degenerate cases of
// reconstruction_fluxes.hpp:151-210) runs only when some lane of the warp
// needs it.  deg: that fallback was taken.
__device__ __forceinline__ Cons hllc_w(const Prim& l, const Prim& r, int axis, double g, double inv_gm1, bool& deg)
{
  const double unl = normal_vel(l, axis), unr = normal_vel(r, axis);
  const double cl = fsound_w(l.rho, l.p, g), cr = fsound_w(r.rho, r.p, g);
  const double sl = smin(unl - cl, unr - cr), sr = smax(unl + cl, unr + cr);
  const bool ordered = sl < sr;
  const bool sup_l = sl >= 0.0, sup_r = sr <= 0.0;
  const bool supersonic = ordered && (sup_l || sup_r);
  const double al = l.rho * (sl - unl), ar = r.rho * (sr - unr);
  const double den = al - ar;
  const double sm = fdiv(r.p - l.p + al * unl - ar * unr, den);
  const double lsd = sl - sm, rsd = sr - sm;
  deg = !ordered || (!supersonic && (fabs(den) <= 1.0e-12 || fabs(lsd) <= 1.0e-12 || fabs(rsd) <= 1.0e-12));
  const bool left = supersonic ? sup_l : sm >= 0.0;
  const Prim q = left ? l : r;
  const double s = left ? sl : sr, un = left ? unl : unr, a = left ? al : ar;
  const Cons u = to_cons_f(q, inv_gm1);
  const Cons f = pflux(q, u, axis);
  const double ps = 0.5 * (l.p + al * (sm - unl) + r.p + ar * (sm - unr));
  const double inv_sd = frcp(left ? lsd : rsd);
  const double rs = a * inv_sd;
  const double es = ((s - un) * u.E - q.p * un + ps * sm) * inv_sd;
  const double tang = axis == 0 ? q.v : q.u;
  const double smx = axis == 0 ? rs * sm : rs * tang;
  const double smy = axis == 0 ? rs * tang : rs * sm;
  Cons out;
  out.rho = supersonic ? f.rho : fma(s, rs - u.rho, f.rho);
  out.mx = supersonic ? f.mx : fma(s, smx - u.mx, f.mx);
  out.my = supersonic ? f.my : fma(s, smy - u.my, f.my);
  out.E = supersonic ? f.E : fma(s, es - u.E, f.E);
  if (__any_sync(0xffffffffu, deg)) {
    const Cons rf = rusanov_i(l, r, axis, g, inv_gm1);
    if (deg) out = rf;
  }
  return out;
}

// Sound speed on the rsqrt path only; `bad` marks states outside (0, 1e300)
// whose speed must come from the IEEE formula instead.
__device__ __forceinline__ double fsound_core(double rho, double p, double g, bool& bad)
{
  const double t = g * p;
  const double q = t * rho;
  bad = !pos_normal_range(q);
  return t * frsqrt(q);
}

// hllc_w without any warp vote: the branch-free HLLC flux of states whose
// sound speeds are on the rsqrt path and whose star state is not degenerate.
// `fallback` marks the faces that must be recomputed by hllc_f instead
// (degenerate star state or a sound speed off the rsqrt path), so two faces
// can be evaluated back to back and repaired by one vote.
__device__ __forceinline__ Cons hllc_core(const Prim& l, const Prim& r, int axis, double g, double inv_gm1,
                                          bool& fallback)
{
  const double unl = normal_vel(l, axis), unr = normal_vel(r, axis);
  bool bl, br;
  const double cl = fsound_core(l.rho, l.p, g, bl), cr = fsound_core(r.rho, r.p, g, br);
  const double sl = smin(unl - cl, unr - cr), sr = smax(unl + cl, unr + cr);
  const bool ordered = sl < sr;
  const bool sup_l = sl >= 0.0, sup_r = sr <= 0.0;
  const bool supersonic = ordered && (sup_l || sup_r);
  const double al = l.rho * (sl - unl), ar = r.rho * (sr - unr);
  const double den = al - ar;
  const double sm = fdiv(r.p - l.p + al * unl - ar * unr, den);
  const double lsd = sl - sm, rsd = sr - sm;
  const bool deg = !ordered || (!supersonic && (fabs(den) <= 1.0e-12 || fabs(lsd) <= 1.0e-12 || fabs(rsd) <= 1.0e-12));
  fallback = deg || bl || br;
  const bool left = supersonic ? sup_l : sm >= 0.0;
  const Prim q = left ? l : r;
  const double s = left ? sl : sr, un = left ? unl : unr, a = left ? al : ar;
  const Cons u = to_cons_f(q, inv_gm1);
  const Cons f = pflux(q, u, axis);
  const double ps = 0.5 * (l.p + al * (sm - unl) + r.p + ar * (sm - unr));
  const double inv_sd = frcp(left ? lsd : rsd);
  const double rs = a * inv_sd;
  const double es = ((s - un) * u.E - q.p * un + ps * sm) * inv_sd;
  const double tang = axis == 0 ? q.v : q.u;
  const double smx = axis == 0 ? rs * sm : rs * tang;
  const double smy = axis == 0 ? rs * tang : rs * sm;
  Cons out;
  out.rho = supersonic ? f.rho : fma(s, rs - u.rho, f.rho);
  out.mx = supersonic ? f.mx : fma(s, smx - u.mx, f.mx);
  out.my = supersonic ? f.my : fma(s, smy - u.my, f.my);
  out.E = supersonic ? f.E : fma(s, es - u.E, f.E);
  return out;
}

// rusanov_i on the rsqrt path; `fallback` as for hllc_core.
__device__ __forceinline__ Cons rusanov_core(const Prim& l, const Prim& r, int axis, double g, double inv_gm1,
                                             bool& fallback)
{
  const Cons ul = to_cons_f(l, inv_gm1), ur = to_cons_f(r, inv_gm1);
  const Cons fl = pflux(l, ul, axis), fr = pflux(r, ur, axis);
  bool bl, br;
  const double cl = fsound_core(l.rho, l.p, g, bl), cr = fsound_core(r.rho, r.p, g, br);
  fallback = bl || br;
  const double sm = smax(fabs(normal_vel(l, axis)) + cl, fabs(normal_vel(r, axis)) + cr);
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
              0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// low_mach_correct_velocity_states (reconstruction_fluxes.hpp:212-232), fast arithmetic.
__device__ __forceinline__ void lowmach_f(Prim& l, Prim& r, double g)
{
  const double al = fsound(l.rho, l.p, g), ar = fsound(r.rho, r.p, g);
  const double ml = fdiv(fsqrt(l.u * l.u + l.v * l.v), smax(al, 1.0e-12));
  const double mr = fdiv(fsqrt(r.u * r.u + r.v * r.v), smax(ar, 1.0e-12));
  const double z = smin(smax(smax(ml, mr), 0.0), 1.0);
  const double ua = 0.5 * (l.u + r.u), va = 0.5 * (l.v + r.v);
  const double hz = 0.5 * z;
  const double lu = ua + hz * (l.u - r.u), ru = ua + hz * (r.u - l.u);
  const double lv = va + hz * (l.v - r.v), rv = va + hz * (r.v - l.v);
  l.u = lu;
  r.u = ru;
  l.v = lv;
  r.v = rv;
}

// xie_am_hllc_p_flux (reconstruction_fluxes.hpp:254-371), fast arithmetic.
static __device__ __noinline__ Cons xie_f(const Prim l, const Prim r, int axis, double g, double inv_gm1,
                                          double sensor, bool& deg)
{
  const double ql = normal_vel(l, axis), qr = normal_vel(r, axis);
  const double pl = l.p, pr = r.p;
  const double cl = fsound(l.rho, pl, g), cr = fsound(r.rho, pr, g);
  const double sl = smin(ql - cl, qr - cr), sr = smax(ql + cl, qr + cr);
  deg = false;
  if (!(sl < sr)) return hllc_f(l, r, axis, g, inv_gm1, deg);
  if (sl >= 0.0) return pflux(l, to_cons_f(l, inv_gm1), axis);
  if (sr <= 0.0) return pflux(r, to_cons_f(r, inv_gm1), axis);
  const double al = l.rho * (sl - ql), ar = r.rho * (sr - qr);
  const double ad = ar - al;
  if (fabs(ad) <= 1.0e-12) {
    deg = true;  // den of the HLLC test is -ad
    bool dummy;
    return hllc_f(l, r, axis, g, inv_gm1, dummy);
  }
  const double inv_ad = frcp(ad);
  {
    const double sm = (r.p - l.p + al * ql - ar * qr) * -inv_ad;
    deg = fabs(sl - sm) <= 1.0e-12 || fabs(sr - sm) <= 1.0e-12;
  }
  bool dummy;
  const double ss = (ar * qr - al * ql + pl - pr) * inv_ad;
  const double dl = sl - ss, dr = sr - ss;
  if (fabs(dl) <= 1.0e-12 || fabs(dr) <= 1.0e-12 || fabs(al) <= 1.0e-12 || fabs(ar) <= 1.0e-12)
    return hllc_f(l, r, axis, g, inv_gm1, dummy);
  const Cons ul = to_cons_f(l, inv_gm1), ur = to_cons_f(r, inv_gm1);
  const double ps = (ar * pl - al * pr - al * ar * (ql - qr)) * inv_ad;
  const double srl = fsqrt(l.rho), srr = fsqrt(r.rho);
  const double rd = srl + srr;
  if (!(rd > 0.0)) return hllc_f(l, r, axis, g, inv_gm1, dummy);
  const double ird = frcp(rd);
  const double uh = (srl * l.u + srr * r.u) * ird;
  const double vh = (srl * l.v + srr * r.v) * ird;
  const double qh = axis == 0 ? uh : vh;
  const double hl = fdiv(ul.E + pl, l.rho), hr = fdiv(ur.E + pr, r.rho);
  const double hh = (srl * hl + srr * hr) * ird;
  const double c2 = (g - 1.0) * (hh - 0.5 * (uh * uh + vh * vh));
  if (!(c2 > 0.0) || !isfinite(c2)) return hllc_f(l, r, axis, g, inv_gm1, dummy);
  const double ch = fsqrt(c2);
  const double mh = fdiv(qh, smax(ch, 1.0e-12));
  const double spl = fsqrt(l.u * l.u + l.v * l.v), spr = fsqrt(r.u * r.u + r.v * r.v);
  const double th = clamp01(smax(fdiv(spl, smax(cl, 1.0e-12)), fdiv(spr, smax(cr, 1.0e-12))));
  const double f = clamp01(sensor);
  const double pss = th * ps + (1.0 - th) * 0.5 * (pl + pr);
  const double psss = f * pss + (1.0 - f) * ps;
  const double bp = fdiv((f - 1.0) * sl * sr * (pr - pl), (sr - sl) * (c2 * (1.0 + fabs(mh))));
  const double nxv = axis == 0 ? 1.0 : 0.0, nyv = axis == 1 ? 1.0 : 0.0;
  const bool left = ss >= 0.0;
  const Prim q = left ? l : r;
  const double qn = left ? ql : qr;
  const double a = left ? al : ar;
  const double rs = fdiv(a, left ? dl : dr);
  const double e = left ? fdiv(ul.E, l.rho) : fdiv(ur.E, r.rho);
  const double es = e + (ss - qn) * (ss + fdiv(left ? pl : pr, a));
  const double rss = rs * ss;
  const Cons out{rss + bp, rss * (q.u + nxv * (ss - qn)) + nxv * psss + bp * uh,
                 rss * (q.v + nyv * (ss - qn)) + nyv * psss + bp * vh,
                 ss * (rs * es + ps) + 0.5 * bp * (uh * uh + vh * vh)};
  if (!isfinite(out.rho) || !isfinite(out.mx) || !isfinite(out.my) || !isfinite(out.E))
    return hllc_f(l, r, axis, g, inv_gm1, dummy);
  return out;
}

// xie_f without branches: the flux of a face whose states take none of
// xie_f's exits (sound speeds on the rsqrt path, ordered wave speeds, and for
// a subsonic face no degenerate denominator, square roots on their fast path
// and a finite result), evaluated with xie_f's arithmetic in xie_f's order;
// a supersonic face selects the upwind physical flux as xie_f returns it.
// `fallback` marks the faces xie_f must evaluate instead (the caller does so
// after one warp vote); deg: the HLLC degeneracy test, valid without fallback.
__device__ __forceinline__ Cons xie_core(const Prim& l, const Prim& r, int axis, double g, double inv_gm1,
                                         double sensor, bool& fallback, bool& deg)
{
  const double ql = normal_vel(l, axis), qr = normal_vel(r, axis);
  const double pl = l.p, pr = r.p;
  bool bl, br;
  const double cl = fsound_core(l.rho, pl, g, bl), cr = fsound_core(r.rho, pr, g, br);
  const double sl = smin(ql - cl, qr - cr), sr = smax(ql + cl, qr + cr);
  const bool ordered = sl < sr;
  const bool sup_l = sl >= 0.0, sup_r = sr <= 0.0;
  const bool supersonic = sup_l || sup_r;
  const double al = l.rho * (sl - ql), ar = r.rho * (sr - qr);
  const double ad = ar - al;
  const double inv_ad = frcp(ad);
  const double sm = (r.p - l.p + al * ql - ar * qr) * -inv_ad;
  deg = !supersonic && (fabs(sl - sm) <= 1.0e-12 || fabs(sr - sm) <= 1.0e-12);
  const double ss = (ar * qr - al * ql + pl - pr) * inv_ad;
  const double dl = sl - ss, dr = sr - ss;
  const Cons ul = to_cons_f(l, inv_gm1), ur = to_cons_f(r, inv_gm1);
  const double ps = (ar * pl - al * pr - al * ar * (ql - qr)) * inv_ad;
  const double srl = l.rho * frsqrt(l.rho), srr = r.rho * frsqrt(r.rho);
  const double rd = srl + srr;
  const double ird = frcp(rd);
  const double uh = (srl * l.u + srr * r.u) * ird;
  const double vh = (srl * l.v + srr * r.v) * ird;
  const double qh = axis == 0 ? uh : vh;
  const double hl = fdiv(ul.E + pl, l.rho), hr = fdiv(ur.E + pr, r.rho);
  const double hh = (srl * hl + srr * hr) * ird;
  const double c2 = (g - 1.0) * (hh - 0.5 * (uh * uh + vh * vh));
  const double ch = c2 * frsqrt(c2);
  const double mh = fdiv(qh, smax(ch, 1.0e-12));
  // |u| of a state at rest is fsqrt's sqrt(0) = 0: kept on the fast path
  const double sp2l = l.u * l.u + l.v * l.v, sp2r = r.u * r.u + r.v * r.v;
  const bool okl = pos_normal_range(sp2l), okr = pos_normal_range(sp2r);
  const double spl = okl ? sp2l * frsqrt(sp2l) : sp2l, spr = okr ? sp2r * frsqrt(sp2r) : sp2r;
  const double th = clamp01(smax(fdiv(spl, smax(cl, 1.0e-12)), fdiv(spr, smax(cr, 1.0e-12))));
  const double f = clamp01(sensor);
  const double pss = th * ps + (1.0 - th) * 0.5 * (pl + pr);
  const double psss = f * pss + (1.0 - f) * ps;
  const double bp = fdiv((f - 1.0) * sl * sr * (pr - pl), (sr - sl) * (c2 * (1.0 + fabs(mh))));
  const double nxv = axis == 0 ? 1.0 : 0.0, nyv = axis == 1 ? 1.0 : 0.0;
  const bool left = ss >= 0.0;
  const Prim q = left ? l : r;
  const double qn = left ? ql : qr;
  const double a = left ? al : ar;
  const double rs = fdiv(a, left ? dl : dr);
  const double e = left ? fdiv(ul.E, l.rho) : fdiv(ur.E, r.rho);
  const double es = e + (ss - qn) * (ss + fdiv(left ? pl : pr, a));
  const double rss = rs * ss;
  const Cons sub{rss + bp, rss * (q.u + nxv * (ss - qn)) + nxv * psss + bp * uh,
                 rss * (q.v + nyv * (ss - qn)) + nyv * psss + bp * vh,
                 ss * (rs * es + ps) + 0.5 * bp * (uh * uh + vh * vh)};
  // xie_f's exits of a subsonic face, and the square roots fsqrt would take
  // off its rsqrt path (l.rho, r.rho, c2, the speeds; 0 < x < 1e300 there)
  const bool sub_exit = fabs(ad) <= 1.0e-12 || fabs(dl) <= 1.0e-12 || fabs(dr) <= 1.0e-12 ||
                        fabs(al) <= 1.0e-12 || fabs(ar) <= 1.0e-12 || !pos_normal_range(l.rho) ||
                        !pos_normal_range(r.rho) || !(rd > 0.0) || !(c2 > 0.0) || !isfinite(c2) ||
                        !pos_normal_range(c2) || !(okl || sp2l == 0.0) || !(okr || sp2r == 0.0) ||
                        !isfinite(sub.rho) || !isfinite(sub.mx) || !isfinite(sub.my) || !isfinite(sub.E);
  fallback = bl || br || !ordered || (!supersonic && sub_exit);
  if (!supersonic) return sub;
  const Prim& w = sup_l ? l : r;
  return pflux(w, sup_l ? ul : ur, axis);
}

// Face pressure ratio of the multiface sensor (reconstruction_fluxes.hpp:390-397):
// min(pl/pr, pr/pl) of the floored face pressures = min/max.
__device__ __forceinline__ double pratio_f(double pl_in, double pr_in)
{
  const double floor = 1.0e-14;
  const double pl = isfinite(pl_in) ? smax(pl_in, floor) : floor;
  const double pr = isfinite(pr_in) ? smax(pr_in, floor) : floor;
  return clamp01(fdiv(smin(pl, pr), smax(pl, pr)));
}

template <int T, bool XIE>
struct FastSmem {
  static constexpr int RW = T + 4, RN = RW * RW;  // primitive region [-2, T+1]^2
  static constexpr int SW = T + 2, SN = SW * SW;  // slope region [-1, T]^2
  static constexpr int NF = T * (T + 1);           // x-faces (= y-faces) per tile
  static constexpr int NT = (NF + 31) / 32 * 32;   // threads: whole warps
  static constexpr int NXR = XIE ? (T + 1) * (T + 2) : 0;  // x-faces [0,T] on rows [-1,T]
  static constexpr int NYR = XIE ? (T + 2) * (T + 1) : 0;  // y-faces [0,T] on columns [-1,T]
  static constexpr int doubles = 4 * RN + 8 * SN + NXR + NYR;
  static constexpr size_t bytes = sizeof(double) * doubles;
  static_assert(SN >= NF, "flux staging reuses the slope region");
};

template <int RK, int T>
__global__ void __launch_bounds__(FastSmem<T, RK == ECG_RIEMANN_XIE_AM_HLLC_P>::NT, 3)
fv_fast_kernel(const EcgFvParams P, const double* __restrict__ u, double* __restrict__ out,
               EcgStepStats* __restrict__ stats, const EcgDtCtl ctl)
{
  constexpr bool XIE = RK == ECG_RIEMANN_XIE_AM_HLLC_P;
  using S = FastSmem<T, XIE>;
  constexpr int NT = S::NT, NF = S::NF, RW = S::RW, SW = S::SW;
  extern __shared__ double smem[];
  __shared__ BlockRed<NT> red;
  double* q_r = smem;
  double* q_u = q_r + S::RN;
  double* q_v = q_u + S::RN;
  double* q_p = q_v + S::RN;
  double* sl = q_p + S::RN;  // 8 planes: x-slopes rho,u,v,p then y-slopes rho,u,v,p
  double* xr = sl + 8 * S::SN;
  double* yr = xr + S::NXR;

  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * T, j0 = blockIdx.y * T;
  const int nx = P.g.nx, ny = P.g.ny;
  const double g = P.gamma, inv_gm1 = frcp(g - 1.0);

  double dt;
  if (!step_control(stats, ctl, dt)) return;

  auto R = [](int x, int y) { return (y + 2) * RW + (x + 2); };
  auto SI = [](int x, int y) { return (y + 1) * SW + (x + 1); };

  // ---- primitives of the halo region ----
  for (int e = tid; e < S::RN; e += NT) {
    const Prim q = to_prim_f(load_cell(P, u, i0 - 2 + e % RW, j0 - 2 + e / RW), g);
    q_r[e] = q.rho;
    q_u[e] = q.u;
    q_v[e] = q.v;
    q_p[e] = q.p;
  }
  __syncthreads();

  // ---- limited slopes, both axes, cells [-1, T]^2 ----
  const int lim = P.limiter;
  const bool second = P.order > 1;
  for (int e = tid; e < S::SN; e += NT) {
    const int c = R(e % SW - 1, e / SW - 1);
    const double* pl[4] = {q_r, q_u, q_v, q_p};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double* q = pl[k];
      const double qc = q[c];
      sl[k * S::SN + e] = second ? limited_slope(qc - q[c - 1], q[c + 1] - qc, lim) : 0.0;
      sl[(4 + k) * S::SN + e] = second ? limited_slope(qc - q[c - RW], q[c + RW] - qc, lim) : 0.0;
    }
  }
  __syncthreads();

  if (XIE) {
    const double* sxp = sl + 3 * S::SN;
    const double* syp = sl + 7 * S::SN;
    for (int e = tid; e < S::NXR; e += NT) {
      const int fx = e % (T + 1), y = e / (T + 1) - 1;
      const double pl = fma(0.5, sxp[SI(fx - 1, y)], q_p[R(fx - 1, y)]);
      const double pr = fma(-0.5, sxp[SI(fx, y)], q_p[R(fx, y)]);
      xr[e] = pratio_f(pl, pr);
    }
    for (int e = tid; e < S::NYR; e += NT) {
      const int x = e % (T + 2) - 1, fy = e / (T + 2);
      const double pl = fma(0.5, syp[SI(x, fy - 1)], q_p[R(x, fy - 1)]);
      const double pr = fma(-0.5, syp[SI(x, fy)], q_p[R(x, fy)]);
      yr[e] = pratio_f(pl, pr);
    }
    __syncthreads();
  }

  // ---- one x-face and one y-face per thread (threads tid < NF) ----
  int degenerate = 0;
  Cons fxv{0.0, 0.0, 0.0, 0.0}, fyv{0.0, 0.0, 0.0, 0.0};
  if constexpr (XIE) {
    // Every thread evaluates the branch-free core of a face (threads past the
    // tile's faces repeat face 0 and discard it), so each warp can send the
    // faces that take one of xie_f's exits through xie_f after one vote.
    const int tf = tid < NF ? tid : 0;
    const double* sy = sl + 4 * S::SN;
    {
      const int fx = tf % (T + 1), y = tf / (T + 1);
      const int wl = (fx >= 1 && i0 + fx - 1 < nx) ? 1 : 0;
      const int wr = (fx < T && i0 + fx < nx) ? 1 : 0;
      const bool valid = tid < NF && j0 + y < ny && (wl | wr);
      const int cl = R(fx - 1, y), cr = R(fx, y), sL = SI(fx - 1, y), sR = SI(fx, y);
      const Prim L{fma(0.5, sl[sL], q_r[cl]), fma(0.5, sl[S::SN + sL], q_u[cl]), fma(0.5, sl[2 * S::SN + sL], q_v[cl]),
                   fma(0.5, sl[3 * S::SN + sL], q_p[cl])};
      const Prim Rr{fma(-0.5, sl[sR], q_r[cr]), fma(-0.5, sl[S::SN + sR], q_u[cr]),
                    fma(-0.5, sl[2 * S::SN + sR], q_v[cr]), fma(-0.5, sl[3 * S::SN + sR], q_p[cr])};
      double m = xr[(y + 1) * (T + 1) + fx];
      m = smin(m, yr[y * (T + 2) + fx]);
      m = smin(m, yr[(y + 1) * (T + 2) + fx]);
      m = smin(m, yr[y * (T + 2) + fx + 1]);
      m = smin(m, yr[(y + 1) * (T + 2) + fx + 1]);
      const double h = clamp01(m);
      bool fb, deg;
      Cons f = xie_core(L, Rr, 0, g, inv_gm1, h * h * h, fb, deg);
      fb = fb && valid;
      if (__any_sync(0xffffffffu, fb)) {
        if (fb) f = xie_f(L, Rr, 0, g, inv_gm1, h * h * h, deg);
      }
      if (valid) {
        fxv = f;
        if (ctl.count_degenerate && deg) degenerate += wl + wr;
      }
    }
    {
      const int x = tf % T, fy = tf / T;
      const int wb = (fy >= 1 && j0 + fy - 1 < ny) ? 1 : 0;
      const int wt = (fy < T && j0 + fy < ny) ? 1 : 0;
      const bool valid = tid < NF && i0 + x < nx && (wb | wt);
      const int cb = R(x, fy - 1), ct = R(x, fy), sB = SI(x, fy - 1), sT = SI(x, fy);
      const Prim L{fma(0.5, sy[sB], q_r[cb]), fma(0.5, sy[S::SN + sB], q_u[cb]), fma(0.5, sy[2 * S::SN + sB], q_v[cb]),
                   fma(0.5, sy[3 * S::SN + sB], q_p[cb])};
      const Prim Rr{fma(-0.5, sy[sT], q_r[ct]), fma(-0.5, sy[S::SN + sT], q_u[ct]),
                    fma(-0.5, sy[2 * S::SN + sT], q_v[ct]), fma(-0.5, sy[3 * S::SN + sT], q_p[ct])};
      // x-face ratios at (x, fy-1), (x+1, fy-1), (x, fy), (x+1, fy)
      double m = yr[fy * (T + 2) + x + 1];
      m = smin(m, xr[fy * (T + 1) + x]);
      m = smin(m, xr[fy * (T + 1) + x + 1]);
      m = smin(m, xr[(fy + 1) * (T + 1) + x]);
      m = smin(m, xr[(fy + 1) * (T + 1) + x + 1]);
      const double h = clamp01(m);
      bool fb, deg;
      Cons f = xie_core(L, Rr, 1, g, inv_gm1, h * h * h, fb, deg);
      fb = fb && valid;
      if (__any_sync(0xffffffffu, fb)) {
        if (fb) f = xie_f(L, Rr, 1, g, inv_gm1, h * h * h, deg);
      }
      if (valid) {
        fyv = f;
        if (ctl.count_degenerate && deg) degenerate += wb + wt;
      }
    }
  }
  if (!XIE && tid < NF) {
    // x-face fx between cells fx-1 and fx, row y
    const int fx = tid % (T + 1), y = tid / (T + 1);
    const int wl = (fx >= 1 && i0 + fx - 1 < nx) ? 1 : 0;
    const int wr = (fx < T && i0 + fx < nx) ? 1 : 0;
    if (j0 + y < ny && (wl | wr)) {
      const int cl = R(fx - 1, y), cr = R(fx, y), sL = SI(fx - 1, y), sR = SI(fx, y);
      Prim L{fma(0.5, sl[sL], q_r[cl]), fma(0.5, sl[S::SN + sL], q_u[cl]), fma(0.5, sl[2 * S::SN + sL], q_v[cl]),
             fma(0.5, sl[3 * S::SN + sL], q_p[cl])};
      Prim Rr{fma(-0.5, sl[sR], q_r[cr]), fma(-0.5, sl[S::SN + sR], q_u[cr]), fma(-0.5, sl[2 * S::SN + sR], q_v[cr]),
              fma(-0.5, sl[3 * S::SN + sR], q_p[cr])};
      bool deg = false;
      if (RK == ECG_RIEMANN_RUSANOV) {
        fxv = rusanov_f(L, Rr, 0, g, inv_gm1);
      } else if (RK == ECG_RIEMANN_XIE_AM_HLLC_P) {
        double m = xr[(y + 1) * (T + 1) + fx];
        m = smin(m, yr[y * (T + 2) + fx]);
        m = smin(m, yr[(y + 1) * (T + 2) + fx]);
        m = smin(m, yr[y * (T + 2) + fx + 1]);
        m = smin(m, yr[(y + 1) * (T + 2) + fx + 1]);
        const double h = clamp01(m);
        fxv = xie_f(L, Rr, 0, g, inv_gm1, h * h * h, deg);
      } else {
        if (RK == ECG_RIEMANN_LOWMACH_HLLC) lowmach_f(L, Rr, g);
        fxv = hllc_f(L, Rr, 0, g, inv_gm1, deg);
      }
      if (ctl.count_degenerate && deg) degenerate += wl + wr;
    }
  }
  if (!XIE && tid < NF) {
    // y-face fy between cells (x, fy-1) and (x, fy)
    const int x = tid % T, fy = tid / T;
    const int wb = (fy >= 1 && j0 + fy - 1 < ny) ? 1 : 0;
    const int wt = (fy < T && j0 + fy < ny) ? 1 : 0;
    if (i0 + x < nx && (wb | wt)) {
      const int cb = R(x, fy - 1), ct = R(x, fy), sB = SI(x, fy - 1), sT = SI(x, fy);
      const double* sy = sl + 4 * S::SN;
      Prim L{fma(0.5, sy[sB], q_r[cb]), fma(0.5, sy[S::SN + sB], q_u[cb]), fma(0.5, sy[2 * S::SN + sB], q_v[cb]),
             fma(0.5, sy[3 * S::SN + sB], q_p[cb])};
      Prim Rr{fma(-0.5, sy[sT], q_r[ct]), fma(-0.5, sy[S::SN + sT], q_u[ct]), fma(-0.5, sy[2 * S::SN + sT], q_v[ct]),
              fma(-0.5, sy[3 * S::SN + sT], q_p[ct])};
      bool deg = false;
      if (RK == ECG_RIEMANN_RUSANOV) {
        fyv = rusanov_f(L, Rr, 1, g, inv_gm1);
      } else if (RK == ECG_RIEMANN_XIE_AM_HLLC_P) {
        // x-face ratios at (x, fy-1), (x+1, fy-1), (x, fy), (x+1, fy)
        double m = yr[fy * (T + 2) + x + 1];
        m = smin(m, xr[fy * (T + 1) + x]);
        m = smin(m, xr[fy * (T + 1) + x + 1]);
        m = smin(m, xr[(fy + 1) * (T + 1) + x]);
        m = smin(m, xr[(fy + 1) * (T + 1) + x + 1]);
        const double h = clamp01(m);
        fyv = xie_f(L, Rr, 1, g, inv_gm1, h * h * h, deg);
      } else {
        if (RK == ECG_RIEMANN_LOWMACH_HLLC) lowmach_f(L, Rr, g);
        fyv = hllc_f(L, Rr, 1, g, inv_gm1, deg);
      }
      if (ctl.count_degenerate && deg) degenerate += wb + wt;
    }
  }
  __syncthreads();  // every slope / primitive read is done: reuse the slope region
  double* F = sl;             // 4 planes of NF x-face fluxes
  double* G = sl + 4 * NF;    // 4 planes of NF y-face fluxes
  if (tid < NF) {
    F[tid] = fxv.rho;
    F[NF + tid] = fxv.mx;
    F[2 * NF + tid] = fxv.my;
    F[3 * NF + tid] = fxv.E;
    G[tid] = fyv.rho;
    G[NF + tid] = fyv.mx;
    G[2 * NF + tid] = fyv.my;
    G[3 * NF + tid] = fyv.E;
  }
  __syncthreads();

  // ---- conservative update + fused reductions ----
  unsigned long long kmax = okey(kLowest), krho = okey(kMax), kp = okey(kMax);
  int nonfinite = 0;
  if (tid < T * T) {
    const int x = tid % T, y = tid / T;
    const int gi = i0 + x, gj = j0 + y;
    if (gi < nx && gj < ny) {
      const long long o = static_cast<long long>(gj) * P.g.pitch + gi;
      const long long pl = P.g.plane;
      const int xl = y * (T + 1) + x, yb = y * T + x;
      const double idx = P.g.inv_dx, idy = P.g.inv_dy;
      Cons n;
      n.rho = __ldg(u + o) - dt * ((F[xl + 1] - F[xl]) * idx + (G[yb + T] - G[yb]) * idy);
      n.mx = __ldg(u + o + pl) - dt * ((F[NF + xl + 1] - F[NF + xl]) * idx + (G[NF + yb + T] - G[NF + yb]) * idy);
      n.my = __ldg(u + o + 2 * pl) -
             dt * ((F[2 * NF + xl + 1] - F[2 * NF + xl]) * idx + (G[2 * NF + yb + T] - G[2 * NF + yb]) * idy);
      n.E = __ldg(u + o + 3 * pl) -
            dt * ((F[3 * NF + xl + 1] - F[3 * NF + xl]) * idx + (G[3 * NF + yb + T] - G[3 * NF + yb]) * idy);
      out[o] = n.rho;
      out[o + pl] = n.mx;
      out[o + 2 * pl] = n.my;
      out[o + 3 * pl] = n.E;
      const Prim q = to_prim_f(n, g);
      const double cs = fsound(q.rho, q.p, g);
      const double rate = (fabs(q.u) + cs) * idx + (fabs(q.v) + cs) * idy;
      if (!isnan(rate)) kmax = okey(rate);
      const bool bad = !isfinite(q.rho) || !isfinite(q.u) || !isfinite(q.v) || !isfinite(q.p) || !isfinite(n.E);
      krho = okey(bad ? -kInf : q.rho);
      kp = okey(bad ? -kInf : q.p);
      nonfinite = bad ? 1 : 0;
    }
  }
  block_commit<NT>(red, kmax, krho, kp, nonfinite, degenerate, &stats[ctl.acc_slot]);
}

template <int RK>
cudaError_t launch_rk(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats, const EcgDtCtl& ctl,
                      cudaStream_t s)
{
  constexpr int T = 16;
  using S = FastSmem<T, RK == ECG_RIEMANN_XIE_AM_HLLC_P>;
  auto kern = fv_fast_kernel<RK, T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::bytes));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  const dim3 grid((p.g.nx + T - 1) / T, (p.g.ny + T - 1) / T);
  kern<<<grid, S::NT, S::bytes, s>>>(p, in, out, stats, ctl);
  return cudaGetLastError();
}

inline cudaError_t launch(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats,
                          const EcgDtCtl& ctl, cudaStream_t s)
{
  switch (p.riemann) {
    case ECG_RIEMANN_RUSANOV: return launch_rk<ECG_RIEMANN_RUSANOV>(p, in, out, stats, ctl, s);
    case ECG_RIEMANN_LOWMACH_HLLC: return launch_rk<ECG_RIEMANN_LOWMACH_HLLC>(p, in, out, stats, ctl, s);
    case ECG_RIEMANN_XIE_AM_HLLC_P: return launch_rk<ECG_RIEMANN_XIE_AM_HLLC_P>(p, in, out, stats, ctl, s);
    default: return launch_rk<ECG_RIEMANN_HLLC>(p, in, out, stats, ctl, s);
  }
}

}  // namespace fast
