// Exact and analytic states of the test problems (problems/exact_riemann.hpp,
// problems/problem_state_functions.hpp, problems/problem_initialization.hpp),
// shared by the ghost rings, the initial states and the direct T1/S2 driver.
// Included inside a namespace that already holds Prim (ecg_device.cuh).
#pragma once

// gresho_state, problems/problem_state_functions.hpp:2-30
__device__ Prim gresho_state(double x, double y, const EcgProblem& c)
{
  const double dx = x - c.vortex_cx, dy = y - c.vortex_cy;
  const double r = sqrt(dx * dx + dy * dy);
  const double rho = c.density_outer;
  const double vs = c.mach * sqrt(c.gamma * c.pressure / c.density_outer);
  double tf = 0.0;
  double pf = -2.0 + 4.0 * log(2.0);
  if (r < 0.2) {
    tf = 5.0 * r;
    pf = 12.5 * r * r;
  } else if (r < 0.4) {
    tf = 2.0 - 5.0 * r;
    pf = 12.5 * r * r + 4.0 * (1.0 - 5.0 * r - log(0.2) + log(r));
  }
  const double vt = vs * tf;
  const double p = c.pressure + rho * vs * vs * pf;
  if (r < 1.0e-14) return Prim{rho, 0.0, 0.0, p};
  return Prim{rho, -vt * dy / r, vt * dx / r, p};
}

// riemann_quadrant_state, problem_state_functions.hpp:74-99
__device__ Prim quadrant_state(double x, double y, const EcgProblem& c)
{
  const bool right = x >= c.interface_x, top = y >= c.interface_y;
  if (right && top) return Prim{1.5, 0.0, 0.0, 1.5};
  if (!right && top) return Prim{0.532258064516129, 1.206045378311055, 0.0, 0.3};
  if (!right && !top) return Prim{0.137992831541219, 1.206045378311055, 1.206045378311055, 0.029032258064516};
  return Prim{0.532258064516129, 0.0, 1.206045378311055, 0.3};
}

// Exact Riemann solution (Toro), problems/exact_riemann.hpp:92-205.
__device__ void pressure_fn(double p, const Prim& q, double g, double& f, double& d)
{
  const double a = sqrt(g * q.p / q.rho);
  if (p > q.p) {
    const double A = 2.0 / ((g + 1.0) * q.rho);
    const double B = (g - 1.0) / (g + 1.0) * q.p;
    const double root = sqrt(A / (p + B));
    f = (p - q.p) * root;
    d = root * (1.0 - 0.5 * (p - q.p) / (p + B));
    return;
  }
  const double ratio = p / q.p;
  f = 2.0 * a / (g - 1.0) * (pow(ratio, (g - 1.0) / (2.0 * g)) - 1.0);
  d = 1.0 / (q.rho * a) * pow(ratio, -(g + 1.0) / (2.0 * g));
}

__device__ Prim riemann_sample(double x, double t, const Prim& l, const Prim& r, double g, double x0)
{
  if (t <= 0.0) return x < x0 ? l : r;
  const double al = sqrt(g * l.p / l.rho), ar = sqrt(g * r.p / r.rho);
  double p = smax(1.0e-12, 0.5 * (l.p + r.p) - 0.125 * (r.u - l.u) * (l.rho + r.rho) * (al + ar));
  for (int it = 0; it < 80; ++it) {
    double fl, dl, fr, dr;
    pressure_fn(p, l, g, fl, dl);
    pressure_fn(p, r, g, fr, dr);
    const double res = fl + fr + r.u - l.u;
    double pn = p - res / (dl + dr);
    if (!(pn > 0.0) || !isfinite(pn)) pn = 0.5 * p;
    if (fabs(pn - p) <= 1.0e-12 * smax(1.0, pn)) {
      p = pn;
      break;
    }
    p = pn;
  }
  double fl, dl, fr, dr;
  pressure_fn(p, l, g, fl, dl);
  pressure_fn(p, r, g, fr, dr);
  const double ps = p, us = 0.5 * (l.u + r.u + fr - fl);
  const double xi = (x - x0) / t;
  const double gm1 = g - 1.0, gp1 = g + 1.0;
  if (xi <= us) {
    if (ps > l.p) {
      const double s = l.u - al * sqrt(gp1 / (2.0 * g) * ps / l.p + gm1 / (2.0 * g));
      if (xi <= s) return l;
      const double ratio = ps / l.p;
      return Prim{l.rho * ((ratio + gm1 / gp1) / ((gm1 / gp1) * ratio + 1.0)), us, l.v, ps};
    }
    const double head = l.u - al;
    const double astar = al * pow(ps / l.p, gm1 / (2.0 * g));
    const double tail = us - astar;
    if (xi <= head) return l;
    if (xi >= tail) return Prim{l.rho * pow(ps / l.p, 1.0 / g), us, l.v, ps};
    const double uu = 2.0 / gp1 * (al + 0.5 * gm1 * l.u + xi);
    const double a = 2.0 / gp1 * (al + 0.5 * gm1 * (l.u - xi));
    return Prim{l.rho * pow(a / al, 2.0 / gm1), uu, l.v, l.p * pow(a / al, 2.0 * g / gm1)};
  }
  if (ps > r.p) {
    const double s = r.u + ar * sqrt(gp1 / (2.0 * g) * ps / r.p + gm1 / (2.0 * g));
    if (xi >= s) return r;
    const double ratio = ps / r.p;
    return Prim{r.rho * ((ratio + gm1 / gp1) / ((gm1 / gp1) * ratio + 1.0)), us, r.v, ps};
  }
  const double head = r.u + ar;
  const double astar = ar * pow(ps / r.p, gm1 / (2.0 * g));
  const double tail = us + astar;
  if (xi >= head) return r;
  if (xi <= tail) return Prim{r.rho * pow(ps / r.p, 1.0 / g), us, r.v, ps};
  const double uu = 2.0 / gp1 * (-ar + 0.5 * gm1 * r.u + xi);
  const double a = 2.0 / gp1 * (ar - 0.5 * gm1 * (r.u - xi));
  return Prim{r.rho * pow(a / ar, 2.0 / gm1), uu, r.v, r.p * pow(a / ar, 2.0 * g / gm1)};
}

// periodic_nearest_delta, problems/problem_state_functions.hpp:32-43
__device__ double nearest_delta(double x, double c, double lo, double hi)
{
  const double L = hi - lo;
  double d = x - c;
  if (L > 0.0) d -= L * floor(d / L + 0.5);
  return d;
}

// isentropic_vortex_state at time t, problem_state_functions.hpp:45-72
__device__ Prim isentropic_vortex_state(double x, double y, const EcgProblem& c, double plo_x, double plo_y,
                                        double t)
{
  const double pi = 3.141592653589793238462643383279502884;
  const double g = c.gamma, s = c.isentropic_vortex_strength;
  const double cx = c.vortex_cx + c.velocity_x * t, cy = c.vortex_cy + c.velocity_y * t;
  const double dx = nearest_delta(x, cx, plo_x, c.prob_hi_x);
  const double dy = nearest_delta(y, cy, plo_y, c.prob_hi_y);
  const double r2 = dx * dx + dy * dy;
  const double eh = exp(0.5 * (1.0 - r2));
  const double ef = exp(1.0 - r2);
  const double temp = 1.0 - (g - 1.0) * s * s / (8.0 * g * pi * pi) * ef;
  const double rho = c.density_outer * pow(temp, 1.0 / (g - 1.0));
  const double p = c.pressure * pow(temp, g / (g - 1.0));
  const double vf = s / (2.0 * pi) * eh;
  return Prim{rho, c.velocity_x - vf * dy, c.velocity_y + vf * dx, p};
}

// periodic_signed_distance / wrap_periodic_coordinate / exact_advection_blob_state,
// problems/problem_initialization.hpp:157-207: the top hat translated with
// (velocity_x, velocity_y), wrapped on periodic axes.
__device__ double periodic_signed_distance(double x, double center, double lo, double hi, bool periodic)
{
  double d = x - center;
  if (periodic) {
    const double length = hi - lo;
    if (length > 0.0) d -= round(d / length) * length;
  }
  return d;
}
__device__ double wrap_periodic_coordinate(double x, double lo, double hi)
{
  const double length = hi - lo;
  if (length <= 0.0) return x;
  double w = lo + fmod(x - lo, length);
  if (w < lo) w += length;
  return w;
}
__device__ Prim exact_blob_state(double x, double y, const EcgProblem& c, double plo_x, double plo_y, double t)
{
  double cx = c.blob_cx + c.velocity_x * t;
  double cy = c.blob_cy + c.velocity_y * t;
  if (c.periodic_x) cx = wrap_periodic_coordinate(cx, plo_x, c.prob_hi_x);
  if (c.periodic_y) cy = wrap_periodic_coordinate(cy, plo_y, c.prob_hi_y);
  const double dx = periodic_signed_distance(x, cx, plo_x, c.prob_hi_x, c.periodic_x != 0);
  const double dy = periodic_signed_distance(y, cy, plo_y, c.prob_hi_y, c.periodic_y != 0);
  const double r2 = dx * dx + dy * dy;
  const double rho = r2 <= c.blob_radius * c.blob_radius ? c.density_inner : c.density_outer;
  return Prim{rho, c.velocity_x, c.velocity_y, c.pressure};
}
