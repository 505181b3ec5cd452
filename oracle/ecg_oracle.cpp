// ecg_oracle.cpp -- CPU restatement of the euler_compare hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
// (amrex_euler_allmach_explicit_imex_b200/csrc) and the "port" CPU baseline;
// only tests/, __graft_entry__.smoke() and bench.py's CPU legs may load it.
// The product never calls it.
//
// It restates the reference's algorithm in plain C++ (no AMReX, no Eigen) on
// ghosted host arrays.  Every floating-point expression keeps the operand
// order of the cited reference line, so that, compiled like the reference
// (gcc -O3, no FMA contraction), explicit-step results are bit-identical to
// the reference build.  The GMRES least-squares solve uses Givens rotations
// instead of the reference's per-iteration colPivHouseholderQr (identical in
// exact arithmetic); its iterates therefore agree with the reference to
// rounding, not bit for bit.
//
// Paths below are relative to amrex/apps/euler_compare/src/euler_compare/.
//
// Host layout of every public function: 4 component planes (rho, mx, my, E)
// of nx*ny doubles, i fastest.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "ecg.h"

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

struct Cons { double rho, mx, my, E; };
struct Prim { double rho, u, v, p; };

inline double cmin(double a, double b) { return std::min(a, b); }  // amrex::min == std::min
inline double cmax(double a, double b) { return std::max(a, b); }  // amrex::max == std::max

// ---- state algebra: core/state_primitives.hpp -------------------------------

// to_primitive, state_primitives.hpp:103-111
inline Prim to_prim(const Cons& c, double g)
{
  const double inv_rho = 1.0 / c.rho;
  const double u = c.mx * inv_rho;
  const double v = c.my * inv_rho;
  const double kin = 0.5 * c.rho * (u * u + v * v);
  return Prim{c.rho, u, v, (g - 1.0) * (c.E - kin)};
}

// to_conserved, state_primitives.hpp:113-117
inline Cons to_cons(const Prim& q, double g)
{
  const double kin = 0.5 * q.rho * (q.u * q.u + q.v * q.v);
  return Cons{q.rho, q.rho * q.u, q.rho * q.v, q.p / (g - 1.0) + kin};
}

// sound_speed, state_primitives.hpp:202-205
inline double csound(const Prim& q, double g) { return std::sqrt(g * q.p / q.rho); }

// minmod, state_primitives.hpp:57-63
inline double mm(double a, double b)
{
  if (a * b <= 0.0) return 0.0;
  return std::abs(a) < std::abs(b) ? a : b;
}

// limited_slope, state_primitives.hpp:71-91
inline double slope1(double bk, double fw, int lim)
{
  if (bk * fw <= 0.0) return 0.0;
  if (lim == ECG_LIMITER_MC) return mm(mm(2.0 * bk, 0.5 * (bk + fw)), 2.0 * fw);
  if (lim == ECG_LIMITER_VANLEER) {
    const double d = bk + fw;
    if (std::abs(d) <= 1.0e-14) return 0.0;
    return 2.0 * bk * fw / d;
  }
  return mm(bk, fw);
}

inline double normal_vel(const Prim& q, int axis) { return axis == 0 ? q.u : q.v; }

// ---- ghosted grid -------------------------------------------------------------

struct Grid {
  int nx = 0, ny = 0;
  static constexpr int ng = 2;
  int jstride = 0;
  std::vector<double> a;  // 4 planes of (nx+4)*(ny+4)
  Grid(int nx_, int ny_) : nx(nx_), ny(ny_), jstride(nx_ + 4) {
    a.assign(static_cast<std::size_t>(4) * jstride * (ny + 4), 0.0);
  }
  std::size_t idx(int i, int j, int n) const {
    return static_cast<std::size_t>(n) * jstride * (ny + 4) + static_cast<std::size_t>(j + ng) * jstride + (i + ng);
  }
  double& at(int i, int j, int n) { return a[idx(i, j, n)]; }
  double at(int i, int j, int n) const { return a[idx(i, j, n)]; }
  Cons cons(int i, int j) const { return Cons{at(i, j, 0), at(i, j, 1), at(i, j, 2), at(i, j, 3)}; }
  void set(int i, int j, const Cons& c) { at(i, j, 0) = c.rho; at(i, j, 1) = c.mx; at(i, j, 2) = c.my; at(i, j, 3) = c.E; }
  void load(const double* u) {
    const std::size_t pl = static_cast<std::size_t>(nx) * ny;
    for (int n = 0; n < 4; ++n)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) at(i, j, n) = u[n * pl + static_cast<std::size_t>(j) * nx + i];
  }
  void store(double* u) const {
    const std::size_t pl = static_cast<std::size_t>(nx) * ny;
    for (int n = 0; n < 4; ++n)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) u[n * pl + static_cast<std::size_t>(j) * nx + i] = at(i, j, n);
  }
};

struct Geo {
  double dx, dy, plo[2], phi[2];
  bool per[2];
  explicit Geo(const ecg_run_config& c) {
    // AMReX Geometry: dx = (hi - lo) / n
    dx = (c.prob_hi[0] - c.prob_lo[0]) / static_cast<double>(c.n_cell[0]);
    dy = (c.prob_hi[1] - c.prob_lo[1]) / static_cast<double>(c.n_cell[1]);
    plo[0] = c.prob_lo[0]; plo[1] = c.prob_lo[1];
    phi[0] = c.prob_hi[0]; phi[1] = c.prob_hi[1];
    per[0] = c.is_periodic[0] != 0; per[1] = c.is_periodic[1] != 0;
  }
  double xc(int i) const { return plo[0] + (static_cast<double>(i) + 0.5) * dx; }
  double yc(int j) const { return plo[1] + (static_cast<double>(j) + 0.5) * dy; }
};

// ---- problem states -----------------------------------------------------------

// shock_density_bubble_post_shock_state, problems/problem_initialization.hpp:51-58
inline Prim bubble_post_shock() { return Prim{2.8181818181818183, 1.6064386578049976, 0.0, 5.0}; }

// shock_density_bubble_fraction / _cell_state, problem_initialization.hpp:66-102
double bubble_fraction(double xc, double yc, double dx, double dy)
{
  double inside = 0.0;
  for (int sy = 0; sy < 4; ++sy) {
    for (int sx = 0; sx < 4; ++sx) {
      const double x = xc + ((static_cast<double>(sx) + 0.5) / 4.0 - 0.5) * dx;
      const double y = yc + ((static_cast<double>(sy) + 0.5) / 4.0 - 0.5) * dy;
      const double rx = x - 0.5, ry = y - 0.0;
      if (x >= 0.2 && rx * rx + ry * ry <= 0.2 * 0.2) inside += 1.0;
    }
  }
  return inside / 16.0;
}
Prim bubble_cell(double x, double y, double dx, double dy)
{
  if (x < 0.2) return bubble_post_shock();
  const double f = bubble_fraction(x, y, dx, dy);
  return Prim{f * 0.1 + (1.0 - f) * 1.0, 0.0, 0.0, 1.0};
}

// Mach 1.22 shock / bubble configuration (ECG_PROBLEM_SHOCK_BUBBLE_MACH122,
// no ProblemKind in the reference): Rankine-Hugoniot state behind a Mach 1.22
// shock into (rho, u, p) = (1, 0, 1), gamma = 1.4; the same sub-cell bubble
// sampling as shock_density_bubble_fraction with the shock at x = 0.5 and a
// rho = 0.138 bubble of radius 0.25 at (1, 0.5).
Prim mach122_post_shock(double gamma)
{
  const double mach = 1.22;
  const double m2 = mach * mach;
  const double rho2 = (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0);
  const double p2 = 1.0 + 2.0 * gamma * (m2 - 1.0) / (gamma + 1.0);
  const double s = mach * std::sqrt(gamma);
  return Prim{rho2, s * (1.0 - 1.0 / rho2), 0.0, p2};
}
Prim mach122_cell(double x, double y, double dx, double dy, double gamma)
{
  if (x < 0.5) return mach122_post_shock(gamma);
  double inside = 0.0;
  for (int sy = 0; sy < 4; ++sy) {
    for (int sx = 0; sx < 4; ++sx) {
      const double xs = x + ((static_cast<double>(sx) + 0.5) / 4.0 - 0.5) * dx;
      const double ys = y + ((static_cast<double>(sy) + 0.5) / 4.0 - 0.5) * dy;
      const double rx = xs - 1.0, ry = ys - 0.5;
      if (xs >= 0.5 && rx * rx + ry * ry <= 0.25 * 0.25) inside += 1.0;
    }
  }
  const double f = inside / 16.0;
  return Prim{f * 0.138 + (1.0 - f) * 1.0, 0.0, 0.0, 1.0};
}

// reference_sound_speed / velocity_scale_from_mach, state_primitives.hpp:207-215
inline double vel_scale(const ecg_run_config& c)
{
  return c.mach * std::sqrt(c.gamma * c.pressure / c.density_outer);
}

// gresho_state, problems/problem_state_functions.hpp:2-30
Prim gresho(double x, double y, const ecg_run_config& c)
{
  const double dx = x - c.vortex_cx, dy = y - c.vortex_cy;
  const double r = std::sqrt(dx * dx + dy * dy);
  const double rho = c.density_outer;
  const double vs = vel_scale(c);
  double tf = 0.0;
  double pf = -2.0 + 4.0 * std::log(2.0);
  if (r < 0.2) {
    tf = 5.0 * r;
    pf = 12.5 * r * r;
  } else if (r < 0.4) {
    tf = 2.0 - 5.0 * r;
    pf = 12.5 * r * r + 4.0 * (1.0 - 5.0 * r - std::log(0.2) + std::log(r));
  }
  const double vt = vs * tf;
  const double p = c.pressure + rho * vs * vs * pf;
  if (r < 1.0e-14) return Prim{rho, 0.0, 0.0, p};
  return Prim{rho, -vt * dy / r, vt * dx / r, p};
}

// periodic_nearest_delta / isentropic_vortex_state, problem_state_functions.hpp:32-72
double nearest_delta(double x, double c, double lo, double hi)
{
  const double L = hi - lo;
  double d = x - c;
  if (L > 0.0) d -= L * std::floor(d / L + 0.5);
  return d;
}
Prim isentropic_vortex(double x, double y, const ecg_run_config& c, double t)
{
  const double pi = 3.141592653589793238462643383279502884;
  const double g = c.gamma, s = c.isentropic_vortex_strength;
  const double cx = c.vortex_cx + c.velocity_x * t, cy = c.vortex_cy + c.velocity_y * t;
  const double dx = nearest_delta(x, cx, c.prob_lo[0], c.prob_hi[0]);
  const double dy = nearest_delta(y, cy, c.prob_lo[1], c.prob_hi[1]);
  const double r2 = dx * dx + dy * dy;
  const double eh = std::exp(0.5 * (1.0 - r2));
  const double ef = std::exp(1.0 - r2);
  const double temp = 1.0 - (g - 1.0) * s * s / (8.0 * g * pi * pi) * ef;
  const double rho = c.density_outer * std::pow(temp, 1.0 / (g - 1.0));
  const double p = c.pressure * std::pow(temp, g / (g - 1.0));
  const double vf = s / (2.0 * pi) * eh;
  return Prim{rho, c.velocity_x - vf * dy, c.velocity_y + vf * dx, p};
}

// riemann_quadrant_state, problem_state_functions.hpp:74-99
Prim quadrant(double x, double y, const ecg_run_config& c)
{
  const bool right = x >= c.riemann_interface_x, top = y >= c.riemann_interface_y;
  if (right && top) return Prim{1.5, 0.0, 0.0, 1.5};
  if (!right && top) return Prim{0.532258064516129, 1.206045378311055, 0.0, 0.3};
  if (!right && !top) return Prim{0.137992831541219, 1.206045378311055, 1.206045378311055, 0.029032258064516};
  return Prim{0.532258064516129, 0.0, 1.206045378311055, 0.3};
}

// toro_state, problems/exact_riemann.hpp:2-35 (as {rho,u,v,p} left, right)
bool toro_states(int id, Prim& l, Prim& r)
{
  switch (id) {
    case 1: l = {1.0, 0.0, 0.0, 1.0}; r = {0.125, 0.0, 0.0, 0.1}; return true;
    case 2: l = {1.0, -2.0, 0.0, 0.4}; r = {1.0, 2.0, 0.0, 0.4}; return true;
    case 3: l = {1.0, 0.0, 0.0, 1000.0}; r = {1.0, 0.0, 0.0, 0.01}; return true;
    case 4: l = {1.0, 0.0, 0.0, 0.01}; r = {1.0, 0.0, 0.0, 100.0}; return true;
    case 5: l = {5.99924, 19.5975, 0.0, 460.894}; r = {5.99242, -6.19633, 0.0, 46.0950}; return true;
    case 93: l = {0.445, 1.698, 0.0, 3.528}; r = {0.5, 0.0, 0.0, 0.571}; return true;
    case 94: l = {1000.0, 1.0, 0.0, 1.0e5}; r = {0.01, 1.0, 0.0, 1.0e5}; return true;
    case 95: l = {1.0, 0.0, 0.0, 1.01}; r = {1.0, 0.0, 0.0, 1.0}; return true;
    case 96: l = {1.0, 0.0, 0.0, 1.0001}; r = {1.0, 0.0, 0.0, 1.0}; return true;
    case 97: l = {1.0, 2.0, 0.0, 0.1}; r = {1.0, -2.0, 0.0, 0.1}; return true;
    case 90: l = {1.0, 0.0, 0.0, 1.0}; r = {1.0, 0.0, 0.0, 1.0}; return true;
    case 91: l = {2.0, 0.0, 0.0, 1.0}; r = {1.0, 0.0, 0.0, 1.0}; return true;
    case 92: l = {2.0, 0.1, 0.0, 1.0}; r = {1.0, 0.1, 0.0, 1.0}; return true;
    default: return false;
  }
}

// Exact Riemann solver (Toro): exact_riemann.hpp:92-205.
void pfun(double p, const Prim& q, double g, double& f, double& d)
{
  const double a = std::sqrt(g * q.p / q.rho);
  if (p > q.p) {
    const double A = 2.0 / ((g + 1.0) * q.rho);
    const double B = (g - 1.0) / (g + 1.0) * q.p;
    const double root = std::sqrt(A / (p + B));
    f = (p - q.p) * root;
    d = root * (1.0 - 0.5 * (p - q.p) / (p + B));
    return;
  }
  const double ratio = p / q.p;
  f = 2.0 * a / (g - 1.0) * (std::pow(ratio, (g - 1.0) / (2.0 * g)) - 1.0);
  d = 1.0 / (q.rho * a) * std::pow(ratio, -(g + 1.0) / (2.0 * g));
}
void star_pu(const Prim& l, const Prim& r, double g, double& ps, double& us)
{
  const double al = std::sqrt(g * l.p / l.rho), ar = std::sqrt(g * r.p / r.rho);
  double p = cmax(1.0e-12, 0.5 * (l.p + r.p) - 0.125 * (r.u - l.u) * (l.rho + r.rho) * (al + ar));
  for (int it = 0; it < 80; ++it) {
    double fl = 0, dl = 0, fr = 0, dr = 0;
    pfun(p, l, g, fl, dl);
    pfun(p, r, g, fr, dr);
    const double res = fl + fr + r.u - l.u;
    double pn = p - res / (dl + dr);
    if (!(pn > 0.0) || !std::isfinite(pn)) pn = 0.5 * p;
    if (std::abs(pn - p) <= 1.0e-12 * cmax(1.0, pn)) { p = pn; break; }
    p = pn;
  }
  double fl = 0, dl = 0, fr = 0, dr = 0;
  pfun(p, l, g, fl, dl);
  pfun(p, r, g, fr, dr);
  ps = p;
  us = 0.5 * (l.u + r.u + fr - fl);
}
Prim riemann_sample(double x, double t, const Prim& l, const Prim& r, double g, double x0)
{
  if (t <= 0.0) return x < x0 ? l : r;
  double ps = 0, us = 0;
  star_pu(l, r, g, ps, us);
  const double xi = (x - x0) / t;
  const double al = std::sqrt(g * l.p / l.rho), ar = std::sqrt(g * r.p / r.rho);
  const double gm1 = g - 1.0, gp1 = g + 1.0;
  auto shock_rho = [&](const Prim& q, double p) {
    const double ratio = p / q.p;
    return q.rho * ((ratio + gm1 / gp1) / ((gm1 / gp1) * ratio + 1.0));
  };
  auto fan_rho = [&](const Prim& q, double p) { return q.rho * std::pow(p / q.p, 1.0 / g); };
  if (xi <= us) {
    if (ps > l.p) {
      const double s = l.u - al * std::sqrt(gp1 / (2.0 * g) * ps / l.p + gm1 / (2.0 * g));
      if (xi <= s) return l;
      return Prim{shock_rho(l, ps), us, l.v, ps};
    }
    const double head = l.u - al;
    const double astar = al * std::pow(ps / l.p, gm1 / (2.0 * g));
    const double tail = us - astar;
    if (xi <= head) return l;
    if (xi >= tail) return Prim{fan_rho(l, ps), us, l.v, ps};
    const double u = 2.0 / gp1 * (al + 0.5 * gm1 * l.u + xi);
    const double a = 2.0 / gp1 * (al + 0.5 * gm1 * (l.u - xi));
    return Prim{l.rho * std::pow(a / al, 2.0 / gm1), u, l.v, l.p * std::pow(a / al, 2.0 * g / gm1)};
  }
  if (ps > r.p) {
    const double s = r.u + ar * std::sqrt(gp1 / (2.0 * g) * ps / r.p + gm1 / (2.0 * g));
    if (xi >= s) return r;
    return Prim{shock_rho(r, ps), us, r.v, ps};
  }
  const double head = r.u + ar;
  const double astar = ar * std::pow(ps / r.p, gm1 / (2.0 * g));
  const double tail = us + astar;
  if (xi >= head) return r;
  if (xi <= tail) return Prim{fan_rho(r, ps), us, r.v, ps};
  const double u = 2.0 / gp1 * (-ar + 0.5 * gm1 * r.u + xi);
  const double a = 2.0 / gp1 * (ar - 0.5 * gm1 * (r.u - xi));
  return Prim{r.rho * std::pow(a / ar, 2.0 / gm1), u, r.v, r.p * std::pow(a / ar, 2.0 * g / gm1)};
}

// Top-hat blob, problem_initialization.hpp:127-155 and exact translated state :157-207
double periodic_signed_distance(double x, double c, double lo, double hi, bool per)
{
  double d = x - c;
  if (per) {
    const double L = hi - lo;
    if (L > 0.0) d -= std::round(d / L) * L;
  }
  return d;
}
double wrap_coord(double x, double lo, double hi)
{
  const double L = hi - lo;
  if (L <= 0.0) return x;
  double w = lo + std::fmod(x - lo, L);
  if (w < lo) w += L;
  return w;
}

// initialize_state dispatch, problem_initialization.hpp:420-435
void initialize(const ecg_run_config& c, Grid& gr)
{
  const Geo geo(c);
  Prim tl{}, tr{};
  if (c.problem == ECG_PROBLEM_TORO1) toro_states(c.toro_test, tl, tr);
  for (int j = 0; j < c.n_cell[1]; ++j) {
    for (int i = 0; i < c.n_cell[0]; ++i) {
      const double x = geo.xc(i), y = geo.yc(j);
      Prim q{};
      switch (c.problem) {
        case ECG_PROBLEM_TORO1: q = x < c.riemann_interface_x ? tl : tr; break;
        case ECG_PROBLEM_GRESHO_VORTEX: q = gresho(x, y, c); break;
        case ECG_PROBLEM_ISENTROPIC_VORTEX: q = isentropic_vortex(x, y, c, 0.0); break;
        case ECG_PROBLEM_RIEMANN_QUADRANT: q = quadrant(x, y, c); break;
        case ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D:
        case ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL: q = bubble_cell(x, y, geo.dx, geo.dy); break;
        case ECG_PROBLEM_SHOCK_BUBBLE_MACH122: q = mach122_cell(x, y, geo.dx, geo.dy, c.gamma); break;
        default: {
          const double r2 = (x - c.blob_cx) * (x - c.blob_cx) + (y - c.blob_cy) * (y - c.blob_cy);
          const double rho = r2 <= c.blob_radius * c.blob_radius ? c.density_inner : c.density_outer;
          gr.at(i, j, 0) = rho;
          gr.at(i, j, 1) = rho * c.velocity_x;
          gr.at(i, j, 2) = rho * c.velocity_y;
          gr.at(i, j, 3) = c.pressure / (c.gamma - 1.0) + 0.5 * rho * (c.velocity_x * c.velocity_x + c.velocity_y * c.velocity_y);
          continue;
        }
      }
      gr.set(i, j, to_cons(q, c.gamma));
    }
  }
}

// ---- ghost fills: problems/boundary_conditions.hpp -----------------------------

inline int wrap(int i, int n) { return ((i % n) + n) % n; }
inline int clampi(int i, int n) { return std::min(std::max(i, 0), n - 1); }

// FillBoundary(periodicity): ghosts whose periodic image is valid.
void fill_periodic(Grid& g, const Geo& geo)
{
  for (int n = 0; n < 4; ++n)
    for (int j = -2; j < g.ny + 2; ++j)
      for (int i = -2; i < g.nx + 2; ++i) {
        const bool vi = i >= 0 && i < g.nx, vj = j >= 0 && j < g.ny;
        if (vi && vj) continue;
        const int ii = geo.per[0] ? wrap(i, g.nx) : i;
        const int jj = geo.per[1] ? wrap(j, g.ny) : j;
        if (ii >= 0 && ii < g.nx && jj >= 0 && jj < g.ny) g.at(i, j, n) = g.at(ii, jj, n);
      }
}

// fill_physical_outflow_ghosts, boundary_conditions.hpp:2-25
void fill_outflow(Grid& g, const Geo& geo)
{
  fill_periodic(g, geo);
  for (int n = 0; n < 4; ++n)
    for (int j = -2; j < g.ny + 2; ++j)
      for (int i = -2; i < g.nx + 2; ++i) {
        const bool xp = !geo.per[0] && (i < 0 || i >= g.nx);
        const bool yp = !geo.per[1] && (j < 0 || j >= g.ny);
        if (xp || yp) g.at(i, j, n) = g.at(xp ? clampi(i, g.nx) : i, yp ? clampi(j, g.ny) : j, n);
      }
}

// fill_shock_density_bubble_ghosts, boundary_conditions.hpp:27-73
void fill_bubble(Grid& g, const Geo& geo, double gamma)
{
  fill_periodic(g, geo);
  const Cons left = to_cons(bubble_post_shock(), gamma);
  for (int j = -2; j < g.ny + 2; ++j)
    for (int i = -2; i < g.nx + 2; ++i) {
      const bool ox = i < 0 || i >= g.nx, oy = j < 0 || j >= g.ny;
      if (!ox && !oy) continue;
      if (i < 0) { g.set(i, j, left); continue; }
      const int ii = i >= g.nx ? g.nx - 1 : i;
      int jj = j;
      bool refl = false;
      if (j < 0) { jj = -j - 1; refl = true; }
      else if (j >= g.ny) { jj = g.ny - 1; }
      jj = clampi(jj, g.ny);
      Cons c = g.cons(ii, jj);
      if (refl) c.my = -c.my;
      g.set(i, j, c);
    }
}

// Mach 1.22 configuration: post-shock inflow left, copy right, mirror walls
// (-rho v) at y = 0 and y = 1.
void fill_mach122(Grid& g, double gamma)
{
  const Cons left = to_cons(mach122_post_shock(gamma), gamma);
  for (int j = -2; j < g.ny + 2; ++j)
    for (int i = -2; i < g.nx + 2; ++i) {
      const bool ox = i < 0 || i >= g.nx, oy = j < 0 || j >= g.ny;
      if (!ox && !oy) continue;
      if (i < 0) { g.set(i, j, left); continue; }
      const int ii = i >= g.nx ? g.nx - 1 : i;
      int jj = j;
      bool refl = false;
      if (j < 0) { jj = -j - 1; refl = true; }
      else if (j >= g.ny) { jj = 2 * g.ny - 1 - j; refl = true; }
      jj = clampi(jj, g.ny);
      Cons c = g.cons(ii, jj);
      if (refl) c.my = -c.my;
      g.set(i, j, c);
    }
}

// exact-state Dirichlet fills, boundary_conditions.hpp:133-163,
// problem_initialization.hpp:209-263,308-375
void fill_exact(Grid& g, const Geo& geo, const ecg_run_config& c, double time)
{
  fill_periodic(g, geo);
  Prim tl{}, tr{};
  if (c.problem == ECG_PROBLEM_TORO1) toro_states(c.toro_test, tl, tr);
  for (int j = -2; j < g.ny + 2; ++j)
    for (int i = -2; i < g.nx + 2; ++i) {
      const bool xp = !geo.per[0] && (i < 0 || i >= g.nx);
      const bool yp = !geo.per[1] && (j < 0 || j >= g.ny);
      Prim q{};
      if (c.problem == ECG_PROBLEM_TORO1) {
        if (!(i < 0 || i >= g.nx || yp)) continue;
        q = riemann_sample(geo.xc(i), time, tl, tr, c.gamma, c.riemann_interface_x);
      } else {
        if (!(xp || yp)) continue;
        if (c.problem == ECG_PROBLEM_GRESHO_VORTEX) {
          q = gresho(geo.xc(i), geo.yc(j), c);
        } else if (c.problem == ECG_PROBLEM_RIEMANN_QUADRANT) {
          q = quadrant(geo.xc(i), geo.yc(j), c);
        } else {  // advection blob
          const int ii = geo.per[0] ? wrap(i, g.nx) : i;
          const int jj = geo.per[1] ? wrap(j, g.ny) : j;
          const double x = geo.xc(ii), y = geo.yc(jj);
          const double cx = c.blob_cx + c.velocity_x * time, cy = c.blob_cy + c.velocity_y * time;
          const double r2 = (x - cx) * (x - cx) + (y - cy) * (y - cy);
          const double rho = r2 <= c.blob_radius * c.blob_radius ? c.density_inner : c.density_outer;
          q = Prim{rho, c.velocity_x, c.velocity_y, c.pressure};
        }
      }
      g.set(i, j, to_cons(q, c.gamma));
    }
}

bool is_bubble(const ecg_run_config& c)
{
  return c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D || c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_CYLINDRICAL;
}

// fill_problem_ghosts dispatch, boundary_conditions.hpp:165-219
void fill_ghosts(Grid& g, const ecg_run_config& c, double time)
{
  const Geo geo(c);
  const bool exact = c.field_boundary == ECG_FIELD_BOUNDARY_EXACT_DIRICHLET && (!geo.per[0] || !geo.per[1]);
  if (is_bubble(c)) {
    fill_bubble(g, geo, c.gamma);
  } else if (c.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122) {
    fill_mach122(g, c.gamma);
  } else if (exact && (c.problem == ECG_PROBLEM_GRESHO_VORTEX || c.problem == ECG_PROBLEM_TORO1 ||
                       c.problem == ECG_PROBLEM_RIEMANN_QUADRANT || c.problem == ECG_PROBLEM_ADVECTION_BLOB)) {
    fill_exact(g, geo, c, time);
  } else {
    fill_outflow(g, geo);
  }
}

// ---- fluxes: numerics/reconstruction_fluxes.hpp --------------------------------

// reconstruct_state, reconstruction_fluxes.hpp:2-24
Prim recon(const Grid& g, int i, int j, int axis, int side, int order, double gm, int lim)
{
  const Prim q = to_prim(g.cons(i, j), gm);
  if (order <= 1) return q;
  const Prim qm = axis == 0 ? to_prim(g.cons(i - 1, j), gm) : to_prim(g.cons(i, j - 1), gm);
  const Prim qp = axis == 0 ? to_prim(g.cons(i + 1, j), gm) : to_prim(g.cons(i, j + 1), gm);
  const double h = 0.5 * side;
  return Prim{q.rho + h * slope1(q.rho - qm.rho, qp.rho - q.rho, lim),
              q.u + h * slope1(q.u - qm.u, qp.u - q.u, lim),
              q.v + h * slope1(q.v - qm.v, qp.v - q.v, lim),
              q.p + h * slope1(q.p - qm.p, qp.p - q.p, lim)};
}

// physical_flux, reconstruction_fluxes.hpp:66-74
Cons pflux(const Prim& q, int axis, double g)
{
  const Cons u = to_cons(q, g);
  if (axis == 0) return Cons{u.mx, u.mx * q.u + q.p, u.my * q.u, (u.E + q.p) * q.u};
  return Cons{u.my, u.mx * q.v, u.my * q.v + q.p, (u.E + q.p) * q.v};
}

// rusanov_flux, reconstruction_fluxes.hpp:82-92
Cons rusanov(const Prim& l, const Prim& r, int axis, double g)
{
  const Cons ul = to_cons(l, g), ur = to_cons(r, g), fl = pflux(l, axis, g), fr = pflux(r, axis, g);
  const double sm = cmax(std::abs(normal_vel(l, axis)) + csound(l, g), std::abs(normal_vel(r, axis)) + csound(r, g));
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
              0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// hllc_star_state_is_degenerate, reconstruction_fluxes.hpp:117-149
bool hllc_degenerate(const Prim& l, const Prim& r, int axis, double g)
{
  const double ul = normal_vel(l, axis), ur = normal_vel(r, axis);
  const double cl = csound(l, g), cr = csound(r, g);
  const double sl = cmin(ul - cl, ur - cr), sr = cmax(ul + cl, ur + cr);
  if (!(sl < sr)) return true;
  if (sl >= 0.0 || sr <= 0.0) return false;
  const double den = l.rho * (sl - ul) - r.rho * (sr - ur);
  if (std::abs(den) <= 1.0e-12) return true;
  const double sm = (r.p - l.p + l.rho * ul * (sl - ul) - r.rho * ur * (sr - ur)) / den;
  return std::abs(sl - sm) <= 1.0e-12 || std::abs(sr - sm) <= 1.0e-12;
}

// hllc_flux, reconstruction_fluxes.hpp:151-210
Cons hllc(const Prim& l, const Prim& r, int axis, double g)
{
  const Cons ul = to_cons(l, g), ur = to_cons(r, g), fl = pflux(l, axis, g), fr = pflux(r, axis, g);
  const double unl = normal_vel(l, axis), unr = normal_vel(r, axis);
  const double cl = csound(l, g), cr = csound(r, g);
  const double sl = cmin(unl - cl, unr - cr), sr = cmax(unl + cl, unr + cr);
  if (!(sl < sr)) return rusanov(l, r, axis, g);
  if (sl >= 0.0) return fl;
  if (sr <= 0.0) return fr;
  const double den = l.rho * (sl - unl) - r.rho * (sr - unr);
  if (std::abs(den) <= 1.0e-12) return rusanov(l, r, axis, g);
  const double sm = (r.p - l.p + l.rho * unl * (sl - unl) - r.rho * unr * (sr - unr)) / den;
  const double lsd = sl - sm, rsd = sr - sm;
  if (std::abs(lsd) <= 1.0e-12 || std::abs(rsd) <= 1.0e-12) return rusanov(l, r, axis, g);
  const double psl = l.p + l.rho * (sl - unl) * (sm - unl);
  const double psr = r.p + r.rho * (sr - unr) * (sm - unr);
  const double ps = 0.5 * (psl + psr);
  // Only the upwind star state enters the flux (reconstruction_fluxes.hpp:206-209).
  const bool use_left = sm >= 0.0;
  const Prim& q = use_left ? l : r;
  const Cons& u = use_left ? ul : ur;
  const Cons& f = use_left ? fl : fr;
  const double s = use_left ? sl : sr, un = use_left ? unl : unr, sd = use_left ? lsd : rsd;
  const double rs = q.rho * (s - un) / sd;
  const double es = ((s - un) * u.E - q.p * un + ps * sm) / sd;
  const double tang = axis == 0 ? q.v : q.u;
  Cons st{};
  if (axis == 0) st = Cons{rs, rs * sm, rs * tang, es};
  else st = Cons{rs, rs * tang, rs * sm, es};
  return Cons{f.rho + s * (st.rho - u.rho), f.mx + s * (st.mx - u.mx), f.my + s * (st.my - u.my), f.E + s * (st.E - u.E)};
}

// low_mach_correct_velocity_states, reconstruction_fluxes.hpp:212-232
void lowmach_correct(const Prim& l, const Prim& r, double g, Prim& cl, Prim& cr)
{
  const double al = csound(l, g), ar = csound(r, g);
  const double sl = std::sqrt(l.u * l.u + l.v * l.v), sr = std::sqrt(r.u * r.u + r.v * r.v);
  const double ml = sl / cmax(al, 1.0e-12), mr = sr / cmax(ar, 1.0e-12);
  const double z = cmin(cmax(cmax(ml, mr), 0.0), 1.0);
  cl = l;
  cr = r;
  const double ua = 0.5 * (l.u + r.u), va = 0.5 * (l.v + r.v);
  cl.u = ua + 0.5 * z * (l.u - r.u);
  cr.u = ua + 0.5 * z * (r.u - l.u);
  cl.v = va + 0.5 * z * (l.v - r.v);
  cr.v = va + 0.5 * z * (r.v - l.v);
}

inline double clamp01(double v) { return cmin(cmax(v, 0.0), 1.0); }

// xie_am_hllc_p_flux, reconstruction_fluxes.hpp:254-371
Cons xie(const Prim& l, const Prim& r, int axis, double g, double sensor)
{
  const Cons ul = to_cons(l, g), ur = to_cons(r, g), fl = pflux(l, axis, g), fr = pflux(r, axis, g);
  const double ql = normal_vel(l, axis), qr = normal_vel(r, axis);
  const double pl = l.p, pr = r.p;
  const double cl = csound(l, g), cr = csound(r, g);
  const double sl = cmin(ql - cl, qr - cr), sr = cmax(ql + cl, qr + cr);
  if (!(sl < sr)) return hllc(l, r, axis, g);
  if (sl >= 0.0) return fl;
  if (sr <= 0.0) return fr;
  const double al = l.rho * (sl - ql), ar = r.rho * (sr - qr);
  const double ad = ar - al;
  if (std::abs(ad) <= 1.0e-12) return hllc(l, r, axis, g);
  const double ss = (ar * qr - al * ql + pl - pr) / ad;
  const double dl = sl - ss, dr = sr - ss;
  if (std::abs(dl) <= 1.0e-12 || std::abs(dr) <= 1.0e-12 || std::abs(al) <= 1.0e-12 || std::abs(ar) <= 1.0e-12)
    return hllc(l, r, axis, g);
  const double rsl = al / dl, rsr = ar / dr;
  const double el = ul.E / l.rho, er = ur.E / r.rho;
  const double esl = el + (ss - ql) * (ss + pl / al);
  const double esr = er + (ss - qr) * (ss + pr / ar);
  const double ps = (ar * pl - al * pr - al * ar * (ql - qr)) / ad;
  const double srl = std::sqrt(l.rho), srr = std::sqrt(r.rho);
  const double rd = srl + srr;
  if (!(rd > 0.0)) return hllc(l, r, axis, g);
  const double uh = (srl * l.u + srr * r.u) / rd;
  const double vh = (srl * l.v + srr * r.v) / rd;
  const double qh = axis == 0 ? uh : vh;
  const double hl = (ul.E + pl) / l.rho, hr = (ur.E + pr) / r.rho;
  const double hh = (srl * hl + srr * hr) / rd;
  const double c2 = (g - 1.0) * (hh - 0.5 * (uh * uh + vh * vh));
  if (!(c2 > 0.0) || !std::isfinite(c2)) return hllc(l, r, axis, g);
  const double ch = std::sqrt(c2);
  const double mh = qh / cmax(ch, 1.0e-12);
  const double spl = std::sqrt(l.u * l.u + l.v * l.v), spr = std::sqrt(r.u * r.u + r.v * r.v);
  const double th = clamp01(cmax(spl / cmax(cl, 1.0e-12), spr / cmax(cr, 1.0e-12)));
  const double f = clamp01(sensor);
  const double pss = th * ps + (1.0 - th) * 0.5 * (pl + pr);
  const double psss = f * pss + (1.0 - f) * ps;
  const double bp = (f - 1.0) * sl * sr / (sr - sl) * (pr - pl) / (c2 * (1.0 + std::abs(mh)));
  const Cons phi{bp, bp * uh, bp * vh, 0.5 * bp * (uh * uh + vh * vh)};
  const double nxv = axis == 0 ? 1.0 : 0.0, nyv = axis == 1 ? 1.0 : 0.0;
  const bool use_left = ss >= 0.0;
  const Prim& q = use_left ? l : r;
  const double qn = use_left ? ql : qr, rs = use_left ? rsl : rsr, es = use_left ? esl : esr;
  const Cons sf{rs * ss, rs * ss * (q.u + nxv * (ss - qn)) + nxv * psss,
                rs * ss * (q.v + nyv * (ss - qn)) + nyv * psss, ss * (rs * es + ps)};
  const Cons out{sf.rho + phi.rho, sf.mx + phi.mx, sf.my + phi.my, sf.E + phi.E};
  if (!std::isfinite(out.rho) || !std::isfinite(out.mx) || !std::isfinite(out.my) || !std::isfinite(out.E))
    return hllc(l, r, axis, g);
  return out;
}

// xie_pressure_ratio_from_states, reconstruction_fluxes.hpp:390-397
double pratio(const Prim& l, const Prim& r)
{
  const double fl = 1.0e-14;
  const double pl = std::isfinite(l.p) ? cmax(l.p, fl) : fl;
  const double pr = std::isfinite(r.p) ? cmax(r.p, fl) : fl;
  return clamp01(cmin(pl / pr, pr / pl));
}

struct FluxCtx {
  const Grid* g;
  double gm;
  int order, lim, riemann;
};

double xratio(const FluxCtx& c, int fi, int j)
{
  return pratio(recon(*c.g, fi - 1, j, 0, +1, c.order, c.gm, c.lim), recon(*c.g, fi, j, 0, -1, c.order, c.gm, c.lim));
}
double yratio(const FluxCtx& c, int i, int fj)
{
  return pratio(recon(*c.g, i, fj - 1, 1, +1, c.order, c.gm, c.lim), recon(*c.g, i, fj, 1, -1, c.order, c.gm, c.lim));
}

// xie_multiface_pressure_sensor, reconstruction_fluxes.hpp:421-440
double xie_sensor(const FluxCtx& c, int fi, int fj, int axis)
{
  double f;
  if (axis == 0) {
    f = xratio(c, fi, fj);
    f = cmin(f, yratio(c, fi - 1, fj));
    f = cmin(f, yratio(c, fi - 1, fj + 1));
    f = cmin(f, yratio(c, fi, fj));
    f = cmin(f, yratio(c, fi, fj + 1));
  } else {
    f = yratio(c, fi, fj);
    f = cmin(f, xratio(c, fi, fj - 1));
    f = cmin(f, xratio(c, fi + 1, fj - 1));
    f = cmin(f, xratio(c, fi, fj));
    f = cmin(f, xratio(c, fi + 1, fj));
  }
  const double h = clamp01(f);
  return h * h * h;
}

// reconstructed_interface_flux + interface_flux, reconstruction_fluxes.hpp:373-388,442-460
Cons face_flux(const FluxCtx& c, int fi, int fj, int axis)
{
  Prim l, r;
  if (axis == 0) {
    l = recon(*c.g, fi - 1, fj, 0, +1, c.order, c.gm, c.lim);
    r = recon(*c.g, fi, fj, 0, -1, c.order, c.gm, c.lim);
  } else {
    l = recon(*c.g, fi, fj - 1, 1, +1, c.order, c.gm, c.lim);
    r = recon(*c.g, fi, fj, 1, -1, c.order, c.gm, c.lim);
  }
  switch (c.riemann) {
    case ECG_RIEMANN_RUSANOV: return rusanov(l, r, axis, c.gm);
    case ECG_RIEMANN_LOWMACH_HLLC: {
      Prim cl, cr;
      lowmach_correct(l, r, c.gm, cl, cr);
      return hllc(cl, cr, axis, c.gm);
    }
    case ECG_RIEMANN_XIE_AM_HLLC_P: return xie(l, r, axis, c.gm, xie_sensor(c, fi, fj, axis));
    default: return hllc(l, r, axis, c.gm);
  }
}

bool face_degenerate(const FluxCtx& c, int fi, int fj, int axis)
{
  Prim l, r;
  if (axis == 0) {
    l = recon(*c.g, fi - 1, fj, 0, +1, c.order, c.gm, c.lim);
    r = recon(*c.g, fi, fj, 0, -1, c.order, c.gm, c.lim);
  } else {
    l = recon(*c.g, fi, fj - 1, 1, +1, c.order, c.gm, c.lim);
    r = recon(*c.g, fi, fj, 1, -1, c.order, c.gm, c.lim);
  }
  if (c.riemann == ECG_RIEMANN_LOWMACH_HLLC) {
    Prim cl, cr;
    lowmach_correct(l, r, c.gm, cl, cr);
    return hllc_degenerate(cl, cr, axis, c.gm);
  }
  return hllc_degenerate(l, r, axis, c.gm);
}

// euler_fv_one_step + count_hllc_degenerate_star_states, numerics/explicit_update.hpp:2-102
int fv_one_step(const ecg_run_config& cfg, Grid& gr, double dt, double time)
{
  fill_ghosts(gr, cfg, time);
  const Geo geo(cfg);
  const FluxCtx fc{&gr, cfg.gamma, cfg.spatial_order, cfg.slope_limiter, cfg.riemann};
  const int nx = gr.nx, ny = gr.ny;
  int degenerate = 0;
  if (cfg.riemann != ECG_RIEMANN_RUSANOV) {
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        degenerate += (face_degenerate(fc, i, j, 0) ? 1 : 0) + (face_degenerate(fc, i + 1, j, 0) ? 1 : 0) +
                      (face_degenerate(fc, i, j, 1) ? 1 : 0) + (face_degenerate(fc, i, j + 1, 1) ? 1 : 0);
  }
  // Each face flux once; (nx+1) x ny x-faces, nx x (ny+1) y-faces.
  std::vector<Cons> fx(static_cast<std::size_t>(nx + 1) * ny), fy(static_cast<std::size_t>(nx) * (ny + 1));
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i <= nx; ++i) fx[static_cast<std::size_t>(j) * (nx + 1) + i] = face_flux(fc, i, j, 0);
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i < nx; ++i) fy[static_cast<std::size_t>(j) * nx + i] = face_flux(fc, i, j, 1);
  const double idx = 1.0 / geo.dx, idy = 1.0 / geo.dy;
  Grid out(nx, ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const Cons& l = fx[static_cast<std::size_t>(j) * (nx + 1) + i];
      const Cons& r = fx[static_cast<std::size_t>(j) * (nx + 1) + i + 1];
      const Cons& b = fy[static_cast<std::size_t>(j) * nx + i];
      const Cons& t = fy[static_cast<std::size_t>(j + 1) * nx + i];
      const Cons o = gr.cons(i, j);
      out.set(i, j, Cons{o.rho - dt * ((r.rho - l.rho) * idx + (t.rho - b.rho) * idy),
                         o.mx - dt * ((r.mx - l.mx) * idx + (t.mx - b.mx) * idy),
                         o.my - dt * ((r.my - l.my) * idx + (t.my - b.my) * idy),
                         o.E - dt * ((r.E - l.E) * idx + (t.E - b.E) * idy)});
    }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) gr.set(i, j, out.cons(i, j));
  return degenerate;
}

// compute_euler_dt, numerics/diagnostic_metrics_timestep.hpp:227-260
double euler_dt(const ecg_run_config& cfg, const Grid& gr, double time)
{
  const Geo geo(cfg);
  double mr = std::numeric_limits<double>::lowest();
  for (int j = 0; j < gr.ny; ++j)
    for (int i = 0; i < gr.nx; ++i) {
      const Prim q = to_prim(gr.cons(i, j), cfg.gamma);
      const double c = csound(q, cfg.gamma);
      mr = cmax(mr, (std::abs(q.u) + c) / geo.dx + (std::abs(q.v) + c) / geo.dy);
    }
  double dt = cfg.stop_time - time;
  if (mr > 0.0) dt = cfg.cfl / mr;
  if (!std::isfinite(dt) || dt <= 0.0) dt = cfg.stop_time - time;
  return std::min(dt, cfg.stop_time - time);
}

// compute_imex_dt, diagnostic_metrics_timestep.hpp:262-326
double imex_dt(const ecg_run_config& cfg, const Grid& gr, double time, ecg_imex_timestep_diag* d)
{
  const Geo geo(cfg);
  const double mdx = std::min(geo.dx, geo.dy);
  const bool eq79 = cfg.method == ECG_METHOD_IMEX && cfg.imex_acoustic_startup == 0 && cfg.imex_acoustic_cfl_cap == 0.0;
  double mat = std::numeric_limits<double>::lowest(), aco = std::numeric_limits<double>::lowest();
  for (int j = 0; j < gr.ny; ++j)
    for (int i = 0; i < gr.nx; ++i) {
      const Prim q = to_prim(gr.cons(i, j), cfg.gamma);
      const double c = csound(q, cfg.gamma);
      const double sp = std::sqrt(q.u * q.u + q.v * q.v);
      const double m = eq79 ? (2.0 * sp / mdx) : (std::abs(q.u) / geo.dx + std::abs(q.v) / geo.dy);
      mat = cmax(mat, m);
      aco = cmax(aco, (std::abs(q.u) + c) / geo.dx + (std::abs(q.v) + c) / geo.dy);
    }
  ecg_imex_timestep_diag td{mat, aco, 0, 0};
  double rate = mat;
  if (cfg.imex_acoustic_startup != 0 && mat <= 1.0e-12 && aco > 0.0) { rate = aco; td.acoustic_startup_used = 1; }
  double dt = cfg.stop_time - time;
  if (rate > 0.0) dt = cfg.imex_cfl / rate;
  if (cfg.imex_acoustic_cfl_cap > 0.0 && aco > 0.0) {
    const double lim = cfg.imex_acoustic_cfl_cap / aco;
    if (lim < dt) { dt = lim; td.acoustic_cap_used = 1; }
  }
  if (!std::isfinite(dt) || dt <= 0.0) dt = cfg.stop_time - time;
  if (d) *d = td;
  return std::min(dt, cfg.stop_time - time);
}

// compute_diagnostics, diagnostic_metrics_timestep.hpp:18-47
ecg_diagnostics diagnostics(const ecg_run_config& cfg, const Grid& gr)
{
  ecg_diagnostics d{std::numeric_limits<double>::max(), std::numeric_limits<double>::max(), 0};
  for (int j = 0; j < gr.ny; ++j)
    for (int i = 0; i < gr.nx; ++i) {
      const Cons u = gr.cons(i, j);
      const Prim q = to_prim(u, cfg.gamma);
      const bool bad = !std::isfinite(q.rho) || !std::isfinite(q.u) || !std::isfinite(q.v) || !std::isfinite(q.p) ||
                       !std::isfinite(u.E);
      d.rho_min = cmin(d.rho_min, bad ? -kInf : q.rho);
      d.pressure_min = cmin(d.pressure_min, bad ? -kInf : q.p);
      d.nonfinite_count += bad ? 1 : 0;
    }
  return d;
}

// compute_admissibility_diagnostics, diagnostic_metrics_timestep.hpp:49-111
ecg_admissibility admissibility(const ecg_run_config& cfg, const Grid& gr)
{
  const double big = std::numeric_limits<double>::max();
  ecg_admissibility a{big, big, big, 0, 0, 0, 0};
  for (int j = 0; j < gr.ny; ++j)
    for (int i = 0; i < gr.nx; ++i) {
      const Cons u = gr.cons(i, j);
      const bool cnf = !std::isfinite(u.rho) || !std::isfinite(u.mx) || !std::isfinite(u.my) || !std::isfinite(u.E);
      const bool dbad = !cnf && u.rho <= 0.0;
      double ie = -kInf, p = -kInf;
      bool tnf = false;
      if (!cnf && !dbad) {
        const double kin = 0.5 * (u.mx * u.mx + u.my * u.my) / u.rho;
        ie = u.E - kin;
        p = (cfg.gamma - 1.0) * ie;
        tnf = !std::isfinite(kin) || !std::isfinite(ie) || !std::isfinite(p);
      }
      const bool nf = cnf || tnf;
      const bool pbad = !nf && !dbad && p <= 0.0;
      const bool ibad = !nf && !dbad && ie <= 0.0;
      a.rho_min = cmin(a.rho_min, nf ? -kInf : u.rho);
      a.pressure_min = cmin(a.pressure_min, (nf || dbad) ? -kInf : p);
      a.internal_energy_min = cmin(a.internal_energy_min, (nf || dbad) ? -kInf : ie);
      a.nonfinite_count += nf ? 1 : 0;
      a.density_failure_count += dbad ? 1 : 0;
      a.pressure_failure_count += pbad ? 1 : 0;
      a.internal_energy_failure_count += ibad ? 1 : 0;
    }
  return a;
}

// ---- IMEX T1/S2 source-map step -------------------------------------------------

// conserved minmod reconstruction (BDLTV20 eq 87-89), reconstruction_fluxes.hpp:26-52
Prim recon_cons_minmod(const Grid& g, int i, int j, int axis, int side, double gm)
{
  const Cons u = g.cons(i, j);
  const Cons um = axis == 0 ? g.cons(i - 1, j) : g.cons(i, j - 1);
  const Cons up = axis == 0 ? g.cons(i + 1, j) : g.cons(i, j + 1);
  const double h = 0.5 * side;
  const Cons s{mm(u.rho - um.rho, up.rho - u.rho), mm(u.mx - um.mx, up.mx - u.mx), mm(u.my - um.my, up.my - u.my),
               mm(u.E - um.E, up.E - u.E)};
  return to_prim(Cons{u.rho + h * s.rho, u.mx + h * s.mx, u.my + h * s.my, u.E + h * s.E}, gm);
}

// pressure_split_explicit_flux + bdltv20_pressure_split_lf_flux (material speed),
// reconstruction_fluxes.hpp:462-484,504-515
Cons split_lf(const Prim& l, const Prim& r, int axis, double g)
{
  const Cons ul = to_cons(l, g), ur = to_cons(r, g);
  auto ef = [axis](const Prim& q) {
    const double mx = q.rho * q.u, my = q.rho * q.v;
    const double kin = 0.5 * q.rho * (q.u * q.u + q.v * q.v);
    if (axis == 0) return Cons{mx, mx * q.u, my * q.u, kin * q.u};
    return Cons{my, mx * q.v, my * q.v, kin * q.v};
  };
  const Cons fl = ef(l), fr = ef(r);
  const double sm = cmax(std::abs(normal_vel(l, axis)), std::abs(normal_vel(r, axis)));
  const double hs = 0.5 * sm;
  return Cons{0.5 * (fl.rho + fr.rho) - hs * (ur.rho - ul.rho), 0.5 * (fl.mx + fr.mx) - hs * (ur.mx - ul.mx),
              0.5 * (fl.my + fr.my) - hs * (ur.my - ul.my), 0.5 * (fl.E + fr.E) - hs * (ur.E - ul.E)};
}

// compute_bdltv20_pressure_split_star, imex/imex_source_map_helpers.hpp:2-68
void imex_star(const ecg_run_config& cfg, const Grid& g, double dt, Grid& star)
{
  const Geo geo(cfg);
  const double idx = 1.0 / geo.dx, idy = 1.0 / geo.dy, gm = cfg.gamma;
  auto lf = [&](int il, int jl, int ir, int jr, int axis) {
    return split_lf(recon_cons_minmod(g, il, jl, axis, +1, gm), recon_cons_minmod(g, ir, jr, axis, -1, gm), axis, gm);
  };
  for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
      const Cons l = lf(i - 1, j, i, j, 0), r = lf(i, j, i + 1, j, 0);
      const Cons b = lf(i, j - 1, i, j, 1), t = lf(i, j, i, j + 1, 1);
      const Cons o = g.cons(i, j);
      star.set(i, j, Cons{o.rho - dt * ((r.rho - l.rho) * idx + (t.rho - b.rho) * idy),
                          o.mx - dt * ((r.mx - l.mx) * idx + (t.mx - b.mx) * idy),
                          o.my - dt * ((r.my - l.my) * idx + (t.my - b.my) * idy),
                          o.E - dt * ((r.E - l.E) * idx + (t.E - b.E) * idy)});
    }
}

// CoupledHostGrid + boundary maps, imex_source_map_helpers.hpp:70-245
struct Host {
  int nx, ny;
  bool px, py, bubble;
  double gamma;
  std::vector<Cons> cell;
  // The Mach 1.22 variant (no reference counterpart): the bubble's policy with
  // its own post-shock inflow state, and a wall at the top as well.
  bool mach122 = false;
  Prim post() const { return mach122 ? mach122_post_shock(gamma) : bubble_post_shock(); }
  int row(int i, int j) const { return j * nx + i; }
  int mi(int i) const { return px ? wrap(i, nx) : clampi(i, nx); }
  int mj(int j) const { return py ? wrap(j, ny) : clampi(j, ny); }
  const Cons& at(int i, int j) const { return cell[static_cast<std::size_t>(row(mi(i), mj(j)))]; }
  // source_map_index: periodic wrap or even Neumann reflection, :169-188
  static int pmap(int k, int n, bool per) {
    if (per) return wrap(k, n);
    if (k < 0) return std::min(-k - 1, n - 1);
    if (k >= n) return std::max(n - (k - n + 1), 0);
    return k;
  }
  int prow(int i, int j) const { return row(pmap(i, nx, px), pmap(j, ny, py)); }
  bool fixed_p(int i) const { return bubble && !px && i < 0; }  // :222-233
  // source_map_state_at_physical_boundary, :98-115
  Cons state_b(int i, int j) const {
    if (bubble) {
      if (!px && i < 0) return to_cons(post(), gamma);
      const int ii = mi(i);
      if (!py && j < 0) { Cons c = at(ii, 0); c.my = -c.my; return c; }
      if (mach122 && !py && j >= ny) { Cons c = at(ii, ny - 1); c.my = -c.my; return c; }
      return at(ii, mj(j));
    }
    return at(i, j);
  }
  // source_map_pressure_at_physical_boundary, :235-245
  double p_b(const std::vector<double>& p, int i, int j) const {
    if (fixed_p(i)) return post().p;
    return p[static_cast<std::size_t>(prow(i, j))];
  }
  // source_map_lagged_momentum_at(_physical_boundary), :293-320
  void m_at(const std::vector<double>& k, int i, int j, double& m0, double& m1) const {
    const std::size_t r = static_cast<std::size_t>(row(mi(i), mj(j)));
    m0 = k[2 * r]; m1 = k[2 * r + 1];
  }
  void m_b(const std::vector<double>& k, int i, int j, double& m0, double& m1) const {
    if (bubble) {
      if (!px && i < 0) { const Cons c = to_cons(post(), gamma); m0 = c.mx; m1 = c.my; return; }
      const int ii = mi(i);
      if (!py && j < 0) { m_at(k, ii, 0, m0, m1); m1 = -m1; return; }
      if (mach122 && !py && j >= ny) { m_at(k, ii, ny - 1, m0, m1); m1 = -m1; return; }
    }
    m_at(k, i, j, m0, m1);
  }
};

Host imex_host(const ecg_run_config& c, int nx, int ny, const Geo& geo)
{
  Host h{nx, ny, geo.per[0], geo.per[1],
         c.problem == ECG_PROBLEM_SHOCK_DENSITY_BUBBLE_2D || c.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122, c.gamma, {}};
  h.mach122 = c.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122;
  return h;
}

struct Face { double h_hat, energy_flux, hl, hr, ql, qr; int guard, flux_nonfinite; };

// source_map_face_flux_detail, imex_source_map_helpers.hpp:359-402
Face face_detail(const Host& h, const std::vector<double>& p, const std::vector<double>& k, int il, int jl, int ir,
                 int jr, int axis)
{
  const double gm1 = h.gamma - 1.0;
  const Cons L = h.state_b(il, jl), R = h.state_b(ir, jr);
  double ml0, ml1, mr0, mr1;
  h.m_b(k, il, jl, ml0, ml1);
  h.m_b(k, ir, jr, mr0, mr1);
  Face f{};
  const double pl = h.p_b(p, il, jl), pr = h.p_b(p, ir, jr);
  f.hl = h.gamma * pl / (gm1 * L.rho);
  f.hr = h.gamma * pr / (gm1 * R.rho);
  f.ql = axis == 0 ? ml0 : ml1;
  f.qr = axis == 0 ? mr0 : mr1;
  const double den = f.ql + f.qr;
  const double scale = std::max({std::abs(f.ql), std::abs(f.qr), 1.0});
  f.guard = std::abs(den) <= 1.0e-14 * scale ? 1 : 0;
  f.h_hat = f.guard != 0 ? 0.5 * (f.hl + f.hr) : (f.hl * f.ql + f.hr * f.qr) / den;
  const double mhat = 0.5 * (f.ql + f.qr);
  f.energy_flux = f.h_hat * mhat;
  f.flux_nonfinite = std::isfinite(f.energy_flux) ? 0 : 1;
  return f;
}

// source_map_eq54_corrected_momentum_field (physical-boundary pressure), :249-268,334-346
std::vector<double> corrected_momentum(const Host& h, const std::vector<double>& p, double dt, double idx, double idy)
{
  std::vector<double> k(static_cast<std::size_t>(2) * h.nx * h.ny);
  for (int j = 0; j < h.ny; ++j)
    for (int i = 0; i < h.nx; ++i) {
      const Cons& s = h.at(i, j);
      const double gx = 0.5 * (h.p_b(p, i + 1, j) - h.p_b(p, i - 1, j)) * idx;
      const double gy = 0.5 * (h.p_b(p, i, j + 1) - h.p_b(p, i, j - 1)) * idy;
      const std::size_t r = static_cast<std::size_t>(h.row(i, j));
      k[2 * r] = s.mx - dt * gx;
      k[2 * r + 1] = s.my - dt * gy;
    }
  return k;
}

// CSR with duplicate columns summed in insertion order and zero coefficients
// dropped, as source_map_build_pressure_system + setFromTriplets build it
// (imex_source_map_step.hpp:8-38).
struct Csr {
  int n = 0;
  std::vector<int> rp, col;
  std::vector<double> val;
  void mul(const std::vector<double>& x, std::vector<double>& y) const {
    y.assign(static_cast<std::size_t>(n), 0.0);
    for (int r = 0; r < n; ++r) {
      double s = 0.0;
      for (int q = rp[r]; q < rp[r + 1]; ++q) s += val[q] * x[col[q]];
      y[r] = s;
    }
  }
};

// source_map_pressure_row_data for every row, imex_source_map_helpers.hpp:473-571
void build_system(const Host& h, const std::vector<double>& p, const std::vector<double>& k, double dt, double idx,
                  double idy, Csr& A, std::vector<double>& rhs, int& nonfinite)
{
  const int n = h.nx * h.ny;
  const double gm1 = h.gamma - 1.0;
  const double xc = 0.25 * dt * dt * idx * idx, yc = 0.25 * dt * dt * idy * idy;
  A.n = n;
  A.rp.assign(static_cast<std::size_t>(n) + 1, 0);
  A.col.clear();
  A.val.clear();
  rhs.assign(static_cast<std::size_t>(n), 0.0);
  nonfinite = 0;
  for (int j = 0; j < h.ny; ++j)
    for (int i = 0; i < h.nx; ++i) {
      const int r = h.row(i, j);
      int rnf = 0;
      double b = 0.0;
      std::vector<std::pair<int, double>> terms;
      auto lhs = [&](int pi, int pj, double coeff) {
        if (h.fixed_p(pi)) {
          const double c = -coeff * h.post().p;
          b += c;
          if (!std::isfinite(c)) ++rnf;
          return;
        }
        terms.emplace_back(h.prow(pi, pj), coeff);
        if (!std::isfinite(coeff)) ++rnf;
      };
      auto add = [&](double v) {
        if (!std::isfinite(v)) ++rnf;
        b += v;
      };
      const double he = face_detail(h, p, k, i, j, i + 1, j, 0).h_hat;
      const double hw = face_detail(h, p, k, i - 1, j, i, j, 0).h_hat;
      const double hn = face_detail(h, p, k, i, j, i, j + 1, 1).h_hat;
      const double hs = face_detail(h, p, k, i, j - 1, i, j, 1).h_hat;
      if (!std::isfinite(he) || !std::isfinite(hw) || !std::isfinite(hn) || !std::isfinite(hs)) ++rnf;
      lhs(i, j, 1.0 / gm1);
      lhs(i + 2, j, -xc * he);
      lhs(i + 1, j, -xc * (he - hw));
      lhs(i, j, xc * (he + hw));
      lhs(i - 1, j, xc * (he - hw));
      lhs(i - 2, j, -xc * hw);
      lhs(i, j + 2, -yc * hn);
      lhs(i, j + 1, -yc * (hn - hs));
      lhs(i, j, yc * (hn + hs));
      lhs(i, j - 1, yc * (hn - hs));
      lhs(i, j - 2, -yc * hs);
      const Cons& s = h.at(i, j);
      double k0, k1;
      h.m_at(k, i, j, k0, k1);
      const double kin = 0.5 * (k0 * k0 + k1 * k1) / s.rho;
      add(s.E);
      add(-kin);
      add(-0.5 * dt * idx * he * h.state_b(i + 1, j).mx);
      add(-0.5 * dt * idx * (he - hw) * h.at(i, j).mx);
      add(0.5 * dt * idx * hw * h.state_b(i - 1, j).mx);
      add(-0.5 * dt * idy * hn * h.state_b(i, j + 1).my);
      add(-0.5 * dt * idy * (hn - hs) * h.at(i, j).my);
      add(0.5 * dt * idy * hs * h.state_b(i, j - 1).my);
      if (!std::isfinite(b)) ++rnf;
      nonfinite += rnf;
      rhs[static_cast<std::size_t>(r)] = b;
      // merge: nonzero terms, duplicates summed in insertion order, sorted by column
      std::vector<std::pair<int, double>> merged;
      for (const auto& t : terms) {
        if (t.second == 0.0) continue;
        bool found = false;
        for (auto& m : merged)
          if (m.first == t.first) { m.second = m.second + t.second; found = true; break; }
        if (!found) merged.push_back(t);
      }
      std::sort(merged.begin(), merged.end(), [](const auto& a, const auto& c) { return a.first < c.first; });
      for (const auto& m : merged) { A.col.push_back(m.first); A.val.push_back(m.second); }
      A.rp[static_cast<std::size_t>(r) + 1] = static_cast<int>(A.col.size());
    }
}

double linf(const std::vector<double>& v)
{
  double m = 0.0;
  for (double x : v) m = std::max(m, std::abs(x));
  return m;
}
bool all_finite(const std::vector<double>& v)
{
  for (double x : v) if (!std::isfinite(x)) return false;
  return true;
}

struct GmresOut {
  std::vector<double> x;
  int iterations = 0;
  bool converged = false, breakdown = false, nonfinite = false;
  double res_linf = kInf, rel_linf = kInf;
};

// solve_host_sparse_gmres, imex/imex_pressure_helpers.hpp:92-217: unrestarted
// GMRES with modified Gram-Schmidt, true infinity-norm residual of every
// iterate, best-iterate return, stop at ||r||inf <= tol or
// ||r||inf / max(||b||inf, 1) <= tol.  The least-squares problem is solved
// with Givens rotations.
GmresOut gmres(const Csr& A, const std::vector<double>& b, const std::vector<double>& x0, int max_iter, double tol)
{
  GmresOut out;
  out.x = x0;
  if (!all_finite(b) || !all_finite(x0)) { out.nonfinite = true; return out; }
  const int n = A.n;
  const double bn = std::max(linf(b), 1.0);
  std::vector<double> ax;
  auto check = [&](const std::vector<double>& t, int it) {
    if (!all_finite(t)) { out.nonfinite = true; return; }
    A.mul(t, ax);
    std::vector<double> r(static_cast<std::size_t>(n));
    for (int q = 0; q < n; ++q) r[q] = ax[q] - b[q];
    if (!all_finite(r)) { out.nonfinite = true; return; }
    const double rl = linf(r), rr = rl / bn;
    if (rl < out.res_linf) { out.x = t; out.iterations = it; out.res_linf = rl; out.rel_linf = rr; }
    if (rl <= tol || rr <= tol) { out.x = t; out.iterations = it; out.res_linf = rl; out.rel_linf = rr; out.converged = true; }
  };
  check(x0, 0);
  if (out.converged || out.nonfinite) return out;
  const int lim = std::max(0, std::min(max_iter, n));
  if (lim == 0) return out;
  A.mul(x0, ax);
  std::vector<double> r0(static_cast<std::size_t>(n));
  for (int q = 0; q < n; ++q) r0[q] = b[q] - ax[q];
  if (!all_finite(r0)) { out.nonfinite = true; return out; }
  double beta2 = 0.0;
  for (double v : r0) beta2 += v * v;
  const double beta = std::sqrt(beta2);
  if (!std::isfinite(beta)) { out.nonfinite = true; return out; }
  if (beta == 0.0) { out.converged = true; out.res_linf = 0.0; out.rel_linf = 0.0; return out; }
  std::vector<std::vector<double>> V;
  V.emplace_back(r0);
  for (double& v : V[0]) v = v / beta;
  const double btol = std::numeric_limits<double>::epsilon() * 100.0 * std::max(beta, 1.0);
  std::vector<std::vector<double>> R(static_cast<std::size_t>(lim), std::vector<double>(static_cast<std::size_t>(lim) + 1, 0.0));
  std::vector<double> cs(static_cast<std::size_t>(lim)), sn(static_cast<std::size_t>(lim)), gv(static_cast<std::size_t>(lim) + 1, 0.0);
  gv[0] = beta;
  std::vector<double> w;
  for (int j = 0; j < lim; ++j) {
    A.mul(V[static_cast<std::size_t>(j)], w);
    if (!all_finite(w)) { out.nonfinite = true; return out; }
    std::vector<double> hcol(static_cast<std::size_t>(j) + 2, 0.0);
    for (int i = 0; i <= j; ++i) {
      double d = 0.0;
      for (int q = 0; q < n; ++q) d += V[static_cast<std::size_t>(i)][q] * w[q];
      hcol[static_cast<std::size_t>(i)] = d;
      for (int q = 0; q < n; ++q) w[q] -= d * V[static_cast<std::size_t>(i)][q];
    }
    double nn2 = 0.0;
    for (double v : w) nn2 += v * v;
    const double nn = std::sqrt(nn2);
    if (!std::isfinite(nn)) { out.nonfinite = true; return out; }
    hcol[static_cast<std::size_t>(j) + 1] = nn;
    if (nn > btol) {
      V.emplace_back(w);
      for (double& v : V.back()) v = v / nn;
    }
    // apply previous rotations, then a new one that zeroes hcol[j+1]
    for (int i = 0; i < j; ++i) {
      const double a = hcol[i], c = hcol[i + 1];
      hcol[i] = cs[i] * a + sn[i] * c;
      hcol[i + 1] = -sn[i] * a + cs[i] * c;
    }
    const double a = hcol[j], c = hcol[j + 1];
    const double rho = std::hypot(a, c);
    cs[j] = rho == 0.0 ? 1.0 : a / rho;
    sn[j] = rho == 0.0 ? 0.0 : c / rho;
    hcol[j] = rho;
    hcol[j + 1] = 0.0;
    gv[j + 1] = -sn[j] * gv[j];
    gv[j] = cs[j] * gv[j];
    for (int i = 0; i <= j; ++i) R[static_cast<std::size_t>(j)][static_cast<std::size_t>(i)] = hcol[i];
    std::vector<double> y(static_cast<std::size_t>(j) + 1);
    for (int i = j; i >= 0; --i) {
      double s = gv[i];
      for (int m = i + 1; m <= j; ++m) s -= R[static_cast<std::size_t>(m)][static_cast<std::size_t>(i)] * y[m];
      y[i] = s / R[static_cast<std::size_t>(i)][static_cast<std::size_t>(i)];
    }
    if (!all_finite(y)) { out.nonfinite = true; return out; }
    std::vector<double> t = x0;
    for (int i = 0; i <= j; ++i)
      for (int q = 0; q < n; ++q) t[q] += y[i] * V[static_cast<std::size_t>(i)][q];
    check(t, j + 1);
    if (out.converged || out.nonfinite) return out;
    if (nn <= btol) { out.breakdown = true; return out; }
  }
  return out;
}

// euler_imex_bdltv20_o1_source_map_picard_one_step, imex/imex_source_map_step.hpp:300-616
int imex_step(const ecg_run_config& cfg, Grid& gr, double dt, ecg_imex_diag& d)
{
  std::memset(&d, 0, sizeof(d));
  d.solver_status = ECG_SOLVER_NOT_RUN;
  d.linear_solver_status_last = -1;
  const Geo geo(cfg);
  const int nx = gr.nx, ny = gr.ny, n = nx * ny;
  const double gm1 = cfg.gamma - 1.0;
  if (is_bubble(cfg) || cfg.problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122) fill_ghosts(gr, cfg, 0.0);
  else fill_outflow(gr, geo);
  Grid sg(nx, ny);
  imex_star(cfg, gr, dt, sg);
  Host h = imex_host(cfg, nx, ny, geo);
  h.cell.resize(static_cast<std::size_t>(n));
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) h.cell[static_cast<std::size_t>(h.row(i, j))] = sg.cons(i, j);
  const double idx = 1.0 / geo.dx, idy = 1.0 / geo.dy;
  std::vector<double> k(static_cast<std::size_t>(2) * n);
  for (int r = 0; r < n; ++r) { k[2 * r] = h.cell[r].mx; k[2 * r + 1] = h.cell[r].my; }
  for (int r = 0; r < n; ++r)
    if (!std::isfinite(k[2 * r]) || !std::isfinite(k[2 * r + 1])) ++d.kinetic_lag_nonfinite_count;
  std::vector<double> p(static_cast<std::size_t>(n));
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) p[static_cast<std::size_t>(h.row(i, j))] = to_prim(gr.cons(i, j), cfg.gamma).p;
  d.trial_density_min = kInf;
  for (const Cons& c : h.cell) {
    if (!std::isfinite(c.rho) || c.rho <= 1.0e-14) ++d.density_denominator_floor_count;
    if (std::isfinite(c.rho)) d.trial_density_min = std::min(d.trial_density_min, c.rho);
  }
  if (d.density_denominator_floor_count > 0) {
    d.solver_status = ECG_SOLVER_DENSITY_DENOMINATOR_FLOOR_USED;
    d.positivity_failure_count = d.density_denominator_floor_count;
    return d.solver_status;
  }
  // source_map_star_pressure_mismatch_linf, imex_source_map_step.hpp:278-298
  {
    double m = 0.0;
    bool inf = false;
    for (int r = 0; r < n && !inf; ++r) {
      const Cons& s = h.cell[r];
      const double kin = 0.5 * (s.mx * s.mx + s.my * s.my) / s.rho;
      const double pe = gm1 * (s.E - kin);
      if (!std::isfinite(pe) || !std::isfinite(p[r])) { inf = true; break; }
      m = std::max(m, std::abs(p[r] - pe));
    }
    d.pressure_energy_residual_before_linf = inf ? kInf : m;
  }
  Csr A;
  std::vector<double> rhs, ax;
  for (int pic = 0; pic < cfg.imex_picard_iterations; ++pic) {
    int nf = 0;
    build_system(h, p, k, dt, idx, idy, A, rhs, nf);
    d.pressure_matrix_rows = n;
    d.pressure_matrix_nonzeros = static_cast<int>(A.val.size());
    d.pressure_matrix_max_row_width = 0;
    d.kinetic_jacobian_abs_max = 0.0;
    for (int r = 0; r < n; ++r) {
      d.pressure_matrix_max_row_width = std::max(d.pressure_matrix_max_row_width, A.rp[r + 1] - A.rp[r]);
      for (int q = A.rp[r]; q < A.rp[r + 1]; ++q) d.kinetic_jacobian_abs_max = std::max(d.kinetic_jacobian_abs_max, std::abs(A.val[q]));
    }
    // ||A - A^T||max over stored entries of both
    {
      double sym = 0.0;
      auto get = [&](int r, int c) {
        for (int q = A.rp[r]; q < A.rp[r + 1]; ++q) if (A.col[q] == c) return A.val[q];
        return 0.0;
      };
      for (int r = 0; r < n; ++r)
        for (int q = A.rp[r]; q < A.rp[r + 1]; ++q) sym = std::max(sym, std::abs(A.val[q] - get(A.col[q], r)));
      d.pressure_matrix_symmetry_linf = sym;
    }
    if (nf > 0 || !all_finite(rhs)) {
      d.solver_status = ECG_SOLVER_SOURCE_MAP_PRESSURE_ROW_NONFINITE;
      d.kinetic_lag_nonfinite_count = nf;
      d.nonfinite_count = nf;
      return d.solver_status;
    }
    A.mul(p, ax);
    std::vector<double> r0(static_cast<std::size_t>(n));
    for (int q = 0; q < n; ++q) r0[q] = ax[q] - rhs[q];
    d.solver_initial_residual = linf(r0);
    d.solver_initial_rhs_norm = std::max(linf(rhs), 1.0);
    const GmresOut g = gmres(A, rhs, p, cfg.imex_solver_max_iter, cfg.imex_solver_tol);
    d.solver_iterations += g.iterations;
    A.mul(g.x, ax);
    std::vector<double> lr(static_cast<std::size_t>(n));
    for (int q = 0; q < n; ++q) lr[q] = ax[q] - rhs[q];
    d.pressure_linear_residual_linf = linf(lr);
    d.pressure_linear_residual_relative_linf = d.pressure_linear_residual_linf / d.solver_initial_rhs_norm;
    d.solver_residual = d.pressure_linear_residual_linf;
    d.solver_relative_residual = d.pressure_linear_residual_relative_linf;
    const bool abs_ok = d.pressure_linear_residual_linf <= cfg.imex_solver_tol;
    const bool rel_ok = d.pressure_linear_residual_relative_linf <= cfg.imex_solver_tol;
    d.linear_solver_status_last = abs_ok ? ECG_SOLVER_CONVERGED_ABSOLUTE
                                         : (rel_ok ? ECG_SOLVER_CONVERGED_RELATIVE : ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED);
    if (!std::isfinite(d.pressure_linear_residual_linf) || !all_finite(g.x)) {
      d.solver_status = ECG_SOLVER_LINEAR_RESIDUAL_NONFINITE;
      d.nonfinite_count = 1;
      return d.solver_status;
    }
    if (!abs_ok && !rel_ok) {
      d.solver_status = g.breakdown ? ECG_SOLVER_GMRES_BREAKDOWN_NOT_CONVERGED : ECG_SOLVER_LINEAR_SOLVE_NOT_CONVERGED;
      return d.solver_status;
    }
    double dl = 0.0, d2 = 0.0, pmax = 1.0;
    for (int q = 0; q < n; ++q) {
      const double dd = g.x[q] - p[q];
      dl = std::max(dl, std::abs(dd));
      d2 += dd * dd;
      pmax = std::max({pmax, std::abs(p[q]), std::abs(g.x[q])});
      p[q] = g.x[q];
    }
    k = corrected_momentum(h, p, dt, idx, idy);
    d.kinetic_lag_nonfinite_count = 0;
    for (int r = 0; r < n; ++r)
      if (!std::isfinite(k[2 * r]) || !std::isfinite(k[2 * r + 1])) ++d.kinetic_lag_nonfinite_count;
    if (d.kinetic_lag_nonfinite_count > 0) {
      d.solver_status = ECG_SOLVER_SOURCE_MAP_LAGGED_MOMENTUM_NONFINITE;
      d.nonfinite_count = d.kinetic_lag_nonfinite_count;
      return d.solver_status;
    }
    ++d.kinetic_lag_update_count;
    d.pressure_picard_delta_linf = dl;
    d.source_picard_delta_l2_relative_to_pmax = std::sqrt(d2 / static_cast<double>(n)) / pmax;
    ++d.source_picard_iterations_used;
    ++d.picard_pressure_solves_used;
  }
  d.solver_status = d.linear_solver_status_last;

  // evaluate_source_map_final, imex_source_map_step.hpp:75-258
  const std::vector<double> km = corrected_momentum(h, p, dt, idx, idy);
  std::vector<Cons> fin(static_cast<std::size_t>(n));
  double rsum = 0.0, msum = 0.0, esum = 0.0;
  double dmin = kInf, spmin = kInf, spmax = -kInf, epmin = kInf, epmax = -kInf, iemin = kInf, iemax = -kInf;
  double rlinf = 0.0, rrel = 0.0, mlinf = 0.0, mrel = 0.0;
  int rcount = 0, nfc = 0, dfail = 0, pfail = 0, ifail = 0, guard = 0, hnf = 0, fnf = 0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      int cg = 0, chnf = 0, cfnf = 0;
      double cfl = 0.0;
      auto ef = [&](int il, int jl, int ir, int jr, int axis) {
        const Face f = face_detail(h, p, km, il, jl, ir, jr, axis);
        cg += f.guard;
        if (!std::isfinite(f.hl) || !std::isfinite(f.hr) || !std::isfinite(f.h_hat) || !std::isfinite(f.ql) ||
            !std::isfinite(f.qr))
          ++chnf;
        if (f.flux_nonfinite != 0) ++cfnf;
        else cfl = std::max(cfl, std::abs(f.energy_flux));
        return f.energy_flux;
      };
      const double fe = ef(i, j, i + 1, j, 0), fw = ef(i - 1, j, i, j, 0);
      const double fn = ef(i, j, i, j + 1, 1), fs = ef(i, j - 1, i, j, 1);
      guard += cg;
      hnf += chnf;
      fnf += cfnf;
      d.energy_flux_linf = std::max(d.energy_flux_linf, cfl);
      const int r = h.row(i, j);
      const Cons& s = h.at(i, j);
      const double m0 = km[2 * static_cast<std::size_t>(r)], m1 = km[2 * static_cast<std::size_t>(r) + 1];
      const double div = (fe - fw) * idx + (fn - fs) * idy;
      const double en = s.E - dt * div;
      const double kin = 0.5 * (m0 * m0 + m1 * m1) / s.rho;
      const double ie = en - kin;
      const double pe = gm1 * ie;
      const double res = p[r] / gm1 - en + kin;
      const double mis = p[r] - pe;
      const double rs = std::max({std::abs(p[r]) / gm1, std::abs(en), std::abs(kin), 1.0});
      const double ms = std::max({std::abs(p[r]), std::abs(pe), std::abs(kin), 1.0});
      const Cons t{s.rho, m0, m1, en};
      fin[static_cast<std::size_t>(r)] = t;
      const bool nfb = !std::isfinite(t.rho) || !std::isfinite(t.mx) || !std::isfinite(t.my) || !std::isfinite(t.E) ||
                       !std::isfinite(p[r]) || !std::isfinite(kin) || !std::isfinite(ie) || !std::isfinite(pe) ||
                       !std::isfinite(res) || !std::isfinite(div);
      if (nfb) { ++nfc; continue; }
      dmin = std::min(dmin, t.rho);
      spmin = std::min(spmin, p[r]);
      spmax = std::max(spmax, p[r]);
      epmin = std::min(epmin, pe);
      epmax = std::max(epmax, pe);
      iemin = std::min(iemin, ie);
      iemax = std::max(iemax, ie);
      d.momentum_correction_linf = std::max(d.momentum_correction_linf,
                                            std::sqrt((t.mx - s.mx) * (t.mx - s.mx) + (t.my - s.my) * (t.my - s.my)));
      const double ed = std::abs(t.E - s.E);
      d.energy_correction_linf = std::max(d.energy_correction_linf, ed);
      d.energy_closeout_delta_linf = std::max(d.energy_closeout_delta_linf, ed);
      d.energy_flux_divergence_linf = std::max(d.energy_flux_divergence_linf, std::abs(div));
      if (t.rho <= 0.0) ++dfail;
      if (p[r] <= 0.0 || pe <= 0.0) ++pfail;
      if (ie <= 0.0) ++ifail;
      rsum += std::abs(res);
      msum += std::abs(mis);
      esum += ed;
      rlinf = std::max(rlinf, std::abs(res));
      rrel = std::max(rrel, std::abs(res) / rs);
      mlinf = std::max(mlinf, std::abs(mis));
      mrel = std::max(mrel, std::abs(mis) / ms);
      ++rcount;
    }
  int eq78 = 0;
  auto vel = [&](int i, int j, int axis) {
    const Cons& s = fin[static_cast<std::size_t>(h.prow(i, j))];
    const double m = axis == 0 ? s.mx : s.my;
    if (!std::isfinite(s.rho) || s.rho == 0.0 || !std::isfinite(m)) return kNaN;
    return m / s.rho;
  };
  double e78 = 0.0, e78s = 0.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const double ue = vel(i + 1, j, 0), uw = vel(i - 1, j, 0), vn = vel(i, j + 1, 1), vs = vel(i, j - 1, 1);
      const double dv = 0.5 * (ue - uw) * idx + 0.5 * (vn - vs) * idy;
      const double sc = std::max({std::abs(ue), std::abs(uw), std::abs(vn), std::abs(vs), 1.0});
      const double den = sc * std::max(idx, idy);
      if (!std::isfinite(dv) || !std::isfinite(den) || den <= 0.0) continue;
      e78 = std::max(e78, std::abs(dv));
      e78s = std::max(e78s, std::abs(dv) / den);
      ++eq78;
    }
  double rl1 = 0.0, ml1 = 0.0, el1 = 0.0;
  if (nfc > 0 || rcount == 0) {
    rl1 = rlinf = rrel = ml1 = mlinf = mrel = el1 = e78 = e78s = kInf;
  } else if (eq78 == 0) {
    e78 = e78s = kInf;
  } else {
    const double ic = 1.0 / static_cast<double>(rcount);
    rl1 = rsum * ic;
    ml1 = msum * ic;
    el1 = esum * ic;
  }
  auto fon = [](double v) { return std::isfinite(v) ? v : kNaN; };
  d.coupled_residual_l1_final = rl1;
  d.coupled_residual_linf_final = rlinf;
  d.coupled_residual_relative_linf_final = rrel;
  d.pressure_energy_residual_l1 = ml1;
  d.pressure_energy_residual_linf = mlinf;
  d.pressure_energy_residual_relative_linf = mrel;
  d.rho_min = fon(dmin);
  d.pressure_min = fon(epmin);
  d.internal_energy_min = fon(iemin);
  d.trial_density_min = fon(dmin);
  d.solved_pressure_min = fon(spmin);
  d.solved_pressure_max = fon(spmax);
  d.eos_pressure_min = fon(epmin);
  d.eos_pressure_max = fon(epmax);
  d.internal_energy_max = fon(iemax);
  d.nonfinite_count = nfc;
  d.positivity_failure_count = dfail + pfail + ifail;
  d.eq78_divergence_linf = e78;
  d.eq78_divergence_scaled_linf = e78s;
  d.energy_closeout_delta_l1 = el1;
  d.face_enthalpy_denominator_guard_count = guard;
  d.face_enthalpy_nonfinite_count = hnf;
  d.energy_flux_nonfinite_count = fnf;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) gr.set(i, j, fin[static_cast<std::size_t>(h.row(i, j))]);
  return d.solver_status;
}

Grid make_grid(const ecg_run_config* c, const double* u)
{
  Grid g(c->n_cell[0], c->n_cell[1]);
  if (u) g.load(u);
  return g;
}

}  // namespace

extern "C" {

void ecgo_default_run_config(ecg_run_config* c)
{
  std::memset(c, 0, sizeof(*c));
  // RunConfig defaults, core/run_config.hpp:2-55
  c->n_cell[0] = 64; c->n_cell[1] = 64;
  c->is_periodic[0] = 1; c->is_periodic[1] = 1;
  c->prob_lo[0] = 0.0; c->prob_lo[1] = 0.0;
  c->prob_hi[0] = 1.0; c->prob_hi[1] = 1.0;
  c->max_step = 8;
  c->spatial_order = 1;
  c->toro_test = 1;
  c->problem = ECG_PROBLEM_ADVECTION_BLOB;
  c->riemann = ECG_RIEMANN_HLLC;
  c->method = ECG_METHOD_EXPLICIT;
  c->slope_limiter = ECG_LIMITER_MINMOD;
  c->field_boundary = ECG_FIELD_BOUNDARY_OUTFLOW;
  c->stop_time = 0.05;
  c->gamma = 1.4;
  c->cfl = 0.4;
  c->imex_cfl = 0.8;
  c->imex_acoustic_cfl_cap = 0.0;
  c->imex_solver_tol = 1.0e-10;
  c->velocity_x = 1.0; c->velocity_y = 0.5;
  c->density_inner = 2.0; c->density_outer = 1.0;
  c->pressure = 1.0;
  c->mach = 0.1;
  c->blob_cx = 0.35; c->blob_cy = 0.35; c->blob_radius = 0.15;
  c->vortex_cx = 0.0; c->vortex_cy = 0.0;
  c->isentropic_vortex_strength = 5.0;
  c->riemann_interface_x = 0.5; c->riemann_interface_y = 0.5;
  c->imex_solver_max_iter = 100;
  c->imex_acoustic_startup = 1;
  c->imex_picard_extra_iterations = 1;
  c->imex_picard_iterations = 2;
}

int ecgo_initialize_state(const ecg_run_config* c, double* u)
{
  Grid g = make_grid(c, nullptr);
  initialize(*c, g);
  g.store(u);
  return 0;
}

void ecgo_fill_problem_ghosts(const ecg_run_config* c, const double* u, double time, double* ghosted)
{
  Grid g = make_grid(c, u);
  fill_ghosts(g, *c, time);
  std::memcpy(ghosted, g.a.data(), g.a.size() * sizeof(double));
}

int ecgo_euler_fv_one_step(const ecg_run_config* c, double* u, double dt, double time)
{
  Grid g = make_grid(c, u);
  const int n = fv_one_step(*c, g, dt, time);
  g.store(u);
  return n;
}

double ecgo_compute_euler_dt(const ecg_run_config* c, const double* u, double time)
{
  const Grid g = make_grid(c, u);
  return euler_dt(*c, g, time);
}

double ecgo_compute_imex_dt(const ecg_run_config* c, const double* u, double time, ecg_imex_timestep_diag* d)
{
  const Grid g = make_grid(c, u);
  return imex_dt(*c, g, time, d);
}

void ecgo_compute_diagnostics(const ecg_run_config* c, const double* u, ecg_diagnostics* out)
{
  const Grid g = make_grid(c, u);
  *out = diagnostics(*c, g);
}

void ecgo_compute_admissibility(const ecg_run_config* c, const double* u, ecg_admissibility* out)
{
  const Grid g = make_grid(c, u);
  *out = admissibility(*c, g);
}

int ecgo_imex_step(const ecg_run_config* c, double* u, double dt, ecg_imex_diag* out)
{
  Grid g = make_grid(c, u);
  Grid keep = g;
  const int s = imex_step(*c, g, dt, *out);
  const bool ok = s == ECG_SOLVER_CONVERGED_ABSOLUTE || s == ECG_SOLVER_CONVERGED_RELATIVE;
  (ok ? g : keep).store(u);
  return s;
}

// solve_host_sparse_gmres restated (see gmres above) on a caller CSR.
int ecgo_gmres_csr(int n, const int* rp, const int* col, const double* val, const double* b, const double* x0,
                   int max_iter, double tol, double* x, int* iterations, int* converged, int* breakdown,
                   int* nonfinite, double* res_linf, double* rel_linf)
{
  Csr A;
  A.n = n;
  A.rp.assign(rp, rp + n + 1);
  A.col.assign(col, col + rp[n]);
  A.val.assign(val, val + rp[n]);
  const GmresOut g = gmres(A, std::vector<double>(b, b + n), std::vector<double>(x0, x0 + n), max_iter, tol);
  std::copy(g.x.begin(), g.x.end(), x);
  *iterations = g.iterations;
  *converged = g.converged;
  *breakdown = g.breakdown;
  *nonfinite = g.nonfinite;
  *res_linf = g.res_linf;
  *rel_linf = g.rel_linf;
  return 0;
}

// The explicit driver loop, app/driver_main.hpp:216-340 (no output).
int ecgo_run_explicit(const ecg_run_config* c, double* u, int max_step, double stop_time, ecg_run_result* out)
{
  ecg_run_config cfg = *c;
  cfg.stop_time = stop_time;
  Grid g = make_grid(c, u);
  std::memset(out, 0, sizeof(*out));
  out->dt_min = kInf;
  double t = 0.0;
  int step = 0;
  ecg_diagnostics d = diagnostics(cfg, g);
  if (d.nonfinite_count > 0 || d.rho_min <= 0.0 || d.pressure_min <= 0.0) { out->failed = 1; }
  while (!out->failed && step < max_step && t < stop_time - 1.0e-14) {
    const double dt = euler_dt(cfg, g, t);
    if (!std::isfinite(dt) || dt <= 0.0) { out->failed = 1; out->failure_code = ECG_FAILURE_INVALID_TIME_STEP; break; }
    out->hllc_degenerate_star_count += fv_one_step(cfg, g, dt, t);
    out->dt_min = std::min(out->dt_min, dt);
    out->dt_max = std::max(out->dt_max, dt);
    out->dt_sum += dt;
    t += dt;
    ++step;
    d = diagnostics(cfg, g);
    if (d.nonfinite_count > 0) { out->failed = 1; out->failure_code = ECG_FAILURE_NONFINITE_STATE; }
    else if (d.rho_min <= 0.0) { out->failed = 1; out->failure_code = ECG_FAILURE_NONPOSITIVE_DENSITY; }
    else if (d.pressure_min <= 0.0) { out->failed = 1; out->failure_code = ECG_FAILURE_NONPOSITIVE_PRESSURE; }
  }
  out->steps = step;
  out->time = t;
  out->diagnostics = d;
  g.store(u);
  return out->failed;
}

// source_map_build_pressure_system on a star state, Picard pressure p and
// lagged momentum k (2 planes); CSR + rhs as the reference assembles them.
int ecgo_imex_build_system(const ecg_run_config* c, const double* star, const double* p, const double* k, double dt,
                           int* rp, int* col, double* val, double* rhs, int cap, int* nonfinite)
{
  const Geo geo(*c);
  const int nx = c->n_cell[0], ny = c->n_cell[1], n = nx * ny;
  Host h = imex_host(*c, nx, ny, geo);
  h.cell.resize(static_cast<std::size_t>(n));
  for (int r = 0; r < n; ++r) h.cell[r] = Cons{star[r], star[n + r], star[2 * n + r], star[3 * n + r]};
  std::vector<double> pv(p, p + n), kv(static_cast<std::size_t>(2) * n);
  for (int r = 0; r < n; ++r) { kv[2 * r] = k[r]; kv[2 * r + 1] = k[n + r]; }
  Csr A;
  std::vector<double> b;
  int nf = 0;
  build_system(h, pv, kv, dt, 1.0 / geo.dx, 1.0 / geo.dy, A, b, nf);
  if (nonfinite) *nonfinite = nf;
  if (static_cast<int>(A.val.size()) > cap) return -1;
  std::copy(A.rp.begin(), A.rp.end(), rp);
  std::copy(A.col.begin(), A.col.end(), col);
  std::copy(A.val.begin(), A.val.end(), val);
  std::copy(b.begin(), b.end(), rhs);
  return static_cast<int>(A.val.size());
}

// compute_bdltv20_pressure_split_star with the IMEX step's ghost policy.
void ecgo_imex_star(const ecg_run_config* c, const double* u, double dt, double* star)
{
  Grid g = make_grid(c, u);
  const Geo geo(*c);
  if (is_bubble(*c) || c->problem == ECG_PROBLEM_SHOCK_BUBBLE_MACH122) fill_ghosts(g, *c, 0.0);
  else fill_outflow(g, geo);
  Grid s(c->n_cell[0], c->n_cell[1]);
  imex_star(*c, g, dt, s);
  s.store(star);
}

// source_map_eq54_corrected_momentum_field (physical-boundary pressure).
void ecgo_corrected_momentum(const ecg_run_config* c, const double* star, const double* p, double dt, double* k)
{
  const Geo geo(*c);
  const int nx = c->n_cell[0], ny = c->n_cell[1], n = nx * ny;
  Host h = imex_host(*c, nx, ny, geo);
  h.cell.resize(static_cast<std::size_t>(n));
  for (int r = 0; r < n; ++r) h.cell[r] = Cons{star[r], star[n + r], star[2 * n + r], star[3 * n + r]};
  const std::vector<double> km = corrected_momentum(h, std::vector<double>(p, p + n), dt, 1.0 / geo.dx, 1.0 / geo.dy);
  for (int r = 0; r < n; ++r) { k[r] = km[2 * r]; k[n + r] = km[2 * r + 1]; }
}

void ecgo_exact_riemann_sample(double x, double t, const double* l, const double* r, double g, double x0, double* out)
{
  const Prim q = riemann_sample(x, t, Prim{l[0], l[1], l[2], l[3]}, Prim{r[0], r[1], r[2], r[3]}, g, x0);
  out[0] = q.rho; out[1] = q.u; out[2] = q.v; out[3] = q.p;
}

void ecgo_gresho_state(const ecg_run_config* c, double x, double y, double* out)
{
  const Prim q = gresho(x, y, *c);
  out[0] = q.rho; out[1] = q.u; out[2] = q.v; out[3] = q.p;
}

// compute_gresho_metrics density_l1_error, diagnostic_metrics_timestep.hpp:150-225
double ecgo_gresho_density_l1(const ecg_run_config* c, const double* u)
{
  const Grid g = make_grid(c, u);
  const Geo geo(*c);
  double s = 0.0;
  for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
      const Prim q = to_prim(g.cons(i, j), c->gamma);
      s += std::abs(q.rho - gresho(geo.xc(i), geo.yc(j), *c).rho);
    }
  return s * (1.0 / static_cast<double>(c->n_cell[0] * c->n_cell[1]));
}

}  // extern "C"
