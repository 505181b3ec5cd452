// Default explicit step of the fast build: warps march up column strips.
// Included inside the ecg_fast namespace of stencil.cuh, after fv_fast.cuh
// (it uses that file's Newton-refined arithmetic and flux functions).
//
// A warp owns the 28 cells [c0, c0+28) of a row strip; lane l holds column
// c0 - 2 + l (lanes 0-1 and 30-31 carry the MUSCL halo).  It walks rows
// j0 .. j0+H-1 keeping, per lane, the primitives of rows j-1 .. j+2 in
// registers:
//   * x-neighbours for the x-slopes and x-face states come by warp shuffles;
//   * the y-slope of a row is computed once and reused by both y-faces;
//   * the y-face flux above row j becomes the flux below row j+1 without
//     leaving registers.
// Every face flux is evaluated once per warp strip (the x-face at a strip
// edge by both strips), with no shared memory and no block barrier in the
// loop.  Reductions (CFL rate, admissibility, degenerate count) accumulate in
// registers and are committed once per block.
namespace march {

constexpr int kLanes = 32;
constexpr int kCells = 28;  // interior cells per warp strip

struct Lane {
  Prim q[4];  // rows j-1, j, j+1, j+2 of this lane's column
};

__device__ __forceinline__ double shup(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shdn(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }

template <int LIM>
__device__ __forceinline__ Prim slope3(const Prim& m, const Prim& c, const Prim& p, bool second)
{
  if (!second) return Prim{0.0, 0.0, 0.0, 0.0};
  return Prim{limited_slope(c.rho - m.rho, p.rho - c.rho, LIM), limited_slope(c.u - m.u, p.u - c.u, LIM),
              limited_slope(c.v - m.v, p.v - c.v, LIM), limited_slope(c.p - m.p, p.p - c.p, LIM)};
}

__device__ __forceinline__ Prim plus_half(const Prim& q, const Prim& s)
{
  return Prim{fma(0.5, s.rho, q.rho), fma(0.5, s.u, q.u), fma(0.5, s.v, q.v), fma(0.5, s.p, q.p)};
}
__device__ __forceinline__ Prim minus_half(const Prim& q, const Prim& s)
{
  return Prim{fma(-0.5, s.rho, q.rho), fma(-0.5, s.u, q.u), fma(-0.5, s.v, q.v), fma(-0.5, s.p, q.p)};
}

// The x-face and the y-face of a row, evaluated back to back on the fast
// path (independent instruction streams the scheduler can interleave); faces
// that need the reference path (degenerate HLLC star state, sound speed off
// the rsqrt path) are recomputed after one warp vote.  deg_*: HLLC fell back
// to Rusanov on that face.  Returns whether the vote fired (the same on every
// lane): deg_* can only be set then.
template <int RK>
__device__ __forceinline__ bool face_pair(Prim xl, Prim xr, Prim yl, Prim yr, double g, double inv_gm1, Cons& fx,
                                          Cons& fy, bool& deg_x, bool& deg_y)
{
  if (RK == ECG_RIEMANN_LOWMACH_HLLC) {
    fast::lowmach_f(xl, xr, g);
    fast::lowmach_f(yl, yr, g);
  }
  bool bx, by;
  if (RK == ECG_RIEMANN_RUSANOV) {
    fx = fast::rusanov_core(xl, xr, 0, g, inv_gm1, bx);
    fy = fast::rusanov_core(yl, yr, 1, g, inv_gm1, by);
  } else {
    fx = fast::hllc_core(xl, xr, 0, g, inv_gm1, bx);
    fy = fast::hllc_core(yl, yr, 1, g, inv_gm1, by);
  }
  deg_x = deg_y = false;
  if (__any_sync(0xffffffffu, bx || by)) {
    if (RK == ECG_RIEMANN_RUSANOV) {
      if (bx) fx = fast::rusanov_f(xl, xr, 0, g, inv_gm1);
      if (by) fy = fast::rusanov_f(yl, yr, 1, g, inv_gm1);
    } else {
      if (bx) fx = fast::hllc_f(xl, xr, 0, g, inv_gm1, deg_x);
      if (by) fy = fast::hllc_f(yl, yr, 1, g, inv_gm1, deg_y);
    }
    return true;
  }
  return false;
}

// One face with the warp-voting flux (faces evaluated one after the other).
template <int RK>
__device__ __forceinline__ Cons face_w(Prim l, Prim r, int axis, double g, double inv_gm1, bool& deg)
{
  deg = false;
  if (RK == ECG_RIEMANN_RUSANOV) return fast::rusanov_i(l, r, axis, g, inv_gm1);
  if (RK == ECG_RIEMANN_LOWMACH_HLLC) fast::lowmach_f(l, r, g);
  return fast::hllc_w(l, r, axis, g, inv_gm1, deg);
}

// One face on its own (the y-face below the first row of a strip).
template <int RK>
__device__ __forceinline__ Cons face_one(Prim l, Prim r, int axis, double g, double inv_gm1, bool& deg)
{
  deg = false;
  if (RK == ECG_RIEMANN_RUSANOV) return fast::rusanov_f(l, r, axis, g, inv_gm1);
  if (RK == ECG_RIEMANN_LOWMACH_HLLC) fast::lowmach_f(l, r, g);
  return fast::hllc_f(l, r, axis, g, inv_gm1, deg);
}

// Reductions of one warp strip over the new state.
struct MarchAcc {
  unsigned long long kmax, krho, kp;
  int nonfinite, degenerate;
  __device__ __forceinline__ void init()
  {
    kmax = okey(kLowest);
    krho = okey(kMax);
    kp = okey(kMax);
    nonfinite = degenerate = 0;
  }
};

// Advances the strip of 28 cells starting at column c0 over rows
// [j0, min(j0 + H, ny)) from u into out.  Called by all 32 lanes of a warp
// (the flux helpers vote across the warp).
template <int RK, int LIM, bool PAIR>
__device__ __forceinline__ void march_strip(const EcgFvParams& P, const double* __restrict__ u,
                                            double* __restrict__ out, int c0, int j0, int H, double dt,
                                            bool count_deg, MarchAcc& acc)
{
  const int lane = threadIdx.x & 31;
  const int x = c0 - 2 + lane;
  const int nx = P.g.nx, ny = P.g.ny;
  const double g = P.gamma, inv_gm1 = fast::frcp(g - 1.0);
  const double idx = P.g.inv_dx, idy = P.g.inv_dy;
  const bool second = P.order > 1;
  const bool inner = lane >= 2 && lane < 2 + kCells;   // owns a cell of the strip
  const bool cell_ok = inner && x < nx;                 // that cell is in the domain
  const bool xface = lane >= 2 && lane <= 2 + kCells;   // its x-face on the left belongs to the strip
  const int xs = x < 0 ? 0 : (x < nx ? x : nx - 1);     // in-bounds column for the old-state reload
  const int rhi = P.row_hi > 0 && P.row_hi < ny ? P.row_hi : ny;  // end of the band of rows being updated
  const int jend = j0 + H < rhi ? j0 + H : rhi;

  // ---- prologue: rows j0-2 .. j0+1, y-slopes of rows j0-1 and j0, the y-face below row j0 ----
  Prim q_m2 = fast::to_prim_f(load_cell(P, u, x, j0 - 2), g);
  Lane L;
  L.q[1] = fast::to_prim_f(load_cell(P, u, x, j0 - 1), g);
  L.q[2] = fast::to_prim_f(load_cell(P, u, x, j0), g);
  L.q[3] = fast::to_prim_f(load_cell(P, u, x, j0 + 1), g);
  const Prim sy_m1 = slope3<LIM>(q_m2, L.q[1], L.q[2], second);
  Prim sy_cur = slope3<LIM>(L.q[1], L.q[2], L.q[3], second);
  Cons gb;
  {
    bool deg;
    gb = face_one<RK>(plus_half(L.q[1], sy_m1), minus_half(L.q[2], sy_cur), 1, g, inv_gm1, deg);
    if (count_deg && deg && cell_ok && j0 < ny) acc.degenerate += 1;
  }
  for (int j = j0; j < jend; ++j) {
    // window rows j-1 .. j+2
    L.q[0] = L.q[1];
    L.q[1] = L.q[2];
    L.q[2] = L.q[3];
    L.q[3] = fast::to_prim_f(load_cell(P, u, x, j + 2), g);
    const Prim& qc = L.q[1];
    // slopes: y of row j+1 (for the y-face above row j), x of this lane's cell
    const Prim sy_next = slope3<LIM>(L.q[1], L.q[2], L.q[3], second);
    const Prim ql{shup(qc.rho), shup(qc.u), shup(qc.v), shup(qc.p)};
    const Prim qr{shdn(qc.rho), shdn(qc.u), shdn(qc.v), shdn(qc.p)};
    const Prim sx = slope3<LIM>(ql, qc, qr, second);
    const Prim sxl{shup(sx.rho), shup(sx.u), shup(sx.v), shup(sx.p)};
    // the x-face on this lane's left and the y-face above row j; every lane
    // evaluates both (lanes 0, 1 and 31 cost nothing extra in lockstep), only
    // lanes 2..30 use or count their x-face
    Cons fl, gt;
    bool deg_x, deg_y, voted = true;
    if (PAIR) {
      voted = face_pair<RK>(plus_half(ql, sxl), minus_half(qc, sx), plus_half(qc, sy_cur), minus_half(L.q[2], sy_next),
                            g, inv_gm1, fl, gt, deg_x, deg_y);
    } else {
      gt = face_w<RK>(plus_half(qc, sy_cur), minus_half(L.q[2], sy_next), 1, g, inv_gm1, deg_y);
      fl = face_w<RK>(plus_half(ql, sxl), minus_half(qc, sx), 0, g, inv_gm1, deg_x);
    }
    const Cons fr{shdn(fl.rho), shdn(fl.mx), shdn(fl.my), shdn(fl.E)};
    if (count_deg && voted) {
      // each face counts once per adjacent cell of this strip in the domain
      // (count_hllc_degenerate_star_states, explicit_update.hpp:2-56)
      const bool left_ok = lane >= 3 && lane <= 2 + kCells && x - 1 < nx;
      if (deg_x && xface) acc.degenerate += (left_ok ? 1 : 0) + (cell_ok ? 1 : 0);
      if (deg_y && cell_ok) acc.degenerate += 1 + (j + 1 < jend ? 1 : 0);
    }
    // update (explicit_update.hpp:92-95) and the reductions of the new state;
    // all lanes compute, lanes outside the strip or the domain neither store
    // nor reduce
    const long long o = static_cast<long long>(j) * P.g.pitch + xs;
    const long long pl = P.g.plane;
    Cons n;
    n.rho = __ldg(u + o) - dt * ((fr.rho - fl.rho) * idx + (gt.rho - gb.rho) * idy);
    n.mx = __ldg(u + o + pl) - dt * ((fr.mx - fl.mx) * idx + (gt.mx - gb.mx) * idy);
    n.my = __ldg(u + o + 2 * pl) - dt * ((fr.my - fl.my) * idx + (gt.my - gb.my) * idy);
    n.E = __ldg(u + o + 3 * pl) - dt * ((fr.E - fl.E) * idx + (gt.E - gb.E) * idy);
    const Prim q = fast::to_prim_f(n, g);
    const double cs = fast::fsound_w(q.rho, q.p, g);
    if (cell_ok) {
      out[o] = n.rho;
      out[o + pl] = n.mx;
      out[o + 2 * pl] = n.my;
      out[o + 3 * pl] = n.E;
      const double rate = (fabs(q.u) + cs) * idx + (fabs(q.v) + cs) * idy;
      if (!isnan(rate)) acc.kmax = umax64(acc.kmax, okey(rate));
      const bool bad = !isfinite(q.rho) || !isfinite(q.u) || !isfinite(q.v) || !isfinite(q.p) || !isfinite(n.E);
      acc.krho = umin64(acc.krho, okey(bad ? -kInf : q.rho));
      acc.kp = umin64(acc.kp, okey(bad ? -kInf : q.p));
      acc.nonfinite += bad ? 1 : 0;
    }
    gb = gt;
    sy_cur = sy_next;
  }
}

// ---- the staged march: rows reach the warp through shared memory --------
//
// Each warp keeps the conserved values of the rows it is about to use in a
// ring of kRing rows in shared memory (slot = row mod kRing, component planes
// of 32 lanes).  A lane requests the cell of its column kAhead rows ahead of
// the one being converted with cp.async (8 bytes per component, straight
// from the state, the exact-Dirichlet ring or a slab halo, whichever the
// ghost policy names); constant ghost states are stored directly.  The load
// latency of a row is thus hidden behind kAhead rows of flux work without
// holding registers, and the old state of the updated row is read back from
// the ring instead of from global memory.  Each lane only reads the slots it
// wrote itself, so cp.async.wait_group is the only synchronisation.
constexpr int kRing = 8;
constexpr int kAhead = 4;
static_assert(kAhead + 4 <= kRing, "the prologue stages rows j0-2 .. j0+1+kAhead");

struct StageRing {
  double v[kRing][4][kLanes];
};

__device__ __forceinline__ void cp_async8(unsigned dst, const double* src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The multiface sensor's pressure ratio (xie_pressure_ratio_from_states,
// reconstruction_fluxes.hpp:390-397) of the x-face on this lane's left in a
// row of which this lane holds the pressure pc: the face pressures of the
// MUSCL states, as the tile kernel forms them.
template <int LIM>
__device__ __forceinline__ double xface_ratio(double pc, bool second)
{
  const double pl = shup(pc), pr = shdn(pc);
  const double s = second ? limited_slope(pc - pl, pr - pc, LIM) : 0.0;
  return fast::pratio_f(fma(0.5, shup(s), pl), fma(-0.5, s, pc));
}

// xie_am_hllc_p flux of one face with sensor h^3 (reconstruction_fluxes.hpp:
// 254-371, 390-440): the branch-free core, repaired by xie_f on the faces a
// warp vote sends back.  deg: the HLLC degeneracy test of the face.
__device__ __forceinline__ Cons face_xie(const Prim& l, const Prim& r, int axis, double g, double inv_gm1, double h,
                                         bool& deg)
{
  const double sensor = h * h * h;
  bool fb;
  Cons f = fast::xie_core(l, r, axis, g, inv_gm1, sensor, fb, deg);
  if (__any_sync(0xffffffffu, fb)) {
    if (fb) f = fast::xie_f(l, r, axis, g, inv_gm1, sensor, deg);
  }
  return f;
}

// RK = xie_am_hllc_p: the faces one at a time, each with its 5-face sensor.
// The pressure ratios it needs come along the march: the y-faces' below and
// above row j (carried, and this row's), and the x-faces' of rows j and j+1
// (row j+1's from the pressure of the window's next row, carried on).
template <int RK, int LIM, bool PAIR>
__device__ __forceinline__ void march_strip_staged(const EcgFvParams& P, const double* __restrict__ u,
                                                   double* __restrict__ out, int c0, int j0, int H, double dt,
                                                   bool count_deg, MarchAcc& acc, StageRing& ring)
{
  const int lane = threadIdx.x & 31;
  const int x = c0 - 2 + lane;
  const int nx = P.g.nx, ny = P.g.ny;
  const double g = P.gamma, inv_gm1 = fast::frcp(g - 1.0);
  const double idx = P.g.inv_dx, idy = P.g.inv_dy;
  const bool second = P.order > 1;
  const bool inner = lane >= 2 && lane < 2 + kCells;
  const bool cell_ok = inner && x < nx;
  const bool xface = lane >= 2 && lane <= 2 + kCells;
  const int xs = x < 0 ? 0 : (x < nx ? x : nx - 1);
  const int rhi = P.row_hi > 0 && P.row_hi < ny ? P.row_hi : ny;
  const int jend = j0 + H < rhi ? j0 + H : rhi;
  const int jlast = jend + 1;  // the last row the strip reads

  double* const col = &ring.v[0][0][lane];
  const unsigned col_s = static_cast<unsigned>(__cvta_generic_to_shared(col));
  unsigned flips = 0;  // bit (row mod kRing): that staged row is a mirror image (my to negate)
  // Strips whose 32 columns all lie in the domain take in-domain rows
  // straight from the state, at a pointer that moves one row a request (the
  // rows are requested in order); the ghost policy decides the rest.
  const bool xin = c0 >= 2 && c0 + kLanes - 2 <= nx;
  const long long pitch = P.g.pitch, pl = P.g.plane;
  const double* rowp = u + static_cast<long long>(j0 - 2) * pitch + x;  // dereferenced only when in the domain
  // request row jr of this lane's column (an empty group past the strip's rows)
  auto put = [&](int jr) {
    if (jr <= jlast) {
      const int sl = jr & (kRing - 1);
      const CellSrc c = xin && static_cast<unsigned>(jr) < static_cast<unsigned>(ny) ? CellSrc{rowp, pl, false}
                                                                                     : cell_src(P, u, x, jr);
      flips = c.flip ? (flips | (1u << sl)) : (flips & ~(1u << sl));
      if (c.p) {
        const unsigned d = col_s + static_cast<unsigned>(sl * 4 * kLanes * 8);
        cp_async8(d, c.p);
        cp_async8(d + kLanes * 8, c.p + c.pl);
        cp_async8(d + 2 * kLanes * 8, c.p + 2 * c.pl);
        cp_async8(d + 3 * kLanes * 8, c.p + 3 * c.pl);
      } else {
        double* d = col + sl * 4 * kLanes;
        d[0] = P.bc.cst[0];
        d[kLanes] = P.bc.cst[1];
        d[2 * kLanes] = P.bc.cst[2];
        d[3 * kLanes] = P.bc.cst[3];
      }
    }
    rowp += pitch;
    cp_async_commit();
  };
  auto get = [&](int jr) {
    const int sl = jr & (kRing - 1);
    const double* d = col + sl * 4 * kLanes;
    Cons c{d[0], d[kLanes], d[2 * kLanes], d[3 * kLanes]};
    if ((flips >> sl) & 1u) c.my = -c.my;
    return c;
  };

  // ---- prologue: stage rows j0-2 .. j0+1+kAhead; rows j0-2 .. j0+1 first ----
#pragma unroll
  for (int r = -2; r <= 1 + kAhead; ++r) put(j0 + r);
  cp_async_wait<kAhead>();
  Prim qa, qb, qc;  // rows j, j+1 and the slot of row j+2, by role
  Prim s0, s1;      // y-slope of row j, and the slot of row j+1's
  Cons g0, g1;      // y-face below row j, and the slot of the face above it
  constexpr bool XIE = RK == ECG_RIEMANN_XIE_AM_HLLC_P;
  double yr_prev = 0.0, xr_cur = 0.0;  // XIE: pressure ratios of the y-face below row j, the x-face left of row j
  {
    const Prim q_m2 = fast::to_prim_f(get(j0 - 2), g);
    const Prim q_m1 = fast::to_prim_f(get(j0 - 1), g);
    qa = fast::to_prim_f(get(j0), g);
    qb = fast::to_prim_f(get(j0 + 1), g);
    const Prim sy_m1 = slope3<LIM>(q_m2, q_m1, qa, second);
    s0 = slope3<LIM>(q_m1, qa, qb, second);
    bool deg;
    if constexpr (XIE) {
      const Prim yl = plus_half(q_m1, sy_m1), yr = minus_half(qa, s0);
      yr_prev = fast::pratio_f(yl.p, yr.p);
      const double xm1 = xface_ratio<LIM>(q_m1.p, second);
      xr_cur = xface_ratio<LIM>(qa.p, second);
      double m = yr_prev;
      m = smin(m, xm1);
      m = smin(m, shdn(xm1));
      m = smin(m, xr_cur);
      m = smin(m, shdn(xr_cur));
      g0 = face_xie(yl, yr, 1, g, inv_gm1, clamp01(m), deg);
    } else {
      g0 = face_one<RK>(plus_half(q_m1, sy_m1), minus_half(qa, s0), 1, g, inv_gm1, deg);
    }
    if (count_deg && deg && cell_ok && j0 < ny) acc.degenerate += 1;
  }
  double* const obase = out + xs;
  double rate_max = kLowest, rho_min = kMax, p_min = kMax;

  // one row: row j's cells from rows j (q0), j+1 (q1) and the new row j+2
  // (into q2), the y-slope of row j (sc; that of row j+1 into sn) and the
  // y-face below row j (gb; the face above it into gt)
  auto row = [&](int j, const Prim& q0, const Prim& q1, Prim& q2, const Prim& sc, Prim& sn, const Cons& gb, Cons& gt) {
    put(j + 2 + kAhead);
    cp_async_wait<kAhead>();  // row j + 2 has landed
    q2 = fast::to_prim_f(get(j + 2), g);
    sn = slope3<LIM>(q0, q1, q2, second);
    const Prim ql{shup(q0.rho), shup(q0.u), shup(q0.v), shup(q0.p)};
    const Prim qr{shdn(q0.rho), shdn(q0.u), shdn(q0.v), shdn(q0.p)};
    const Prim sx = slope3<LIM>(ql, q0, qr, second);
    const Prim sxl{shup(sx.rho), shup(sx.u), shup(sx.v), shup(sx.p)};
    Cons fl;
    bool deg_x, deg_y, voted = true;
    if constexpr (XIE) {
      // sensors: the x-face on the left, from its own ratio and the y-faces'
      // below and above cells i-1 and i; the y-face above, from its own ratio
      // and the x-faces' left and right of cell i in rows j and j+1
      const Prim xl = plus_half(ql, sxl), xrs = minus_half(q0, sx);
      const Prim yl = plus_half(q0, sc), yrs = minus_half(q1, sn);
      const double yr_cur = fast::pratio_f(yl.p, yrs.p);
      const double xr_next = xface_ratio<LIM>(q1.p, second);
      double my = yr_cur;
      my = smin(my, xr_cur);
      my = smin(my, shdn(xr_cur));
      my = smin(my, xr_next);
      my = smin(my, shdn(xr_next));
      double mx = xr_cur;
      mx = smin(mx, shup(yr_prev));
      mx = smin(mx, shup(yr_cur));
      mx = smin(mx, yr_prev);
      mx = smin(mx, yr_cur);
      gt = face_xie(yl, yrs, 1, g, inv_gm1, clamp01(my), deg_y);
      fl = face_xie(xl, xrs, 0, g, inv_gm1, clamp01(mx), deg_x);
      yr_prev = yr_cur;
      xr_cur = xr_next;
    } else if (PAIR) {
      voted = face_pair<RK>(plus_half(ql, sxl), minus_half(q0, sx), plus_half(q0, sc), minus_half(q1, sn), g, inv_gm1,
                            fl, gt, deg_x, deg_y);
    } else {
      gt = face_w<RK>(plus_half(q0, sc), minus_half(q1, sn), 1, g, inv_gm1, deg_y);
      fl = face_w<RK>(plus_half(ql, sxl), minus_half(q0, sx), 0, g, inv_gm1, deg_x);
    }
    const Cons fr{shdn(fl.rho), shdn(fl.mx), shdn(fl.my), shdn(fl.E)};
    if (count_deg && voted) {
      // each face counts once per adjacent cell of this strip in the domain
      // (count_hllc_degenerate_star_states, explicit_update.hpp:2-56); a
      // face is degenerate only where the warp's fallback vote fired
      const bool left_ok = lane >= 3 && lane <= 2 + kCells && x - 1 < nx;
      if (deg_x && xface) acc.degenerate += (left_ok ? 1 : 0) + (cell_ok ? 1 : 0);
      if (deg_y && cell_ok) acc.degenerate += 1 + (j + 1 < jend ? 1 : 0);
    }
    // update (explicit_update.hpp:92-95) from the staged old state of row j
    const Cons old = get(j);
    Cons n;
    n.rho = old.rho - dt * ((fr.rho - fl.rho) * idx + (gt.rho - gb.rho) * idy);
    n.mx = old.mx - dt * ((fr.mx - fl.mx) * idx + (gt.mx - gb.mx) * idy);
    n.my = old.my - dt * ((fr.my - fl.my) * idx + (gt.my - gb.my) * idy);
    n.E = old.E - dt * ((fr.E - fl.E) * idx + (gt.E - gb.E) * idy);
    const Prim q = fast::to_prim_f(n, g);
    const double cs = fast::fsound_w(q.rho, q.p, g);
    if (cell_ok) {
      double* o = obase + static_cast<long long>(j) * P.g.pitch;
      o[0] = n.rho;
      o[pl] = n.mx;
      o[2 * pl] = n.my;
      o[3 * pl] = n.E;
      // running extrema as doubles (max/min skip a NaN operand, as the keys'
      // NaN test does), turned into ordered keys once, after the strip
      const double rate = (fabs(q.u) + cs) * idx + (fabs(q.v) + cs) * idy;
      rate_max = fmax(rate_max, rate);
      const bool bad = !isfinite(q.rho) || !isfinite(q.u) || !isfinite(q.v) || !isfinite(q.p) || !isfinite(n.E);
      rho_min = fmin(rho_min, bad ? -kInf : q.rho);
      p_min = fmin(p_min, bad ? -kInf : q.p);
      acc.nonfinite += bad ? 1 : 0;
    }
  };

  // (Six rows a trip, which hands the roles round by name with no register
  // moves, measured 112.7 us against 75.8 us: the larger loop body costs
  // more than the moves it saves.)
  for (int j = j0; j < jend; ++j) {
    row(j, qa, qb, qc, s0, s1, g0, g1);
    qa = qb;
    qb = qc;
    s0 = s1;
    g0 = g1;
  }
  cp_async_wait<0>();  // no request outlives the strip
  acc.kmax = umax64(acc.kmax, okey(rate_max));
  acc.krho = umin64(acc.krho, okey(rho_min));
  acc.kp = umin64(acc.kp, okey(p_min));
}

// Registers: the register-loaded strips at most 128 a thread (4 blocks of 4
// warps per SM), measured faster than the 166-register schedule the paired
// faces get unbounded; the staged strips at most 168 (3 blocks), measured
// faster than 128 for them (fewer registers spill).
// STAGE: rows through the shared-memory ring (march_strip_staged), else
// straight from global memory into registers (march_strip).
template <int RK, int LIM, int WPB, bool PAIR, bool STAGE>
__global__ void __launch_bounds__(WPB * 32, (STAGE ? 12 : 16) / WPB)
fv_march_kernel(const EcgFvParams P, const double* __restrict__ u, double* __restrict__ out,
                EcgStepStats* __restrict__ stats, const EcgDtCtl ctl, const int H)
{
  __shared__ BlockRed<WPB * 32> red;
  __shared__ StageRing ring[STAGE ? WPB : 1];
  const int strip = blockIdx.x * WPB + (threadIdx.x >> 5);
  const int c0 = strip * kCells;
  const int j0 = (P.row_hi > 0 ? P.row_lo : 0) + blockIdx.y * H;

  double dt;
  if (!step_control(stats, ctl, dt)) return;

  MarchAcc acc;
  acc.init();
  if (c0 < P.g.nx) {
    if constexpr (STAGE)
      march_strip_staged<RK, LIM, PAIR>(P, u, out, c0, j0, H, dt, ctl.count_degenerate != 0, acc,
                                        ring[STAGE ? threadIdx.x >> 5 : 0]);
    else
      march_strip<RK, LIM, PAIR>(P, u, out, c0, j0, H, dt, ctl.count_degenerate != 0, acc);
  }
  block_commit<WPB * 32>(red, acc.kmax, acc.krho, acc.kp, acc.nonfinite, acc.degenerate, &stats[ctl.acc_slot]);
}

// Rows per warp: the given march_rows, else the smallest count that lets all
// warp strips of the grid run in a single wave of resident warps (so no SM
// idles in a tail), at least 8 so the per-strip prologue stays cheap.
template <int RK, int LIM, bool PAIR, bool STAGE>
cudaError_t launch_lim(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats, const EcgDtCtl& ctl,
                       cudaStream_t s)
{
  constexpr int WPB = 4;
  const int strips = (p.g.nx + kCells - 1) / kCells;
  // a band of rows (the pipelined host step) or the whole grid
  const int rlo = p.row_hi > 0 ? p.row_lo : 0;
  const int rhi = p.row_hi > 0 && p.row_hi < p.g.ny ? p.row_hi : p.g.ny;
  const int rows = rhi - rlo;
  if (rows <= 0) return cudaSuccess;
  int H = p.march_rows;
  if (H <= 0) {
    static int blocks_per_sm = 0;
    if (blocks_per_sm == 0) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fv_march_kernel<RK, LIM, WPB, PAIR, STAGE>, WPB * 32, 0) !=
              cudaSuccess ||
          b < 1)
        b = 1;
      blocks_per_sm = b;
    }
    const long long slots = static_cast<long long>(p.sm_count > 0 ? p.sm_count : 148) * blocks_per_sm * WPB;
    const long long per_col = slots / strips;  // warps available per strip column
    H = per_col > 0 ? static_cast<int>((rows + per_col - 1) / per_col) : rows;
    if (H < 8) H = 8;
  }
  const dim3 grid((strips + WPB - 1) / WPB, (rows + H - 1) / H);
  fv_march_kernel<RK, LIM, WPB, PAIR, STAGE><<<grid, WPB * 32, 0, s>>>(p, in, out, stats, ctl, H);
  return cudaGetLastError();
}

template <int RK, bool PAIR, bool STAGE>
cudaError_t launch_rk(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats, const EcgDtCtl& ctl,
                      cudaStream_t s)
{
  switch (p.limiter) {
    case ECG_LIMITER_MC: return launch_lim<RK, ECG_LIMITER_MC, PAIR, STAGE>(p, in, out, stats, ctl, s);
    case ECG_LIMITER_VANLEER: return launch_lim<RK, ECG_LIMITER_VANLEER, PAIR, STAGE>(p, in, out, stats, ctl, s);
    default: return launch_lim<RK, ECG_LIMITER_MINMOD, PAIR, STAGE>(p, in, out, stats, ctl, s);
  }
}

template <int RK>
cudaError_t launch_mode(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats, const EcgDtCtl& ctl,
                        cudaStream_t s, bool pair, bool stage)
{
  if (stage) return launch_rk<RK, true, true>(p, in, out, stats, ctl, s);
  return pair ? launch_rk<RK, true, false>(p, in, out, stats, ctl, s) : launch_rk<RK, false, false>(p, in, out, stats, ctl, s);
}

// pair: evaluate the x- and y-face of a row together (one vote for both);
// otherwise one after the other.  stage: paired faces, rows staged through
// shared memory (march_strip_staged).
inline cudaError_t launch(const EcgFvParams& p, const double* in, double* out, EcgStepStats* stats,
                          const EcgDtCtl& ctl, cudaStream_t s, bool pair, bool stage)
{
  switch (p.riemann) {
    case ECG_RIEMANN_RUSANOV: return launch_mode<ECG_RIEMANN_RUSANOV>(p, in, out, stats, ctl, s, pair, stage);
    case ECG_RIEMANN_LOWMACH_HLLC: return launch_mode<ECG_RIEMANN_LOWMACH_HLLC>(p, in, out, stats, ctl, s, pair, stage);
    case ECG_RIEMANN_XIE_AM_HLLC_P: {
      // Staged strips carry the 5-face sensor along, on grids whose strips
      // fill a wave of resident warps with runs of 8 rows or more (2560x640:
      // 139 us against the tile kernel's 176 us), and for a band of rows
      // (the pipelined host step: the tile kernel steps whole grids only);
      // smaller grids, and the other variants, use the 16x16 tile kernel
      // (Gresho 256^2: 19 us against 34 us on strips).
      const long long strips = (p.g.nx + kCells - 1) / kCells;
      const int rlo = p.row_hi > 0 ? p.row_lo : 0;
      const int rhi = p.row_hi > 0 && p.row_hi < p.g.ny ? p.row_hi : p.g.ny;
      const long long slots = static_cast<long long>(p.sm_count > 0 ? p.sm_count : 148) * 12;
      if (stage && (p.row_hi > 0 || strips * ((rhi - rlo + 7) / 8) >= slots))
        return launch_rk<ECG_RIEMANN_XIE_AM_HLLC_P, false, true>(p, in, out, stats, ctl, s);
      return fast::launch(p, in, out, stats, ctl, s);
    }
    default: return launch_mode<ECG_RIEMANN_HLLC>(p, in, out, stats, ctl, s, pair, stage);
  }
}

}  // namespace march
