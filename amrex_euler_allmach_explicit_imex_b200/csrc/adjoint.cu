// Adjoint of the explicit step: ecg_explicit_step_device (the forward on
// caller arrays) and ecg_explicit_step_vjp_device (include/ecg.h).
//
// U1 = U0 - dt [ (F_{i+1/2} - F_{i-1/2}) / dx + (G_{j+1/2} - G_{j-1/2}) / dy ]
// (numerics/explicit_update.hpp:58-102) with dt held fixed, so
//   gU0 = gU1 + (dq/dU)^T gq,   gq = sum over faces f of (dF_f/dq)^T gF_f,
//   gF_{i+1/2} = dt/dx (gU1_{i+1} - gU1_i)   (and the same along y).
// One thread per face evaluates the face's 4 x 16 Jacobian column by column
// (forward-mode duals through the same limiter / Riemann branches the forward
// takes, adjoint.cuh) and scatters (dF/dq)^T gF into the primitive gradients
// of the four cells of its stencil, mapped through the boundary policy
// (periodic images and outflow copies add to their source cell, the bubble
// wall mirror flips the v component, constant inflow states receive nothing).
// The scatter uses FP64 atomics, so the summation order and the last bits of
// gU0 vary from run to run.  A second kernel applies (dq/dU)^T per cell.
#include <cuda_runtime.h>

#include <cstring>

#include "ctx.h"
#include "ecg.h"

#include "adjoint.cuh"

namespace {

using ecg_adj::C4;
using ecg_adj::Dual;
using ecg_adj::P4;

struct Src {
  int i, j;
  bool valid, flip;
};

__device__ __forceinline__ int wrapi(int i, int n)
{
  int r = i % n;
  return r < 0 ? r + n : r;
}

// Source cell of (i, j) under the ghost policy: the map of load_cell
// (problems/boundary_conditions.hpp:2-73) for the policies without a ring.
__device__ Src source_of(const EcgFvParams& P, int i, int j)
{
  const int nx = P.g.nx, ny = P.g.ny;
  Src s{i, j, true, false};
  if (i < 0) {
    if (P.bc.x_lo == BC_CONST) return Src{0, 0, false, false};
    s.i = P.bc.x_lo == BC_PERIODIC ? wrapi(i, nx) : 0;
  } else if (i >= nx) {
    if (P.bc.x_hi == BC_CONST) return Src{0, 0, false, false};
    s.i = P.bc.x_hi == BC_PERIODIC ? wrapi(i, nx) : nx - 1;
  }
  if (j < 0) {
    if (P.bc.y_lo == BC_CONST) return Src{0, 0, false, false};
    if (P.bc.y_lo == BC_PERIODIC) {
      s.j = wrapi(j, ny);
    } else if (P.bc.y_lo == BC_REFLECT) {
      s.j = -j - 1 > ny - 1 ? ny - 1 : -j - 1;
      s.flip = true;
    } else {
      s.j = 0;
    }
  } else if (j >= ny) {
    if (P.bc.y_hi == BC_CONST) return Src{0, 0, false, false};
    if (P.bc.y_hi == BC_PERIODIC) {
      s.j = wrapi(j, ny);
    } else if (P.bc.y_hi == BC_REFLECT) {
      s.j = 2 * ny - 1 - j < 0 ? 0 : 2 * ny - 1 - j;
      s.flip = true;
    } else {
      s.j = ny - 1;
    }
  }
  return s;
}

// Primitive state of (i, j), ghosts included (to_primitive, core/state_primitives.hpp:103-111).
__device__ P4<double> prim_at(const EcgFvParams& P, const double* __restrict__ u, const Src& s)
{
  double rho, mx, my, E;
  if (!s.valid) {
    rho = P.bc.cst[0];
    mx = P.bc.cst[1];
    my = P.bc.cst[2];
    E = P.bc.cst[3];
  } else {
    const long long o = static_cast<long long>(s.j) * P.g.pitch + s.i;
    rho = u[o];
    mx = u[o + P.g.plane];
    my = u[o + 2 * P.g.plane];
    E = u[o + 3 * P.g.plane];
    if (s.flip) my = -my;
  }
  const double inv_rho = 1.0 / rho;
  const double uu = mx * inv_rho, vv = my * inv_rho;
  const double kin = 0.5 * rho * (uu * uu + vv * vv);
  return P4<double>{rho, uu, vv, (P.gamma - 1.0) * (E - kin)};
}

__device__ __forceinline__ double comp(const P4<double>& q, int m)
{
  return m == 0 ? q.rho : (m == 1 ? q.u : (m == 2 ? q.v : q.p));
}

// One thread per face of `axis`: gq of the face's 4-cell stencil += (dF/dq)^T gF.
template <int AXIS>
__global__ void face_vjp_kernel(const EcgFvParams P, const double* __restrict__ u0, const double* __restrict__ gu1,
                                double dt, double* __restrict__ gq)
{
  const int nx = P.g.nx, ny = P.g.ny;
  const int fw = AXIS == 0 ? nx + 1 : nx;
  const int fh = AXIS == 0 ? ny : ny + 1;
  const long long nf = static_cast<long long>(fw) * fh;
  const long long n = static_cast<long long>(nx) * ny;
  const double coef = dt * (AXIS == 0 ? P.g.inv_dx : P.g.inv_dy);
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nf;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int fi = static_cast<int>(e % fw), fj = static_cast<int>(e / fw);
    // cells L = c[1] (index f-1 along the axis) and R = c[2] (index f)
    const int li = AXIS == 0 ? fi - 1 : fi, lj = AXIS == 0 ? fj : fj - 1;
    const bool l_in = li >= 0 && lj >= 0;
    const bool r_in = AXIS == 0 ? fi < nx : fj < ny;
    double gF[4];
    for (int m = 0; m < 4; ++m) {
      const double gr = r_in ? gu1[static_cast<long long>(fj) * nx + fi + m * n] : 0.0;
      const double gl = l_in ? gu1[static_cast<long long>(lj) * nx + li + m * n] : 0.0;
      gF[m] = coef * (gr - gl);
    }
    if (gF[0] == 0.0 && gF[1] == 0.0 && gF[2] == 0.0 && gF[3] == 0.0) continue;
    Src src[4];
    P4<double> q[4];
    for (int k = 0; k < 4; ++k) {
      const int ci = AXIS == 0 ? fi - 2 + k : fi, cj = AXIS == 0 ? fj : fj - 2 + k;
      src[k] = source_of(P, ci, cj);
      q[k] = prim_at(P, u0, src[k]);
    }
    const int k0 = P.order > 1 ? 0 : 1, k1 = P.order > 1 ? 4 : 3;
    for (int k = k0; k < k1; ++k) {
      if (!src[k].valid) continue;
      for (int m = 0; m < 4; ++m) {
        P4<Dual> c[4];
        for (int kk = 0; kk < 4; ++kk) {
          c[kk] = P4<Dual>{Dual{q[kk].rho, 0.0}, Dual{q[kk].u, 0.0}, Dual{q[kk].v, 0.0}, Dual{q[kk].p, 0.0}};
        }
        Dual* slot = m == 0 ? &c[k].rho : (m == 1 ? &c[k].u : (m == 2 ? &c[k].v : &c[k].p));
        slot->d = 1.0;
        const C4<Dual> F = ecg_adj::t_face_flux(c, AXIS, P.gamma, P.riemann, P.order, P.limiter);
        double g = gF[0] * F.rho.d + gF[1] * F.mx.d + gF[2] * F.my.d + gF[3] * F.E.d;
        if (g == 0.0) continue;
        if (src[k].flip && m == 2) g = -g;
        atomicAdd(&gq[static_cast<long long>(src[k].j) * nx + src[k].i + m * n], g);
      }
    }
  }
}

// gU0 = gU1 + (dq/dU)^T gq per cell.
__global__ void cell_vjp_kernel(const EcgFvParams P, const double* __restrict__ u0, const double* __restrict__ gu1,
                                const double* __restrict__ gq, double* __restrict__ gu0)
{
  const long long n = static_cast<long long>(P.g.nx) * P.g.ny;
  const double gm1 = P.gamma - 1.0;
  for (long long r = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double rho = u0[r], mx = u0[r + n], my = u0[r + 2 * n];
    const double inv_rho = 1.0 / rho;
    const double uu = mx * inv_rho, vv = my * inv_rho;
    const double g0 = gq[r], g1 = gq[r + n], g2 = gq[r + 2 * n], g3 = gq[r + 3 * n];
    gu0[r] = gu1[r] + g0 - (g1 * uu + g2 * vv) * inv_rho + g3 * gm1 * 0.5 * (uu * uu + vv * vv);
    gu0[r + n] = gu1[r + n] + g1 * inv_rho - g3 * gm1 * uu;
    gu0[r + 2 * n] = gu1[r + 2 * n] + g2 * inv_rho - g3 * gm1 * vv;
    gu0[r + 3 * n] = gu1[r + 3 * n] + g3 * gm1;
  }
}

int blocks_for(long long n, int nt)
{
  long long b = (n + nt - 1) / nt;
  if (b > 148 * 16) b = 148 * 16;
  return static_cast<int>(b < 1 ? 1 : b);
}

// Compact planes (i fastest, no padding) of the context's grid.
EcgFvParams compact_params(ecg_ctx* c)
{
  EcgFvParams p = ecgi::fv_params(c, false);
  p.g.pitch = c->grid.nx;
  p.g.plane = static_cast<long long>(c->grid.nx) * c->grid.ny;
  return p;
}

bool ensure_adj(ecg_ctx* c)
{
  if (c->adj_gq) return true;
  const size_t n = static_cast<size_t>(c->grid.nx) * c->grid.ny;
  return ecgi::cuda_ok(c, cudaMalloc(&c->adj_gq, sizeof(double) * 4 * n), "alloc adjoint") &&
         ecgi::cuda_ok(c, cudaMalloc(&c->adj_stats, sizeof(EcgStepStats)), "alloc adjoint stats");
}

}  // namespace

extern "C" {

ecg_status ecg_explicit_step_device(ecg_ctx* c, const double* u0, double dt, double* u1)
{
  if (!c || !u0 || !u1 || u0 == u1) return ECG_ERR_BAD_ARG;
  const EcgFvParams p = compact_params(c);
  if (p.bc.ring) {
    c->err = "exact-Dirichlet ghost rings are not supported on caller arrays";
    return ECG_ERR_UNSUPPORTED;
  }
  if (!ensure_adj(c)) return ECG_ERR_CUDA;
  EcgDtCtl ctl;
  std::memset(&ctl, 0, sizeof(ctl));
  ctl.dt = dt;
  ctl.count_degenerate = c->cfg.riemann != ECG_RIEMANN_RUSANOV;
  ctl.read_slot = 0;
  ctl.acc_slot = 0;
  ctl.reset_slot = -1;
  if (!ecgi::cuda_ok(c, c->ops->init_stats(c->adj_stats, 1, 0.0, c->stream), "init stats")) return ECG_ERR_CUDA;
  if (!ecgi::cuda_ok(c, c->ops->fv_step(p, u0, u1, c->adj_stats, ctl, c->tile_y, c->stream), "fv_step"))
    return ECG_ERR_CUDA;
  return ECG_OK;
}

ecg_status ecg_explicit_step_vjp_device(ecg_ctx* c, const double* u0, double dt, const double* g_u1, double* g_u0)
{
  if (!c || !u0 || !g_u1 || !g_u0 || g_u1 == g_u0) return ECG_ERR_BAD_ARG;
  const EcgFvParams p = compact_params(c);
  if (p.bc.ring) {
    c->err = "exact-Dirichlet ghost rings are not supported by the adjoint";
    return ECG_ERR_UNSUPPORTED;
  }
  if (c->cfg.riemann == ECG_RIEMANN_XIE_AM_HLLC_P) {
    c->err = "the adjoint covers rusanov, hllc and lowmach_hllc";
    return ECG_ERR_UNSUPPORTED;
  }
  if (!ensure_adj(c)) return ECG_ERR_CUDA;
  const long long n = static_cast<long long>(c->grid.nx) * c->grid.ny;
  if (!ecgi::cuda_ok(c, cudaMemsetAsync(c->adj_gq, 0, sizeof(double) * 4 * n, c->stream), "memset")) return ECG_ERR_CUDA;
  const long long nfx = static_cast<long long>(c->grid.nx + 1) * c->grid.ny;
  const long long nfy = static_cast<long long>(c->grid.nx) * (c->grid.ny + 1);
  face_vjp_kernel<0><<<blocks_for(nfx, 128), 128, 0, c->stream>>>(p, u0, g_u1, dt, c->adj_gq);
  if (!ecgi::cuda_ok(c, cudaGetLastError(), "face vjp x")) return ECG_ERR_CUDA;
  face_vjp_kernel<1><<<blocks_for(nfy, 128), 128, 0, c->stream>>>(p, u0, g_u1, dt, c->adj_gq);
  if (!ecgi::cuda_ok(c, cudaGetLastError(), "face vjp y")) return ECG_ERR_CUDA;
  cell_vjp_kernel<<<blocks_for(n, 256), 256, 0, c->stream>>>(p, u0, g_u1, c->adj_gq, g_u0);
  if (!ecgi::cuda_ok(c, cudaGetLastError(), "cell vjp")) return ECG_ERR_CUDA;
  return ECG_OK;
}

}  // extern "C"
