"""Synthetic workloads of the batched and differentiable paths.

The reference runs one solve per process and has no batched or adjoint
driver, so these inputs are defined here: seeded Riemann problems on a
ladder of uneven grids (the batched configuration) and the Gaussian density
blob (the adjoint configuration).  States are returned as numpy arrays in the
Array4 layout (4, ny, nx) that ecg_upload_state takes."""
import numpy as np

from .config import read_config

BATCH_GRIDS = [(64, 64), (128, 32), (256, 256), (512, 128), (1024, 256)]


def riemann_batch(nsolve=64, seed=0, grids=BATCH_GRIDS, gamma=1.4, cfl=0.5, stop_time=1.0e9, riemann="hllc"):
    """`nsolve` explicit O2 solves, grid (nx, ny) drawn from `grids`; per solve
    rho, p ~ U[0.1, 1] and u, v ~ U[-1, 1] on each side of an interface at
    x0 ~ U[0.3, 0.7] on [0, 1] x [0, ny/nx]; transmissive x, periodic y.
    Returns (list of RunSettings, list of states)."""
    rng = np.random.default_rng(seed)
    cfgs, states = [], []
    for _ in range(nsolve):
        nx, ny = grids[int(rng.integers(len(grids)))]
        rho = rng.uniform(0.1, 1.0, 2)
        p = rng.uniform(0.1, 1.0, 2)
        u = rng.uniform(-1.0, 1.0, 2)
        v = rng.uniform(-1.0, 1.0, 2)
        x0 = rng.uniform(0.3, 0.7)
        kv = (f"amr.n_cell={nx} {ny}\ngeometry.prob_lo=0 0\ngeometry.prob_hi=1 {ny / nx!r}\n"
              "geometry.is_periodic=0 1\neuler.problem=toro1\neuler.method=explicit\neuler.spatial_order=2\n"
              f"euler.riemann={riemann}\neuler.slope_limiter=minmod\neuler.cfl={cfl!r}\neuler.gamma={gamma!r}\n"
              f"stop_time={stop_time!r}\nmax_step=100000000\neuler.field_boundary=outflow\n"
              f"prob.x0={x0!r}\n")
        cfgs.append(read_config(kv))
        x = (np.arange(nx) + 0.5) / nx
        left = (x < x0)[None, :].repeat(ny, 0)
        r_ = np.where(left, rho[0], rho[1])
        u_ = np.where(left, u[0], u[1])
        v_ = np.where(left, v[0], v[1])
        p_ = np.where(left, p[0], p[1])
        states.append(np.stack([r_, r_ * u_, r_ * v_, p_ / (gamma - 1.0) + 0.5 * r_ * (u_ * u_ + v_ * v_)]))
    return cfgs, states
