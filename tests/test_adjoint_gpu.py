"""Hand-written adjoint of the explicit O2 step against central finite
differences, through the torch.autograd.Function of the package.

The reference has no adjoint; the forward it differentiates is the
parity-tested fast explicit step (ecg_explicit_step_device).  dt is held fixed
per step, as the adjoint defines it.  Tolerances: one step, 1e-7 relative
(FD with h = 1e-6 on smooth states); the 256^2 blob rollout of 400 steps,
1e-5 relative per direction (minmod switches near the blob's extrema make the
objective only piecewise smooth)."""
import math

import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200.config import read_config

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _smooth_state(torch, nx, ny, seed, gamma=1.4):
    g = torch.Generator().manual_seed(seed)
    x = (torch.arange(nx, dtype=torch.float64) + 0.5) / nx
    y = (torch.arange(ny, dtype=torch.float64) + 0.5) / ny
    X, Y = torch.meshgrid(x, y, indexing="xy")
    a = torch.rand(8, generator=g, dtype=torch.float64)
    rho = 1.0 + 0.3 * torch.sin(2 * math.pi * (X + a[0])) * torch.cos(2 * math.pi * (Y + a[1]))
    u = 0.4 * torch.sin(2 * math.pi * (Y + a[2])) + 0.2 * a[3]
    v = 0.4 * torch.cos(2 * math.pi * (X + a[4])) - 0.2 * a[5]
    p = 1.0 + 0.2 * torch.cos(2 * math.pi * (X + Y + a[6]))
    return torch.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)]).cuda()


CASES = [
    ("periodic-hllc", "geometry.is_periodic=1 1\neuler.riemann=hllc\neuler.problem=advection_blob\n"),
    ("outflow-lowmach", "geometry.is_periodic=0 0\neuler.riemann=lowmach_hllc\neuler.problem=advection_blob\n"),
    ("outflow-rusanov-mc", "geometry.is_periodic=0 1\neuler.riemann=rusanov\neuler.slope_limiter=mc\n"
                           "euler.problem=toro1\n"),
    ("bubble-hllc", "euler.riemann=hllc\neuler.problem=shock_density_bubble_2d\ngeometry.prob_hi=2 0.5\n"),
]


@pytest.mark.parametrize("name,kv", CASES, ids=[c[0] for c in CASES])
def test_step_vjp_matches_finite_differences(gpu, name, kv):
    torch = _torch()
    from amrex_euler_allmach_explicit_imex_b200 import autograd as ad

    nx, ny = 40, 24
    cfg = read_config(f"amr.n_cell={nx} {ny}\neuler.spatial_order=2\n" + kv).cfg
    ectx = ad.make_context(cfg)
    try:
        u0 = _smooth_state(torch, nx, ny, 1)
        dt = 2.0e-3
        gen = torch.Generator().manual_seed(2)
        g1 = torch.randn(4, ny, nx, generator=gen, dtype=torch.float64).cuda()
        g0 = ad._vjp(ectx, u0, dt, g1)
        h = 1.0e-6
        for r in range(3):
            d = torch.randn(4, ny, nx, generator=gen, dtype=torch.float64).cuda() * u0.abs().mean(dim=(1, 2), keepdim=True)
            up = ad._step(ectx, u0 + h * d, dt)
            um = ad._step(ectx, u0 - h * d, dt)
            fd = float(((up - um) / (2 * h) * g1).sum())
            an = float((g0 * d).sum())
            assert an == pytest.approx(fd, rel=1e-7, abs=1e-9), (name, r)
    finally:
        ectx.close()


def _blob(torch, n, gamma=1.4):
    x = (torch.arange(n, dtype=torch.float64) + 0.5) / n
    X, Y = torch.meshgrid(x, x, indexing="xy")
    return 1.0 + 0.5 * torch.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)


def _u_of_rho(torch, rho, gamma=1.4):
    # (u, v) = (1, 1), p = 1
    return torch.stack([rho, rho, rho, 1.0 / (gamma - 1.0) + rho * torch.ones_like(rho)])


def test_blob_rollout_gradient_against_central_differences(gpu):
    """Gaussian blob on the periodic unit square, 256^2, 400 O2 HLLC steps at
    the CFL-0.5 dt of the initial state, J = sum(rho^2), dJ/drho0 with a
    checkpoint every 20 steps, against central differences (h = 1e-6) along
    16 seeded random directions."""
    torch = _torch()
    from amrex_euler_allmach_explicit_imex_b200 import autograd as ad

    n, steps = 256, 400
    cfg = read_config(f"amr.n_cell={n} {n}\ngeometry.is_periodic=1 1\neuler.problem=advection_blob\n"
                      "euler.riemann=hllc\neuler.spatial_order=2\neuler.cfl=0.5\nstop_time=10\n").cfg
    ectx = ad.make_context(cfg)
    try:
        rho0 = _blob(torch, n).cuda()
        u0 = _u_of_rho(torch, rho0)
        ctx2 = api.Context(cfg)
        ctx2.upload(u0.cpu().numpy())
        dt = api.compute_euler_dt(ctx2, 0.0)
        ctx2.close()
        dts = [dt] * steps

        r = rho0.clone().requires_grad_(True)
        uN = ad.explicit_rollout(ectx, _u_of_rho(torch, r), dts, checkpoint_every=20)
        J = (uN[0] ** 2).sum()
        J.backward()
        grad = r.grad.detach()

        def J_of(rho):
            with torch.no_grad():
                u = _u_of_rho(torch, rho).contiguous()
                for dtk in dts:
                    u = ad._step(ectx, u, dtk)
                return float((u[0] ** 2).sum())

        gen = torch.Generator().manual_seed(16)
        h = 1.0e-6
        errs = []
        for _ in range(16):
            d = torch.randn(n, n, generator=gen, dtype=torch.float64).cuda()
            fd = (J_of(rho0 + h * d) - J_of(rho0 - h * d)) / (2 * h)
            an = float((grad * d).sum())
            errs.append(abs(an - fd) / max(abs(fd), 1e-12))
        assert max(errs) <= 1e-5, errs
    finally:
        ectx.close()
