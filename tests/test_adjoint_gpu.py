"""Hand-written adjoint of the explicit O2 step against central finite
differences, through the torch.autograd.Function of the package.

The reference has no adjoint; the forward it differentiates is the
parity-tested fast explicit step (ecg_explicit_step_device), with dt held
fixed per step as the adjoint defines it.  The step is only piecewise
differentiable: a limited slope switches branch where a one-sided difference
changes sign or (minmod, MC) where the two one-sided differences tie in
magnitude, and a central difference that straddles such a switch is not the
derivative of either branch.  The one-step tests therefore use states on
which no switch lies close to the base state (quadratic profiles for minmod,
whose one-sided differences never tie; van Leer, which has no tie switch),
with a small FD step (h = 1e-7), and hold the adjoint to 2e-6 relative.  The 256^2 blob rollout (uniform velocity
and pressure, density exactly 1 far from the blob) sits on switches by
construction; there the check is along 16 smooth seeded directions, at 1e-4
for van Leer and 5e-3 for minmod (measured worst cases 6.6e-5 and 2.9e-3).
A wrong adjoint term shows at 1e-3 and above on the one-step tests."""
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
    """Sines along both axes: smooth, with one-sided differences that can
    tie in magnitude near inflection points (use with van Leer)."""
    g = torch.Generator().manual_seed(seed)
    x = (torch.arange(nx, dtype=torch.float64) + 0.5) / nx
    y = (torch.arange(ny, dtype=torch.float64) + 0.5) / ny
    X, Y = torch.meshgrid(x, y, indexing="xy")
    a = torch.rand(8, generator=g, dtype=torch.float64)
    rho = 1.0 + 0.3 * torch.sin(2 * math.pi * (X + a[0])) * torch.cos(2 * math.pi * (Y + a[1]))
    u = 0.4 * torch.sin(2 * math.pi * (Y + 0.7 * X + a[2])) + 0.2 * a[3]
    v = 0.4 * torch.cos(2 * math.pi * (X - 0.6 * Y + a[4])) - 0.2 * a[5]
    p = 1.0 + 0.2 * torch.cos(2 * math.pi * (X + 1.3 * Y + a[6]))
    return torch.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)]).cuda()


def _quadratic_state(torch, nx, ny, gamma=1.4, hx=1.0, hy=1.0):
    """Quadratic profiles: one-sided differences differ by a constant second
    difference, so minmod never ties; the vertices sit off the cell faces."""
    x = (torch.arange(nx, dtype=torch.float64) + 0.5) / nx * hx
    y = (torch.arange(ny, dtype=torch.float64) + 0.5) / ny * hy
    X, Y = torch.meshgrid(x, y, indexing="xy")
    rho = 1.0 + 0.3 * (X / hx - 0.313) ** 2 + 0.2 * (Y / hy - 0.627) ** 2
    u = 0.3 - 0.5 * (X / hx - 0.571) ** 2 + 0.2 * (Y / hy - 0.119) ** 2
    v = -0.2 + 0.4 * (X / hx - 0.847) ** 2 - 0.3 * (Y / hy - 0.433) ** 2
    p = 1.0 + 0.25 * (X / hx - 0.662) ** 2 + 0.15 * (Y / hy - 0.281) ** 2
    return torch.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)]).cuda()


CASES = [
    ("periodic-hllc-vanleer", "geometry.is_periodic=1 1\neuler.riemann=hllc\neuler.slope_limiter=vanleer\n"
                              "euler.problem=advection_blob\n", "sines"),
    ("outflow-hllc-minmod", "geometry.is_periodic=0 0\neuler.riemann=hllc\neuler.problem=advection_blob\n",
     "quadratic"),
    ("outflow-lowmach-minmod", "geometry.is_periodic=0 0\neuler.riemann=lowmach_hllc\neuler.problem=advection_blob\n",
     "quadratic"),
    ("outflow-rusanov-vanleer", "geometry.is_periodic=0 1\neuler.riemann=rusanov\neuler.slope_limiter=vanleer\n"
                                "euler.problem=toro1\n", "sines"),
    ("bubble-hllc-minmod", "euler.riemann=hllc\neuler.problem=shock_density_bubble_2d\ngeometry.prob_hi=2 0.5\n",
     "quadratic"),
]


@pytest.mark.parametrize("name,kv,state", CASES, ids=[c[0] for c in CASES])
def test_step_vjp_matches_finite_differences(gpu, name, kv, state):
    """<g1, (step(u0 + h d) - step(u0 - h d)) / 2h> = <vjp(u0, g1), d> along
    random directions d, one direction per conserved component and one mixed."""
    torch = _torch()
    from amrex_euler_allmach_explicit_imex_b200 import autograd as ad

    nx, ny = 40, 24
    cfg = read_config(f"amr.n_cell={nx} {ny}\neuler.spatial_order=2\n" + kv).cfg
    ectx = ad.make_context(cfg)
    try:
        hx = cfg.prob_hi[0] - cfg.prob_lo[0]
        hy = cfg.prob_hi[1] - cfg.prob_lo[1]
        u0 = _smooth_state(torch, nx, ny, 1) if state == "sines" else _quadratic_state(torch, nx, ny, hx=hx, hy=hy)
        dt = 2.0e-3 * hx
        gen = torch.Generator().manual_seed(2)
        g1 = torch.randn(4, ny, nx, generator=gen, dtype=torch.float64).cuda()
        g0 = ad._vjp(ectx, u0, dt, g1)
        h = 1.0e-7
        scale = u0.abs().mean(dim=(1, 2), keepdim=True)
        for comp in range(5):
            d = torch.randn(4, ny, nx, generator=gen, dtype=torch.float64).cuda() * scale
            if comp < 4:
                mask = torch.zeros(4, 1, 1, dtype=torch.float64, device=d.device)
                mask[comp] = 1.0
                d = d * mask
            up = ad._step(ectx, u0 + h * d, dt)
            um = ad._step(ectx, u0 - h * d, dt)
            fd = float(((up - um) / (2 * h) * g1).sum())
            an = float((g0 * d).sum())
            assert an == pytest.approx(fd, rel=2e-6, abs=1e-9), (name, comp)
    finally:
        ectx.close()


def _blob(torch, n, gamma=1.4):
    x = (torch.arange(n, dtype=torch.float64) + 0.5) / n
    X, Y = torch.meshgrid(x, x, indexing="xy")
    return 1.0 + 0.5 * torch.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)


def _u_of_rho(torch, rho, gamma=1.4):
    # (u, v) = (1, 1), p = 1
    return torch.stack([rho, rho, rho, 1.0 / (gamma - 1.0) + rho * torch.ones_like(rho)])


@pytest.mark.parametrize("limiter,tol", [("minmod", 5e-3), ("vanleer", 1e-4)])
def test_blob_rollout_gradient_against_central_differences(gpu, limiter, tol):
    """Gaussian blob rho = 1 + 0.5 exp(-|x - c|^2 / 0.01) on the periodic unit
    square, 256^2, (u, v) = (1, 1), p = 1; 400 O2 HLLC steps at the CFL-0.5 dt
    of the initial state; J = sum(rho^2); dJ/drho0 with a checkpoint every 20
    steps, against central differences (h = 1e-6) along 16 seeded smooth
    random directions (random Fourier modes)."""
    torch = _torch()
    from amrex_euler_allmach_explicit_imex_b200 import autograd as ad

    n, steps = 256, 400
    cfg = read_config(f"amr.n_cell={n} {n}\ngeometry.is_periodic=1 1\neuler.problem=advection_blob\n"
                      f"euler.riemann=hllc\neuler.spatial_order=2\neuler.cfl=0.5\nstop_time=10\n"
                      f"euler.slope_limiter={limiter}\n").cfg
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
        x = (torch.arange(n, dtype=torch.float64) + 0.5) / n
        X, Y = torch.meshgrid(x, x, indexing="xy")
        h = 1.0e-6
        errs = []
        for _ in range(16):
            d = torch.zeros(n, n, dtype=torch.float64)
            for _m in range(3):
                kx, ky = (int(k) for k in torch.randint(1, 6, (2,), generator=gen))
                ph = torch.rand(2, generator=gen, dtype=torch.float64)
                amp = float(torch.randn(1, generator=gen, dtype=torch.float64))
                d += amp * torch.sin(2 * math.pi * (kx * X + ph[0])) * torch.cos(2 * math.pi * (ky * Y + ph[1]))
            d = d.cuda()
            fd = (J_of(rho0 + h * d) - J_of(rho0 - h * d)) / (2 * h)
            an = float((grad * d).sum())
            errs.append(abs(an - fd) / max(abs(fd), 1e-12))
        assert max(errs) <= tol, errs
    finally:
        ectx.close()
