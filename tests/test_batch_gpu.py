"""Batched independent solves (ecg_batch_*) against the single-solve path.

Every solve of a batch runs the same per-cell formulas as a context's
device-resident loop (ecg_run, ECG_ARITH_FAST): same fluxes, same fused
reductions, same device-side compute_euler_dt.  The two are separate kernel
instantiations, and FMA contraction may fuse an inlined expression
differently in each, so they agree to rounding, not bit for bit: 1e-12
relative over the 30 steps, the fast path's per-step bound.  The single-solve
path itself is held to the reference by test_explicit_gpu.py; a few steps are
also checked against the oracle directly."""
import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api, workloads
from amrex_euler_allmach_explicit_imex_b200._lib import EcgError
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu

GRIDS = [(64, 64), (128, 32), (96, 40), (200, 8), (33, 17), (29, 5)]


def _batch(seed=3, n=6, **kw):
    return workloads.riemann_batch(n, seed, grids=GRIDS, **kw)


def _single(cfg, u0, steps):
    with api.Context(cfg, arith="fast") as ctx:
        ctx.upload(u0)
        r = api.run(ctx, steps, cfg.stop_time)
        return ctx.download(), r


@pytest.mark.parametrize("riemann", ["hllc", "rusanov", "lowmach_hllc", "xie_am_hllc_p"])
def test_batch_matches_single_solves(gpu, riemann):
    cfgs, states = _batch(riemann=riemann)
    with api.Batch(cfgs) as b:
        for k, u in enumerate(states):
            b.upload(k, u)
        res = b.run(30)
        got = [b.download(k) for k in range(len(cfgs))]
    for k, (c, u0) in enumerate(zip(cfgs, states)):
        want, r = _single(c.cfg, u0, 30)
        assert res[k].steps == r.steps == 30
        assert res[k].failed == 0
        assert res[k].time == pytest.approx(r.time, rel=1e-12)
        assert abs(res[k].hllc_degenerate_star_count - r.hllc_degenerate_star_count) <= max(
            2, 1e-3 * r.hllc_degenerate_star_count)
        assert golden_io.state_rel_err(got[k], want) <= 1e-12, f"solve {k} {c.cfg.n_cell[0]}x{c.cfg.n_cell[1]}"
        assert res[k].diagnostics.rho_min == pytest.approx(r.diagnostics.rho_min, rel=1e-12)


def test_batch_split_runs_equal_one_run(gpu):
    cfgs, states = _batch(seed=5)
    outs = []
    for split in [(20,), (7, 13)]:
        with api.Batch(cfgs) as b:
            for k, u in enumerate(states):
                b.upload(k, u)
            for s in split:
                res = b.run(s)
            outs.append(([b.download(k) for k in range(len(cfgs))], [(r.steps, r.time) for r in res]))
    assert outs[0][1] == outs[1][1]
    for a, c in zip(outs[0][0], outs[1][0]):
        assert np.array_equal(a, c)


def test_batch_stop_time_per_solve(gpu):
    cfgs, states = _batch(seed=7)
    # solve 0 stops early at its own stop_time; the others run all steps
    cfgs[0].cfg.stop_time = 2.0e-3
    with api.Batch(cfgs) as b:
        for k, u in enumerate(states):
            b.upload(k, u)
        res = b.run(40)
        u0 = b.download(0)
    assert res[0].time == pytest.approx(2.0e-3, rel=0, abs=1e-15)
    assert res[0].steps < 40
    assert all(r.steps == 40 for r in res[1:])
    want, r = _single(cfgs[0].cfg, states[0], 40)
    assert r.steps == res[0].steps and golden_io.state_rel_err(u0, want) <= 1e-12


def test_batch_against_oracle(gpu, oracle):
    cfgs, states = _batch(seed=11, n=4)
    with api.Batch(cfgs) as b:
        for k, u in enumerate(states):
            b.upload(k, u)
        b.run(3)
        got = [b.download(k) for k in range(len(cfgs))]
    for k, (c, u0) in enumerate(zip(cfgs, states)):
        u, t = u0, 0.0
        for _ in range(3):
            dt = oracle.euler_dt(c.cfg, u, t)
            u, _ = oracle.step(c.cfg, u, dt, t)
            t += dt
        assert golden_io.state_rel_err(got[k], u) <= 3e-12


def test_batch_rejects_mixed_solvers(gpu):
    cfgs, _ = _batch(n=2)
    cfgs[1] = read_config("amr.n_cell=32 8\neuler.problem=toro1\neuler.riemann=rusanov\n")
    with pytest.raises(EcgError):
        api.Batch(cfgs)
