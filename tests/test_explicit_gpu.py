"""GPU parity of the explicit path through the C ABI against the reference's
outputs (golden fixtures from the reference code) and the CPU oracle.

Tolerances: ECG_ARITH_EXACT (no FMA contraction) must be bit-identical to the
reference CPU build; ECG_ARITH_FAST must agree within 1e-12 relative per
step (field-family relative error, tests/golden_io.state_rel_err)."""
import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu

CASES = list(golden_io.explicit_cases())
FAST_TOL = 1e-12


# (arith, explicit kernel): exact tile kernel; fast column-strip kernel with
# rows staged through shared memory (default); the same with rows loaded into
# registers; fast square-tile kernel
KERNELS = [("exact", 0), ("fast", 0), ("fast", 3), ("fast", 1)]


@pytest.mark.parametrize("arith,kernel", KERNELS, ids=["exact", "fast-strip", "fast-strip-regs", "fast-tile"])
@pytest.mark.parametrize("key,case", CASES, ids=[k for k, _ in CASES])
def test_explicit_step_parity(gpu, arith, kernel, key, case):
    cfg = read_config(golden_io.kv_of(case["kv"])).cfg
    t, dt = float(case["t"]), float(case["dt"])
    with api.Context(cfg, arith=arith, tile_y=kernel) as ctx:
        ctx.upload(case["u0"])
        g = api.fill_problem_ghosts(ctx, t)
        deg = api.euler_fv_one_step(ctx, dt, t)
        u1 = ctx.download()
        edt = api.compute_euler_dt(ctx, t)
        d = api.compute_diagnostics(ctx)
        a = api.compute_admissibility_diagnostics(ctx)
        idt, td = api.compute_imex_dt(ctx, t)
    assert np.array_equal(g, case["ghost"]), "ghost fill"
    if arith == "exact":
        assert np.array_equal(u1, case["u1"])
        assert edt == float(case["edt"])
        assert [d.rho_min, d.pressure_min, d.nonfinite_count] == list(case["diag"])
        assert [idt, td.material_rate_max, td.acoustic_rate_max] == list(case["imexdt"])
        assert [a.rho_min, a.pressure_min, a.internal_energy_min] == list(case["adm"][:3])
    else:
        assert golden_io.state_rel_err(u1, case["u1"]) <= FAST_TOL
        assert abs(edt - float(case["edt"])) <= FAST_TOL * float(case["edt"])
        assert d.nonfinite_count == int(case["diag"][2])
    assert deg == int(case["deg"])
    assert [a.nonfinite_count, a.density_failure_count, a.pressure_failure_count,
            a.internal_energy_failure_count] == [int(x) for x in case["adm"][3:]]


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_sod_reference_loop_through_abi(gpu, arith):
    """The reference driver's loop (compute_euler_dt -> euler_fv_one_step ->
    compute_diagnostics) issued call by call through the C ABI."""
    z = golden_io.load("sod_400x4.npz")
    cfg = read_config(golden_io.kv_of(z["kv"])).cfg
    with api.Context(cfg, arith=arith) as ctx:
        ctx.upload(z["u0"])
        t, n, dts, degs = 0.0, 0, [], []
        while n < 100000 and t < cfg.stop_time - 1e-14:
            dt = api.compute_euler_dt(ctx, t)
            degs.append(api.euler_fv_one_step(ctx, dt, t))
            d = api.compute_diagnostics(ctx)
            assert d.nonfinite_count == 0 and d.rho_min > 0 and d.pressure_min > 0
            dts.append(dt)
            t += dt
            n += 1
        u = ctx.download()
    assert n == 553
    l1 = np.abs(u[0] - z["exact_rho"][None, :]).mean()
    if arith == "exact":
        assert np.array_equal(np.array(dts), z["dts"])
        assert np.array_equal(u, z["u_final"])
        assert l1 == float(z["l1_rho"])
    else:
        assert abs(l1 - float(z["l1_rho"])) <= 1e-9 * float(z["l1_rho"])
    assert degs == list(z["degs"])


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_sod_device_loop(gpu, arith):
    """ecg_run: the same loop kept on the device (graph-captured chunks)."""
    z = golden_io.load("sod_400x4.npz")
    cfg = read_config(golden_io.kv_of(z["kv"])).cfg
    with api.Context(cfg, arith=arith) as ctx:
        ctx.upload(z["u0"])
        r = api.run(ctx, 100000, cfg.stop_time)
        u = ctx.download()
    assert r.steps == 553 and not r.failed
    assert r.time == pytest.approx(0.2, abs=1e-15)
    if arith == "exact":
        assert np.array_equal(u, z["u_final"])
        assert r.dt_sum == sum(z["dts"].tolist()) or abs(r.dt_sum - z["dts"].sum()) < 1e-15
        assert r.hllc_degenerate_star_count == int(z["degs"].sum())
    else:
        l1 = np.abs(u[0] - z["exact_rho"][None, :]).mean()
        assert abs(l1 - float(z["l1_rho"])) <= 1e-9 * float(z["l1_rho"])


def test_device_loop_max_step_and_failure(gpu):
    """max_step stops the device loop; a negative-density state fails fast."""
    z = golden_io.load("sod_400x4.npz")
    cfg = read_config(golden_io.kv_of(z["kv"])).cfg
    with api.Context(cfg) as ctx:
        ctx.upload(z["u0"])
        r = api.run(ctx, 37, cfg.stop_time)
        assert r.steps == 37 and not r.failed
        bad = z["u0"].copy()
        bad[0, 2, 100] = -1.0
        ctx.upload(bad)
        r = api.run(ctx, 10, cfg.stop_time)
        assert r.failed and r.steps == 0


def _smooth_periodic(nx, ny, rng):
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    rho = 1 + 0.3 * np.sin(2 * np.pi * X) * np.cos(4 * np.pi * Y) + 0.01 * rng.standard_normal((ny, nx))
    u = 0.5 * np.cos(2 * np.pi * Y)
    v = 0.3 * np.sin(2 * np.pi * X)
    p = 1 + 0.2 * np.cos(2 * np.pi * (X + Y))
    return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])


@pytest.mark.parametrize("riemann", ["hllc", "xie_am_hllc_p", "rusanov", "lowmach_hllc"])
def test_full_size_properties(gpu, riemann):
    """2560x640 (the benchmark size): fast vs exact arithmetic within 1e-12
    per step, and periodic mass/momentum/energy conservation to rounding."""
    rng = np.random.default_rng(5)
    nx, ny = 2560, 640
    u0 = _smooth_periodic(nx, ny, rng)
    kv = {"amr.n_cell": f"{nx} {ny}", "geometry.prob_hi": "4 1", "euler.riemann": riemann, "euler.spatial_order": 2}
    cfg = read_config(kv).cfg
    out = {}
    for arith in ("exact", "fast"):
        with api.Context(cfg, arith=arith) as ctx:
            ctx.upload(u0)
            dt = api.compute_euler_dt(ctx, 0.0)
            api.euler_fv_one_step(ctx, dt, 0.0)
            out[arith] = ctx.download()
    assert golden_io.state_rel_err(out["fast"], out["exact"]) <= FAST_TOL
    for k in range(4):
        s0, s1 = u0[k].sum(), out["exact"][k].sum()
        assert abs(s1 - s0) <= 1e-12 * np.abs(u0[k]).sum()


def test_hllcp_strips_match_the_tile_kernel(gpu):
    """xie_am_hllc_p on the 2560x640 bubble: the staged strips (default; the
    5-face sensor carried along the march) against the 16x16 tile kernel
    (tile_y 1) over three steps: the same face formulas, so the states agree
    to rounding and the degenerate counts and time steps are equal."""
    kv = {"euler.problem": "shock_density_bubble_2d", "amr.n_cell": "2560 640", "geometry.prob_hi": "2 0.5",
          "euler.riemann": "xie_am_hllc_p"}
    cfg = read_config(kv).cfg
    runs = {}
    for tile in (0, 1):
        with api.Context(cfg, tile_y=tile) as ctx:
            api.initialize_state(ctx)
            t, rec = 0.0, []
            for _ in range(3):
                dt = api.compute_euler_dt(ctx, t)
                deg = api.euler_fv_one_step(ctx, dt, t)
                rec.append((dt, deg))
                t += dt
            runs[tile] = (ctx.download(), rec)
    assert golden_io.state_rel_err(runs[0][0], runs[1][0]) <= 3e-13
    for (dt0, deg0), (dt1, deg1) in zip(runs[0][1], runs[1][1]):
        assert dt0 == pytest.approx(dt1, rel=1e-13)
        assert deg0 == deg1


def test_full_size_bubble_matches_oracle_on_a_band(gpu, oracle):
    """The 2560x640 bubble step against the oracle on the full grid."""
    kv = {"euler.problem": "shock_density_bubble_2d", "amr.n_cell": "2560 640"}
    cfg = read_config(kv).cfg
    u0 = oracle.initialize(cfg)
    dt = oracle.euler_dt(cfg, u0, 0.0)
    ref_u1, ref_deg = oracle.step(cfg, u0, dt, 0.0)
    with api.Context(cfg, arith="exact") as ctx:
        ctx.upload(u0)
        assert api.compute_euler_dt(ctx, 0.0) == dt
        deg = api.euler_fv_one_step(ctx, dt, 0.0)
        u1 = ctx.download()
    assert np.array_equal(u1, ref_u1)
    assert deg == ref_deg


INIT_PROBLEMS = [
    ("toro1", "geometry.prob_hi=1 0.1\namr.n_cell=37 5\nprob.test=3\n", 0.0),
    ("gresho_vortex", "amr.n_cell=33 29\neuler.mach=0.01\n", 1e-14),
    ("isentropic_vortex", "amr.n_cell=40 24\ngeometry.prob_lo=-5 -5\ngeometry.prob_hi=5 5\n"
                          "euler.vortex_center=0 0\n", 1e-14),
    ("riemann_quadrant", "amr.n_cell=30 30\n", 0.0),
    ("shock_density_bubble_2d", "amr.n_cell=160 40\ngeometry.prob_hi=2 0.5\n", 0.0),
    ("advection_blob", "amr.n_cell=45 45\n", 0.0),
]


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("problem,extra,tol", INIT_PROBLEMS, ids=[p for p, _, _ in INIT_PROBLEMS])
def test_initialize_state_on_device(gpu, oracle, arith, problem, extra, tol):
    """initialize_state on the device against the oracle's restatement of
    problem_initialization.hpp: exact where the profile needs only + - * /
    sqrt (in ECG_ARITH_EXACT), to rounding of log/exp/pow otherwise."""
    cfg = read_config(f"euler.problem={problem}\n" + extra).cfg
    want = oracle.initialize(cfg)
    with api.Context(cfg, arith=arith) as ctx:
        api.initialize_state(ctx)
        got = ctx.download()
    if arith == "exact" and tol == 0.0:
        assert np.array_equal(got, want)
    else:
        assert golden_io.state_rel_err(got, want) <= max(tol, 1e-15)


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("riemann", ["hllc", "xie_am_hllc_p"])
def test_mach122_variant_steps(gpu, oracle, arith, riemann):
    """The Mach 1.22 shock / bubble configuration: device initial state and
    three steps against the oracle's restatement (bit-identical in
    ECG_ARITH_EXACT, 1e-12 relative per step in ECG_ARITH_FAST)."""
    cfg = read_config(f"euler.problem=shock_bubble_mach122\namr.n_cell=96 24\neuler.riemann={riemann}\n").cfg
    u = oracle.initialize(cfg)
    with api.Context(cfg, arith=arith) as ctx:
        api.initialize_state(ctx)
        assert np.array_equal(ctx.download(), u) if arith == "exact" else golden_io.state_rel_err(ctx.download(), u) <= 1e-15
        ctx.upload(u)
        t = 0.0
        for _ in range(3):
            dt = oracle.euler_dt(cfg, u, t)
            want, _ = oracle.step(cfg, u, dt, t)
            ctx.upload(u)
            api.euler_fv_one_step(ctx, dt, t)
            got = ctx.download()
            if arith == "exact":
                assert np.array_equal(got, want)
            else:
                assert golden_io.state_rel_err(got, want) <= FAST_TOL
            u, t = want, t + dt
