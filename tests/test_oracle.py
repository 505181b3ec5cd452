"""The CPU restatement (oracle/ecg_oracle.cpp) against the reference's own
outputs: golden fixtures generated from the reference code, and the live
reference build (oracle/_ref) where it exists."""
import os

import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import abi
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io


def test_sod_pin(oracle):
    """Sod 400x4, explicit O2 HLLC, CFL 0.5 to t=0.2: the reference takes 553
    steps and reaches L1(rho) = 1.5946047357576687e-3 against the exact
    solution; the oracle reproduces every dt and the final state bit for bit."""
    z = golden_io.load("sod_400x4.npz")
    cfg = read_config(golden_io.kv_of(z["kv"])).cfg
    u0 = oracle.initialize(cfg)
    assert np.array_equal(u0, z["u0"])
    u, t, dts = u0, 0.0, []
    while t < cfg.stop_time - 1e-14:
        dt = oracle.euler_dt(cfg, u, t)
        u, _ = oracle.step(cfg, u, dt, t)
        dts.append(dt)
        t += dt
    assert len(dts) == int(z["steps"]) == 553
    assert np.array_equal(np.array(dts), z["dts"])
    assert np.array_equal(u, z["u_final"])
    ex = np.array([oracle.exact_riemann(x, t, [1, 0, 0, 1], [0.125, 0, 0, 0.1], 1.4, 0.5)[0]
                   for x in (np.arange(400) + 0.5) / 400])
    assert np.array_equal(ex, z["exact_rho"])
    l1 = np.abs(u[0] - ex[None, :]).mean()
    assert l1 == float(z["l1_rho"])
    assert abs(l1 - 1.594604735757667e-3) < 1e-17


def test_sod_run_loop(oracle):
    """ecgo_run_explicit (the driver loop) equals the step-by-step loop."""
    z = golden_io.load("sod_400x4.npz")
    cfg = read_config(golden_io.kv_of(z["kv"])).cfg
    u, r = oracle.run_explicit(cfg, z["u0"], 100000, cfg.stop_time)
    assert r.steps == 553 and not r.failed
    assert np.array_equal(u, z["u_final"])
    assert r.hllc_degenerate_star_count == int(z["degs"].sum())


@pytest.mark.parametrize("key,case", list(golden_io.explicit_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_explicit_case_bitwise(oracle, key, case):
    cfg = read_config(golden_io.kv_of(case["kv"])).cfg
    t, dt = float(case["t"]), float(case["dt"])
    u1, deg = oracle.step(cfg, case["u0"], dt, t)
    assert np.array_equal(u1, case["u1"]), key
    assert deg == int(case["deg"])
    assert np.array_equal(oracle.fill_ghosts(cfg, case["u0"], t), case["ghost"])
    assert oracle.euler_dt(cfg, u1, t) == float(case["edt"])
    d = oracle.diagnostics(cfg, u1)
    assert [d.rho_min, d.pressure_min, d.nonfinite_count] == list(case["diag"])
    a = oracle.admissibility(cfg, u1)
    assert [a.rho_min, a.pressure_min, a.internal_energy_min, a.nonfinite_count, a.density_failure_count,
            a.pressure_failure_count, a.internal_energy_failure_count] == list(case["adm"])
    idt, td = oracle.imex_dt(cfg, u1, t)
    assert [idt, td.material_rate_max, td.acoustic_rate_max] == list(case["imexdt"])


@pytest.mark.parametrize("name", golden_io.IMEX_NAMES)
def test_imex_pieces_bitwise(oracle, name):
    """Star update, pressure system (CSR + rhs) and eq54 momentum are the
    reference's bit for bit; GMRES agrees to rounding."""
    c = golden_io.imex_case(name)
    cfg = read_config(golden_io.kv_of(c["kv"])).cfg
    dt = float(c["dt"])
    star = oracle.imex_star(cfg, c["pu"], dt)
    assert np.array_equal(star, c["pstar"])
    rp, col, val, rhs, nf = oracle.build_system(cfg, c["pstar"], c["pp"], c["pk"], dt)
    assert nf == 0
    assert np.array_equal(rp, c["prp"]) and np.array_equal(col, c["pcol"])
    assert np.array_equal(val, c["pval"]) and np.array_equal(rhs, c["prhs"])
    assert np.array_equal(oracle.corrected_momentum(cfg, c["pstar"], c["pp"], dt), c["pkcorr"])
    g = oracle.gmres_csr(rp, col, val, rhs, c["pp"].ravel(), 200, 1e-10)
    assert g["converged"]
    assert abs(g["iterations"] - int(c["giters"])) <= 1
    assert np.abs(g["x"] - c["gx"]).max() <= 1e-9 * np.abs(c["gx"]).max()


@pytest.mark.parametrize("name", golden_io.IMEX_NAMES)
def test_imex_step_vs_reference(oracle, name):
    """One IMEX T1/S2 step: same solver status and Picard count, GMRES
    iterations within one per Picard solve, state within 1e-9 relative
    (GMRES tolerance 1e-10; iterates differ by rounding)."""
    c = golden_io.imex_case(name)
    cfg = read_config(golden_io.kv_of(c["kv"])).cfg
    u1, d = oracle.imex_step(cfg, c["u0"], float(c["dt"]))
    assert d.solver_status == int(c["d_solver_status"])
    assert d.picard_pressure_solves_used == int(c["d_picard_pressure_solves_used"])
    assert abs(d.solver_iterations - int(c["d_solver_iterations"])) <= cfg.imex_picard_iterations
    assert golden_io.state_rel_err(u1, c["u1"]) <= 1e-9
    assert d.pressure_linear_residual_relative_linf <= cfg.imex_solver_tol


def test_live_reference_random_states(oracle, ref):
    """Fresh random states through the reference build and the oracle."""
    rng = np.random.default_rng(99)
    for riem in ["hllc", "xie_am_hllc_p", "lowmach_hllc", "rusanov"]:
        kv = {"amr.n_cell": "11 6", "euler.riemann": riem, "euler.spatial_order": 2, "geometry.is_periodic": "0 1"}
        cfg = ref.configure(kv)
        rho = rng.uniform(0.3, 2, (6, 11))
        u = rng.uniform(-1, 1, (3, 6, 11))
        st = np.stack([rho, rho * u[0], rho * u[1], rng.uniform(2, 4, (6, 11))])
        dt = 0.4 * ref.euler_dt(st)
        a, na = ref.step(st, dt)
        b, nb = oracle.step(cfg, st, dt)
        assert np.array_equal(a, b) and na == nb


INIT_KV = [
    "euler.problem=toro1\ngeometry.prob_hi=1 0.1\namr.n_cell=37 5\nprob.test=3\n",
    "euler.problem=gresho_vortex\namr.n_cell=33 29\neuler.mach=0.01\n",
    "euler.problem=isentropic_vortex\namr.n_cell=40 24\ngeometry.prob_lo=-5 -5\ngeometry.prob_hi=5 5\n"
    "euler.vortex_center=0 0\n",
    "euler.problem=riemann_quadrant\namr.n_cell=30 30\n",
    "euler.problem=shock_density_bubble_2d\namr.n_cell=160 40\ngeometry.prob_hi=2 0.5\n",
    "euler.problem=advection_blob\namr.n_cell=45 45\n",
]


@pytest.mark.parametrize("kv", INIT_KV, ids=lambda s: s.split("\n")[0].split("=")[1])
def test_oracle_initialize_matches_reference(oracle, ref, kv):
    """The restated initialize_state is bit-identical to the reference's
    (problems/problem_initialization.hpp:420-435) for every problem."""
    cfg = ref.configure(kv)
    assert np.array_equal(oracle.initialize(cfg), ref.initialize())


def test_oracle_mach122_configuration(oracle):
    """The Mach 1.22 shock / bubble configuration (no ProblemKind in the
    reference): Rankine-Hugoniot post-shock state left of x = 0.5, the
    rho = 0.138 bubble at (1, 0.5), reflecting walls at y = 0 and y = 1."""
    cfg = read_config("euler.problem=shock_bubble_mach122\namr.n_cell=64 16\n").cfg
    u = oracle.initialize(cfg)
    g, m = 1.4, 1.22
    rho2 = (g + 1) * m * m / ((g - 1) * m * m + 2)
    p2 = 1 + 2 * g * (m * m - 1) / (g + 1)
    u2 = m * np.sqrt(g) * (1 - 1 / rho2)
    assert u[0, 5, 3] == pytest.approx(rho2, rel=1e-15)          # x = 0.1875 < 0.5
    assert u[1, 5, 3] == pytest.approx(rho2 * u2, rel=1e-15)
    assert u[3, 5, 3] == pytest.approx(p2 / (g - 1) + 0.5 * rho2 * u2 * u2, rel=1e-15)
    assert u[0, 8, 16] == pytest.approx(0.138)                     # (1.03, 0.53): inside the bubble
    assert u[0, 2, 60] == 1.0 and u[3, 2, 60] == pytest.approx(2.5)  # ambient
    # walls: ghost row -1 mirrors row 0, ghost row ny mirrors row ny-1, my negated
    w = np.array(u)
    w[2] = 0.1 + 0.01 * np.arange(64)[None, :] * np.ones((16, 1))
    gh = oracle.fill_ghosts(cfg, w)
    assert np.array_equal(gh[2, 1, 2:-2], -w[2, 0]) and np.array_equal(gh[2, 0, 2:-2], -w[2, 1])
    assert np.array_equal(gh[2, -2, 2:-2], -w[2, -1]) and np.array_equal(gh[2, -1, 2:-2], -w[2, -2])
    assert np.array_equal(gh[0, 2:-2, 0], np.full(16, rho2))      # inflow column


def test_paper_fixture_covers_every_mode():
    """tests/golden/paper_cases.json: one reference run per direct-driver mode."""
    import json
    import os

    with open(os.path.join(os.path.dirname(__file__), "golden", "paper_cases.json")) as f:
        cases = json.load(f)
    modes = {c["report"]["bdltv20_paper_t1_s2"] for c in cases.values()}
    assert modes == set(abi.PAPER_MODE) - {"off"}
    for c in cases.values():
        s = read_config(c["kv"])
        assert s.bdltv20_paper_t1_s2 == c["report"]["bdltv20_paper_t1_s2"]
        assert int(c["report"]["bdltv20_paper_steps"]) >= 3


def test_paper_fixture_reproduces_live_reference(ref):
    """The reference driver, run again here, prints the committed report."""
    import json
    import os

    with open(os.path.join(os.path.dirname(__file__), "golden", "paper_cases.json")) as f:
        cases = json.load(f)
    for name in ("toro_xy", "gresho_eps", "vortex"):
        ref.configure(cases[name]["kv"])
        rc, rep = ref.paper_run()
        assert rc == cases[name]["rc"]
        assert rep == cases[name]["report"], name


def test_output_fixture_is_the_reference_writers(ref, tmp_path):
    """tests/golden/output_cases.npz: the reference's Toro and blob writers,
    run again here, print the committed files."""
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "output_cases.npz"))
    for name in ("toro", "blob"):
        ref.configure(str(d[name + "_kv"]))
        step, time, *trial = d[name + "_meta"]
        p = str(tmp_path / (name + ".csv"))
        ref.write_final_csv(d[name + "_u"], int(step), float(time), p, tuple(trial))
        with open(p) as f:
            assert f.read() == str(d[name + "_csv"])


def _baseline(name):
    z = golden_io.load("baseline_cases.npz")
    return {k[len(name) + 1:]: z[k] for k in z.files if k.startswith(name + "_")}


def test_baseline_explicit_hllcp_fixture_is_the_oracle_step(oracle):
    """The restatement reproduces the reference's explicit HLLC-P step of the
    256^2 Gresho vortex (M = 0.01) bit for bit, from its own initial state."""
    c = _baseline("gresho256_m0p01_hllcp")
    cfg = read_config(golden_io.kv_of(c["kv"])).cfg
    u0 = oracle.initialize(cfg)
    assert oracle.euler_dt(cfg, u0, 0.0) == float(c["dt"])
    u1, deg = oracle.step(cfg, u0, float(c["dt"]), 0.0)
    assert np.array_equal(u1, c["u1"])
    assert deg == int(c["deg"])


def test_baseline_bubble_imex_fixture_vs_oracle(oracle):
    """The restated IMEX step on the 640 x 160 bubble against the reference's
    (GMRES rounding: 1e-9 relative), with the reference's dt."""
    c = _baseline("bubble640x160")
    cfg = read_config(golden_io.kv_of(c["kv"])).cfg
    u0 = oracle.initialize(cfg)
    dt, _ = oracle.imex_dt(cfg, u0)
    assert dt == float(c["dt"])
    u1, d = oracle.imex_step(cfg, u0, dt)
    assert d.solver_status in (1, 2)
    assert golden_io.state_rel_err(u1, c["u1"]) <= 1e-9


def test_gresho_l1_restatement_matches_reference(oracle, ref):
    """compute_gresho_metrics' density L1 error (diagnostic_metrics_timestep.hpp:
    150-225), restated in the oracle, on a perturbed periodic Gresho state."""
    kv = golden_io.load("baseline_cases.npz")["gresho256_m0p1_kv"]
    text = golden_io.kv_of(kv).replace("amr.n_cell=256 256", "amr.n_cell=48 40")
    cfg = ref.configure(text)
    rng = np.random.default_rng(3)
    u = ref.initialize() * (1 + 1e-3 * rng.standard_normal((4, 40, 48)))
    want = ref.gresho_density_l1(u)
    assert want > 0
    assert oracle.gresho_density_l1(cfg, u) == pytest.approx(want, rel=1e-13)
