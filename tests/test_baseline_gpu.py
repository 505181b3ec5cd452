"""The BASELINE configurations at their own sizes against the reference's own
code (fixtures from tests/golden/make_golden.py, `baseline` and `gresho_l1`).

* One IMEX T1/S2 step (4 Picard passes, GMRES tol 1e-10, 200 iterations) of
  the periodic Gresho vortex on 256^2 at M = 0.1, 0.01 and 0.001, and of the
  shock-density bubble on 640 x 160, from the device's own initial state with
  the reference's dt.  The reference's initial state goes through `log` in
  the Gresho pressure, which CUDA and glibc may round an ulp apart, so the
  states are compared at the IMEX tolerance (1e-9 relative, field families)
  rather than bit for bit.
* One explicit HLLC-P step of the Gresho vortex at 256^2, M = 0.01 (1e-12).
* The density L1 error against the exact Gresho state after whole runs on
  64^2, M = 0.1 (explicit HLLC-P to t = 1, IMEX to t = 0.1), computed from the
  downloaded state by the oracle's restatement of compute_gresho_metrics.
"""
import json
import os

import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu

IMEX_NAMES = ["gresho256_m0p1", "gresho256_m0p01", "gresho256_m0p001", "bubble640x160"]
CONVERGED = (1, 2)  # converged_absolute, converged_relative


def _case(name):
    z = golden_io.load("baseline_cases.npz")
    return {k[len(name) + 1:]: z[k] for k in z.files if k.startswith(name + "_")}


def _imex_step(case, **gpu):
    cfg = read_config(golden_io.kv_of(case["kv"])).cfg
    with api.Context(cfg, **gpu) as ctx:
        api.initialize_state(ctx)
        u0 = ctx.download()
        d = api.euler_imex_bdltv20_o1_source_map_picard_one_step(ctx, float(case["dt"]))
        u1 = ctx.download()
    return cfg, u0, u1, d


@pytest.mark.parametrize("name", IMEX_NAMES)
def test_baseline_imex_fp64_vs_reference(gpu, name):
    c = _case(name)
    cfg, u0, u1, d = _imex_step(c)
    ref_status = int(c["d_solver_status"])
    ref_its = int(c["d_solver_iterations"])
    if ref_status in CONVERGED:
        assert d.solver_status in CONVERGED, api.solver_status_str(d.solver_status)
        assert golden_io.state_rel_err(u1, c["u1"]) <= 1e-9
        # same Krylov method up to rounding (classical Gram-Schmidt with one
        # reorthogonalisation against the reference's modified Gram-Schmidt):
        # the iteration counts of the four solves agree to a few
        assert abs(d.solver_iterations - ref_its) <= max(cfg.imex_picard_iterations, 0.1 * ref_its)
        assert d.picard_pressure_solves_used == int(c["d_picard_pressure_solves_used"])
        for f in ["rho_min", "pressure_min", "solved_pressure_min", "solved_pressure_max",
                  "energy_flux_linf", "momentum_correction_linf"]:
            ref = float(c["d_" + f])
            assert getattr(d, f) == pytest.approx(ref, rel=1e-6, abs=1e-9 * max(1.0, abs(ref))), f
    else:
        # M = 0.001: the reference's GMRES(200) does not reach 1e-10 in the
        # first Picard pass; neither does this one, and the state stays.  The
        # reported iterate is the best one of the 200, whose index rounding
        # may move by a few.
        assert d.solver_status == ref_status, api.solver_status_str(d.solver_status)
        assert ref_its == cfg.imex_solver_max_iter
        assert abs(d.solver_iterations - ref_its) <= cfg.imex_picard_iterations
        assert np.array_equal(u1, u0)
        assert golden_io.state_rel_err(u1, c["u1"]) <= 1e-12
    assert d.pressure_matrix_rows == int(c["d_pressure_matrix_rows"])
    # The stored entries drop coefficients that are exactly zero, such as
    # -xc*(he - hw) where the two face enthalpies are equal: in the uniform
    # parts of these states that equality follows the last bits of the Picard
    # iterate, so the counts agree to 1 % (measured: 0.2 %).
    ref_nnz = int(c["d_pressure_matrix_nonzeros"])
    assert abs(d.pressure_matrix_nonzeros - ref_nnz) <= 0.01 * ref_nnz
    assert abs(d.pressure_matrix_max_row_width - int(c["d_pressure_matrix_max_row_width"])) <= 1


@pytest.mark.parametrize("name", ["gresho256_m0p1", "gresho256_m0p01", "bubble640x160"])
def test_baseline_imex_mixed_vs_reference(gpu, name):
    """The FP32-basis solve applies the reference's stopping rule to the true
    FP64 residual.  Its cycles restart, so it stops at another iterate than
    the reference's unrestarted solve, with a residual under the same 1e-10:
    at M = 0.01 (the worst-conditioned of these systems) the two states lie
    1.4e-9 apart, so the bound here is 3e-9.  (At M = 0.001 the reference's
    solve fails, so there is no state to pin.)"""
    c = _case(name)
    cfg, _, u1, d = _imex_step(c, imex_precision="mixed")
    assert d.solver_status in CONVERGED, api.solver_status_str(d.solver_status)
    assert golden_io.state_rel_err(u1, c["u1"]) <= 3e-9
    assert d.pressure_linear_residual_relative_linf <= cfg.imex_solver_tol or \
        d.pressure_linear_residual_linf <= cfg.imex_solver_tol


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_baseline_explicit_hllcp_vs_reference(gpu, arith):
    c = _case("gresho256_m0p01_hllcp")
    cfg = read_config(golden_io.kv_of(c["kv"])).cfg
    with api.Context(cfg, arith=arith) as ctx:
        api.initialize_state(ctx)
        dt = api.compute_euler_dt(ctx, 0.0)
        deg = api.euler_fv_one_step(ctx, float(c["dt"]), 0.0)
        u1 = ctx.download()
    assert dt == pytest.approx(float(c["dt"]), rel=1e-13)
    assert golden_io.state_rel_err(u1, c["u1"]) <= 1e-12
    assert deg == int(c["deg"])


def _l1_cases():
    with open(os.path.join(golden_io.GOLDEN, "gresho_l1.json")) as f:
        return json.load(f)


# Explicit: exact arithmetic follows the reference step for step (its L1 error
# agrees to 1e-10; the device's initial state may differ from the reference's
# in the last bit of the log in the Gresho pressure).  Fast arithmetic agrees
# to 1e-12 per step, and 2793 steps of a low-Mach flow carry that to 6e-9 of
# the L1 error (measured), so 1e-7.  IMEX: every GMRES solve stops at a
# relative residual below 1e-10 at an iterate that differs from the
# reference's by rounding, so the states agree to about 1e-9 after 32 steps;
# the L1 error is 2e-3, so 1e-6.
L1_RUNS = [("explicit_hllcp", {"arith": "exact"}, 1e-10), ("explicit_hllcp", {"arith": "fast"}, 1e-7),
           ("imex", {"imex_precision": "fp64"}, 1e-6), ("imex", {"imex_precision": "mixed"}, 1e-6)]


@pytest.mark.parametrize("name,gpu_opts,rtol", L1_RUNS,
                         ids=["explicit-exact", "explicit-fast", "imex-fp64", "imex-mixed"])
def test_gresho_density_l1_vs_reference(gpu, oracle, name, gpu_opts, rtol):
    ref = _l1_cases()[name]
    cfg = read_config(ref["kv"]).cfg
    with api.Context(cfg, **gpu_opts) as ctx:
        api.initialize_state(ctx)
        r = api.run(ctx, 100000, float(ref["stop_time"]))
        u = ctx.download()
    assert not r.failed
    assert r.steps == ref["steps"]
    assert r.time == pytest.approx(ref["time"], rel=1e-12)
    l1 = oracle.gresho_density_l1(cfg, u)
    assert l1 == pytest.approx(ref["density_l1_error"], rel=rtol)
