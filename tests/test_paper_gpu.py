"""The direct BDLTV20 T1/S2 driver (ecg_paper_t1s2_run) against the
reference's own run_bdltv20_paper_t1_s2 (imex/imex_bdltv20_direct_driver.hpp:44-779).

tests/golden/paper_cases.json holds the reference's key=value report for a
short run of every mode (tests/golden/make_golden.py, from the reference
built in oracle/_ref).  The device run reproduces the report: step counts,
guard and failure counts, and pass/fail exactly; the final time, minima and
error norms to GMRES rounding (the pressure solves use the reference's
stopping rule but classical Gram-Schmidt and a matrix-free operator, so the
states agree to about 1e-12 per step, well inside the 1e-8 used here)."""
import json
import os

import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200._lib import EcgError
from amrex_euler_allmach_explicit_imex_b200.config import read_config

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "paper_cases.json")) as f:
    CASES = json.load(f)

P = "bdltv20_paper_"


def _run(kv, arith="exact"):
    s = read_config(kv)
    with api.Context(s.cfg, arith=arith) as ctx:
        r = api.run_bdltv20_paper_t1_s2(ctx, s)
        u = ctx.download()
    return r, u


@pytest.mark.parametrize("name", sorted(CASES))
def test_paper_driver_matches_reference_report(gpu, name):
    case = CASES[name]
    ref = case["report"]
    r, u = _run(case["kv"])
    assert r.steps == int(ref[P + "steps"])
    assert r.final_time == pytest.approx(float(ref[P + "final_time"]), rel=1e-10)
    assert r.solver_failure_count == int(ref[P + "solver_failure_count"])
    assert r.nonfinite_count == int(ref[P + "nonfinite_count"])
    assert r.nonpositive_count == int(ref[P + "nonpositive_count"])
    assert bool(r.passed) == (ref[P + "t1_s2_status"] == "passed")
    assert (r.passed == 1) == (case["rc"] == 0)
    g_ref = int(ref[P + "enthalpy_guard_count"])
    assert abs(r.enthalpy_guard_count - g_ref) <= max(2, 0.01 * g_ref)
    it_ref = int(ref[P + "gmres_iterations_max"])
    assert abs(r.gmres_iterations_max - it_ref) <= max(2, 0.15 * it_ref)
    for f in ("density_l1_error", "velocity_l1_error", "pressure_l1_error", "density_l2_error", "velocity_l2_error",
              "pressure_l2_error", "density_linf_error", "pressure_linf_error", "rho_min", "pressure_min"):
        assert getattr(r, f) == pytest.approx(float(ref[P + f]), rel=1e-8, abs=1e-13), f
    assert r.pressure_residual_linf_max <= max(1e-8, 100 * float(ref[P + "pressure_residual_linf_max"]))


def test_paper_driver_fast_initial_state(gpu):
    """The context's fast arithmetic only changes the initial state's last
    bits (initialize_state with FMA); the driver itself has one build."""
    case = CASES["gresho"]
    r, _ = _run(case["kv"], arith="fast")
    assert r.steps == int(case["report"][P + "steps"])
    assert r.density_l1_error == pytest.approx(float(case["report"][P + "density_l1_error"]), rel=1e-8)


@pytest.mark.parametrize("name,old,new", [("blob", "advection_blob_periodic_2d", "gresho_exact_dirichlet_2d"),
                                          ("gresho", "max_steps=4", "max_steps=0"),
                                          ("vortex", "max_steps=3", "max_steps=3\neuler.bdltv20_paper_t1_s2_dt=0")])
def test_paper_driver_rejects_mismatched_configuration(gpu, name, old, new):
    """The config reader's checks (core/config_reader.hpp:143-250, which abort
    there): a mode on the wrong problem, no steps, a zero fixed dt; BAD_ARG with
    the reference's message, before any launch."""
    s = read_config(CASES[name]["kv"].replace(old, new))
    with api.Context(s.cfg) as ctx:
        with pytest.raises(EcgError, match="requires|must be"):
            api.run_bdltv20_paper_t1_s2(ctx, s)
