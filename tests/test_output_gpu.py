"""Output writers (io/output_cases.hpp) against the reference's own writers.

tests/golden/output_cases.npz holds, for seeded states, the files the
reference writes (tests/golden/make_golden.py, oracle/_ref): the Gresho (explicit
and IMEX), Toro, Riemann-quadrant and advection-blob final CSVs, and the
shock-density-bubble snapshot, metrics and summary.  Our files must have the
same header, row count and string columns; numbers are printed with %.17g
from columns computed on the device in the reference's arithmetic, so they
are the same text except where an exact state goes through log or exp (one
ulp) or a sum runs in another order (the bubble's area and centroid)."""
import json
import os

import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200.config import read_config

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "output_cases.npz"))
FINAL = ["gresho_explicit", "gresho_imex", "toro", "quadrant", "blob"]
REL = 1e-14


def compare_csv(ours, ref, rel=REL):
    """Same header, rows and string fields; numbers within rel.  Returns the
    fraction of fields that are the same text."""
    a, b = ours.splitlines(), ref.splitlines()
    assert len(a) == len(b)
    assert a[0] == b[0]
    same = total = 0
    for la, lb in zip(a[1:], b[1:]):
        ta, tb = la.split(","), lb.split(",")
        assert len(ta) == len(tb), (la, lb)
        for x, y in zip(ta, tb):
            total += 1
            if x == y:
                same += 1
                continue
            fx, fy = float(x), float(y)  # a differing string field raises here
            assert abs(fx - fy) <= rel * max(abs(fx), abs(fy), 1.0), (x, y, la)
    return same / max(total, 1)


@pytest.mark.parametrize("name", FINAL)
def test_final_csv_matches_reference_writer(gpu, name, tmp_path):
    cfg = read_config(str(G[name + "_kv"])).cfg
    step, time, *trial = G[name + "_meta"]
    with api.Context(cfg, arith="exact") as ctx:
        ctx.upload(G[name + "_u"])
        path = tmp_path / (name + ".csv")
        api.write_final_csv(ctx, str(path), int(step), float(time), trial)
    same = compare_csv(path.read_text(), str(G[name + "_csv"]))
    # the Gresho exact pressure goes through log; everything else is the same text
    assert same >= (0.9 if name.startswith("gresho") else 1.0), same


def _bubble():
    cfg = read_config(str(G["bubble_kv"])).cfg
    return cfg, G["bubble_u"], json.loads(str(G["bubble_run"]))


def test_bubble_snapshot_matches_reference_writer(gpu, tmp_path):
    cfg, u, b = _bubble()
    with api.Context(cfg, arith="exact") as ctx:
        ctx.upload(u)
        api.write_bubble_snapshot(ctx, str(tmp_path), b["index"], b["step"], b["time"])
    files = os.listdir(tmp_path)
    assert files == [str(G["bubble_snapshot_name"])]
    assert compare_csv((tmp_path / files[0]).read_text(), str(G["bubble_snapshot_csv"])) == 1.0


def test_bubble_snapshot_async_keeps_the_state_of_the_call(gpu, tmp_path):
    """The asynchronous writer copies the columns on a side stream and formats
    them on a host thread: the caller steps on meanwhile, and the file still
    holds the state at the call."""
    cfg, u, b = _bubble()
    with api.Context(cfg, arith="exact") as ctx:
        ctx.upload(u)
        api.write_bubble_snapshot(ctx, str(tmp_path / "a"), b["index"], b["step"], b["time"], asynchronous=True)
        t = b["time"]
        for k in range(3):
            dt = api.compute_euler_dt(ctx, t)
            api.euler_fv_one_step(ctx, dt, t)
            t += dt
            api.write_bubble_snapshot(ctx, str(tmp_path / "b"), b["index"] + 1 + k, b["step"] + 1 + k, t,
                                      asynchronous=True)
        api.output_wait(ctx)
    first = tmp_path / "a" / str(G["bubble_snapshot_name"])
    assert compare_csv(first.read_text(), str(G["bubble_snapshot_csv"])) == 1.0
    assert len(os.listdir(tmp_path / "b")) == 3


def test_bubble_metrics_match_reference(gpu):
    cfg, u, b = _bubble()
    with api.Context(cfg, arith="exact") as ctx:
        ctx.upload(u)
        m = api.shock_bubble_metrics(ctx, b["time"])
    ref = G["bubble_metrics"]
    got = [m.rho_min, m.rho_max, m.pressure_min, m.pressure_max, m.internal_energy_min, m.density_bubble_centroid_x,
           m.density_bubble_centroid_y, m.density_bubble_area, m.schlieren_max]
    # extrema are exact; the area and centroid sums run in another order
    np.testing.assert_array_equal(got[:5], ref[:5])
    np.testing.assert_allclose(got[5:8], ref[5:8], rtol=1e-13)
    assert got[8] == ref[8]
    assert m.nonfinite_count == int(G["bubble_nonfinite"])
    assert m.density_bubble_area_threshold == 0.55


def test_bubble_summary_matches_reference_writer(gpu, tmp_path):
    cfg, u, b = _bubble()
    with api.Context(cfg, arith="exact") as ctx:
        ctx.upload(u)
        path = tmp_path / "summary.csv"
        api.write_bubble_summary_csv(ctx, str(path), b["step"], b["time"], status=b["status"],
                                     failure_category=b["failure"], steps_rejected=b["rejected"],
                                     wall_time_sec=b["wall"], dt_min=b["dt_min"], dt_max=b["dt_max"],
                                     dt_mean=b["dt_mean"], snapshot_status=b["snapshot_status"],
                                     snapshot_dir=b["snapshot_dir"], snapshot_times=b["snapshot_times"])
    # the quoted snapshot_times field splits the same way in both files
    compare_csv(path.read_text(), str(G["bubble_summary_csv"]), rel=1e-13)


def test_writers_reject_other_problems(gpu, tmp_path):
    cfg, u, _ = _bubble()
    with api.Context(cfg) as ctx:
        ctx.upload(u)
        with pytest.raises(api.EcgError):
            api.write_final_csv(ctx, str(tmp_path / "x.csv"), 0, 0.0)
    gcfg = read_config(str(G["toro_kv"])).cfg
    with api.Context(gcfg) as ctx:
        ctx.upload(G["toro_u"])
        with pytest.raises(api.EcgError):
            api.write_bubble_snapshot(ctx, str(tmp_path), 0, 0, 0.0)
        with pytest.raises(api.EcgError):
            api.shock_bubble_metrics(ctx)
