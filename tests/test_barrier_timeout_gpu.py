"""The bounded wait of the GMRES grid barrier, the only device-side wait of
the path: a block that never arrives makes the others' wait run out after
spin_limit polls, the kernel reports it, and the device stays usable.  No
fault, trap or hang is involved: the missing arrival is the block returning
early, and every wait is bounded."""
import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_reports(gpu):
    first, out = api.check_grid_barrier_timeout(spin_limit=4096)
    assert first == 4  # every block passed the barrier all of them reached
    assert out == 3    # the three blocks left waiting for block 0 gave up


def test_device_usable_after_a_timed_out_barrier(gpu):
    api.check_grid_barrier_timeout(spin_limit=1024)
    c = golden_io.imex_case("gresho_m0p1")
    cfg = read_config(golden_io.kv_of(c["kv"])).cfg
    with api.Context(cfg) as ctx:
        ctx.upload(c["u0"])
        d = api.euler_imex_bdltv20_o1_source_map_picard_one_step(ctx, float(c["dt"]))
        u1 = ctx.download()
    assert d.solver_status in (1, 2)
    assert golden_io.state_rel_err(u1, c["u1"]) <= 1e-9


def test_barrier_check_rejects_unbounded_limits(gpu):
    for bad in (0, -1, (1 << 25) + 1):
        with pytest.raises(api.EcgError):
            api.check_grid_barrier_timeout(spin_limit=bad)


def test_barrier_check_rejects_a_missing_device(gpu):
    with pytest.raises(api.EcgError):
        api.check_grid_barrier_timeout(device=1 << 20)
