"""ecg_euler_fv_one_step_host: the upload, step and download of a host state
in one call, pipelined over row bands, against the device-resident step on
the same state.  Band edges are strip edges of the column-strip kernel, whose
y-faces there go through the one-face flux: fast arithmetic agrees to 1e-12
per step, as between any two strip partitions."""
import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu

CASES = {
    "bubble": "amr.n_cell=320 80\ngeometry.prob_hi=2 0.5\neuler.problem=shock_density_bubble_2d\neuler.riemann=hllc\n",
    "toro_periodic_y": "amr.n_cell=200 96\ngeometry.prob_hi=1 0.48\neuler.problem=toro1\neuler.riemann=lowmach_hllc\n"
                       "geometry.is_periodic=0 1\n",
    "gresho_hllcp": "amr.n_cell=96 96\ngeometry.is_periodic=1 1\neuler.problem=gresho_vortex\neuler.vortex_center=0.5 0.5\n"
                    "euler.riemann=xie_am_hllc_p\n",
    # HLLC-P on a grid whose device step takes the strips as well: the host
    # step's bands run on the strips with the sensor carried across band edges
    "bubble_hllcp": "amr.n_cell=1280 320\ngeometry.prob_hi=2 0.5\neuler.problem=shock_density_bubble_2d\n"
                    "euler.riemann=xie_am_hllc_p\n",
}


@pytest.mark.parametrize("arith", ["fast", "exact"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_host_step_matches_device_step(gpu, name, arith):
    cfg = read_config(CASES[name]).cfg
    with api.Context(cfg, arith=arith) as ctx:
        api.initialize_state(ctx)
        u0 = ctx.download()
        t, states, degs = 0.0, [], []
        for _ in range(3):
            dt = api.compute_euler_dt(ctx, t)
            degs.append(api.euler_fv_one_step(ctx, dt, t))
            states.append(ctx.download())
            t += dt
    with api.Context(cfg, arith=arith) as ctx:
        a = np.ascontiguousarray(u0)
        b = np.empty_like(a)
        ctx.upload(a)
        t = 0.0
        for k in range(3):
            dt = api.compute_euler_dt(ctx, t)  # the fused reduction of the previous host step
            deg = api.euler_fv_one_step_host(ctx, a, b, dt, t)
            tol = 0.0 if arith == "exact" else 1e-12 * (k + 1)
            assert golden_io.state_rel_err(b, states[k]) <= tol
            assert abs(deg - degs[k]) <= (0 if arith == "exact" else 2)
            np.testing.assert_array_equal(ctx.download(), b)
            a, b = b, a
            t += dt


def test_host_step_in_place(gpu):
    cfg = read_config(CASES["bubble"]).cfg
    with api.Context(cfg) as ctx:
        api.initialize_state(ctx)
        u = np.ascontiguousarray(ctx.download())
        ref = u.copy()
        dt = api.compute_euler_dt(ctx)
        api.euler_fv_one_step(ctx, dt)
        want = ctx.download()
        ctx.upload(ref)
        api.euler_fv_one_step_host(ctx, u, u, dt)
        assert golden_io.state_rel_err(u, want) <= 1e-12


def _pinned(shape):
    import torch

    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


def _padded(u, g, extra):
    """u inside a ghost-padded box: lo = -g, rows nx + 2g + extra long,
    planes one row apart more than the box needs."""
    _, ny, nx = u.shape
    js = nx + 2 * g + extra
    ns = js * (ny + 2 * g + 1)
    buf = np.full(4 * ns, np.nan)
    box = np.lib.stride_tricks.as_strided(buf[g * js + g:], shape=u.shape, strides=(8 * ns, 8 * js, 8))
    box[...] = u
    return buf, box, js, ns


@pytest.mark.parametrize("name", ["bubble", "toro_periodic_y"])
def test_pageable_boxes_cross_like_pinned_ones(gpu, name):
    """Pageable host boxes go through the library's pinned stage in bands of
    rows; the bits that cross are those of a pinned box, and a ghost-padded
    Array4 box (lo = -2, padded rows and planes) keeps its ghosts."""
    from amrex_euler_allmach_explicit_imex_b200._lib import check, load

    lib = load()
    cfg = read_config(CASES[name]).cfg
    with api.Context(cfg) as ctx:
        api.initialize_state(ctx)
        u0 = ctx.download(_pinned((4, ctx.ny, ctx.nx)))
        dt = api.compute_euler_dt(ctx)
        pin_out = _pinned(u0.shape)
        api.euler_fv_one_step_host(ctx, u0, pin_out, dt)
        page_out = np.empty_like(u0)
        api.euler_fv_one_step_host(ctx, np.array(u0), page_out, dt)
        np.testing.assert_array_equal(page_out, pin_out)
        # a padded pageable box: upload, host step in place, download
        g = 2
        buf, box, js, ns = _padded(u0, g, 3)
        base = buf.ctypes.data  # the Array4 base: cell (lo_x, lo_y)
        check(lib.ecg_upload_state(ctx.handle, base, -g, -g, js, ns), "upload", ctx.handle)
        np.testing.assert_array_equal(ctx.download(), u0)
        check(lib.ecg_euler_fv_one_step_host(ctx.handle, base, base, -g, -g, js, ns, dt, 0.0, None), "host step",
              ctx.handle)
        np.testing.assert_array_equal(box, pin_out)
        box[...] = 0.0
        check(lib.ecg_download_state(ctx.handle, base, -g, -g, js, ns), "download", ctx.handle)
        np.testing.assert_array_equal(box, pin_out)
        # the ghosts and the row and plane padding are untouched
        inside = np.zeros(buf.size, dtype=bool)
        np.lib.stride_tricks.as_strided(inside[g * js + g:], shape=u0.shape, strides=(ns, js, 1))[...] = True
        assert np.isnan(buf[~inside]).all()


# A periodic-y grid whose bands are large enough that the last upload chunk
# lands well after the first band's step could start.
WRAP_Y = ("amr.n_cell=1280 320\ngeometry.prob_hi=4 1\ngeometry.is_periodic=1 1\neuler.problem=gresho_vortex\n"
          "euler.vortex_center=0.5 0.5\neuler.riemann=hllc\n")


@pytest.mark.parametrize("memory", ["pinned", "pageable"])
def test_host_step_reads_only_the_host_state(gpu, memory):
    """Nothing the device buffer held before a host step reaches its result:
    before each call the context holds a decoy (the host state rolled by half
    the grid in y).  Under periodic y the first band's ghost rows are the
    grid's last two rows; they must cross before that band is stepped."""
    cfg = read_config(WRAP_Y).cfg
    with api.Context(cfg) as ctx:
        api.initialize_state(ctx)
        u0 = ctx.download()
        t, dts, states = 0.0, [], []
        for _ in range(3):
            dt = api.compute_euler_dt(ctx, t)
            api.euler_fv_one_step(ctx, dt, t)
            dts.append(dt)
            states.append(ctx.download())
            t += dt
    with api.Context(cfg) as ctx:
        if memory == "pinned":
            a, b = _pinned(u0.shape), _pinned(u0.shape)
            a[...] = u0
        else:
            a, b = np.ascontiguousarray(u0), np.empty_like(u0)
        t = 0.0
        for k in range(3):
            ctx.upload(np.ascontiguousarray(np.roll(a, a.shape[1] // 2, axis=1)))
            api.euler_fv_one_step_host(ctx, a, b, dts[k], t)
            assert golden_io.state_rel_err(b, states[k]) <= 1e-12 * (k + 1)
            np.testing.assert_array_equal(ctx.download(), b)
            a, b = b, a
            t += dts[k]
