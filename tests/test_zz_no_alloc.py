"""The allocation-free explicit step, ecg_euler_fv_one_step_noalloc, against
the context entry point ecg_euler_fv_one_step on the same inputs.

Both are called through the C ABI.  The caller's state lives in an AMReX-style
FArrayBox with two ghost cells (lo = (-2, -2)); two calls in a row
(in -> out, then out -> in) must reproduce two context steps: bit-identical in
ECG_ARITH_EXACT, within 1e-12 relative per step in ECG_ARITH_FAST.  The file
name sorts last so the suite also runs it after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

from amrex_euler_allmach_explicit_imex_b200 import _lib, api
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-12
CASES = list(golden_io.explicit_cases())


def _noalloc(cfg, opt, src, dst, nx, ny, dt, t, ghost=2):
    """One call; the Array4 base is the box's lower corner (-ghost, -ghost)
    and the box is (nx + 2 ghost) x (ny + 2 ghost) cells per plane."""
    lib = _lib.load()
    err = C.create_string_buffer(512)
    deg = C.c_int32(-1)
    w, h = nx + 2 * ghost, ny + 2 * ghost
    st = lib.ecg_euler_fv_one_step_noalloc(C.byref(cfg), C.byref(opt), C.c_void_p(src.data_ptr()),
                                           C.c_void_p(dst.data_ptr()), -ghost, -ghost, w, w * h, dt, t,
                                           C.byref(deg), err, len(err))
    return st, deg.value, err.value.decode()


def _fab(torch, u):
    """(4, ny, nx) valid data -> device FArrayBox (4, ny+4, nx+4) with NaN ghosts."""
    _, ny, nx = u.shape
    f = torch.full((4, ny + 4, nx + 4), float("nan"), dtype=torch.float64, device="cuda")
    f[:, 2:ny + 2, 2:nx + 2] = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    return f


def _check(arith, got, want):
    if arith == "exact":
        assert np.array_equal(got, want)
    else:
        assert golden_io.state_rel_err(got, want) <= FAST_TOL


def _two_steps(cfg, u0, dt, t, arith, tile_y=0):
    import torch

    nx, ny = cfg.n_cell[0], cfg.n_cell[1]
    with api.Context(cfg, arith=arith, tile_y=tile_y) as ctx:
        ctx.upload(u0)
        deg1 = api.euler_fv_one_step(ctx, dt, t)
        u1 = ctx.download()
        deg2 = api.euler_fv_one_step(ctx, dt, t + dt)
        u2 = ctx.download()

    a = _fab(torch, u0)
    b = torch.full_like(a, float("nan"))
    opt = api.gpu_options(arith=arith, tile_y=tile_y, stream=torch.cuda.current_stream().cuda_stream)
    st, d1, msg = _noalloc(cfg, opt, a, b, nx, ny, dt, t)
    assert st == 0, msg
    torch.cuda.synchronize()
    _check(arith, b[:, 2:ny + 2, 2:nx + 2].cpu().numpy(), u1)
    assert d1 == deg1
    st, d2, msg = _noalloc(cfg, opt, b, a, nx, ny, dt, t + dt)
    assert st == 0, msg
    torch.cuda.synchronize()
    _check(arith, a[:, 2:ny + 2, 2:nx + 2].cpu().numpy(), u2)
    assert d2 == deg2
    # the caller's ghost cells are never written
    assert torch.isnan(a[:, :2]).all() and torch.isnan(b[:, :, -2:]).all()
    return u1


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("key,case", CASES[:8], ids=[k for k, _ in CASES[:8]])
def test_noalloc_matches_golden(gpu, arith, key, case):
    """The first call against the reference's own step (the golden u1)
    directly: bit-identical in exact arithmetic, 1e-12 in fast."""
    import torch

    cfg = read_config(golden_io.kv_of(case["kv"])).cfg
    nx, ny = cfg.n_cell[0], cfg.n_cell[1]
    a = _fab(torch, case["u0"])
    b = torch.full_like(a, float("nan"))
    opt = api.gpu_options(arith=arith, stream=torch.cuda.current_stream().cuda_stream)
    st, deg, msg = _noalloc(cfg, opt, a, b, nx, ny, float(case["dt"]), float(case["t"]))
    assert st == 0, msg
    torch.cuda.synchronize()
    _check(arith, b[:, 2:ny + 2, 2:nx + 2].cpu().numpy(), case["u1"])
    assert deg == int(case["deg"])


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("key,case", CASES, ids=[k for k, _ in CASES])
def test_noalloc_matches_context_step(gpu, arith, key, case):
    cfg = read_config(golden_io.kv_of(case["kv"])).cfg
    _two_steps(cfg, case["u0"], float(case["dt"]), float(case["t"]), arith)


def _random_state(nx, ny, seed):
    rng = np.random.default_rng(seed)
    rho = rng.uniform(1.0, 2.0, (ny, nx))
    u = rng.uniform(-0.5, 0.5, (ny, nx))
    v = rng.uniform(-0.5, 0.5, (ny, nx))
    p = rng.uniform(1.0, 2.0, (ny, nx))
    return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])


def _kv(problem, riemann, nx, ny):
    hi = "2 0.5" if problem.startswith("shock") else "1 0.6"
    return (f"amr.n_cell={nx} {ny}\neuler.problem={problem}\neuler.riemann={riemann}\n"
            "euler.spatial_order=2\neuler.field_boundary=exact_dirichlet\ngeometry.is_periodic=0 0\n"
            f"geometry.prob_hi={hi}\n")


PROBLEMS = [("gresho_vortex", "hllc"), ("toro1", "xie_am_hllc_p"), ("shock_density_bubble_2d", "hllc"),
            ("advection_blob", "lowmach_hllc")]


# tile_y selects the explicit kernel: 0 column strips with paired faces and
# rows staged through shared memory, 3 the same with rows loaded into
# registers, 2 column strips with faces one at a time, 1 square 16x16 tiles, 8
# the 32x8 tiles
@pytest.mark.parametrize("tile_y", [0, 1, 2, 3, 8])
@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("problem,riemann", PROBLEMS)
def test_noalloc_larger_grid(gpu, arith, problem, riemann, tile_y):
    """A 200 x 120 grid: strips and tiles that overhang the domain, the
    exact-Dirichlet ghost ring in the static scratch, every kernel the entry
    point can select, reading and writing with the caller's strides."""
    cfg = read_config(_kv(problem, riemann, 200, 120)).cfg
    _two_steps(cfg, _random_state(200, 120, 5), 2.0e-4, 0.01, arith, tile_y)


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("problem,riemann", [("shock_density_bubble_2d", "hllc"), ("toro1", "xie_am_hllc_p")])
def test_noalloc_tight_layout(gpu, arith, problem, riemann):
    """A caller box with no ghost cells and no padding (lo = (0, 0),
    jstride = nx, nstride = nx ny) on an odd 201 x 119 grid, between guard
    values: every write lands inside the box and matches the context step."""
    import torch

    nx, ny = 201, 119
    cfg = read_config(_kv(problem, riemann, nx, ny)).cfg
    u0 = _random_state(nx, ny, 11)
    dt, t = 2.0e-4, 0.01
    with api.Context(cfg, arith=arith) as ctx:
        ctx.upload(u0)
        api.euler_fv_one_step(ctx, dt, t)
        want = ctx.download()
    guard = 4096
    n = 4 * nx * ny
    src = torch.full((n + 2 * guard,), 7.5, dtype=torch.float64, device="cuda")
    dst = torch.full((n + 2 * guard,), -3.25, dtype=torch.float64, device="cuda")
    src[guard:guard + n] = torch.from_numpy(u0.reshape(-1)).cuda()
    opt = api.gpu_options(arith=arith, stream=torch.cuda.current_stream().cuda_stream)
    st, _, msg = _noalloc(cfg, opt, src[guard:], dst[guard:], nx, ny, dt, t, ghost=0)
    assert st == 0, msg
    torch.cuda.synchronize()
    got = dst[guard:guard + n].cpu().numpy().reshape(4, ny, nx)
    _check(arith, got, want)
    assert (dst[:guard] == -3.25).all() and (dst[guard + n:] == -3.25).all()
    assert torch.equal(src[guard:guard + n].cpu(), torch.from_numpy(u0.reshape(-1)))


def test_noalloc_rejects_ring_beyond_scratch(gpu):
    import torch

    kv = "amr.n_cell=2048 300\neuler.problem=toro1\neuler.field_boundary=exact_dirichlet\ngeometry.is_periodic=0 0\n"
    cfg = read_config(kv).cfg
    a = torch.zeros(16, dtype=torch.float64, device="cuda")
    b = torch.zeros(16, dtype=torch.float64, device="cuda")
    opt = api.gpu_options()
    lib = _lib.load()
    err = C.create_string_buffer(512)
    st = lib.ecg_euler_fv_one_step_noalloc(C.byref(cfg), C.byref(opt), C.c_void_p(a.data_ptr()),
                                           C.c_void_p(b.data_ptr()), 0, 0, 2048, 2048 * 300, 1e-4, 0.0, None, err,
                                           len(err))
    assert st == 1  # ECG_ERR_BAD_ARG, before any launch
    assert "exceeds" in err.value.decode()
    st = lib.ecg_euler_fv_one_step_noalloc(C.byref(cfg), C.byref(opt), C.c_void_p(a.data_ptr()),
                                           C.c_void_p(a.data_ptr()), 0, 0, 2048, 2048 * 300, 1e-4, 0.0, None, err,
                                           len(err))
    assert st == 1


def test_noalloc_rejects_overlapping_arrays(gpu):
    """state_out starting inside state_in (or the reverse) would let the step
    overwrite cells it still has to read: rejected before any launch."""
    import torch

    nx, ny = 64, 32
    cfg = read_config(_kv("shock_density_bubble_2d", "hllc", nx, ny)).cfg
    n = 4 * nx * ny
    buf = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    lib = _lib.load()
    opt = api.gpu_options()
    err = C.create_string_buffer(512)
    base = buf.data_ptr()
    for src, dst in [(base, base + 8 * nx * ny), (base + 8 * (n - 1), base), (base, base + 8 * n)]:
        st = lib.ecg_euler_fv_one_step_noalloc(C.byref(cfg), C.byref(opt), C.c_void_p(src), C.c_void_p(dst), 0, 0,
                                               nx, nx * ny, 1e-4, 0.0, None, err, len(err))
        if dst - src >= 8 * n or src - dst >= 8 * n:
            assert st == 0, err.value.decode()  # adjacent, disjoint arrays
        else:
            assert st == 1 and "overlap" in err.value.decode()
    torch.cuda.synchronize()
