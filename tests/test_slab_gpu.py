"""Slab contexts (ecg_create_slab) on one GPU against the undivided grid.

The grid is split into 2 or 3 slab contexts in one process. Each step packs
every slab's edge columns (ecg_slab_pack), copies them into the neighbours'
halo blocks (the exchange NCCL does between GPUs), and steps every slab. No
kernel waits on another, since the copies are ordered on one stream.
dt is the minimum of the slabs' dt, and the degenerate count is the sum.

Against the whole-grid context: exact arithmetic is bit-identical.
Fast arithmetic agrees to 1e-12 per step: the column strips of a slab start
at its own first column, and a strip-edge face goes through the one-face
flux."""
import numpy as np
import pytest
import torch

from amrex_euler_allmach_explicit_imex_b200 import api, slab
from amrex_euler_allmach_explicit_imex_b200.config import read_config
from tests import golden_io

pytestmark = pytest.mark.gpu

CASES = {
    "bubble": "amr.n_cell=256 64\ngeometry.prob_hi=2 0.5\neuler.problem=shock_density_bubble_2d\neuler.riemann=hllc\n",
    "toro_periodic_y": "amr.n_cell=200 40\ngeometry.prob_hi=1 0.2\neuler.problem=toro1\neuler.riemann=lowmach_hllc\n"
                       "geometry.is_periodic=0 1\n",
    "gresho_periodic": "amr.n_cell=96 96\ngeometry.is_periodic=1 1\neuler.problem=gresho_vortex\n"
                       "euler.vortex_center=0.5 0.5\neuler.riemann=hllc\n",
    "blob_hllcp": "amr.n_cell=96 64\ngeometry.prob_hi=1 0.6666666666666666\ngeometry.is_periodic=1 1\n"
                  "euler.problem=advection_blob\neuler.riemann=xie_am_hllc_p\n",
}
SPLITS = [("bubble", 2), ("bubble", 3), ("toro_periodic_y", 3), ("gresho_periodic", 2), ("blob_hllcp", 3)]


def _whole(cfg, arith, stream, steps):
    with api.Context(cfg, arith=arith, stream=stream.cuda_stream) as ctx:
        api.initialize_state(ctx)
        u0 = ctx.download()
        t, out = 0.0, []
        for _ in range(steps):
            dt = api.compute_euler_dt(ctx, t)
            deg = api.euler_fv_one_step(ctx, dt, t)
            out.append((dt, deg, ctx.download()))
            t += dt
    return u0, out


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("name,nslab", SPLITS)
def test_slabs_on_one_gpu_match_the_whole_grid(gpu, name, nslab, arith):
    cfg = read_config(CASES[name]).cfg
    nx, ny = cfg.n_cell[0], cfg.n_cell[1]
    periodic = cfg.is_periodic[0] != 0
    stream = torch.cuda.current_stream()
    u0, want = _whole(cfg, arith, stream, 3)
    parts = []
    for r in range(nslab):
        x0, x1 = slab.partition(nx, nslab, r)
        left, right = slab.neighbours(nslab, r, periodic)
        ctx = api.Context(cfg, slab=(x0, x1, left is not None, right is not None), arith=arith,
                          stream=stream.cuda_stream)
        b = {k: torch.zeros(8 * ny, dtype=torch.float64, device="cuda") for k in ("send_lo", "send_hi", "lo", "hi")}
        ctx.bind_halo(b["lo"] if left is not None else None, b["hi"] if right is not None else None)
        ctx.upload(np.ascontiguousarray(u0[:, :, x0:x1]))
        parts.append((ctx, left, right, b))
    try:
        t = 0.0
        for k, (dt_ref, deg_ref, u_ref) in enumerate(want):
            dt = min(api.compute_euler_dt(ctx, t) for ctx, *_ in parts)
            assert dt == dt_ref
            for ctx, _, _, b in parts:
                ctx.pack(b["send_lo"], b["send_hi"])
            for ctx, left, right, b in parts:
                if left is not None:
                    b["lo"].copy_(parts[left][3]["send_hi"])
                if right is not None:
                    b["hi"].copy_(parts[right][3]["send_lo"])
            deg = sum(api.euler_fv_one_step(ctx, dt, t) for ctx, *_ in parts)
            got = np.concatenate([ctx.download() for ctx, *_ in parts], axis=2)
            if arith == "exact":
                assert np.array_equal(got, u_ref)
                assert deg == deg_ref
            else:
                assert golden_io.state_rel_err(got, u_ref) <= 1e-12 * (k + 1)
                assert abs(deg - deg_ref) <= 2
            t += dt
    finally:
        for ctx, *_ in parts:
            ctx.close()


def test_slab_refuses_what_needs_the_whole_grid(gpu):
    imex = read_config("amr.n_cell=64 64\ngeometry.is_periodic=1 1\neuler.problem=gresho_vortex\n"
                       "euler.vortex_center=0.5 0.5\neuler.method=imex\neuler.spatial_order=2\n"
                       "euler.imex_acoustic_startup=0\n").cfg
    with pytest.raises(api.EcgError):
        api.Context(imex, slab=(0, 32, True, True))
    ring = read_config("amr.n_cell=64 8\neuler.problem=toro1\neuler.field_boundary=exact_dirichlet\n"
                       "geometry.is_periodic=0 0\n").cfg
    with pytest.raises(api.EcgError):
        api.Context(ring, slab=(0, 32, False, True))
    cfg = read_config(CASES["bubble"]).cfg
    with api.Context(cfg, slab=(0, 128, False, True)) as ctx:
        api.initialize_state(ctx)
        with pytest.raises(api.EcgError):
            api.run(ctx, 2, 1.0)
    with pytest.raises(api.EcgError):
        api.Context(cfg, slab=(10, 11, True, True))  # a slab of one column


def test_slab_initial_state_is_its_part_of_the_grid(gpu):
    """initialize_state of a slab writes its columns of the whole grid's state
    (coordinates from the slab's origin and the grid's dx)."""
    cfg = read_config(CASES["bubble"]).cfg
    with api.Context(cfg, arith="exact") as ctx:
        api.initialize_state(ctx)
        whole = ctx.download()
    with api.Context(cfg, slab=(96, 192, True, True), arith="exact") as ctx:
        api.initialize_state(ctx)
        part = ctx.download()
    np.testing.assert_allclose(part, whole[:, :, 96:192], rtol=1e-15, atol=0)


def _solver_rank(rank, world, port, u0, out):
    """One rank of a gloo group; every rank on cuda:0 (the host moves the
    halos, so no kernel waits on another rank's)."""
    import os

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        cfg = read_config(CASES["gresho_periodic"]).cfg
        s = slab.SlabSolver(cfg, arith="exact")
        s.scatter(u0)
        t, dts, degs = 0.0, [], []
        for _ in range(3):
            dt = s.compute_euler_dt(t)
            degs.append(s.euler_fv_one_step(dt, t))
            dts.append(dt)
            t += dt
        u = s.gather()
        s.close()
        if rank == 0:
            out.put((dts, degs, u))
    finally:
        dist.destroy_process_group()


def test_slab_solver_over_a_gloo_group(gpu):
    """SlabSolver end to end (partition, binding, pack, exchange, dt and count
    reductions, gather) with two gloo ranks sharing one GPU, against the
    whole grid in exact arithmetic."""
    import socket

    import torch.multiprocessing as mp

    cfg = read_config(CASES["gresho_periodic"]).cfg
    u0, want = _whole(cfg, "exact", torch.cuda.current_stream(), 3)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_solver_rank, args=(r, 2, port, u0, out)) for r in range(2)]
    for p in procs:
        p.start()
    dts, degs, u = out.get(timeout=300)
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs)
    assert dts == [w[0] for w in want]
    assert degs == [w[1] for w in want]
    assert np.array_equal(u, want[-1][2])
