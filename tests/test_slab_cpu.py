"""The slab decomposition's host logic on gloo ranks (CPU): partition,
neighbours, the halo exchange (including two ranks with periodic x, where
both neighbours are one rank) and the dt reduction.

Each rank packs its edge columns, exchanges them through
slab.HaloExchange, and steps its slab extended by the received halo columns
with the CPU oracle. The physical x sides stay physical. The slabs' cells
must equal the oracle's step of the undivided grid bit for bit, and the
reduced dt must equal its compute_euler_dt. The extended slab's halo cells
see the wrong boundary, but no slab cell reads them: the stencil reaches two
cells."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from amrex_euler_allmach_explicit_imex_b200 import slab
from amrex_euler_allmach_explicit_imex_b200.config import read_config

# dx and dy powers of two, so every slab's and extended slab's (hi - lo) / n
# is the undivided grid's cell size exactly
CASES = {
    "toro_outflow": "amr.n_cell=64 8\ngeometry.prob_hi=1 0.125\neuler.problem=toro1\neuler.riemann=hllc\n"
                    "geometry.is_periodic=0 1\n",
    "bubble": "amr.n_cell=64 16\ngeometry.prob_hi=2 0.5\neuler.problem=shock_density_bubble_2d\neuler.riemann=hllc\n",
    "blob_periodic": "amr.n_cell=64 32\ngeometry.prob_hi=1 0.5\ngeometry.is_periodic=1 1\neuler.problem=advection_blob\n"
                     "euler.riemann=xie_am_hllc_p\n",
}


def test_partition_and_neighbours():
    assert [slab.partition(10, 3, r) for r in range(3)] == [(0, 3), (3, 6), (6, 10)]
    assert slab.neighbours(3, 0, False) == (None, 1)
    assert slab.neighbours(3, 2, False) == (1, None)
    assert slab.neighbours(3, 0, True) == (2, 1)
    assert slab.neighbours(2, 1, True) == (0, 0)
    assert slab.neighbours(1, 0, True) == (None, None)
    with pytest.raises(ValueError):
        slab.partition(5, 3, 0)


def _rank(rank, world, port, name, out):
    from tests.oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        oracle = Oracle()
        cfg = read_config(CASES[name]).cfg
        nx, ny = cfg.n_cell[0], cfg.n_cell[1]
        periodic = cfg.is_periodic[0] != 0
        dx = (cfg.prob_hi[0] - cfg.prob_lo[0]) / nx
        rng = np.random.default_rng(5)
        u = oracle.initialize(cfg)
        u = u * (1.0 + 0.01 * rng.standard_normal(u.shape))
        x0, x1 = slab.partition(nx, world, rank)
        left, right = slab.neighbours(world, rank, periodic)
        local = np.ascontiguousarray(u[:, :, x0:x1])
        send_lo = torch.from_numpy(np.ascontiguousarray(local[:, :, :2]).ravel())
        send_hi = torch.from_numpy(np.ascontiguousarray(local[:, :, -2:]).ravel())
        recv_lo = torch.zeros(8 * ny, dtype=torch.float64)
        recv_hi = torch.zeros(8 * ny, dtype=torch.float64)
        slab.HaloExchange(world, rank, periodic).exchange(send_lo, send_hi, recv_lo, recv_hi)

        def sub(a, b, arr):
            c = cfg.copy()
            c.n_cell[0] = arr.shape[2]
            c.prob_lo[0] = cfg.prob_lo[0] + a * dx
            c.prob_hi[0] = cfg.prob_lo[0] + b * dx
            c.is_periodic[0] = cfg.is_periodic[0] if world == 1 else 0
            return c

        # dt: each slab's own, reduced as the minimum
        t = torch.tensor([oracle.euler_dt(sub(x0, x1, local), local, 0.0)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        dt = float(t.item())
        parts, a, b = [], x0, x1
        if left is not None:
            parts.append(recv_lo.numpy().reshape(4, ny, 2))
            a -= 2
        parts.append(local)
        if right is not None:
            parts.append(recv_hi.numpy().reshape(4, ny, 2))
            b += 2
        ext = np.concatenate(parts, axis=2)
        u1, _ = oracle.step(sub(a, b, ext), ext, dt, 0.0)
        off = 2 if left is not None else 0
        mine = u1[:, :, off:off + (x1 - x0)]
        gathered = [None] * world
        dist.all_gather_object(gathered, (x0, mine))
        if rank == 0:
            whole = np.concatenate([m for _, m in sorted(gathered, key=lambda g: g[0])], axis=2)
            ref, _ = oracle.step(cfg, u, dt, 0.0)
            out.put((float(dt), float(oracle.euler_dt(cfg, u, 0.0)), bool(np.array_equal(whole, ref)),
                     float(np.abs(whole - ref).max())))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_slab_step_equals_undivided_step(name, world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    dt, dt_ref, equal, diff = out.get(timeout=10)
    assert dt == dt_ref
    assert equal, diff

