"""One grid's explicit steps split over the ranks of a torch.distributed
group as slabs along x.

Each rank holds columns [x0, x1) in a slab context (ecg_create_slab), whose
inner x sides take their two ghost columns from the neighbour slabs. Each
step:
1. packs the slab's two edge columns on each side (ecg_slab_pack);
2. swaps them with the neighbours by send/recv: NCCL between GPUs, any
   backend for the host logic;
3. steps the slab, which reads the received halo blocks in place.

The CFL dt is the minimum over ranks of each slab's dt. This equals the
whole grid's dt bit for bit: dt = cfl / max rate is monotone, and the max is
exact. The degenerate-star count is the sum over ranks: a face between two
slabs is counted once by each side's cell, as in the undivided grid.

No counterpart in the reference: it runs one box in one process, and its
IMEX path requires NProcs() == 1. The IMEX pressure system couples the whole
grid, so slabs run the explicit method only."""
import numpy as np
import torch
import torch.distributed as dist

from . import api

TAG_LO = 11  # a slab's low edge columns, to its left neighbour
TAG_HI = 12  # its high edge columns, to its right neighbour


def partition(nx, world, rank):
    """Columns [x0, x1) of `rank`: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the group")
    if nx < 2 * world:
        raise ValueError(f"{nx} columns cannot give {world} slabs of at least two columns")
    return nx * rank // world, nx * (rank + 1) // world


def neighbours(world, rank, periodic_x):
    """(left, right) neighbour ranks, None at a physical x boundary; a single
    rank has none (its periodic wrap stays inside its context)."""
    if world == 1:
        return None, None
    left = rank - 1 if rank > 0 else (world - 1 if periodic_x else None)
    right = rank + 1 if rank < world - 1 else (0 if periodic_x else None)
    return left, right


class HaloExchange:
    """Swaps edge columns with the x-neighbours.  Sends go out in the order
    (low edge to the left, high edge to the right) and receives are posted as
    (high halo from the right, low halo from the left).  Backends that match
    messages per peer in order (NCCL) then pair them correctly, including
    when both neighbours are one rank (two ranks, periodic x).  Tags pair them
    on backends that use tags."""

    def __init__(self, world, rank, periodic_x, group=None):
        self.left, self.right = neighbours(world, rank, periodic_x)
        self.group = group
        self.nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"

    def exchange(self, send_lo, send_hi, recv_lo, recv_hi):
        if self.left is None and self.right is None:
            return
        ops = []
        if self.left is not None:
            ops.append((dist.isend, send_lo, self.left, TAG_LO))
        if self.right is not None:
            ops.append((dist.isend, send_hi, self.right, TAG_HI))
        if self.right is not None:
            ops.append((dist.irecv, recv_hi, self.right, TAG_LO))
        if self.left is not None:
            ops.append((dist.irecv, recv_lo, self.left, TAG_HI))
        if self.nccl:
            reqs = dist.batch_isend_irecv([dist.P2POp(op, t, peer, self.group, tag) for op, t, peer, tag in ops])
            for r in reqs:
                r.wait()
            return
        # host backends move host tensors: device blocks go through host copies
        staged = [(op, t.cpu() if t.is_cuda else t, t, peer, tag) for op, t, peer, tag in ops]
        reqs = [op(h, peer, group=self.group, tag=tag) for op, h, _, peer, tag in staged]
        for r in reqs:
            r.wait()
        for op, h, t, _, _ in staged:
            if op is dist.irecv and t.is_cuda:
                t.copy_(h)


class SlabSolver:
    """The explicit step of one grid, split over the group's ranks (one GPU
    each).  cfg: the whole grid's run configuration."""

    def __init__(self, cfg, group=None, device=None, **gpu):
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        nx, ny = cfg.n_cell[0], cfg.n_cell[1]
        periodic = cfg.is_periodic[0] != 0
        self.x0, self.x1 = partition(nx, self.world, self.rank)
        left, right = neighbours(self.world, self.rank, periodic)
        self.stream = torch.cuda.current_stream(self.device)
        self.ctx = api.Context(cfg, slab=(self.x0, self.x1, left is not None, right is not None),
                               device=self.device.index, stream=self.stream.cuda_stream, **gpu)
        blk = lambda: torch.zeros(8 * ny, dtype=torch.float64, device=self.device)
        self.send_lo, self.send_hi, self.recv_lo, self.recv_hi = blk(), blk(), blk(), blk()
        self.ctx.bind_halo(self.recv_lo if left is not None else None, self.recv_hi if right is not None else None)
        self.xchg = HaloExchange(self.world, self.rank, periodic, group)

    def close(self):
        self.ctx.close()

    def scatter(self, u):
        """This rank's columns of a whole-grid state (4, ny, nx)."""
        self.ctx.upload(np.ascontiguousarray(u[:, :, self.x0:self.x1]))

    def initialize_state(self):
        api.initialize_state(self.ctx)

    def gather(self):
        """The whole-grid state on every rank."""
        dev = self.device if self.xchg.nccl else torch.device("cpu")
        local = torch.from_numpy(np.ascontiguousarray(self.ctx.download())).to(dev)
        if self.world == 1:
            return local.cpu().numpy()
        nx = self.x1 - self.x0
        wmax = max(b - a for a, b in (partition(self._nx(), self.world, r) for r in range(self.world)))
        pad = torch.zeros((4, local.shape[1], wmax), dtype=torch.float64, device=dev)
        pad[:, :, :nx] = local
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(parts, pad, group=self.group)
        cols = []
        for r in range(self.world):
            a, b = partition(self._nx(), self.world, r)
            cols.append(parts[r][:, :, :b - a])
        return torch.cat(cols, dim=2).cpu().numpy()

    def _nx(self):
        return self.ctx.cfg.n_cell[0]

    def _reduce(self, value, dtype, op):
        """All-reduce of one number: on the device over NCCL, on the host otherwise."""
        dev = self.device if self.xchg.nccl else torch.device("cpu")
        t = torch.tensor([value], dtype=dtype, device=dev)
        dist.all_reduce(t, op=op, group=self.group)
        return t.item()

    def compute_euler_dt(self, time=0.0):
        """compute_euler_dt of the whole grid: the minimum of the slabs' dt."""
        dt = api.compute_euler_dt(self.ctx, time)
        if self.world == 1:
            return dt
        return float(self._reduce(dt, torch.float64, dist.ReduceOp.MIN))

    def euler_fv_one_step(self, dt, time=0.0):
        """One explicit step of the whole grid; returns its degenerate count."""
        if self.world > 1:
            self.ctx.pack(self.send_lo, self.send_hi)
            self.xchg.exchange(self.send_lo, self.send_hi, self.recv_lo, self.recv_hi)
        deg = api.euler_fv_one_step(self.ctx, dt, time)
        if self.world == 1:
            return deg
        return int(self._reduce(deg, torch.int64, dist.ReduceOp.SUM))
