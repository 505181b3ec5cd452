"""Differentiable explicit rollouts: torch.autograd.Function over the C ABI.

U_N = step_{dt_{N-1}} o ... o step_{dt_0} (U_0), each step the explicit O2
update of euler_fv_one_step (numerics/explicit_update.hpp:58-102) with its dt
held fixed.  The forward keeps every k-th state (a checkpoint); the backward
walks the segments last to first, recomputes the states inside a segment
from its checkpoint and applies the hand-written step adjoint
(ecg_explicit_step_vjp_device) step by step.  Memory: N/k checkpoints plus k
states of one segment.

States are CUDA float64 tensors of shape (4, ny, nx) (component planes, i
fastest).  The context's kernels run on the stream the context was created
with; create it on the current torch stream (the default of `make_context`).
"""
import ctypes as C

import torch

from . import api
from ._lib import check, load


def make_context(cfg, **gpu):
    """A context whose kernels are ordered with torch's current CUDA stream."""
    gpu.setdefault("stream", torch.cuda.current_stream().cuda_stream)
    return api.Context(cfg, **gpu)


def _step(ectx, u, dt):
    out = torch.empty_like(u)
    check(load().ecg_explicit_step_device(ectx.handle, C.c_void_p(u.data_ptr()), float(dt),
                                          C.c_void_p(out.data_ptr())), "explicit_step_device", ectx.handle)
    return out


def _vjp(ectx, u, dt, g):
    out = torch.empty_like(g)
    check(load().ecg_explicit_step_vjp_device(ectx.handle, C.c_void_p(u.data_ptr()), float(dt),
                                              C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr())),
          "explicit_step_vjp_device", ectx.handle)
    return out


class ExplicitRollout(torch.autograd.Function):
    """apply(u0, ectx, dts, k) -> U_N; gradients flow to u0 only."""

    @staticmethod
    def forward(fctx, u0, ectx, dts, k):
        if u0.dtype != torch.float64 or not u0.is_cuda or u0.shape != (4, ectx.ny, ectx.nx):
            raise ValueError("u0 must be a CUDA float64 tensor of shape (4, ny, nx)")
        dts = [float(d) for d in dts]
        k = max(1, int(k))
        u = u0.detach().contiguous()
        checkpoints = [u]
        for n, dt in enumerate(dts):
            u = _step(ectx, u, dt)
            if (n + 1) % k == 0 and n + 1 < len(dts):
                checkpoints.append(u)
        fctx.ectx, fctx.dts, fctx.k, fctx.checkpoints = ectx, dts, k, checkpoints
        return u

    @staticmethod
    def backward(fctx, g):
        ectx, dts, k = fctx.ectx, fctx.dts, fctx.k
        g = g.contiguous()
        nseg = len(fctx.checkpoints)
        for s in range(nseg - 1, -1, -1):
            start = s * k
            end = min(start + k, len(dts))
            states = [fctx.checkpoints[s]]
            for n in range(start, end - 1):
                states.append(_step(ectx, states[-1], dts[n]))
            for n in range(end - 1, start - 1, -1):
                g = _vjp(ectx, states[n - start], dts[n], g)
        return g, None, None, None


def explicit_rollout(ectx, u0, dts, checkpoint_every=20):
    """U_N after len(dts) explicit steps from u0, differentiable in u0."""
    return ExplicitRollout.apply(u0, ectx, list(dts), checkpoint_every)
