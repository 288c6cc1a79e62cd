"""Differentiable space-charge step for PyTorch: E at the particles as a function of their
positions (and charges), with the backward pass computed by the native adjoint
(``osc_space_charge_step_vjp_dev``).  The mesh is held fixed (no refit inside the graph).

Both passes run on the caller's current CUDA stream, so they order with the surrounding
torch work.  The FP32 backward reuses E on the grid from its forward step when no other step
ran on the context in between (OPT_VJP_REUSE_FORWARD, set for the backward call only): the
tensors saved for backward cannot change in between, torch checks their versions."""
from __future__ import annotations

import ctypes

import torch

from .mesh import Mesh3D, _ctx, _tp
from .native import OPT_VJP_REUSE_FORWARD, PREC_FP32


def _on_stream(octx):
    s = torch.cuda.current_stream()
    octx.set_stream(s.cuda_stream)


class _SpaceChargeField(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x, y, z, q, octx, mesh: Mesh3D, precision: int):
        for t in (x, y, z, q):
            if t.dtype != torch.float64 or not t.is_cuda:
                raise ValueError("space_charge_field needs float64 CUDA tensors")
        x, y, z, q = (t.contiguous() for t in (x, y, z, q))
        _on_stream(octx)
        E = torch.empty((x.numel(), 3), dtype=torch.float64, device=x.device)
        m = mesh.to_c()
        octx.call("osc_space_charge_step_dev", ctypes.byref(m), ctypes.c_int64(x.numel()), _tp(x), _tp(y), _tp(z),
                  _tp(q), None, 0, 0, int(precision), _tp(E), None)
        fctx.save_for_backward(x, y, z, q)
        fctx.octx = octx
        fctx.cmesh = m
        fctx.precision = precision
        return E

    @staticmethod
    def backward(fctx, gE):
        x, y, z, q = fctx.saved_tensors
        octx = fctx.octx
        _on_stream(octx)
        gE = gE.contiguous().to(torch.float64)
        gx, gy, gz = torch.empty_like(x), torch.empty_like(y), torch.empty_like(z)
        gq = torch.empty_like(q) if fctx.needs_input_grad[3] else None
        prev = octx.get_option(OPT_VJP_REUSE_FORWARD)
        octx.set_option(OPT_VJP_REUSE_FORWARD, 1)
        try:
            octx.call("osc_space_charge_step_vjp_dev", ctypes.byref(fctx.cmesh), ctypes.c_int64(x.numel()),
                      _tp(x), _tp(y), _tp(z), _tp(q), ctypes.c_double(0.0), int(fctx.precision), _tp(gE), _tp(gx),
                      _tp(gy), _tp(gz), _tp(gq))
        finally:
            octx.set_option(OPT_VJP_REUSE_FORWARD, prev)
        return gx, gy, gz, gq, None, None, None


def space_charge_field(x, y, z, q, mesh: Mesh3D, ctx, precision: int = PREC_FP32):
    """E (np, 3) at the particles for positions x, y, z and charges q (float64 CUDA tensors),
    on the fixed mesh `mesh`; differentiable with respect to x, y, z and q.  The context's
    stream is set to torch's current stream."""
    return _SpaceChargeField.apply(x, y, z, q, _ctx(ctx), mesh, precision)
