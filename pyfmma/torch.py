"""Differentiable FMM for PyTorch: c = FMM(targets, sources, weights) with a
hand-written adjoint.

    from pyfmma.torch import fmm
    c = fmm(x, y, w, kernel=pyfmma.kernels.gaussian(0.01), poly_ord=4, depth=6)
    (g * c).sum().backward()        # x.grad, y.grad, w.grad

Backward (L = sum_i g_i c_i):
  dL/dw_j = sum_i g_i f(x_i, y_j)          the transposed FMM: targets and
                                           sources swapped, weights g
  dL/dy_j = w_j sum_i g_i d f(x_i, y_j)/dy the gradient of that transposed
                                           field at y_j (L2P and P2P on grad f)
  dL/dx_i = g_i sum_j w_j d f(x_i, y_j)/dx the gradient of the forward field
For the built-in kernels f(x, y) = s f(y, x) with s = -1 for 1/(x-y) and
sum_d (x-y)_d/|x-y|^2, s = +1 otherwise.  Trees and interaction lists are
rebuilt in every call, not stored.  No counterpart in the reference (which has
no derivatives).
"""
from __future__ import annotations

import torch

import fmma_b200

from . import kernels as _k

_ANTISYMMETRIC = {_k.inv_diff.kernel_id, _k.sum_over_r2.kernel_id}


class FMMAFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, y, w, spec):
        fc = spec["context"]
        with fc.lock:
            fc.set_kernel(spec["kernel"].kernel_id, spec["kernel"].p0)
            c, used = fc.solve(x.contiguous(), y.contiguous(), w.contiguous(), solver=spec["solver"],
                               poly_ord=spec["poly_ord"], depth=spec["depth"], trans_sym=spec["trans_sym"],
                               precision=spec["precision"])
        ctx.spec = dict(spec, depth=used)
        ctx.save_for_backward(x, y, w)
        return c

    @staticmethod
    def backward(ctx, g):
        x, y, w = ctx.saved_tensors
        spec = ctx.spec
        fc = spec["context"]
        sign = -1.0 if spec["kernel"].kernel_id in _ANTISYMMETRIC else 1.0
        g = g.contiguous().to(torch.float64)
        kw = dict(solver=spec["solver"], poly_ord=spec["poly_ord"], depth=spec["depth"],
                  trans_sym=spec["trans_sym"], precision=spec["precision"])
        dx = dy = dw = None
        with fc.lock:
            fc.set_kernel(spec["kernel"].kernel_id, spec["kernel"].p0)
            if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
                # transposed field u(y) = sum_i g_i f(y, x_i) and its gradient at y
                u, ug, _ = fc.solve_grad(y.contiguous(), x.contiguous(), g, want_potential=ctx.needs_input_grad[2],
                                         **kw)
                if ctx.needs_input_grad[2]:
                    dw = sign * u
                if ctx.needs_input_grad[1]:
                    dy = sign * (w.unsqueeze(-1) * ug)
                    if dy.dim() == 3:
                        dy = dy.sum(0)
            if ctx.needs_input_grad[0]:
                _, cg, _ = fc.solve_grad(x.contiguous(), y.contiguous(), w.contiguous(), want_potential=False, **kw)
                dx = g.unsqueeze(-1) * cg
                if dx.dim() == 3:
                    dx = dx.sum(0)
        return dx, dy, dw, None


def fmm(x, y, w, *, kernel=_k.laplace, poly_ord=4, depth=-1, trans_sym=0, precision="fp64", solver="fmm",
        context=None):
    """c[r, i] = sum_j w[r, j] f(x_i, y_j) on CUDA float64 tensors, differentiable in x, y and w."""
    if not (x.is_cuda and y.is_cuda and w.is_cuda):
        raise ValueError("pyfmma.torch.fmm takes CUDA tensors")
    if x.dtype != torch.float64 or y.dtype != torch.float64 or w.dtype != torch.float64:
        raise TypeError("pyfmma.torch.fmm takes float64 tensors")
    spec = dict(context=context or fmma_b200.default_context(x.device.index or 0), kernel=kernel,
                poly_ord=int(poly_ord), depth=int(depth), trans_sym=int(trans_sym), precision=precision,
                solver=solver)
    return FMMAFunction.apply(x, y, w, spec)
