"""``torch.autograd.Function`` wrappers of the gradient entries.

The forward pass calls ``ttg_grad_xAx`` / ``ttg_grad_xb`` /
``ttg_grad_sampled``, which return the functional's value AND its gradient
with respect to every core in one device pass (the adjoint sweeps share the
interfaces of the forward sweep); the gradient is kept for ``backward``.
The differentiable input is the flat core vector of x (the layout of
``@tt_tensor/tt_tensor.m:33-41``) as a float64 tensor on any device.

This module loads libttgpu before torch so that the library's CUDA 12.9
cuBLAS/cuSOLVER are the ones the process binds.
"""
from . import lib as _lib

_lib()

import numpy as np  # noqa: E402
import torch  # noqa: E402

from . import TensorTrain, grad_sampled, grad_xAx, grad_xb  # noqa: E402


class TTFunctional(torch.autograd.Function):
    """``f(core)`` for one of the functionals ``"xAx"``, ``"xb"``,
    ``"sampled"`` of the TT tensor with shape (n, r) and flat ``core``."""

    @staticmethod
    def forward(ctx, core, n, r, kind, operand, idx=None, y=None):
        x = TensorTrain(np.asarray(n), np.asarray(r),
                        core.detach().to("cpu", torch.float64).numpy())
        if kind == "xAx":
            v, g = grad_xAx(x, operand)
        elif kind == "xb":
            v, g = grad_xb(x, operand)
        elif kind == "sampled":
            v, g = grad_sampled(x, idx, y)
        else:
            raise ValueError("unknown functional %r" % (kind,))
        ctx.save_for_backward(torch.from_numpy(g.core).to(core.device))
        return torch.tensor(v, dtype=torch.float64, device=core.device)

    @staticmethod
    def backward(ctx, gout):
        (g,) = ctx.saved_tensors
        return gout * g, None, None, None, None, None, None


def xAx(core, n, r, A):
    """``<x, A x>`` (A a ``ttgpu.TTMatrix`` or ``DeviceTT``)."""
    return TTFunctional.apply(core, n, r, "xAx", A)


def xb(core, n, r, b):
    """``<x, b>`` (b a ``ttgpu.TensorTrain`` or ``DeviceTT``)."""
    return TTFunctional.apply(core, n, r, "xb", b)


def sampled_loss(core, n, r, idx, y):
    """``sum_s (X[idx[s]] - y[s])^2``; ``idx`` [S, d] 0-based, ``y`` [S]."""
    return TTFunctional.apply(core, n, r, "sampled", None, idx, y)
