"""The MOP-alpha objective as a differentiable torch function.

``mop_objective(struct, theta_est, keys, J, alpha)`` returns the (F,)
MOP-alpha negative log-likelihoods for the F rows of ``theta_est`` (a CUDA
tensor on the estimation scale).  Its backward is the library's hand-written
adjoint (``ppf_mop_backward``): it replays the ancestors, first-child offsets
and state checkpoints that the forward left in its workspace, so no autodiff
tape is built.  This is the role ``jax.value_and_grad`` of ``_mop_internal``
plays in the reference (``pypomp/core/algorithms/ad_helpers.py:6-54``,
``pypomp/core/algorithms/mop.py:19-135``).
"""

from __future__ import annotations

import numpy as np

from . import _ffi
from .functional import MopCall, PompStruct



def _torch():
    import torch as _t

    return _t


class _MopFunction:
    """Holder of the autograd.Function subclass (created on first use)."""

    cls = None

    @classmethod
    def get(cls):
        if cls.cls is None:
            t = _torch()

            class MopFunction(t.autograd.Function):
                @staticmethod
                def forward(ctx, theta, struct, seeds, J, alpha, ckpt_every):
                    call = MopCall(struct, theta, seeds, J, alpha, ckpt_every=ckpt_every)
                    out = call.forward(grad=False)
                    ctx.call = call
                    ctx.dtype = theta.dtype
                    return out["value"].clone()

                @staticmethod
                def backward(ctx, gvalue):
                    call = ctx.call
                    ctx.call = None
                    grad = call.backward(gvalue.detach())
                    return grad.to(ctx.dtype).clone(), None, None, None, None, None

            cls.cls = MopFunction
        return cls.cls


def mop_objective(struct: PompStruct, theta_est, keys, J: int, alpha: float, ckpt_every: int = 0):
    """(F,) MOP-alpha negative log-likelihood, differentiable in ``theta_est``.

    ``theta_est`` (F, P) CUDA tensor (estimation scale), ``keys`` (F,) uint64
    keys.  Backward runs the adjoint kernels on the forward's saved state."""
    _ffi.require_cuda()
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if theta_est.dim() != 2 or theta_est.shape[0] != keys.shape[0]:
        raise ValueError("theta_est must be (F, P) with one key per row")
    return _MopFunction.get().apply(theta_est, struct, keys, int(J), float(alpha), int(ckpt_every))
