"""MOP-alpha through torch autograd (GPU).

``mop_objective`` runs ``ppf_mop`` in its forward and ``ppf_mop_backward`` (the
adjoint sweep over the forward's saved ancestors and checkpoints) in its
backward.  The gradient must equal the one ``ppf_mop`` computes in a single
call (float64 sums, cast to the parameters' float32), scale with the upstream
gradient row by row, and leave the values unchanged.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
f32 = np.float32


def _case():
    import pypomp_b200 as pp

    m = pp.SV(T=40, key=1)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    th = np.repeat(th, 3, axis=0)
    th[1, 0] += f32(0.05)
    th[2, 3] -= f32(0.1)
    return st, th


def test_autograd_matches_single_call_gradient():
    import torch

    from pypomp_b200 import functional as F
    from pypomp_b200.autograd import mop_objective

    st, th = _case()
    keys = np.array([4, 5, 6], np.uint64)
    J = 3000
    want = F.run_mop(st, th, keys, J, 0.97, grad=True)
    theta = torch.tensor(th, device="cuda", requires_grad=True)
    v = mop_objective(st, theta, keys, J, 0.97)
    np.testing.assert_array_equal(v.detach().cpu().numpy(), want["value"])
    v.sum().backward()
    np.testing.assert_allclose(theta.grad.cpu().numpy(), want["grad"].astype(f32), rtol=1e-6, atol=1e-6)


def test_autograd_scales_by_upstream_gradient():
    import torch

    from pypomp_b200 import functional as F
    from pypomp_b200.autograd import mop_objective

    st, th = _case()
    keys = np.array([7, 8, 9], np.uint64)
    J = 2048
    want = F.run_mop(st, th, keys, J, 0.5, grad=True)["grad"]
    w = torch.tensor([1.0, -2.0, 0.25], dtype=torch.float64, device="cuda")
    theta = torch.tensor(th, device="cuda", requires_grad=True)
    (mop_objective(st, theta, keys, J, 0.5) * w).sum().backward()
    np.testing.assert_allclose(theta.grad.cpu().numpy(), (want * w.cpu().numpy()[:, None]).astype(f32),
                               rtol=1e-6, atol=1e-6)


def test_mopcall_backward_equals_forward_with_gradient():
    from pypomp_b200.functional import MopCall

    st, th = _case()
    keys = np.array([1, 2, 3], np.uint64)
    a = MopCall(st, th, keys, 1500, 0.97)
    a.forward(grad=True)
    g1 = a.out["grad"].cpu().numpy().copy()
    b = MopCall(st, th, keys, 1500, 0.97)
    b.forward(grad=False)
    g2 = b.backward().cpu().numpy()
    np.testing.assert_allclose(g2, g1, rtol=1e-12, atol=1e-12)
