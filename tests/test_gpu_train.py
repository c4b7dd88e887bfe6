"""Train (MOP-alpha gradient steps + Adam) against the reference's fixture (GPU).

The reference's locked train run (``test_train_regression.py``: LG 1-D, J=12,
three Adam steps with alpha=0 on the MOP gradient) is replayed through the
product path: for each iteration the reference's own draws (its JAX key tree,
restated in ``oracle/jaxrng.py``) are injected into the CUDA MOP forward and
adjoint, and the gradient drives ``pypomp_b200.optim.Adam``.  Matching the
locked final parameters to the fixtures' tolerance pins the adjoint against the
reference's ``jax.value_and_grad``.
"""

import numpy as np
import pytest

from oracle import jaxrng as jr, refpath as rp

pytestmark = pytest.mark.gpu


def test_train_reference_fixture_through_injection(ref_values, ref_lg1d):
    from pypomp_b200 import functional as F
    from pypomp_b200.functional import PompStruct
    from pypomp_b200.models import lg_spec
    from pypomp_b200.optim import Adam, cosine_alpha

    st = PompStruct(spec=lg_spec(1, 1), ys=ref_lg1d["ys"], times=np.arange(1, 5.0), t0=0.0)
    th = ref_lg1d["theta"].astype(np.float64)
    T, J, M = 4, 12, 3
    opt = Adam(scale=False, ls=False, c=0.0, max_ls_itn=1)
    state = opt.init_state(th)
    key = jr.split(jr.key(20260811), 1)[0]        # keys = split(key, n_reps)
    nll = None
    for m in range(M):
        alpha_m = 1.0 - (1.0 - 0.0) * cosine_alpha(m, M, 1.0)
        s = jr.split(key)                           # train.py:89
        key, sub = s[0], s[1]
        rec = rp.RecordingNoise(rp.JaxKeyNoise(sub, J, 1, 1))
        rp.mop("LG", th.astype(np.float32), ref_lg1d["ys"], J, alpha_m, rec)
        z0, z, u = rec.arrays()
        res = F.run_mop(st, th.astype(np.float32)[None], np.zeros(1, np.uint64), J, alpha_m,
                        inject=dict(z0=z0[None], z=z[None], u=u[None]), grad=True)
        nll = res["value"][0]
        grad = res["grad"][0] / T
        key = jr.split(key)[0]                      # train.py:118 (Hessian subkey)
        direction, state = opt.step(grad, state, m)
        th = th + 0.01 * direction
    tol = ref_values["tolerance"]
    np.testing.assert_allclose(nll, ref_values["train"]["final_neg_loglik"][0], **tol)
    np.testing.assert_allclose(th[:4], ref_values["train"]["final_theta"][:4], **tol)


def test_functional_train_moves_toward_kalman_mle():
    """A short train run on the 1-D LG model increases the exact likelihood."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import Adam, LearningRate
    from oracle import kalman

    m = pp.LG(T=60, A=np.array([[0.8]]), C=np.array([[1.0]]), Q=np.array([[0.04]]),
              R=np.array([[0.09]]), key=7)
    st = m.to_struct()
    names = m.canonical_param_names
    start = m.theta.to_array(names)[0].copy()
    start[0] = 0.4                                       # A11 far from the truth
    th0 = m.spec.to_est(start[None])
    eta = LearningRate({n: (0.02 if n == "A11" else 0.0) for n in names})
    nll, traces = F.train(st, th0, 2000, Adam(), 40, eta, 0.97, np.array([3], np.uint64))

    def exact(theta_est):
        A, C, Q, R, X0 = kalman.lg_matrices(m.spec.from_est(theta_est), 1, 1)
        return kalman.kalman_loglik(st.ys, A, C, Q, R, X0)

    assert exact(traces[0, -1]) > exact(traces[0, 0]) + 1.0
    assert traces[0, -1, 0] > 0.55
