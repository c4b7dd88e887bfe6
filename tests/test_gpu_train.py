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


@pytest.mark.parametrize("name", ["FullMatrixAdam", "BFGS", "Newton", "WeightedNewton", "SGD_ls", "Adam_ls"])
def test_train_every_optimizer_and_line_search(name):
    """Each optimiser of the reference drives the GPU MOP gradient; the line
    search backtracks on the GPU particle filter.  Traces stay finite and the
    final parameters do not fall far below the start in exact log-likelihood."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200 import optim
    from oracle.kalman import kalman_loglik, lg_matrices

    m = pp.LG(T=40, A=[[0.8]], C=[[1.0]], Q=[[0.5]], R=[[0.5]], X0=[0.0], key=3)
    st = m.to_struct()
    spec = st.spec
    names = m.canonical_param_names
    th = m.theta.to_array(names)[0] * np.array([0.9, 1.0, 1.3, 0.8, 1.0])
    est = np.repeat(spec.to_est(th)[None], 2, axis=0)
    opt = {"FullMatrixAdam": optim.FullMatrixAdam(), "BFGS": optim.BFGS(), "Newton": optim.Newton(),
           "WeightedNewton": optim.WeightedNewton(), "SGD_ls": optim.SGD(ls=True),
           "Adam_ls": optim.Adam(ls=True, c=0.01)}[name]
    rate = 0.02 if name in ("FullMatrixAdam", "BFGS", "SGD_ls", "Adam_ls") else 0.3
    eta = optim.LearningRate({n: rate for n in names})
    nll, tr = F.train(st, est, 4000, opt, 4, eta, 0.97, np.array([11, 12], np.uint64))
    assert nll.shape == (2, 5) and tr.shape == (2, 5, 5)
    assert np.all(np.isfinite(nll[:, 1:])) and np.all(np.isfinite(tr))

    def kal(e):
        A, C, Q, R, X0 = lg_matrices(spec.from_est(e), 1, 1)
        return kalman_loglik(st.ys, A, C, Q, R, X0)
    start = kal(est[0])
    for i in range(2):
        assert kal(tr[i, -1]) > start - 2.0, (name, start, kal(tr[i, -1]))


def test_hessian_fd_symmetric_and_finite():
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F

    m = pp.SV(T=60, key=1)
    st = m.to_struct()
    est = st.spec.to_est(m.theta.to_array(m.canonical_param_names))
    H = F.mop_hessian_fd(st, np.repeat(est, 2, axis=0), np.array([3, 4], np.uint64), 3000, 0.97)
    assert H.shape == (2, 6, 6) and np.all(np.isfinite(H))
    assert np.allclose(H, np.swapaxes(H, 1, 2))


def test_hessian_fd_near_exact_kalman_hessian():
    """The central-difference MOP Hessian (alpha = 1, J = 1e5, h = 1e-2) against
    the exact Kalman Hessian of LG 1-D: the diagonal within a factor of two."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from oracle.kalman import kalman_loglik, lg_matrices

    m = pp.LG(T=50, A=[[0.8]], C=[[1.0]], Q=[[0.5]], R=[[0.5]], X0=[0.0], key=3)
    st = m.to_struct()
    spec = st.spec
    est = spec.to_est(m.theta.to_array(m.canonical_param_names)[0])

    def nll(e):
        A, C, Q, R, X0 = lg_matrices(spec.from_est(e), 1, 1)
        return -kalman_loglik(st.ys, A, C, Q, R, X0)
    h = 1e-4
    exact = np.array([(nll(est + h * np.eye(5)[i]) - 2 * nll(est) + nll(est - h * np.eye(5)[i])) / h ** 2
                      for i in range(4)])
    H = F.mop_hessian_fd(st, est[None], np.array([7], np.uint64), 100000, 1.0)[0] * 50
    ratio = np.diag(H)[:4] / exact
    assert np.all((ratio > 0.5) & (ratio < 2.0)), (np.diag(H), exact)


def test_train_reused_mop_call_equals_fresh_calls():
    """With one alpha for the run, functional.train reuses one MOP call per step
    (MopCall.update, graph replay); the trace equals fresh run_mop calls under
    the same key tree (train.py:86-90: a MOP key, then a Hessian key per step)."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom
    from pypomp_b200.optim import SGD, LearningRate

    m = pp.SV(T=40, key=1)
    st = m.to_struct()
    names = m.canonical_param_names
    est = np.repeat(st.spec.to_est(m.theta.to_array(names)), 2, axis=0)
    est[1, 0] += 0.1
    keys = np.array([31, 32], np.uint64)
    J, M, rate = 3000, 4, 0.05
    eta = LearningRate({n: rate for n in names})
    nll, tr = F.train(st, est, J, SGD(), M, eta, 0.97, keys)
    th = est.copy()
    chain = [int(k) for k in keys]
    for step in range(M):
        subs = np.zeros(2, np.uint64)
        for i in range(2):
            chain[i], subs[i] = (int(v) for v in pprandom.split(chain[i]))
        res = F.run_mop(st, th.astype(np.float32), subs, J, 0.97, grad=True)
        assert np.array_equal(res["value"], nll[:, step + 1])
        for i in range(2):
            chain[i] = int(pprandom.split(chain[i])[0])
        th = th + rate * (-res["grad"] / 40)
        assert np.array_equal(th, tr[:, step + 1])


@pytest.mark.parametrize("opt_name,alpha_cooling", [("Adam", 1.0), ("SGD", 0.5)])
def test_train_device_loop_equals_host_loop(opt_name, alpha_cooling):
    """The device-side training loop (parameters, optimiser state and traces in
    device memory, one synchronisation at the end) gives the host loop's
    negative log-likelihoods and parameter traces bit for bit, with a
    constant alpha (graph replay) and with cosine-cooled alpha."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200 import optim

    m = pp.SV(T=80, key=3)
    st = m.to_struct()
    est = np.repeat(m.spec.to_est(m.theta.to_array(m.canonical_param_names)), 2, axis=0)
    opt = optim.Adam(clip_norm=5.0) if opt_name == "Adam" else optim.SGD()
    eta = optim.LearningRate({n: 0.01 for n in m.canonical_param_names})
    keys = np.array([8, 9], np.uint64)
    a = F.train(st, est, 4096, opt, 5, eta, 0.97, keys, alpha_cooling=alpha_cooling, device_loop=True)
    b = F.train(st, est, 4096, opt, 5, eta, 0.97, keys, alpha_cooling=alpha_cooling, device_loop=False)
    assert np.array_equal(a[0], b[0], equal_nan=True)
    assert np.array_equal(a[1], b[1])
