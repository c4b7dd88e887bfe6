"""The linear Gaussian model above 4 x 4 (up to dx = dy = 9, the reference's
``MAX_DIM``, ``pypomp/models/linear_gaussian.py:48``) on the GPU.

The wide instantiation (matrix row stride 9, run-time dy <= 9) runs the
streaming and plain filters, MOP-alpha with its adjoint, IF2 and simulation.
Each is checked against the C oracle, which restates the same arithmetic:

* Philox-mode filters bit for bit (ancestors, log-weights, CLL, ESS and the
  filter / prediction means) on both paths, for square and non-square shapes;
* the log-likelihood of a 9 x 9 model within Monte Carlo error of the exact
  FP64 Kalman value;
* the MOP adjoint against central differences of the oracle's frozen-ancestry
  surrogate, and MOP's forward ancestors bit for bit;
* IF2 swarms and ancestors bit for bit; simulated trajectories bit for bit;
* the object API on a 7-D model end to end, and the dimension limit's error.
"""

import numpy as np
import pytest

from oracle import cora, kalman

pytestmark = pytest.mark.gpu
f32 = np.float32


def _model(dx, dy, T, key):
    import pypomp_b200 as pp

    return pp.LG(T=T, A=0.9 * np.eye(dx), C=np.eye(dy, dx) + 0.1, Q=np.eye(dx) * 0.05,
                 R=np.eye(dy) * 0.2 + 0.02, key=key)


def _thetas(m, F):
    th = np.repeat(m.theta.to_array(m.canonical_param_names), F, axis=0).astype(f32)
    for f in range(1, F):
        th[f, 0] *= f32(1.0 - 0.03 * f)
    return th


@pytest.mark.parametrize("path", ["stream", "plain"])
@pytest.mark.parametrize("dx,dy", [(6, 7), (2, 5), (9, 9), (5, 1)])
def test_wide_lg_philox_bit_exact(dx, dy, path):
    from pypomp_b200 import functional as F

    m = _model(dx, dy, 8, key=dx * 10 + dy)
    st = m.to_struct()
    th = _thetas(m, 2)
    seeds = np.array([5, 6], np.uint64)
    J = 3000
    want = cora.pfilter(m.spec.kind, dx, dy, th, st.ys, J, seeds=seeds, anc=True, logw=True, CLL=True, ESS=True,
                        fmean=True, pmean=True)
    got = F.run_pfilter(st, th, seeds, J, path=path, save_ancestors=True, save_weights=True, CLL=True,
                        ESS=True, filter_mean=True, prediction_mean=True)
    assert np.array_equal(got["anc"], want["anc"])
    assert np.array_equal(got["logw"].view(np.uint32), want["logw"].view(np.uint32))
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12)
    np.testing.assert_allclose(got["cll"], want["cll"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got["ess"], want["ess"], rtol=1e-5)
    for k in ("fmean", "pmean"):
        np.testing.assert_allclose(got[k], want[k], rtol=1e-5, atol=1e-6)


def test_wide_lg_loglik_against_kalman():
    """9 x 9: log-mean-exp of 16 filters of 200000 particles within 5
    standard errors of the exact FP64 Kalman log-likelihood."""
    from pypomp_b200 import functional as F
    from pypomp_b200.maths import logmeanexp, logmeanexp_se

    m = _model(9, 9, 30, key=99)
    st = m.to_struct()
    th = _thetas(m, 1)
    ll = F.run_pfilter(st, np.repeat(th, 16, axis=0), np.arange(16, dtype=np.uint64) + 1, 200000)["loglik"]
    A, C, Q, R, X0 = kalman.lg_matrices(th[0].astype(np.float64), 9, 9)
    exact = kalman.kalman_loglik(st.ys, A, C, Q, R, X0)
    lme, se = logmeanexp(ll), logmeanexp_se(ll)
    assert np.all(np.isfinite(ll))
    assert abs(lme - exact) <= 5 * se + 1e-3, (lme, exact, se)


@pytest.mark.parametrize("dx,dy", [(5, 6), (3, 5)])
def test_wide_lg_mop_gradient_vs_finite_differences(dx, dy):
    from pypomp_b200 import functional as F

    m = _model(dx, dy, 10, key=7)
    st, spec = m.to_struct(), m.spec
    th = spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    seeds = np.array([11], np.uint64)
    J, alpha = 800, 0.9
    fwd = cora.pfilter(spec.kind, dx, dy, th, st.ys, J, seeds=seeds, est=True, mop=True, anc=True)
    got = F.run_mop(st, th, seeds, J, alpha, grad=True, save_ancestors=True)
    assert np.array_equal(got["anc"], fwd["anc"])
    np.testing.assert_allclose(got["value"], -fwd["loglik"], rtol=1e-12)
    base, m0 = cora.mop_surrogate(spec.kind, dx, dy, th, st.ys, J, alpha, got["anc"], seeds=seeds)
    np.testing.assert_allclose(base[0], got["value"][0], rtol=1e-7)
    h, P = 1e-3, th.shape[1]
    fd = np.zeros(P)
    for p in range(P):
        tp, tm = th.copy(), th.copy()
        tp[0, p] += f32(h)
        tm[0, p] -= f32(h)
        hp, hm = float(tp[0, p]) - float(th[0, p]), float(th[0, p]) - float(tm[0, p])
        vp = cora.mop_surrogate(spec.kind, dx, dy, tp, st.ys, J, alpha, got["anc"], m0, seeds=seeds)[0]
        vm = cora.mop_surrogate(spec.kind, dx, dy, tm, st.ys, J, alpha, got["anc"], m0, seeds=seeds)[0]
        fd[p] = (vp[0] - vm[0]) / (hp + hm)
    g = got["grad"][0]
    err = np.linalg.norm(g - fd) / np.linalg.norm(fd)
    assert err <= 1e-3, (err, g, fd)


@pytest.mark.parametrize("dx,dy", [(1, 5), (5, 5), (9, 9)])
def test_wide_lg_perfilter_bit_exact(dx, dy):
    from pypomp_b200 import functional as F

    m = _model(dx, dy, 6, key=3)
    st, spec = m.to_struct(), m.spec
    th = spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    nF, P, T, J = 2, th.shape[1], st.ys.shape[0], 1500
    rng = np.random.default_rng(5)
    swarm = (np.repeat(th[:, :, None], J, axis=2).repeat(nF, axis=0)
             + f32(0.01) * rng.standard_normal((nF, P, J)).astype(f32)).astype(f32)
    sig = np.full(P, 0.02, f32)
    sig0 = np.zeros(P, f32)
    cool = (0.98 ** np.arange(T)).astype(f32)
    seeds = np.array([11, 12], np.uint64)
    want = cora.perfilter(spec.kind, dx, dy, swarm, st.ys, J, sig, sig0, cool, f32(0.99), seeds=seeds,
                          CLL=True, anc=True)
    got = F.run_perfilter(st, swarm.transpose(0, 2, 1), seeds, J, sig, sig0, cool, f32(0.99), CLL=True,
                          save_ancestors=True)
    assert np.array_equal(got["anc"], want["anc"])
    assert np.array_equal(got["swarm"], want["swarm"].transpose(0, 2, 1))
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12)


def test_wide_lg_simulate_bit_exact():
    from pypomp_b200 import functional as F

    m = _model(6, 7, 9, key=4)
    st = m.to_struct()
    th = _thetas(m, 2)
    seeds = np.array([21, 22], np.uint64)
    X, Y = F.simulate(st, th, 300, seeds)
    Xo, Yo = cora.simulate(m.spec.kind, 6, 7, th, 300, 9, seeds)
    assert np.array_equal(X, Xo) and np.array_equal(Y, Yo)


def test_wide_lg_object_api_and_limits():
    import pypomp_b200 as pp
    from pypomp_b200.optim import LearningRate, RWSigma

    m = _model(7, 3, 20, key=8)
    assert m.canonical_param_names[:2] == ["A11", "A12"] and len(m.statenames) == 7
    m.pfilter(J=2000, key=1, reps=2)
    assert np.all(np.isfinite(m.results()["logLik"]))
    names = m.canonical_param_names
    m.mif(J=1000, M=2, rw_sd=RWSigma({n: 0.01 for n in names}).geometric_cooling(0.5), key=2)
    m.train(J=1000, M=2, eta=LearningRate({n: 0.001 for n in names}), key=3)
    assert np.all(np.isfinite(m.theta.to_array(names)))
    with pytest.raises(ValueError, match="dimensions up to 9"):
        pp.LG(T=5, A=np.eye(10))
