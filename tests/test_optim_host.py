"""Optimiser steps and the train line search on the CPU.

References: pypomp/core/optimizer.py:95-320 (SGD, Adam, FullMatrixAdam,
BFGS, Newton, WeightedNewton) and pypomp/core/algorithms/train.py:38-52
(preconditions), :139-170 and :442-500 (_line_search).  The line search runs
on the C oracle's particle filter in place of the GPU one.
"""

import math

import numpy as np
import pytest

from oracle import cora


def test_full_matrix_adam_step():
    from pypomp_b200.optim import FullMatrixAdam

    opt = FullMatrixAdam()
    g = np.array([[0.5, -1.0, 2.0], [0.1, 0.2, 0.3]])
    m, v = opt.init_state(g)
    assert m.shape == (2, 3) and v.shape == (2, 3, 3)
    d, (m1, v1) = opt.step(g, (m, v), 0)
    for i in range(2):
        mh = (0.1 * g[i]) / (1 - 0.9)
        F = (0.001 * np.outer(g[i], g[i])) / (1 - 0.999)
        w, V = np.linalg.eigh(F)
        want = -(V @ np.diag(1 / np.sqrt(np.maximum(w, 0) + 1e-4)) @ V.T) @ mh
        assert np.allclose(d[i], want)
    assert np.allclose(v1[0], 0.001 * np.outer(g[0], g[0]))


def test_bfgs_steps():
    from pypomp_b200.optim import BFGS

    opt = BFGS()
    g0, g1, g2 = np.array([[1.0, 2.0]]), np.array([[0.5, 1.0]]), np.array([[0.2, 0.7]])
    st = opt.init_state(np.zeros((1, 2)))
    eta = np.array([0.1, 0.3])
    with pytest.raises(ValueError, match="eta_i"):
        opt.step(g0, st, 0)
    d, st = opt.step(g0, st, 0, eta_i=eta)
    assert np.array_equal(d, -g0)
    d, st = opt.step(g1, st, 1, eta_i=eta)
    assert np.array_equal(d, -g1) and np.array_equal(st[0][0], np.eye(2))
    d, st = opt.step(g2, st, 2, eta_i=eta)
    s = 0.2 * (-g1[0])
    y = g2[0] - g1[0]
    rho = 1 / np.dot(y, s)
    H = np.eye(2)
    Hy = H @ y
    H = H - rho * np.outer(s, Hy) - rho * np.outer(Hy, s) + rho * (rho * (y @ Hy) + 1) * np.outer(s, s)
    assert np.allclose(st[0][0], H) and np.allclose(d[0], -H @ g2[0])
    # y . s == 0: the update is skipped
    _, st2 = opt.step(g2, (np.eye(2)[None], g2), 3, eta_i=eta)
    assert np.array_equal(st2[0][0], np.eye(2))


def test_newton_and_weighted_newton():
    from pypomp_b200.optim import Newton, WeightedNewton

    H0 = np.array([[[4.0, 1.0], [1.0, 3.0]]])
    H1 = np.array([[[2.0, 0.0], [0.0, 5.0]]])
    g = np.array([[1.0, -1.0]])
    with pytest.raises(ValueError, match="compute_hessian_fn"):
        Newton().step(g, (), 0)
    d, _ = Newton().step(g, (), 0, compute_hessian_fn=lambda: H0)
    assert np.allclose(d[0], -np.linalg.solve(H0[0], g[0]))
    wn = WeightedNewton()
    st = wn.init_state(np.zeros((1, 2)))
    d, st = wn.step(g, st, 0, compute_hessian_fn=lambda: H0)
    assert np.allclose(d[0], -np.linalg.solve(H0[0], g[0])) and np.array_equal(st[0], H0)
    d, st = wn.step(g, st, 1, compute_hessian_fn=lambda: H1)
    wt = 1.0 / 2.0 ** math.log(2.0)
    assert np.allclose(d[0], -np.linalg.solve(wt * H0[0] + (1 - wt) * H1[0], g[0]))


def test_train_preconditions():
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import SGD, LearningRate, Newton

    m = pp.LG(T=5, key=0)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names))
    eta = LearningRate({n: 0.01 for n in m.canonical_param_names})
    with pytest.raises(ValueError, match="at least one monitor"):
        F.train(st, th, 100, SGD(ls=True), 2, eta, 0.97, [1], n_monitors=0)

    from pypomp_b200.optim import Optimizer

    class Other(Optimizer):
        pass
    with pytest.raises(ValueError, match="not supported"):
        F.train(st, th, 100, Other(), 2, eta, 0.97, [1])
    assert Newton.needs_hessian and not SGD.needs_hessian


def test_line_search_follows_armijo(monkeypatch):
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F

    m = pp.Ricker(T=30, key=4)
    st = m.to_struct()
    spec = st.spec
    ycon = spec.ycon(st.ys[None])

    def fake_run_pfilter(struct, theta_f, seeds_f, J, *, thresh=0.0, est=False, **kw):
        return {"loglik": cora.pfilter(spec.kind, 1, 1, theta_f, struct.ys, J, seeds=seeds_f, ycon=ycon,
                                       thresh=thresh, est=est)["loglik"]}

    monkeypatch.setattr(F, "run_pfilter", fake_run_pfilter)
    th0 = spec.to_est(m.theta.to_array(m.canonical_param_names))
    th = np.concatenate([th0, th0 + 0.3])
    keys = np.array([7, 8], np.uint64)
    J = 400
    curr = -fake_run_pfilter(st, th.astype(np.float32), keys, J, est=True)["loglik"]
    grad = np.array([[0.5, -0.2, 0.1, 0.0], [-3.0, 1.0, 0.5, 0.2]])
    direction = -grad * np.array([[1.0], [8.0]])
    got = F._line_search(st, th, keys, J, 0.0, curr, grad, direction, 0.5, 10, 0.1, 0.5)
    for i in range(2):     # the reference's while-loop, row by row
        eta, itn, cont = 0.5, 0, True
        while cont:
            pt = (th[i] + eta * direction[i])[None].astype(np.float32)
            nxt = -fake_run_pfilter(st, pt, keys[i:i + 1], J, est=True)["loglik"][0]
            sc = (nxt > curr[i] + eta * 0.1 * np.sum(grad[i] * direction[i])) or np.isnan(nxt)
            eta = eta * 0.5 if (sc and itn < 10) else eta
            cont = sc and itn < 10
            itn += 1
        assert got[i] == eta
    assert got[1] < 0.5      # the long step on row 1 had to be cut back
