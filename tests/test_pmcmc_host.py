"""PMCMC host logic on the CPU: proposals, the prior's change of variables,
and the Metropolis-Hastings chains driven by the C oracle's particle filter.

References: pypomp/proposals.py (MVNDiagRW, MVNRWFull, MVNRWAdaptive),
pypomp/core/algorithms/pmcmc.py:30-163 (_pmcmc_internal / _pmcmc_step),
pypomp/functional/pmcmc.py:18-113, pypomp/core/model_mechanics.py:798-862
(_DPrior: log-Jacobian of the back-transform on the estimation scale).
"""

import math

import numpy as np
import pytest

from oracle import cora


def test_diag_proposal_validation_and_canonical_order():
    from pypomp_b200.proposals import MVNDiagRW

    with pytest.raises(ValueError, match="at least one positive"):
        MVNDiagRW({"a": 0.0, "b": -1.0})
    p = MVNDiagRW({"b": 0.2, "a": 0.1, "c": 0.0})
    assert p.param_names == ("b", "a")
    q = p.canonicalize(["a", "b", "z"])
    assert q.param_names == ("a", "b", "z") and np.array_equal(q.sd_arr, [0.1, 0.2, 0.0])
    with pytest.raises(ValueError, match="not in model"):
        p.canonicalize(["a"])
    th = np.array([1.0, 2.0, 3.0])
    prop, st = q.step((), th, np.uint64(99), 1, 0)
    z = np.random.default_rng(99).standard_normal(3)
    assert np.array_equal(prop, th + z * q.sd_arr) and prop[2] == 3.0 and st == ()


def test_full_proposal_validation_and_draw():
    from pypomp_b200.proposals import MVNRWFull

    with pytest.raises(ValueError, match="square"):
        MVNRWFull(np.ones((2, 3)), ["a", "b"])
    with pytest.raises(ValueError, match="len\\(param_names\\)"):
        MVNRWFull(np.eye(2), ["a"])
    V = np.array([[0.04, 0.01], [0.01, 0.09]])
    p = MVNRWFull(V, ["y", "x"]).canonicalize(["x", "y"])
    L = np.linalg.cholesky(V)
    assert np.allclose(p.chol, [[L[1, 1], L[1, 0]], [L[0, 1], L[0, 0]]])
    prop, _ = p.step((), np.zeros(2), np.uint64(5), 1, 0)
    assert np.allclose(prop, p.chol @ np.random.default_rng(5).standard_normal(2))


def test_adaptive_proposal_phases_and_welford():
    from pypomp_b200.proposals import MVNRWAdaptive

    for kw in ({}, {"rw_sd": {"a": 1.0}, "rw_var": np.eye(1)}):
        with pytest.raises(ValueError, match="Exactly one"):
            MVNRWAdaptive(**kw)
    for bad in ({"scale_start": 0}, {"scale_cooling": 0.0}, {"shape_start": 0}, {"target": 1.0}):
        with pytest.raises(ValueError):
            MVNRWAdaptive(rw_sd={"a": 1.0}, **bad)
    p = MVNRWAdaptive(rw_sd={"a": 0.5, "b": 0.2}, scale_start=2, shape_start=4, target=0.3)
    p = p.canonicalize(["a", "b", "c"])
    st = p.init_state(np.zeros(3))
    rng = np.random.default_rng(0)
    thetas = rng.normal(size=(8, 3))
    thetas[:, 2] = 0.0
    accepts = [0, 0, 1, 2, 3, 4, 5, 5]
    scaling, mean, cov = 1.0, None, np.zeros((3, 3))
    for n, (th, acc) in enumerate(zip(thetas, accepts), start=1):
        prop, st2 = p.step(st, th, np.uint64(1000 + n), n, acc)
        nf = float(n)
        in1 = n >= 2 and acc < 4
        if in1:
            cool = 0.999 ** max(n - 2.0, 0.0)
            scaling = min(scaling * math.exp(cool * (acc / nf - 0.3)), 50.0)
        C = (2.38 ** 2 / 3) * cov if acc >= 4 else (scaling ** 2 * p.init_rw_var if in1 else p.init_rw_var)
        m0 = th if mean is None else mean
        mean = m0 + (th - m0) / nf
        cov = ((nf - 1.0) * cov + np.outer(th - m0, th - mean)) / nf
        z = np.random.default_rng(1000 + n).standard_normal(3)
        want = th + (np.linalg.cholesky(C + 1e-10 * np.eye(3)) @ z) * np.array([1.0, 1.0, 0.0])
        assert np.allclose(prop, want, rtol=1e-12, atol=1e-12), n
        assert st2.scaling == pytest.approx(scaling) and np.allclose(st2.theta_mean, mean)
        assert np.allclose(st2.covmat_emp, cov)
        st = st2


def test_log_jacobian_matches_finite_differences():
    import pypomp_b200 as pp

    spec = pp.SV(T=5).spec
    th = np.array([0.3, -3.0, -1.1, -0.4, 0.05, -3.2])
    J = np.zeros((6, 6))
    h = 1e-6
    for i in range(6):
        e = np.zeros(6)
        e[i] = h
        J[:, i] = (spec.from_est(th + e) - spec.from_est(th - e)) / (2 * h)
    assert spec.log_det_jac_from_est(th) == pytest.approx(np.linalg.slogdet(J)[1], abs=1e-6)


def _oracle_loglik(spec, ys, J):
    ycon = spec.ycon(ys[None] if ys.ndim == 2 else ys)

    def fn(th_est, keys):
        return cora.pfilter(spec.kind, spec.dx, spec.dy, np.asarray(th_est, np.float32), ys, J,
                            seeds=np.asarray(keys, np.uint64), ycon=ycon, dt=spec.dt, est=True)["loglik"]
    return fn


def test_chains_follow_the_metropolis_hastings_rule():
    """Chains driven by the oracle's filter, rebuilt step by step from the
    reference's rule: accept iff log u < ll' + lp' - ll - lp (both finite)."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom
    from pypomp_b200.proposals import MVNDiagRW

    m = pp.Ricker(T=25, key=3)
    st = m.to_struct()
    spec = st.spec
    names = m.canonical_param_names
    th0 = m.theta.to_array(names)
    thetas = np.concatenate([th0, th0 * np.array([1.1, 1.0, 0.9, 1.0])])
    prior = lambda p: -0.5 * (math.log(p["sigma"]) + 1.0) ** 2      # noqa: E731
    prop = MVNDiagRW({"r": 0.05, "sigma": 0.1, "phi": 0.05})
    keys = np.array([11, 12], np.uint64)
    fn = _oracle_loglik(spec, st.ys, 300)
    ll, lp, th, acc = F._pmcmc_run(spec, thetas, prop, 12, keys, fn, dprior=prior)
    assert ll.shape == (2, 13) and th.shape == (2, 13, 4) and acc.shape == (2,)
    canon = prop.canonicalize(names)
    for c in range(2):
        carry, k0 = pprandom.split(keys[c], 2)
        cur = spec.to_est(thetas[c])
        ll_c = fn(cur[None], [k0])[0]
        lpc = prior(dict(zip(names, spec.from_est(cur)))) + spec.log_det_jac_from_est(cur)
        n_acc = 0
        for it in range(1, 13):
            carry, kp, kf, ka = pprandom.split(carry, 4)
            new, _ = canon.step((), cur, kp, it, n_acc)
            lpn = prior(dict(zip(names, spec.from_est(new)))) + spec.log_det_jac_from_est(new)
            lln = fn(new[None], [kf])[0]
            u = np.random.default_rng(int(ka)).random()
            la = lln + lpn - ll_c - lpc
            if np.isfinite(la) and np.isfinite(lpn) and math.log(u) < la:
                cur, ll_c, lpc, n_acc = new, lln, lpn, n_acc + 1
            assert ll[c, it] == ll_c and np.allclose(th[c, it], spec.from_est(cur))
            assert lp[c, it] == pytest.approx(prior(dict(zip(names, th[c, it]))))
        assert acc[c] == n_acc
    assert 0 < acc.sum() < 24      # some moves accepted, some rejected
