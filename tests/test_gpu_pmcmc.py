"""PMCMC on the GPU: the chains equal those driven by the C oracle's filter.

Every iteration filters all chains in one batched ppf_pfilter launch
(replayed from a CUDA graph).  The GPU log-likelihoods equal the oracle's to
float64 rounding of log(), so the accept decisions, and with them the
parameter traces, are the same.  The OO method is checked for the
reference's result layout (pypomp/core/estimation_mixin.py:823-935,
pypomp/core/results/render.py:419-440).
"""

import math

import numpy as np
import pytest

from oracle import cora

pytestmark = pytest.mark.gpu


def _oracle_loglik(spec, ys, J):
    ycon = spec.ycon(ys[None] if ys.ndim == 2 else ys)

    def fn(th_est, keys):
        return cora.pfilter(spec.kind, spec.dx, spec.dy, np.asarray(th_est, np.float32), ys, J,
                            seeds=np.asarray(keys, np.uint64), ycon=ycon, dt=spec.dt, est=True)["loglik"]
    return fn


@pytest.mark.parametrize("model", ["ricker", "lg2"])
def test_gpu_chains_equal_oracle_chains(model):
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.proposals import MVNDiagRW, MVNRWAdaptive

    if model == "ricker":
        m = pp.Ricker(T=40, key=2)
        prop = MVNRWAdaptive(rw_sd={"r": 0.05, "sigma": 0.1, "phi": 0.05}, scale_start=3, shape_start=5)
        prior = lambda p: -0.5 * (math.log(p["sigma"]) + 1.0) ** 2      # noqa: E731
    else:
        m = pp.LG(T=30, key=2)
        prop = MVNDiagRW({"A11": 0.02, "A22": 0.02, "Q11": 0.05, "R11": 0.05})
        prior = None
    st = m.to_struct()
    names = m.canonical_param_names
    th0 = m.theta.to_array(names)
    thetas = np.concatenate([th0, th0, th0])
    keys = np.array([5, 6, 7], np.uint64)
    J, M = 700, 15
    got = F.pmcmc(st, thetas, prop, M, J, keys, dprior=prior)
    want = F._pmcmc_run(st.spec, thetas, prop, M, keys, _oracle_loglik(st.spec, st.ys, J), dprior=prior)
    assert np.allclose(got[0], want[0], rtol=1e-12, atol=0)
    assert np.allclose(got[1], want[1], rtol=1e-12, atol=0)
    assert np.array_equal(got[2], want[2])
    assert np.array_equal(got[3], want[3])
    assert got[3].sum() > 0


def test_pomp_pmcmc_results_layout():
    import pypomp_b200 as pp
    from pypomp_b200.proposals import MVNDiagRW

    m = pp.Ricker(T=30, key=1)
    th = m.theta.params()[0]
    m.pmcmc(J=400, M=8, proposal=MVNDiagRW({"r": 0.05, "sigma": 0.05}), key=3, theta=[th, th])
    res = m.results()
    assert list(res.columns) == ["theta_idx", "iteration", "logLik", "log_prior"] + m.canonical_param_names
    assert len(res) == 2 * 9 and np.all(res["log_prior"] == 0.0)
    tr = m.traces()
    assert list(tr.columns[:6]) == ["theta_idx", "iteration", "method", "logLik", "se", "log_prior"]
    r = m.results_history[-1]
    assert r.acceptance_rate.shape == (2,) and np.all((0 <= r.acceptance_rate) & (r.acceptance_rate <= 1))
    assert m.theta.num_replicates() == 2 and np.all(np.isfinite(m.theta.logLik))
    with pytest.raises(ValueError, match="M must be"):
        m.pmcmc(J=10, M=0, proposal=MVNDiagRW({"r": 0.1}), key=1)
