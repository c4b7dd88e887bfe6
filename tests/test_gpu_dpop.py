"""DPOP objective and gradient on the GPU against the oracle and the reference.

DPOP (``pypomp/core/algorithms/dpop.py:34-243``) runs MOP-alpha's filter and
adds the transition log-weight held in one state component of the predicted
particles to the carried weights as ``pw - stop_gradient(pw)``.

* its value equals MOP-alpha's bit for bit on the same draws, and the
  reference's locked DPOP value (``test_dpop_regression.csv``) is reproduced
  through the injection mode;
* the adjoint gradient (``PPF_F_DPOP``) matches central finite differences
  (h = 1e-3) of the DPOP surrogate with frozen ancestry, frozen
  stop_gradient(m) and frozen stop_gradient(pw) (``oracle/ppf_oracle.c``,
  ``ppfo_dpop_surrogate``) to relative error <= 1e-3, for every state
  component of LG, SV and Ricker, on the persistent and the per-step kernels;
* the reference's locked ``dpop_train`` run (``test_dpop_train_regression.csv``:
  LG 1-D, J = 12, three Adam steps at alpha = 0.8 with process_weight_index 0)
  is replayed with the reference's own draws injected into every gradient
  call and the final objective;
* ``Pomp._dpop_train`` records a ``dpop_train`` result and refuses a missing
  or unknown process-weight state as the reference does.
"""

import numpy as np
import pytest

from oracle import cora, jaxrng as jr, refpath as rp

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore:dpop")]
f32 = np.float32


def _case(model):
    import pypomp_b200 as pp

    from tests.conftest import LG2_Q, LG2_R

    if model == "LG":
        m = pp.LG(T=15, Q=LG2_Q, R=LG2_R, key=3)
        J = 1500
    elif model == "SV":
        m = pp.SV(T=30, key=1)
        J = 2048
    else:
        m = pp.Ricker(T=20, r=6.0, key=2)     # out of the chaotic regime
        J = 1600
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    return m, st, th, J


def _oracle_kw(m, st):
    spec = m.spec
    kw = {}
    if spec.name == "Ricker":
        kw["ycon"] = spec.ycon(st.ys)
    if getattr(spec, "dt", 0.0):
        kw["dt"] = spec.dt
    return kw


@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
def test_dpop_value_and_ancestors_equal_mop(model):
    from pypomp_b200 import functional as F

    m, st, th, J = _case(model)
    seeds = np.array([5, 6], np.uint64)
    th2 = np.repeat(th, 2, axis=0)
    mop = F.run_mop(st, th2, seeds, J, 0.8, grad=True, save_ancestors=True)
    for pwi in range(m.spec.dx):
        dp = F.run_mop(st, th2, seeds, J, 0.8, grad=True, save_ancestors=True, process_weight_index=pwi)
        assert np.array_equal(dp["value"], mop["value"])
        assert np.array_equal(dp["anc"], mop["anc"])
        assert np.all(np.isfinite(dp["grad"]))


@pytest.mark.parametrize("persistent", [True, False])
@pytest.mark.parametrize("alpha", [0.5, 0.97])
@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
def test_dpop_gradient_vs_finite_differences(model, alpha, persistent):
    from pypomp_b200 import functional as F

    m, st, th, J = _case(model)
    spec = m.spec
    seeds = np.array([11], np.uint64)
    kw = _oracle_kw(m, st)
    for pwi in range(spec.dx):
        got = F.run_mop(st, th, seeds, J, alpha, grad=True, save_ancestors=True, persistent=persistent,
                        process_weight_index=pwi)
        anc = got["anc"]
        base, m0, p0 = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, th, st.ys, J, alpha, anc, seeds=seeds,
                                          pwi=pwi, **kw)
        np.testing.assert_allclose(base[0], got["value"][0], rtol=1e-7)
        h = 1e-3
        P = th.shape[1]
        fd = np.zeros(P)
        for p in range(P):
            tp, tm = th.copy(), th.copy()
            tp[0, p] += f32(h)
            tm[0, p] -= f32(h)
            hp = float(tp[0, p]) - float(th[0, p])
            hm = float(th[0, p]) - float(tm[0, p])
            vp = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, tp, st.ys, J, alpha, anc, m0, seeds=seeds,
                                    pwi=pwi, p0=p0, **kw)[0]
            vm = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, tm, st.ys, J, alpha, anc, m0, seeds=seeds,
                                    pwi=pwi, p0=p0, **kw)[0]
            fd[p] = (vp[0] - vm[0]) / (hp + hm)
        g = got["grad"][0]
        err = np.linalg.norm(g - fd) / np.linalg.norm(fd)
        assert err <= 1e-3, (model, alpha, pwi, err, g, fd)
        # a transition log-weight that depends on theta changes the gradient
        # (SV's second component is the step's normal itself: no dependence)
        if not (model == "SV" and pwi == 1):
            mop = F.run_mop(st, th, seeds, J, alpha, grad=True, persistent=persistent)
            assert not np.allclose(mop["grad"], g, rtol=1e-6, atol=0), (model, pwi)


@pytest.mark.parametrize("J", [1500, 262144])
def test_dpop_persistent_forms_equal_per_step_launches(J):
    """Every adjoint form -- one launch per step, the split-phase sweep (all
    particles resident, small J) and the strided persistent sweep (large J) --
    gives the same DPOP gradient to the float64 summation order."""
    from pypomp_b200 import functional as F

    m, st, th, _ = _case("LG")
    st.ys = st.ys[:8]
    seeds = np.array([31, 32], np.uint64)
    th2 = np.repeat(th, 2, axis=0)
    th2[1, 0] += f32(0.02)
    a = F.run_mop(st, th2, seeds, J, 0.9, grad=True, persistent=True, process_weight_index=1)
    b = F.run_mop(st, th2, seeds, J, 0.9, grad=True, persistent=False, process_weight_index=1)
    assert np.array_equal(a["value"], b["value"])
    np.testing.assert_allclose(a["grad"], b["grad"], rtol=1e-9, atol=1e-12)


def _lg1d_struct(ref_lg1d):
    from pypomp_b200.functional import PompStruct
    from pypomp_b200.models import lg_spec

    return PompStruct(spec=lg_spec(1, 1), ys=ref_lg1d["ys"], times=np.arange(1, 5.0), t0=0.0)


def test_dpop_reference_fixture_through_injection(ref_values, ref_lg1d):
    from pypomp_b200 import functional as F

    st = _lg1d_struct(ref_lg1d)
    inj = dict(z0=ref_lg1d["mop_z0"][None], z=ref_lg1d["mop_z"][None], u=ref_lg1d["mop_u"][None])
    # test_dpop_regression.py passes theta0 (natural values) as estimation-scale input
    res = F.run_mop(st, ref_lg1d["theta"][None], np.zeros(1, np.uint64), 12, 0.5, inject=inj, grad=True,
                    process_weight_index=0)
    np.testing.assert_allclose(res["value"][0], ref_values["dpop"]["dpop"][0], **ref_values["tolerance"])
    assert np.all(np.isfinite(res["grad"]))


def test_dpop_train_reference_fixture_through_injection(ref_values, ref_lg1d):
    """The locked dpop_train run, step by step as ``_dpop_train_scan_step``
    (``train_dpop.py:118-171``) takes it: split the key, value and gradient of
    the mean objective, NaN -> 0, Adam, theta += 0.01 direction; then one more
    split for the final objective (``train_dpop.py:197-220``)."""
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import Adam

    st = _lg1d_struct(ref_lg1d)
    th = ref_lg1d["theta"].astype(np.float64)
    T, J, M, alpha = 4, 12, 3, 0.8
    opt = Adam()
    state = opt.init_state(th)
    key = jr.split(jr.key(20260811), 1)[0]        # keys = split(key, n_reps)

    def objective(theta, sub, grad):
        rec = rp.RecordingNoise(rp.JaxKeyNoise(sub, J, 1, 1))
        rp.mop("LG", theta.astype(np.float32), ref_lg1d["ys"], J, alpha, rec)
        z0, z, u = rec.arrays()
        return F.run_mop(st, theta.astype(np.float32)[None], np.zeros(1, np.uint64), J, alpha,
                         inject=dict(z0=z0[None], z=z[None], u=u[None]), grad=grad, process_weight_index=0)

    for m in range(M):
        s = jr.split(key)
        key, sub = s[0], s[1]
        res = objective(th, sub, True)
        grad = np.where(np.isnan(res["grad"][0]), 0.0, res["grad"][0] / T)
        direction, state = opt.step(grad, state, m)
        th = th + 0.01 * direction
    s = jr.split(key)
    final = objective(th, s[1], False)["value"][0]
    tol = ref_values["tolerance"]
    np.testing.assert_allclose(final, ref_values["dpop_train"]["final_neg_loglik"][0], **tol)
    np.testing.assert_allclose(th, ref_values["dpop_train"]["final_theta"], **tol)


def test_functional_dpop_train_shapes_and_keys():
    """functional.dpop_train: traces of shape (n, M+1, P) starting at the
    input, a final entry evaluated at the last parameters, and the same
    gradients as dpop_value_and_grad under the same key splits."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom
    from pypomp_b200.optim import SGD, LearningRate

    m = pp.LG(T=20, A=np.array([[0.8]]), C=np.array([[1.0]]), Q=np.array([[0.04]]), R=np.array([[0.09]]), key=4)
    st = m.to_struct()
    names = m.canonical_param_names
    th0 = m.spec.to_est(np.repeat(m.theta.to_array(names), 2, axis=0))
    keys = np.array([3, 4], np.uint64)
    eta = LearningRate({n: 0.01 for n in names})
    nll, tr = F.dpop_train(st, th0, 500, SGD(), 2, eta, 0.9, 0, keys)
    assert nll.shape == (2, 3) and tr.shape == (2, 3, len(names))
    np.testing.assert_allclose(tr[:, 0], th0)
    assert np.all(np.isfinite(nll)) and np.all(np.isfinite(tr))
    # step 0 by hand: first split of each key, mean objective's gradient
    subs = np.array([pprandom.split(int(k))[1] for k in keys], np.uint64)
    v, g = F.dpop_value_and_grad(st, th0, 500, 0.9, 0, subs)
    np.testing.assert_allclose(nll[:, 0], v * st.ys.shape[0], rtol=1e-12)
    direction, _ = SGD().step(g, SGD().init_state(th0), 0, eta_i=eta.to_array(names, 2)[0])
    np.testing.assert_allclose(tr[:, 1], th0 + eta.to_array(names, 2)[0] * direction, rtol=1e-6, atol=1e-9)


def test_pomp_dpop_train_result_and_errors():
    import pypomp_b200 as pp
    from pypomp_b200.optim import LearningRate

    m = pp.LG(T=25, key=6)
    eta = LearningRate({n: 0.005 for n in m.canonical_param_names})
    with pytest.raises(ValueError, match="process-weight state"):
        m._dpop_train(J=200, M=2, eta=eta)
    with pytest.raises(ValueError, match="not found in statenames"):
        m._dpop_train(J=200, M=2, eta=eta, process_weight_state="logw")
    with pytest.warns(FutureWarning, match="experimental"):
        m._dpop_train(J=400, M=3, eta=eta, process_weight_state=m.statenames[0], key=9)
    r = m.results_history[-1]
    assert r.method == "dpop_train" and r.config["process_weight_state"] == m.statenames[0]
    tr = m.results_history.traces()
    assert set(tr["method"]) == {"dpop_train"} and tr["iteration"].max() == 3
    assert np.all(np.isfinite(m.theta.logLik))


def test_panel_dpop_train_first_iteration_by_hand():
    """Panel DPOP training (``train_panel_dpop.py:152-322``) on a ragged
    Ricker panel: the first entry is the summed DPOP objective of all units at
    the start under iteration 0's keys, the first chunk's shared and unit
    update follows from one batched DPOP gradient by hand, and
    ``PanelPomp._dpop_train`` fills the panel result tables."""
    import pandas as pd

    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.functional import _panel_thetas
    from pypomp_b200.optim import SGD, LearningRate

    units = {f"u{i}": pp.Ricker(T=T, r=6.0, key=50 + i) for i, T in enumerate((20, 30, 25))}
    shared = pd.DataFrame({"shared": [0.3, 10.0]}, index=["sigma", "phi"])
    spec_df = pd.DataFrame([[6.0, 5.5, 6.5], [7.0, 6.0, 8.0]], index=["r", "N_0"], columns=list(units))
    pan = pp.PanelPomp(units, pp.PanelParameters({"shared": shared, "unit_specific": spec_df}))
    st = pan.to_struct()
    names = st.unit_names
    sn, un = pan.canonical_shared_param_names, pan.canonical_unit_param_names
    sh, ua = pan.theta.shared_array(sn), pan.theta.unit_array(names, un)
    keys = (np.arange(2 * 3, dtype=np.uint64) + np.uint64(70)).reshape(1, 2, 3)
    J, U = 1000, 3
    eta = LearningRate({n: 0.01 for n in list(sn) + list(un)})
    nll, hs, hu = F.panel_dpop_train(st, sh, ua, J, SGD(), 2, eta, 0.9, 0, keys, chunk_size=U)
    assert nll.shape == (1, 3) and np.all(np.isfinite(nll)) and np.all(np.isfinite(hu))
    # the objective at the start, iteration 0's keys, every unit
    th0 = _panel_thetas(sh, ua, st.permutations).reshape(U, -1)
    est0 = st.spec.to_est(th0).astype(np.float32)
    v0 = F.run_mop(st.all_units(), est0, keys[0, 0], J, 0.9, grad=True, unit_f=np.arange(U, dtype=np.int32),
                   process_weight_index=0)
    np.testing.assert_allclose(nll[0, 0], v0["value"].sum(), rtol=1e-12)
    # iteration 0 is one chunk of all units: its value is the same call's
    np.testing.assert_allclose(nll[0, 1], v0["value"].sum(), rtol=1e-12)
    with pytest.warns(FutureWarning, match="experimental"):
        pan._dpop_train(J=800, M=2, eta=eta, chunk_size=2, process_weight_state="N", key=4)
    assert pan.results_history[-1].method == "dpop_train"
    assert pan.results_history[-1].config["chunk_size"] == 1       # 2 does not divide 3
    assert np.all(np.isfinite(pan.results()["shared logLik"]))
    with pytest.raises(ValueError, match="not found in statenames"):
        pan._dpop_train(J=800, M=1, eta=eta, process_weight_state="logw")
