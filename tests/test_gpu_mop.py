"""MOP-alpha value and adjoint gradient on the GPU against the oracle.

* the reference's locked MOP value (``test_mop_regression.csv``) is reproduced
  by feeding the reference's own draws through the injection mode;
* forward ancestors are bit-identical to the C oracle's MOP run;
* the adjoint gradient matches central finite differences (h = 1e-3) of the
  MOP-alpha surrogate with frozen ancestry and frozen stop_gradient(m)
  (``oracle/ppf_oracle.c``, ``ppfo_mop_surrogate``) to relative error <= 1e-3;
* the gradient does not depend on the checkpoint spacing (to float64 rounding
  of the cross-block accumulation).
"""

import numpy as np
import pytest

from oracle import cora

pytestmark = pytest.mark.gpu
f32 = np.float32


def _F():
    from pypomp_b200 import functional as F

    return F


def test_mop_reference_fixture_through_injection(ref_values, ref_lg1d):
    F = _F()
    from pypomp_b200.functional import PompStruct
    from pypomp_b200.models import lg_spec

    st = PompStruct(spec=lg_spec(1, 1), ys=ref_lg1d["ys"], times=np.arange(1, 5.0), t0=0.0)
    inj = dict(z0=ref_lg1d["mop_z0"][None], z=ref_lg1d["mop_z"][None], u=ref_lg1d["mop_u"][None])
    # test_mop_regression.py passes theta0 (natural values) as estimation-scale input
    res = F.run_mop(st, ref_lg1d["theta"][None], np.zeros(1, np.uint64), 12, 0.5, inject=inj, grad=True)
    np.testing.assert_allclose(res["value"][0], ref_values["mop"]["mop"][0], **ref_values["tolerance"])
    assert np.all(np.isfinite(res["grad"]))


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
        # r = 6 keeps the map out of its chaotic regime (log r = 3.8 is chaotic:
        # pathwise derivatives grow ~40x per step and central differences with
        # h = 1e-3 leave the linear regime)
        m = pp.Ricker(T=20, r=6.0, key=2)
        J = 1600
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    return m, st, th, J


def _oracle_kw(m, st):
    spec = m.spec
    return dict(ycon=spec.ycon(st.ys), dt=spec.dt)


@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
def test_mop_forward_ancestors_bit_exact(model):
    F = _F()
    m, st, th, J = _case(model)
    spec = m.spec
    seeds = np.array([5, 6], np.uint64)
    th2 = np.repeat(th, 2, axis=0)
    th2[1, 0] += f32(0.01)
    want = cora.pfilter(spec.kind, spec.dx, spec.dy, th2, st.ys, J, seeds=seeds, est=True, mop=True,
                        anc=True, **_oracle_kw(m, st))
    got = F.run_mop(st, th2, seeds, J, 0.97, grad=False, save_ancestors=True)
    assert np.array_equal(got["anc"], want["anc"])
    np.testing.assert_allclose(got["value"], -want["loglik"], rtol=1e-12)


@pytest.mark.parametrize("alpha", [0.0, 0.5, 0.97, 1.0])
@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
def test_mop_gradient_vs_finite_differences(model, alpha):
    F = _F()
    m, st, th, J = _case(model)
    spec = m.spec
    seeds = np.array([11], np.uint64)
    kw = _oracle_kw(m, st)
    got = F.run_mop(st, th, seeds, J, alpha, grad=True, save_ancestors=True)
    anc = got["anc"]
    base, m0 = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, th, st.ys, J, alpha, anc, seeds=seeds, **kw)
    np.testing.assert_allclose(base[0], got["value"][0], rtol=1e-7)
    h = 1e-3
    P = th.shape[1]
    fd = np.zeros(P)
    for p in range(P):
        tp = th.copy()
        tm = th.copy()
        tp[0, p] += f32(h)
        tm[0, p] -= f32(h)
        hp = float(tp[0, p]) - float(th[0, p])
        hm = float(th[0, p]) - float(tm[0, p])
        vp, _ = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, tp, st.ys, J, alpha, anc, m0, seeds=seeds, **kw)
        vm, _ = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, tm, st.ys, J, alpha, anc, m0, seeds=seeds, **kw)
        fd[p] = (vp[0] - vm[0]) / (hp + hm)
    g = got["grad"][0]
    err = np.linalg.norm(g - fd) / np.linalg.norm(fd)
    assert err <= 1e-3, (model, alpha, err, g, fd)


def test_mop_gradient_independent_of_checkpoint_spacing():
    F = _F()
    m, st, th, J = _case("SV")
    seeds = np.array([3], np.uint64)
    ref = F.run_mop(st, th, seeds, J, 0.97, grad=True, ckpt_every=1)
    for ck in (2, 7, 0, 30):
        got = F.run_mop(st, th, seeds, J, 0.97, grad=True, ckpt_every=ck)
        # recomputation is bit-exact; only the cross-block float64 atomic
        # accumulation of the gradient sums may change the last bits
        np.testing.assert_allclose(got["grad"], ref["grad"], rtol=1e-12, atol=1e-12, err_msg=str(ck))
        assert np.array_equal(got["value"], ref["value"])


def test_mop_gradient_finite_for_chaotic_ricker_with_zero_counts():
    """Chaotic Ricker series have runs of zero counts and particles whose
    predicted count all but vanishes; their weights underflow, and the adjoint
    must form y / N' products without overflowing (no 0 * inf or inf - inf).
    The series are kept to 120 steps: along a chaotic lineage the pathwise
    state derivative grows by the map's Lyapunov factor every step and leaves
    float32 range after a few hundred steps, whatever the arithmetic order."""
    import math

    import pypomp_b200 as pp

    F = _F()
    for i, logr in enumerate((3.75, 3.87, 4.12)):
        m = pp.Ricker(T=120, r=math.exp(logr), key=1000 + i)
        st = m.to_struct()
        assert np.any(st.ys == 0)
        th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
        got = F.run_mop(st, th, np.array([i], np.uint64), 8192, 0.97, grad=True)
        assert np.all(np.isfinite(got["value"])) and np.all(np.isfinite(got["grad"])), (logr, got["grad"])


@pytest.mark.parametrize("alpha", [0.5, 0.97])
@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
def test_persistent_form_equals_per_step_launches(model, alpha):
    """The persistent MOP (forward and adjoint sweep as two cooperative
    launches) against one launch per step: values and ancestors bit for bit;
    the gradient to the float64 summation order of its terms."""
    F = _F()
    m, st, th, J = _case(model)
    seeds = np.array([21, 22], np.uint64)
    th2 = np.repeat(th, 2, axis=0)
    th2[1, 0] += f32(0.02)
    a = F.run_mop(st, th2, seeds, J, alpha, grad=True, save_ancestors=True, persistent=True)
    b = F.run_mop(st, th2, seeds, J, alpha, grad=True, save_ancestors=True, persistent=False)
    assert np.array_equal(a["anc"], b["anc"])
    assert np.array_equal(a["value"], b["value"])
    tol = 1e-9
    for f in range(2):
        assert np.linalg.norm(a["grad"][f] - b["grad"][f]) <= tol * np.linalg.norm(b["grad"][f]), \
            (a["grad"][f], b["grad"][f])


def test_persistent_form_on_ragged_panel_units():
    """Panel MOP with units of different lengths through the persistent form
    (filters stop at their own T_u inside the launch) against per-step launches."""
    import pypomp_b200 as pp
    from pypomp_b200.functional import PompStruct

    F = _F()
    units = [pp.Ricker(T=T, r=6.0, key=30 + i) for i, T in enumerate((25, 40, 13))]
    spec = units[0].spec
    Tmax = 40
    ys = np.zeros((3, Tmax, 1), f32)
    for i, mm in enumerate(units):
        y = mm.to_struct().ys
        ys[i, :y.shape[0]] = y
    st = PompStruct(spec=spec, ys=ys, times=np.arange(1, Tmax + 1.0), t0=0.0,
                    T_u=np.array([25, 40, 13], np.int32))
    th = np.stack([spec.to_est(mm.theta.to_array(mm.canonical_param_names))[0] for mm in units]).astype(f32)
    seeds = np.array([5, 6, 7], np.uint64)
    unit_f = np.arange(3, dtype=np.int32)
    a = F.run_mop(st, th, seeds, 3000, 0.97, grad=True, unit_f=unit_f, persistent=True)
    b = F.run_mop(st, th, seeds, 3000, 0.97, grad=True, unit_f=unit_f, persistent=False)
    assert np.array_equal(a["value"], b["value"])
    np.testing.assert_allclose(a["grad"], b["grad"], rtol=1e-9, atol=1e-12)


def test_persistent_form_at_config_size_equals_per_step_launches():
    """C3's shape (SV, T = 2000, J = 65536): the persistent form gives the
    per-step launches' value bit for bit and their gradient to 1e-9."""
    import pypomp_b200 as pp

    F = _F()
    m = pp.SV(T=2000, key=0)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    seeds = np.array([1], np.uint64)
    a = F.run_mop(st, th, seeds, 65536, 0.97, grad=True, persistent=True)
    b = F.run_mop(st, th, seeds, 65536, 0.97, grad=True, persistent=False)
    assert np.array_equal(a["value"], b["value"])
    np.testing.assert_allclose(a["grad"], b["grad"], rtol=1e-9)


def test_persistent_form_replays_from_a_cuda_graph():
    """PPF_F_GRAPH captures the persistent form's two cooperative launches once
    and replays them: the replay equals a direct call."""
    import pypomp_b200 as pp
    from pypomp_b200.functional import MopCall

    m = pp.SV(T=200, key=4)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    seeds = np.array([3], np.uint64)
    direct = MopCall(st, th, seeds, 16384, 0.97)
    want = {k: v.cpu().numpy() for k, v in direct.forward(grad=True).items()}
    g = MopCall(st, th, seeds, 16384, 0.97, graph=True)
    for _ in range(3):
        got = {k: v.cpu().numpy() for k, v in g.forward(grad=True).items()}
        assert np.array_equal(got["value"], want["value"])
        np.testing.assert_allclose(got["grad"], want["grad"], rtol=1e-12)
