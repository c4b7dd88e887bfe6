"""IF2 (perturbed filter + mif loop) on the GPU against the oracle.

* ``ppf_perfilter`` is bit-identical to the C oracle's restatement
  (``oracle/ppf_oracle.c`` ``ppfo_perfilter``) for LG 2-D, SV and Ricker:
  ancestors, conditional log-likelihoods, log-likelihood and final swarm,
  with one and several tiles per swarm, thresh 0 and 20, on the
  cluster-resident path (chosen for these few small swarms) and on the
  streaming kernels;
* with zero random-walk sds the perturbed filter is the bootstrap filter
  (same ancestors and log-likelihoods bit for bit);
* ``functional.mif`` replaying the reference's own draws reproduces the
  locked ``test_mif_regression.csv`` and ``test_mif_full_trace_regression.csv``
  (tolerance of the reference's regression tests);
* ``Pomp.mif`` runs end to end on Philox draws and fills the result tables.
"""

import numpy as np
import pytest

from oracle import cora

pytestmark = pytest.mark.gpu
f32 = np.float32


def _F():
    from pypomp_b200 import functional as F

    return F


def _case(model):
    import pypomp_b200 as pp

    from tests.conftest import LG2_Q, LG2_R

    if model == "LG":
        m = pp.LG(T=12, Q=LG2_Q, R=LG2_R, key=3)
    elif model == "SV":
        m = pp.SV(T=25, key=1)
    else:
        m = pp.Ricker(T=15, key=2)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    return m, st, th


def _swarm(th, F, J, seed):
    rng = np.random.default_rng(seed)
    P = th.shape[1]
    return (np.repeat(th[:, :, None], J, axis=2).repeat(F, axis=0)
            + f32(0.01) * rng.standard_normal((F, P, J)).astype(f32)).astype(f32)


@pytest.mark.parametrize("stream_only", [False, True])
@pytest.mark.parametrize("thresh", [0.0, 20.0])
@pytest.mark.parametrize("J", [1000, 5000])
@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
def test_perfilter_bit_exact_vs_oracle(model, J, thresh, stream_only):
    F = _F()
    m, st, th = _case(model)
    spec = m.spec
    nF, P, T = 3, th.shape[1], st.ys.shape[0]
    swarm = _swarm(th, nF, J, 5)
    sig = np.full(P, 0.02, f32)
    sig0 = np.zeros(P, f32)
    sig0[-1] = 0.05
    cool = (0.98 ** np.arange(T)).astype(f32)
    seeds = np.array([11, 12, 13], np.uint64)
    want = cora.perfilter(spec.kind, spec.dx, spec.dy, swarm, st.ys, J, sig, sig0, cool, f32(0.99),
                          seeds=seeds, ycon=spec.ycon(st.ys), dt=spec.dt, thresh=thresh, CLL=True, anc=True)
    got = F.run_perfilter(st, swarm.transpose(0, 2, 1), seeds, J, sig, sig0, cool, f32(0.99), thresh=thresh,
                          CLL=True, save_ancestors=True, stream_only=stream_only)
    assert np.array_equal(got["anc"], want["anc"])
    assert np.array_equal(got["swarm"], want["swarm"].transpose(0, 2, 1))
    np.testing.assert_allclose(got["cll"], want["cll"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12)


@pytest.mark.parametrize("thresh", [0.0, 20.0])
def test_perfilter_without_perturbation_is_pfilter(lg2d, thresh):
    F = _F()
    st = lg2d.to_struct()
    th = lg2d.spec.to_est(lg2d.theta.to_array(lg2d.canonical_param_names)).astype(f32)
    P, J, T = th.shape[1], 4096, st.ys.shape[0]
    th2 = np.repeat(th, 2, axis=0)
    th2[1, 0] += f32(0.01)
    seeds = np.array([7, 8], np.uint64)
    zero = np.zeros(P, f32)
    swarm = np.repeat(th2[:, None, :], J, axis=1)
    got = F.run_perfilter(st, swarm, seeds, J, zero, zero, np.ones(T, f32), 1.0, thresh=thresh,
                          CLL=True, save_ancestors=True)
    want = F.run_pfilter(st, th2, seeds, J, thresh=thresh, est=True, CLL=True, save_ancestors=True,
                         path="stream")
    assert np.array_equal(got["anc"], want["anc"])
    assert np.array_equal(got["cll"], want["cll"])
    assert np.array_equal(got["loglik"], want["loglik"])


def _rw():
    from pypomp_b200.optim import RWSigma

    return RWSigma({n: 0.02 for n in ("A11", "C11", "Q11", "R11", "X0_1")}).geometric_cooling(0.5)


def _struct(ref_lg1d):
    from pypomp_b200.functional import PompStruct
    from pypomp_b200.models import lg_spec

    return PompStruct(spec=lg_spec(1, 1), ys=ref_lg1d["ys"], times=np.arange(1, 5.0), t0=0.0)


def test_mif_reference_fixture_through_injection(ref_values, ref_lg1d):
    F = _F()
    tol = ref_values["tolerance"]
    st = _struct(ref_lg1d)
    theta = ref_lg1d["theta"]
    inj = [{"perfilter": {k: ref_lg1d[f"mif_{k}"][it][None] for k in ("zp0", "zp", "z0", "z", "u")},
            "monitors": []} for it in range(3)]
    swarm = np.repeat(theta[None, None, :], 12, axis=1)
    ll, tr, final = F.mif(st, swarm, _rw(), 3, 12, np.zeros(1, np.uint64), 0.0, 0, inject=inj)
    np.testing.assert_allclose(ll[0, -1], ref_values["mif"]["final_loglik"][0], **tol)
    np.testing.assert_allclose(tr[0, -1], ref_values["mif"]["final_theta"], **tol)
    assert final.shape == (1, 12, 5)


def test_mif_full_trace_fixture_through_injection(ref_values, ref_lg1d):
    F = _F()
    tol = ref_values["tolerance"]
    gold = ref_values["mif_full_trace"]
    st = _struct(ref_lg1d)
    theta = ref_lg1d["theta"]
    thetas = np.stack([theta, (theta * f32(1.05)).astype(f32)])
    inj = [{"perfilter": {k: ref_lg1d[f"mift_{k}"][:, it] for k in ("zp0", "zp", "z0", "z", "u")},
            "monitors": [{k: ref_lg1d[f"mift_mon_{k}"][:, it] for k in ("z0", "z", "u")}]}
           for it in range(4)]
    swarm = np.repeat(thetas[:, None, :], 12, axis=1)
    ll, tr, _ = F.mif(st, swarm, _rw(), 4, 12, np.zeros(2, np.uint64), 0.0, 1, inject=inj)
    names = ["A11", "C11", "Q11", "R11", "X0_1"]
    for r in range(2):
        np.testing.assert_allclose(ll[r], [gold[f"loglik_rep{r}_m{m}"][0] for m in range(4)], **tol)
        want = [[gold[f"{n}_rep{r}_m{m}"][0] for n in names] for m in range(5)]
        np.testing.assert_allclose(tr[r], want, **tol)


def test_pomp_mif_end_to_end(lg2d):
    import copy

    from pypomp_b200.optim import RWSigma

    m = copy.deepcopy(lg2d)
    names = m.canonical_param_names
    rw = RWSigma({n: 0.02 for n in names}, init_names=[names[-1]]).geometric_cooling(0.5)
    th = m.theta.params()[0]
    m.mif(J=2000, M=3, rw_sd=rw, key=5, theta=[th, th], n_monitors=1)
    res = m.results()
    assert list(res.columns[:3]) == ["theta_idx", "logLik", "se"]
    assert len(res) == 2 and np.all(np.isfinite(res["logLik"]))
    tr = m.traces()
    assert len(tr) == 2 * 4 and np.isnan(tr[tr["iteration"] == 0]["logLik"]).all()
    assert m.theta.num_replicates() == 2


def test_mif_moves_toward_kalman_mle():
    """IF2 from a perturbed start raises the exact (Kalman) log-likelihood of
    its final mean parameters (the reference's accuracy check,
    tests/test_accuracy/test_accuracy_pomp.py:73-97)."""
    import pypomp_b200 as pp
    from oracle.kalman import kalman_loglik, lg_matrices
    from pypomp_b200.optim import RWSigma

    m = pp.LG(T=100, A=[[0.8]], C=[[1.0]], Q=[[0.5]], R=[[0.5]], X0=[0.0], key=11)
    names = m.canonical_param_names
    truth = m.theta.params()[0]
    start = {**truth, "A11": 0.4, "Q11": 1.2, "R11": 0.2}

    def kal(p):
        A, C, Q, R, X0 = lg_matrices(np.array([p[n] for n in names]), 1, 1)
        return kalman_loglik(m.to_struct().ys, A, C, Q, R, X0)
    rw = RWSigma({"A11": 0.02, "C11": 0.0, "Q11": 0.02, "R11": 0.02, "X0_1": 0.0}).geometric_cooling(0.5)
    m.mif(J=2000, M=25, rw_sd=rw, key=3, theta=[start])
    end = m.theta.params()[0]
    assert kal(end) > kal(start) + 5.0, (kal(start), kal(end), end)


def test_oo_and_functional_pfilter_agree_exactly(lg2d):
    """Pomp.pfilter is functional.pfilter under the keys it derives
    (the reference's tests/test_properties/test_layer_parity.py)."""
    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom

    th = lg2d.theta.to_array(lg2d.canonical_param_names)
    lg2d.pfilter(J=700, key=5, reps=3)
    oo = lg2d.results_history[-1].payload["logLiks"]
    keys = pprandom.split(pprandom.split(pprandom.as_key(5))[1], 3).reshape(1, 3)
    fn = F.pfilter(lg2d.to_struct(), th, 700, keys)["logLik"]
    assert np.array_equal(oo, fn)


@pytest.mark.parametrize("J", [3000, 40000])
def test_mif_graph_replay_equals_per_iteration_calls(J):
    """functional.mif runs its iterations on persistent device buffers
    (PerfilterCall); the result equals separate ppf_perfilter calls exactly,
    on the cluster path (J = 3000) and the stream path (J = 40000), and so
    does a graph-replayed PerfilterCall."""
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom
    from pypomp_b200.optim import RWSigma

    m = pp.Ricker(T=30, key=4)
    st = m.to_struct()
    names = m.canonical_param_names
    th = m.theta.to_array(names)
    starts = np.repeat(np.repeat(th[:, None, :], J, axis=1), 2, axis=0).astype(np.float32)
    rw = RWSigma({n: 0.03 for n in names}).geometric_cooling(0.5)
    keys = np.array([8, 9], np.uint64)
    M = 3
    ll, traces, final = F.mif(st, starts, rw, M, J, keys)
    rw_sig, rw_sig0 = rw.arrays(names)
    est = st.spec.to_est(starts.reshape(-1, 4)).reshape(starts.shape).astype(np.float32)
    swarm = torch.from_numpy(np.ascontiguousarray(est.transpose(0, 2, 1))).cuda()
    m_keys = np.stack([pprandom.split(k, M + 1)[1:] for k in keys])
    for it in range(M):
        cool = np.array([rw.cooling_factor(i, it, 30) for i in range(30)], dtype=np.float32)
        res = F.run_perfilter(st, swarm, m_keys[:, it], J, rw_sig, rw_sig0, cool, cool[0])
        assert np.array_equal(res["loglik"].cpu().numpy(), ll[:, it])
        swarm = res["swarm"]
    want = st.spec.from_est(swarm.cpu().numpy().transpose(0, 2, 1).reshape(-1, 4)).reshape(final.shape)
    assert np.array_equal(want, final)
    sw0 = torch.from_numpy(np.ascontiguousarray(est.transpose(0, 2, 1))).cuda()
    call = F.PerfilterCall(st, sw0, J, rw_sig, rw_sig0, graph=True)
    for it in range(M):
        cool = np.array([rw.cooling_factor(i, it, 30) for i in range(30)], dtype=np.float32)
        assert np.array_equal(call(m_keys[:, it], cool, cool[0]), ll[:, it])
    assert np.array_equal(call.swarm.cpu().numpy(), swarm.cpu().numpy())


def test_mif_device_loop_equals_host_loop():
    """The device-side IF2 loop (cooling factors and keys uploaded once, no
    host wait per iteration) gives the host loop's traces, log-likelihoods and
    final swarm bit for bit."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import RWSigma

    m = pp.Ricker(T=60, key=5)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names)[:, None, :], 3000, axis=1)
    th = np.repeat(th, 2, axis=0)
    rw = RWSigma({n: 0.03 for n in m.canonical_param_names}).geometric_cooling(0.5)
    keys = np.array([4, 5], np.uint64)
    a = F.mif(st, th, rw, 4, 3000, keys, device_loop=True)
    b = F.mif(st, th, rw, 4, 3000, keys, device_loop=False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
