"""Parity of the CUDA particle filter with the oracle (GPU).

Every execution path (plain, stream, resident) is compared with the C oracle
bit for bit on log-weights and resampling ancestors, in both noise-injection
and Philox modes; log-likelihoods agree to float64 rounding of log().  The
reference's own locked fixtures are reproduced by feeding the reference's
draws through the injection mode.  Edge cases: J=1, T=1, partial tiles,
thresh > 1 (steps without resampling), ragged panels, collapsed weights,
non-finite parameters; the stream path with each of its tile sizes; the
cluster-resident path (swarm split over a thread-block cluster's shared
memory).
"""

import numpy as np
import pytest

from oracle import cora, kalman

pytestmark = pytest.mark.gpu

PATHS = ["plain", "stream", "stream@2048", "stream@512", "stream@256", "resident", "cluster"]
f32 = np.float32


def _F():
    from pypomp_b200 import functional as F

    return F


def _bits_equal(a, b):
    a = np.asarray(a, f32)
    b = np.asarray(b, f32)
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    return bool(np.all(same))


def _compare(got, want, what):
    assert np.array_equal(got["anc"], want["anc"]), f"{what}: ancestors differ"
    assert _bits_equal(got["logw"], want["logw"]), f"{what}: log-weights differ"
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12, atol=1e-12, err_msg=what)
    if "cll" in want:
        np.testing.assert_allclose(got["cll"], want["cll"], rtol=1e-12, atol=1e-12, err_msg=what)
    if "ess" in want:
        np.testing.assert_allclose(got["ess"], want["ess"], rtol=1e-5, err_msg=what)
    for k in ("fmean", "pmean"):
        if k in want:
            np.testing.assert_allclose(got[k], want[k], rtol=1e-5, atol=1e-6, err_msg=what)


def _models():
    import pypomp_b200 as pp

    from tests.conftest import LG2_Q, LG2_R

    lg = pp.LG(T=12, Q=LG2_Q, R=LG2_R, key=3)
    sv = pp.SV(T=12, key=1)
    rk = pp.Ricker(T=12, key=2)
    return {"LG": lg, "SV": sv, "Ricker": rk}


def _thetas(m, F):
    th = np.repeat(m.theta.to_array(m.canonical_param_names), F, axis=0).astype(f32)
    for f in range(1, F):
        th[f, 0] *= f32(1.0 - 0.03 * f)
    return th


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("model", ["LG", "SV", "Ricker"])
@pytest.mark.parametrize("J", [1, 777, 5000])
def test_philox_mode_bit_exact(path, model, J):
    F = _F()
    m = _models()[model]
    st = m.to_struct()
    th = _thetas(m, 3)
    seeds = np.array([3, 1000, 77], np.uint64)
    spec = m.spec
    ycon = spec.ycon(st.ys)
    want = cora.pfilter(spec.kind, spec.dx, spec.dy, th, st.ys, J, seeds=seeds, ycon=ycon,
                        dt=spec.dt, anc=True, logw=True, CLL=True, ESS=True, fmean=True, pmean=True)
    got = F.run_pfilter(st, th, seeds, J, path=path, save_ancestors=True, save_weights=True,
                        CLL=True, ESS=True, filter_mean=True, prediction_mean=True)
    _compare(got, want, f"{model}/{path}/J={J}")


@pytest.mark.parametrize("path", PATHS)
def test_injection_mode_bit_exact_lg2d(path, lg2d):
    F = _F()
    st = lg2d.to_struct()
    th = lg2d.theta.to_array(lg2d.canonical_param_names).astype(f32)
    J, T = 4096, 50
    rng = np.random.default_rng(1234)
    inj = dict(z0=rng.standard_normal((1, J, 2)).astype(f32),
               z=rng.standard_normal((1, T, J, 2)).astype(f32), u=rng.random((1, T)).astype(f32))
    want = cora.pfilter(1, 2, 2, th, st.ys, J, inject=inj, anc=True, logw=True, CLL=True, ESS=True)
    got = F.run_pfilter(st, th, np.zeros(1, np.uint64), J, path=path, inject=inj,
                        save_ancestors=True, save_weights=True, CLL=True, ESS=True)
    _compare(got, want, f"inject/{path}")


@pytest.mark.parametrize("path", PATHS)
def test_reference_fixtures_through_injection(path, ref_values, ref_lg1d):
    """The reference's own normals and uniforms reproduce its locked values."""
    F = _F()
    from pypomp_b200.models import lg_spec
    from pypomp_b200.functional import PompStruct

    tol = ref_values["tolerance"]
    st = PompStruct(spec=lg_spec(1, 1), ys=ref_lg1d["ys"], times=np.arange(1, 5.0), t0=0.0)
    inj = dict(z0=ref_lg1d["diag_z0"], z=ref_lg1d["diag_z"], u=ref_lg1d["diag_u"])
    got = F.run_pfilter(st, ref_lg1d["diag_theta"], np.zeros(2, np.uint64), 12, path=path,
                        inject=inj, CLL=True, ESS=True, filter_mean=True, prediction_mean=True)
    gold = ref_values["pfilter_diagnostics"]
    for r in range(2):
        np.testing.assert_allclose(got["loglik"][r], gold["logLik"][r], **tol)
        for t in range(4):
            np.testing.assert_allclose(got["cll"][r, t], gold[f"CLL_rep{r}_t{t}"][0], **tol)
            np.testing.assert_allclose(got["ess"][r, t], gold[f"ESS_rep{r}_t{t}"][0], **tol)
            np.testing.assert_allclose(got["fmean"][r, t, 0], gold[f"filter_mean_rep{r}_t{t}"][0], **tol)
            np.testing.assert_allclose(got["pmean"][r, t, 0], gold[f"prediction_mean_rep{r}_t{t}"][0], **tol)
    inj = dict(z0=ref_lg1d["pf_z0"][None], z=ref_lg1d["pf_z"][None], u=ref_lg1d["pf_u"][None])
    got = F.run_pfilter(st, ref_lg1d["theta"][None], np.zeros(1, np.uint64), 12, path=path, inject=inj)
    np.testing.assert_allclose(got["loglik"][0], ref_values["pfilter"]["logLik"][0], **tol)


@pytest.mark.parametrize("path", PATHS)
def test_thresh_ragged_panel_and_T1(path):
    F = _F()
    import pypomp_b200 as pp
    from pypomp_b200.functional import PompStruct

    units = [pp.Ricker(T=9, key=k) for k in range(3)]
    ys = np.stack([u.ys.to_numpy(dtype=f32) for u in units])
    T_u = np.array([5, 9, 1], np.int32)
    st = PompStruct(spec=units[0].spec, ys=ys, times=np.arange(1, 10.0), t0=0.0, T_u=T_u)
    th = _thetas(units[0], 6)
    unit = np.array([0, 1, 2, 0, 1, 2], np.int32)
    seeds = np.arange(6, dtype=np.uint64) * 7 + 1
    spec = units[0].spec
    for thresh in (0.0, 20.0):
        want = cora.pfilter(spec.kind, 1, 1, th, ys, 3000, seeds=seeds, ycon=spec.ycon(ys), unit=unit,
                            T_u=T_u, thresh=thresh, anc=True, logw=True, CLL=True)
        got = F.run_pfilter(st, th, seeds, 3000, thresh=thresh, unit_f=unit, path=path,
                            save_ancestors=True, save_weights=True, CLL=True)
        for f in range(6):
            Tf = T_u[unit[f]]
            assert np.array_equal(got["anc"][f, :Tf], want["anc"][f, :Tf]), (path, thresh, f)
            assert _bits_equal(got["logw"][f, :Tf], want["logw"][f, :Tf]), (path, thresh, f)
        np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12)


@pytest.mark.parametrize("path", PATHS)
def test_collapsed_and_nonfinite(path):
    F = _F()
    import pypomp_b200 as pp

    m = pp.Ricker(T=6, key=5)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names), 3, axis=0).astype(f32)
    th[1, 2] = 0.0          # phi = 0: every particle has zero likelihood for y > 0
    th[2, 0] = np.nan       # r = NaN: NaN weights
    seeds = np.array([1, 2, 3], np.uint64)
    want = cora.pfilter(3, 1, 1, th, st.ys, 700, seeds=seeds, ycon=m.spec.ycon(st.ys), anc=True, CLL=True)
    got = F.run_pfilter(st, th, seeds, 700, path=path, save_ancestors=True, CLL=True)
    assert np.array_equal(got["anc"], want["anc"])
    assert np.isneginf(want["loglik"][1]) and np.isnan(want["loglik"][2])
    assert np.isneginf(got["loglik"][1]) and np.isnan(got["loglik"][2])
    np.testing.assert_allclose(got["loglik"][0], want["loglik"][0], rtol=1e-12)


def test_lg_c1_against_kalman(lg2d):
    """Config 1 through the public Pomp API: logLik within MC error of FP64 Kalman."""
    th = lg2d.theta.to_array(lg2d.canonical_param_names)
    A, C, Q, R, X0 = kalman.lg_matrices(th[0], 2, 2)
    exact = kalman.kalman_loglik(lg2d.to_struct().ys, A, C, Q, R, X0)
    lg2d.pfilter(J=1000, key=2024, reps=32, CLL=True, ESS=True)
    df = lg2d.results()
    assert list(df.columns[:3]) == ["theta_idx", "logLik", "se"]
    lls = lg2d.results_history[-1].payload["logLiks"][0]
    assert abs(np.mean(lls) - exact) < 4 * np.std(lls) / np.sqrt(lls.size) + 0.05
    cll = lg2d.CLL()          # tidy frame: theta_idx, rep, time, CLL
    assert list(cll.columns) == ["theta_idx", "rep", "time", "CLL"] and len(cll) == 32 * 50
    sums = cll.groupby(["theta_idx", "rep"])["CLL"].sum().to_numpy()
    np.testing.assert_allclose(sums, lg2d.results_history[-1].payload["logLiks"][0], rtol=1e-10)
    avg = lg2d.CLL(average=True)
    assert list(avg.columns) == ["theta_idx", "time", "CLL"] and len(avg) == 50
    ess = lg2d.ESS()
    assert np.all(ess["ESS"] >= 1) and np.all(ess["ESS"] <= 1000)
    assert list(lg2d.time().columns) == ["method", "time"]
    # prune keeps the best parameter sets by log-likelihood
    th2 = lg2d.theta.params()[0]
    starts = [th2, {**th2, "A11": 0.2}, {**th2, "A11": 0.5}]
    lg2d.pfilter(J=300, key=1, theta=starts)
    lls = np.asarray(lg2d.theta.logLik)
    best = int(np.argmax(lls))
    lg2d.prune(n=1)
    assert lg2d.theta.num_replicates() == 3
    assert np.all(lg2d.theta.logLik == lls[best])
    assert all(p["A11"] == starts[best]["A11"] for p in lg2d.theta.params())


def test_lg_c2_full_width_properties(lg2d):
    """Config 2 width (J=262144) on a short horizon: bit-exact vs oracle, sorted ancestors."""
    F = _F()
    st = lg2d.to_struct()
    st.ys = st.ys[:6]
    th = np.repeat(lg2d.theta.to_array(lg2d.canonical_param_names), 2, axis=0).astype(f32)
    seeds = np.array([0, 1], np.uint64)
    J = 262144
    want = cora.pfilter(1, 2, 2, th, st.ys, J, seeds=seeds, anc=True, CLL=True, nthreads=2)
    got = F.run_pfilter(st, th, seeds, J, path="stream", save_ancestors=True, CLL=True)
    assert np.array_equal(got["anc"], want["anc"])
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12)
    assert np.all(np.diff(got["anc"], axis=-1) >= 0)
    np.testing.assert_allclose(got["cll"].sum(-1), got["loglik"], rtol=1e-12)


def test_j_validation():
    F = _F()
    import pypomp_b200 as pp

    m = pp.Ricker(T=3)
    th = m.theta.to_array(m.canonical_param_names)
    with pytest.raises(ValueError, match="J should be greater than 0"):
        F.run_pfilter(m.to_struct(), th, np.array([1], np.uint64), 0)
    with pytest.raises(ValueError):
        F.run_pfilter(m.to_struct(), th, np.array([1], np.uint64), (1 << 21) + 1)


def test_autotune_picks_a_tile_and_keeps_results():
    F = _F()
    m = _models()["SV"]
    st = m.to_struct()
    # 16 filters x 20 large tiles: enough CTAs that the automatic choice is the stream path
    th = np.repeat(_thetas(m, 2), 8, axis=0)
    seeds = np.arange(5, 21, dtype=np.uint64)
    J = 40000
    best = F.autotune(st, th, seeds, J)
    assert best in (2048, 512, 256)
    auto = F.run_pfilter(st, th, seeds, J, path="stream", save_ancestors=True)
    fixed = F.run_pfilter(st, th, seeds, J, path=f"stream@{best}", save_ancestors=True)
    assert np.array_equal(auto["anc"], fixed["anc"])
    assert np.array_equal(auto["loglik"], fixed["loglik"])
    # two filters of the same size run cluster-resident: nothing to tune
    assert F.autotune(st, th[:2], seeds[:2], J) == 0


@pytest.mark.parametrize("path", ["stream", "resident"])
def test_graph_replay_matches_direct_launches(path):
    """PPF_F_GRAPH: the first call captures, later calls with the same
    descriptor replay the graph; results equal direct launches bit for bit."""
    import torch

    from pypomp_b200 import _ffi

    m = _models()["SV"]
    st = m.to_struct()
    th = _thetas(m, 2)
    seeds = np.array([21, 22], np.uint64)
    J = 3000 if path == "stream" else 1500
    want = _F().run_pfilter(st, th, seeds, J, path=path, save_ancestors=True)
    dev = torch.device("cuda", 0)
    ys = torch.from_numpy(np.ascontiguousarray(st.ys[None], dtype=f32)).to(dev)
    thd = torch.from_numpy(th).to(dev)
    sd = torch.from_numpy(seeds.view(np.int64).copy()).to(dev)
    ll = torch.zeros(2, dtype=torch.float64, device=dev)
    anc = torch.zeros(2, st.ys.shape[0], J, dtype=torch.int32, device=dev)
    d = _ffi.PfilterDesc()
    d.model = m.spec.ffi_model()
    d.J, d.F, d.T, d.U = J, 2, st.ys.shape[0], 1
    d.path = _ffi.PATHS[path]
    d.flags = _ffi.F_GRAPH | _ffi.F_SAVE_ANC
    d.theta, d.ys, d.seeds, d.loglik, d.anc = _ffi.ptr(thd), _ffi.ptr(ys), _ffi.ptr(sd), _ffi.ptr(ll), _ffi.ptr(anc)
    ws = torch.empty(_ffi.LIB.ppf_pfilter_workspace_bytes(d), dtype=torch.uint8, device=dev)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(3):
        ll.zero_()
        anc.zero_()
        _ffi.check(_ffi.LIB.ppf_pfilter(d, stream), "ppf_pfilter")
        _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_pfilter")
        assert np.array_equal(anc.cpu().numpy(), want["anc"]), call
        assert np.array_equal(ll.cpu().numpy(), want["loglik"]), call


def test_largest_swarm_bit_exact():
    """J = 2^21 (PPF_MAX_J, the largest swarm the 128-bit offset arithmetic
    admits): stream path against the oracle, ancestors bit for bit."""
    from pypomp_b200 import _ffi

    F = _F()
    m = _models()["Ricker"]
    st = m.to_struct()
    st.ys = np.ascontiguousarray(st.ys[:3])
    th = _thetas(m, 1)
    seeds = np.array([99], np.uint64)
    J = _ffi.PPF_MAX_J
    want = cora.pfilter(m.spec.kind, 1, 1, th, st.ys, J, seeds=seeds, ycon=m.spec.ycon(st.ys), anc=True)
    got = F.run_pfilter(st, th, seeds, J, path="stream", save_ancestors=True)
    assert np.array_equal(got["anc"], want["anc"])
    np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12)


def test_fast_arithmetic_first_step_log_weights_close_to_exact(lg2d):
    """PPF_F_FAST (hardware special functions, contraction): the first step's
    log-weights of the same particles (same Philox words) agree with the exact
    arithmetic within 1e-5 relative (1e-5 absolute near zero), and the
    resampling ancestors stay sorted and in range."""
    F = _F()
    st = lg2d.to_struct()
    st.ys = st.ys[:5]
    th = np.repeat(lg2d.theta.to_array(lg2d.canonical_param_names), 3, axis=0).astype(f32)
    seeds = np.array([3, 4, 5], np.uint64)
    J = 65536
    ex = F.run_pfilter(st, th, seeds, J, path="stream", save_weights=True)
    fa = F.run_pfilter(st, th, seeds, J, path="stream", save_weights=True, save_ancestors=True, fast=True)
    w_ex, w_fa = ex["logw"][:, 0], fa["logw"][:, 0]
    assert np.all(np.isfinite(w_fa))
    assert np.all(np.abs(w_fa - w_ex) <= 1e-5 * np.maximum(np.abs(w_ex), 1.0))
    assert not np.array_equal(w_fa, w_ex)          # the fast kernels really ran
    anc = fa["anc"]
    assert np.all(np.diff(anc, axis=-1) >= 0) and anc.min() >= 0 and anc.max() < J


def test_fast_arithmetic_loglik_against_kalman():
    """LG 2-D, T = 300, J = 262144, 32 seeds with PPF_F_FAST: the log-mean-exp
    of the log-likelihoods is within Monte Carlo error of the exact Kalman
    value and within 1e-4 of it relative, as the exact arithmetic is."""
    import pypomp_b200 as pp
    from pypomp_b200.maths import logmeanexp, logmeanexp_se
    from tests.conftest import LG2_Q, LG2_R

    F = _F()
    m = pp.LG(T=300, Q=LG2_Q, R=LG2_R, key=7)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names), 32, axis=0).astype(f32)
    A, C, Q, R, X0 = kalman.lg_matrices(th[0].astype(np.float64), 2, 2)
    exact = kalman.kalman_loglik(st.ys, A, C, Q, R, X0)
    for fast in (False, True):
        ll = F.run_pfilter(st, th, np.arange(32, dtype=np.uint64) + 500, 262144, path="stream", fast=fast)["loglik"]
        lme, se = logmeanexp(ll), logmeanexp_se(ll)
        assert abs(lme - exact) <= 5 * se + 1e-3, (fast, lme, exact, se)
        assert abs(lme - exact) / abs(exact) <= 1e-4, (fast, lme, exact)
