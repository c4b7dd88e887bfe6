"""Pin the oracle before trusting it (CPU only).

* oracle/jaxrng.py reproduces the reference's simulate fixture, so the
  restated Threefry key trees are the reference's own random streams;
* oracle/refpath.py (the float32 restatement of pfilter / mop) reproduces the
  reference's locked pfilter, per-step diagnostics and MOP values;
* the C oracle (the CUDA path's exact arithmetic), fed the reference's own
  normals and uniforms, reproduces the same fixtures;
* Philox4x32-10 matches the published known-answer vectors, and the
  deterministic elementary functions are within 2 ulp of float64 libm;
* the C oracle agrees with the FP64 Kalman log-likelihood within Monte Carlo
  error, and keeps the reference's invariants (sum CLL = logLik, ESS in [1,J]).
"""

import numpy as np
import pytest

from oracle import cora, jaxrng as jr, kalman, refpath as rp

f32 = np.float32


def _close(a, b, tol):
    return abs(a - b) <= tol["atol"] + tol["rtol"] * abs(b)


def test_jax_streams_reproduce_simulate_fixture(ref_values):
    # tests/test_regression/test_simulate_regression.py:7-21
    theta = np.array([0.9, 1.0, 0.1, np.sqrt(0.1), 0.0], f32)
    k = jr.split(jr.key(20260811), 1)[0]
    X, Y = rp.simulate("LG", theta, 4, k, nsim=1)
    tol = ref_values["tolerance"]
    assert _close(float(X[-1, 0, 0]), ref_values["simulate"]["X_final"][0], tol)
    for got, want in zip(Y[:, 0, 0], ref_values["simulate"]["Y"]):
        assert _close(float(got), want, tol)


def test_refpath_reproduces_pfilter_fixture(ref_values, ref_lg1d):
    k = jr.split(jr.key(20260811), 1)[0]
    res = rp.pfilter("LG", ref_lg1d["theta"], ref_lg1d["ys"], 12, rp.JaxKeyNoise(k, 12, 1, 1))
    assert _close(float(res["logLik"]), ref_values["pfilter"]["logLik"][0], ref_values["tolerance"])


def test_refpath_reproduces_diagnostics_fixture(ref_values, ref_lg1d):
    tol = ref_values["tolerance"]
    gold = ref_values["pfilter_diagnostics"]
    ks = jr.split(jr.key(20260812), 2)
    for r in range(2):
        res = rp.pfilter("LG", ref_lg1d["diag_theta"][r], ref_lg1d["ys"], 12,
                         rp.JaxKeyNoise(ks[r], 12, 1, 1), diagnostics=True)
        assert _close(float(res["logLik"]), gold["logLik"][r], tol)
        for t in range(4):
            for name, key in (("CLL", "CLL"), ("ESS", "ESS")):
                assert _close(float(res[key][t]), gold[f"{name}_rep{r}_t{t}"][0], tol)
            assert _close(float(res["filter_mean"][t, 0]), gold[f"filter_mean_rep{r}_t{t}"][0], tol)
            assert _close(float(res["prediction_mean"][t, 0]), gold[f"prediction_mean_rep{r}_t{t}"][0], tol)


def test_refpath_reproduces_mop_fixture(ref_values, ref_lg1d):
    k = jr.split(jr.key(20260811), 1)[0]
    v = rp.mop("LG", ref_lg1d["theta"], ref_lg1d["ys"], 12, 0.5, rp.JaxKeyNoise(k, 12, 1, 1))
    assert _close(float(v), ref_values["mop"]["mop"][0], ref_values["tolerance"])



def test_refpath_reproduces_dpop_fixture(ref_values, ref_lg1d):
    """DPOP's forward is MOP's (the transition log-weight enters the carried
    weights as pw - stop_gradient(pw), value 0; same key tree,
    ``pypomp/core/algorithms/dpop.py:85-134``), so the MOP restatement
    reproduces the locked DPOP value (alpha = 0.5, process_weight_index = 0)."""
    k = jr.split(jr.key(20260811), 1)[0]
    v = rp.mop("LG", ref_lg1d["theta"], ref_lg1d["ys"], 12, 0.5, rp.JaxKeyNoise(k, 12, 1, 1))
    assert _close(float(v), ref_values["dpop"]["dpop"][0], ref_values["tolerance"])


def test_dpop_surrogate_value_equals_mop_surrogate():
    """At the base parameters the frozen DPOP surrogate of the C oracle has the
    MOP surrogate's value, and its recorded pw are the predicted states'
    component pwi."""
    import pypomp_b200 as pp

    m = pp.LG(T=8, key=5)
    st, spec = m.to_struct(), m.spec
    th = spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(np.float32)
    seeds = np.array([2], np.uint64)
    J = 300
    w = cora.pfilter(spec.kind, spec.dx, spec.dy, th, st.ys, J, seeds=seeds, est=True, mop=True, anc=True)
    v_mop, m0 = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, th, st.ys, J, 0.5, w["anc"], seeds=seeds)
    for pwi in range(spec.dx):
        v_dp, m0_dp, p0 = cora.mop_surrogate(spec.kind, spec.dx, spec.dy, th, st.ys, J, 0.5, w["anc"],
                                             seeds=seeds, pwi=pwi)
        assert v_dp[0] == v_mop[0]
        assert np.array_equal(m0_dp, m0) and p0.shape == m0.shape and np.all(np.isfinite(p0))

def test_recorded_streams_replay_identically(ref_lg1d):
    # the committed injection arrays are the draws of the key tree above
    res = rp.pfilter("LG", ref_lg1d["theta"], ref_lg1d["ys"], 12,
                     rp.ArrayNoise(ref_lg1d["pf_z0"], ref_lg1d["pf_z"], ref_lg1d["pf_u"]))
    k = jr.split(jr.key(20260811), 1)[0]
    res2 = rp.pfilter("LG", ref_lg1d["theta"], ref_lg1d["ys"], 12, rp.JaxKeyNoise(k, 12, 1, 1))
    assert res["logLik"] == res2["logLik"]


def test_c_oracle_reproduces_reference_fixtures(ref_values, ref_lg1d):
    """The exact-arithmetic C oracle, fed the reference's own draws."""
    tol = ref_values["tolerance"]
    inj = dict(z0=ref_lg1d["pf_z0"][None], z=ref_lg1d["pf_z"][None], u=ref_lg1d["pf_u"][None])
    r = cora.pfilter(1, 1, 1, ref_lg1d["theta"], ref_lg1d["ys"], 12, inject=inj)
    assert _close(float(r["loglik"][0]), ref_values["pfilter"]["logLik"][0], tol)
    gold = ref_values["pfilter_diagnostics"]
    inj = dict(z0=ref_lg1d["diag_z0"], z=ref_lg1d["diag_z"], u=ref_lg1d["diag_u"])
    r = cora.pfilter(1, 1, 1, ref_lg1d["diag_theta"], ref_lg1d["ys"], 12, inject=inj,
                     CLL=True, ESS=True, fmean=True, pmean=True)
    for rep in range(2):
        assert _close(float(r["loglik"][rep]), gold["logLik"][rep], tol)
        for t in range(4):
            assert _close(r["cll"][rep, t], gold[f"CLL_rep{rep}_t{t}"][0], tol)
            assert _close(float(r["ess"][rep, t]), gold[f"ESS_rep{rep}_t{t}"][0], tol)
            assert _close(float(r["fmean"][rep, t, 0]), gold[f"filter_mean_rep{rep}_t{t}"][0], tol)
            assert _close(float(r["pmean"][rep, t, 0]), gold[f"prediction_mean_rep{rep}_t{t}"][0], tol)
    inj = dict(z0=ref_lg1d["mop_z0"][None], z=ref_lg1d["mop_z"][None], u=ref_lg1d["mop_u"][None])
    r = cora.pfilter(1, 1, 1, ref_lg1d["theta"], ref_lg1d["ys"], 12, inject=inj, est=True, mop=True)
    assert _close(-float(r["loglik"][0]), ref_values["mop"]["mop"][0], tol)


def test_c_oracle_ancestors_match_reference_restatement(ref_lg1d):
    inj = dict(z0=ref_lg1d["diag_z0"], z=ref_lg1d["diag_z"], u=ref_lg1d["diag_u"])
    r = cora.pfilter(1, 1, 1, ref_lg1d["diag_theta"], ref_lg1d["ys"], 12, inject=inj, anc=True)
    for rep in range(2):
        ref = rp.pfilter("LG", ref_lg1d["diag_theta"][rep], ref_lg1d["ys"], 12,
                         rp.ArrayNoise(ref_lg1d["diag_z0"][rep], ref_lg1d["diag_z"][rep],
                                       ref_lg1d["diag_u"][rep]), diagnostics=True)
        np.testing.assert_array_equal(r["anc"][rep][:3], ref["ancestors"][:3])


# Random123 known-answer vectors for Philox4x32-10 (counter, key -> output).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    np.testing.assert_array_equal(cora.philox(ctr, key), np.array(want, np.uint32))


def _ulp_err(got, want):
    got = np.float32(got)
    want64 = float(want)
    if not np.isfinite(want64):
        return 0.0 if got == np.float32(want64) else np.inf
    spacing = np.spacing(np.float32(want64))
    return abs(float(got) - want64) / float(abs(spacing))


def test_detmath_exp_log_accuracy():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-100, 88, 4000), rng.uniform(-1, 1, 2000),
                         [0.0, -0.0, 1e-30, -87.5, 88.7, -103.0]]).astype(f32)
    worst = max(_ulp_err(cora.expf(x), np.exp(np.float64(x))) for x in xs
                if np.exp(np.float64(x)) > 1.2e-38)
    assert worst <= 2.0, worst
    ys = np.concatenate([np.exp(rng.uniform(-80, 80, 4000)), rng.uniform(0.5, 2.0, 2000),
                         [1.0, 2.0, 0.70710677, 1e-40]]).astype(f32)
    worst = max(_ulp_err(cora.logf(y), np.log(np.float64(y))) for y in ys if y != 1.0)
    assert worst <= 2.0, worst
    assert cora.logf(1.0) == 0.0 and np.isneginf(cora.logf(0.0)) and np.isnan(cora.logf(-1.0))
    assert cora.expf(-200.0) == 0.0 and np.isinf(cora.expf(100.0))


def test_detmath_sincos_accuracy():
    us = np.linspace(0, 1, 5001, endpoint=False).astype(f32)
    for u in us:
        s, c = cora.sincos2pi(u)
        a = 2 * np.pi * np.float64(u)
        assert abs(float(s) - np.sin(a)) < 4e-7 and abs(float(c) - np.cos(a)) < 4e-7


def test_philox_normals_are_standard_normal():
    z = np.concatenate([cora.normals(42, j, 1, 0, 4) for j in range(20000)])
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1.0) < 0.02
    assert abs(np.mean(z ** 4) - 3.0) < 0.15


def test_c_oracle_matches_kalman_lg2d(lg2d):
    st = lg2d.to_struct()
    th = lg2d.theta.to_array(lg2d.canonical_param_names)
    A, C, Q, R, X0 = kalman.lg_matrices(th[0], 2, 2)
    exact = kalman.kalman_loglik(st.ys, A, C, Q, R, X0)
    F = 16
    r = cora.pfilter(1, 2, 2, np.repeat(th, F, 0), st.ys, 2000,
                     seeds=np.arange(F, dtype=np.uint64) + 99, CLL=True, ESS=True, nthreads=4)
    ll = r["loglik"]
    # MC error of one filter at J=2000, T=50 is ~0.1; the replicate mean is closer
    assert abs(np.mean(ll) - exact) < 4 * np.std(ll) / np.sqrt(F) + 0.05
    np.testing.assert_allclose(r["cll"].sum(axis=1), ll, rtol=1e-12)
    assert np.all(r["ess"] >= 1.0) and np.all(r["ess"] <= 2000.0)


def test_c_oracle_thresh_and_identity_ancestors(lg2d):
    st = lg2d.to_struct()
    th = lg2d.theta.to_array(lg2d.canonical_param_names)
    r = cora.pfilter(1, 2, 2, th, st.ys, 256, seeds=np.array([5], np.uint64), thresh=20.0,
                     anc=True, ESS=True)
    anc = r["anc"][0]
    ident = np.all(anc == np.arange(256)[None, :], axis=1)
    assert ident.any() and (~ident).any()   # some steps resample, some do not
    for t in range(anc.shape[0]):
        assert np.all(np.diff(anc[t]) >= 0)  # systematic ancestors are sorted


def test_weight_quantiser_exp_equals_expf():
    """pp_expq (the fixed-point weights' exp) gives the same quantised weight
    rint(e 2^40) as pp_expf for every argument at or below 0: exhaustive over
    the float32 values in [-40, 0] at a 1/4096 stride plus edge cases."""
    import ctypes

    lib = cora._L()
    lib.ppfo_expq.argtypes = [ctypes.c_float]
    lib.ppfo_expq.restype = ctypes.c_float
    xs = np.concatenate([-np.arange(0, 40 * 4096, dtype=np.float64) / 4096.0,
                         [-32.0, -31.999998, -32.000004, -0.0, -1e-30, -np.inf]]).astype(f32)
    for x in xs:
        e1 = np.float32(lib.ppfo_expf(float(x)))
        e2 = np.float32(lib.ppfo_expq(float(x)))
        q1 = np.rint(np.float32(e1 * np.float32(2.0 ** 40)))
        q2 = np.rint(np.float32(e2 * np.float32(2.0 ** 40)))
        assert q1 == q2, (x, e1, e2)
        if x >= -32.0:
            assert e1 == e2, (x, e1, e2)


@pytest.mark.parametrize("dx,dy", [(6, 7), (9, 9), (2, 5)])
def test_c_oracle_wide_lg_against_kalman(dx, dy):
    """The C oracle's LG above 4 x 4 (up to the reference's MAX_DIM = 9,
    ``pypomp/models/linear_gaussian.py:48``): log-mean-exp of 8 filters within
    5 standard errors of the exact FP64 Kalman log-likelihood."""
    import pypomp_b200 as pp
    from pypomp_b200.maths import logmeanexp, logmeanexp_se

    m = pp.LG(T=15, A=0.9 * np.eye(dx), C=np.eye(dy, dx) + 0.1, Q=np.eye(dx) * 0.05,
              R=np.eye(dy) * 0.2 + 0.02, key=5)
    st = m.to_struct()
    th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    r = cora.pfilter(m.spec.kind, dx, dy, np.repeat(th, 8, 0), st.ys, 20000, seeds=np.arange(8, dtype=np.uint64),
                     nthreads=8)
    A, C, Q, R, X0 = kalman.lg_matrices(th[0].astype(np.float64), dx, dy)
    exact = kalman.kalman_loglik(st.ys, A, C, Q, R, X0)
    lme, se = logmeanexp(r["loglik"]), logmeanexp_se(r["loglik"])
    assert abs(lme - exact) <= 5 * se, (lme, exact, se)
