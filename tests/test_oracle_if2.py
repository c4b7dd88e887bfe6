"""Pin the IF2 oracle (CPU only).

* oracle/refpath.py's ``mif`` (the float32 restatement of
  ``pypomp/core/algorithms/mif.py:16-258`` over the reference's own key tree)
  reproduces the reference's locked ``test_mif_regression.csv`` and
  ``test_mif_full_trace_regression.csv``;
* the C oracle's perturbed filter (the CUDA path's exact arithmetic), fed the
  same draws through injection, reproduces both fixtures when the mif loop is
  driven around it;
* with zero random-walk sds the perturbed filter is the bootstrap filter: the
  C oracle's ``perfilter`` and ``pfilter`` agree bit for bit.
"""

import numpy as np

from oracle import cora, jaxrng as jr, refpath as rp

f32 = np.float32
SIG = np.full(5, 0.02, f32)
SIG0 = np.zeros(5, f32)
NAMES = ["A11", "C11", "Q11", "R11", "X0_1"]


def _cool(nt, m, ntimes):
    frac = f32(f32(nt) / f32(ntimes) + f32(m))
    return f32(f32(0.5 ** (1.0 / 50.0)) ** frac)


def _close(got, want, tol):
    np.testing.assert_allclose(np.asarray(got, np.float64), np.asarray(want, np.float64), **tol)


def _trace_gold(gold, r, M):
    ll = [gold[f"loglik_rep{r}_m{m}"][0] for m in range(M)]
    tr = [[gold[f"{n}_rep{r}_m{m}"][0] for n in NAMES] for m in range(M + 1)]
    return np.array(ll), np.array(tr)


def test_refpath_mif_reproduces_reference_fixtures(ref_values, ref_lg1d):
    tol = ref_values["tolerance"]
    theta, ys = ref_lg1d["theta"], ref_lg1d["ys"]
    k = jr.split(jr.key(20260811), 1)[0]
    ll, tr, _, _ = rp.mif("LG", theta, ys, 12, 3, SIG, SIG0, _cool, k, 0)
    _close(ll[-1], ref_values["mif"]["final_loglik"][0], tol)
    _close(tr[-1], ref_values["mif"]["final_theta"], tol)
    ks = jr.split(jr.key(20260812), 2)
    thetas = [theta, (theta * f32(1.05)).astype(f32)]
    for r in range(2):
        ll, tr, _, _ = rp.mif("LG", thetas[r], ys, 12, 4, SIG, SIG0, _cool, ks[r], 1)
        want_ll, want_tr = _trace_gold(ref_values["mif_full_trace"], r, 4)
        _close(ll, want_ll, tol)
        _close(tr, want_tr, tol)


def _c_oracle_mif(theta, ys, M, draws, mon=None):
    """The mif loop (mif.py:16-85) around the C oracle's perturbed filter."""
    from oracle.models_np import MODELS

    m = MODELS["LG"]
    J = 12
    swarm = np.repeat(m.to_est(theta)[:, None], J, axis=1)[None].astype(f32)    # (1, P, J)
    means = [swarm[0].mean(axis=1, dtype=f32)]
    lls = []
    for it in range(M):
        cool = np.array([_cool(i, it, 4) for i in range(4)], f32)
        inj = {k: draws[k][it][None] for k in ("zp0", "zp", "z0", "z", "u")}
        res = cora.perfilter(1, 1, 1, swarm, ys, J, SIG, SIG0, cool, cool[0], inject=inj)
        if mon is not None:
            minj = {k: mon[k][it][None] for k in ("z0", "z", "u")}
            pf = cora.pfilter(1, 1, 1, means[-1][None], ys, J, est=True, inject=minj)
            lls.append(pf["loglik"][0])
        else:
            lls.append(res["loglik"][0])
        swarm = res["swarm"]
        means.append(swarm[0].mean(axis=1, dtype=f32))
    return np.array(lls), m.from_est(np.stack(means))


def test_c_oracle_perfilter_reproduces_reference_mif(ref_values, ref_lg1d):
    tol = ref_values["tolerance"]
    theta, ys = ref_lg1d["theta"], ref_lg1d["ys"]
    draws = {k: ref_lg1d[f"mif_{k}"] for k in ("zp0", "zp", "z0", "z", "u")}
    ll, tr = _c_oracle_mif(theta, ys, 3, draws)
    _close(ll[-1], ref_values["mif"]["final_loglik"][0], tol)
    _close(tr[-1], ref_values["mif"]["final_theta"], tol)
    thetas = [theta, (theta * f32(1.05)).astype(f32)]
    for r in range(2):
        draws = {k: ref_lg1d[f"mift_{k}"][r] for k in ("zp0", "zp", "z0", "z", "u")}
        mon = {k: ref_lg1d[f"mift_mon_{k}"][r] for k in ("z0", "z", "u")}
        ll, tr = _c_oracle_mif(thetas[r], ys, 4, draws, mon)
        want_ll, want_tr = _trace_gold(ref_values["mif_full_trace"], r, 4)
        _close(ll, want_ll, tol)
        _close(tr, want_tr, tol)


def test_c_oracle_perfilter_without_perturbation_is_pfilter(lg2d):
    st = lg2d.to_struct()
    spec = lg2d.spec
    th = spec.to_est(lg2d.theta.to_array(lg2d.canonical_param_names)).astype(f32)
    P, J, T = th.shape[1], 3000, st.ys.shape[0]
    seeds = np.array([7, 8], np.uint64)
    th2 = np.repeat(th, 2, axis=0)
    th2[1, 0] += f32(0.01)
    swarm = np.repeat(th2[:, :, None], J, axis=2)
    zero = np.zeros(P, f32)
    for thresh in (0.0, 20.0):
        got = cora.perfilter(spec.kind, spec.dx, spec.dy, swarm, st.ys, J, zero, zero, np.ones(T, f32), 1.0,
                             seeds=seeds, thresh=thresh, CLL=True, anc=True)
        want = cora.pfilter(spec.kind, spec.dx, spec.dy, th2, st.ys, J, seeds=seeds, est=True, thresh=thresh,
                            CLL=True, anc=True)
        assert np.array_equal(got["anc"], want["anc"])
        assert np.array_equal(got["cll"], want["cll"])
        assert np.array_equal(got["loglik"], want["loglik"])
        assert np.array_equal(got["swarm"], swarm)
