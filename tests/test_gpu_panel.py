"""Panels on the GPU.

* ``panel_pfilter``, ``panel_mif`` and ``panel_train`` fed the reference's
  own draws reproduce its locked panel fixtures (two LG units, J = 12,
  identity host transform as in the fixtures);
* a ragged panel (units of 20, 35 and 50 observations in one launch) gives
  each unit the log-likelihood its own single-unit filter gives, bit for bit,
  and the panel filter is bit-exact with the C oracle;
* ``PanelPomp.pfilter / mif / train`` run end to end on a ragged Ricker panel
  and fill the reference's panel result tables;
* the natural-scale option of the IF2 kernels (``PPF_F_NATURAL``) is
  bit-exact with the C oracle.
"""

import dataclasses

import numpy as np
import pandas as pd
import pytest

from oracle import cora

pytestmark = pytest.mark.gpu
f32 = np.float32


def _lg_panel_struct(ref_lg1d):
    from pypomp_b200.functional import PanelPompStruct
    from pypomp_b200.models import lg_spec

    spec = dataclasses.replace(lg_spec(1, 1), natural=True)
    ys = np.stack([ref_lg1d["ys"], ref_lg1d["panel_ys2"]]).astype(f32)
    return PanelPompStruct(spec=spec, ys=ys, T_u=np.array([4, 4], np.int32), times=[np.arange(1, 5.0)] * 2,
                           t0=0.0, unit_names=["unit1", "unit2"], shared_param_names=["A11", "C11"],
                           unit_param_names=["Q11", "R11", "X0_1"],
                           permutations=np.array([[0, 1, 2, 3, 4]] * 2))


def test_panel_pfilter_fixture_through_injection(ref_values, ref_lg1d):
    from pypomp_b200 import functional as F

    st = _lg_panel_struct(ref_lg1d)
    th = ref_lg1d["theta"]
    inj = {k: ref_lg1d[f"ppf_{k}"] for k in ("z0", "z", "u")}
    res = F.panel_pfilter(st, np.stack([th, th])[None], 12, np.zeros((1, 2), np.uint64), inject=inj)
    np.testing.assert_allclose(res["logLik"][0], ref_values["panel_pfilter"]["logLik"], **ref_values["tolerance"])


def test_panel_mif_fixture_through_injection(ref_values, ref_lg1d):
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import RWSigma

    st = _lg_panel_struct(ref_lg1d)
    th = ref_lg1d["theta"].astype(np.float64)
    rw = RWSigma({n: 0.02 for n in st.param_names}).geometric_cooling(0.5)
    inj = [[{"perfilter": {k: ref_lg1d[f"pmif_{k}"][m, u][None] for k in ("zp0", "zp", "z0", "z", "u")},
             "monitors": []} for u in range(2)] for m in range(3)]
    sh = np.repeat(th[None, None, :2], 12, axis=1)
    un = np.repeat(np.stack([th[2:]] * 2)[None, None], 12, axis=1)
    s_tr, u_tr, fs, fu = F.panel_mif(st, sh, un, rw, 3, 12, np.zeros(1, np.uint64), 0.0, 0, True, inject=inj)
    g = ref_values["panel_mif"]
    tol = ref_values["tolerance"]
    np.testing.assert_allclose(s_tr[0, -1], g["final_shared"], **tol)
    np.testing.assert_allclose(u_tr[0, -1].ravel(), g["final_unit"], **tol)
    assert fs.shape == (1, 12, 2) and fu.shape == (1, 12, 2, 3)


def test_panel_train_fixture_through_injection(ref_values, ref_lg1d):
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import Adam, LearningRate

    st = _lg_panel_struct(ref_lg1d)
    th = ref_lg1d["theta"].astype(np.float64)
    eta = LearningRate({n: 0.01 for n in st.param_names})
    inj = [[{k: ref_lg1d[f"ptrain_{k}"][m, c][None] for k in ("z0", "z", "u")} for c in range(2)]
           for m in range(3)]
    nll, hs, hu = F.panel_train(st, th[None, :2], np.stack([th[2:]] * 2)[None], 12, Adam(), 3, eta, 0.97,
                                np.zeros((1, 3, 2), np.uint64), 1.0, 1, inject=inj)
    g = ref_values["panel_train"]
    tol = ref_values["tolerance"]
    np.testing.assert_allclose(nll[0, -1], g["final_neg_loglik"][0], **tol)
    np.testing.assert_allclose(hs[0, -1], g["final_shared"], **tol)
    np.testing.assert_allclose(hu[0, -1].ravel(), g["final_unit"], **tol)


def _ricker_panel(lengths=(20, 35, 50)):
    import pypomp_b200 as pp

    units = {f"u{i}": pp.Ricker(T=T, key=i) for i, T in enumerate(lengths)}
    shared = pd.DataFrame({"shared": [0.3, 10.0]}, index=["sigma", "phi"])
    spec = pd.DataFrame([[44.7, 40.0, 50.0], [7.0, 6.0, 8.0]], index=["r", "N_0"], columns=list(units))
    return pp.PanelPomp(units, pp.PanelParameters({"shared": shared, "unit_specific": spec}))


def test_ragged_panel_pfilter_matches_single_units_and_oracle():
    from pypomp_b200 import functional as F
    from pypomp_b200.functional import _panel_thetas

    pan = _ricker_panel()
    st = pan.to_struct()
    th = _panel_thetas(pan.theta.shared_array(), pan.theta.unit_array(st.unit_names), st.permutations)
    th = np.repeat(th, 2, axis=0).astype(f32)                   # (2 reps, U, P)
    th[1, :, 0] *= f32(0.9)
    keys = np.arange(6, dtype=np.uint64).reshape(2, 3) + np.uint64(40)
    J = 3000
    res = F.panel_pfilter(st, th, J, keys, CLL=True)
    for r in range(2):
        for u in range(3):
            one = F.run_pfilter(st.unit(u), th[r, u][None], keys[r, u:u + 1], J, CLL=True)
            assert res["logLik"][r, u] == one["loglik"][0]
            T = int(st.T_u[u])
            np.testing.assert_array_equal(res["CLL"][r, u, :T], one["cll"][0])
            assert np.all(np.isnan(res["CLL"][r, u, T:]))
    want = cora.pfilter(st.spec.kind, 1, 1, th.reshape(6, 4), st.ys, J, seeds=keys.reshape(-1),
                        unit=np.tile(np.arange(3), 2), T_u=st.T_u, ycon=st.spec.ycon(st.ys))
    np.testing.assert_allclose(res["logLik"].reshape(-1), want["loglik"], rtol=1e-12)


def test_panelpomp_methods_end_to_end():
    from pypomp_b200.optim import LearningRate, RWSigma

    pan = _ricker_panel()
    pan.pfilter(J=2000, key=1, reps=2, CLL=True)
    r = pan.results()
    assert list(r.columns[:6]) == ["theta_idx", "shared logLik", "shared logLik se", "unit", "unit logLik",
                                   "unit logLik se"]
    assert len(r) == 3 and np.all(np.isfinite(r["unit logLik"]))
    names = pan.canonical_param_names
    rw = RWSigma({n: 0.02 for n in names}).geometric_cooling(0.5)
    for block in (True, False):
        pan.mif(J=1000, M=2, rw_sd=rw, key=2, block=block, n_monitors=1)
        tr = pan.traces()
        assert set(tr["unit"]) == {"shared", "u0", "u1", "u2"}
        assert np.all(np.isfinite(pan.results()["unit logLik"]))
    pan.train(J=1000, M=2, eta=LearningRate({n: 0.01 for n in names}), key=3)
    res = pan.results()
    assert np.all(np.isfinite(res["shared logLik"]))
    assert pan.theta.num_replicates() == 1


def test_perfilter_natural_scale_bit_exact():
    from pypomp_b200 import functional as F
    import pypomp_b200 as pp

    m = pp.Ricker(T=15, key=2)
    st = m.to_struct()
    th = m.theta.to_array(m.canonical_param_names).astype(f32)
    J = 2000
    swarm = np.repeat(th[:, :, None], J, axis=2)
    sig = np.array([0.5, 0.01, 0.1, 0.1], f32)
    cool = np.ones(15, f32)
    seeds = np.array([3], np.uint64)
    want = cora.perfilter(st.spec.kind, 1, 1, swarm, st.ys, J, sig, sig, cool, 1.0, seeds=seeds,
                          ycon=st.spec.ycon(st.ys), anc=True, natural=True)
    got = F.run_perfilter(st, swarm.transpose(0, 2, 1), seeds, J, sig, sig, cool, 1.0, save_ancestors=True,
                          natural=True)
    assert np.array_equal(got["anc"], want["anc"])
    assert np.array_equal(got["swarm"], want["swarm"].transpose(0, 2, 1))


@pytest.mark.parametrize("block", [True, False])
def test_panel_mif_queued_units_equal_separate_calls(block):
    """panel_mif queues its unit filters on device-resident inputs without
    waiting between them; its swarms and unit log-likelihoods equal the
    unit-by-unit run_perfilter calls they replace, bit for bit (ragged units)."""
    import torch

    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom
    from pypomp_b200.optim import RWSigma

    pan = _ricker_panel()
    st = pan.to_struct()
    names = pan.get_unit_names()
    J, M = 1500, 2
    rw = RWSigma({n: 0.03 for n in pan.canonical_param_names}).geometric_cooling(0.5)
    sh = np.repeat(pan.theta.shared_array()[:, None, :], J, axis=1)
    un = np.repeat(pan.theta.unit_array(names)[:, None], J, axis=1)
    keys = np.array([17], np.uint64)
    s_tr, u_tr, s_fin, u_fin = F.panel_mif(st, sh, un, rw, M, J, keys, block=block)
    # the same iterations unit by unit (the loop panel_mif runs with injected draws)
    spec, U = st.spec, st.U
    perms = np.asarray(st.permutations)
    inv = np.argsort(perms, axis=1)
    ns, nu = sh.shape[2], un.shape[3]
    sig_p, sig0_p = rw.arrays(st.param_names)
    panel0 = np.concatenate([sh[:, :, None, :].repeat(U, axis=2), un], axis=3)
    est = np.empty_like(panel0)
    for u in range(U):
        est[:, :, u, :] = spec.to_est(panel0[:, :, u, perms[u]])[:, :, inv[u]]
    S = torch.tensor(est[:, :, 0, :ns].transpose(0, 2, 1).copy(), dtype=torch.float32).cuda()
    Us = torch.tensor(est[:, :, :, ns:].transpose(0, 2, 3, 1).copy(), dtype=torch.float32).cuda()
    m_keys = np.stack([pprandom.split(k, M + 1)[1:] for k in keys])
    for it in range(M):
        unit_keys = np.stack([pprandom.split(k, U) for k in m_keys[:, it]])
        for u in range(U):
            st_u = st.unit(u)
            T = st_u.ys.shape[0]
            swarm = torch.cat([S, Us[:, u]], dim=1)[:, torch.tensor(perms[u]).cuda()].contiguous()
            cool = np.array([rw.cooling_factor(i, it, T) for i in range(T)], dtype=np.float32)
            res = F.run_perfilter(st_u, swarm, unit_keys[:, u], J, sig_p[perms[u]], sig0_p[perms[u]], cool,
                                  cool[0], save_ancestors=not block)
            assert res["loglik"].cpu().numpy()[0] == u_tr[0, it + 1, u, 0]
            new = res["swarm"][:, torch.tensor(inv[u]).cuda()]
            S = new[:, :ns].contiguous()
            if not block:
                origin = torch.arange(J).cuda().expand(1, J).contiguous()
                for t in range(T):
                    origin = torch.gather(origin, 1, res["anc"][:, t].long())
                Us = torch.gather(Us, 3, origin[:, None, None, :].expand(1, U, nu, J))
            Us = Us.clone()
            Us[:, u] = new[:, ns:]
    # final swarms on the natural scale, converted as panel_mif converts them
    s_e = S.cpu().numpy().transpose(0, 2, 1)
    u_e = Us.cpu().numpy().transpose(0, 3, 1, 2)
    for u in range(U):
        nat = spec.from_est(np.concatenate([s_e, u_e[:, :, u]], axis=2)[:, :, perms[u]])[:, :, inv[u]]
        assert np.array_equal(nat[:, :, ns:], u_fin[:, :, u])
        if u == 0:
            assert np.array_equal(nat[:, :, :ns], s_fin)


def test_panel_mif_parallel_units_equal_single_unit_filters():
    """mode='parallel' (not in the reference): all units of all replicates in
    one batched perturbed-filter call per iteration.  Each unit's filter is
    the single-unit filter from the iteration's swarms, bit for bit (the first
    unit's also against the C oracle); the unit-specific swarms are those
    filters' outputs, and the shared swarm follows the documented
    recombination (inverse-variance weighted centre, deviations of unit
    j mod U)."""
    import torch

    from pypomp_b200 import functional as F
    from pypomp_b200 import random as pprandom
    from pypomp_b200.optim import RWSigma

    pan = _ricker_panel()
    st = pan.to_struct()
    names = pan.get_unit_names()
    J, M = 1500, 2
    rw = RWSigma({n: 0.03 for n in pan.canonical_param_names}).geometric_cooling(0.5)
    sh = np.repeat(pan.theta.shared_array()[:, None, :], J, axis=1)
    un = np.repeat(pan.theta.unit_array(names)[:, None], J, axis=1)
    keys = np.array([23], np.uint64)
    s_tr, u_tr, s_fin, u_fin = F.panel_mif(st, sh, un, rw, M, J, keys, mode="parallel")
    spec, U = st.spec, st.U
    perm = np.asarray(st.permutations)[0]
    inv = np.argsort(perm)
    ns, nu = sh.shape[2], un.shape[3]
    sig_p, sig0_p = rw.arrays(st.param_names)
    panel0 = np.concatenate([sh[:, :, None, :].repeat(U, axis=2), un], axis=3)
    est = spec.to_est(panel0[..., perm])[..., inv]
    S = est[0, :, 0, :ns].T.astype(f32)                       # (ns, J)
    Us = est[0, :, :, ns:].transpose(1, 2, 0).astype(f32)     # (U, nu, J)
    m_keys = pprandom.split(int(keys[0]), M + 1)[1:]
    for it in range(M):
        unit_keys = pprandom.split(int(m_keys[it]), U)
        outs = []
        for u in range(U):
            st_u = st.unit(u)
            T = st_u.ys.shape[0]
            swarm = np.concatenate([S, Us[u]], axis=0)[perm]  # (P, J) unit order
            cool = np.array([rw.cooling_factor(i, it, T) for i in range(T)], dtype=np.float32)
            one = F.run_perfilter(st_u, torch.from_numpy(swarm[None].copy()).cuda(), unit_keys[u:u + 1], J,
                                  sig_p[perm], sig0_p[perm], cool, cool[0])
            assert one["loglik"].cpu().numpy()[0] == u_tr[0, it + 1, u, 0]
            if it == 0 and u == 0:
                want = cora.perfilter(spec.kind, 1, 1, swarm[None], st_u.ys, J, sig_p[perm].astype(f32),
                                      sig0_p[perm].astype(f32), cool, cool[0], seeds=unit_keys[u:u + 1],
                                      ycon=spec.ycon(st_u.ys))
                assert np.array_equal(one["swarm"].cpu().numpy()[0], want["swarm"][0])
            outs.append(one["swarm"].cpu().numpy()[0][inv])       # panel order (P, J)
        outs = np.stack(outs)                                     # (U, P, J)
        Us = outs[:, ns:].copy()
        su = outs[:, :ns].astype(np.float64)
        mu = su.mean(axis=2)
        var = su.var(axis=2)
        w = np.where(var > 0, 1.0 / np.where(var > 0, var, 1.0), 0.0)
        centre = (w * mu).sum(axis=0) / w.sum(axis=0)
        S = (centre[:, None] + (su - mu[..., None])[np.arange(J) % U, :, np.arange(J)].T).astype(f32)
    s_e = S.T.astype(np.float64)                                  # (J, ns)
    for u in range(U):
        nat = spec.from_est(np.concatenate([s_e, Us[u].T.astype(np.float64)], axis=1)[:, perm])[:, inv]
        assert np.array_equal(nat[:, ns:], u_fin[0, :, u])
        if u == 0:
            np.testing.assert_allclose(nat[:, :ns], s_fin[0], rtol=1e-6)


def test_panel_mif_parallel_raises_the_panel_loglik():
    """From a perturbed start, parallel-mode panel IF2 raises the summed unit
    log-likelihood of the panel (PanelPomp.mif end to end, mode='parallel')."""
    import pypomp_b200 as pp
    from pypomp_b200.optim import RWSigma

    units = {f"u{i}": pp.Ricker(T=60 + 10 * i, r=np.exp(3.0), sigma=0.3, phi=10.0, key=100 + i) for i in range(6)}
    shared = pd.DataFrame({"shared": [0.6, 6.0]}, index=["sigma", "phi"])
    spec = pd.DataFrame([[np.exp(2.6)] * 6, [7.0] * 6], index=["r", "N_0"], columns=list(units))
    pan = pp.PanelPomp(units, pp.PanelParameters({"shared": shared, "unit_specific": spec}))
    rw = RWSigma({"r": 0.05, "sigma": 0.05, "phi": 0.05, "N_0": 0.0}).geometric_cooling(0.5)
    pan.pfilter(J=2000, key=1, reps=4)
    before = pan.results()["shared logLik"].iloc[0]
    pan.mif(J=2000, M=15, rw_sd=rw, key=2, mode="parallel")
    tr = pan.traces()
    ll = tr.loc[(tr["unit"] == "shared") & (tr["method"] == "mif"), "logLik"].to_numpy()
    assert ll.shape == (16,) and np.all(np.isfinite(ll[1:]))        # iteration 0 has no log-likelihood
    assert ll[-1] > ll[1]
    pan.pfilter(J=2000, key=3, reps=4)
    after = pan.results()["shared logLik"].iloc[0]
    assert after > before + 5.0, (before, after)
