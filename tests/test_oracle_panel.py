"""Panels on the CPU: oracle pins and host logic.

* oracle/refpath.py's panel filter and panel IF2 (``pfilter.py:248-304``,
  ``panel_mif.py:17-247``) reproduce the reference's locked
  ``test_panel_pfilter_regression.csv`` and ``test_panel_mif_regression.csv``
  (two LG units, J = 12).  Those fixtures replace ``par_trans`` by
  ``ParTrans()`` after building the units, which changes the host-side
  transforms only: the model mechanics keep LG's log transform of the
  covariance-factor diagonals;
* the C oracle fed the same draws reproduces both;
* ``PanelPomp.to_struct`` pads ragged units and builds the parameter
  permutations; ``_panel_thetas`` maps [shared | unit] blocks to unit order.
"""

import numpy as np
import pandas as pd

from oracle import cora, jaxrng as jr, refpath as rp

f32 = np.float32
SIG = np.full(5, 0.02, f32)
SIG0 = np.zeros(5, f32)


def _cool(nt, m, ntimes):
    return f32(f32(0.5 ** (1.0 / 50.0)) ** f32(f32(nt) / f32(ntimes) + f32(m)))


def _close(got, want, tol):
    np.testing.assert_allclose(np.asarray(got, np.float64), np.asarray(want, np.float64), **tol)


def _gold_mif(ref_values):
    g = ref_values["panel_mif"]
    return np.array(g["final_shared"]), np.array(g["final_unit"])


def test_refpath_panel_fixtures(ref_values, ref_lg1d):
    tol = ref_values["tolerance"]
    th, ys1, ys2 = ref_lg1d["theta"], ref_lg1d["ys"], ref_lg1d["panel_ys2"]
    key = jr.key(20260811)
    ll, _ = rp.panel_pfilter("LG", np.stack([th, th]), [ys1, ys2], 12, jr.split(key, 2))
    _close(ll, ref_values["panel_pfilter"]["logLik"], tol)
    s_tr, u_tr, _ = rp.panel_mif("LG", th[:2], np.stack([th[2:]] * 2), [ys1, ys2], 12, 3, SIG, SIG0, _cool,
                                 jr.split(key, 1)[0], host_identity=True)
    want_s, want_u = _gold_mif(ref_values)
    _close(s_tr[-1], want_s, tol)
    _close(u_tr[-1].ravel(), want_u, tol)


def test_c_oracle_panel_fixtures(ref_values, ref_lg1d):
    tol = ref_values["tolerance"]
    th, ys1, ys2 = ref_lg1d["theta"], ref_lg1d["ys"], ref_lg1d["panel_ys2"]
    ys = np.stack([ys1, ys2])
    inj = {k: ref_lg1d[f"ppf_{k}"] for k in ("z0", "z", "u")}
    res = cora.pfilter(1, 1, 1, np.stack([th, th]), ys, 12, unit=np.array([0, 1]), inject=inj)
    _close(res["loglik"], ref_values["panel_pfilter"]["logLik"], tol)
    # panel IF2 loop around the C oracle's perturbed filter (block, no monitors)
    S = np.repeat(th[:2, None], 12, axis=1)[None].astype(f32)              # (1, ns, J)
    Us = np.repeat(th[2:, None], 12, axis=1)[None, None].repeat(2, axis=1).astype(f32)   # (1, U, nu, J)
    for it in range(3):
        lls = []
        for u in range(2):
            swarm = np.concatenate([S, Us[:, u]], axis=1)
            cool = np.array([_cool(i, it, 4) for i in range(4)], f32)
            dr = {k: ref_lg1d[f"pmif_{k}"][it, u][None] for k in ("zp0", "zp", "z0", "z", "u")}
            out = cora.perfilter(1, 1, 1, swarm, ys[u], 12, SIG, SIG0, cool, cool[0], inject=dr)
            S = out["swarm"][:, :2]
            Us[:, u] = out["swarm"][:, 2:]
            lls.append(out["loglik"][0])
    want_s, want_u = _gold_mif(ref_values)
    got_s = np.concatenate([[sum(lls)], S[0].mean(axis=1, dtype=f32)])
    got_u = np.concatenate([np.concatenate([[lls[u]], Us[0, u].mean(axis=1, dtype=f32)]) for u in range(2)])
    _close(got_s, want_s, tol)
    _close(got_u, want_u, tol)


def _ricker_panel(lengths=(20, 35, 50)):
    import pypomp_b200 as pp

    units = {f"u{i}": pp.Ricker(T=T, key=i) for i, T in enumerate(lengths)}
    shared = pd.DataFrame({"shared": [0.3, 10.0]}, index=["sigma", "phi"])
    spec = pd.DataFrame([[44.7, 40.0, 50.0], [7.0, 6.0, 8.0]], index=["r", "N_0"], columns=list(units))
    return pp.PanelPomp(units, pp.PanelParameters({"shared": shared, "unit_specific": spec}))


def test_panel_struct_padding_and_permutations():
    from pypomp_b200.functional import _panel_thetas

    pan = _ricker_panel()
    st = pan.to_struct()
    assert st.ys.shape == (3, 50, 1)
    assert list(st.T_u) == [20, 35, 50]
    assert np.all(st.ys[0, 20:] == 0)
    # panel order [sigma, phi | r, N_0]; Ricker canonical order [r, sigma, phi, N_0]
    assert st.param_names == ["sigma", "phi", "r", "N_0"]
    assert st.permutations[0].tolist() == [2, 0, 1, 3]
    th = _panel_thetas(pan.theta.shared_array()[:, None, :].repeat(2, 1),
                       pan.theta.unit_array(st.unit_names)[:, None].repeat(2, 1), st.permutations)
    assert th.shape == (1, 2, 3, 4)
    np.testing.assert_allclose(th[0, 0, 1], [40.0, 0.3, 10.0, 6.0])


def test_panel_parameters_round_trip():
    import pypomp_b200 as pp

    pan = _ricker_panel()
    names = pan.get_unit_names()
    sh = np.array([[0.2, 9.0], [0.4, 11.0]])
    un = np.arange(12, dtype=float).reshape(2, 3, 2)
    p = pp.PanelParameters.from_arrays(sh, un, ["sigma", "phi"], ["r", "N_0"], names)
    assert p.num_replicates() == 2
    np.testing.assert_array_equal(p.shared_array(), sh)
    np.testing.assert_array_equal(p.unit_array(names), un)
