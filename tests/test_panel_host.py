"""Panel parameter housekeeping on the CPU: prune and mix-and-match
(pypomp/core/parameters/base.py:138-181, pypomp/core/parameters/panel.py:504-585)."""

import numpy as np
import pandas as pd
import pytest


def _params():
    import pypomp_b200 as pp

    units = ["a", "b", "c"]
    reps = []
    for r in range(3):
        sh = pd.DataFrame({"shared": [0.1 * (r + 1), 10.0 + r]}, index=["sigma", "phi"])
        us = pd.DataFrame([[40.0 + r, 41.0 + r, 42.0 + r], [7.0 + r, 8.0 + r, 9.0 + r]],
                          index=["r", "N_0"], columns=units)
        reps.append({"shared": sh, "unit_specific": us})
    ll = np.array([[-10.0, -20.0, -30.0],     # replicate 0
                   [-12.0, -15.0, -31.0],     # replicate 1
                   [-11.0, -25.0, -29.0]])    # replicate 2
    return pp.PanelParameters(reps, logLik_unit=ll), units, ll


def test_mixed_and_matched_pairs_ranks():
    p, units, ll = _params()
    m = p.mixed_and_matched(units)
    # shared by panel log-likelihood: totals -60, -58, -65 -> order 1, 0, 2
    assert [d["shared"].loc["sigma", "shared"] for d in m.params()] == pytest.approx([0.2, 0.1, 0.3])
    # unit a ranks 0, 2, 1; unit b ranks 1, 0, 2; unit c ranks 2, 0, 1
    want_r = {"a": [40.0, 42.0, 41.0], "b": [42.0, 41.0, 43.0], "c": [44.0, 42.0, 43.0]}
    for u in units:
        assert [d["unit_specific"].loc["r", u] for d in m.params()] == want_r[u]
    assert m.logLik_unit[0].tolist() == [-10.0, -15.0, -29.0]
    assert m.logLik[0] == pytest.approx(ll.max(axis=0).sum())


def test_pruned_keeps_the_best_and_refills():
    p, units, ll = _params()
    q = p.pruned(n=1)
    assert q.num_replicates() == 3
    assert all(d["shared"].loc["sigma", "shared"] == pytest.approx(0.2) for d in q.params())
    assert np.all(q.logLik == ll[1].sum())
    q2 = p.pruned(n=2, refill=False)
    assert q2.num_replicates() == 2
    assert [d["shared"].loc["sigma", "shared"] for d in q2.params()] == pytest.approx([0.2, 0.1])
    with pytest.raises(ValueError):
        p.pruned(n=0)


def test_align_params_orders_and_reports_missing_names():
    from pypomp_b200 import functional as F

    assert F.align_params({"beta": 0.5, "gamma": 0.1}, ["gamma", "beta"]).tolist() == [0.1, 0.5]
    out = F.align_params({"beta": np.array([0.5, 0.6]), "gamma": np.array([0.1, 0.2])}, ["gamma", "beta"])
    assert out.shape == (2, 2) and out[:, 0].tolist() == [0.1, 0.2] and out[:, 1].tolist() == [0.5, 0.6]
    with pytest.raises(KeyError, match="required by the model structure"):
        F.align_params({"beta": 0.5}, ["gamma", "beta"])
