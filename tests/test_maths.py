"""logmeanexp / logmeanexp_se against their definitions and the edge cases the
reference's own tests fix (pypomp tests/test_maths.py: the R pomp value for
100..104, empty / all-NaN / -inf / single-value samples, ignore_nan)."""

import math
import time
import warnings

import numpy as np
import pytest

from pypomp_b200.maths import logmeanexp, logmeanexp_se


def _lme_direct(v):
    v = [float(t) for t in v]
    c = max(v)
    return c + math.log(math.fsum(math.exp(t - c) for t in v) / len(v))


def _se_direct(v):
    n = len(v)
    loo = [_lme_direct(v[:i] + v[i + 1:]) for i in range(n)]
    m = math.fsum(loo) / n
    return math.sqrt(n - 1) * math.sqrt(math.fsum((t - m) ** 2 for t in loo) / n)


def test_r_pomp_value():
    x = np.array([100.0, 101.0, 102.0, 103.0, 104.0])
    assert round(logmeanexp(x), 2) == 102.84
    assert round(logmeanexp_se(x), 2) == 0.75


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_matches_definition(seed):
    rng = np.random.default_rng(seed)
    v = list(rng.normal(-200.0, 3.0, size=37))
    assert logmeanexp(np.array(v)) == pytest.approx(_lme_direct(v), rel=1e-13)
    assert logmeanexp_se(np.array(v)) == pytest.approx(_se_direct(v), rel=1e-9)


def test_dominant_maximum():
    v = [100.0, 101.0, 1e10 + 2]
    se = logmeanexp_se(np.array(v))
    assert np.isfinite(se)
    assert se == pytest.approx(_se_direct(v), rel=1e-9)


@pytest.mark.parametrize("arr, lme_nan, se_nan", [
    (np.array([100.0]), False, True),
    (np.array([]), True, True),
    (np.array([np.nan, np.nan]), True, True),
    (np.array([100.0, 101.0, -np.inf]), False, False),
    (np.array([1.0, np.nan, -np.inf]), True, True),
    (np.array([42.0]), False, True),
])
def test_edge_cases(arr, lme_nan, se_nan):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)
        lme, se = logmeanexp(arr), logmeanexp_se(arr)
    assert np.isnan(lme) == lme_nan and (lme_nan or np.isfinite(lme))
    assert np.isnan(se) == se_nan and (se_nan or np.isfinite(se))


def test_ignore_nan_drops_entries():
    a = np.array([1.0, np.nan, 2.0, 3.0])
    b = np.array([1.0, 2.0, 3.0])
    assert logmeanexp(a, ignore_nan=True) == pytest.approx(logmeanexp(b), abs=1e-12)
    assert logmeanexp_se(a, ignore_nan=True) == pytest.approx(logmeanexp_se(b), abs=1e-12)
    assert np.isnan(logmeanexp(np.array([np.nan, np.nan]), ignore_nan=True))
    assert np.isnan(logmeanexp_se(np.array([np.nan, np.nan]), ignore_nan=True))


def test_axis_and_shift():
    rng = np.random.default_rng(5)
    x = rng.normal(size=(3, 4, 6))
    got = logmeanexp(x, axis=-1)
    assert got.shape == (3, 4)
    for i in range(3):
        for j in range(4):
            assert got[i, j] == pytest.approx(_lme_direct(list(x[i, j])), rel=1e-13)
    se = logmeanexp_se(x, axis=1)
    assert se.shape == (3, 6)
    assert se[1, 2] == pytest.approx(_se_direct(list(x[1, :, 2])), rel=1e-9)
    assert logmeanexp(x[0, 0] + 37.5) == pytest.approx(logmeanexp(x[0, 0]) + 37.5, rel=1e-12)


def test_large_sample_is_fast():
    v = np.random.default_rng(0).normal(size=10000)
    t0 = time.perf_counter()
    logmeanexp_se(v)
    assert time.perf_counter() - t0 < 2.0
