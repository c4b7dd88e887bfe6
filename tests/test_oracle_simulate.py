"""The oracle's simulation and the shared Poisson sampler (CPU).

The sampler (include/ppf_sample.h) is pinned by its distribution: chi-square
goodness of fit to the Poisson pmf on both branches (inversion below a mean
of 10, PTRS at and above it), its special cases, and log k! against lgamma.
The trajectories are pinned by their construction: the initial state and
every transition and observation follow the model's formulas from the
documented draw streams, and their moments match the model's.
"""

import math

import numpy as np
import pytest
from scipy import stats

from oracle import cora

LG, SV, RICKER = 1, 2, 3


@pytest.mark.parametrize("lam", [0.05, 0.7, 4.0, 9.99, 10.0, 23.0, 150.0, 4000.0])
def test_poisson_sampler_fits_the_pmf(lam):
    n = 20000
    draws = np.array([cora.poisson(lam, 11, k, 5) for k in range(n)])
    assert np.all(draws == np.floor(draws)) and draws.min() >= 0
    lo, hi = int(stats.poisson.ppf(1e-4, lam)), int(stats.poisson.ppf(1 - 1e-4, lam))
    edges = np.arange(lo, hi + 2)
    # merge cells until each expects at least 20 draws
    cells, cur = [], []
    for k in edges[:-1]:
        cur.append(k)
        if n * stats.poisson.pmf(cur, lam).sum() >= 20:
            cells.append(cur)
            cur = []
    if cur:
        cells[-1].extend(cur)
    obs = [np.isin(draws, c).sum() for c in cells]
    obs[0] += (draws < cells[0][0]).sum()
    obs[-1] += (draws > cells[-1][-1]).sum()
    exp = [n * stats.poisson.pmf(c, lam).sum() for c in cells]
    exp[0] += n * stats.poisson.cdf(cells[0][0] - 1, lam)
    exp[-1] += n * stats.poisson.sf(cells[-1][-1], lam)
    chi2 = sum((o - e) ** 2 / e for o, e in zip(obs, exp))
    p = stats.chi2.sf(chi2, len(cells) - 1)
    assert p > 1e-4, (lam, chi2, len(cells), p)


def test_poisson_special_values_and_determinism():
    assert cora.poisson(0.0, 1, 0, 1) == 0.0
    assert math.isnan(cora.poisson(float("nan"), 1, 0, 1))
    assert math.isnan(cora.poisson(-1.0, 1, 0, 1))
    assert cora.poisson(float("inf"), 1, 0, 1) == float("inf")
    a = [cora.poisson(37.0, 5, k, 9) for k in range(100)]
    b = [cora.poisson(37.0, 5, k, 9) for k in range(100)]
    c = [cora.poisson(37.0, 5, k, 10) for k in range(100)]
    assert a == b and a != c


def test_logfact_matches_lgamma():
    for k in list(range(40)) + [100, 1000, 12345, 10 ** 6]:
        want = math.lgamma(k + 1)
        assert abs(cora.logfact(k) - want) <= 4e-7 * max(1.0, want), k


def _lg_theta(dx, dy, A, C, LQ, LR, X0):
    th = list(np.asarray(A, float).ravel()) + list(np.asarray(C, float).ravel())
    for M, d in ((LQ, dx), (LR, dy)):
        M = np.asarray(M, float)
        th += [M[i, k] for i in range(d) for k in range(i + 1)]
    return np.asarray(th + list(X0), np.float32)


def test_lg_trajectories_follow_the_model_draws():
    """X_0 = X0 + L_Q z0, X_t = A X_{t-1} + L_Q z_t, Y_t = C X_t + L_R w_t with
    z from the process stream and w from the measurement stream (float64
    reconstruction; float32 rounding only)."""
    A = np.array([[0.9, 0.1], [-0.2, 0.8]])
    C = np.array([[1.0, 0.5], [0.0, 1.0]])
    LQ = np.array([[0.3, 0.0], [0.1, 0.2]])
    LR = np.array([[0.5, 0.0], [0.2, 0.4]])
    X0 = np.array([1.0, -1.0])
    th = _lg_theta(2, 2, A, C, LQ, LR, X0)
    seeds = np.array([77, 78], np.uint64)
    X, Y = cora.simulate(LG, 2, 2, np.stack([th, th]), 3, 12, seeds)
    assert X.shape == (2, 3, 13, 2) and Y.shape == (2, 3, 12, 2)
    L = cora._L()
    for f in range(2):
        for k in range(3):
            z = np.zeros(2, np.float32)
            L.ppfo_normals(int(seeds[f]), k, 0, 0, 2, z.ctypes.data)
            x = X0 + LQ @ z
            assert np.allclose(X[f, k, 0], x, atol=1e-5)
            for t in range(12):
                L.ppfo_normals(int(seeds[f]), k, t + 1, 0, 2, z.ctypes.data)
                x = A @ X[f, k, t].astype(float) + LQ @ z
                assert np.allclose(X[f, k, t + 1], x, atol=1e-5)
                w = np.zeros(2, np.float32)
                L.ppfo_normals(int(seeds[f]), k, t + 1, 3, 2, w.ctypes.data)
                assert np.allclose(Y[f, k, t], C @ X[f, k, t + 1].astype(float) + LR @ w, atol=1e-5)
    assert not np.array_equal(X[0], X[1])   # different keys, different paths


def test_sv_and_ricker_moments():
    # SV: the standardised return given (v, eps) is N(0, 1)
    dt = 1.0 / 252.0
    th = np.array([2.0, 0.04, 0.3, -0.7, 0.05, math.log(0.04)], np.float32)
    X, Y = cora.simulate(SV, 2, 1, th[None], 400, 50, [3], dt=dt)
    v, eps = X[0, :, 1:, 0].astype(float), X[0, :, 1:, 1].astype(float)
    sd = np.exp(0.5 * v) * math.sqrt(dt)
    r = (Y[0, :, :, 0] - (0.05 * dt + -0.7 * sd * eps)) / (math.sqrt(1 - 0.49) * sd)
    assert abs(r.mean()) < 0.03 and abs(r.std() - 1.0) < 0.03
    assert abs(eps.mean()) < 0.03 and abs(eps.std() - 1.0) < 0.03
    # Ricker: counts are Poisson(phi N): mean and variance of y - phi N
    th = np.array([math.exp(2.5), 0.3, 10.0, 7.0], np.float32)
    X, Y = cora.simulate(RICKER, 1, 1, th[None], 500, 40, [4])
    lam = 10.0 * X[0, :, 1:, 0].astype(float)
    resid = Y[0, :, :, 0] - lam
    assert abs(resid.mean()) < 0.1
    assert abs((resid ** 2).mean() / lam.mean() - 1.0) < 0.05
    assert np.all(Y == np.floor(Y))
