"""Parity at the benchmark configurations' own sizes (GPU).

* C2 -- LG 2-D, T = 1000, J = 262144, 64 seeds in one call: the log-mean-exp
  of the 64 log-likelihoods is within Monte Carlo error of the exact FP64
  Kalman log-likelihood and within 1e-4 of it relative; two of the seeds are
  re-run by the C oracle over the whole horizon and agree bit for bit (every
  conditional log-likelihood to float64 rounding of log(), which any changed
  ancestor anywhere in the run would break).
* C3 -- SV MOP-alpha (alpha = 0.97), T = 2000, J = 65536: the adjoint gradient
  of every parameter against central finite differences (h = 1e-3) of the
  MOP-alpha surrogate with the ancestry and stop_gradient(m) of the GPU run
  frozen, relative error <= 1e-3 (the surrogate evaluated in float64 on the
  same injected normals, the perturbed evaluations in parallel threads).
* C4 -- Ricker 32 x 32 (log r, sigma) grid, J = 16384, T = 500, all 1024
  filters in one call: four grid points re-run by the C oracle agree bit for
  bit.
"""

import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import cora, kalman

pytestmark = pytest.mark.gpu
f32 = np.float32


def test_c2_full_configuration_against_kalman_and_oracle():
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.maths import logmeanexp, logmeanexp_se
    from tests.conftest import LG2_Q, LG2_R

    T, J, NS = 1000, 262144, 64
    m = pp.LG(T=T, Q=LG2_Q, R=LG2_R, key=0)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names), NS, axis=0).astype(f32)
    seeds = np.arange(NS, dtype=np.uint64)
    got = F.run_pfilter(st, th, seeds, J, path="stream", CLL=True)
    ll = got["loglik"]
    A, C, Q, R, X0 = kalman.lg_matrices(th[0].astype(np.float64), 2, 2)
    exact = kalman.kalman_loglik(st.ys, A, C, Q, R, X0)
    lme, se = logmeanexp(ll), logmeanexp_se(ll)
    assert abs(lme - exact) <= 5 * se, (lme, exact, se)
    assert abs(lme - exact) / abs(exact) <= 1e-4, (lme, exact)
    assert np.all(np.isfinite(ll))
    np.testing.assert_allclose(got["cll"].sum(axis=1), ll, rtol=1e-12)
    pick = np.array([0, 37])
    want = cora.pfilter(1, 2, 2, th[pick], st.ys, J, seeds=seeds[pick], CLL=True, nthreads=2)
    np.testing.assert_allclose(got["cll"][pick], want["cll"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(ll[pick], want["loglik"], rtol=1e-12)


def test_c3_sv_mop_gradient_against_frozen_ancestry_differences():
    """The adjoint at T = 2000, J = 65536 against central differences (h = 1e-3)
    of the surrogate evaluated in float64 (oracle/mop_fp64.py) with the GPU
    run's ancestors and stop_gradient(m) frozen, on injected normals.  (In
    float32 the quotient of a 2000-step series carries a rounding error of
    about 0.1 in the rho component: rho enters every log-density through one
    rounded constant, so T ulps of it move the objective coherently.)"""
    import os

    import pypomp_b200 as pp
    from oracle.mop_fp64 import sv_surrogate
    from pypomp_b200 import functional as F

    T, J, alpha = 2000, 65536, 0.97
    m = pp.SV(T=T, key=0)
    st = m.to_struct()
    spec = m.spec
    th = spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    rng = np.random.default_rng(2000)
    z = rng.standard_normal((1, T, J, 1)).astype(f32)
    u = rng.random((1, T)).astype(f32)
    got = F.run_mop(st, th, np.zeros(1, np.uint64), J, alpha, grad=True, save_ancestors=True,
                    inject={"z": z, "u": u})
    g = got["grad"][0]
    assert np.all(np.isfinite(g))
    anc = got["anc"][0]
    zz = z[0, :, :, 0]
    base, m0 = sv_surrogate(th[0].astype(np.float64), st.ys, spec.dt, zz, anc, alpha)
    np.testing.assert_allclose(base, got["value"][0], rtol=1e-5)
    h = 1e-3
    P = th.shape[1]
    pts = []
    for p in range(P):
        for sgn in (1.0, -1.0):
            t = th[0].astype(np.float64)
            t[p] += sgn * h
            pts.append(t)

    def surrogate(t):
        return sv_surrogate(t, st.ys, spec.dt, zz, anc, alpha, m0)[0]

    with ThreadPoolExecutor(max_workers=min(len(pts), max(1, os.cpu_count() or 1))) as ex:
        vals = list(ex.map(surrogate, pts))
    fd = np.array([(vals[2 * p] - vals[2 * p + 1]) / (2 * h) for p in range(P)])
    err = np.linalg.norm(g - fd) / np.linalg.norm(fd)
    print("C3 gradient", g.tolist(), "central differences (float64 surrogate)", fd.tolist(),
          "relative error", err)
    assert err <= 1e-3, (err, g, fd)


def test_c4_ricker_grid_points_bit_exact():
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F

    T, J = 500, 16384
    m = pp.Ricker(T=T, key=0)
    st = m.to_struct()
    lr = np.linspace(3.0, 4.6, 32)
    sg = np.linspace(0.05, 0.8, 32)
    grid = np.array([[math.exp(a), b, 10.0, 7.0] for a in lr for b in sg], f32)
    seeds = np.arange(grid.shape[0], dtype=np.uint64)
    got = F.run_pfilter(st, grid, seeds, J, CLL=True)
    pick = np.array([0, 333, 700, 1023])
    want = cora.pfilter(m.spec.kind, 1, 1, grid[pick], st.ys, J, seeds=seeds[pick],
                        ycon=m.spec.ycon(st.ys), CLL=True, nthreads=4)
    np.testing.assert_allclose(got["loglik"][pick], want["loglik"], rtol=1e-12)
    np.testing.assert_allclose(got["cll"][pick], want["cll"], rtol=1e-12, atol=1e-12)
