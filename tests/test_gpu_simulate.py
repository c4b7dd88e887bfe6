"""ppf_simulate on the GPU against the oracle: trajectories bit for bit.

The kernel and the oracle (oracle/ppf_oracle.c, ``ppfo_simulate``) draw from
the same streams with the same float32 arithmetic, so states and observations
must be identical -- LG in 1-4 dimensions (static and run-time dy), SV, and
Ricker with Poisson means on both sides of the sampler's switch at 10.  The
reference-facing API (``functional.simulate``, ``Pomp.simulate``) is checked
for the reference's layouts and DataFrame columns
(pypomp/functional/simulate.py:8-72, pypomp/core/estimation_mixin.py:1101-1222).
"""

import math

import numpy as np
import pytest

from oracle import cora

pytestmark = pytest.mark.gpu


def _struct(model):
    return model.to_struct()


def _cases():
    import pypomp_b200 as pp

    return {
        "lg1": pp.LG(T=6, A=[[0.9]], C=[[1.0]], Q=[[0.2]], R=[[0.3]], X0=[0.5], key=0),
        "lg2": pp.LG(T=6, key=0),
        "lg3x2": pp.LG(T=6, A=np.eye(3) * 0.8, C=np.ones((2, 3)) * 0.5, Q=np.eye(3) * 0.1,
                       R=np.eye(2) * 0.2, X0=np.zeros(3), key=0),
        "lg4": pp.LG(T=6, A=np.eye(4) * 0.7, C=np.eye(4), Q=np.eye(4) * 0.1, R=np.eye(4) * 0.2,
                     X0=np.ones(4), key=0),
        "sv": pp.SV(T=6, key=0),
        "ricker": pp.Ricker(T=6, key=0),
        "ricker_small": pp.Ricker(T=6, r=math.exp(2.0), phi=0.8, key=0),
    }


@pytest.mark.parametrize("name", ["lg1", "lg2", "lg3x2", "lg4", "sv", "ricker", "ricker_small"])
@pytest.mark.parametrize("nsim,T", [(1, 1), (5, 0), (130, 19), (300, 64)])
def test_simulate_matches_oracle_bit_for_bit(name, nsim, T):
    from pypomp_b200 import functional as F

    m = _cases()[name]
    st = _struct(m)
    th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    thetas = np.concatenate([th, th * np.float32(1.01)], axis=0)
    seeds = np.array([3, 99], np.uint64)
    times = np.arange(1, T + 1, dtype=float)
    X, Y = F.simulate(st, thetas, nsim, seeds, times=times)
    spec = st.spec
    Xo, Yo = cora.simulate(spec.kind, spec.dx, spec.dy, thetas, nsim, T, seeds, dt=spec.dt)
    assert X.shape == (2, nsim, T + 1, spec.dx) and Y.shape == (2, nsim, T, spec.dy)
    assert np.array_equal(X, Xo, equal_nan=True)
    assert np.array_equal(Y, Yo, equal_nan=True)


def test_simulate_estimation_scale_equals_natural():
    from pypomp_b200 import functional as F

    # Ricker on the estimation scale: bit for bit against the oracle
    m = _cases()["ricker"]
    st = _struct(m)
    th = m.theta.to_array(m.canonical_param_names)
    X2, Y2 = F.simulate(st, np.log(th).astype(np.float32), 40, [5], est=True)
    Xo, Yo = cora.simulate(3, 1, 1, np.log(th).astype(np.float32), 40, 6, [5], est=True)
    assert np.array_equal(X2, Xo) and np.array_equal(Y2, Yo)
    # LG (stable, linear): natural and estimation scale agree to float32 rounding
    # of exp(log(.)); chaotic Ricker paths would amplify that rounding
    m = _cases()["lg2"]
    st = _struct(m)
    th = m.theta.to_array(m.canonical_param_names)
    X1, Y1 = F.simulate(st, th.astype(np.float32), 40, [5])
    X3, Y3 = F.simulate(st, st.spec.to_est(th).astype(np.float32), 40, [5], est=True)
    assert np.allclose(X1, X3, rtol=1e-4, atol=1e-5) and np.allclose(Y1, Y3, rtol=1e-4, atol=1e-5)


def test_pomp_simulate_frames_and_as_pomp():
    m = _cases()["lg2"]
    states, obs = m.simulate(key=4, nsim=3)
    T = len(m.ys)
    assert list(states.columns) == ["theta_idx", "sim", "time"] + m.statenames
    assert list(obs.columns) == ["theta_idx", "sim", "time"] + list(m.ys.columns)
    assert len(states) == 3 * (T + 1) and len(obs) == 3 * T
    assert states["time"].iloc[0] == m.t0
    assert np.array_equal(obs["time"].to_numpy()[:T], m.ys.index.to_numpy())
    with pytest.warns(UserWarning, match="as_pomp overrides nsim"):
        new = m.simulate(key=4, nsim=2, as_pomp=True)
    assert new.ys.shape == m.ys.shape and list(new.ys.columns) == list(m.ys.columns)
    # the first replicate of the first parameter set, under the same key
    _, obs1 = m.simulate(key=4, nsim=1)
    assert np.array_equal(new.ys.to_numpy(), obs1[list(m.ys.columns)].to_numpy())
    # a model built on simulated data filters to a finite log-likelihood
    new.pfilter(J=500, key=1)
    assert np.isfinite(new.results()["logLik"].iloc[0])


def test_simulate_rejects_bad_arguments():
    from pypomp_b200 import functional as F

    m = _cases()["lg2"]
    st = _struct(m)
    th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    with pytest.raises(ValueError):
        F.simulate(st, th, 0, [1])
    with pytest.raises(ValueError):
        F.simulate(st, th, 2, [1, 2])


def test_panel_simulate_units_and_as_pomp():
    import pandas as pd

    import pypomp_b200 as pp
    from pypomp_b200 import random as pprandom
    from pypomp_b200.pomp import PompParameters

    units = {f"u{i}": pp.Ricker(T=8 + 3 * i, key=i) for i in range(3)}
    sh = pd.DataFrame({"shared": [0.3, 10.0]}, index=["sigma", "phi"])
    sp = pd.DataFrame([[40.0, 45.0, 50.0], [7.0, 7.0, 7.0]], index=["r", "N_0"], columns=list(units))
    pan = pp.PanelPomp(units, pp.PanelParameters({"shared": sh, "unit_specific": sp}))
    X, Y = pan.simulate(key=9, nsim=2)
    assert list(X.columns) == ["unit", "theta_idx", "sim", "time", "N"]
    assert list(Y.columns) == ["unit", "theta_idx", "sim", "time", "y"]
    for i, u in enumerate(units):
        T = 8 + 3 * i
        assert (X["unit"] == u).sum() == 2 * (T + 1) and (Y["unit"] == u).sum() == 2 * T
    # unit u1 equals its own Pomp.simulate under the key the panel derives for it
    k = pprandom.as_key(9)
    k, _ = pprandom.split(k)
    k, sub = pprandom.split(k)
    one = pp.Ricker(T=11, key=1)
    _, Y1 = one.simulate(key=sub, theta=PompParameters(pan.get_unit_parameters("u1")), nsim=2)
    assert np.array_equal(Y[Y["unit"] == "u1"]["y"].to_numpy(), Y1["y"].to_numpy())
    new = pan.simulate(key=9, as_pomp=True)
    assert [len(new.unit_objects[u].ys) for u in units] == [8, 11, 14]
    new.pfilter(J=300, key=2)
    assert np.all(np.isfinite(new.results()["unit logLik"].to_numpy(dtype=float)))
