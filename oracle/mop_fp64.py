"""FP64 MOP-alpha surrogate with frozen ancestry -- TEST INFRASTRUCTURE ONLY.

The gradient check of the MOP-alpha adjoint compares it with central finite
differences of the surrogate objective whose resampling ancestors and
stop_gradient(m) are frozen at the values of the run being differentiated
(``pypomp/core/algorithms/mop.py:69-135``: carried weight
``wF = (wP + m - stop_gradient(m))[a]``, ``wP = alpha wF``, per-step term
``LSE(wP + m) - LSE(wP)``).  In float32 the difference quotient of a long
series is dominated by rounding: a parameter that enters every particle's
log-density through one rounded constant (the SV model's
``-log sqrt(1 - rho^2)``) moves the objective by T x ulp of that constant, so
at T = 2000 and h = 1e-3 the float32 quotient is off by about 0.1.  This
module evaluates the same surrogate with the model arithmetic in float64 on
injected normals, so the quotient is accurate to the truncation error.

``sv_surrogate`` restates the SV model of ``oracle/models_np.py`` (state
``(v, eps)``, ``v' = v + kappa dt (theta e^{-v} - 1) + xi sqrt(dt) e^{-v/2} z``,
``eps' = z``, returns ``N(mu dt + rho sd eps', (1 - rho^2) sd^2)`` with
``sd = e^{v'/2} sqrt(dt)``) on the estimation scale
``(log kappa, log theta, log xi, atanh rho, mu, v0)``.
"""

from __future__ import annotations

import numpy as np


def _lse(v: np.ndarray) -> float:
    m = np.max(v)
    if not np.isfinite(m):
        return float(m)
    return float(m + np.log(np.sum(np.exp(v - m))))


def sv_surrogate(theta_est, ys, dt: float, z, anc, alpha: float, m0=None):
    """Negative MOP-alpha surrogate of one SV filter in float64.

    ``theta_est`` (6,), ``ys`` (T,) or (T, 1), ``z`` (T, J) process normals
    (the normal of particle j on the step into observation t), ``anc`` (T, J)
    frozen ancestors, ``m0`` (T, J) frozen stop_gradient(m) or None (recorded
    at these parameters).  Returns ``(value, m0)``.
    """
    th = np.asarray(theta_est, dtype=np.float64)
    kappa, theta, xi = np.exp(th[0]), np.exp(th[1]), np.exp(th[2])
    rho, mu, v0 = np.tanh(th[3]), th[4], th[5]
    ys = np.asarray(ys, dtype=np.float64).reshape(-1)
    z = np.asarray(z, dtype=np.float64)
    anc = np.asarray(anc)
    T, J = z.shape
    rc = np.sqrt(1.0 - rho * rho)
    sqdt = np.sqrt(dt)
    c0 = -0.5 * np.log(2.0 * np.pi) - np.log(rc) - 0.5 * np.log(dt)
    rec = np.empty((T, J)) if m0 is None else None
    v = np.full(J, v0)
    wF = np.full(J, -np.log(J))
    ll = 0.0
    for t in range(T):
        wP = alpha * wF
        emh = np.exp(-0.5 * v)
        vp = v + kappa * dt * (theta * emh * emh - 1.0) + xi * sqdt * emh * z[t]
        eps = z[t]
        sd = np.exp(0.5 * vp) * sqdt
        r = (ys[t] - (mu * dt + rho * sd * eps)) / (rc * sd)
        m = -0.5 * r * r - 0.5 * vp + c0
        ll += _lse(wP + m) - _lse(wP)
        mt = m if m0 is None else m0[t]
        if rec is not None:
            rec[t] = m
        a = anc[t]
        wF = (wP + m - mt)[a]
        v = vp[a]
    return -ll, (rec if m0 is None else m0)


def central_differences(fn, theta, h: float = 1e-3):
    """(f(theta + h e_p) - f(theta - h e_p)) / 2h for every p, in float64."""
    theta = np.asarray(theta, dtype=np.float64)
    g = np.zeros(theta.size)
    for p in range(theta.size):
        e = np.zeros(theta.size)
        e[p] = h
        g[p] = (fn(theta + e) - fn(theta - e)) / (2.0 * h)
    return g
