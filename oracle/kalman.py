"""FP64 Kalman filter: the exact log-likelihood of the LG model.

TEST INFRASTRUCTURE ONLY.  Generalises the reference's 1-D helper
(``tests/helpers/kalman.py:13-32``) to matrices, with LG's convention that the
initial state is drawn from N(X0, Q) at t0 and propagated once before the first
observation (so the filter starts from P0 = Q, ``tests/helpers/lg_accuracy.py:26-28``).
"""

from __future__ import annotations

import numpy as np


def kalman_loglik(ys, A, C, Q, R, X0, P0=None) -> float:
    ys = np.asarray(ys, dtype=np.float64)
    A, C, Q, R = (np.atleast_2d(np.asarray(M, dtype=np.float64)) for M in (A, C, Q, R))
    x = np.asarray(X0, dtype=np.float64).reshape(-1)
    P = Q.copy() if P0 is None else np.atleast_2d(np.asarray(P0, dtype=np.float64))
    ll = 0.0
    for y in ys:
        xp = A @ x
        Pp = A @ P @ A.T + Q
        v = np.atleast_1d(y) - C @ xp
        S = C @ Pp @ C.T + R
        Sc = np.linalg.cholesky(S)
        sol = np.linalg.solve(Sc, v)
        ll += -0.5 * (len(v) * np.log(2 * np.pi) + 2 * np.sum(np.log(np.diag(Sc))) + sol @ sol)
        K = Pp @ C.T @ np.linalg.inv(S)
        x = xp + K @ v
        P = (np.eye(len(x)) - K @ C) @ Pp
    return float(ll)


def lg_matrices(theta: np.ndarray, dx: int, dy: int):
    """(A, C, Q, R, X0) from LG's canonical natural-scale vector."""
    t = np.asarray(theta, dtype=np.float64)
    p = 0
    A = t[p:p + dx * dx].reshape(dx, dx); p += dx * dx
    C = t[p:p + dy * dx].reshape(dy, dx); p += dy * dx
    LQ = np.zeros((dx, dx))
    for i in range(dx):
        for j in range(i + 1):
            LQ[i, j] = t[p]; p += 1
    LR = np.zeros((dy, dy))
    for i in range(dy):
        for j in range(i + 1):
            LR[i, j] = t[p]; p += 1
    X0 = t[p:p + dx]
    return A, C, LQ @ LQ.T, LR @ LR.T, X0
