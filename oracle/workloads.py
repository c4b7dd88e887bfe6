"""Benchmark workloads built without the product package -- TEST INFRASTRUCTURE.

``bench.py --impl reference`` times the CPU restatement of the path and must
not load the CUDA library, so it builds its inputs here.  The data follow the
same recipe as ``pypomp_b200.models.LG`` (``numpy.random.default_rng(seed)``:
x0 ~ N(X0, Q), then per observation x = A x + L_Q z, y = C x + L_R z), and
``tests/test_bench_reference.py`` checks that both give identical arrays.
"""

from __future__ import annotations

import numpy as np

# The headline LG configuration: A = rot(0.2), C = I, Q = [[1, 1e-4], [1e-4, 1]] / 100,
# R = [[1, 0.1], [0.1, 1]] / 10, X0 = 0.
LG2_A = np.array([[np.cos(0.2), -np.sin(0.2)], [np.sin(0.2), np.cos(0.2)]])
LG2_Q = np.array([[1.0, 1e-4], [1e-4, 1.0]]) / 100
LG2_R = np.array([[1.0, 0.1], [0.1, 1.0]]) / 10


def lg_theta_vector(A, C, Q, R, X0) -> np.ndarray:
    """LG's canonical natural-scale vector: A and C row-major, the lower
    triangles of the Cholesky factors of Q and R row by row, X0."""
    LQ, LR = np.linalg.cholesky(Q), np.linalg.cholesky(R)
    dx, dy = A.shape[0], C.shape[0]
    tri = lambda L, d: [L[i, j] for i in range(d) for j in range(i + 1)]   # noqa: E731
    return np.array(list(A.ravel()) + list(C.ravel()) + tri(LQ, dx) + tri(LR, dy) + list(X0), dtype=np.float64)


def lg_simulate(A, C, Q, R, X0, T: int, seed: int) -> np.ndarray:
    """(T, dy) observations from the seeded generator, float64."""
    rng = np.random.default_rng(seed)
    LQ, LR = np.linalg.cholesky(Q), np.linalg.cholesky(R)
    dx, dy = A.shape[0], C.shape[0]
    x = np.asarray(X0, dtype=float) + LQ @ rng.standard_normal(dx)
    Y = np.zeros((T, dy))
    for t in range(T):
        x = A @ x + LQ @ rng.standard_normal(dx)
        Y[t] = C @ x + LR @ rng.standard_normal(dy)
    return Y


def headline_lg(T: int, seed: int = 0):
    """Canonical parameters (float32) and data (float32, (T, 2)) of the 2-D LG workload."""
    A, C, X0 = LG2_A, np.eye(2), np.zeros(2)
    theta = lg_theta_vector(A, C, LG2_Q, LG2_R, X0).astype(np.float32)
    ys = lg_simulate(A, C, LG2_Q, LG2_R, X0, T, seed).astype(np.float32)
    return theta, ys
