"""Float32 NumPy restatements of the built-in models, vectorised over particles.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

* ``LG``: ``pypomp/models/linear_gaussian.py:139-215``.  Parameters are the
  natural-scale vector in LG's canonical order ``A`` (row-major), ``C``
  (row-major), lower triangle of the Cholesky factor of ``Q`` and ``R``
  (row-major), ``X0``.  ``_to_est`` takes the log of the factor diagonals
  (``linear_gaussian.py:202-215``).  ``dmeas`` restates
  ``jax.scipy.stats.multivariate_normal.logpdf`` with ``cov = L_R L_R^T``:
  Cholesky of cov, triangular solve, ``-|y|^2/2 - n/2 log(2 pi) - sum log diag``.
* ``SV``: discretised Heston-type log-variance model (no reference counterpart;
  its structure follows ``pypomp/models/spx.py:66-158``).  State ``(v, eps)``
  where ``eps`` is the latest volatility shock; parameters
  ``kappa, theta, xi, rho, mu, v0`` on the natural scale.  Per step
  ``v' = v + kappa (theta - e^v) e^{-v} dt + xi e^{-v/2} sqrt(dt) eps'`` and
  the return density is ``N(mu dt + rho sqrt(e^{v'} dt) eps', (1-rho^2) e^{v'} dt)``.
  Estimation scale: log kappa, log theta, log xi, atanh rho, mu, v0.
* ``Ricker``: ``N' = r N exp(-N + sigma e)``, ``y ~ Poisson(phi N')``.
  Parameters ``r, sigma, phi, N_0``; estimation scale takes logs of all four.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

f32 = np.float32


def _lg_dims(P: int):
    for dx in range(1, 10):
        for dy in range(1, 10):
            if dx * dx + dy * dx + dx * (dx + 1) // 2 + dy * (dy + 1) // 2 + dx == P:
                return dx, dy
    raise ValueError(f"no LG dims for {P} parameters")


class _LG:
    name = "LG"

    @staticmethod
    def layout(dx, dy):
        return {
            "A": (0, dx * dx),
            "C": (dx * dx, dx * dx + dy * dx),
            "Q": (dx * dx + dy * dx, dx * dx + dy * dx + dx * (dx + 1) // 2),
            "R": (dx * dx + dy * dx + dx * (dx + 1) // 2,
                  dx * dx + dy * dx + dx * (dx + 1) // 2 + dy * (dy + 1) // 2),
            "X0": (dx * dx + dy * dx + dx * (dx + 1) // 2 + dy * (dy + 1) // 2,
                   dx * dx + dy * dx + dx * (dx + 1) // 2 + dy * (dy + 1) // 2 + dx),
        }

    @staticmethod
    def _tril(v, d):
        L = np.zeros((d, d), f32)
        k = 0
        for i in range(d):
            for j in range(i + 1):
                L[i, j] = v[k]
                k += 1
        return L

    def unpack(self, theta):
        theta = np.asarray(theta, f32)
        dx, dy = _lg_dims(theta.shape[-1])
        lay = self.layout(dx, dy)
        A = theta[slice(*lay["A"])].reshape(dx, dx)
        C = theta[slice(*lay["C"])].reshape(dy, dx)
        LQ = self._tril(theta[slice(*lay["Q"])], dx)
        LR = self._tril(theta[slice(*lay["R"])], dy)
        X0 = theta[slice(*lay["X0"])]
        return {"dx": dx, "dy": dy, "A": A, "C": C, "LQ": LQ, "LR": LR, "X0": X0}

    def diag_index(self, P):
        dx, dy = _lg_dims(P)
        lay = self.layout(dx, dy)
        idx = []
        for key, d in (("Q", dx), ("R", dy)):
            k = lay[key][0]
            for i in range(d):
                for j in range(i + 1):
                    if i == j:
                        idx.append(k)
                    k += 1
        return idx

    def to_est(self, theta):
        t = np.array(theta, f32, copy=True)
        idx = self.diag_index(t.shape[-1])
        t[..., idx] = np.log(t[..., idx])
        return t

    def from_est(self, theta):
        t = np.array(theta, f32, copy=True)
        idx = self.diag_index(t.shape[-1])
        t[..., idx] = np.exp(t[..., idx])
        return t

    def n_init(self, p):
        return p["dx"]

    def n_step(self, p):
        return p["dx"]

    def n_meas(self, p):
        return p["dy"]

    def rinit(self, p, z):
        # X0 + L_Q @ z  (linear_gaussian.py:139-148)
        return (p["X0"][None, :] + z @ p["LQ"].T).astype(f32)

    def rproc(self, p, X, z, t):
        # A @ X + L_Q @ z  (linear_gaussian.py:151-163)
        return (X @ p["A"].T + z @ p["LQ"].T).astype(f32)

    def dmeas(self, p, y, X):
        # multivariate_normal.logpdf(y; C X, L_R L_R^T)  (linear_gaussian.py:166-177)
        cov = (p["LR"] @ p["LR"].T).astype(f32)
        L = np.linalg.cholesky(cov.astype(f32)).astype(f32)
        r = (np.asarray(y, f32)[None, :] - X @ p["C"].T).astype(f32)
        sol = np.linalg.solve(L, r.T).T.astype(f32)
        n = p["dy"]
        return (f32(-0.5) * np.sum(sol * sol, axis=1, dtype=f32)
                - f32(n / 2) * f32(math.log(2 * math.pi))
                - np.sum(np.log(np.diag(L)), dtype=f32)).astype(f32)

    def rmeas(self, p, X, z):
        return (X @ p["C"].T + z @ p["LR"].T).astype(f32)


@dataclass
class SVConst:
    dt: float = 1.0 / 252.0


class _SV:
    name = "SV"
    names = ["kappa", "theta", "xi", "rho", "mu", "v0"]
    dt = f32(1.0 / 252.0)

    def unpack(self, theta):
        t = np.asarray(theta, f32)
        return dict(zip(self.names, t))

    def to_est(self, theta):
        t = np.array(theta, f32, copy=True)
        t[..., 0:3] = np.log(t[..., 0:3])
        t[..., 3] = np.arctanh(t[..., 3])
        return t

    def from_est(self, theta):
        t = np.array(theta, f32, copy=True)
        t[..., 0:3] = np.exp(t[..., 0:3])
        t[..., 3] = np.tanh(t[..., 3])
        return t

    def n_init(self, p):
        return 0

    def n_step(self, p):
        return 1

    def n_meas(self, p):
        return 1

    def rinit(self, p, z):
        J = z.shape[0]
        X = np.zeros((J, 2), f32)
        X[:, 0] = p["v0"]
        return X

    def rproc(self, p, X, z, t):
        v = X[:, 0]
        eps = z[:, 0]
        dt = self.dt
        ev = np.exp(-v).astype(f32)
        vn = (v + p["kappa"] * (p["theta"] - np.exp(v)) * ev * dt
              + p["xi"] * np.exp(f32(-0.5) * v) * np.sqrt(dt) * eps).astype(f32)
        return np.stack([vn, eps], axis=1).astype(f32)

    def dmeas(self, p, y, X):
        v = X[:, 0]
        eps = X[:, 1]
        dt = self.dt
        sd = np.sqrt(np.exp(v) * dt).astype(f32)
        mean = (p["mu"] * dt + p["rho"] * sd * eps).astype(f32)
        s = (np.sqrt(f32(1.0) - p["rho"] * p["rho"]) * sd).astype(f32)
        r = ((f32(y[0]) - mean) / s).astype(f32)
        return (f32(-0.5) * r * r - np.log(s) - f32(0.5 * math.log(2 * math.pi))).astype(f32)

    def rmeas(self, p, X, z):
        v = X[:, 0]
        eps = X[:, 1]
        dt = self.dt
        sd = np.sqrt(np.exp(v) * dt)
        return (p["mu"] * dt + sd * (p["rho"] * eps + np.sqrt(1 - p["rho"] ** 2) * z[:, 0]))[:, None].astype(f32)


class _Ricker:
    name = "Ricker"
    names = ["r", "sigma", "phi", "N_0"]

    def unpack(self, theta):
        t = np.asarray(theta, f32)
        return dict(zip(self.names, t))

    def to_est(self, theta):
        return np.log(np.asarray(theta, f32)).astype(f32)

    def from_est(self, theta):
        return np.exp(np.asarray(theta, f32)).astype(f32)

    def n_init(self, p):
        return 0

    def n_step(self, p):
        return 1

    def n_meas(self, p):
        return 1

    def rinit(self, p, z):
        return np.full((z.shape[0], 1), p["N_0"], f32)

    def rproc(self, p, X, z, t):
        N = X[:, 0]
        return (p["r"] * N * np.exp(-N + p["sigma"] * z[:, 0]))[:, None].astype(f32)

    def dmeas(self, p, y, X):
        lam = (p["phi"] * X[:, 0]).astype(f32)
        yv = f32(y[0])
        with np.errstate(divide="ignore", invalid="ignore"):
            ll = yv * np.log(lam) - lam - f32(math.lgamma(float(yv) + 1.0))
        if yv == 0:
            ll = -lam
        return ll.astype(f32)

    def rmeas(self, p, X, z):
        raise NotImplementedError("Ricker observations are simulated with numpy Poisson draws")


MODELS = {"LG": _LG(), "SV": _SV(), "Ricker": _Ricker()}
