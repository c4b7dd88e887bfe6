"""Built-in models whose mechanics run as CUDA device functions.

Each factory mirrors the reference's model constructors
(``pypomp/models/linear_gaussian.py:337`` ``LG``; the SV and Ricker factories
follow the same pattern as ``pypomp/models/spx.py:161``) and returns a
:class:`pypomp_b200.pomp.Pomp` whose ``rinit/rproc/dmeas`` are the device code
in ``pypomp_b200/csrc/ppf_models.cuh``.  A ``ModelSpec`` carries what the C
ABI needs (kind, dims, parameter count) plus the canonical parameter names and
the natural <-> estimation transforms (``ParTrans``,
``pypomp/core/par_trans.py:70``).

Data are simulated on the host from a seeded NumPy generator (the reference
simulates with JAX, ``linear_gaussian.py:448``; its streams are not available
here).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import pandas as pd

from . import _ffi
from .pomp import Pomp

#: Largest LG state or observation dimension (pypomp/models/linear_gaussian.py:48).
MAX_DIM = 9


@dataclass(frozen=True)
class ModelSpec:
    kind: int
    dx: int
    dy: int
    param_names: tuple
    statenames: tuple
    obsnames: tuple
    dt: float = 0.0
    est_log: tuple = ()     # indices transformed by log / exp
    est_atanh: tuple = ()   # indices transformed by atanh / tanh
    name: str = ""
    natural: bool = False   # host-side identity transform (ParTrans() assigned after construction)

    @property
    def n_params(self) -> int:
        return len(self.param_names)

    def ffi_model(self) -> _ffi.PpfModel:
        return _ffi.PpfModel(self.kind, self.dx, self.dy, self.n_params, float(self.dt), 0)

    def _apply(self, theta, f_log, f_atanh) -> np.ndarray:
        t = np.array(theta, dtype=np.float64, copy=True)
        if self.natural:
            return t
        P = t.shape[-1]
        for cols, f in ((self.est_log, f_log), (self.est_atanh, f_atanh)):
            if not cols:
                continue
            if sorted(cols) == list(range(P)):
                t = f(t)                          # every column: one contiguous pass
            else:
                t[..., list(cols)] = f(t[..., list(cols)])
        return t

    def to_est(self, theta: np.ndarray) -> np.ndarray:
        return self._apply(theta, np.log, np.arctanh)

    def from_est(self, theta: np.ndarray) -> np.ndarray:
        return self._apply(theta, np.exp, np.tanh)

    def log_det_jac_from_est(self, theta_est: np.ndarray) -> np.ndarray:
        """log |det d from_est / d theta_est| (the change of variables a prior on
        the natural scale picks up on the estimation scale; the transforms are
        element-wise, so the Jacobian is diagonal: d exp(x) = exp(x),
        d tanh(x) = 1 - tanh(x)^2)."""
        t = np.asarray(theta_est, dtype=np.float64)
        out = np.zeros(t.shape[:-1])
        if self.natural:
            return out
        if self.est_log:
            out = out + t[..., list(self.est_log)].sum(axis=-1)
        if self.est_atanh:
            out = out + np.log1p(-np.tanh(t[..., list(self.est_atanh)]) ** 2).sum(axis=-1)
        return out

    def ycon(self, ys: np.ndarray) -> np.ndarray | None:
        """Per-observation constant of dmeas (Ricker: log y!), else None."""
        if self.kind == _ffi.MODEL_RICKER:
            # counts repeat: lgamma once per distinct finite value (0 where missing)
            y = np.asarray(ys, dtype=np.float64)[..., 0]
            out = np.zeros(y.shape, np.float64)
            fin = np.isfinite(y)
            vals, inv = np.unique(y[fin], return_inverse=True)
            out[fin] = np.array([math.lgamma(v + 1.0) for v in vals.tolist()], np.float64)[inv]
            return out.astype(np.float32)
        return None


# ---------------------------------------------------------------------------
# LG
# ---------------------------------------------------------------------------


def _lg_names(dx: int, dy: int):
    names = [f"A{i}{j}" for i in range(1, dx + 1) for j in range(1, dx + 1)]
    names += [f"C{i}{j}" for i in range(1, dy + 1) for j in range(1, dx + 1)]
    q = [f"Q{i}{j}" for i in range(1, dx + 1) for j in range(1, i + 1)]
    r = [f"R{i}{j}" for i in range(1, dy + 1) for j in range(1, i + 1)]
    names += q + r + [f"X0_{i}" for i in range(1, dx + 1)]
    return names


def lg_spec(dx: int, dy: int) -> ModelSpec:
    names = _lg_names(dx, dy)
    diag = [i for i, n in enumerate(names) if len(n) == 3 and n[0] in "QR" and n[1] == n[2]]
    return ModelSpec(
        kind=_ffi.MODEL_LG, dx=dx, dy=dy, param_names=tuple(names),
        statenames=tuple(f"X{i}" for i in range(1, dx + 1)),
        obsnames=tuple(f"Y{j}" for j in range(1, dy + 1)),
        est_log=tuple(diag), name="LG",
    )


def _default_A(dx):
    A = np.zeros((dx, dx))
    c, s = math.cos(0.2), math.sin(0.2)
    i = 0
    while i + 1 < dx:
        A[i:i + 2, i:i + 2] = [[c, -s], [s, c]]
        i += 2
    if i < dx:
        A[i, i] = c
    return A


def _default_cov(d, diag, off):
    M = np.eye(d) * diag
    if d > 1:
        M = M + (np.ones((d, d)) - np.eye(d)) * (off / (d - 1))
    return M


def lg_theta(A, C, Q, R, X0) -> dict:
    """LG's canonical parameter dict from matrices (Cholesky factors of Q, R)."""
    A, C, Q, R, X0 = (np.asarray(v, dtype=float) for v in (A, C, Q, R, X0))
    dx, dy = A.shape[0], C.shape[0]
    for nm, M in (("Q", Q), ("R", R)):
        if not np.allclose(M, M.T, atol=1e-8, rtol=1e-5):
            raise ValueError(f"Covariance matrix {nm} must be symmetric.")
        try:
            np.linalg.cholesky(M)
        except np.linalg.LinAlgError as e:
            raise ValueError(f"Covariance matrix {nm} must be positive-definite.") from e
    LQ, LR = np.linalg.cholesky(Q), np.linalg.cholesky(R)
    th = {}
    for i in range(dx):
        for j in range(dx):
            th[f"A{i+1}{j+1}"] = float(A[i, j])
    for i in range(dy):
        for j in range(dx):
            th[f"C{i+1}{j+1}"] = float(C[i, j])
    for i in range(dx):
        for j in range(i + 1):
            th[f"Q{i+1}{j+1}"] = float(LQ[i, j])
    for i in range(dy):
        for j in range(i + 1):
            th[f"R{i+1}{j+1}"] = float(LR[i, j])
    for i in range(dx):
        th[f"X0_{i+1}"] = float(X0[i])
    return th


def simulate_lg(theta: dict, dx: int, dy: int, T: int, seed: int):
    """Host simulation of LG data (x0 ~ N(X0, Q), x_t = A x + N(0,Q), y = C x + N(0,R))."""
    rng = np.random.default_rng(seed)
    A = np.array([[theta[f"A{i+1}{j+1}"] for j in range(dx)] for i in range(dx)])
    C = np.array([[theta[f"C{i+1}{j+1}"] for j in range(dx)] for i in range(dy)])
    LQ = np.zeros((dx, dx))
    LR = np.zeros((dy, dy))
    for i in range(dx):
        for j in range(i + 1):
            LQ[i, j] = theta[f"Q{i+1}{j+1}"]
    for i in range(dy):
        for j in range(i + 1):
            LR[i, j] = theta[f"R{i+1}{j+1}"]
    x = np.array([theta[f"X0_{i+1}"] for i in range(dx)]) + LQ @ rng.standard_normal(dx)
    Y = np.zeros((T, dy))
    for t in range(T):
        x = A @ x + LQ @ rng.standard_normal(dx)
        Y[t] = C @ x + LR @ rng.standard_normal(dy)
    return Y


def LG(T: int = 4, A=None, C=None, Q=None, R=None, X0=None, key=None, ys=None) -> Pomp:
    """Linear Gaussian model (``pypomp/models/linear_gaussian.py:337-451``).

    Dimensions are inferred from the arrays given, as in the reference, and are
    limited to 4 (the CUDA device code's register budget).  ``ys`` may be given
    to use existing data; otherwise data are simulated with seed ``key``.
    """
    dims = set()
    if A is not None:
        dims.add(np.asarray(A).shape[0])
    if Q is not None:
        dims.add(np.asarray(Q).shape[0])
    if X0 is not None:
        dims.add(np.asarray(X0).shape[0])
    if C is not None:
        dims.add(np.asarray(C).shape[1])
    if len(dims) > 1:
        raise ValueError(f"Inconsistent state dimension: {sorted(dims)}.")
    dyc = set()
    if C is not None:
        dyc.add(np.asarray(C).shape[0])
    if R is not None:
        dyc.add(np.asarray(R).shape[0])
    if len(dyc) > 1:
        raise ValueError(f"Inconsistent observation dimension: {sorted(dyc)}.")
    dx = dims.pop() if dims else (dyc.copy().pop() if dyc else 2)
    dy = dyc.pop() if dyc else dx
    for kind, d in (("state", dx), ("observation", dy)):
        if d < 1:
            raise ValueError(f"The {kind} dimension must be at least 1, but is {d}.")
        if d > MAX_DIM:
            raise ValueError(
                f"LG supports dimensions up to {MAX_DIM}, but the {kind} dimension is "
                f"{d}. Above {MAX_DIM} the 'A11' style parameter names are ambiguous.")
    A_ = _default_A(dx) if A is None else np.asarray(A, float)
    C_ = np.eye(dy, dx) if C is None else np.asarray(C, float)
    Q_ = _default_cov(dx, 1.0, 0.02) / 100 if Q is None else np.asarray(Q, float)
    R_ = _default_cov(dy, 1.0, 0.1) / 10 if R is None else np.asarray(R, float)
    X0_ = np.zeros(dx) if X0 is None else np.asarray(X0, float)
    theta = lg_theta(A_, C_, Q_, R_, X0_)
    spec = lg_spec(dx, dy)
    if ys is None:
        seed = 1 if key is None else int(np.asarray(key, dtype=np.uint64) % (1 << 63))
        Y = simulate_lg(theta, dx, dy, T, seed)
        ys = pd.DataFrame(Y, index=np.arange(1, T + 1, dtype=float), columns=list(spec.obsnames))
    return Pomp(spec=spec, ys=ys, theta=theta, t0=0.0)


# ---------------------------------------------------------------------------
# Heston-type stochastic volatility (log variance)
# ---------------------------------------------------------------------------

SV_DT = 1.0 / 252.0


def sv_spec(dt: float = SV_DT) -> ModelSpec:
    return ModelSpec(
        kind=_ffi.MODEL_SV, dx=2, dy=1,
        param_names=("kappa", "theta", "xi", "rho", "mu", "v0"),
        statenames=("v", "eps"), obsnames=("r",), dt=dt,
        est_log=(0, 1, 2), est_atanh=(3,), name="SV",
    )


def simulate_sv(theta: dict, T: int, seed: int, dt: float = SV_DT):
    rng = np.random.default_rng(seed)
    k, th, xi, rho, mu = (theta[n] for n in ("kappa", "theta", "xi", "rho", "mu"))
    v = theta["v0"]
    r = np.zeros((T, 1))
    for t in range(T):
        e = rng.standard_normal()
        v = v + k * (th - math.exp(v)) * math.exp(-v) * dt + xi * math.exp(-v / 2) * math.sqrt(dt) * e
        eta = rng.standard_normal()
        sd = math.sqrt(math.exp(v) * dt)
        r[t, 0] = mu * dt + sd * (rho * e + math.sqrt(1 - rho * rho) * eta)
    return r


def SV(T: int = 2000, kappa=2.0, theta=0.04, xi=0.3, rho=-0.7, mu=0.05, v0=None,
       key=0, ys=None, dt: float = SV_DT) -> Pomp:
    """Discretised Heston-type stochastic-volatility model on log variance.

    ``v_t = v + kappa (theta - e^v) e^-v dt + xi e^{-v/2} sqrt(dt) eps_t`` and
    daily log-returns ``r_t ~ N(mu dt, e^{v_t} dt)`` with correlation ``rho``
    between ``eps_t`` and the return noise.  The latent state carries
    ``(v, eps)`` so the measurement density can condition on ``eps_t``.
    ``v0`` defaults to ``log(theta)``.  Estimation scale: log kappa, log theta,
    log xi, atanh rho, mu, v0.
    """
    par = {"kappa": float(kappa), "theta": float(theta), "xi": float(xi), "rho": float(rho),
           "mu": float(mu), "v0": float(math.log(theta) if v0 is None else v0)}
    spec = sv_spec(dt)
    if ys is None:
        Y = simulate_sv(par, T, int(key), dt)
        ys = pd.DataFrame(Y, index=np.arange(1, T + 1, dtype=float), columns=["r"])
    return Pomp(spec=spec, ys=ys, theta=par, t0=0.0)


# ---------------------------------------------------------------------------
# Stochastic Ricker
# ---------------------------------------------------------------------------


def ricker_spec() -> ModelSpec:
    return ModelSpec(
        kind=_ffi.MODEL_RICKER, dx=1, dy=1, param_names=("r", "sigma", "phi", "N_0"),
        statenames=("N",), obsnames=("y",), est_log=(0, 1, 2, 3), name="Ricker",
    )


def simulate_ricker(theta: dict, T: int, seed: int):
    rng = np.random.default_rng(seed)
    N = theta["N_0"]
    y = np.zeros((T, 1))
    for t in range(T):
        N = theta["r"] * N * math.exp(-N + theta["sigma"] * rng.standard_normal())
        y[t, 0] = rng.poisson(theta["phi"] * N)
    return y


def Ricker(T: int = 500, r=math.exp(3.8), sigma=0.3, phi=10.0, N_0=7.0, key=0, ys=None) -> Pomp:
    """Stochastic Ricker model: ``N_t = r N_{t-1} exp(-N_{t-1} + sigma e_t)``,
    ``y_t ~ Poisson(phi N_t)``; estimation scale is the log of every parameter."""
    par = {"r": float(r), "sigma": float(sigma), "phi": float(phi), "N_0": float(N_0)}
    spec = ricker_spec()
    if ys is None:
        Y = simulate_ricker(par, T, int(key))
        ys = pd.DataFrame(Y, index=np.arange(1, T + 1, dtype=float), columns=["y"])
    return Pomp(spec=spec, ys=ys, theta=par, t0=0.0)
