"""Random-walk proposals for PMCMC (``pypomp/proposals.py``).

The same three proposals as the reference, with its constructors, validation
and update rules, on NumPy float64:

* :class:`MVNDiagRW` -- diagonal normal random walk (``proposals.py:67-143``);
* :class:`MVNRWFull` -- full-covariance normal random walk (``:146-233``);
* :class:`MVNRWAdaptive` -- the two-phase adaptive walk of Roberts & Rosenthal
  (2009) (``:264-516``): scale adaptation towards a target acceptance rate,
  then the scaled empirical covariance (2.38^2 / d) Cov once enough proposals
  were accepted; Welford updates of the running mean and covariance.

``step(state, theta, key, n, accepts)`` returns the proposed parameter vector
(estimation scale) and the new state.  Normals come from a NumPy generator
seeded with the 64-bit step key, so a chain is reproducible from its key.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np


def _normals(key, d: int) -> np.ndarray:
    return np.random.default_rng(int(np.asarray(key, dtype=np.uint64))).standard_normal(d)


class MVNDiagRW:
    """Diagonal multivariate normal random walk; entries with ``sd <= 0`` are dropped."""

    def __init__(self, rw_sd: dict):
        rw_sd = {k: float(v) for k, v in rw_sd.items() if v > 0}
        if not rw_sd:
            raise ValueError("rw_sd must contain at least one positive entry.")
        self.param_names = tuple(rw_sd)
        self.sd_arr = np.asarray([rw_sd[p] for p in self.param_names])

    def __eq__(self, other):
        if not isinstance(other, MVNDiagRW):
            return NotImplemented
        return self.param_names == other.param_names and np.array_equal(self.sd_arr, other.sd_arr)

    def init_state(self, theta_arr):
        return ()

    def step(self, state, theta_arr, key, n, accepts):
        return np.asarray(theta_arr, float) + _normals(key, len(theta_arr)) * self.sd_arr, state

    def canonicalize(self, canonical_names: Sequence[str]) -> "MVNDiagRW":
        names = tuple(canonical_names)
        idx = {p: i for i, p in enumerate(names)}
        sd = np.zeros(len(names))
        for p, v in zip(self.param_names, self.sd_arr):
            if p not in idx:
                raise ValueError(f"Proposal parameter {p!r} not in model.")
            sd[idx[p]] = v
        out = object.__new__(MVNDiagRW)
        out.param_names, out.sd_arr = names, sd
        return out


def _expand(mat: np.ndarray, local: Sequence[str], names: Sequence[str]) -> np.ndarray:
    idx = {p: i for i, p in enumerate(names)}
    full = np.zeros((len(names), len(names)))
    for a, pa in enumerate(local):
        if pa not in idx:
            raise ValueError(f"Proposal parameter {pa!r} not in model.")
        for b, pb in enumerate(local):
            full[idx[pa], idx[pb]] = mat[a, b]
    return full


class MVNRWFull:
    """Full-covariance multivariate normal random walk from a covariance matrix."""

    def __init__(self, rw_var, param_names):
        rw_var = np.asarray(rw_var, dtype=float)
        if rw_var.ndim != 2 or rw_var.shape[0] != rw_var.shape[1]:
            raise ValueError("rw_var must be a square matrix.")
        if rw_var.shape[0] != len(param_names):
            raise ValueError("rw_var dimensions must match len(param_names).")
        self.chol = np.linalg.cholesky(rw_var)
        self.param_names = tuple(param_names)

    def __eq__(self, other):
        if not isinstance(other, MVNRWFull):
            return NotImplemented
        return self.param_names == other.param_names and np.array_equal(self.chol, other.chol)

    def init_state(self, theta_arr):
        return ()

    def step(self, state, theta_arr, key, n, accepts):
        return np.asarray(theta_arr, float) + self.chol @ _normals(key, len(theta_arr)), state

    def canonicalize(self, canonical_names: Sequence[str]) -> "MVNRWFull":
        out = object.__new__(MVNRWFull)
        out.param_names = tuple(canonical_names)
        out.chol = _expand(self.chol, self.param_names, out.param_names)
        return out


@dataclass(frozen=True)
class AdaptiveState:
    """State carried by :class:`MVNRWAdaptive` from step to step."""

    scaling: float
    theta_mean: np.ndarray
    covmat_emp: np.ndarray
    initialized: bool


class MVNRWAdaptive:
    """Adaptive multivariate normal random walk (Roberts & Rosenthal 2009)."""

    def __init__(self, rw_sd: dict | None = None, rw_var=None, param_names=None, scale_start: int = 200,
                 scale_cooling: float = 0.999, shape_start: int = 200, target: float = 0.234,
                 max_scaling: float = 50.0):
        if (rw_sd is None) == (rw_var is None):
            raise ValueError("Exactly one of rw_sd and rw_var must be given.")
        if rw_sd is not None:
            rw_sd = {k: float(v) for k, v in rw_sd.items() if v > 0}
            names = tuple(rw_sd)
            init_var = np.diag([rw_sd[p] ** 2 for p in names])
        else:
            if param_names is None:
                raise ValueError("param_names required when rw_var is given.")
            init_var = np.asarray(rw_var, dtype=float)
            if init_var.shape != (len(param_names), len(param_names)):
                raise ValueError("rw_var shape must match param_names.")
            names = tuple(param_names)
        if scale_start < 1:
            raise ValueError("scale_start must be a positive integer.")
        if not (0 < scale_cooling <= 1):
            raise ValueError("scale_cooling must be in (0, 1].")
        if shape_start < 1:
            raise ValueError("shape_start must be a positive integer.")
        if not (0 < target < 1):
            raise ValueError("target must be in (0, 1).")
        self.init_rw_var = np.asarray(init_var)
        self.param_names = names
        self.scale_start, self.scale_cooling = int(scale_start), float(scale_cooling)
        self.shape_start, self.target, self.max_scaling = int(shape_start), float(target), float(max_scaling)

    def __eq__(self, other):
        if not isinstance(other, MVNRWAdaptive):
            return NotImplemented
        return (self.param_names == other.param_names and self.scale_start == other.scale_start
                and self.scale_cooling == other.scale_cooling and self.shape_start == other.shape_start
                and self.target == other.target and self.max_scaling == other.max_scaling
                and np.array_equal(self.init_rw_var, other.init_rw_var))

    def init_state(self, theta_arr) -> AdaptiveState:
        d = len(theta_arr)
        return AdaptiveState(1.0, np.zeros(d), np.zeros((d, d)), False)

    def step(self, state: AdaptiveState, theta_arr, key, n, accepts):
        th = np.asarray(theta_arr, float)
        d = th.shape[0]
        nf = max(float(n), 1.0)
        mean0 = state.theta_mean if state.initialized else th
        # phase 1: scale towards the target acceptance rate
        cool = self.scale_cooling ** max(float(n) - self.scale_start, 0.0)
        scaling_p1 = min(state.scaling * np.exp(cool * (float(accepts) / nf - self.target)), self.max_scaling)
        in_p1 = (n >= self.scale_start) and (accepts < self.shape_start)
        scaling = scaling_p1 if in_p1 else state.scaling
        # covariance of this proposal
        if accepts >= self.shape_start:
            cov = (2.38 ** 2 / d) * state.covmat_emp
        elif in_p1:
            cov = scaling ** 2 * self.init_rw_var
        else:
            cov = self.init_rw_var
        # Welford updates of the running mean and covariance
        mean1 = mean0 + (th - mean0) / nf
        cov_emp = ((nf - 1.0) * state.covmat_emp + np.outer(th - mean0, th - mean1)) / nf
        active = (np.any(self.init_rw_var != 0, axis=0) | np.any(self.init_rw_var != 0, axis=1)).astype(float)
        try:
            chol = np.linalg.cholesky(cov + 1e-10 * np.eye(d))
        except np.linalg.LinAlgError:       # not positive definite: a NaN proposal, rejected
            chol = np.full((d, d), np.nan)
        prop = th + (chol @ _normals(key, d)) * active
        return prop, AdaptiveState(scaling, mean1, cov_emp, True)

    def canonicalize(self, canonical_names: Sequence[str]) -> "MVNRWAdaptive":
        out = object.__new__(MVNRWAdaptive)
        out.__dict__.update(self.__dict__)
        out.param_names = tuple(canonical_names)
        out.init_rw_var = _expand(self.init_rw_var, self.param_names, out.param_names)
        return out
