"""Host-side configuration objects of the estimation loops.

Mirrors the reference's optimiser, learning-rate and random-walk classes that
sit around the hot path (the math here runs once per iteration on a
parameter vector; the particle work is in the CUDA library):

* ``SGD``, ``Adam``, ``FullMatrixAdam``, ``BFGS``, ``Newton``, ``WeightedNewton``
                         -- ``pypomp/core/optimizer.py:95-320`` (update rules,
                            bias correction, ``clip_norm`` / ``scale`` / ``ls``
                            options).  Steps take a batch of parameter vectors
                            (leading dimensions) and treat each row on its own,
                            as the reference's vmapped train does.
* ``LearningRate``       -- ``pypomp/core/learning_rate.py`` (per-parameter
                            rates, cosine / geometric / linear / hyperbolic decay)
* ``RWSigma``            -- ``pypomp/core/rw_sigma.py`` (IF2 random-walk sds,
                            initial-value parameters, cooling schedules,
                            ``cooling_factor`` at ``rw_sigma.py:193-224``)
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np


# ---------------------------------------------------------------------------
# Optimisers
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class Optimizer:
    clip_norm: float | None = None
    scale: bool = False
    ls: bool = False
    c: float = 0.1
    max_ls_itn: int = 10

    needs_hessian = False

    def init_state(self, theta: np.ndarray):
        raise NotImplementedError

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        raise NotImplementedError


@dataclass(frozen=True)
class SGD(Optimizer):
    def init_state(self, theta):
        return ()

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        return -np.asarray(grad, dtype=np.float64), ()

    def step_device(self, grad, state, step_num):
        """``step`` on float64 torch tensors (device-side training loop)."""
        return -grad, ()


@dataclass(frozen=True)
class Adam(Optimizer):
    beta1: float = 0.9
    beta2: float = 0.999
    epsilon: float = 1e-8

    def init_state(self, theta):
        z = np.zeros_like(np.asarray(theta, dtype=np.float64))
        return (z, z.copy())

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        m, v = state
        g = np.asarray(grad, dtype=np.float64)
        m_new = self.beta1 * m + (1 - self.beta1) * g
        v_new = self.beta2 * v + (1 - self.beta2) * (g ** 2)
        m_hat = m_new / (1 - self.beta1 ** (step_num + 1))
        v_hat = v_new / (1 - self.beta2 ** (step_num + 1))
        return -m_hat / (np.sqrt(v_hat) + self.epsilon), (m_new, v_new)

    def init_state_device(self, theta):
        return (theta.new_zeros(theta.shape), theta.new_zeros(theta.shape))

    def step_device(self, grad, state, step_num):
        """``step`` on float64 torch tensors, operation for operation (the
        same IEEE float64 results as the NumPy form)."""
        m, v = state
        m_new = self.beta1 * m + (1 - self.beta1) * grad
        v_new = self.beta2 * v + (1 - self.beta2) * (grad * grad)
        # divisors as device tensors: torch turns division by a host scalar
        # into multiplication by its reciprocal, which can differ in the last bit
        m_hat = m_new / grad.new_full((), 1 - self.beta1 ** (step_num + 1))
        v_hat = v_new / grad.new_full((), 1 - self.beta2 ** (step_num + 1))
        return -m_hat / (v_hat.sqrt() + self.epsilon), (m_new, v_new)


def _rows(a):
    a = np.asarray(a, dtype=np.float64)
    return a.reshape(-1, a.shape[-1])


def _pinv_sym(h):
    """Pseudo-inverse of a symmetric matrix (``jnp.linalg.pinv(..., hermitian=True)``)."""
    w, V = np.linalg.eigh(h)
    cut = np.finfo(np.float64).eps * h.shape[-1] * (np.max(np.abs(w)) if w.size else 0.0)
    inv = np.where(np.abs(w) > cut, 1.0 / np.where(np.abs(w) > cut, w, 1.0), 0.0)
    return (V * inv) @ V.T


@dataclass(frozen=True)
class FullMatrixAdam(Optimizer):
    """Adam with a full second-moment matrix (``optimizer.py:157-213``):
    direction = -F_hat^{-1/2} m_hat, F_hat from the outer products of the
    gradients, the inverse root through an eigendecomposition."""

    beta1: float = 0.9
    beta2: float = 0.999
    epsilon: float = 1e-4

    def init_state(self, theta):
        t = np.asarray(theta, dtype=np.float64)
        return np.zeros_like(t), np.zeros(t.shape + (t.shape[-1],))

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        m, v = state
        g = np.asarray(grad, dtype=np.float64)
        shape, P = g.shape, g.shape[-1]
        m_new = self.beta1 * m + (1 - self.beta1) * g
        m_hat = m_new / (1 - self.beta1 ** (step_num + 1))
        v_new = self.beta2 * v + (1 - self.beta2) * (g[..., :, None] * g[..., None, :])
        F_hat = v_new / (1 - self.beta2 ** (step_num + 1))
        out = np.empty((int(np.prod(shape[:-1], dtype=int)), P))
        for i, (Fh, mh) in enumerate(zip(F_hat.reshape(-1, P, P), _rows(m_hat))):
            w, V = np.linalg.eigh(Fh)
            out[i] = -(V @ np.diag(1.0 / np.sqrt(np.maximum(w, 0.0) + self.epsilon)) @ V.T) @ mh
        return out.reshape(shape), (m_new, v_new)


@dataclass(frozen=True)
class BFGS(Optimizer):
    """Quasi-Newton BFGS (``optimizer.py:216-267``), with the reference's
    choices: from the third step on, s_k = mean(eta) * (-previous gradient),
    y_k = grad - previous gradient, the inverse-Hessian update kept only when
    1 / (y_k . s_k) is finite; earlier steps go along -grad."""

    def init_state(self, theta):
        t = np.asarray(theta, dtype=np.float64)
        eye = np.broadcast_to(np.eye(t.shape[-1]), t.shape + (t.shape[-1],)).copy()
        return eye, np.zeros_like(t)

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        if eta_i is None:
            raise ValueError("BFGS optimizer requires eta_i")
        hess, prev_grad = state
        g = np.asarray(grad, dtype=np.float64)
        shape, P = g.shape, g.shape[-1]
        if step_num <= 1:
            return -g, (hess, g)
        eta_bar = float(np.mean(eta_i))
        H = hess.reshape(-1, P, P).copy()
        out = np.empty((H.shape[0], P))
        for i, (gi, pg) in enumerate(zip(_rows(g), _rows(prev_grad))):
            s_k = eta_bar * (-pg)
            y_k = gi - pg
            with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                rho = 1.0 / np.dot(y_k, s_k)
                Hy = H[i] @ y_k
                new = (H[i] - rho * np.outer(s_k, Hy) - rho * np.outer(Hy, s_k)
                       + rho * (rho * np.dot(y_k, Hy) + 1.0) * np.outer(s_k, s_k))
            if np.isfinite(rho):
                H[i] = new
            out[i] = -H[i] @ gi
        return out.reshape(shape), (H.reshape(hess.shape), g)


@dataclass(frozen=True)
class Newton(Optimizer):
    """Newton-Raphson (``optimizer.py:270-289``): direction = -pinv(H) grad."""

    needs_hessian = True

    def init_state(self, theta):
        return ()

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        if compute_hessian_fn is None:
            raise ValueError("Newton optimizer requires compute_hessian_fn")
        g = np.asarray(grad, dtype=np.float64)
        P = g.shape[-1]
        H = np.asarray(compute_hessian_fn(), dtype=np.float64).reshape(-1, P, P)
        out = np.stack([-_pinv_sym(h) @ gi for h, gi in zip(H, _rows(g))])
        return out.reshape(g.shape), ()


@dataclass(frozen=True)
class WeightedNewton(Optimizer):
    """Newton on a decaying mixture of the previous and current Hessians
    (``optimizer.py:292-320``): weight i^log(i) / (i+1)^log(i+1) on the
    previous one from the second step on."""

    needs_hessian = True

    def init_state(self, theta):
        t = np.asarray(theta, dtype=np.float64)
        return (np.broadcast_to(np.eye(t.shape[-1]), t.shape + (t.shape[-1],)).copy(),)

    def step(self, grad, state, step_num, compute_hessian_fn=None, eta_i=None):
        if compute_hessian_fn is None:
            raise ValueError("WeightedNewton optimizer requires compute_hessian_fn")
        (prev,) = state
        g = np.asarray(grad, dtype=np.float64)
        P = g.shape[-1]
        H = np.asarray(compute_hessian_fn(), dtype=np.float64).reshape(-1, P, P)
        if step_num == 0:
            use = H
        else:
            i = float(step_num)
            wt = (i ** math.log(i)) / ((i + 1.0) ** math.log(i + 1.0))
            use = wt * prev.reshape(-1, P, P) + (1.0 - wt) * H
        out = np.stack([-_pinv_sym(h) @ gi for h, gi in zip(use, _rows(g))])
        return out.reshape(g.shape), (H.reshape(prev.shape),)


# ---------------------------------------------------------------------------
# Learning rates
# ---------------------------------------------------------------------------


class LearningRate:
    """Per-parameter learning rates, constant or as an (M,) schedule."""

    def __init__(self, rates: dict):
        if not isinstance(rates, dict):
            raise ValueError("rates must be a dictionary")
        self._rates = {}
        for k, v in rates.items():
            arr = np.asarray(v, dtype=np.float64)
            if np.any(arr < 0):
                raise ValueError("learning rates must be non-negative")
            self._rates[str(k)] = arr

    def to_array(self, param_names: Sequence[str], M: int) -> np.ndarray:
        """(M, P) schedule in ``param_names`` order (``learning_rate.py:113-167``);
        every requested name must have a rate, extra rates are ignored."""
        names = list(param_names)
        for n in names:
            if n not in self._rates:
                raise ValueError(f"Parameter '{n}' not found in learning rates")
        M_eff = max(int(M), 1)
        cols = []
        for n in names:
            a = self._rates[n]
            if a.ndim == 0:
                cols.append(np.full(M_eff, float(a)))
            else:
                if a.shape[0] != M:
                    raise ValueError(f"Learning rate schedule for '{n}' has length {a.shape[0]}, expected M={M}")
                cols.append(a)
        return np.stack(cols, axis=1)

    def _apply(self, factor: np.ndarray) -> "LearningRate":
        out = {}
        for k, a in self._rates.items():
            out[k] = (float(a) * factor) if a.ndim == 0 else a * factor
        return LearningRate(out)

    def cosine_decay(self, final_factor: float, M: int) -> "LearningRate":
        if not 0 <= final_factor <= 1:
            raise ValueError("final_factor should be between 0 and 1")
        it = np.arange(M)
        return self._apply(final_factor + (1.0 - final_factor) * 0.5 * (1.0 + np.cos(np.pi * it / M)))

    def geometric_decay(self, decay_rate: float, M: int) -> "LearningRate":
        if not 0 <= decay_rate <= 1:
            raise ValueError("decay_rate should be between 0 and 1")
        return self._apply(decay_rate ** np.arange(M))

    def linear_decay(self, final_factor: float, M: int) -> "LearningRate":
        if not 0 <= final_factor <= 1:
            raise ValueError("final_factor should be between 0 and 1")
        return self._apply(np.linspace(1.0, final_factor, M))

    def hyperbolic_decay(self, decay_rate: float, M: int) -> "LearningRate":
        if decay_rate < 0:
            raise ValueError("decay_rate must be non-negative")
        return self._apply(1.0 / (1.0 + decay_rate * np.arange(M)))

    @property
    def rates(self):
        return dict(self._rates)


def cosine_alpha(m: int, M: int, c: float) -> float:
    """``_cosine_cooling`` (``pypomp/core/algorithms/helpers.py:302-314``)."""
    return c + (1.0 - c) * 0.5 * (1.0 + math.cos(math.pi * m / M))


# ---------------------------------------------------------------------------
# IF2 random-walk standard deviations
# ---------------------------------------------------------------------------


class RWSigma:
    """Random-walk sds for IF2 perturbations with a cooling schedule.

    ``sigmas`` maps parameter names to sds (estimation scale); ``init_names``
    are perturbed only at t0 with their sd (``mif.py:113-120``), the rest at
    every observation (``mif.py:178-181``).  Default cooling: geometric 0.5.
    """

    def __init__(self, sigmas: dict, init_names: Sequence[str] = (), cooling_fn: Callable | None = None):
        if not isinstance(sigmas, dict):
            raise ValueError("sigmas must be a dictionary")
        if not isinstance(init_names, (list, tuple)):
            raise ValueError("init_names must be a list or tuple")
        clean = {}
        for name, value in sigmas.items():
            if not isinstance(name, str):
                raise ValueError("All keys in sigmas must be strings")
            if isinstance(value, bool):
                raise ValueError(f"Value for '{name}' must be a float, got bool")
            v = float(value)
            if v < 0:
                raise ValueError("All values in sigmas dictionary must be non-negative")
            clean[name] = v
        if len(init_names) != len(set(init_names)):
            raise ValueError("Duplicate names found in init_names")
        if not all(n in clean for n in init_names):
            raise ValueError("All init_names names must be in sigmas dictionary")
        self.param_names = tuple(clean)
        self.init_names = tuple(init_names)
        self._sig = clean
        self.cooling_type = "geometric"
        self.a, self.s, self.c, self.M = 0.5, None, None, None
        self._custom = None
        if cooling_fn is not None:
            self.cooling_type = "custom"
            self._custom = cooling_fn

    def _copy(self):
        o = RWSigma(dict(self._sig), list(self.init_names))
        o.cooling_type, o.a, o.s, o.c, o.M, o._custom = (self.cooling_type, self.a, self.s, self.c,
                                                         self.M, self._custom)
        return o

    def geometric_cooling(self, a: float) -> "RWSigma":
        if not 0 <= a <= 1:
            raise ValueError("a should be between 0 and 1")
        o = self._copy()
        o.cooling_type, o.a = "geometric", float(a)
        return o

    def cosine_cooling(self, c: float, M: int) -> "RWSigma":
        if not 0 <= c <= 1:
            raise ValueError("c should be between 0 and 1")
        if M <= 0:
            raise ValueError("M must be positive")
        o = self._copy()
        o.cooling_type, o.c, o.M = "cosine", float(c), int(M)
        return o

    def hyperbolic_cooling(self, s: float) -> "RWSigma":
        if s < 0:
            raise ValueError("s must be non-negative")
        o = self._copy()
        o.cooling_type, o.s = "hyperbolic", float(s)
        return o

    def cooling_factor(self, nt, m, ntimes) -> float:
        """``rw_sigma.py:193-224``: factor at time index nt of iteration m."""
        frac = nt / ntimes + m
        if self.cooling_type == "geometric":
            return (self.a ** (1.0 / 50.0)) ** frac
        if self.cooling_type == "cosine":
            return self.c + (1.0 - self.c) * 0.5 * (1.0 + math.cos(math.pi * frac / self.M))
        if self.cooling_type == "hyperbolic":
            return 1.0 / (1.0 + self.s * frac)
        if self.cooling_type == "custom":
            return float(self._custom(nt, m, ntimes))
        return 1.0

    def cooling_factors(self, ntimes: int, m: int) -> list:
        """``cooling_factor(nt, m, ntimes)`` for nt = 0 .. ntimes-1, the same
        float64 arithmetic with the loop-invariant parts taken out."""
        if self.cooling_type == "geometric":
            base = self.a ** (1.0 / 50.0)
            return [base ** (nt / ntimes + m) for nt in range(ntimes)]
        return [self.cooling_factor(nt, m, ntimes) for nt in range(ntimes)]

    def arrays(self, canonical_names: Sequence[str]):
        """(sigmas for per-step perturbation, sigmas for t0 only) in canonical order."""
        names = list(canonical_names)
        if set(names) != set(self.param_names):
            raise ValueError(
                "RWSigma parameter names must match canonical_param_names up to reordering. "
                f"Got {sorted(self.param_names)}, expected {sorted(names)}.")
        sig = np.array([self._sig[n] for n in names], dtype=np.float64)
        init = np.array([1.0 if n in self.init_names else 0.0 for n in names])
        return sig * (1.0 - init), sig * init

    @property
    def sigmas(self):
        return dict(self._sig)
