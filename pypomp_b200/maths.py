"""Averages of replicate log-likelihoods on the likelihood scale.

pypomp reports a parameter set's log-likelihood as the log of the mean of the
replicate likelihoods, with a jackknife standard error
(``pypomp/maths.py:24-157``).  Both are written here from their definitions:

* ``logmeanexp(x) = log((1/n) sum_i exp(x_i))``, evaluated as
  ``c + log((1/n) sum_i exp(x_i - c))`` with ``c = max_i x_i`` so that no
  exponential overflows;
* the jackknife SE: with ``L_(i)`` the log-mean-exp of the sample without
  entry i, ``se = sqrt(n - 1) * sd(L_(1), ..., L_(n))`` (sd with divisor n).

Conventions kept from the reference: NaN entries make the result NaN unless
``ignore_nan`` drops them; an empty sample gives NaN (with a warning when no
axis is given); a sample of fewer than two values has no standard error (NaN).
"""

from __future__ import annotations

import warnings

import numpy as np


def _shift(a: np.ndarray, keep: np.ndarray, axis):
    """Largest kept entry along ``axis`` (keepdims); NaN where nothing is kept."""
    masked = np.where(keep, a, -np.inf)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        c = np.max(masked, axis=axis, keepdims=True)
    none_kept = ~np.any(keep, axis=axis, keepdims=True)
    return np.where(none_kept, np.nan, c)


def logmeanexp(x, axis=None, ignore_nan: bool = False):
    """``log(mean(exp(x)))`` over ``axis`` (all entries when None), without
    overflow.  A float for ``axis=None``, else an array with ``axis`` removed.
    With ``ignore_nan`` the mean runs over the non-NaN entries only."""
    a = np.asarray(x, dtype=float)
    if a.size == 0 and axis is None and not ignore_nan:
        warnings.warn("x is an empty array, returning nan", stacklevel=2)
        return np.nan
    keep = ~np.isnan(a) if ignore_nan else np.ones(a.shape, dtype=bool)
    c = _shift(a, keep, axis) if ignore_nan else np.max(a, axis=axis, keepdims=True)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        terms = np.where(keep, np.exp(a - c), 0.0)
        total = np.sum(terms, axis=axis, keepdims=True)
        count = np.sum(keep, axis=axis, keepdims=True)
        out = c + np.log(total / count)
    return out.item() if axis is None else np.squeeze(out, axis=axis)


def _jackknife_se(v: np.ndarray) -> float:
    """Jackknife SE of the log-mean-exp of the 1-D sample ``v``."""
    n = v.size
    if n < 2:
        return np.nan
    order = np.argsort(v)
    top = v[order[-1]]
    if not np.isfinite(top):   # NaN, or an infinite maximum: no finite estimate
        return np.nan
    # Leaving out any entry but a unique maximum keeps the maximum as the shift:
    # the sum of the others is the full sum less the entry's own term.  Leaving
    # out a unique maximum shifts by the runner-up instead and sums the others
    # directly, so a dominant maximum cannot cancel its own sum to zero.
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        e = np.exp(v - top)
        full = np.sum(e)
        loo = top + np.log((full - e) / (n - 1))
        second = v[order[-2]]
        if second < top:
            i = order[-1]
            rest = np.delete(v, i)
            loo[i] = second + np.log(np.sum(np.exp(rest - second)) / (n - 1)) if np.isfinite(second) \
                else -np.inf
    return float(np.sqrt(n - 1) * np.std(loo))


def logmeanexp_se(x, axis=None, ignore_nan: bool = False):
    """Jackknife standard error of :func:`logmeanexp` over ``axis`` (all
    entries when None).  NaN for fewer than two values; with ``ignore_nan``
    NaN entries are dropped first."""
    a = np.asarray(x, dtype=float)
    if axis is None:
        v = a.ravel()
        return _jackknife_se(v[~np.isnan(v)] if ignore_nan else v)
    rows = np.moveaxis(a, axis, -1)
    flat = rows.reshape(-1, rows.shape[-1])
    out = np.empty(flat.shape[0])
    for r, v in enumerate(flat):
        out[r] = _jackknife_se(v[~np.isnan(v)] if ignore_nan else v)
    return out.reshape(rows.shape[:-1])
