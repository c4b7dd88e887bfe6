"""Host reductions over replicate log-likelihoods (``pypomp/maths.py:24-157``)."""

from __future__ import annotations

import warnings

import numpy as np


def logmeanexp(x, axis=None, ignore_nan: bool = False):
    """``log(mean(exp(x)))`` computed stably (``pypomp/maths.py:24-83``)."""
    x_array = np.asarray(x, dtype=float)
    if ignore_nan:
        with warnings.catch_warnings():
            warnings.filterwarnings("ignore", message="All-NaN slice encountered")
            x_max = np.nanmax(x_array, axis=axis, keepdims=True)
        mask = np.isnan(x_array)
        x_safe = np.where(mask, -np.inf, x_array)
        counts = np.sum(~mask, axis=axis, keepdims=True)
        with np.errstate(divide="ignore", invalid="ignore"):
            mean_exp = np.sum(np.exp(x_safe - x_max), axis=axis, keepdims=True) / counts
            res = np.log(mean_exp) + x_max
    else:
        if axis is None and x_array.size == 0:
            warnings.warn("x is an empty array, returning nan", stacklevel=2)
            return np.nan
        x_max = np.max(x_array, axis=axis, keepdims=True)
        with np.errstate(divide="ignore", invalid="ignore"):
            res = np.log(np.mean(np.exp(x_array - x_max), axis=axis, keepdims=True)) + x_max
    if axis is None:
        return res.item()
    return np.squeeze(res, axis=axis)


def logmeanexp_se(x, axis=None, ignore_nan: bool = False):
    """Jackknife standard error of :func:`logmeanexp` (``pypomp/maths.py:95-157``)."""
    if axis is not None:
        return np.apply_along_axis(logmeanexp_se, axis, x, ignore_nan=ignore_nan)
    x_array = np.asarray(x, dtype=float)
    if ignore_nan:
        x_array = x_array[~np.isnan(x_array)]
    n = x_array.size
    if n <= 1:
        return np.nan
    x_max = np.max(x_array)
    s = np.exp(x_array - x_max)
    S = np.sum(s)
    with np.errstate(divide="ignore", invalid="ignore"):
        jack = np.log((S - s) / (n - 1)) + x_max
    is_max = x_array == x_max
    if np.sum(is_max) == 1:
        idx_max = int(np.argmax(x_array))
        if S - s[idx_max] <= 0:
            jack[idx_max] = logmeanexp(np.delete(x_array, idx_max))
    return float(np.sqrt(n - 1) * np.std(jack, ddof=0))
