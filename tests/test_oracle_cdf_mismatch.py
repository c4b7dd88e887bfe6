"""How often the exact fixed-point resampling CDF and the reference's float32
running-sum CDF choose different ancestors (CPU).

The reference resamples with ``cumsum`` of the float32 normalised weights
divided by its last entry, then ``searchsorted((U + k) / J, side="right")``
(``pypomp/core/algorithms/helpers.py:14-31``; restated in
``oracle/refpath.py``).  This library uses the exact fixed-point CDF of
``include/ppf.h`` (restated in ``oracle/ppf_oracle.c``).  The float32 running
sum carries a rounding error that grows with J and reaches the spacing of the
systematic points (1/J) at a few thousand particles, so the two definitions
move some children to a neighbouring parent.

Two figures per J, printed and bounded:
* the per-step rate: the same log-weights (the C oracle's first step) through
  both definitions, fraction of the J children whose parent differs;
* the whole-run divergence: the C oracle and the float32 restatement fed the
  same injected draws for T = 4 steps (once one child differs, its subtree
  differs, so this fraction grows with t), and the log-likelihood difference,
  which stays within Monte Carlo error.
"""

import numpy as np
import pytest

from oracle import cora, refpath

f32 = np.float32


def _exact_parents(w: np.ndarray, u: float) -> np.ndarray:
    """The fixed-point systematic parents of include/ppf.h, in exact integers."""
    J = w.size
    M = float(np.max(w))
    q = [int(np.rint(np.float64(cora.expf(f32(x - f32(M)))) * 2.0 ** 40)) for x in w]
    C = np.cumsum(np.array(q, dtype=object))
    tot = int(C[-1])
    u32 = int(np.float64(u) * 2.0 ** 32)
    chi = (u32 * tot) >> 32
    # parent(k) = #{ j : C_j J <= k tot + chi }
    CJ = [int(c) * J for c in C]
    out = np.empty(J, np.int64)
    j = 0
    for k in range(J):
        lim = k * tot + chi
        while j < J and CJ[j] <= lim:
            j += 1
        out[k] = j
    return out


def _lg1d(T, seed):
    rng = np.random.default_rng(seed)
    x, ys = 0.0, []
    for _ in range(T):
        x = 0.9 * x + np.sqrt(0.1) * rng.standard_normal()
        ys.append([x + np.sqrt(0.1) * rng.standard_normal()])
    theta = np.array([0.9, 1.0, np.sqrt(0.1), np.sqrt(0.1), 0.0], f32)   # A, C, L_Q, L_R, X0
    return theta, np.asarray(ys, f32)


@pytest.mark.parametrize("J, per_step_max, logdiff_max", [(1000, 0.002, 0.05), (4096, 0.01, 0.05),
                                                          (65536, 0.2, 0.05)])
def test_exact_vs_float32_cdf(J, per_step_max, logdiff_max, capsys):
    T = 4
    theta, ys = _lg1d(T, 7)
    rng = np.random.default_rng(1234)
    z0 = rng.standard_normal((1, J, 1)).astype(f32)
    z = rng.standard_normal((1, T, J, 1)).astype(f32)
    u = rng.random((1, T)).astype(f32)
    exact = cora.pfilter(1, 1, 1, theta[None], ys, J, inject={"z0": z0, "z": z, "u": u},
                         anc=True, logw=True)
    # per step: the C oracle's first-step log-weights through both CDFs
    w0 = exact["logw"][0, 0]
    mine = _exact_parents(w0, float(u[0, 0]))
    assert np.array_equal(mine, exact["anc"][0, 0]), "numpy restatement of the exact CDF"
    theirs = refpath.resample(refpath.normalize(w0)[0], u[0, 0])
    per_step = float(np.mean(mine != theirs))
    shift = np.abs(mine - theirs)
    # whole run: same draws through the float32 restatement
    ref = refpath.pfilter("LG", theta, ys, J, refpath.ArrayNoise(z0[0], z[0], u[0]), diagnostics=True)
    whole = float(np.mean(exact["anc"][0] != ref["ancestors"]))
    dl = abs(float(exact["loglik"][0]) - float(ref["logLik"]))
    with capsys.disabled():
        print(f"\n  J={J}: per-step parent mismatch {per_step:.4%} (max shift {int(shift.max())}); "
              f"whole run (T={T}) {whole:.2%} of ancestors differ; "
              f"logLik {float(exact['loglik'][0]):.5f} vs {float(ref['logLik']):.5f}")
    assert shift.max() <= 1 + J // 4096        # neighbouring parents only
    assert per_step <= per_step_max
    assert dl <= logdiff_max
