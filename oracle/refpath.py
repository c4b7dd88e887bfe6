"""Float32 NumPy restatement of the reference's particle-filter hot path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

This module follows the reference's algorithms operation by operation, in
float32 like the reference's JAX defaults, vectorised over particles:

* ``pfilter``      -- ``pypomp/core/algorithms/pfilter.py:15-182``
* ``normalize``    -- ``pypomp/core/algorithms/helpers.py:34-57``
* ``resample``     -- ``pypomp/core/algorithms/helpers.py:14-31`` (float32
  cumsum, ``searchsorted(..., side="right")``)
* ``mop``          -- ``pypomp/core/algorithms/mop.py:19-135``
* ``perfilter``    -- ``pypomp/core/algorithms/mif.py:88-258``
* ``mif``          -- ``pypomp/core/algorithms/mif.py:16-85``
* ``simulate``     -- ``pypomp/core/algorithms/simulate.py:15-142``

Random numbers come from a *noise source*.  ``JaxKeyNoise`` replays the
reference's own key tree (``pfilter.py:23-25,105,160``;
``model_mechanics.py:904`` per-sub-step split and ``:586`` per-particle split;
``mif.py:113-120,179``) through ``oracle/jaxrng.py``, which is what lets the
oracle reproduce the reference's regression fixtures.  ``ArrayNoise`` reads
injected arrays: it is how the same draws are fed to the CUDA kernels'
noise-injection mode.  ``RecordingNoise`` wraps a source and records every draw
into injection arrays.

The resampling CDF here is the reference's float32 running sum.  The CUDA path
uses an exact fixed-point CDF instead (defined in ``include/ppf.h``); the C
oracle (``oracle/ppf_oracle.c``) restates that definition for bit-exact
comparisons.  ``tests/test_oracle_cdf_mismatch.py`` measures how often the two
pick different ancestors on the same weights (none of 1000, about 0.1 % of
4096 and 10 % of 65536 children on its LG case, always a neighbouring parent)
and how far whole runs then diverge.
"""

from __future__ import annotations

import numpy as np

from . import jaxrng as jr
from .models_np import MODELS

f32 = np.float32


# ---------------------------------------------------------------------------
# Noise sources
# ---------------------------------------------------------------------------


class JaxKeyNoise:
    """The reference pfilter/mop key tree, replayed with ``oracle.jaxrng``."""

    def __init__(self, key: jr.Key, J: int, n_init: int, n_step: int):
        # pfilter.py:23-25 / mop.py:30-32: split(key, J+1) -> carry key, J rinit keys
        sk = jr.split(key, J + 1)
        self.key = sk[0]
        self.init_keys = sk[1:]
        self.J = J
        self.n_init = n_init
        self.n_step = n_step

    def init_normals(self):
        J = self.J
        if self.n_init == 0:
            return np.zeros((J, 0), f32)
        return np.stack([jr.normal(self.init_keys[j], (self.n_init,)) for j in range(J)])

    def step_normals(self, t):
        # pfilter.py:105 then model_mechanics.py:904 (one sub-step) and :586
        s = jr.split(self.key)
        self.key, sub = s[0], s[1]
        s2 = jr.split(sub)
        sub2 = s2[1]
        pk = jr.split(sub2, self.J)
        if self.n_step == 0:
            return np.zeros((self.J, 0), f32)
        return np.stack([jr.normal(pk[j], (self.n_step,)) for j in range(self.J)])

    def resample_uniform(self, t):
        # pfilter.py:160 (and mop.py:123) then helpers.py:28
        s = jr.split(self.key)
        self.key, sub = s[0], s[1]
        return f32(jr.uniform(sub))


class ArrayNoise:
    """Injected draws: ``z0`` (J,n_init), ``z`` (T,J,n_step), ``u`` (T,)."""

    def __init__(self, z0, z, u):
        self.z0 = np.asarray(z0, f32)
        self.z = np.asarray(z, f32)
        self.u = np.asarray(u, f32)

    def init_normals(self):
        return self.z0

    def step_normals(self, t):
        return self.z[t]

    def resample_uniform(self, t):
        return f32(self.u[t])


class RecordingNoise:
    """Wraps a source and records its draws as injection arrays."""

    def __init__(self, src):
        self.src = src
        self.z0 = None
        self.z = []
        self.u = []

    def init_normals(self):
        self.z0 = self.src.init_normals()
        return self.z0

    def step_normals(self, t):
        z = self.src.step_normals(t)
        self.z.append(z)
        return z

    def resample_uniform(self, t):
        u = self.src.resample_uniform(t)
        self.u.append(u)
        return u

    def arrays(self):
        return (self.z0, np.stack(self.z), np.asarray(self.u, f32))


# ---------------------------------------------------------------------------
# Weight helpers (helpers.py)
# ---------------------------------------------------------------------------


def normalize(w: np.ndarray):
    """``_normalize_weights`` (helpers.py:34-57)."""
    w = w.astype(f32)
    mw = np.max(w)
    collapsed = mw == -np.inf
    mw_safe = f32(0.0) if collapsed else mw
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        lt = f32(mw_safe + np.log(np.nansum(np.exp(w - mw_safe), dtype=f32)))
    if collapsed:
        lt = f32(-np.inf)
        nw = np.full(w.shape, -np.log(f32(w.shape[-1])), f32)
    else:
        nw = (w - lt).astype(f32)
    return nw, lt


def resample(nw: np.ndarray, u: np.float32):
    """``_resample`` (helpers.py:14-31): systematic, float32 CDF, side=right."""
    J = nw.shape[-1]
    unifs = ((u + np.arange(J, dtype=f32)) / f32(J)).astype(f32)
    csum = np.cumsum(np.exp(nw).astype(f32), dtype=f32)
    return np.searchsorted((csum / csum[-1]).astype(f32), unifs, side="right")


# ---------------------------------------------------------------------------
# pfilter
# ---------------------------------------------------------------------------


def pfilter(model, theta, ys, J, noise, thresh=0.0, diagnostics=False):
    """``_pfilter_internal`` + ``_pfilter_step`` (pfilter.py:15-182).

    ``model`` is a name in ``MODELS``; ``theta`` is on the natural scale.
    Returns a dict with ``logLik`` (float32 like the reference), and when
    ``diagnostics`` is set ``CLL``, ``ESS``, ``filter_mean``,
    ``prediction_mean`` and the per-step ``ancestors`` and ``log_weights``
    (unnormalised, before normalisation).
    """
    m = MODELS[model]
    ys = np.asarray(ys, f32)
    T = ys.shape[0]
    par = m.unpack(np.asarray(theta, f32))
    X = m.rinit(par, noise.init_normals())
    nw = np.log(np.ones(J, f32) / f32(J)).astype(f32)
    loglik = f32(0.0)
    logthresh = np.log(f32(thresh)) if thresh > 0 else f32(-np.inf)
    out = {"CLL": [], "ESS": [], "filter_mean": [], "prediction_mean": [],
           "ancestors": [], "log_weights": []}
    for i in range(T):
        X = m.rproc(par, X, noise.step_normals(i), i)
        meas = m.dmeas(par, ys[i], X)
        w = (nw + meas).astype(f32)
        nwn, lt = normalize(w)
        loglik = f32(loglik + lt)
        if diagnostics:
            out["log_weights"].append(w)
            out["CLL"].append(lt)
            with np.errstate(over="ignore"):
                out["ESS"].append(f32(1.0) / np.sum(np.exp(f32(2.0) * nwn), dtype=f32))
            out["filter_mean"].append((X * np.exp(nwn)[:, None]).sum(axis=0, dtype=f32))
            out["prediction_mean"].append(X.mean(axis=0, dtype=f32))
        with np.errstate(invalid="ignore"):
            do_resample = bool(np.max(nwn) - np.min(nwn) > logthresh)
        u = noise.resample_uniform(i)
        if do_resample:
            counts = resample(nwn, u)
            X = X[counts]
            nw = np.full(J, -np.log(f32(J)), f32)
        else:
            counts = np.arange(J)
            nw = nwn
        if diagnostics:
            out["ancestors"].append(counts)
    res = {"logLik": loglik}
    if diagnostics:
        for k, v in out.items():
            res[k] = np.asarray(v)
    return res


def mop(model, theta_est, ys, J, alpha, noise, with_ancestors=False):
    """``_mop_internal`` + ``_mop_step`` (mop.py:19-135): value only.

    ``theta_est`` is on the estimation scale (``SHOULD_TRANS = True``,
    mop.py:16).  Returns the negative MOP log-likelihood (float32).
    """
    m = MODELS[model]
    ys = np.asarray(ys, f32)
    T = ys.shape[0]
    par = m.unpack(m.from_est(np.asarray(theta_est, f32)))
    X = m.rinit(par, noise.init_normals())
    wF = np.log(np.ones(J, f32) / f32(J)).astype(f32)
    loglik = f32(0.0)
    anc = []
    a = f32(alpha)
    for i in range(T):
        wP = (a * wF).astype(f32)
        X = m.rproc(par, X, noise.step_normals(i), i)
        meas = m.dmeas(par, ys[i], X)
        loglik = f32(loglik + _lse(wP + meas) - _lse(wP))
        nw, _ = normalize(meas)
        u = noise.resample_uniform(i)
        counts = resample(nw, u)
        X = X[counts]
        wF = wP[counts]
        anc.append(counts)
    if with_ancestors:
        return f32(-loglik), np.asarray(anc)
    return f32(-loglik)


def _lse(v):
    v = np.asarray(v, f32)
    mx = np.max(v)
    if not np.isfinite(mx):
        mx = f32(0.0)
    return f32(mx + np.log(np.sum(np.exp(v - mx), dtype=f32)))


# ---------------------------------------------------------------------------
# simulate (used to make the reference's own LG data sets)
# ---------------------------------------------------------------------------


def simulate(model, theta, T, key: jr.Key, nsim=1):
    """``_simulate_internal`` (simulate.py:15-142) with nstep=1 and no covariates.

    Returns ``(X (T+1, nsim, dx), Y (T, nsim, dy))`` in float32.
    """
    m = MODELS[model]
    par = m.unpack(np.asarray(theta, f32))
    sk = jr.split(key, nsim + 1)
    key, keys = sk[0], sk[1:]
    X = m.rinit(par, np.stack([jr.normal(keys[s], (m.n_init(par),)) for s in range(nsim)]))
    Xs = [X]
    Ys = []
    for i in range(T):
        s = jr.split(key)
        key, sub = s[0], s[1]
        s2 = jr.split(sub)
        pk = jr.split(s2[1], nsim)
        z = np.stack([jr.normal(pk[j], (m.n_step(par),)) for j in range(nsim)])
        X = m.rproc(par, X, z, i)
        s3 = jr.split(key, nsim + 1)
        key, mk = s3[0], s3[1:]
        zm = np.stack([jr.normal(mk[j], (m.n_meas(par),)) for j in range(nsim)])
        Ys.append(m.rmeas(par, X, zm))
        Xs.append(X)
    return np.stack(Xs), np.stack(Ys)


def pomp_simulate_data(model, theta, T, key: jr.Key):
    """Data as ``Pomp.simulate(key=key, nsim=1, as_pomp=True)`` makes it.

    ``estimation_mixin.py:1173-1182``: ``_update_fresh_key`` splits ``key`` and
    uses the second half, which is split once more per parameter set
    (``pomp.py:391-408``).
    """
    new_key = jr.split(key)[1]
    k = jr.split(new_key, 1)[0]
    X, Y = simulate(model, theta, T, k, nsim=1)
    return X[:, 0, :], Y[:, 0, :]


# ---------------------------------------------------------------------------
# IF2: perturbed filter and the mif loop
# ---------------------------------------------------------------------------


class JaxPerfilterNoise:
    """The key tree of one IF2 iteration (``mif.py:112-140`` and ``:171-181``).

    ``split(key)`` -> carry key, t0-perturbation key (normal (J, P)); then
    ``split(key, J+1)`` -> carry key, J rinit keys; then
    ``split(key, T+1)[1:]`` are the step keys, each split in 3 (perturbation
    normal (J, P), process key, resampling key).  Inside ``rprocess_interp``
    the process key is split once per sub-step and then per particle
    (``model_mechanics.py:904`` and ``:586``), as in the bootstrap filter.
    """

    def __init__(self, key: jr.Key, J: int, P: int, n_init: int, n_step: int, T: int):
        s = jr.split(key)
        key, sub = s[0], s[1]
        self.zp0 = jr.normal(sub, (J, P))
        sk = jr.split(key, J + 1)
        key, self.init_keys = sk[0], sk[1:]
        self.step_keys = jr.split(key, T + 1)[1:]
        self.J, self.P, self.n_init, self.n_step = J, P, n_init, n_step

    def perturb0(self):
        return self.zp0

    def init_normals(self):
        if self.n_init == 0:
            return np.zeros((self.J, 0), f32)
        return np.stack([jr.normal(self.init_keys[j], (self.n_init,)) for j in range(self.J)])

    def _keys(self, t):
        k3 = jr.split(self.step_keys[t], 3)
        return k3[0], k3[1], k3[2]

    def perturb(self, t):
        return jr.normal(self._keys(t)[0], (self.J, self.P))

    def step_normals(self, t):
        if self.n_step == 0:
            return np.zeros((self.J, 0), f32)
        sub2 = jr.split(self._keys(t)[1])[1]
        pk = jr.split(sub2, self.J)
        return np.stack([jr.normal(pk[j], (self.n_step,)) for j in range(self.J)])

    def resample_uniform(self, t):
        return f32(jr.uniform(self._keys(t)[2]))


class ArrayPerfilterNoise:
    """Injected IF2 draws: ``zp0`` (J,P), ``zp`` (T,J,P), ``z0``, ``z``, ``u``."""

    def __init__(self, zp0, zp, z0, z, u):
        self.zp0, self.zp = np.asarray(zp0, f32), np.asarray(zp, f32)
        self.z0, self.z, self.u = np.asarray(z0, f32), np.asarray(z, f32), np.asarray(u, f32)

    def perturb0(self):
        return self.zp0

    def init_normals(self):
        return self.z0

    def perturb(self, t):
        return self.zp[t]

    def step_normals(self, t):
        return self.z[t]

    def resample_uniform(self, t):
        return f32(self.u[t])


class RecordingPerfilterNoise:
    """Wraps an IF2 noise source and records its draws as injection arrays."""

    def __init__(self, src):
        self.src = src
        self.rec = {"zp0": None, "z0": None, "zp": [], "z": [], "u": []}

    def perturb0(self):
        self.rec["zp0"] = self.src.perturb0()
        return self.rec["zp0"]

    def init_normals(self):
        self.rec["z0"] = self.src.init_normals()
        return self.rec["z0"]

    def perturb(self, t):
        v = self.src.perturb(t)
        self.rec["zp"].append(v)
        return v

    def step_normals(self, t):
        v = self.src.step_normals(t)
        self.rec["z"].append(v)
        return v

    def resample_uniform(self, t):
        v = self.src.resample_uniform(t)
        self.rec["u"].append(v)
        return v

    def arrays(self):
        r = self.rec
        return {"zp0": r["zp0"], "zp": np.stack(r["zp"]), "z0": r["z0"], "z": np.stack(r["z"]),
                "u": np.asarray(r["u"], f32)}


def _per_particle(m, th_est, fn, natural=False):
    """Apply ``fn(par, j)`` for each particle's natural-scale parameters."""
    nat = th_est if natural else m.from_est(th_est)
    return [fn(m.unpack(nat[j]), j) for j in range(th_est.shape[0])]


def perfilter(model, swarm_est, ys, J, rw_sig, rw_sig0, cool, cool0, noise, thresh=0.0, natural=False):
    """``_perfilter_internal`` + ``_perfilter_scan_body`` (mif.py:88-258).

    ``swarm_est`` (J, P) on the estimation scale (the natural scale with
    ``natural``: an identity ``ParTrans``); ``cool`` (T,) and ``cool0`` are the
    cooling factors.  Returns ``(swarm (J, P) after the last resampling,
    loglik float32)``.
    """
    m = MODELS[model]
    ys = np.asarray(ys, f32)
    T = ys.shape[0]
    rw_sig = np.asarray(rw_sig, f32)
    rw_sig0 = np.asarray(rw_sig0, f32)
    th = np.asarray(swarm_est, f32)
    th = (th + (f32(cool0) * rw_sig0)[None, :] * noise.perturb0()).astype(f32)
    z0 = noise.init_normals()
    X = np.concatenate(_per_particle(m, th, lambda p, j: m.rinit(p, z0[j:j + 1]), natural), axis=0).astype(f32)
    nw = np.full(J, -np.log(f32(J)), f32)
    loglik = f32(0.0)
    logthresh = np.log(f32(thresh)) if thresh > 0 else f32(-np.inf)
    log1e18 = np.log(f32(1e-18))
    for t in range(T):
        thp = (th + (f32(cool[t]) * rw_sig)[None, :] * noise.perturb(t)).astype(f32)
        z = noise.step_normals(t)
        X = np.concatenate(_per_particle(m, thp, lambda p, j: m.rproc(p, X[j:j + 1], z[j:j + 1], t), natural),
                           axis=0).astype(f32)
        meas = np.concatenate(_per_particle(m, thp, lambda p, j: m.dmeas(p, ys[t], X[j:j + 1]),
                                            natural)).astype(f32)
        meas = np.nan_to_num(meas, nan=log1e18).astype(f32)
        w = (nw + meas).astype(f32)
        nwn, lt = normalize(w)
        loglik = f32(loglik + lt)
        with np.errstate(invalid="ignore"):
            do_resample = bool(np.max(nwn) - np.min(nwn) > logthresh)
        u = noise.resample_uniform(t)
        if do_resample:
            counts = resample(nwn, u)
            X = X[counts]
            th = thp[counts]
            nw = (nwn[counts] - nwn[counts] - np.log(f32(J))).astype(f32)
        else:
            th = thp
            nw = nwn
    return th, loglik


def mif(model, theta, ys, J, M, rw_sig, rw_sig0, cooling, key: jr.Key, n_monitors=0, thresh=0.0):
    """``_mif_internal`` + ``_mif_scan_body`` (mif.py:16-85) for one replicate.

    ``theta`` (P,) natural scale; ``cooling(nt, m, ntimes)`` the schedule.
    Returns ``(logliks (M,), traces (M+1, P) natural, final swarm (J, P)
    natural, draws)`` where ``draws`` lists, per iteration, the recorded
    perturbed-filter draws and the monitors' draws.
    """
    m = MODELS[model]
    ys = np.asarray(ys, f32)
    T = ys.shape[0]
    th_est = m.to_est(np.asarray(theta, f32))
    P = th_est.shape[0]
    par0 = m.unpack(np.asarray(theta, f32))
    n_init, n_step = m.n_init(par0), m.n_step(par0)
    swarm = np.repeat(th_est[None, :], J, axis=0).astype(f32)
    m_keys = jr.split(key, M + 1)[1:]
    means = [swarm.mean(axis=0, dtype=f32)]
    logliks, draws = [], []
    for it in range(M):
        cool = np.array([cooling(i, it, T) for i in range(T)], f32)
        rec = RecordingPerfilterNoise(JaxPerfilterNoise(m_keys[it], J, P, n_init, n_step, T))
        new_swarm, ll = perfilter(model, swarm, ys, J, rw_sig, rw_sig0, cool, cool[0], rec, thresh)
        mon = []
        if n_monitors >= 1:
            mean = swarm.mean(axis=0, dtype=f32)
            mon_keys = jr.split(m_keys[it], n_monitors)
            nll = []
            for i in range(n_monitors):
                r = RecordingNoise(JaxKeyNoise(mon_keys[i], J, n_init, n_step))
                nll.append(-pfilter(model, m.from_est(mean), ys, J, r, thresh)["logLik"])
                z0, z, u = r.arrays()
                mon.append({"z0": z0, "z": z, "u": u})
            ll = -np.mean(np.asarray(nll, f32), dtype=f32)
        logliks.append(f32(ll))
        draws.append({"perfilter": rec.arrays(), "monitors": mon})
        swarm = new_swarm
        means.append(swarm.mean(axis=0, dtype=f32))
    traces = m.from_est(np.stack(means))
    return np.asarray(logliks, f32), traces, m.from_est(swarm), draws


def panel_pfilter(model, thetas, ys_units, J, keys, thresh=0.0):
    """``_chunked_panel_pfilter_internal`` (pfilter.py:248-304): one bootstrap
    filter per unit, natural-scale ``thetas`` (U, P), ``keys`` (U,) jaxrng
    keys.  Returns (logLiks (U,), recorded draws per unit)."""
    lls, draws = [], []
    for u, ys in enumerate(ys_units):
        rec = RecordingNoise(JaxKeyNoise(keys[u], J, 1, 1))
        lls.append(pfilter(model, thetas[u], ys, J, rec, thresh)["logLik"])
        z0, z, uu = rec.arrays()
        draws.append({"z0": z0, "z": z, "u": uu})
    return np.asarray(lls, f32), draws


def panel_mif(model, shared0, unit0, ys_units, J, M, rw_sig, rw_sig0, cooling, key: jr.Key,
              host_identity=False, thresh=0.0):
    """``_panel_mif_internal`` (panel_mif.py:17-247) for one replicate with
    ``block=True``, no monitors, and units whose canonical order is
    [shared | unit-specific] (the identity permutation).

    ``shared0`` (ns,) and ``unit0`` (U, nu) natural scale.  ``host_identity``
    restates a unit whose ``par_trans`` was replaced by ``ParTrans()`` after
    construction: the host-side transforms are the identity while the model
    mechanics keep the model's own transform (``pomp.py:271-313`` binds it to
    the components at construction).  Returns ``(shared_traces (M+1, ns+1),
    unit_traces (M+1, U, nu+1), draws[m][u])``.
    """
    m_ = MODELS[model]
    ns, U = len(shared0), len(ys_units)
    natural = False
    to_e = (lambda v: np.asarray(v, f32)) if host_identity else m_.to_est
    from_e = (lambda v: np.asarray(v, f32)) if host_identity else m_.from_est
    est = [to_e(np.concatenate([shared0, unit0[u]]).astype(f32)) for u in range(U)]
    S = np.repeat(est[0][None, :ns], J, axis=0).astype(f32)
    Us = np.stack([np.repeat(est[u][None, ns:], J, axis=0) for u in range(U)], axis=1).astype(f32)
    P = ns + Us.shape[2]
    par0 = m_.unpack(m_.from_est(est[0]))
    n_init, n_step = m_.n_init(par0), m_.n_step(par0)
    m_keys = jr.split(key, M + 1)[1:]

    def trace_row(ll_units):
        s_row = np.concatenate([[np.sum(ll_units)], S.mean(axis=0, dtype=f32)]) if ll_units is not None \
            else np.concatenate([[np.nan], S.mean(axis=0, dtype=f32)])
        u_rows = [np.concatenate([[np.nan if ll_units is None else ll_units[u]], Us[:, u].mean(axis=0, dtype=f32)])
                  for u in range(U)]
        return s_row, np.stack(u_rows)

    s_tr, u_tr = [], []
    a, b = trace_row(None)
    s_tr.append(a)
    u_tr.append(b)
    draws = []
    for it in range(M):
        unit_keys = jr.split(m_keys[it], U)
        lls = np.zeros(U, f32)
        dm = []
        for u in range(U):
            ys = np.asarray(ys_units[u], f32)
            T = ys.shape[0]
            cool = np.array([cooling(i, it, T) for i in range(T)], f32)
            th = np.concatenate([S, Us[:, u]], axis=1).astype(f32)
            rec = RecordingPerfilterNoise(JaxPerfilterNoise(unit_keys[u], J, P, n_init, n_step, T))
            new, ll = perfilter(model, th, ys, J, rw_sig, rw_sig0, cool, cool[0], rec, thresh, natural)
            S = new[:, :ns].astype(f32)
            Us[:, u] = new[:, ns:]
            lls[u] = ll
            dm.append({"perfilter": rec.arrays(), "monitors": []})
        draws.append(dm)
        a, b = trace_row(lls)
        s_tr.append(a)
        u_tr.append(b)
    s_tr, u_tr = np.stack(s_tr), np.stack(u_tr)
    if not host_identity:
        raise NotImplementedError("trace back-transform is only restated for identity host transforms")
    del from_e
    return s_tr, u_tr, draws
