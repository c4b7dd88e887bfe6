"""ctypes wrapper of the C oracle (``oracle/_build/libppf_oracle.so``).

TEST INFRASTRUCTURE ONLY.  Runs the restatement on HOST arrays with the same
descriptor layout as the CUDA library's ``ppf_pfilter_desc`` (include/ppf.h).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_SO = Path(__file__).resolve().parent / "_build" / "libppf_oracle.so"
_vp = ctypes.c_void_p


class _Model(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("dx", ctypes.c_int32), ("dy", ctypes.c_int32),
                ("n_params", ctypes.c_int32), ("dt", ctypes.c_float), ("reserved", ctypes.c_int32)]


class _Desc(ctypes.Structure):
    _fields_ = [("model", _Model), ("J", ctypes.c_int32), ("F", ctypes.c_int32),
                ("T", ctypes.c_int32), ("U", ctypes.c_int32), ("path", ctypes.c_int32),
                ("flags", ctypes.c_uint32), ("thresh", ctypes.c_float), ("tile", ctypes.c_int32)] + [
        (n, _vp) for n in ("theta", "ys", "ycon", "unit", "T_u", "seeds", "inj_z0", "inj_z",
                           "inj_u", "loglik", "cll", "ess", "fmean", "pmean", "anc", "logw",
                           "workspace")] + [("ws_bytes", ctypes.c_size_t)]


class _IF2Desc(ctypes.Structure):
    _fields_ = [("model", _Model), ("J", ctypes.c_int32), ("F", ctypes.c_int32),
                ("T", ctypes.c_int32), ("U", ctypes.c_int32), ("flags", ctypes.c_uint32),
                ("thresh", ctypes.c_float)] + [
        (n, _vp) for n in ("swarm_in", "swarm_out", "rw_sig", "rw_sig0", "cool", "cool0", "ys",
                           "ycon", "unit", "T_u", "seeds", "inj_zp0", "inj_zp", "inj_z0", "inj_z",
                           "inj_u", "loglik", "cll", "anc", "workspace")] + [("ws_bytes", ctypes.c_size_t)]


class _SimDesc(ctypes.Structure):
    _fields_ = [("model", _Model), ("F", ctypes.c_int32), ("nsim", ctypes.c_int32),
                ("T", ctypes.c_int32), ("flags", ctypes.c_uint32)] + [
        (n, _vp) for n in ("theta", "seeds", "X", "Y")]


def lib():
    if not _SO.exists():
        raise ImportError(f"oracle library missing: {_SO} (run `make -C oracle`)")
    L = ctypes.CDLL(str(_SO))
    L.ppfo_pfilter.argtypes = [ctypes.POINTER(_Desc), ctypes.c_int, ctypes.c_int]
    L.ppfo_pfilter.restype = ctypes.c_int
    L.ppfo_mop_surrogate.argtypes = [ctypes.POINTER(_Desc), ctypes.c_float, _vp, _vp, _vp, _vp]
    L.ppfo_mop_surrogate.restype = ctypes.c_int
    L.ppfo_dpop_surrogate.argtypes = [ctypes.POINTER(_Desc), ctypes.c_float, ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
                                      _vp]
    L.ppfo_dpop_surrogate.restype = ctypes.c_int
    L.ppfo_perfilter.argtypes = [ctypes.POINTER(_IF2Desc), ctypes.c_int]
    L.ppfo_perfilter.restype = ctypes.c_int
    L.ppfo_expf.argtypes = [ctypes.c_float]
    L.ppfo_expf.restype = ctypes.c_float
    L.ppfo_logf.argtypes = [ctypes.c_float]
    L.ppfo_logf.restype = ctypes.c_float
    L.ppfo_sincos2pif.argtypes = [ctypes.c_float, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    L.ppfo_philox.argtypes = [_vp, _vp, _vp]
    L.ppfo_normals.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                               ctypes.c_int, _vp]
    L.ppfo_simulate.argtypes = [ctypes.POINTER(_SimDesc)]
    L.ppfo_simulate.restype = ctypes.c_int
    L.ppfo_poisson.argtypes = [ctypes.c_float, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
    L.ppfo_poisson.restype = ctypes.c_float
    L.ppfo_logfact.argtypes = [ctypes.c_float]
    L.ppfo_logfact.restype = ctypes.c_float
    return L


_LIB = None


def _L():
    global _LIB
    if _LIB is None:
        _LIB = lib()
    return _LIB


def _p(a):
    return 0 if a is None else a.ctypes.data


def pfilter(kind, dx, dy, theta_f, ys, J, *, seeds=None, ycon=None, unit=None, T_u=None,
            dt=0.0, thresh=0.0, est=False, inject=None, mop=False, CLL=False, ESS=False,
            fmean=False, pmean=False, anc=False, logw=False, nthreads=1):
    """Run the oracle over F filters; arrays on the host.  Returns a dict."""
    theta_f = np.ascontiguousarray(np.atleast_2d(theta_f), dtype=np.float32)
    F, P = theta_f.shape
    ys = np.ascontiguousarray(ys, dtype=np.float32)
    if ys.ndim == 2:
        ys = ys[None]
    U, T, _ = ys.shape
    keep = [theta_f, ys]
    d = _Desc()
    d.model = _Model(kind, dx, dy, P, dt, 0)
    d.J, d.F, d.T, d.U = J, F, T, U
    flags = (1 if CLL else 0) | (2 if ESS else 0) | (4 if fmean else 0) | (8 if pmean else 0)
    flags |= (32 if anc else 0) | (64 if logw else 0) | (128 if est else 0)
    d.thresh = thresh
    d.theta, d.ys = _p(theta_f), _p(ys)
    if ycon is not None:
        ycon = np.ascontiguousarray(ycon, dtype=np.float32)
        keep.append(ycon)
        d.ycon = _p(ycon)
    if unit is not None:
        unit = np.ascontiguousarray(unit, dtype=np.int32)
        keep.append(unit)
        d.unit = _p(unit)
    if T_u is not None:
        T_u = np.ascontiguousarray(T_u, dtype=np.int32)
        keep.append(T_u)
        d.T_u = _p(T_u)
    if seeds is not None:
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        keep.append(seeds)
        d.seeds = _p(seeds)
    if inject is not None:
        flags |= 16
        for k, name in (("z0", "inj_z0"), ("z", "inj_z"), ("u", "inj_u")):
            if inject.get(k) is not None:
                a = np.ascontiguousarray(inject[k], dtype=np.float32)
                keep.append(a)
                setattr(d, name, _p(a))
    d.flags = flags
    out = {"loglik": np.zeros(F, np.float64)}
    if CLL:
        out["cll"] = np.zeros((F, T), np.float64)
    if ESS:
        out["ess"] = np.zeros((F, T), np.float32)
    if fmean:
        out["fmean"] = np.zeros((F, T, dx), np.float32)
    if pmean:
        out["pmean"] = np.zeros((F, T, dx), np.float32)
    if anc:
        out["anc"] = np.zeros((F, T, J), np.int32)
    if logw:
        out["logw"] = np.zeros((F, T, J), np.float32)
    d.loglik = _p(out["loglik"])
    d.cll, d.ess = _p(out.get("cll")), _p(out.get("ess"))
    d.fmean, d.pmean = _p(out.get("fmean")), _p(out.get("pmean"))
    d.anc, d.logw = _p(out.get("anc")), _p(out.get("logw"))
    rc = _L().ppfo_pfilter(ctypes.byref(d), 1 if mop else 0, int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle returned {rc}")
    del keep
    return out


def mop_surrogate(kind, dx, dy, theta_est, ys, J, alpha, anc, m0=None, *, seeds=None,
                  ycon=None, dt=0.0, inject=None, natural=False, pwi=None, p0=None):
    """MOP-alpha surrogate value (frozen ancestry, frozen stop_gradient(m)).

    ``anc`` (F,T,J) ancestors; ``m0`` (F,T,J) or None to record it.  Returns
    ``(value (F,), m0 (F,T,J))``.  With ``pwi`` (a state component) it is the
    DPOP surrogate: the predicted state's component ``pwi`` enters the carried
    weights as ``pw - p0`` (``p0`` (F,T,J) frozen, or None to record it), and
    the return is ``(value, m0, p0)``."""
    theta_est = np.ascontiguousarray(np.atleast_2d(theta_est), dtype=np.float32)
    F, P = theta_est.shape
    ys = np.ascontiguousarray(ys, dtype=np.float32)
    if ys.ndim == 2:
        ys = ys[None]
    U, T, _ = ys.shape
    keep = [theta_est, ys]
    d = _Desc()
    d.model = _Model(kind, dx, dy, P, dt, 0)
    d.J, d.F, d.T, d.U = J, F, T, U
    flags = 0 if natural else 128
    d.theta, d.ys = _p(theta_est), _p(ys)
    if ycon is not None:
        ycon = np.ascontiguousarray(ycon, dtype=np.float32)
        keep.append(ycon)
        d.ycon = _p(ycon)
    if seeds is not None:
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        keep.append(seeds)
        d.seeds = _p(seeds)
    if inject is not None:
        flags |= 16
        for k, name in (("z0", "inj_z0"), ("z", "inj_z"), ("u", "inj_u")):
            if inject.get(k) is not None:
                a = np.ascontiguousarray(inject[k], dtype=np.float32)
                keep.append(a)
                setattr(d, name, _p(a))
    d.flags = flags
    anc = np.ascontiguousarray(anc, dtype=np.int32)
    m0_out = np.zeros((F, T, J), np.float32) if m0 is None else None
    m0_in = None if m0 is None else np.ascontiguousarray(m0, dtype=np.float32)
    value = np.zeros(F, np.float64)
    if pwi is None:
        rc = _L().ppfo_mop_surrogate(ctypes.byref(d), float(alpha), _p(anc), _p(m0_in), _p(m0_out), _p(value))
    else:
        p0_out = np.zeros((F, T, J), np.float32) if p0 is None else None
        p0_in = None if p0 is None else np.ascontiguousarray(p0, dtype=np.float32)
        rc = _L().ppfo_dpop_surrogate(ctypes.byref(d), float(alpha), int(pwi), _p(anc), _p(m0_in), _p(m0_out),
                                      _p(p0_in), _p(p0_out), _p(value))
    if rc != 0:
        raise RuntimeError(f"oracle returned {rc}")
    del keep
    if pwi is not None:
        return value, (m0_out if m0 is None else m0_in), (p0_out if p0 is None else p0_in)
    return value, (m0_out if m0 is None else m0_in)


def perfilter(kind, dx, dy, swarm, ys, J, rw_sig, rw_sig0, cool, cool0, *, seeds=None,
              ycon=None, unit=None, T_u=None, dt=0.0, thresh=0.0, inject=None, CLL=False,
              anc=False, nthreads=1, natural=False):
    """One IF2 iteration over F swarms (``swarm`` (F, P, J), estimation scale).

    ``cool`` (U, T) and ``cool0`` (U,) are the cooling factors; ``inject`` may
    hold ``zp0`` (F,J,P), ``zp`` (F,T,J,P), ``z0``, ``z``, ``u``.  Returns a
    dict with ``loglik`` (F,), ``swarm`` (F, P, J) and optional ``cll``/``anc``."""
    swarm = np.ascontiguousarray(swarm, dtype=np.float32)
    F, P, Jc = swarm.shape
    assert Jc == J
    ys = np.ascontiguousarray(ys, dtype=np.float32)
    if ys.ndim == 2:
        ys = ys[None]
    U, T, _ = ys.shape
    rw_sig = np.ascontiguousarray(rw_sig, dtype=np.float32)
    rw_sig0 = np.ascontiguousarray(rw_sig0, dtype=np.float32)
    cool = np.ascontiguousarray(np.broadcast_to(np.asarray(cool, np.float32), (U, T)))
    cool0 = np.ascontiguousarray(np.broadcast_to(np.asarray(cool0, np.float32), (U,)))
    keep = [swarm, ys, rw_sig, rw_sig0, cool, cool0]
    d = _IF2Desc()
    d.model = _Model(kind, dx, dy, P, dt, 0)
    d.J, d.F, d.T, d.U = J, F, T, U
    d.thresh = thresh
    flags = (1 if CLL else 0) | (32 if anc else 0) | (256 if natural else 0)
    d.swarm_in, d.ys = _p(swarm), _p(ys)
    d.rw_sig, d.rw_sig0, d.cool, d.cool0 = _p(rw_sig), _p(rw_sig0), _p(cool), _p(cool0)
    for name, a, dt_ in (("ycon", ycon, np.float32), ("unit", unit, np.int32), ("T_u", T_u, np.int32),
                         ("seeds", seeds, np.uint64)):
        if a is not None:
            a = np.ascontiguousarray(a, dtype=dt_)
            keep.append(a)
            setattr(d, name, _p(a))
    if inject is not None:
        flags |= 16
        for k in ("zp0", "zp", "z0", "z", "u"):
            if inject.get(k) is not None:
                a = np.ascontiguousarray(inject[k], dtype=np.float32)
                keep.append(a)
                setattr(d, "inj_" + k, _p(a))
    d.flags = flags
    out = {"loglik": np.zeros(F, np.float64), "swarm": np.zeros((F, P, J), np.float32)}
    if CLL:
        out["cll"] = np.zeros((F, T), np.float64)
    if anc:
        out["anc"] = np.zeros((F, T, J), np.int32)
    d.loglik, d.swarm_out = _p(out["loglik"]), _p(out["swarm"])
    d.cll, d.anc = _p(out.get("cll")), _p(out.get("anc"))
    rc = _L().ppfo_perfilter(ctypes.byref(d), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle returned {rc}")
    del keep
    return out


def expf(x):
    return np.float32(_L().ppfo_expf(float(x)))


def logf(x):
    return np.float32(_L().ppfo_logf(float(x)))


def sincos2pi(u):
    s, c = ctypes.c_float(), ctypes.c_float()
    _L().ppfo_sincos2pif(float(u), ctypes.byref(s), ctypes.byref(c))
    return np.float32(s.value), np.float32(c.value)


def philox(ctr, key):
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32)
    key = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    _L().ppfo_philox(_p(ctr), _p(key), _p(out))
    return out


def normals(seed, j, s, tag, n):
    z = np.zeros(n, np.float32)
    _L().ppfo_normals(int(seed), int(j), int(s), int(tag), int(n), _p(z))
    return z


def simulate(kind, dx, dy, theta_f, nsim, T, seeds, *, dt=0.0, est=False):
    """Trajectories of F parameter sets x nsim replicates (``ppfo_simulate``):
    returns X (F, nsim, T+1, dx) and Y (F, nsim, T, dy) as float32."""
    theta_f = np.ascontiguousarray(np.atleast_2d(theta_f), dtype=np.float32)
    F, P = theta_f.shape
    seeds = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(F))
    X = np.zeros((F, nsim, T + 1, dx), np.float32)
    Y = np.zeros((F, nsim, T, dy), np.float32)
    d = _SimDesc()
    d.model = _Model(kind, dx, dy, P, dt, 0)
    d.F, d.nsim, d.T, d.flags = F, nsim, T, (1 << 7) if est else 0
    d.theta, d.seeds, d.X, d.Y = _p(theta_f), _p(seeds), _p(X), _p(Y)
    rc = _L().ppfo_simulate(ctypes.byref(d))
    if rc != 0:
        raise RuntimeError(f"ppfo_simulate returned {rc}")
    return X, Y


def poisson(lam, seed, k, s):
    """One draw of the shared Poisson sampler (include/ppf_sample.h)."""
    return float(_L().ppfo_poisson(float(lam), int(seed), int(k), int(s)))


def logfact(k):
    return float(_L().ppfo_logfact(float(k)))
