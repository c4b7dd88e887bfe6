"""Stateless drop-ins for ``pypomp.functional`` on the CUDA library.

Signatures and return layouts follow the reference
(``pypomp/functional/pfilter.py:11-90``, ``mop.py:8-62``, ``mif.py:15-122``,
``train.py:14-110``); the work is one call into ``libppf.so`` per batch of
filters instead of a jitted XLA program.  Arrays come back as NumPy.

``struct`` is a :class:`PompStruct` (from ``Pomp.to_struct()``), ``keys`` are
uint64 key arrays (``pypomp_b200.random``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _ffi
from .models import ModelSpec


@dataclass
class PompStruct:
    """What the kernels need from a model (``pypomp/functional/structs.py:10``)."""

    spec: ModelSpec
    ys: np.ndarray            # (T, dy) float32, or (U, T, dy) for panels
    times: np.ndarray
    t0: float
    T_u: np.ndarray | None = None   # (U,) lengths for ragged panels

    @property
    def param_names(self):
        return list(self.spec.param_names)


def align_params(params, names, axis: int = -1) -> np.ndarray:
    """Stack named parameter values in the order ``names``
    (``pypomp/functional/utils.py:7-48``), e.g. ``struct.param_names``."""
    try:
        return np.stack([np.asarray(params[name]) for name in names], axis=axis)
    except KeyError as e:
        raise KeyError(
            f"Parameter '{e.args[0]}' is required by the model structure but missing from inputs.") from e


def _device_inputs(torch, struct: PompStruct, dev):
    ys = np.asarray(struct.ys, dtype=np.float32)
    if ys.ndim == 2:
        ys = ys[None]
    U, T, _ = ys.shape
    ycon = struct.spec.ycon(ys)
    ys_d = torch.from_numpy(np.ascontiguousarray(ys)).to(dev)
    ycon_d = torch.from_numpy(np.ascontiguousarray(ycon)).to(dev) if ycon is not None else None
    Tu_d = None
    if struct.T_u is not None:
        Tu_d = torch.from_numpy(np.asarray(struct.T_u, dtype=np.int32)).to(dev)
    return ys_d, ycon_d, Tu_d, U, T


def run_pfilter(struct: PompStruct, theta_f: np.ndarray, seeds_f: np.ndarray, J: int, *,
                thresh: float = 0.0, CLL=False, ESS=False, filter_mean=False,
                prediction_mean=False, est=False, unit_f=None, path=None, inject=None,
                save_ancestors=False, save_weights=False, return_torch=False, fast=False):
    """One batched call of ``ppf_pfilter`` over F filters.

    ``theta_f`` (F, P) parameters, ``seeds_f`` (F,) keys.  ``inject`` is an
    optional dict of host arrays ``z0`` (F,J,n0), ``z`` (F,T,J,nz), ``u``
    (F,T) that replaces the Philox draws.  ``path`` is "plain", "stream",
    "resident", "cluster", "stream@<tile>" (tile 2048, 512 or 256 particles
    per CTA) or None (automatic).  ``fast`` sets ``PPF_F_FAST`` (streaming
    path, Philox draws: hardware special-function approximations, not
    bit-identical with the oracle).  Returns a dict of NumPy arrays.
    """
    torch = _ffi.require_cuda()
    if J < 1:
        raise ValueError("J should be greater than 0.")
    if J > _ffi.PPF_MAX_J:
        raise ValueError(f"J must be at most {_ffi.PPF_MAX_J}.")
    dev = torch.device("cuda", torch.cuda.current_device())
    spec = struct.spec
    theta_f = np.ascontiguousarray(theta_f, dtype=np.float32)
    F = theta_f.shape[0]
    ys_d, ycon_d, Tu_d, U, T = _device_inputs(torch, struct, dev)
    th_d = torch.from_numpy(theta_f).to(dev)
    seeds_d = torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).copy()).to(dev)
    unit_d = None
    if unit_f is not None:
        unit_d = torch.from_numpy(np.asarray(unit_f, dtype=np.int32)).to(dev)
    flags = (_ffi.F_CLL if CLL else 0) | (_ffi.F_ESS if ESS else 0)
    flags |= (_ffi.F_FMEAN if filter_mean else 0) | (_ffi.F_PMEAN if prediction_mean else 0)
    flags |= (_ffi.F_EST if est else 0)
    flags |= (_ffi.F_SAVE_ANC if save_ancestors else 0) | (_ffi.F_SAVE_W if save_weights else 0)
    flags |= _ffi.F_FAST if fast else 0
    out = {"loglik": torch.zeros(F, dtype=torch.float64, device=dev)}
    f32 = dict(dtype=torch.float32, device=dev)
    if CLL:
        out["cll"] = torch.zeros(F, T, dtype=torch.float64, device=dev)
    if ESS:
        out["ess"] = torch.zeros(F, T, **f32)
    if filter_mean:
        out["fmean"] = torch.zeros(F, T, spec.dx, **f32)
    if prediction_mean:
        out["pmean"] = torch.zeros(F, T, spec.dx, **f32)
    if save_ancestors:
        out["anc"] = torch.zeros(F, T, J, dtype=torch.int32, device=dev)
    if save_weights:
        out["logw"] = torch.zeros(F, T, J, **f32)
    inj = {}
    if inject is not None:
        flags |= _ffi.F_INJECT
        for k in ("z0", "z", "u"):
            if inject.get(k) is not None:
                inj[k] = torch.from_numpy(np.ascontiguousarray(inject[k], dtype=np.float32)).to(dev)
    d = _ffi.PfilterDesc()
    d.model = spec.ffi_model()
    d.J, d.F, d.T, d.U = J, F, T, U
    tile = 0
    if isinstance(path, str) and "@" in path:     # "stream@512": stream path with a fixed tile
        path, tile = path.split("@")
        tile = int(tile)
    d.path = _ffi.env_path() if path is None else _ffi.PATHS[path] if isinstance(path, str) else int(path)
    d.tile = tile
    d.flags = flags
    d.thresh = float(max(0.0, thresh))
    d.theta, d.ys, d.ycon = _ffi.ptr(th_d), _ffi.ptr(ys_d), _ffi.ptr(ycon_d)
    d.unit, d.T_u, d.seeds = _ffi.ptr(unit_d), _ffi.ptr(Tu_d), _ffi.ptr(seeds_d)
    d.inj_z0, d.inj_z, d.inj_u = _ffi.ptr(inj.get("z0")), _ffi.ptr(inj.get("z")), _ffi.ptr(inj.get("u"))
    d.loglik = _ffi.ptr(out["loglik"])
    d.cll, d.ess = _ffi.ptr(out.get("cll")), _ffi.ptr(out.get("ess"))
    d.fmean, d.pmean = _ffi.ptr(out.get("fmean")), _ffi.ptr(out.get("pmean"))
    d.anc, d.logw = _ffi.ptr(out.get("anc")), _ffi.ptr(out.get("logw"))
    nbytes = _ffi.LIB.ppf_pfilter_workspace_bytes(d)
    ws = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    stream = torch.cuda.current_stream(dev).cuda_stream
    _ffi.check(_ffi.LIB.ppf_pfilter(d, stream), "ppf_pfilter")
    _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_pfilter")
    if return_torch:
        return out
    return {k: v.cpu().numpy() for k, v in out.items()}


def autotune(struct: PompStruct, theta_f: np.ndarray, seeds_f: np.ndarray, J: int, *, unit_f=None,
             thresh: float = 0.0) -> int:
    """Time the stream path's tile sizes for this shape (``ppf_autotune``) and
    keep the fastest for later calls of the same shape; returns the tile (0 if
    the shape runs on the resident or cluster path)."""
    import ctypes

    torch = _ffi.require_cuda()
    dev = torch.device("cuda", torch.cuda.current_device())
    theta_f = np.ascontiguousarray(theta_f, dtype=np.float32)
    F = theta_f.shape[0]
    ys_d, ycon_d, Tu_d, U, T = _device_inputs(torch, struct, dev)
    th_d = torch.from_numpy(theta_f).to(dev)
    seeds_d = torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).copy()).to(dev)
    unit_d = None if unit_f is None else torch.from_numpy(np.asarray(unit_f, dtype=np.int32)).to(dev)
    ll = torch.zeros(F, dtype=torch.float64, device=dev)
    d = _ffi.PfilterDesc()
    d.model = struct.spec.ffi_model()
    d.J, d.F, d.T, d.U = J, F, T, U
    d.path = _ffi.env_path()
    d.thresh = float(max(0.0, thresh))
    d.theta, d.ys, d.ycon = _ffi.ptr(th_d), _ffi.ptr(ys_d), _ffi.ptr(ycon_d)
    d.unit, d.T_u, d.seeds, d.loglik = _ffi.ptr(unit_d), _ffi.ptr(Tu_d), _ffi.ptr(seeds_d), _ffi.ptr(ll)
    # zeroed: on a shape that runs on another path nothing is launched, and the
    # status word read below must then read as success
    ws = torch.zeros(max(int(_ffi.LIB.ppf_pfilter_workspace_bytes(d)), 256), dtype=torch.uint8, device=dev)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    best = ctypes.c_int(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    _ffi.check(_ffi.LIB.ppf_autotune(d, stream, ctypes.byref(best)), "ppf_autotune")
    _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_autotune")
    return int(best.value)


def pfilter(struct: PompStruct, thetas_array, J: int, keys, thresh: float = 0.0,
            CLL: bool = False, ESS: bool = False, filter_mean: bool = False,
            prediction_mean: bool = False, *, path=None, fast: bool = False) -> dict:
    """Bootstrap particle filter (``pypomp/functional/pfilter.py:11-90``).

    ``thetas_array`` (n_theta, P) natural scale; ``keys`` (n_theta, reps).
    Returns ``logLik`` (n_theta, reps) and, when requested, ``CLL``/``ESS``
    (n_theta, reps, T) and ``filter_mean``/``prediction_mean``
    (n_theta, reps, T, dx).  ``fast`` (not in the reference) uses the
    ``PPF_F_FAST`` kernels on the streaming path.
    """
    thetas = np.atleast_2d(np.asarray(thetas_array, dtype=np.float32))
    keys = np.asarray(keys, dtype=np.uint64)
    if keys.ndim == 1:
        keys = keys.reshape(thetas.shape[0], -1)
    n, reps = keys.shape
    if n != thetas.shape[0]:
        raise ValueError("keys must have shape (n_theta, reps)")
    theta_f = np.repeat(thetas, reps, axis=0)
    res = run_pfilter(struct, theta_f, keys.reshape(-1), J, thresh=thresh, CLL=CLL, ESS=ESS,
                      filter_mean=filter_mean, prediction_mean=prediction_mean, path=path, fast=fast)
    T = res.get("cll", res.get("ess", np.zeros((0, 0)))).shape[-1] if (CLL or ESS) else None
    out = {"logLik": res["loglik"].reshape(n, reps)}
    if CLL:
        out["CLL"] = res["cll"].reshape(n, reps, -1)
    if ESS:
        out["ESS"] = res["ess"].reshape(n, reps, -1)
    if filter_mean:
        out["filter_mean"] = res["fmean"].reshape(n, reps, res["fmean"].shape[1], -1)
    if prediction_mean:
        out["prediction_mean"] = res["pmean"].reshape(n, reps, res["pmean"].shape[1], -1)
    del T
    return out


def simulate(struct: PompStruct, thetas_array, nsim: int, keys, times=None, *, est: bool = False,
             return_torch: bool = False):
    """Simulated states and observations (``pypomp/functional/simulate.py:8-72``).

    ``thetas_array`` (n_reps, P) on the natural scale (estimation scale with
    ``est``), ``keys`` one key per row.  ``times`` only sets the number of
    observation times, since the built-in models take one process step per
    observation; it defaults to ``struct.times``.  Returns ``X_sims``
    (n_reps, nsim, T+1, dx), the initial state first, and ``Y_sims``
    (n_reps, nsim, T, dy): NumPy arrays, or CUDA tensors with
    ``return_torch``.  One ``ppf_simulate`` launch per 65535 parameter sets.
    """
    torch = _ffi.require_cuda()
    if int(nsim) < 1:
        raise ValueError("nsim must be at least 1.")
    nsim = int(nsim)
    thetas = np.ascontiguousarray(np.atleast_2d(np.asarray(thetas_array, dtype=np.float32)))
    n = thetas.shape[0]
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != n:
        raise ValueError("keys must hold one key per parameter set")
    spec = struct.spec
    if thetas.shape[1] != spec.n_params:
        raise ValueError(f"thetas_array must have {spec.n_params} columns")
    T = len(struct.times if times is None else times)
    dev = torch.device("cuda", torch.cuda.current_device())
    th_d = torch.from_numpy(thetas).to(dev)
    seeds_d = torch.from_numpy(keys.view(np.int64).copy()).to(dev)
    X = torch.empty(n, nsim, T + 1, spec.dx, dtype=torch.float32, device=dev)
    Y = torch.empty(n, nsim, T, spec.dy, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for f0 in range(0, n, 65535):
        f1 = min(n, f0 + 65535)
        d = _ffi.SimulateDesc()
        d.model = spec.ffi_model()
        d.F, d.nsim, d.T = f1 - f0, nsim, T
        d.flags = _ffi.F_EST if est else 0
        d.theta, d.seeds = _ffi.ptr(th_d[f0:f1]), _ffi.ptr(seeds_d[f0:f1])
        d.X, d.Y = _ffi.ptr(X[f0:f1]), (_ffi.ptr(Y[f0:f1]) if T > 0 else 0)
        _ffi.check(_ffi.LIB.ppf_simulate(d, stream), "ppf_simulate")
    if return_torch:
        return X, Y
    return X.cpu().numpy(), Y.cpu().numpy()


class PfilterCall:
    """Repeated ``ppf_pfilter`` calls of one shape: device buffers, workspace
    and descriptor made once, the launch sequence captured into a CUDA graph
    on the first call (``PPF_F_GRAPH``) and replayed after copying the new
    parameters and keys into the same buffers.  Used by :func:`pmcmc`, which
    filters every chain once per iteration."""

    def __init__(self, struct: PompStruct, F: int, J: int, *, thresh: float = 0.0, est: bool = False):
        torch = _ffi.require_cuda()
        if J < 1:
            raise ValueError("J should be greater than 0.")
        if J > _ffi.PPF_MAX_J:
            raise ValueError(f"J must be at most {_ffi.PPF_MAX_J}.")
        self.torch = torch
        dev = torch.device("cuda", torch.cuda.current_device())
        spec = struct.spec
        self.P = spec.n_params
        ys_d, ycon_d, Tu_d, U, T = _device_inputs(torch, struct, dev)
        self.keep = [ys_d, ycon_d, Tu_d]
        self.theta = torch.zeros(F, self.P, dtype=torch.float32, device=dev)
        self.seeds = torch.zeros(F, dtype=torch.int64, device=dev)
        self.ll = torch.zeros(F, dtype=torch.float64, device=dev)
        d = _ffi.PfilterDesc()
        d.model = spec.ffi_model()
        d.J, d.F, d.T, d.U = J, F, T, U
        d.path = _ffi.env_path()
        d.flags = (_ffi.F_EST if est else 0) | _ffi.F_GRAPH
        d.thresh = float(max(0.0, thresh))
        d.theta, d.ys, d.ycon = _ffi.ptr(self.theta), _ffi.ptr(ys_d), _ffi.ptr(ycon_d)
        d.T_u, d.seeds, d.loglik = _ffi.ptr(Tu_d), _ffi.ptr(self.seeds), _ffi.ptr(self.ll)
        self.ws = torch.empty(max(int(_ffi.LIB.ppf_pfilter_workspace_bytes(d)), 256), dtype=torch.uint8,
                              device=dev)
        d.workspace, d.ws_bytes = _ffi.ptr(self.ws), self.ws.numel()
        self.d = d
        self.stream = torch.cuda.current_stream(dev).cuda_stream

    def __call__(self, theta_f: np.ndarray, seeds_f: np.ndarray) -> np.ndarray:
        torch = self.torch
        self.theta.copy_(torch.from_numpy(np.ascontiguousarray(theta_f, dtype=np.float32)))
        self.seeds.copy_(torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).copy()))
        _ffi.check(_ffi.LIB.ppf_pfilter(self.d, self.stream), "ppf_pfilter")
        _ffi.check(_ffi.LIB.ppf_workspace_status(self.d.workspace, self.stream), "ppf_pfilter")
        return self.ll.cpu().numpy().copy()


def _split4(keys: np.ndarray):
    from . import random as pprandom

    out = np.stack([pprandom.split(k, 4) for k in keys])
    return out[:, 0], out[:, 1], out[:, 2], out[:, 3]


def pmcmc(struct: PompStruct, thetas_array, proposal, M: int, J: int, keys, thresh: float = 0.0,
          dprior=None):
    """Particle marginal Metropolis-Hastings (``pypomp/functional/pmcmc.py:18-113``,
    ``pypomp/core/algorithms/pmcmc.py:30-163``; Andrieu, Doucet & Holenstein 2010).

    One chain per row of ``thetas_array`` (natural scale), each with its own
    key.  Chains move on the estimation scale; the acceptance ratio uses the
    prior there (``dprior`` of the natural parameters plus the log-Jacobian of
    the back-transform).  Per chain and iteration the key splits four ways
    (carry, proposal, filter, acceptance), as the reference's scan does.  All
    chains' particle filters of one iteration run as one batched
    ``ppf_pfilter`` launch, replayed from a CUDA graph.

    ``dprior`` is a callable on a dict of natural-scale parameters returning
    a log density (``None``: flat).  Returns ``(loglik_traces (n, M+1),
    log_prior_traces (n, M+1), theta_traces (n, M+1, d), accepts (n,))``,
    traces on the natural scale, the log-prior recomputed there without the
    Jacobian.
    """
    if int(M) < 1:
        raise ValueError("M must be >= 1.")
    thetas = np.atleast_2d(np.asarray(thetas_array, dtype=np.float64))
    call = PfilterCall(struct, thetas.shape[0], J, thresh=thresh, est=True)
    return _pmcmc_run(struct.spec, thetas, proposal, int(M), keys, call, dprior)


def _pmcmc_run(spec, thetas, proposal, M: int, keys, loglik_fn, dprior=None):
    """The chains of :func:`pmcmc` given ``loglik_fn(theta_est (n, d), keys (n,))``
    -> log-likelihoods (n,): the batched GPU filter in the product, the C
    oracle's filter in the CPU tests."""
    from . import random as pprandom

    names = list(spec.param_names)
    thetas = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
    n, d = thetas.shape
    if d != len(names):
        raise ValueError(f"thetas_array must have {len(names)} columns")
    keys = np.asarray(keys, dtype=np.uint64).reshape(n)
    prop = proposal.canonicalize(names)

    def prior_nat(th):
        if dprior is None:
            return 0.0
        return float(dprior({nm: float(v) for nm, v in zip(names, th)}))

    def prior_est(th_est):
        return prior_nat(spec.from_est(th_est)) + float(spec.log_det_jac_from_est(th_est))

    call = loglik_fn
    th_cur = spec.to_est(thetas)
    carry = np.empty(n, np.uint64)
    pf0 = np.empty(n, np.uint64)
    for c in range(n):
        carry[c], pf0[c] = pprandom.split(keys[c], 2)
    ll_cur = call(th_cur, pf0)
    lp_cur = np.array([prior_est(t) for t in th_cur])
    state = [prop.init_state(t) for t in th_cur]
    accepts = np.zeros(n, np.int64)
    ll_tr = np.empty((n, M + 1))
    lp_tr = np.empty((n, M + 1))
    th_tr = np.empty((n, M + 1, d))
    ll_tr[:, 0], lp_tr[:, 0], th_tr[:, 0] = ll_cur, lp_cur, th_cur
    for it in range(1, M + 1):
        carry, k_prop, k_pf, k_acc = _split4(carry)
        th_prop = np.empty_like(th_cur)
        for c in range(n):
            th_prop[c], state[c] = prop.step(state[c], th_cur[c], k_prop[c], it, int(accepts[c]))
        lp_prop = np.array([prior_est(t) for t in th_prop])
        ll_prop = call(th_prop, k_pf)
        log_alpha = ll_prop + lp_prop - ll_cur - lp_cur
        u = np.array([np.random.default_rng(int(k)).random() for k in k_acc])
        with np.errstate(divide="ignore", invalid="ignore"):
            acc = np.isfinite(log_alpha) & np.isfinite(lp_prop) & (np.log(u) < log_alpha)
        th_cur = np.where(acc[:, None], th_prop, th_cur)
        ll_cur = np.where(acc, ll_prop, ll_cur)
        lp_cur = np.where(acc, lp_prop, lp_cur)
        accepts += acc
        ll_tr[:, it], lp_tr[:, it], th_tr[:, it] = ll_cur, lp_cur, th_cur
    th_nat = spec.from_est(th_tr)
    lp_nat = np.array([[prior_nat(t) for t in chain] for chain in th_nat])
    return ll_tr, lp_nat, th_nat, accepts.astype(np.int32)


class MopCall:
    """One batched MOP-alpha evaluation on the device: inputs, outputs and the
    workspace that keeps the forward's saves (ancestors, first-child offsets,
    state checkpoints) for a later adjoint sweep.

    ``theta_est`` is a (F, P) host array or CUDA tensor on the estimation
    scale (natural scale with ``natural``, ``PPF_F_NATURAL``).  ``forward(grad)`` runs ``ppf_mop`` (the adjoint too when
    ``grad``); ``backward(dvalue)`` runs ``ppf_mop_backward`` on the same
    workspace and returns ``dvalue[f] * d value[f] / d theta[f]``.
    """

    def __init__(self, struct: PompStruct, theta_est, seeds_f, J: int, alpha: float, *, unit_f=None,
                 inject=None, ckpt_every: int = 0, save_ancestors: bool = False, natural: bool = False,
                 graph: bool = False, persistent: bool = True, process_weight_index: int | None = None):
        torch = _ffi.require_cuda()
        if J < 1:
            raise ValueError("J should be greater than 0.")
        if J > _ffi.PPF_MAX_J:
            raise ValueError(f"J must be at most {_ffi.PPF_MAX_J}.")
        if not 0.0 <= float(alpha) <= 1.0:
            raise ValueError("alpha must be in [0, 1]")
        self.torch = torch
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        spec = struct.spec
        if hasattr(theta_est, "is_cuda"):
            th_d = theta_est.detach().to(dev, torch.float32).reshape(-1, spec.n_params).contiguous()
        else:
            th = np.ascontiguousarray(np.atleast_2d(theta_est), dtype=np.float32)
            th_d = torch.from_numpy(th).to(dev)
        F = th_d.shape[0]
        ys_d, ycon_d, Tu_d, U, T = _device_inputs(torch, struct, dev)
        seeds_d = torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).copy()).to(dev)
        unit_d = None
        if unit_f is not None:
            unit_d = torch.from_numpy(np.asarray(unit_f, dtype=np.int32)).to(dev)
        self.out = {"value": torch.zeros(F, dtype=torch.float64, device=dev),
                    "grad": torch.zeros(F, spec.n_params, dtype=torch.float64, device=dev)}
        if save_ancestors:
            self.out["anc"] = torch.zeros(F, T, J, dtype=torch.int32, device=dev)
        inj = {}
        flags = (_ffi.F_NATURAL if natural else 0) | (_ffi.F_GRAPH if graph else 0)
        if not persistent:
            flags |= _ffi.F_NO_PERSIST
        pwi = -1
        if process_weight_index is not None:
            pwi = int(process_weight_index)
            if not 0 <= pwi < spec.dx:
                raise ValueError(f"process_weight_index must be a state index in [0, {spec.dx})")
            flags |= _ffi.F_DPOP
        if inject is not None:
            flags |= _ffi.F_INJECT
            for k in ("z0", "z", "u"):
                if inject.get(k) is not None:
                    inj[k] = torch.from_numpy(np.ascontiguousarray(inject[k], dtype=np.float32)).to(dev)
        d = _ffi.MopDesc()
        d.model = spec.ffi_model()
        d.J, d.F, d.T, d.U = J, F, T, U
        d.flags = flags
        d.alpha = float(alpha)
        d.ckpt_every = int(ckpt_every)
        d.theta, d.ys, d.ycon = _ffi.ptr(th_d), _ffi.ptr(ys_d), _ffi.ptr(ycon_d)
        d.unit, d.T_u, d.seeds = _ffi.ptr(unit_d), _ffi.ptr(Tu_d), _ffi.ptr(seeds_d)
        d.inj_z0, d.inj_z, d.inj_u = _ffi.ptr(inj.get("z0")), _ffi.ptr(inj.get("z")), _ffi.ptr(inj.get("u"))
        d.value, d.anc = _ffi.ptr(self.out["value"]), _ffi.ptr(self.out.get("anc"))
        d.process_weight_index = pwi
        nbytes = _ffi.LIB.ppf_mop_workspace_bytes(d)
        self.ws = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
        d.workspace, d.ws_bytes = _ffi.ptr(self.ws), self.ws.numel()
        self.d = d
        self.keep = (th_d, ys_d, ycon_d, Tu_d, seeds_d, unit_d, inj)
        self.forward_done = False

    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def update(self, theta_est, seeds_f) -> None:
        """New parameters and keys of the same shape, copied into this call's
        device buffers: the descriptor stays byte-identical, so with ``graph``
        the next forward replays the captured launch sequence on them.  (A call
        built on a CUDA tensor reads that tensor, so this writes into it.)"""
        torch = self.torch
        th_d, seeds_d = self.keep[0], self.keep[4]
        if hasattr(theta_est, "is_cuda"):
            th_d.copy_(theta_est.detach().reshape(th_d.shape))
        else:
            th_d.copy_(torch.from_numpy(np.ascontiguousarray(theta_est, dtype=np.float32).reshape(th_d.shape)))
        seeds_d.copy_(torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).reshape(-1).copy()))
        self.forward_done = False

    def launch(self, grad: bool, err_acc) -> None:
        """``ppf_mop`` queued on the stream without waiting; the workspace's
        status word is OR-ed into the device flag ``err_acc`` (int32)."""
        d = self.d
        d.grad = _ffi.ptr(self.out["grad"]) if grad else 0
        _ffi.check(_ffi.LIB.ppf_mop(d, self._stream()), "ppf_mop")
        err_acc.bitwise_or_(self.ws[:4].view(self.torch.int32))
        self.forward_done = True

    def forward(self, grad: bool = False) -> dict:
        d = self.d
        d.grad = _ffi.ptr(self.out["grad"]) if grad else 0
        stream = self._stream()
        _ffi.check(_ffi.LIB.ppf_mop(d, stream), "ppf_mop")
        _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_mop")
        self.forward_done = True
        return self.out

    def backward(self, dvalue=None):
        if not self.forward_done:
            raise RuntimeError("MopCall.backward needs a forward pass on the same workspace first")
        d = self.d
        d.grad = _ffi.ptr(self.out["grad"])
        dv = None
        if dvalue is not None:
            dv = self.torch.as_tensor(dvalue, dtype=self.torch.float64, device=self.dev).reshape(-1).contiguous()
        stream = self._stream()
        _ffi.check(_ffi.LIB.ppf_mop_backward(d, _ffi.ptr(dv), stream), "ppf_mop_backward")
        _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_mop_backward")
        return self.out["grad"]


def run_mop(struct: PompStruct, theta_est_f: np.ndarray, seeds_f: np.ndarray, J: int, alpha: float,
            *, grad: bool = True, unit_f=None, inject=None, ckpt_every: int = 0,
            save_ancestors: bool = False, return_torch: bool = False, persistent: bool = True,
            process_weight_index: int | None = None):
    """One batched call of ``ppf_mop``: MOP-alpha value (negative log-likelihood,
    summed over time) and, when ``grad``, its gradient on the estimation scale.
    ``persistent=False`` keeps one launch per step where the library would use
    its persistent form (same results; for comparisons).  With
    ``process_weight_index`` the objective is DPOP's (``PPF_F_DPOP``): same
    value, gradient with the transition log-weight held in that state
    component."""
    call = MopCall(struct, theta_est_f, seeds_f, J, alpha, unit_f=unit_f, inject=inject,
                   ckpt_every=ckpt_every, save_ancestors=save_ancestors, persistent=persistent,
                   process_weight_index=process_weight_index)
    out = dict(call.forward(grad=grad))
    if not grad:
        out.pop("grad")
    if return_torch:
        return out
    return {k: v.cpu().numpy() for k, v in out.items()}


def mop(struct: PompStruct, thetas_array, J: int, alpha: float, keys) -> np.ndarray:
    """MOP-alpha negative log-likelihood (``pypomp/functional/mop.py:8-62``).

    ``thetas_array`` (n, P) on the estimation scale, ``keys`` (n,).
    """
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float32))
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != th.shape[0]:
        raise ValueError("keys must have one key per parameter set")
    return run_mop(struct, th, keys, J, alpha, grad=False)["value"]


def mop_value_and_grad(struct: PompStruct, thetas_array, J: int, alpha: float, keys, mean: bool = True):
    """Value and gradient of the (mean) MOP objective
    (``pypomp/core/algorithms/ad_helpers.py:32-54`` ``_jvg_mop``): with
    ``mean`` both are divided by the series length as ``_mop_internal_mean``
    does (``mop.py:148-158``)."""
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float32))
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    res = run_mop(struct, th, keys, J, alpha, grad=True)
    T = np.asarray(struct.ys).shape[-2]
    scale = 1.0 / T if mean else 1.0
    return res["value"] * scale, res["grad"] * scale


def dpop(struct: PompStruct, thetas_array, J: int, alpha: float, process_weight_index: int,
         keys) -> np.ndarray:
    """DPOP negative log-likelihood (``pypomp/functional/dpop.py:13-90`` ->
    ``_dpop_internal``, ``pypomp/core/algorithms/dpop.py:34-134``).

    ``thetas_array`` (n, P) on the estimation scale, ``keys`` (n,).  DPOP adds
    the transition log-weight held in state component ``process_weight_index``
    to the carried weights as ``pw - stop_gradient(pw)``: its value is zero,
    so the objective's value equals MOP-alpha's with the same draws; only its
    gradient differs (:func:`dpop_value_and_grad`).  Experimental in the
    reference, which warns; so does this function."""
    import warnings

    warnings.warn("dpop is experimental and its API and behavior are subject to change.",
                  category=FutureWarning, stacklevel=2)
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float32))
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != th.shape[0]:
        raise ValueError("keys must have one key per parameter set")
    return run_mop(struct, th, keys, J, alpha, grad=False, process_weight_index=process_weight_index)["value"]


def dpop_value_and_grad(struct: PompStruct, thetas_array, J: int, alpha: float, process_weight_index: int,
                        keys, mean: bool = True):
    """Value and gradient of the (mean) DPOP objective, the
    ``jax.value_and_grad(_dpop_internal_mean)`` of
    ``pypomp/core/algorithms/train_dpop.py:130-146``: one ``ppf_mop`` call with
    ``PPF_F_DPOP`` (forward and adjoint) for all n parameter sets."""
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float32))
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    res = run_mop(struct, th, keys, J, alpha, grad=True, process_weight_index=process_weight_index)
    T = np.asarray(struct.ys).shape[-2]
    scale = 1.0 / T if mean else 1.0
    return res["value"] * scale, res["grad"] * scale


def dpop_train(struct: PompStruct, thetas_array, J: int, optimizer, M: int, eta, alpha: float,
               process_weight_index: int, keys, alpha_cooling: float = 1.0, thresh: float = 0.0,
               n_monitors: int = 1):
    """DPOP gradient training (``pypomp/functional/dpop.py:93-185`` ->
    ``_dpop_train_internal``, ``pypomp/core/algorithms/train_dpop.py:118-227``).

    ``thetas_array`` (n, P) on the estimation scale, ``keys`` (n,).  Iteration
    m splits the key, cools alpha (cosine, ``alpha_cooling``), takes the mean
    DPOP objective's value and gradient in one batched ``ppf_mop`` call,
    replaces NaN gradient entries by 0, clips elementwise (``clip_norm``),
    takes the optimiser's step (scaled to unit norm with ``scale``) and moves
    ``theta += eta[m] * direction``.  After the M steps one more split gives
    the key of the final objective at the last parameters.  Returns
    ``(neg_logliks (n, M+1), thetas (n, M+1, P))``: entry m < M is the total
    negative DPOP log-likelihood at the parameters before step m, entry M the
    one at the final parameters.  ``thresh`` and ``n_monitors`` are accepted
    for the reference's signature and, as there, unused.  First-order
    optimisers only (the reference's scan passes no Hessian)."""
    import warnings

    from . import random as pprandom
    from .optim import LearningRate, cosine_alpha

    warnings.warn("dpop_train is experimental and its API and behavior are subject to change.",
                  category=FutureWarning, stacklevel=2)
    if getattr(optimizer, "needs_hessian", False):
        raise ValueError(f"Optimizer '{optimizer.__class__.__name__}' needs a Hessian; dpop_train "
                         "supports first-order optimizers")
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float64)).copy()
    n, P = th.shape
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != n:
        raise ValueError("keys must have one key per parameter set")
    names = list(struct.spec.param_names)
    eta_arr = eta.to_array(names, M) if isinstance(eta, LearningRate) else np.broadcast_to(
        np.asarray(eta, dtype=np.float64), (max(M, 1), P))
    T = np.asarray(struct.ys).shape[-2]
    state = optimizer.init_state(th)
    nll = np.zeros((n, M + 1))
    traces = np.zeros((n, M + 1, P))
    traces[:, 0] = th
    chain = [int(k) for k in keys]

    def split_all():
        subs = np.zeros(n, np.uint64)
        for i in range(n):
            chain[i], subs[i] = (int(v) for v in pprandom.split(chain[i]))
        return subs

    alphas = [1.0 - (1.0 - alpha) * cosine_alpha(m, M, alpha_cooling) for m in range(M + 1)]
    reuse = len(set(alphas)) == 1
    call = None
    for m in range(M):
        subs = split_all()
        if reuse and call is not None:
            call.update(th.astype(np.float32), subs)
        else:
            call = MopCall(struct, th.astype(np.float32), subs, J, alphas[m], graph=reuse,
                           process_weight_index=process_weight_index)
        res = {k: v.cpu().numpy() for k, v in call.forward(grad=True).items()}
        nll[:, m] = res["value"]
        grad = np.where(np.isnan(res["grad"]), 0.0, res["grad"] / T)
        if optimizer.clip_norm is not None:
            grad = np.clip(grad, -optimizer.clip_norm, optimizer.clip_norm)
        direction, state = optimizer.step(grad, state, m, eta_i=eta_arr[m])
        if optimizer.scale:
            direction = direction / np.maximum(np.linalg.norm(direction, axis=-1, keepdims=True), 1e-8)
        th = th + eta_arr[m] * direction
        traces[:, m + 1] = th
    subs = split_all()
    nll[:, M] = run_mop(struct, th.astype(np.float32), subs, J, alphas[M], grad=False,
                        process_weight_index=process_weight_index)["value"]
    return nll, traces


def _warn_nonfinite(grad, m: int) -> None:
    """The reference applies a MOP gradient as it comes (its clip is
    elementwise, ``train.py:115-116``, and lets NaN through), so a gradient
    that overflowed float32 -- as pathwise derivatives along chaotic
    trajectories do over long series -- turns the parameters into NaN.  Same
    semantics here, but the caller is told."""
    bad = ~np.isfinite(np.asarray(grad))
    if bad.any():
        import warnings

        rows = np.unique(np.nonzero(bad.reshape(bad.shape[0], -1))[0]) if bad.ndim > 1 else [0]
        warnings.warn(f"train iteration {m}: non-finite MOP gradient entries ({int(bad.sum())}) in "
                      f"{len(rows)} parameter set(s); the update propagates them, as the reference does",
                      RuntimeWarning, stacklevel=3)


def train(struct: PompStruct, thetas_array, J: int, optimizer, M: int, eta, alpha: float, keys,
          alpha_cooling: float = 1.0, thresh: float = 0.0, n_monitors: int = 1, *, device_loop: bool = True):
    """MOP-alpha gradient training (``pypomp/functional/train.py:14-110`` /
    ``_train_internal``, ``train.py:38-180``).

    ``thetas_array`` (n, P) on the estimation scale, ``keys`` (n,).  Each
    iteration: cosine-cooled alpha (``train.py:82-85``), one batched MOP value
    and gradient for all n parameter sets (the gradient of the mean objective,
    ``_mop_internal_mean``), optional clipping, the optimiser step and
    ``theta += eta[m] * direction``.  The recorded negative log-likelihood is
    the MOP value at the current parameters (n_monitors == 1) or the mean of
    ``n_monitors`` particle filters (n_monitors > 1; NaN for 0).  Returns
    ``(neg_logliks (n, M+1), thetas (n, M+1, P))`` with a NaN first entry.

    ``optimizer.ls`` replaces the fixed step by the reference's Armijo
    backtracking (``train.py:442-500``, :func:`_line_search`) on the particle
    filter's negative log-likelihood under the iteration's MOP key.  Newton and
    WeightedNewton get the Hessian of the mean MOP objective as central
    differences of its gradient under the iteration's Hessian key (common
    random numbers), all 2P perturbed gradients of all parameter sets in one
    batched launch (:func:`mop_hessian_fd`).

    SGD and Adam without line search and with at most one monitor run the
    loop on the device side (:func:`_train_device`); ``device_loop=False``
    keeps the host loop (same results).
    """
    from . import random as pprandom
    from .optim import LearningRate, cosine_alpha

    from .optim import BFGS, SGD, Adam, FullMatrixAdam, Newton, WeightedNewton

    if n_monitors < 1 and optimizer.ls:
        raise ValueError("Line search requires at least one monitor")
    if not isinstance(optimizer, (SGD, Adam, FullMatrixAdam, Newton, WeightedNewton, BFGS)):
        raise ValueError(f"Optimizer '{optimizer.__class__.__name__}' not supported")
    if device_loop and type(optimizer) in (SGD, Adam) and not optimizer.ls and n_monitors <= 1 and M > 0:
        return _train_device(struct, thetas_array, J, optimizer, M, eta, alpha, keys, alpha_cooling, n_monitors)
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float64)).copy()
    n, P = th.shape
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != n:
        raise ValueError("keys must have one key per parameter set")
    names = list(struct.spec.param_names)
    eta_arr = eta.to_array(names, M) if isinstance(eta, LearningRate) else np.broadcast_to(
        np.asarray(eta, dtype=np.float64), (max(M, 1), P))
    T = np.asarray(struct.ys).shape[-2]
    state = optimizer.init_state(th)
    nll = np.full((n, M + 1), np.nan)
    traces = np.zeros((n, M + 1, P))
    traces[:, 0] = th
    chain = [int(k) for k in keys]
    alphas = [1.0 - (1.0 - alpha) * cosine_alpha(m, M, alpha_cooling) for m in range(M)]
    # with one alpha for the whole run every step reuses one MOP call (its
    # buffers, workspace and captured launch sequence)
    reuse = len(set(alphas)) == 1
    call = None
    for m in range(M):
        alpha_m = alphas[m]
        subs = np.zeros(n, np.uint64)
        for i in range(n):
            chain[i], subs[i] = (int(v) for v in pprandom.split(chain[i]))
        if reuse and call is not None:
            call.update(th.astype(np.float32), subs)
        else:
            call = MopCall(struct, th.astype(np.float32), subs, J, alpha_m, graph=reuse)
        res = {k: v.cpu().numpy() for k, v in call.forward(grad=True).items()}
        grad = res["grad"] / T
        if n_monitors == 1:
            nll[:, m + 1] = res["value"]
        elif n_monitors > 1:
            mon = np.zeros((n, n_monitors), np.uint64)
            for i in range(n):
                ks = pprandom.split(chain[i], n_monitors + 1)
                chain[i] = int(ks[0])
                mon[i] = ks[1:]
            pf = run_pfilter(struct, np.repeat(th.astype(np.float32), n_monitors, axis=0),
                             mon.reshape(-1), J, thresh=thresh, est=True)
            nll[:, m + 1] = -pf["loglik"].reshape(n, n_monitors).mean(axis=1)
        hkeys = np.zeros(n, np.uint64)
        for i in range(n):
            chain[i], hkeys[i] = (int(v) for v in pprandom.split(chain[i]))
        _warn_nonfinite(grad, m)
        if optimizer.clip_norm is not None:
            grad = np.clip(grad, -optimizer.clip_norm, optimizer.clip_norm)
        hess_fn = (lambda: mop_hessian_fd(struct, th, hkeys, J, alpha_m)) if optimizer.needs_hessian else None
        direction, state = optimizer.step(grad, state, m, compute_hessian_fn=hess_fn, eta_i=eta_arr[m])
        if optimizer.scale:
            direction = direction / np.linalg.norm(direction, axis=-1, keepdims=True)
        if optimizer.ls:
            step = _line_search(struct, th, subs, J, thresh, nll[:, m + 1], grad, direction,
                                float(np.mean(eta_arr[m])), optimizer.max_ls_itn, optimizer.c, 0.5)
            th = th + step[:, None] * direction
        else:
            th = th + eta_arr[m] * direction
        traces[:, m + 1] = th
    return nll, traces


def _train_device(struct: PompStruct, thetas_array, J: int, optimizer, M: int, eta, alpha: float, keys,
                  alpha_cooling: float, n_monitors: int):
    """:func:`train` for SGD / Adam without line search and with at most one
    monitor, with the loop on the device side: the parameters, optimiser
    state, learning rates, keys and traces stay in device memory, each
    iteration's MOP value + gradient (one ``ppf_mop`` call, its launch
    sequence replayed from a CUDA graph when alpha is constant), clipping and
    update are queued on the stream, and the host synchronises once at the
    end.  The keys come from the same splits as the host loop and every update
    is the same float64 arithmetic, so the results are the host loop's."""
    from . import random as pprandom
    from .optim import LearningRate, cosine_alpha

    torch = _ffi.require_cuda()
    th = np.atleast_2d(np.asarray(thetas_array, dtype=np.float64)).copy()
    n, P = th.shape
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != n:
        raise ValueError("keys must have one key per parameter set")
    names = list(struct.spec.param_names)
    eta_arr = eta.to_array(names, M) if isinstance(eta, LearningRate) else np.broadcast_to(
        np.asarray(eta, dtype=np.float64), (max(M, 1), P))
    T = np.asarray(struct.ys).shape[-2]
    dev = torch.device("cuda", torch.cuda.current_device())
    # the key chain of the host loop: per iteration one split for the MOP key,
    # one for the (unused) Hessian key
    chain = [int(k) for k in keys]
    subs = np.zeros((M, n), np.uint64)
    for m in range(M):
        for i in range(n):
            chain[i], subs[m, i] = (int(v) for v in pprandom.split(chain[i]))
            chain[i], _ = (int(v) for v in pprandom.split(chain[i]))
    alphas = [1.0 - (1.0 - alpha) * cosine_alpha(m, M, alpha_cooling) for m in range(M)]
    reuse = len(set(alphas)) == 1
    th_d = torch.tensor(th, dtype=torch.float64, device=dev)
    subs_d = torch.from_numpy(subs.view(np.int64)).to(dev)
    eta_d = torch.tensor(np.ascontiguousarray(eta_arr[:M]), dtype=torch.float64, device=dev)
    nll_d = torch.full((n, M + 1), float("nan"), dtype=torch.float64, device=dev)
    tr_d = torch.zeros(n, M + 1, P, dtype=torch.float64, device=dev)
    tr_d[:, 0] = th_d
    bad = torch.zeros(1, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    T_d = torch.tensor(float(T), dtype=torch.float64, device=dev)
    call = MopCall(struct, th.astype(np.float32), subs[0], J, alphas[0], graph=reuse)
    th32_d, seeds_d = call.keep[0], call.keep[4]
    state = optimizer.init_state_device(th_d) if hasattr(optimizer, "init_state_device") else ()
    for m in range(M):
        th32_d.copy_(th_d)
        seeds_d.copy_(subs_d[m])
        call.d.alpha = float(alphas[m])
        call.launch(True, err)
        grad = call.out["grad"] / T_d     # a device divisor: true division, as on the host
        if n_monitors == 1:
            nll_d[:, m + 1] = call.out["value"]
        bad += (~torch.isfinite(grad)).sum()
        if optimizer.clip_norm is not None:
            grad = grad.clamp(-optimizer.clip_norm, optimizer.clip_norm)
        direction, state = optimizer.step_device(grad, state, m)
        if optimizer.scale:
            direction = direction / (direction * direction).sum(dim=-1, keepdim=True).sqrt()
        th_d = th_d + eta_d[m] * direction
        tr_d[:, m + 1] = th_d
    e = int(err.item())
    if e:
        _ffi.check(_ffi.PPF_ETIMEOUT if e & 1 else _ffi.PPF_EINTERNAL, "ppf_mop")
    nbad = int(bad.item())
    if nbad:
        import warnings

        warnings.warn(f"train: {nbad} non-finite MOP gradient entries over {M} iterations; the updates "
                      "propagate them, as the reference does", RuntimeWarning, stacklevel=3)
    return nll_d.cpu().numpy(), tr_d.cpu().numpy()


def mop_hessian_fd(struct: PompStruct, theta_est, keys, J: int, alpha: float, h: float = 1e-2):
    """Hessian of the mean MOP-alpha objective at each row of ``theta_est``
    (n, P) by central differences of its gradient, h_j = h max(1, |theta_j|),
    every perturbed point under its row's key (common random numbers):
    one ``ppf_mop`` launch of 2 n P filters.  Returns (n, P, P), symmetrised.
    (The reference differentiates its estimator twice with jax.hessian,
    ``ad_helpers.py``; there is no second-order adjoint kernel here.)  The
    estimator's gradient jumps where a perturbation moves a resampling
    boundary, so a small h amplifies those jumps; h = 1e-2 averages over them
    (on LG 1-D with J = 1e5 the diagonal lands within 0.8-1.5x of the exact
    Kalman Hessian; at h = 1e-3 it is dominated by the jumps)."""
    th = np.atleast_2d(np.asarray(theta_est, dtype=np.float64))
    n, P = th.shape
    T = np.asarray(struct.ys).shape[-2]
    step = h * np.maximum(1.0, np.abs(th))                       # (n, P)
    pts = np.repeat(th[:, None, None, :], 2, axis=1).repeat(P, axis=2)   # (n, 2, P, P)
    idx = np.arange(P)
    pts[:, 0, idx, idx] += step
    pts[:, 1, idx, idx] -= step
    seeds = np.repeat(np.asarray(keys, dtype=np.uint64).reshape(n), 2 * P)
    res = run_mop(struct, pts.reshape(-1, P).astype(np.float32), seeds, J, alpha, grad=True)
    g = res["grad"].reshape(n, 2, P, P) / T
    H = (g[:, 0] - g[:, 1]) / (2.0 * step[:, :, None])           # H[i, j, :] = d grad / d theta_j
    return 0.5 * (H + np.swapaxes(H, 1, 2))


def _line_search(struct, th, keys, J, thresh, curr_obj, grad, direction, eta0, tau, c, frac):
    """Armijo backtracking of every row at once (``train.py:442-500``, stoch=False):
    evaluate the particle filter's negative log-likelihood at
    theta + eta direction under the row's key; while it exceeds
    curr + eta c <grad, direction> (or is NaN) and fewer than tau reductions
    were made, eta *= frac.  Rows still searching share one batched launch
    per round."""
    n = th.shape[0]
    eta = np.full(n, eta0)
    itn = np.zeros(n, np.int64)
    active = np.ones(n, bool)
    slope = np.sum(grad * direction, axis=-1)
    keys = np.asarray(keys, dtype=np.uint64).reshape(n)
    while active.any():
        rows = np.nonzero(active)[0]
        pts = th[rows] + eta[rows, None] * direction[rows]
        res = run_pfilter(struct, pts.astype(np.float32), keys[rows], J, thresh=thresh, est=True)
        nxt = -res["loglik"]
        with np.errstate(invalid="ignore"):
            cont = (nxt > curr_obj[rows] + eta[rows] * c * slope[rows]) | np.isnan(nxt)
        more = cont & (itn[rows] < tau)
        eta[rows] = np.where(more, eta[rows] * frac, eta[rows])
        itn[rows] += 1
        active[rows] = more
    return eta


# ---------------------------------------------------------------------------
# IF2
# ---------------------------------------------------------------------------


def run_perfilter(struct: PompStruct, swarm, seeds_f: np.ndarray, J: int, rw_sig, rw_sig0, cool, cool0,
                  *, thresh: float = 0.0, unit_f=None, inject=None, CLL: bool = False,
                  save_ancestors: bool = False, natural: bool = False, stream_only: bool = False):
    """One batched call of ``ppf_perfilter``: one IF2 iteration over F swarms.

    ``swarm`` is either a CUDA tensor (F, P, J) on the estimation scale (kept
    on the device; the result swarm comes back the same way) or a host array
    (F, J, P).  ``cool`` (T,) or (U, T) and ``cool0`` (scalar or (U,)) are the
    cooling factors of the step and t0 perturbations.  ``inject`` optionally
    holds host arrays ``zp0`` (F,J,P), ``zp`` (F,T,J,P), ``z0``, ``z``, ``u``
    replacing the Philox draws.  ``natural`` hands the kernels natural-scale
    parameters (``PPF_F_NATURAL``: no transform inside the mechanics);
    ``stream_only`` keeps the streaming kernels where few small swarms would
    otherwise run cluster-resident (``PPF_F_NO_CLUSTER``).
    Returns a dict with ``loglik`` (F,), ``swarm`` and optionally ``cll`` /
    ``anc``.
    """
    torch = _ffi.require_cuda()
    if J < 1:
        raise ValueError("J should be greater than 0.")
    if J > _ffi.PPF_MAX_J:
        raise ValueError(f"J must be at most {_ffi.PPF_MAX_J}.")
    dev = torch.device("cuda", torch.cuda.current_device())
    spec = struct.spec
    P = spec.n_params
    device_swarm = hasattr(swarm, "is_cuda")
    if device_swarm:
        sw_d = swarm.to(dev, torch.float32).contiguous()
        F = sw_d.shape[0]
    else:
        sw = np.asarray(swarm, dtype=np.float32)
        F = sw.shape[0]
        sw_d = torch.from_numpy(np.ascontiguousarray(sw.transpose(0, 2, 1))).to(dev)
    if tuple(sw_d.shape) != (F, P, J):
        raise ValueError(f"swarm must hold {P} parameters of {J} particles per filter")
    ys_d, ycon_d, Tu_d, U, T = _device_inputs(torch, struct, dev)
    cool_h = np.array(np.broadcast_to(np.asarray(cool, np.float32), (U, T)), dtype=np.float32)
    cool0_h = np.array(np.broadcast_to(np.asarray(cool0, np.float32), (U,)), dtype=np.float32)
    f32d = dict(dtype=torch.float32, device=dev)
    keep = {
        "rw_sig": torch.tensor(np.asarray(rw_sig, np.float32), **f32d),
        "rw_sig0": torch.tensor(np.asarray(rw_sig0, np.float32), **f32d),
        "cool": torch.from_numpy(cool_h).to(dev),
        "cool0": torch.from_numpy(cool0_h).to(dev),
        "seeds": torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).copy()).to(dev),
    }
    unit_d = None
    if unit_f is not None:
        unit_d = torch.from_numpy(np.asarray(unit_f, dtype=np.int32)).to(dev)
    out = {"loglik": torch.zeros(F, dtype=torch.float64, device=dev),
           "swarm": torch.empty(F, P, J, **f32d)}
    flags = (_ffi.F_NATURAL if natural else 0) | (_ffi.F_NO_CLUSTER if stream_only else 0)
    if CLL:
        flags |= _ffi.F_CLL
        out["cll"] = torch.zeros(F, T, dtype=torch.float64, device=dev)
    if save_ancestors:
        flags |= _ffi.F_SAVE_ANC
        out["anc"] = torch.zeros(F, T, J, dtype=torch.int32, device=dev)
    inj = {}
    if inject is not None:
        flags |= _ffi.F_INJECT
        for k in ("zp0", "zp", "z0", "z", "u"):
            if inject.get(k) is not None:
                inj[k] = torch.from_numpy(np.ascontiguousarray(inject[k], dtype=np.float32)).to(dev)
    d = _ffi.PerfilterDesc()
    d.model = spec.ffi_model()
    d.J, d.F, d.T, d.U = J, F, T, U
    d.flags = flags
    d.thresh = float(max(0.0, thresh))
    d.swarm_in, d.swarm_out = _ffi.ptr(sw_d), _ffi.ptr(out["swarm"])
    d.rw_sig, d.rw_sig0 = _ffi.ptr(keep["rw_sig"]), _ffi.ptr(keep["rw_sig0"])
    d.cool, d.cool0 = _ffi.ptr(keep["cool"]), _ffi.ptr(keep["cool0"])
    d.ys, d.ycon, d.unit, d.T_u = _ffi.ptr(ys_d), _ffi.ptr(ycon_d), _ffi.ptr(unit_d), _ffi.ptr(Tu_d)
    d.seeds = _ffi.ptr(keep["seeds"])
    for k in ("zp0", "zp", "z0", "z", "u"):
        setattr(d, "inj_" + k, _ffi.ptr(inj.get(k)))
    d.loglik, d.cll, d.anc = _ffi.ptr(out["loglik"]), _ffi.ptr(out.get("cll")), _ffi.ptr(out.get("anc"))
    nbytes = _ffi.LIB.ppf_perfilter_workspace_bytes(d)
    ws = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    stream = torch.cuda.current_stream(dev).cuda_stream
    _ffi.check(_ffi.LIB.ppf_perfilter(d, stream), "ppf_perfilter")
    _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_perfilter")
    if device_swarm:
        return out
    res = {k: v.cpu().numpy() for k, v in out.items() if k != "swarm"}
    res["swarm"] = out["swarm"].cpu().numpy().transpose(0, 2, 1).copy()
    return res


class PerfilterCall:
    """The iterations of one IF2 run on the device.  Two swarm buffers are used
    in turn (iteration m reads one and writes the other), and the keys,
    cooling factors, log-likelihoods and workspace stay allocated; a call
    copies its keys and cooling factors into the same buffers.  With ``graph``
    each buffer direction's launch sequence is captured into a CUDA graph on
    first use (``PPF_F_GRAPH``) and replayed afterwards.  Measured on Ricker
    (T = 500) the graph did not pay for IF2, whose kernels dominate (J = 32768
    x 8: 17-20 ms per iteration either way), so ``mif`` leaves it off; the
    persistent buffers alone save 5-8 % against separate calls."""

    def __init__(self, struct: PompStruct, swarm, J: int, rw_sig, rw_sig0, *, thresh: float = 0.0,
                 graph: bool = False, unit_f=None):
        torch = _ffi.require_cuda()
        self.torch = torch
        dev = torch.device("cuda", torch.cuda.current_device())
        spec = struct.spec
        P = spec.n_params
        first = swarm.to(dev, torch.float32).contiguous()
        F = first.shape[0]
        if tuple(first.shape) != (F, P, J):
            raise ValueError(f"swarm must hold {P} parameters of {J} particles per filter")
        ys_d, ycon_d, Tu_d, U, T = _device_inputs(torch, struct, dev)
        f32d = dict(dtype=torch.float32, device=dev)
        self.U, self.T = U, T
        self.swarms = [first.clone(), torch.empty_like(first)]
        self.seeds = torch.zeros(F, dtype=torch.int64, device=dev)
        self.cool = torch.zeros(U, T, **f32d)
        self.cool0 = torch.zeros(U, **f32d)
        self.ll = torch.zeros(F, dtype=torch.float64, device=dev)
        unit_d = None if unit_f is None else torch.from_numpy(np.asarray(unit_f, dtype=np.int32)).to(dev)
        self.keep = [ys_d, ycon_d, Tu_d, torch.tensor(np.asarray(rw_sig, np.float32), **f32d),
                     torch.tensor(np.asarray(rw_sig0, np.float32), **f32d), unit_d]
        self.descs = []
        self.ws = None
        for i in (0, 1):
            d = _ffi.PerfilterDesc()
            d.model = spec.ffi_model()
            d.J, d.F, d.T, d.U = J, F, T, U
            d.flags = _ffi.F_GRAPH if graph else 0
            d.thresh = float(max(0.0, thresh))
            d.swarm_in, d.swarm_out = _ffi.ptr(self.swarms[i]), _ffi.ptr(self.swarms[1 - i])
            d.rw_sig, d.rw_sig0 = _ffi.ptr(self.keep[3]), _ffi.ptr(self.keep[4])
            d.cool, d.cool0 = _ffi.ptr(self.cool), _ffi.ptr(self.cool0)
            d.ys, d.ycon, d.T_u = _ffi.ptr(ys_d), _ffi.ptr(ycon_d), _ffi.ptr(Tu_d)
            d.unit = _ffi.ptr(unit_d)
            d.seeds, d.loglik = _ffi.ptr(self.seeds), _ffi.ptr(self.ll)
            if self.ws is None:
                self.ws = torch.empty(max(int(_ffi.LIB.ppf_perfilter_workspace_bytes(d)), 256),
                                      dtype=torch.uint8, device=dev)
            d.workspace, d.ws_bytes = _ffi.ptr(self.ws), self.ws.numel()
            self.descs.append(d)
        self.cur = 0
        self.stream = torch.cuda.current_stream(dev).cuda_stream

    @property
    def swarm(self):
        """The current swarm (F, P, J), estimation scale."""
        return self.swarms[self.cur]

    def run_device(self, seeds_d, cool_d, err_acc) -> None:
        """One iteration from device-resident keys (F,) int64 and cooling
        factors (U, T): the copies and the launch are queued on the stream and
        the host does not wait; the workspace's status word is OR-ed into the
        device flag ``err_acc`` (int32) for one check after the loop."""
        self.seeds.copy_(seeds_d)
        self.cool.copy_(cool_d)
        self.cool0.copy_(cool_d[:, 0])
        d = self.descs[self.cur]
        _ffi.check(_ffi.LIB.ppf_perfilter(d, self.stream), "ppf_perfilter")
        err_acc.bitwise_or_(self.ws[:4].view(self.torch.int32))
        self.cur ^= 1

    def __call__(self, seeds_f, cool, cool0) -> np.ndarray:
        torch = self.torch
        self.seeds.copy_(torch.from_numpy(np.asarray(seeds_f, dtype=np.uint64).view(np.int64).copy()))
        self.cool.copy_(torch.from_numpy(np.array(np.broadcast_to(np.asarray(cool, np.float32),
                                                                  (self.U, self.T)), dtype=np.float32)))
        self.cool0.copy_(torch.from_numpy(np.array(np.broadcast_to(np.asarray(cool0, np.float32), (self.U,)),
                                                   dtype=np.float32)))
        d = self.descs[self.cur]
        _ffi.check(_ffi.LIB.ppf_perfilter(d, self.stream), "ppf_perfilter")
        _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, self.stream), "ppf_perfilter")
        self.cur ^= 1
        return self.ll.cpu().numpy().copy()


def mif(struct: PompStruct, thetas_array, rw_sd, M: int, J: int, keys, thresh: float = 0.0,
        n_monitors: int = 0, *, inject=None, device_loop: bool = True):
    """Iterated filtering 2 (``pypomp/functional/mif.py:15-122``,
    ``_mif_internal`` / ``_mif_scan_body`` at ``pypomp/core/algorithms/mif.py:16-85``).

    ``thetas_array`` (n_reps, J, P) starting swarms on the natural scale,
    ``rw_sd`` an :class:`~pypomp_b200.optim.RWSigma`, ``keys`` (n_reps,).
    Each iteration m runs one perturbed filter per replicate (all replicates
    in one ``ppf_perfilter`` call, swarms resident on the GPU) with cooling
    factors ``rw_sd.cooling_factor(t, m, T)``; with ``n_monitors`` >= 1 the
    recorded log-likelihood is the mean over ``n_monitors`` unperturbed
    filters at the swarm mean before the iteration (mean of the negative
    log-likelihoods, as the reference averages them), else the perturbed
    filter's.  Key tree per replicate: ``split(key, M+1)[1:]`` iteration keys;
    the monitors use ``split(iteration key, n_monitors)``.  ``inject``
    optionally replays external draws: one dict per iteration with
    ``"perfilter"`` (arrays ``zp0``, ``zp``, ``z0``, ``z``, ``u`` with a
    leading replicate axis) and ``"monitors"`` (a list of ``z0``/``z``/``u``
    dicts, leading replicate axis).  Returns ``(logliks (n_reps, M), traces
    (n_reps, M+1, P), final swarm (n_reps, J, P))``, natural scale.
    Without monitors or injected draws the loop runs on the device side
    (:func:`_mif_device`); ``device_loop=False`` keeps the host loop (same
    results).
    """
    from . import random as pprandom

    torch = _ffi.require_cuda()
    spec = struct.spec
    names = list(spec.param_names)
    th = np.asarray(thetas_array, dtype=np.float32)
    if th.ndim != 3 or th.shape[1] != J or th.shape[2] != len(names):
        raise ValueError(f"thetas_array must have shape (n_reps, {J}, {len(names)})")
    if M < 0:
        raise ValueError("M must be non-negative")
    n = th.shape[0]
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    if keys.shape[0] != n:
        raise ValueError("keys must have one key per replicate")
    rw_sig, rw_sig0 = rw_sd.arrays(names)
    T = np.asarray(struct.ys).shape[-2]
    dev = torch.device("cuda", torch.cuda.current_device())
    est = spec.to_est(th.reshape(-1, len(names))).reshape(th.shape).astype(np.float32)
    swarm = torch.from_numpy(np.ascontiguousarray(est.transpose(0, 2, 1))).to(dev)   # (n, P, J)
    m_keys = np.stack([pprandom.split(k, M + 1)[1:] for k in keys]) if M > 0 else np.zeros((n, 0), np.uint64)
    means = [swarm.mean(dim=2)]
    logliks = np.zeros((n, M))
    if device_loop and inject is None and n_monitors < 1 and M > 0:
        return _mif_device(struct, swarm, rw_sd, rw_sig, rw_sig0, M, J, m_keys, T, thresh)
    # without injected draws the iterations share one set of device buffers
    call = PerfilterCall(struct, swarm, J, rw_sig, rw_sig0, thresh=thresh) if inject is None and M > 0 else None
    for it in range(M):
        cool = np.array([rw_sd.cooling_factor(i, it, T) for i in range(T)], dtype=np.float32)
        inj = inject[it] if inject is not None else None
        if call is not None:
            ll_it = call(m_keys[:, it], cool, cool[0])
            res = {"loglik": ll_it, "swarm": call.swarm}
        else:
            res = run_perfilter(struct, swarm, m_keys[:, it], J, rw_sig, rw_sig0, cool, cool[0], thresh=thresh,
                                inject=None if inj is None else inj["perfilter"])
            res["loglik"] = res["loglik"].cpu().numpy()
        if n_monitors >= 1:
            mean = means[-1].cpu().numpy()
            mon = np.stack([pprandom.split(k, n_monitors) for k in m_keys[:, it]])
            minj = None
            if inj is not None:
                minj = {k: np.stack([np.stack([inj["monitors"][i][k][r] for i in range(n_monitors)])
                                     for r in range(n)]).reshape((n * n_monitors,) + inj["monitors"][0][k].shape[1:])
                        for k in ("z0", "z", "u")}
            pf = run_pfilter(struct, np.repeat(mean, n_monitors, axis=0), mon.reshape(-1), J,
                             thresh=thresh, est=True, inject=minj)
            logliks[:, it] = -(-pf["loglik"].reshape(n, n_monitors)).mean(axis=1)
        else:
            logliks[:, it] = res["loglik"]
        swarm = res["swarm"]
        means.append(swarm.mean(dim=2))
    traces = torch.stack(means, dim=1).cpu().numpy()                       # (n, M+1, P) est
    traces = spec.from_est(traces.reshape(-1, len(names))).reshape(traces.shape)
    final = swarm.cpu().numpy().transpose(0, 2, 1)
    final = spec.from_est(final.reshape(-1, len(names))).reshape(final.shape)
    return logliks, traces, final


def _cooling_rows(rw_sd, m: int, T_u, width: int | None = None, out=None) -> np.ndarray:
    """(U, width) cooling factors of iteration m for every unit and step (zero
    past a unit's length; width defaults to max T_u), written into ``out``
    when given."""
    T_u = np.atleast_1d(np.asarray(T_u, dtype=np.int64))
    if out is None:
        out = np.empty((T_u.size, int(width or T_u.max())), np.float32)
    out.fill(0.0)
    rows = {}                      # units of equal length share their rows
    for u, Tu in enumerate(T_u.tolist()):
        if Tu not in rows:
            rows[Tu] = np.array(rw_sd.cooling_factors(Tu, m), dtype=np.float32)
        out[u, :Tu] = rows[Tu]
    return out


def _cooling_table(rw_sd, M: int, T_u, width: int | None = None) -> np.ndarray:
    """(M, U, width) cooling factors of every iteration, unit and step (zero
    past a unit's length; width defaults to max T_u)."""
    T_u = np.atleast_1d(np.asarray(T_u, dtype=np.int64))
    out = np.zeros((M, T_u.size, int(width or T_u.max())), np.float32)
    for m in range(M):
        _cooling_rows(rw_sd, m, T_u, out=out[m])
    return out


def _mif_device(struct, swarm, rw_sd, rw_sig, rw_sig0, M, J, m_keys, T, thresh):
    """The IF2 iterations of :func:`mif` (no monitors, no injected draws) with
    the loop on the device side: the cooling factors of all M iterations and
    all iteration keys are uploaded once, every iteration's launch, swarm
    means and log-likelihoods are queued on the stream without a host wait,
    and one synchronisation at the end reads the traces and the status.
    Same kernels and inputs as the host loop, so the same results bit for bit."""
    torch = _ffi.require_cuda()
    spec = struct.spec
    names = list(spec.param_names)
    dev = swarm.device
    n = swarm.shape[0]
    call = PerfilterCall(struct, swarm, J, rw_sig, rw_sig0, thresh=thresh)
    cool_d = torch.from_numpy(_cooling_table(rw_sd, M, [T])).to(dev)                 # (M, 1, T)
    keys_d = torch.from_numpy(np.ascontiguousarray(m_keys.T).view(np.int64)).to(dev)  # (M, n)
    ll_d = torch.zeros(M, n, dtype=torch.float64, device=dev)
    means_d = torch.zeros(M + 1, n, spec.n_params, dtype=torch.float32, device=dev)
    means_d[0] = swarm.mean(dim=2)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    for it in range(M):
        call.run_device(keys_d[it], cool_d[it], err)
        ll_d[it].copy_(call.ll)
        means_d[it + 1] = call.swarm.mean(dim=2)
    e = int(err.item())
    if e:
        _ffi.check(_ffi.PPF_ETIMEOUT if e & 1 else _ffi.PPF_EINTERNAL, "ppf_perfilter")
    logliks = ll_d.T.cpu().numpy()
    traces = means_d.transpose(0, 1).cpu().numpy()
    traces = spec.from_est(traces.reshape(-1, len(names))).reshape(traces.shape)
    final = call.swarm.cpu().numpy().transpose(0, 2, 1)
    final = spec.from_est(final.reshape(-1, len(names))).reshape(final.shape)
    return logliks, traces, final


# ---------------------------------------------------------------------------
# Panels
# ---------------------------------------------------------------------------


@dataclass
class PanelPompStruct:
    """What the kernels need from a panel (``pypomp/functional/structs.py:156``).

    Units share one built-in model; their series may have different lengths:
    ``ys`` is (U, Tmax, dy) padded after ``T_u[u]`` observations (the
    reference stacks equal-length units only).  ``permutations[u][i]`` is the
    panel-order index ([shared | unit-specific] names) of the unit model's
    canonical parameter i.
    """

    spec: ModelSpec
    ys: np.ndarray
    T_u: np.ndarray
    times: list
    t0: float
    unit_names: list
    shared_param_names: list
    unit_param_names: list
    permutations: np.ndarray

    @property
    def param_names(self):
        return list(self.shared_param_names) + list(self.unit_param_names)

    @property
    def U(self):
        return len(self.unit_names)

    def all_units(self) -> PompStruct:
        return PompStruct(spec=self.spec, ys=self.ys, times=np.arange(self.ys.shape[1]), t0=self.t0,
                          T_u=np.asarray(self.T_u, np.int32))

    def unit(self, u: int) -> PompStruct:
        T = int(self.T_u[u])
        return PompStruct(spec=self.spec, ys=np.ascontiguousarray(self.ys[u, :T]),
                          times=np.asarray(self.times[u]), t0=self.t0)


def _mask_ragged(arr, T_u, unit_of_row):
    """NaN after each row's own series length (diagnostics of ragged panels)."""
    arr = np.array(arr, dtype=np.float64 if arr.dtype == np.float64 else np.float32, copy=True)
    for i, u in enumerate(unit_of_row):
        arr[i, int(T_u[u]):] = np.nan
    return arr


def panel_pfilter(struct: PanelPompStruct, thetas_array, J: int, keys, thresh: float = 0.0,
                  chunk_size: int = 1, CLL: bool = False, ESS: bool = False, filter_mean: bool = False,
                  prediction_mean: bool = False, *, inject=None) -> dict:
    """Panel particle filter (``pypomp/functional/pfilter.py:93-140``).

    ``thetas_array`` (n_reps, U, P) in each unit's canonical order, natural
    scale; ``keys`` (n_reps, U).  All n_reps x U filters run in one call
    (``chunk_size`` is accepted for signature compatibility; there is nothing
    to chunk).  Returns ``logLik`` (n_reps, U) and the requested diagnostics
    with a (n_reps, U, Tmax[, dx]) layout, NaN after a unit's last observation.
    ``inject`` optionally replays external draws (``run_pfilter``'s arrays
    with a leading n_reps * U filter axis).
    """
    del chunk_size
    th = np.asarray(thetas_array, dtype=np.float32)
    n, U, P = th.shape
    keys = np.asarray(keys, dtype=np.uint64).reshape(n, U)
    unit_f = np.tile(np.arange(U, dtype=np.int32), n)
    res = run_pfilter(struct.all_units(), th.reshape(n * U, P), keys.reshape(-1), J, thresh=thresh,
                      CLL=CLL, ESS=ESS, filter_mean=filter_mean, prediction_mean=prediction_mean,
                      unit_f=unit_f, inject=inject)
    out = {"logLik": res["loglik"].reshape(n, U)}
    for name, key in (("CLL", "cll"), ("ESS", "ess"), ("filter_mean", "fmean"), ("prediction_mean", "pmean")):
        if key in res:
            a = _mask_ragged(res[key], struct.T_u, unit_f)
            out[name] = a.reshape((n, U) + a.shape[1:])
    return out


def _panel_thetas(shared, unit, perms):
    """Unit-order parameters from [shared | unit] panel blocks.

    ``shared`` (..., ns), ``unit`` (..., U, nu) -> (..., U, P) with
    theta_u[i] = panel_u[perms[u][i]]."""
    U = unit.shape[-2]
    sh = np.broadcast_to(shared[..., None, :], shared.shape[:-1] + (U, shared.shape[-1]))
    panel = np.concatenate([sh, unit], axis=-1)
    out = np.empty(panel.shape[:-1] + (perms.shape[1],), dtype=panel.dtype)
    for u in range(U):
        out[..., u, :] = panel[..., u, perms[u]]
    return out


def panel_mop(struct: PanelPompStruct, thetas_array, J: int, alpha: float, keys, grad: bool = False):
    """MOP-alpha values of every (replicate, unit) filter in one call
    (``_panel_mop_internal_vmap``, ``pypomp/core/algorithms/mop.py:161-179``).

    ``thetas_array`` (n, U, P) on the estimation scale, unit order; ``keys``
    (n, U).  Returns value (n, U) and, with ``grad``, d value / d theta
    (n, U, P)."""
    th = np.asarray(thetas_array, dtype=np.float32)
    n, U, P = th.shape
    keys = np.asarray(keys, dtype=np.uint64).reshape(n, U)
    unit_f = np.tile(np.arange(U, dtype=np.int32), n)
    res = run_mop(struct.all_units(), th.reshape(n * U, P), keys.reshape(-1), J, alpha, grad=grad,
                  unit_f=unit_f)
    out = {"value": res["value"].reshape(n, U)}
    if grad:
        out["grad"] = res["grad"].reshape(n, U, P)
    return out


def _perfilter_queued(st_u, unit_in, swarm, seeds_d, J, sig_d, sig0_d, cool_d, thresh, save_anc, ll_out,
                      err_acc, stream):
    """Queue one unit's ``ppf_perfilter`` on device-resident inputs without
    waiting for it: the log-likelihoods land in ``ll_out`` (n,), the status
    word is OR-ed into ``err_acc``.  ``cool_d`` is the unit's row of cooling
    factors; its first entry is the t0 factor."""
    torch = _ffi.require_cuda()
    ys_d, ycon_d, Tu_d, U1, T = unit_in
    spec = st_u.spec
    F, P = swarm.shape[0], spec.n_params
    out = {"swarm": torch.empty(F, P, J, dtype=torch.float32, device=swarm.device)}
    d = _ffi.PerfilterDesc()
    d.model = spec.ffi_model()
    d.J, d.F, d.T, d.U = J, F, T, U1
    d.flags = _ffi.F_SAVE_ANC if save_anc else 0
    d.thresh = float(max(0.0, thresh))
    if save_anc:
        out["anc"] = torch.zeros(F, T, J, dtype=torch.int32, device=swarm.device)
    d.swarm_in, d.swarm_out = _ffi.ptr(swarm), _ffi.ptr(out["swarm"])
    d.rw_sig, d.rw_sig0 = _ffi.ptr(sig_d), _ffi.ptr(sig0_d)
    d.cool, d.cool0 = _ffi.ptr(cool_d), _ffi.ptr(cool_d)
    d.ys, d.ycon, d.T_u = _ffi.ptr(ys_d), _ffi.ptr(ycon_d), _ffi.ptr(Tu_d)
    d.seeds, d.loglik, d.anc = _ffi.ptr(seeds_d), _ffi.ptr(ll_out), _ffi.ptr(out.get("anc"))
    ws = torch.empty(max(int(_ffi.LIB.ppf_perfilter_workspace_bytes(d)), 256), dtype=torch.uint8,
                     device=swarm.device)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    _ffi.check(_ffi.LIB.ppf_perfilter(d, stream), "ppf_perfilter")
    err_acc.bitwise_or_(ws[:4].view(torch.int32))
    out["loglik"] = ll_out
    return out


def panel_mif(struct: PanelPompStruct, shared_array, unit_array, rw_sd, M: int, J: int, keys,
              thresh: float = 0.0, n_monitors: int = 0, block: bool = True, *, inject=None,
              mode: str = "sequential"):
    """Panel iterated filtering (``pypomp/functional/mif.py:125-259``;
    ``_panel_mif_internal`` / ``_panel_mif_unit_scan_fn`` at
    ``pypomp/core/algorithms/panel_mif.py:17-247``).

    ``shared_array`` (n_reps, J, n_shared) and ``unit_array``
    (n_reps, J, U, n_spec), natural scale.  Every iteration visits the units
    in order; for unit u the swarms [shared | unit u] are permuted to the
    unit's canonical order, run through one perturbed filter (all replicates
    in one ``ppf_perfilter`` call, swarms resident on the GPU), and written
    back; the shared swarm carries from unit to unit.  With ``block=False``
    the other units' swarms are reordered by unit u's resampling ancestry.
    Keys: per replicate ``split(key, M+1)[1:]`` iteration keys, then
    ``split(iteration key, U)`` unit keys (monitors ``split(unit key,
    n_monitors)``).  The cooling factor of a unit uses that unit's own
    series length.  ``inject``, for replaying external draws, is indexed
    ``inject[m][u]`` like ``mif``'s.  Returns (shared_traces (n, M+1, ns+1),
    unit_traces (n, M+1, U, nu+1), final shared swarm (n, J, ns), final unit
    swarm (n, J, U, nu)); column 0 of the traces is the log-likelihood
    (summed over units for the shared trace), the rest are swarm means.

    ``mode="parallel"`` is not in the reference (see :func:`_panel_mif_parallel`):
    every unit of every replicate is filtered in one batched call per
    iteration, all from the iteration's shared swarm, and the units' shared
    swarms are then combined.
    """
    if mode == "parallel":
        if inject is not None:
            raise ValueError("mode='parallel' does not replay injected draws")
        return _panel_mif_parallel(struct, shared_array, unit_array, rw_sd, M, J, keys, thresh, n_monitors)
    if mode != "sequential":
        raise ValueError("mode must be 'sequential' or 'parallel'")
    from . import random as pprandom

    torch = _ffi.require_cuda()
    spec = struct.spec
    dev = torch.device("cuda", torch.cuda.current_device())
    sh = np.asarray(shared_array, dtype=np.float64)
    un = np.asarray(unit_array, dtype=np.float64)
    n = sh.shape[0]
    ns, nu, U = sh.shape[2], un.shape[3], struct.U
    if sh.shape[1] != J or un.shape[1] != J or un.shape[2] != U:
        raise ValueError("shared_array must be (n_reps, J, n_shared) and unit_array (n_reps, J, U, n_spec)")
    if M < 1:
        raise ValueError("M must be greater than 0.")
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    perms = np.asarray(struct.permutations, dtype=np.int64)
    inv_perms = np.argsort(perms, axis=1)
    names = struct.param_names
    sig_p, sig0_p = rw_sd.arrays(names)                      # panel order
    # estimation-scale swarms on the device: shared (n, ns, J), unit (n, U, nu, J)
    panel0 = np.concatenate([sh[:, :, None, :].repeat(U, axis=2), un], axis=3)   # (n, J, U, Pp)
    est_unit = np.empty_like(panel0)
    for u in range(U):
        th_u = spec.to_est(panel0[:, :, u, perms[u]])        # unit order
        est_unit[:, :, u, :] = th_u[:, :, inv_perms[u]]      # back to panel order
    S = torch.tensor(est_unit[:, :, 0, :ns].transpose(0, 2, 1).copy(), dtype=torch.float32, device=dev)
    Us = torch.tensor(est_unit[:, :, :, ns:].transpose(0, 2, 3, 1).copy(), dtype=torch.float32, device=dev)
    m_keys = np.stack([pprandom.split(k, M + 1)[1:] for k in keys])        # (n, M)

    def means():
        return S.mean(dim=2).cpu().numpy(), Us.mean(dim=3).cpu().numpy()  # (n, ns), (n, U, nu)

    def nat_means(s_mean, u_mean):
        s_out = np.empty((n, ns))
        u_out = np.empty((n, U, nu))
        for u in range(U):
            panel = np.concatenate([s_mean, u_mean[:, u]], axis=1)
            nat = spec.from_est(panel[:, perms[u]])[:, inv_perms[u]]
            u_out[:, u] = nat[:, ns:]
            if u == 0:
                s_out = nat[:, :ns]
        return s_out, u_out

    s0, u0 = nat_means(*means())
    shared_tr = np.full((n, M + 1, ns + 1), np.nan)
    unit_tr = np.full((n, M + 1, U, nu + 1), np.nan)
    shared_tr[:, 0, 1:], unit_tr[:, 0, :, 1:] = s0, u0
    perm_t = [torch.tensor(perms[u], device=dev) for u in range(U)]
    inv_t = [torch.tensor(inv_perms[u], device=dev) for u in range(U)]
    # Without injected draws the unit filters are queued back to back: every
    # unit's data and sds are uploaded once, each iteration's keys and cooling
    # factors in one pinned copy, and the status words are folded into one
    # device flag read once per iteration, so the host never waits for a unit
    # filter before preparing the next.
    fast = inject is None
    if fast:
        units_st = [struct.unit(u) for u in range(U)]
        unit_in = [_device_inputs(torch, units_st[u], dev) for u in range(U)]
        f32d = dict(dtype=torch.float32, device=dev)
        sig_d = [torch.tensor(sig_p[perms[u]], **f32d) for u in range(U)]
        sig0_d = [torch.tensor(sig0_p[perms[u]], **f32d) for u in range(U)]
        Tmax = max(u_in[4] for u_in in unit_in)
        err_acc = torch.zeros(1, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream

        def unit_cooling(it):
            c = np.zeros((U, Tmax), np.float32)
            for u in range(U):
                Tu = unit_in[u][4]
                c[u, :Tu] = [rw_sd.cooling_factor(i, it, Tu) for i in range(Tu)]
            return c
        cool_next = unit_cooling(0)
    for it in range(M):
        unit_keys = np.stack([pprandom.split(k, U) for k in m_keys[:, it]])    # (n, U)
        ll_units = np.zeros((n, U))
        if fast:
            cool_h = cool_next
            pinned = (torch.from_numpy(cool_h).pin_memory(),
                      torch.from_numpy(np.ascontiguousarray(unit_keys.T).view(np.int64)).pin_memory())
            cool_d = pinned[0].to(dev, non_blocking=True)                       # (U, Tmax)
            keys_d = pinned[1].to(dev, non_blocking=True)                       # (U, n)
            ll_d = torch.zeros(U, n, dtype=torch.float64, device=dev)
        for u in range(U):
            st_u = struct.unit(u)
            T = st_u.ys.shape[0]
            panel = torch.cat([S, Us[:, u]], dim=1)                             # (n, Pp, J)
            swarm = panel.index_select(1, perm_t[u]).contiguous()               # unit order
            if fast:
                inj = None
                res = _perfilter_queued(units_st[u], unit_in[u], swarm, keys_d[u], J, sig_d[u], sig0_d[u],
                                        cool_d[u], thresh, not block, ll_d[u], err_acc, stream)
            else:
                cool = np.array([rw_sd.cooling_factor(i, it, T) for i in range(T)], dtype=np.float32)
                inj = inject[it][u]
                res = run_perfilter(st_u, swarm, unit_keys[:, u], J, sig_p[perms[u]], sig0_p[perms[u]], cool,
                                    cool[0], thresh=thresh, save_ancestors=not block,
                                    inject=None if inj is None else inj["perfilter"])
            if n_monitors >= 1:
                mean = swarm.mean(dim=2).cpu().numpy()
                mon = np.stack([pprandom.split(k, n_monitors) for k in unit_keys[:, u]])
                minj = None
                if inj is not None:
                    minj = {k: np.stack([np.stack([inj["monitors"][i][k][r] for i in range(n_monitors)])
                                         for r in range(n)]).reshape(
                                             (n * n_monitors,) + inj["monitors"][0][k].shape[1:])
                            for k in ("z0", "z", "u")}
                pf = run_pfilter(st_u, np.repeat(mean, n_monitors, axis=0), mon.reshape(-1), J, thresh=thresh,
                                 est=True, inject=minj)
                ll_units[:, u] = -(-pf["loglik"].reshape(n, n_monitors)).mean(axis=1)
            elif not fast:
                ll_units[:, u] = res["loglik"].cpu().numpy()
            new_panel = res["swarm"].index_select(1, inv_t[u])                  # panel order
            if ns > 0:
                S = new_panel[:, :ns].contiguous()
            if nu > 0:
                if not block:
                    anc = res["anc"]                                           # (n, T, J)
                    origin = torch.arange(J, device=dev).expand(n, J).contiguous()
                    for t in range(T):
                        origin = torch.gather(origin, 1, anc[:, t].long())
                    idx = origin[:, None, None, :].expand(n, U, nu, J)
                    Us = torch.gather(Us, 3, idx)
                Us = Us.clone()
                Us[:, u] = new_panel[:, ns:]
        if fast:
            # the next iteration's cooling factors while this one's filters run
            if it + 1 < M:
                cool_next = unit_cooling(it + 1)
            err = int(err_acc.item())
            if err:
                _ffi.check(_ffi.PPF_ETIMEOUT if err & 1 else _ffi.PPF_EINTERNAL, "ppf_perfilter")
            if n_monitors < 1:
                ll_units = ll_d.T.cpu().numpy()
            del pinned
        s_mean, u_mean = nat_means(*means())
        shared_tr[:, it + 1, 0] = ll_units.sum(axis=1)
        shared_tr[:, it + 1, 1:] = s_mean
        unit_tr[:, it + 1, :, 0] = ll_units
        unit_tr[:, it + 1, :, 1:] = u_mean
    # final swarms on the natural scale
    s_fin = S.cpu().numpy().transpose(0, 2, 1)                 # (n, J, ns)
    u_fin = Us.cpu().numpy().transpose(0, 3, 1, 2)             # (n, J, U, nu)
    fs = np.empty((n, J, ns))
    fu = np.empty((n, J, U, nu))
    for u in range(U):
        panel = np.concatenate([s_fin, u_fin[:, :, u]], axis=2)
        nat = spec.from_est(panel[:, :, perms[u]])[:, :, inv_perms[u]]
        fu[:, :, u] = nat[:, :, ns:]
        if u == 0:
            fs = nat[:, :, :ns]
    return shared_tr, unit_tr, fs, fu


def _panel_mif_parallel(struct: PanelPompStruct, shared_array, unit_array, rw_sd, M: int, J: int, keys,
                        thresh: float = 0.0, n_monitors: int = 0):
    """Panel IF2 with the units filtered side by side -- a mode the reference
    does not have (its unit scan carries the shared swarm from unit to unit,
    ``pypomp/core/algorithms/panel_mif.py:119-123, 216-219``).

    Iteration m, replicate r:

    * one ``ppf_perfilter`` call filters all U units of all replicates
      (n x U swarms, ragged series masked per unit), each from
      [shared swarm S_r | unit u's swarm] with unit u's key (the sequential
      mode's ``split(iteration key, U)[u]``) and cooling (its own length);
    * unit u's unit-specific swarm becomes its filter's output, as in the
      sequential mode with ``block=True`` (no reordering across units);
    * the shared swarm is recombined from the units' outputs S'_{r,u}: per
      shared parameter (estimation scale), the centre is the inverse-variance
      weighted mean of the units' swarm means, sum_u mu_u / v_u / sum_u 1 / v_u
      (the maximiser of the sum of the units' quadratic log-likelihood
      approximations; a plain mean when no unit's swarm has spread), and
      particle j is that centre plus the deviation of particle j of unit
      (j mod U) from its unit's mean, so the swarm keeps the units' spread.

    Without shared parameters the units never interact and each unit's swarm
    is exactly what a single-unit IF2 iteration gives it.  The log-likelihood
    columns are each unit's perturbed-filter log-likelihood (or, with
    monitors, the mean of ``n_monitors`` filters at the unit's input swarm
    mean, all units in one batched call).  Returns what :func:`panel_mif`
    returns.
    """
    from . import random as pprandom

    torch = _ffi.require_cuda()
    spec = struct.spec
    dev = torch.device("cuda", torch.cuda.current_device())
    sh = np.asarray(shared_array, dtype=np.float64)
    un = np.asarray(unit_array, dtype=np.float64)
    n = sh.shape[0]
    ns, nu, U = sh.shape[2], un.shape[3], struct.U
    if sh.shape[1] != J or un.shape[1] != J or un.shape[2] != U:
        raise ValueError("shared_array must be (n_reps, J, n_shared) and unit_array (n_reps, J, U, n_spec)")
    if M < 1:
        raise ValueError("M must be greater than 0.")
    perms = np.asarray(struct.permutations, dtype=np.int64)
    if not np.all(perms == perms[0]):
        raise ValueError("mode='parallel' needs the same parameter order in every unit")
    perm, inv = perms[0], np.argsort(perms[0])
    perm_t, inv_t = torch.tensor(perm, device=dev), torch.tensor(inv, device=dev)
    keys = np.asarray(keys, dtype=np.uint64).reshape(-1)
    sig_p, sig0_p = rw_sd.arrays(struct.param_names)
    sig_u, sig0_u = sig_p[perm], sig0_p[perm]
    # the transforms act column by column: panel column j is canonical
    # parameter inv[j], so apply that parameter's transform to it directly (no
    # gathers of the J x U swarm); the shared block (n, J, ns) and the unit
    # block (n, J, U, nu) are transformed apart (the shared columns are not
    # repeated per unit) and transposed on the device
    import dataclasses

    def colspec(cols):
        cols = list(cols)
        return dataclasses.replace(spec, est_log=tuple(i for i, j in enumerate(cols) if inv[j] in spec.est_log),
                                   est_atanh=tuple(i for i, j in enumerate(cols) if inv[j] in spec.est_atanh))

    pspec = colspec(range(ns + nu))
    sspec, uspec = colspec(range(ns)), colspec(range(ns, ns + nu))
    S = torch.from_numpy(sspec.to_est(np.ascontiguousarray(sh))).to(dev).float().permute(0, 2, 1).contiguous()
    Us = torch.from_numpy(uspec.to_est(np.ascontiguousarray(un))).to(dev).float().permute(0, 2, 3, 1).contiguous()
    m_keys = np.stack([pprandom.split(k, M + 1)[1:] for k in keys])               # (n, M)
    all_units = struct.all_units()
    T_u = np.asarray(struct.T_u, dtype=np.int64)
    Tmax = int(struct.ys.shape[1])
    unit_f = np.tile(np.arange(U, dtype=np.int32), n)
    jmod = torch.arange(J, device=dev) % U

    def nat(s_est, u_est):        # (n, ns), (n, U, nu) estimation scale -> natural, panel order
        panel = np.concatenate([np.repeat(s_est[:, None], U, axis=1), u_est], axis=2)
        out = pspec.from_est(panel)
        return out[:, 0, :ns], out[:, :, ns:]

    # device-side loop: the keys of all iterations are uploaded once, the
    # swarms stay in one PerfilterCall's buffers, and without monitors nothing
    # waits for the GPU until the end.  Each iteration's cooling factors are
    # formed on the host while the previous iterations run, in a ring of two
    # pinned buffers (a buffer is refilled once its copy two iterations back
    # has run)
    unit_keys_all = np.stack([np.stack([pprandom.split(k, U) for k in m_keys[:, it]]) for it in range(M)])
    keys_d = torch.from_numpy(np.ascontiguousarray(unit_keys_all.reshape(M, n * U)).view(np.int64)).to(dev)
    cool_h = [torch.empty((U, Tmax), dtype=torch.float32).pin_memory() for _ in range(2)]
    cool_ev = [None, None]
    cool_d = torch.empty((M, U, Tmax), dtype=torch.float32, device=dev)
    panel = torch.cat([S[:, None].expand(n, U, ns, J), Us], dim=2)
    call = PerfilterCall(all_units, panel.reshape(n * U, ns + nu, J).index_select(1, perm_t), J, sig_u, sig0_u,
                         thresh=thresh, unit_f=unit_f)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    ll_d = torch.zeros(M, n, U, dtype=torch.float64, device=dev)
    smeans = torch.zeros(M + 1, n, ns, dtype=torch.float64, device=dev)
    umeans = torch.zeros(M + 1, n, U, nu, dtype=torch.float64, device=dev)
    smeans[0], umeans[0] = S.mean(dim=2).double(), Us.mean(dim=3).double()
    for it in range(M):
        r = it & 1
        if cool_ev[r] is not None:
            cool_ev[r].synchronize()
        _cooling_rows(rw_sd, it, T_u, Tmax, out=cool_h[r].numpy())
        cool_d[it].copy_(cool_h[r], non_blocking=True)
        cool_ev[r] = torch.cuda.Event()
        cool_ev[r].record()
        if it > 0:
            panel = torch.cat([S[:, None].expand(n, U, ns, J), Us], dim=2)
            call.swarm.copy_(panel.reshape(n * U, ns + nu, J).index_select(1, perm_t))
        if n_monitors >= 1:
            mean = call.swarm.mean(dim=2).cpu().numpy()                              # (n U, P) unit order
            mon = np.stack([pprandom.split(k, n_monitors) for k in unit_keys_all[it].reshape(-1)])
            pf = run_pfilter(all_units, np.repeat(mean, n_monitors, axis=0), mon.reshape(-1), J,
                             thresh=thresh, est=True, unit_f=np.repeat(unit_f, n_monitors))
            ll_d[it] = torch.from_numpy(pf["loglik"].reshape(n, U, n_monitors).mean(axis=2)).to(dev)
        call.run_device(keys_d[it], cool_d[it], err)
        if n_monitors < 1:
            ll_d[it] = call.ll.view(n, U)
        out = call.swarm.index_select(1, inv_t).reshape(n, U, ns + nu, J)            # panel order
        if nu > 0:
            Us = out[:, :, ns:].contiguous()
        if ns > 0:
            su = out[:, :, :ns].double()                                              # (n, U, ns, J)
            mu = su.mean(dim=3)
            var = su.var(dim=3, unbiased=False)
            w = torch.where(var > 0, 1.0 / var.clamp_min(1e-300), torch.zeros_like(var))
            wsum = w.sum(dim=1)
            centre = torch.where(wsum > 0, (w * mu).sum(dim=1) / wsum.clamp_min(1e-300), mu.mean(dim=1))
            dev_j = su - mu[..., None]                                                # deviations from unit means
            pick = dev_j.gather(1, jmod.view(1, 1, 1, J).expand(n, 1, ns, J)).squeeze(1)   # (n, ns, J)
            S = (centre[..., None] + pick).float().contiguous()
        smeans[it + 1], umeans[it + 1] = S.mean(dim=2).double(), Us.mean(dim=3).double()
    e = int(err.item())
    if e:
        _ffi.check(_ffi.PPF_ETIMEOUT if e & 1 else _ffi.PPF_EINTERNAL, "ppf_perfilter")
    shared_tr = np.full((n, M + 1, ns + 1), np.nan)
    unit_tr = np.full((n, M + 1, U, nu + 1), np.nan)
    sm, um = smeans.cpu().numpy(), umeans.cpu().numpy()
    ll_units = ll_d.cpu().numpy()                                                     # (M, n, U)
    for it in range(M + 1):
        s_mean, u_mean = nat(sm[it], um[it])
        shared_tr[:, it, 1:], unit_tr[:, it, :, 1:] = s_mean, u_mean
        if it > 0:
            shared_tr[:, it, 0] = ll_units[it - 1].sum(axis=1)
            unit_tr[:, it, :, 0] = ll_units[it - 1]
    s_fin = sspec.from_est(S.permute(0, 2, 1).contiguous().double().cpu().numpy())        # (n, J, ns)
    u_fin = uspec.from_est(Us.permute(0, 3, 1, 2).contiguous().double().cpu().numpy())    # (n, J, U, nu)
    return shared_tr, unit_tr, s_fin, u_fin


def panel_train(struct: PanelPompStruct, shared_array, unit_array, J: int, optimizer, M: int, eta,
                alpha: float, keys, alpha_cooling: float = 1.0, chunk_size: int = 1, *, inject=None,
                process_weight_index: int | None = None):
    """Panel MOP-alpha gradient training (``pypomp/functional/train.py:112-190``;
    ``_panel_train_internal`` / ``_chunk_scan_step`` at
    ``pypomp/core/algorithms/train.py:191-413``).

    ``shared_array`` (n_reps, n_shared), ``unit_array`` (n_reps, U, n_spec),
    natural scale; ``keys`` (n_reps, M, U) (or (n_reps,), split into M x U).
    Each iteration walks the units in chunks of ``chunk_size``; a chunk's
    MOP values and gradients for every replicate come from one ``ppf_mop``
    call.  Chunk loss = sum of its units' MOP values / (chunk_size * Tmax);
    the shared parameters take one optimiser step per chunk with rate
    eta / n_chunks (global step count), the unit parameters one step with the
    gradient scaled by chunk_size (iteration count).  Returns
    (neg_logliks (n, M+1), shared (n, M+1, ns), unit (n, M+1, U, nu)),
    natural scale, NaN first log-likelihood.  ``inject[m][c]`` optionally
    replays external draws for chunk c of iteration m.

    With ``process_weight_index`` it is the panel DPOP training of
    ``_panel_dpop_train_internal`` (``pypomp/core/algorithms/train_panel_dpop.py:152-322``):
    the chunks' values and gradients are DPOP's (``PPF_F_DPOP``), gradients
    are not clipped, SGD and Adam only, and the first log-likelihood entry is
    the summed DPOP objective of all units at the initial parameters under
    iteration 0's keys and the uncooled alpha (``train_panel_dpop.py:295-316``).
    """
    from . import random as pprandom
    from .optim import SGD, Adam, FullMatrixAdam, LearningRate, cosine_alpha

    dpop_mode = process_weight_index is not None
    if dpop_mode and inject is not None:
        raise ValueError("panel DPOP training does not replay injected draws")
    # as _panel_train_internal (train.py:191-200): these three only; `ls` is not used by panel train
    allowed = (SGD, Adam) if dpop_mode else (SGD, Adam, FullMatrixAdam)
    if not isinstance(optimizer, allowed):
        what = "panel dpop_train" if dpop_mode else "panel train"
        raise ValueError(f"Optimizer '{optimizer.__class__.__name__}' not supported for {what}")
    spec = struct.spec
    U, Tn = struct.U, struct.ys.shape[1]
    cs = max(1, int(chunk_size))
    if U % cs:
        raise ValueError("chunk_size must divide the number of units")
    nch = U // cs
    sh = np.asarray(shared_array, dtype=np.float64)
    un = np.asarray(unit_array, dtype=np.float64)
    n, ns = sh.shape
    nu = un.shape[2]
    keys = np.asarray(keys, dtype=np.uint64)
    if keys.ndim == 1:
        keys = np.stack([pprandom.split(k, M * U) for k in keys]).reshape(n, M, U)
    keys = keys.reshape(n, M, U)
    perms = np.asarray(struct.permutations, dtype=np.int64)
    inv_perms = np.argsort(perms, axis=1)
    eta_s = eta.to_array(struct.shared_param_names, M) if (ns and isinstance(eta, LearningRate)) else \
        np.broadcast_to(np.asarray(eta, np.float64), (max(M, 1), ns)) if ns else np.zeros((max(M, 1), 0))
    eta_u = eta.to_array(struct.unit_param_names, M) if (nu and isinstance(eta, LearningRate)) else \
        np.broadcast_to(np.asarray(eta, np.float64), (max(M, 1), nu)) if nu else np.zeros((max(M, 1), 0))

    def to_est_blocks(s_nat, u_nat):
        th = _panel_thetas(s_nat, u_nat, perms)                       # (n, U, P) unit order
        est = spec.to_est(th)
        panel = np.stack([est[:, u, inv_perms[u]] for u in range(U)], axis=1)   # (n, U, Pp)
        return panel[:, 0, :ns].copy(), panel[:, :, ns:].copy()

    def from_est_blocks(s_est, u_est):
        th = _panel_thetas(s_est, u_est, perms)
        nat = spec.from_est(th)
        panel = np.stack([nat[:, u, inv_perms[u]] for u in range(U)], axis=1)
        return panel[:, 0, :ns].copy(), panel[:, :, ns:].copy()

    s_est, u_est = to_est_blocks(sh, un)
    st_s = optimizer.init_state(s_est)
    st_u = optimizer.init_state(u_est)
    gstep = 0
    nll = np.full((n, M + 1), np.nan)
    hist_s = np.zeros((n, M + 1, ns))
    hist_u = np.zeros((n, M + 1, U, nu))
    hist_s[:, 0], hist_u[:, 0] = sh, un
    all_units = struct.all_units()
    alphas = [1.0 - (1.0 - alpha) * cosine_alpha(m, M, alpha_cooling) for m in range(M)]
    # one alpha for the whole run and no injected draws: each chunk reuses one
    # MOP call (buffers, workspace, captured launch sequence) across iterations
    reuse = len(set(alphas)) == 1 and inject is None
    calls = [None] * nch
    for m in range(M):
        alpha_m = alphas[m]
        chunk_nll = np.zeros((n, nch))
        for c in range(nch):
            units = np.arange(c * cs, (c + 1) * cs)
            th = _panel_thetas(s_est, u_est[:, units], perms[units])    # (n, cs, P)
            inj = inject[m][c] if inject is not None else None
            th32 = th.reshape(n * cs, -1).astype(np.float32)
            ks = keys[:, m, units].reshape(-1)
            if reuse and calls[c] is not None:
                calls[c].update(th32, ks)
                res = {k: v.cpu().numpy() for k, v in calls[c].forward(grad=True).items()}
            elif reuse:
                calls[c] = MopCall(all_units, th32, ks, J, alpha_m, unit_f=np.tile(units.astype(np.int32), n),
                                   graph=True, process_weight_index=process_weight_index)
                res = {k: v.cpu().numpy() for k, v in calls[c].forward(grad=True).items()}
            else:
                res = run_mop(all_units, th32, ks, J, alpha_m, grad=True,
                              unit_f=np.tile(units.astype(np.int32), n), inject=inj,
                              process_weight_index=process_weight_index)
            val = res["value"].reshape(n, cs)
            g = res["grad"].reshape(n, cs, -1)
            gp = np.zeros((n, cs, ns + nu))
            for j, u in enumerate(units):
                gp[:, j, perms[u]] = g[:, j]
            scale = 1.0 / (cs * Tn)
            grad_s = gp[:, :, :ns].sum(axis=1) * scale
            grad_u = gp[:, :, ns:] * scale * cs
            chunk_nll[:, c] = val.sum(axis=1) * scale * (Tn * U)
            _warn_nonfinite(gp, m)
            if optimizer.clip_norm is not None and not dpop_mode:
                grad_s = np.clip(grad_s, -optimizer.clip_norm, optimizer.clip_norm)
                grad_u = np.clip(grad_u, -optimizer.clip_norm, optimizer.clip_norm)
            d_s, st_s = optimizer.step(grad_s, st_s, gstep)
            st_uc = tuple(x[:, units] for x in st_u)
            d_u, st_uc = optimizer.step(grad_u, st_uc, m)
            for x, y in zip(st_u, st_uc):
                x[:, units] = y
            if optimizer.scale:
                d_s = d_s / np.maximum(np.linalg.norm(d_s, axis=-1, keepdims=True), 1e-8)
                d_u = d_u / np.maximum(np.linalg.norm(d_u, axis=-1, keepdims=True), 1e-8)
            s_est = s_est + (eta_s[m] / nch) * d_s
            u_est[:, units] = u_est[:, units] + eta_u[m] * d_u
            gstep += 1
        nll[:, m + 1] = chunk_nll.mean(axis=1)
        hist_s[:, m + 1], hist_u[:, m + 1] = from_est_blocks(s_est, u_est)
    if dpop_mode:
        s0, u0 = to_est_blocks(sh, un)
        units = np.arange(U)
        th0 = _panel_thetas(s0, u0, perms).reshape(n * U, -1).astype(np.float32)
        v0 = run_mop(all_units, th0, keys[:, 0, :].reshape(-1), J, alpha, grad=False,
                     unit_f=np.tile(units.astype(np.int32), n), process_weight_index=process_weight_index)["value"]
        nll[:, 0] = v0.reshape(n, U).sum(axis=1)
    return nll, hist_s, hist_u


def panel_dpop_train(struct: PanelPompStruct, shared_array, unit_array, J: int, optimizer, M: int, eta,
                     alpha: float, process_weight_index: int, keys, alpha_cooling: float = 1.0,
                     chunk_size: int = 1):
    """Panel DPOP gradient training (``_panel_dpop_train_internal``,
    ``pypomp/core/algorithms/train_panel_dpop.py:152-322``, behind
    ``PanelPomp._dpop_train``): :func:`panel_train`'s chunk loop on the DPOP
    objective.  Returns ``(neg_logliks (n, M+1), shared (n, M+1, ns),
    unit (n, M+1, U, nu))``, natural scale."""
    import warnings

    warnings.warn("dpop_train is experimental and its API and behavior are subject to change.",
                  category=FutureWarning, stacklevel=2)
    return panel_train(struct, shared_array, unit_array, J, optimizer, M, eta, alpha, keys, alpha_cooling,
                       chunk_size, process_weight_index=int(process_weight_index))
