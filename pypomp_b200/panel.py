"""``PanelPomp``: panels of units that share one built-in CUDA model.

Mirrors the reference's panel interface on the hot path
(``pypomp/panel/panel.py:15`` ``PanelPomp``,
``pypomp/panel/estimation_mixin.py:384`` ``pfilter``, ``:597`` ``mif``,
``:775`` ``train``; parameters as in ``pypomp/core/parameters/panel.py``,
result tables as in ``pypomp/core/results/render.py:179-400``), with pandas
frames instead of xarray.  Units may have series of different lengths; the
kernels mask each unit after its own last observation.
"""

from __future__ import annotations

import time
from copy import deepcopy

import numpy as np
import pandas as pd

from . import random as pprandom
from .maths import logmeanexp, logmeanexp_se
from .pomp import ResultsHistory


class PanelParameters:
    """Shared and unit-specific parameter sets, one entry per replicate.

    Each entry is ``{"shared": DataFrame (index: shared names, one column) or
    None, "unit_specific": DataFrame (index: unit parameter names, columns:
    unit names) or None}``, as the reference's constructor takes them.
    """

    def __init__(self, theta, logLik_unit=None):
        if isinstance(theta, PanelParameters):
            self._list = deepcopy(theta._list)
            self.logLik_unit = None if theta.logLik_unit is None else np.array(theta.logLik_unit)
            return
        if isinstance(theta, dict):
            theta = [theta]
        self._list = []
        for t in theta:
            sh = t.get("shared")
            us = t.get("unit_specific")
            self._list.append({"shared": None if sh is None else sh.copy(),
                               "unit_specific": None if us is None else us.copy()})
        if not self._list:
            raise ValueError("theta must hold at least one replicate")
        self.logLik_unit = None if logLik_unit is None else np.asarray(logLik_unit, dtype=float)

    # -- names -------------------------------------------------------------
    def get_shared_param_names(self):
        sh = self._list[0]["shared"]
        return [] if sh is None else [str(x) for x in sh.index]

    def get_unit_param_names(self):
        us = self._list[0]["unit_specific"]
        return [] if us is None else [str(x) for x in us.index]

    def get_unit_names(self):
        us = self._list[0]["unit_specific"]
        return [] if us is None else [str(x) for x in us.columns]

    def get_param_names(self):
        return self.get_shared_param_names() + self.get_unit_param_names()

    def num_replicates(self) -> int:
        return len(self._list)

    @property
    def logLik(self):
        return None if self.logLik_unit is None else self.logLik_unit.sum(axis=1)

    # -- arrays ------------------------------------------------------------
    def shared_array(self, names=None) -> np.ndarray:
        names = self.get_shared_param_names() if names is None else names
        if not names:
            return np.zeros((len(self._list), 0))
        return np.stack([t["shared"].loc[names].iloc[:, 0].to_numpy(dtype=float) for t in self._list])

    def unit_array(self, unit_names, names=None) -> np.ndarray:
        names = self.get_unit_param_names() if names is None else names
        if not names:
            return np.zeros((len(self._list), len(unit_names), 0))
        return np.stack([t["unit_specific"].loc[names, list(unit_names)].to_numpy(dtype=float).T
                         for t in self._list])

    @classmethod
    def from_arrays(cls, shared_values, unit_specific_values, shared_names, unit_specific_names, unit_names,
                    logLik_unit=None):
        """(n, ns) and (n, U, nu) arrays to parameter frames."""
        out = []
        for i in range(np.asarray(shared_values).shape[0]):
            sh = (pd.DataFrame({"shared": np.asarray(shared_values)[i]}, index=list(shared_names))
                  if len(shared_names) else None)
            us = (pd.DataFrame(np.asarray(unit_specific_values)[i].T, index=list(unit_specific_names),
                               columns=list(unit_names)) if len(unit_specific_names) else None)
            out.append({"shared": sh, "unit_specific": us})
        return cls(out, logLik_unit=logLik_unit)

    def params(self, as_list: bool = True):
        return deepcopy(self._list)

    def pruned(self, n: int = 1, refill: bool = True) -> "PanelParameters":
        """The top ``n`` replicates by panel log-likelihood, repeated to the previous
        count with ``refill`` (``pypomp/core/parameters/base.py:138-181``; without
        log-likelihoods every replicate ranks equal)."""
        n_reps = self.num_replicates()
        if n < 1:
            raise ValueError("n must be at least 1.")
        ll = self.logLik
        if ll is None or np.all(np.isnan(ll)):
            ll = np.zeros(n_reps)
        top = np.asarray(ll).argsort()[-n:][::-1]
        idx = np.tile(top, (n_reps + n - 1) // n)[:n_reps] if refill else top
        return PanelParameters([self._list[i] for i in idx],
                               logLik_unit=None if self.logLik_unit is None else self.logLik_unit[idx])

    def mixed_and_matched(self, unit_names=None) -> "PanelParameters":
        """Rank the shared parameters by panel log-likelihood and, unit by unit,
        the unit-specific parameters by that unit's log-likelihood; replicate r
        of the result pairs the r-th best of each
        (``pypomp/core/parameters/panel.py:504-585``).  ``unit_names`` is the
        order of the columns of ``logLik_unit`` (default: the unit-specific
        frame's columns)."""
        if self.logLik_unit is None:
            raise ValueError("mix_and_match needs unit log-likelihoods (run pfilter first)")
        units = list(self.get_unit_names() if unit_names is None else unit_names)
        reps = self.num_replicates()
        shared_ranks = self.logLik.argsort()[::-1]
        unit_ranks = [self.logLik_unit[:, u].argsort()[::-1] for u in range(len(units))]
        out, ll_unit = [], np.zeros_like(self.logLik_unit)
        for r in range(reps):
            sh = self._list[shared_ranks[r]]["shared"]
            us = None
            if self._list[0]["unit_specific"] is not None:
                us = self._list[0]["unit_specific"].copy()
                for u, name in enumerate(units):
                    us[name] = self._list[unit_ranks[u][r]]["unit_specific"][name].to_numpy()
            out.append({"shared": None if sh is None else sh.copy(), "unit_specific": us})
            for u in range(len(units)):
                ll_unit[r, u] = self.logLik_unit[unit_ranks[u][r], u]
        return PanelParameters(out, logLik_unit=ll_unit)

    def __len__(self):
        return len(self._list)

    def __repr__(self):
        return f"PanelParameters({self.num_replicates()} replicates, shared={self.get_shared_param_names()}, " \
               f"unit_specific={self.get_unit_param_names()})"


class PanelResult:
    """One panel run: tables in the reference's panel layout."""

    def __init__(self, method, theta, payload, config, execution_time, key):
        self.method, self.theta, self.payload = method, theta, payload
        self.config, self.execution_time, self.key = config, execution_time, key

    def to_dataframe(self, ignore_nan: bool = False) -> pd.DataFrame:
        unit_names = self.payload["unit_names"]
        if self.method == "pfilter":
            ll = self.payload["logLiks"]                                  # (n, U, reps)
            lme = logmeanexp(ll, axis=-1, ignore_nan=ignore_nan)
            se = (logmeanexp_se(ll, axis=-1, ignore_nan=ignore_nan) if ll.shape[-1] > 1
                  else np.full(lme.shape, np.nan))
            shared_ll = lme.sum(axis=1)
            shared_se = np.sqrt(np.sum(se ** 2, axis=1))
            rows = [{"theta_idx": i, "shared logLik": shared_ll[i], "shared logLik se": shared_se[i],
                     "unit": un, "unit logLik": lme[i, u], "unit logLik se": se[i, u]}
                    for i in range(ll.shape[0]) for u, un in enumerate(unit_names)]
            df = pd.DataFrame(rows)
            return _attach_params(df, self.theta, unit_names)
        s_tr, u_tr = self.payload["shared_traces"], self.payload["unit_traces"]
        n = s_tr.shape[0]
        rows = []
        for i in range(n):
            for u, un in enumerate(unit_names):
                r = {"theta_idx": i, "iteration": s_tr.shape[1] - 1, "shared logLik": s_tr[i, -1, 0],
                     "shared logLik se": np.nan, "unit": un, "unit logLik": u_tr[i, -1, u, 0],
                     "unit logLik se": np.nan}
                r.update({nm: s_tr[i, -1, 1 + p] for p, nm in enumerate(self.payload["shared_names"])})
                r.update({nm: u_tr[i, -1, u, 1 + p] for p, nm in enumerate(self.payload["unit_param_names"])})
                rows.append(r)
        return pd.DataFrame(rows)

    def traces(self) -> pd.DataFrame:
        unit_names = self.payload["unit_names"]
        if self.method == "pfilter":
            df = self.to_dataframe()
            rows = []
            for i in df["theta_idx"].unique():
                d = df[df["theta_idx"] == i]
                rows.append({"theta_idx": i, "unit": "shared", "iteration": 0, "method": "pfilter",
                             "logLik": d["shared logLik"].iloc[0], "se": d["shared logLik se"].iloc[0]})
                for _, r in d.iterrows():
                    rows.append({"theta_idx": i, "unit": r["unit"], "iteration": 0, "method": "pfilter",
                                 "logLik": r["unit logLik"], "se": r["unit logLik se"]})
            return pd.DataFrame(rows)
        s_tr, u_tr = self.payload["shared_traces"], self.payload["unit_traces"]
        sn, un_ = self.payload["shared_names"], self.payload["unit_param_names"]
        rows = []
        n, M1 = s_tr.shape[:2]
        for i in range(n):
            for m in range(M1):
                r = {"theta_idx": i, "unit": "shared", "iteration": m, "method": self.method,
                     "logLik": s_tr[i, m, 0], "se": np.nan}
                r.update({nm: s_tr[i, m, 1 + p] for p, nm in enumerate(sn)})
                rows.append(r)
                for u, uname in enumerate(unit_names):
                    r = {"theta_idx": i, "unit": uname, "iteration": m, "method": self.method,
                         "logLik": u_tr[i, m, u, 0], "se": np.nan}
                    r.update({nm: s_tr[i, m, 1 + p] for p, nm in enumerate(sn)})
                    r.update({nm: u_tr[i, m, u, 1 + p] for p, nm in enumerate(un_)})
                    rows.append(r)
        return pd.DataFrame(rows)


def _attach_params(df, theta, unit_names):
    sn = theta.get_shared_param_names()
    un = theta.get_unit_param_names()
    sh = theta.shared_array(sn)
    us = theta.unit_array(unit_names, un)
    for p, nm in enumerate(sn):
        df[nm] = [sh[i, p] for i in df["theta_idx"]]
    uidx = {u: k for k, u in enumerate(unit_names)}
    for p, nm in enumerate(un):
        df[nm] = [us[i, uidx[u], p] for i, u in zip(df["theta_idx"], df["unit"])]
    return df


class PanelPomp:
    """A panel of ``Pomp`` units on one built-in model with shared and
    unit-specific parameters (``pypomp/panel/panel.py:15``)."""

    def __init__(self, Pomp_dict: dict, theta: PanelParameters):
        if not isinstance(theta, PanelParameters):
            raise TypeError("theta must be a PanelParameters instance")
        if not Pomp_dict:
            raise ValueError("Pomp_dict must hold at least one unit")
        self.unit_objects = dict(Pomp_dict)
        self.theta = theta
        self.results_history = ResultsHistory()
        self.fresh_key = None
        self.canonical_shared_param_names = theta.get_shared_param_names()
        self.canonical_unit_param_names = theta.get_unit_param_names()
        self.canonical_param_names = theta.get_param_names()
        specs = {u.spec.kind for u in self.unit_objects.values()}
        if len(specs) != 1:
            raise ValueError("all units must use the same built-in model")
        rep = next(iter(self.unit_objects.values()))
        if set(self.canonical_param_names) != set(rep.canonical_param_names):
            raise ValueError("shared + unit-specific names must be the units' parameter names")
        if theta.get_unit_param_names() and set(theta.get_unit_names()) != set(self.unit_objects):
            raise ValueError("unit-specific columns must name the units")

    def get_unit_names(self):
        return list(self.unit_objects.keys())

    def to_struct(self):
        from .functional import PanelPompStruct

        names = self.get_unit_names()
        units = [self.unit_objects[u] for u in names]
        rep = units[0]
        Tmax = max(len(u.ys) for u in units)
        dy = rep.spec.dy
        ys = np.zeros((len(units), Tmax, dy), np.float32)
        T_u = np.zeros(len(units), np.int32)
        for k, u in enumerate(units):
            y = u.ys.to_numpy(dtype=np.float32)
            ys[k, :len(y)] = y
            T_u[k] = len(y)
        panel_names = self.canonical_param_names
        perms = np.array([[panel_names.index(nm) for nm in u.canonical_param_names] for u in units], np.int64)
        return PanelPompStruct(spec=rep.spec, ys=ys, T_u=T_u, times=[u.ys.index.to_numpy(float) for u in units],
                               t0=rep.t0, unit_names=names, shared_param_names=self.canonical_shared_param_names,
                               unit_param_names=self.canonical_unit_param_names, permutations=perms)

    def _update_fresh_key(self, key=None):
        old = self.fresh_key if key is None else pprandom.as_key(key)
        if old is None:
            raise ValueError("Both the key argument and the fresh_key attribute are None. "
                             "At least one key must be given.")
        self.fresh_key, new = pprandom.split(old)
        return new, old

    def _theta_in(self, theta):
        t = self.theta if theta is None else theta
        if not isinstance(t, PanelParameters):
            t = PanelParameters(t)
        return deepcopy(t)

    def get_unit_parameters(self, unit: str, theta=None) -> list:
        """Each replicate's parameters of ``unit``: shared values updated with
        the unit's own (``pypomp/panel/estimation_mixin.py:104-142``)."""
        t = self._theta_in(theta)
        out = []
        for d in t.params(as_list=True):
            p = {}
            if d["shared"] is not None:
                p.update({str(k): float(v) for k, v in d["shared"].iloc[:, 0].items()})
            if d["unit_specific"] is not None:
                p.update({str(k): float(v) for k, v in d["unit_specific"][unit].items()})
            out.append(p)
        return out

    def simulate(self, key, theta=None, times=None, nsim: int = 1, as_pomp: bool = False):
        """Simulated states and observations of every unit
        (``pypomp/panel/estimation_mixin.py:229-311``): unit by unit with the
        unit's parameters and a key split off the panel key, through
        ``Pomp.simulate`` (one ``ppf_simulate`` launch per unit).  Returns
        long-format frames with a leading ``unit`` column, or with
        ``as_pomp`` a copy of the panel whose units hold the first replicate's
        simulated data."""
        import warnings

        from .pomp import PompParameters

        if as_pomp:
            if nsim > 1:
                warnings.warn(
                    "as_pomp is True, but nsim > 1. Only 1 simulation will be performed as_pomp overrides nsim.",
                    UserWarning, stacklevel=2)
            nsim = 1
        t = self._theta_in(theta)
        key = pprandom.as_key(key)
        xs, ys, units = [], [], {}
        for unit, obj in self.unit_objects.items():
            key, sub = pprandom.split(key)
            res = obj.simulate(key=sub, theta=PompParameters(self.get_unit_parameters(unit, theta=t)),
                               times=times, nsim=nsim, as_pomp=as_pomp)
            if as_pomp:
                units[unit] = res
            else:
                X, Y = res
                X.insert(0, "unit", unit)
                Y.insert(0, "unit", unit)
                xs.append(X)
                ys.append(Y)
        if as_pomp:
            out = deepcopy(self)
            out.unit_objects = units
            out.theta = PanelParameters(t.params(as_list=True)[:1])
            return out
        return pd.concat(xs), pd.concat(ys)

    # -- estimation ----------------------------------------------------------
    def pfilter(self, J: int, key=None, theta=None, thresh: float = 0.0, reps: int = 1, chunk_size: int = 1,
                CLL: bool = False, ESS: bool = False, filter_mean: bool = False,
                prediction_mean: bool = False) -> None:
        """Panel particle filter (``pypomp/panel/estimation_mixin.py:384-595``)."""
        from . import functional as F

        start = time.time()
        thresh = float(max(0.0, thresh))
        th = self._theta_in(theta)
        new_key, old_key = self._update_fresh_key(key)
        if J < 1:
            raise ValueError("J should be greater than 0.")
        struct = self.to_struct()
        names = self.get_unit_names()
        U = len(names)
        n = th.num_replicates()
        sh = th.shared_array(self.canonical_shared_param_names)
        us = th.unit_array(names, self.canonical_unit_param_names)
        from .functional import _panel_thetas

        thetas = _panel_thetas(sh, us, struct.permutations)            # (n, U, P)
        thetas = np.repeat(thetas, reps, axis=0)
        keys = pprandom.split(new_key, n * reps * U).reshape(n * reps, U)
        res = F.panel_pfilter(struct, thetas, J, keys, thresh, chunk_size, CLL, ESS, filter_mean,
                              prediction_mean)
        ll = res["logLik"].reshape(n, reps, U).transpose(0, 2, 1)      # (n, U, reps)
        th.logLik_unit = logmeanexp(ll, axis=-1)
        self.theta = th
        payload = {"logLiks": ll, "unit_names": names}
        for k in ("CLL", "ESS", "filter_mean", "prediction_mean"):
            if k in res:
                a = res[k].reshape((n, reps, U) + res[k].shape[2:])
                payload[k] = np.moveaxis(a, 1, 2)
        self.results_history.add(PanelResult("pfilter", deepcopy(th), payload,
                                             {"J": J, "reps": reps, "thresh": thresh},
                                             time.time() - start, old_key))

    def mif(self, J: int, M: int, rw_sd, key=None, theta=None, thresh: float = 0.0, n_monitors: int = 0,
            block: bool = True, mode: str = "sequential") -> None:
        """Panel iterated filtering (``pypomp/panel/estimation_mixin.py:597-773``).

        ``mode="parallel"`` (not in the reference) filters all units side by
        side in one batched call per iteration and recombines the shared
        swarm afterwards (``functional._panel_mif_parallel``)."""
        from . import functional as F

        start = time.time()
        thresh = float(max(0.0, thresh))
        th = self._theta_in(theta)
        theta_for_result = deepcopy(th)
        n = th.num_replicates()
        names = self.get_unit_names()
        if J < 1 or M < 1:
            raise ValueError("J and M must be greater than 0.")
        sn, un = self.canonical_shared_param_names, self.canonical_unit_param_names
        sh = np.repeat(th.shared_array(sn)[:, None, :], J, axis=1)
        us = np.repeat(th.unit_array(names, un)[:, None, :, :], J, axis=1)
        key, old_key = self._update_fresh_key(key)
        keys = pprandom.split(key, n)
        s_tr, u_tr, _, _ = F.panel_mif(self.to_struct(), sh, us, rw_sd, M, J, keys, thresh, n_monitors, block,
                                       mode=mode)
        self.theta = PanelParameters.from_arrays(s_tr[:, -1, 1:], u_tr[:, -1, :, 1:], sn, un, names,
                                                 logLik_unit=u_tr[:, -1, :, 0])
        self.results_history.add(PanelResult(
            "mif", theta_for_result,
            {"shared_traces": s_tr, "unit_traces": u_tr, "unit_names": names, "shared_names": sn,
             "unit_param_names": un},
            {"J": J, "M": M, "rw_sd": rw_sd, "thresh": thresh, "n_monitors": n_monitors, "block": block,
             "mode": mode},
            time.time() - start, old_key))

    def train(self, J: int, M: int, eta, chunk_size: int = 1, optimizer=None, alpha: float = 0.97, key=None,
              theta=None, alpha_cooling: float = 1.0) -> None:
        """Panel MOP-alpha training (``pypomp/panel/estimation_mixin.py:775-1000``)."""
        from . import functional as F
        from .optim import Adam

        start = time.time()
        optimizer = optimizer or Adam()
        th = self._theta_in(theta)
        theta_for_result = deepcopy(th)
        n = th.num_replicates()
        key, old_key = self._update_fresh_key(key)
        if J < 1 or M < 1:
            raise ValueError("J and M must be greater than 0.")
        names = self.get_unit_names()
        U = len(names)
        sn, un = self.canonical_shared_param_names, self.canonical_unit_param_names
        keys = pprandom.split(key, n * M * U).reshape(n, M, U)
        nll, hs, hu = F.panel_train(self.to_struct(), th.shared_array(sn), th.unit_array(names, un), J,
                                    optimizer, M, eta, alpha, keys, alpha_cooling, chunk_size)
        s_tr = np.concatenate([-nll[:, :, None], hs], axis=2)
        u_tr = np.concatenate([np.full(hu.shape[:3] + (1,), np.nan), hu], axis=3)
        self.theta = PanelParameters.from_arrays(hs[:, -1], hu[:, -1], sn, un, names)
        self.results_history.add(PanelResult(
            "train", theta_for_result,
            {"shared_traces": s_tr, "unit_traces": u_tr, "unit_names": names, "shared_names": sn,
             "unit_param_names": un},
            {"J": J, "M": M, "eta": eta, "alpha": alpha, "chunk_size": chunk_size,
             "alpha_cooling": alpha_cooling, "optimizer": optimizer},
            time.time() - start, old_key))

    def _dpop_train(self, J: int, M: int, eta, chunk_size: int = 1, optimizer=None, alpha: float = 0.97,
                    alpha_cooling: float = 1.0, process_weight_state: str | None = None, key=None,
                    theta=None) -> None:
        """Panel DPOP training (``pypomp/panel/estimation_mixin.py:995-1180``,
        experimental there too): :meth:`train`'s chunked loop on the DPOP
        objective with the transition log-weight in state component
        ``process_weight_state``.  A ``chunk_size`` that does not divide the
        number of units is lowered to the largest divisor below it, with a
        warning, as the reference does."""
        import warnings

        from . import functional as F
        from .optim import Adam

        warnings.warn("dpop_train is experimental and its API and behavior are subject to change.",
                      category=FutureWarning, stacklevel=2)
        start = time.time()
        optimizer = optimizer or Adam()
        th = self._theta_in(theta)
        theta_for_result = deepcopy(th)
        n = th.num_replicates()
        key, old_key = self._update_fresh_key(key)
        if J < 1:
            raise ValueError("J should be greater than 0.")
        if M < 1:
            raise ValueError("M should be greater than 0.")
        names = self.get_unit_names()
        U = len(names)
        cs = min(max(int(chunk_size), 1), U)
        if U % cs:
            orig = cs
            cs = max(d for d in range(cs, 0, -1) if U % d == 0)
            warnings.warn("chunk_size does not divide the number of units; "
                          f"using chunk_size={cs} instead of {orig}.", UserWarning, stacklevel=2)
        if process_weight_state is None:
            raise ValueError(
                "dpop_train requires a process-weight state. Please provide `process_weight_state` as the "
                "name of the state variable that accumulates the transition log-weight (e.g. 'logw').")
        statenames = list(self.unit_objects[names[0]].statenames)
        if process_weight_state not in statenames:
            raise ValueError(f"process_weight_state '{process_weight_state}' not found in statenames: "
                             f"{statenames}")
        pwi = statenames.index(process_weight_state)
        sn, un = self.canonical_shared_param_names, self.canonical_unit_param_names
        keys = pprandom.split(key, n * M * U).reshape(n, M, U)
        nll, hs, hu = F.panel_train(self.to_struct(), th.shared_array(sn), th.unit_array(names, un), J,
                                    optimizer, M, eta, alpha, keys, alpha_cooling, cs, process_weight_index=pwi)
        s_tr = np.concatenate([-nll[:, :, None], hs], axis=2)
        u_tr = np.concatenate([np.full(hu.shape[:3] + (1,), np.nan), hu], axis=3)
        self.theta = PanelParameters.from_arrays(hs[:, -1], hu[:, -1], sn, un, names)
        self.results_history.add(PanelResult(
            "dpop_train", theta_for_result,
            {"shared_traces": s_tr, "unit_traces": u_tr, "unit_names": names, "shared_names": sn,
             "unit_param_names": un},
            {"J": J, "M": M, "eta": eta, "alpha": alpha, "chunk_size": cs, "alpha_cooling": alpha_cooling,
             "optimizer": optimizer, "process_weight_state": process_weight_state},
            time.time() - start, old_key))

    # -- analysis ------------------------------------------------------------
    def time(self) -> pd.DataFrame:
        return self.results_history.time()

    def prune(self, n: int = 1, refill: bool = True) -> None:
        """Keep the top ``n`` parameter sets (``pypomp/panel/analysis_mixin.py:38-49``)."""
        self.theta = self.theta.pruned(n=n, refill=refill)

    def mix_and_match(self) -> None:
        """Cross-combine the best shared and unit-specific parameters
        (``pypomp/panel/analysis_mixin.py:51-72``)."""
        self.theta = self.theta.mixed_and_matched(self.get_unit_names())

    def results(self, index: int = -1, ignore_nan: bool = False) -> pd.DataFrame:
        return self.results_history[index].to_dataframe(ignore_nan=ignore_nan)

    def traces(self) -> pd.DataFrame:
        frames = []
        offset = 0
        for r in self.results_history._results:
            tr = r.traces().copy()
            tr["iteration"] = tr["iteration"] + offset
            offset = int(tr["iteration"].max()) + (1 if r.method == "pfilter" else 0)
            frames.append(tr)
        return pd.concat(frames, ignore_index=True) if frames else pd.DataFrame()
