"""``Pomp``: the object-oriented interface for the built-in CUDA models.

Mirrors the reference's ``Pomp`` methods on the hot path
(``pypomp/core/estimation_mixin.py:101`` ``pfilter``, ``:274`` ``mif``,
``:446`` ``train``) and its result tables (``pypomp/core/analysis_mixin.py``,
``pypomp/core/results/render.py:145-162``).  Methods keep their keyword
arguments, return ``None``, update ``self.theta`` and append a ``Result`` to
``self.results_history``.  ``results()`` has the columns
``theta_idx, logLik, se, <params>``.
"""

from __future__ import annotations

import time
from copy import deepcopy
from dataclasses import dataclass, field

import numpy as np
import pandas as pd

from . import random as pprandom
from .maths import logmeanexp, logmeanexp_se


class PompParameters:
    """A list of parameter dicts plus their log-likelihoods
    (``pypomp/core/parameters/pomp.py``; pandas/numpy instead of xarray)."""

    def __init__(self, theta, logLik=None):
        if isinstance(theta, dict):
            theta = [theta]
        self._list = [dict(t) for t in theta]
        self.logLik = None if logLik is None else np.asarray(logLik, dtype=float)

    def num_replicates(self) -> int:
        return len(self._list)

    def get_param_names(self):
        return list(self._list[0].keys()) if self._list else []

    def params(self, as_list: bool = True):
        return [dict(t) for t in self._list] if as_list else pd.DataFrame(self._list)

    def to_array(self, names) -> np.ndarray:
        return np.asarray([[t[n] for n in names] for t in self._list], dtype=np.float64)

    @classmethod
    def from_array(cls, arr, names):
        arr = np.atleast_2d(np.asarray(arr, dtype=float))
        return cls([{n: float(v) for n, v in zip(names, row)} for row in arr])

    def subset(self, idx):
        return PompParameters([self._list[i] for i in idx])

    def pruned(self, n: int = 1, refill: bool = True) -> "PompParameters":
        """The top ``n`` replicates by log-likelihood, repeated to the previous
        count with ``refill`` (``pypomp/core/parameters/base.py:138-181``)."""
        n_reps = self.num_replicates()
        if n_reps == 0:
            raise ValueError("No parameter sets available to prune.")
        if n < 1:
            raise ValueError("n must be at least 1.")
        ll = self.logLik
        if ll is None or np.all(np.isnan(ll)):
            raise ValueError("No valid log-likelihoods available to prune (all nan).")
        top = np.asarray(ll).argsort()[-n:][::-1]
        idx = np.tile(top, (n_reps + n - 1) // n)[:n_reps] if refill else top
        out = PompParameters([self._list[i] for i in idx])
        out.logLik = np.asarray(ll)[idx]
        return out

    def __len__(self):
        return len(self._list)

    def __repr__(self):
        return f"PompParameters({self._list}, logLik={self.logLik})"


@dataclass
class Result:
    method: str
    theta: PompParameters
    payload: dict
    config: dict = field(default_factory=dict)
    execution_time: float | None = None
    key: object = None

    def to_dataframe(self, ignore_nan: bool = False) -> pd.DataFrame:
        if self.method == "pfilter":
            arr = np.asarray(self.payload["logLiks"])
            logLik = np.atleast_1d(logmeanexp(arr, axis=-1, ignore_nan=ignore_nan))
            se = (logmeanexp_se(arr, axis=-1, ignore_nan=ignore_nan)
                  if arr.shape[-1] > 1 else np.full_like(logLik, np.nan))
            df = pd.DataFrame({"theta_idx": np.arange(len(self.theta)), "logLik": logLik,
                               "se": np.atleast_1d(se)})
            return pd.concat([df, pd.DataFrame(self.theta.params(as_list=True))], axis=1)
        if self.method == "pmcmc":
            # every iteration (pypomp/core/results/render.py:419-430)
            df = self._pmcmc_frame()
            return df.dropna() if ignore_nan else df
        # mif / train: final iteration of the trace
        tr = self.traces()
        last = tr[tr["iteration"] == tr["iteration"].max()].drop(columns=["iteration", "method"])
        return last.reset_index(drop=True)

    def _pmcmc_frame(self) -> pd.DataFrame:
        ll = np.asarray(self.payload["logLiks"])          # (n, M+1)
        lp = np.asarray(self.payload["log_prior"])        # (n, M+1)
        th = np.asarray(self.payload["traces"])           # (n, M+1, P)
        n, M1 = ll.shape
        df = pd.DataFrame({"theta_idx": np.repeat(np.arange(n), M1),
                           "iteration": np.tile(np.arange(M1), n),
                           "logLik": ll.reshape(-1), "log_prior": lp.reshape(-1)})
        for p, nm in enumerate(self.payload["param_names"]):
            df[nm] = th[:, :, p].reshape(-1)
        return df

    @property
    def acceptance_rate(self) -> np.ndarray:
        """Per-chain acceptance rate (pmcmc)."""
        acc = self.payload.get("accepts")
        if acc is None:
            return np.zeros(0)
        M = self.config.get("M")
        return np.asarray(acc, float) / float(M) if M else np.zeros(len(acc))

    def traces(self) -> pd.DataFrame:
        if self.method == "pmcmc":
            df = self._pmcmc_frame()
            df.insert(2, "method", "pmcmc")
            df.insert(4, "se", np.nan)
            return df
        if self.method == "pfilter":
            df = self.to_dataframe()
            df.insert(1, "iteration", 0)
            df.insert(2, "method", "pfilter")
            return df
        logliks = np.asarray(self.payload["logLiks"])      # (n, M+1)
        traces = np.asarray(self.payload["traces"])        # (n, M+1, P)
        names = self.payload["param_names"]
        rows = []
        n, M1 = logliks.shape
        for i in range(n):
            for m in range(M1):
                r = {"theta_idx": i, "iteration": m, "method": self.method,
                     "logLik": logliks[i, m], "se": np.nan}
                r.update({nm: traces[i, m, p] for p, nm in enumerate(names)})
                rows.append(r)
        return pd.DataFrame(rows)


class ResultsHistory:
    def __init__(self):
        self._results: list[Result] = []

    def add(self, r: Result):
        self._results.append(r)

    def __getitem__(self, i):
        return self._results[i]

    def __len__(self):
        return len(self._results)

    def results(self, index: int = -1, ignore_nan: bool = False) -> pd.DataFrame:
        return self._results[index].to_dataframe(ignore_nan=ignore_nan)

    def traces(self) -> pd.DataFrame:
        frames = []
        offset = 0
        for r in self._results:
            tr = r.traces().copy()
            tr["iteration"] = tr["iteration"] + offset
            offset = int(tr["iteration"].max()) + (1 if r.method == "pfilter" else 0)
            frames.append(tr)
        return pd.concat(frames, ignore_index=True) if frames else pd.DataFrame()

    def time(self) -> pd.DataFrame:
        """Execution time of every run (``results/history.py:38-54``)."""
        if not self._results:
            return pd.DataFrame()
        df = pd.DataFrame([{"method": r.method, "time": r.execution_time} for r in self._results])
        df.index.name = "history_index"
        return df


class ParTrans:
    """Parameter transform between the natural and the estimation scale
    (``pypomp/core/par_trans.py:70``).

    ``ParTrans()`` is the identity, as in the reference.  The built-in models
    carry their own default transform (logs / atanh, in their ``ModelSpec``).
    Assigning ``ParTrans()`` to ``Pomp.par_trans`` after construction behaves
    as it does in the reference: the host-side conversions (``to_est`` /
    ``from_est`` of the swarms, traces and results) become the identity, while
    the model mechanics keep the transform the model was built with (the
    reference binds it to the rinit/rproc/dmeas components when the ``Pomp``
    is constructed, ``pypomp/core/pomp.py:271-313``).  User-written transform
    functions cannot reach the device code, so they are refused.
    """

    def __init__(self, to_est=None, from_est=None):
        if to_est is not None or from_est is not None:
            raise NotImplementedError(
                "custom parameter transforms are not supported by the CUDA path; "
                "use the model's default transform or ParTrans() (identity)")
        self.identity = True

    def __repr__(self):
        return "ParTrans()"


class Pomp:
    """A partially observed Markov process on one of the built-in CUDA models."""

    @property
    def par_trans(self):
        """``ParTrans()`` when the host-side identity transform is active, else
        the model's default transform (represented by its ``ModelSpec``)."""
        return ParTrans() if self.spec.natural else self.spec

    @par_trans.setter
    def par_trans(self, value):
        from dataclasses import replace

        if isinstance(value, ParTrans):
            self.spec = replace(self.spec, natural=True)
        elif value is None or value is self.spec or getattr(value, "kind", None) == self.spec.kind:
            self.spec = replace(self.spec, natural=False)
        else:
            raise TypeError("par_trans must be a ParTrans instance")

    def __init__(self, spec, ys: pd.DataFrame, theta, t0: float = 0.0, fresh_key=None):
        self.spec = spec
        if not isinstance(ys, pd.DataFrame):
            ys = pd.DataFrame(np.asarray(ys, dtype=float),
                              index=np.arange(1, len(ys) + 1, dtype=float),
                              columns=list(spec.obsnames))
        self.ys = ys
        self.t0 = float(t0)
        self.theta = theta if isinstance(theta, PompParameters) else PompParameters(theta)
        self.fresh_key = None if fresh_key is None else pprandom.as_key(fresh_key)
        self.results_history = ResultsHistory()

    # -- reference-facing attributes --------------------------------------
    @property
    def canonical_param_names(self):
        return list(self.spec.param_names)

    @property
    def statenames(self):
        return list(self.spec.statenames)

    def to_struct(self):
        from .functional import PompStruct

        # C-contiguous (row-major [T][dy]): pandas hands out column-major views
        ys = np.ascontiguousarray(self.ys.to_numpy(dtype=np.float32, copy=True))
        return PompStruct(spec=self.spec, ys=ys,
                          times=self.ys.index.to_numpy(dtype=float), t0=self.t0)

    def _update_fresh_key(self, key=None):
        """``pypomp/core/pomp.py:391-408``: split the key, keep one half."""
        old_key = self.fresh_key if key is None else pprandom.as_key(key)
        if old_key is None:
            raise ValueError(
                "Both the key argument and the fresh_key attribute are None. "
                "At least one key must be given.")
        self.fresh_key, new_key = pprandom.split(old_key)
        return new_key, old_key

    def _prepare_theta_input(self, theta):
        if theta is None:
            return self.theta
        if isinstance(theta, dict) or isinstance(theta, list):
            theta = PompParameters(theta)
        if not isinstance(theta, PompParameters):
            raise TypeError("theta must be a PompParameters object or None")
        if set(theta.get_param_names()) != set(self.canonical_param_names):
            raise ValueError("theta parameter names must match canonical_param_names up to reordering")
        return theta

    # -- estimation ----------------------------------------------------------
    def pfilter(self, J: int, key=None, theta=None, thresh: float = 0.0, reps: int = 1,
                CLL: bool = False, ESS: bool = False, filter_mean: bool = False,
                prediction_mean: bool = False, track_time: bool = True) -> None:
        """Bootstrap particle filter (``pypomp/core/estimation_mixin.py:101-272``)."""
        from . import functional as F

        start = time.time()
        thresh = float(max(0.0, thresh))
        theta_in = deepcopy(self._prepare_theta_input(theta))
        theta_for_results = deepcopy(theta_in)
        new_key, old_key = self._update_fresh_key(key)
        if J < 1:
            raise ValueError("J should be greater than 0.")
        n = theta_in.num_replicates()
        thetas = theta_in.to_array(self.canonical_param_names)
        keys = pprandom.split(new_key, n * reps).reshape(n, reps)
        res = F.pfilter(self.to_struct(), thetas, J, keys, thresh, CLL, ESS, filter_mean, prediction_mean)
        logliks = res["logLik"]
        theta_in.logLik = logmeanexp(logliks, axis=-1)
        self.theta = theta_in
        payload = {"logLiks": logliks}
        for k in ("CLL", "ESS", "filter_mean", "prediction_mean"):
            if k in res:
                payload[k] = res[k]
        self.results_history.add(Result(
            method="pfilter", theta=theta_for_results, payload=payload,
            config={"J": J, "reps": reps, "thresh": thresh},
            execution_time=(time.time() - start) if track_time else None, key=old_key))

    def mif(self, J: int, M: int, rw_sd, key=None, theta=None, thresh: float = 0.0,
            n_monitors: int = 0, track_time: bool = True) -> None:
        """Iterated filtering 2 (``pypomp/core/estimation_mixin.py:274-445``).

        Starts every particle of replicate i at ``theta[i]``, runs
        ``functional.mif`` with one key per replicate (``split(new_key,
        n_reps)``), sets ``self.theta`` to the final swarm means with the
        last iteration's log-likelihoods, and records the traces
        (``logLik`` is NaN at iteration 0)."""
        from . import functional as F

        start = time.time()
        thresh = float(max(0.0, thresh))
        if set(rw_sd.param_names) != set(self.canonical_param_names):
            raise ValueError(
                "rw_sd.sigmas keys must match canonical_param_names up to reordering. "
                f"Got {sorted(rw_sd.param_names)}, expected {sorted(self.canonical_param_names)}.")
        theta_in = deepcopy(self._prepare_theta_input(theta))
        theta_for_results = deepcopy(theta_in)
        new_key, old_key = self._update_fresh_key(key)
        n = theta_in.num_replicates()
        if J < 1:
            raise ValueError("J should be greater than 0.")
        keys = pprandom.split(new_key, n)
        thetas = theta_in.to_array(self.canonical_param_names)
        swarms = np.repeat(thetas[:, None, :], J, axis=1)
        logliks, traces, _ = F.mif(self.to_struct(), swarms, rw_sd, M, J, keys, thresh, n_monitors)
        lls = np.concatenate([np.full((n, 1), np.nan), logliks], axis=1)
        self.theta = PompParameters.from_array(traces[:, M, :], self.canonical_param_names)
        self.theta.logLik = logliks[:, -1] if M > 0 else None
        self.results_history.add(Result(
            method="mif", theta=theta_for_results,
            payload={"logLiks": lls, "traces": traces, "param_names": self.canonical_param_names},
            config={"J": J, "M": M, "rw_sd": rw_sd, "thresh": thresh, "n_monitors": n_monitors},
            execution_time=(time.time() - start) if track_time else None, key=old_key))

    def train(self, J: int, M: int, eta, key=None, theta=None, optimizer=None, alpha: float = 0.97,
              thresh: float = 0.0, alpha_cooling: float = 1.0, n_monitors: int = 1,
              track_time: bool = True) -> None:
        """MOP-alpha gradient training (``pypomp/core/estimation_mixin.py:446-620``)."""
        from . import functional as F
        from .optim import Adam, LearningRate

        start = time.time()
        optimizer = optimizer or Adam()
        thresh = float(max(0.0, thresh))
        theta_in = deepcopy(self._prepare_theta_input(theta))
        theta_for_results = deepcopy(theta_in)
        n = theta_in.num_replicates()
        if J < 1:
            raise ValueError("J should be greater than 0")
        if not isinstance(eta, LearningRate):
            raise TypeError("eta must be a LearningRate object")
        new_key, old_key = self._update_fresh_key(key)
        keys = pprandom.split(new_key, n)
        th_est = self.spec.to_est(theta_in.to_array(self.canonical_param_names))
        nll, traces = F.train(self.to_struct(), th_est, J, optimizer, M, eta, alpha, keys,
                              alpha_cooling, thresh, n_monitors)
        nat = self.spec.from_est(traces.reshape(-1, traces.shape[-1])).reshape(traces.shape)
        self.theta = PompParameters.from_array(nat[:, -1, :], self.canonical_param_names)
        self.theta.logLik = -nll[:, -1]
        self.results_history.add(Result(
            method="train", theta=theta_for_results,
            payload={"logLiks": -nll, "traces": nat, "param_names": self.canonical_param_names},
            config={"J": J, "M": M, "eta": eta, "alpha": alpha, "thresh": thresh,
                    "alpha_cooling": alpha_cooling, "optimizer": optimizer},
            execution_time=(time.time() - start) if track_time else None, key=old_key))

    def _dpop_train(self, J: int, M: int, eta, optimizer=None, alpha: float = 0.8, alpha_cooling: float = 1.0,
                    process_weight_state: str | None = None, key=None, theta=None,
                    track_time: bool = True) -> None:
        """DPOP gradient training (``pypomp/core/estimation_mixin.py:637-820``,
        experimental there too).  ``process_weight_state`` names the state
        component that holds the transition log-weight of an interval.  Sets
        ``self.theta`` to the final parameters with the final objective as
        ``logLik`` and records a ``dpop_train`` result with the traces."""
        import warnings

        from . import functional as F
        from .optim import Adam, LearningRate

        warnings.warn("dpop_train is experimental and its API and behavior are subject to change.",
                      category=FutureWarning, stacklevel=2)
        start = time.time()
        optimizer = optimizer or Adam()
        theta_in = deepcopy(self._prepare_theta_input(theta))
        theta_for_results = deepcopy(theta_in)
        n = theta_in.num_replicates()
        if J < 1:
            raise ValueError("J should be greater than 0")
        if not isinstance(eta, LearningRate):
            raise TypeError("eta must be a LearningRate object")
        if process_weight_state is None:
            raise ValueError(
                "dpop_train requires a process-weight state. Please provide `process_weight_state` as the "
                "name of the state variable that accumulates the transition log-weight (e.g. 'logw').")
        if process_weight_state not in self.statenames:
            raise ValueError(f"State '{process_weight_state}' not found in statenames {self.statenames}")
        pwi = self.statenames.index(process_weight_state)
        new_key, old_key = self._update_fresh_key(key)
        keys = pprandom.split(new_key, n)
        th_est = self.spec.to_est(theta_in.to_array(self.canonical_param_names))
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", FutureWarning)
            nll, traces = F.dpop_train(self.to_struct(), th_est, J, optimizer, M, eta, alpha, pwi, keys,
                                       alpha_cooling)
        nat = self.spec.from_est(traces.reshape(-1, traces.shape[-1])).reshape(traces.shape)
        self.theta = PompParameters.from_array(nat[:, -1, :], self.canonical_param_names)
        self.theta.logLik = -nll[:, -1]
        self.results_history.add(Result(
            method="dpop_train", theta=theta_for_results,
            payload={"logLiks": -nll, "traces": nat, "param_names": self.canonical_param_names},
            config={"J": J, "M": M, "eta": eta, "alpha": alpha, "alpha_cooling": alpha_cooling,
                    "optimizer": optimizer, "process_weight_state": process_weight_state},
            execution_time=(time.time() - start) if track_time else None, key=old_key))

    # -- analysis ------------------------------------------------------------
    def pmcmc(self, J: int, M: int, proposal, dprior=None, key=None, theta=None, thresh: float = 0.0,
              track_time: bool = True) -> None:
        """Particle marginal Metropolis-Hastings (``pypomp/core/estimation_mixin.py:823-935``).

        One chain per parameter replicate of ``theta``, one key per chain
        split from the model's key.  Sets ``self.theta`` to the chains' final
        parameters with their last log-likelihoods and records a ``pmcmc``
        result: traces of ``logLik``, ``log_prior`` (natural scale, no
        Jacobian) and the parameters, plus accept counts."""
        from . import functional as F

        start = time.time()
        if J < 1:
            raise ValueError("J must be >= 1.")
        if M < 1:
            raise ValueError("M must be >= 1.")
        theta_in = deepcopy(self._prepare_theta_input(theta))
        theta_for_result = deepcopy(theta_in)
        n = theta_in.num_replicates()
        if n < 1:
            raise ValueError("pmcmc requires at least one starting parameter set.")
        new_key, old_key = self._update_fresh_key(key)
        names = self.canonical_param_names
        keys = pprandom.split(new_key, n)
        ll, lp, th, acc = F.pmcmc(self.to_struct(), theta_in.to_array(names), proposal, M, J, keys,
                                  thresh=thresh, dprior=dprior)
        self.theta = PompParameters.from_array(th[:, -1], names)
        self.theta.logLik = ll[:, -1]
        self.results_history.add(Result(
            method="pmcmc", theta=theta_for_result,
            payload={"logLiks": ll, "log_prior": lp, "traces": th, "param_names": names, "accepts": acc},
            config={"M": M, "J": J}, execution_time=(time.time() - start) if track_time else None,
            key=old_key))

    def simulate(self, key=None, theta=None, times=None, nsim: int = 1, as_pomp: bool = False):
        """Simulated states and observations (``pypomp/core/estimation_mixin.py:1101-1222``).

        Returns ``(states_df, obs_df)``, long-format DataFrames with columns
        ``theta_idx``, ``sim``, ``time`` and one column per state (the initial
        state at ``t0`` included) or observation variable; with ``as_pomp`` a
        copy of the model whose ``ys`` is the first replicate of the first
        parameter set (``nsim`` forced to 1).  One key per parameter set,
        split from the model's key as the reference does."""
        import warnings

        from . import functional as F

        if as_pomp:
            if nsim > 1:
                warnings.warn(
                    "as_pomp is True, but nsim > 1. Only 1 simulation will be performed as_pomp overrides nsim.",
                    UserWarning, stacklevel=2)
            nsim = 1
        theta_in = self._prepare_theta_input(theta)
        thetas = theta_in.to_array(self.canonical_param_names)
        new_key, _ = self._update_fresh_key(key)
        keys = pprandom.split(new_key, thetas.shape[0])
        times_array = self.ys.index.to_numpy(dtype=float) if times is None else np.asarray(times, dtype=float)
        X, Y = F.simulate(self.to_struct(), thetas, nsim, keys, times=times_array)

        def to_long(vals, times_vec, columns):
            n_theta, n_sim, n_time, n_feat = vals.shape
            df = pd.DataFrame(vals.reshape(n_theta * n_sim * n_time, n_feat), columns=pd.Index(columns))
            df.insert(0, "time", np.tile(np.asarray(times_vec, dtype=float), n_theta * n_sim))
            df.insert(0, "sim", np.tile(np.repeat(np.arange(n_sim), n_time), n_theta))
            df.insert(0, "theta_idx", np.repeat(np.arange(n_theta), n_sim * n_time))
            return df

        times0 = np.concatenate([np.array([self.t0]), times_array])
        states = to_long(X, times0, self.statenames)
        obs = to_long(Y, times_array, list(self.ys.columns))
        if as_pomp:
            first = obs[(obs["theta_idx"] == 0) & (obs["sim"] == 0)]
            ys = pd.DataFrame(first.drop(columns=["theta_idx", "sim", "time"]).to_numpy(),
                              index=pd.Index(first["time"].to_numpy()), columns=self.ys.columns)
            out = deepcopy(self)
            out.ys = ys
            out.theta = theta_in.subset([0])
            return out
        return states, obs

    def results(self, index: int = -1, ignore_nan: bool = False) -> pd.DataFrame:
        return self.results_history.results(index=index, ignore_nan=ignore_nan)

    def traces(self) -> pd.DataFrame:
        return self.results_history.traces()

    def _per_step(self, key: str, index: int, average: bool) -> pd.DataFrame:
        r = self.results_history[index]
        if key not in r.payload:
            return pd.DataFrame()
        vals = np.asarray(r.payload[key])                  # (n_theta, reps, T)
        times = self.ys.index.to_numpy(dtype=float)
        n, reps, T = vals.shape
        if average:
            agg = logmeanexp(vals, axis=1) if key == "CLL" else vals.mean(axis=1)
            return pd.DataFrame({"theta_idx": np.repeat(np.arange(n), T), "time": np.tile(times, n),
                                 key: agg.reshape(-1)})
        return pd.DataFrame({"theta_idx": np.repeat(np.arange(n), reps * T),
                             "rep": np.tile(np.repeat(np.arange(reps), T), n),
                             "time": np.tile(times, n * reps), key: vals.reshape(-1)})

    def CLL(self, index: int = -1, average: bool = False) -> pd.DataFrame:
        """Conditional log-likelihoods of a pfilter run with ``CLL=True`` as a tidy
        frame (``theta_idx``, ``rep``, ``time``, ``CLL``); ``average`` takes the
        log-mean-exp over replicates (``pypomp/core/results/render.py:77-95``)."""
        return self._per_step("CLL", index, average)

    def ESS(self, index: int = -1, average: bool = False) -> pd.DataFrame:
        """Effective sample sizes of a pfilter run with ``ESS=True`` (columns as
        :meth:`CLL`); ``average`` takes the mean over replicates."""
        return self._per_step("ESS", index, average)

    def time(self) -> pd.DataFrame:
        return self.results_history.time()

    def prune(self, n: int = 1, refill: bool = True) -> None:
        """Keep the top ``n`` parameter sets by log-likelihood (``analysis_mixin.py:134-150``)."""
        self.theta = self.theta.pruned(n=n, refill=refill)
