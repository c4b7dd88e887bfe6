"""Benchmark: batched particle filter throughput on B200 (particle-steps/s).

Workload (the headline configuration): the 2-D linear Gaussian model
(A = rot(0.2), Q = [[1,1e-4],[1e-4,1]]/100, R = [[1,.1],[.1,1]]/10, C = I,
X0 = 0), T = 1000 simulated observations, J = 262144 particles, 64
independent seeds per launch, float32 state, float64 log-likelihood sums.  One
"step" is one full batched filter over all 64 seeds (1.68e10 particle-steps).
Per-rank work is fixed (each rank runs its own 64 seeds): weak scaling, no
collective on the data path; ranks only meet for the timing barrier and the
max-over-ranks of the device time.

Printed JSON line: ``value`` is whole-job particle-steps/s with inputs resident
in HBM; ``e2e`` is the same metric through the public API
``pypomp_b200.functional.pfilter`` with host inputs (H2D of data, parameters
and keys, D2H of the log-likelihoods inside the timed region); ``roofline``
is for the dominant kernel (resample + propagate) from CUDA events around its
launches; ``cpu_baseline`` times the C restatement of the path on this host's
cores; ``plain`` times the one-filter-at-a-time baseline kernels.

``--impl reference`` times the reference's CPU path.  The reference (pypomp on
JAX) cannot run on this image (no jax), so the arm times the oracle's C
restatement of the path with every host thread, on a bounded sample of the
workload (a prefix of the observations for a subset of the seeds), and reports
the same metric and config.  The restatement uses this library's exact
arithmetic (fixed-point resampling CDF, polynomial exp / log), not the
reference's float32 running-sum CDF.  That arm builds its inputs from
``oracle/workloads.py`` and never loads the CUDA library.

Accuracy: the LG lines state the particle filter's log-likelihood error
against the exact FP64 Kalman log-likelihood of the same data
(``loglik_err_vs_kalman``: relative error of the mean over the filters, and
its z-score against the Monte Carlo standard error).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s pfilter & MOP grad vs plain kernel, same GPU, ≤1e-4 logLik err"
UNIT = "particle-steps/s"
J, T, NSEED = 262144, 1000, 64
LG_Q = np.array([[1.0, 1e-4], [1e-4, 1.0]]) / 100
LG_R = np.array([[1.0, 0.1], [0.1, 1.0]]) / 10
LG_A = np.array([[math.cos(0.2), -math.sin(0.2)], [math.sin(0.2), math.cos(0.2)]])
# algorithmic bytes per particle of the resample+propagate kernel (LG, dx=2):
# read parent log-weight 4 + parent state 8, write child state 8 + log-weight 4
RESPROP_BYTES = 24
SUM_BYTES = 4
# DRAM traffic of one k_resprop launch per particle, from an ncu capture of a
# 24-seed case (dram__bytes_read.sum + dram__bytes_write.sum = 109.1 MB for
# 6.29 M particles); traffic is proportional to the particles processed
RESPROP_TRAFFIC_PER_PARTICLE = 17.35
# DRAM traffic of one k_simulate launch per trajectory-step, from an ncu capture
# of LG 2-D, 1 parameter set x 65536 replicates x T = 200 (188.0 MB written +
# 37.0 MB read for 13.1 M trajectory-steps); the writes and the partial-sector
# reads both grow with the trajectory-steps written
SIM_TRAFFIC_PER_TRAJ_STEP = 225.0e6 / (65536 * 200)


def rank_seeds(rank: int) -> np.ndarray:
    """Each rank filters its own 64 seeds (weak scaling, disjoint streams)."""
    return np.arange(NSEED, dtype=np.uint64) + np.uint64(1000 * rank)


def max_over_ranks(x: float, dev) -> float:
    """The slowest rank's value (device time is reported as the max over ranks)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=dev)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank_step: float, world: int, steps: int, ms_max: float) -> float:
    """Units all ranks processed per second of the slowest rank's device time."""
    return units_per_rank_step * world * steps / (ms_max / 1e3)


def workload():
    import pypomp_b200 as pp

    m = pp.LG(T=T, Q=LG_Q, R=LG_R, key=0)
    return m


def headline_config(world: int) -> dict:
    """The workload's config, printed identically by both arms."""
    return {"workload": "LG 2-D pfilter, T=1000, J=262144, 64 seeds per GPU",
            "model": "LG", "global_batch": NSEED * world, "seq_len": T, "particles": J,
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (state 2x64x262144x12 B = 403 MB per step)"}


def kalman_loglik(ys, A, C, Q, R, X0) -> float:
    """Exact FP64 log-likelihood of the LG model (x0 ~ N(X0, Q) at t0, one
    transition before the first observation, so the filter starts from P = Q)."""
    ys = np.asarray(ys, dtype=np.float64)
    x = np.asarray(X0, dtype=np.float64).copy()
    P = np.asarray(Q, dtype=np.float64).copy()
    ll = 0.0
    for y in ys:
        xp, Pp = A @ x, A @ P @ A.T + Q
        S = C @ Pp @ C.T + R
        L = np.linalg.cholesky(S)
        v = y - C @ xp
        a = np.linalg.solve(L, v)
        ll -= 0.5 * (len(v) * math.log(2 * math.pi) + a @ a) + float(np.sum(np.log(np.diag(L))))
        K = np.linalg.solve(S, C @ Pp).T
        x, P = xp + K @ v, Pp - K @ C @ Pp
    return float(ll)


def loglik_error(logliks, exact: float) -> dict:
    """The filters' log-likelihood estimate against the exact value: the
    log-mean-exp over the filters (pypomp's logLik over replicates) with its
    jackknife standard error, its relative error and the z-score of the
    difference; the plain mean and sd of the estimates are listed beside."""
    from pypomp_b200.maths import logmeanexp, logmeanexp_se

    ll = np.asarray(logliks, dtype=np.float64)
    lme, se = float(logmeanexp(ll)), float(logmeanexp_se(ll))
    return {"kalman": exact, "pf_logmeanexp": lme, "se": se, "n_filters": int(ll.size),
            "rel_err": abs(lme - exact) / abs(exact),
            "z": (lme - exact) / se if se > 0 else None,
            "pf_mean": float(np.mean(ll)), "pf_sd": float(np.std(ll, ddof=1)) if ll.size > 1 else None}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples taken during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5).stdout
                self.samples.append([v.strip() for v in out.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def cpu_baseline(nthreads: int, Tsample: int = 40, F: int | None = None):
    """C restatement (oracle) on the host's cores, bounded sample of the
    workload: F seeds (one per thread) over the first Tsample observations."""
    from oracle import cora
    from oracle.workloads import headline_lg

    th, ys = headline_lg(T, seed=0)
    F = F or nthreads
    t0 = time.perf_counter()
    cora.pfilter(1, 2, 2, np.repeat(th[None], F, 0), ys[:Tsample], J,
                 seeds=np.arange(F, dtype=np.uint64), nthreads=nthreads)
    dt = time.perf_counter() - t0
    return F * J * Tsample / dt, dt, F, Tsample


def run_reference(args):
    """The reference arm: the C restatement on every host thread.  Each step
    filters one seed per thread over the first REF_T_SAMPLE observations (a few
    seconds of CPU work); ``ms_per_step`` is the time of that sample."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    Ts = args.ref_t
    times = []
    for i in range(args.warmup + args.steps):
        v, dt, F, _ = cpu_baseline(nthreads, Tsample=Ts, F=nthreads)
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    units = nthreads * J * Ts
    value = units * len(times) / total
    sample = (f"per step {nthreads} of the 64 seeds (one per thread) x J={J} x the first {Ts} of "
              f"T={T} observations = {units:.3g} particle-steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / len(times) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": headline_config(world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": sample,
                         "note": "the reference's JAX CPU path cannot run here (jax not installed); "
                                 "C restatement of the path with this library's exact arithmetic "
                                 "(fixed-point resampling CDF, polynomial exp / log), not the "
                                 "reference's float32 running-sum CDF; all host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args):
    import torch
    import torch.distributed as dist

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from pypomp_b200 import functional as F

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    m = workload()
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names), NSEED, axis=0).astype(np.float32)
    seeds = rank_seeds(rank)

    # ---- device-resident inputs, one descriptor, C-ABI calls -------------
    ys_d = torch.from_numpy(np.ascontiguousarray(st.ys)).to(dev)
    th_d = torch.from_numpy(th).to(dev)
    seeds_d = torch.from_numpy(seeds.view(np.int64).copy()).to(dev)
    ll_d = torch.zeros(NSEED, dtype=torch.float64, device=dev)
    d = _ffi.PfilterDesc()
    d.model = m.spec.ffi_model()
    d.J, d.F, d.T, d.U = J, NSEED, T, 1
    d.path = _ffi.PATH_STREAM
    d.tile = args.tile
    d.flags = (_ffi.F_GRAPH if args.graph else 0) | (_ffi.F_FAST if args.fast else 0)
    d.theta, d.ys, d.seeds, d.loglik = _ffi.ptr(th_d), _ffi.ptr(ys_d), _ffi.ptr(seeds_d), _ffi.ptr(ll_d)
    ws = torch.empty(_ffi.LIB.ppf_pfilter_workspace_bytes(d), dtype=torch.uint8, device=dev)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    stream = torch.cuda.current_stream(dev)

    def step():
        _ffi.check(_ffi.LIB.ppf_pfilter(d, stream.cuda_stream), "ppf_pfilter")

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream.cuda_stream), "warmup")

    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, dev)
    units_per_step = NSEED * J * T * world
    value = whole_job_rate(NSEED * J * T, world, args.steps, ms_max)
    loglik = ll_d.cpu().numpy()
    launches_per_step = 1 + 2 * T

    # ---- per-kernel durations (CUDA events around each launch) -----------
    torch.cuda.synchronize()
    _ffi.profile_begin()
    step()
    prof = _ffi.profile_end()
    rp_ms, rp_n = prof["resample_propagate"]
    sum_ms, sum_n = prof["weight_sum"]
    peak, peak_kind = peaks()
    rp_avg = rp_ms / rp_n
    achieved = RESPROP_BYTES * J * NSEED / (rp_avg / 1e3) / 1e9
    sum_avg = sum_ms / sum_n

    # ---- end to end through the public API (host inputs) -----------------
    struct = m.to_struct()
    thetas_host = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    keys_host = seeds.reshape(1, NSEED)
    F.pfilter(struct, thetas_host, J, keys_host, fast=args.fast)  # warm (allocator, module)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        out = F.pfilter(struct, thetas_host, J, keys_host, fast=args.fast)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = units_per_step * e2e_steps / max_over_ranks(e2e_s, dev)
    assert np.allclose(out["logLik"].ravel(), loglik, rtol=1e-12, equal_nan=True)
    h2d = struct.ys.nbytes + thetas_host.nbytes + keys_host.nbytes
    d2h = NSEED * 8

    # ---- plain (one filter at a time) baseline on the same GPU -----------
    plain = None
    if rank == 0 and not args.skip_plain:
        Fp = 2
        dp = _ffi.PfilterDesc()
        ctypes_copy = bytes(d)
        import ctypes

        ctypes.memmove(ctypes.addressof(dp), ctypes_copy, ctypes.sizeof(d))
        dp.F = Fp
        dp.path = _ffi.PATH_PLAIN
        wsp = torch.empty(_ffi.LIB.ppf_pfilter_workspace_bytes(dp), dtype=torch.uint8, device=dev)
        dp.workspace, dp.ws_bytes = _ffi.ptr(wsp), wsp.numel()
        llp = torch.zeros(Fp, dtype=torch.float64, device=dev)
        dp.loglik = _ffi.ptr(llp)
        _ffi.check(_ffi.LIB.ppf_pfilter(dp, stream.cuda_stream), "plain warmup")
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        _ffi.check(_ffi.LIB.ppf_pfilter(dp, stream.cuda_stream), "plain")
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        plain_value = Fp * J * T / (pms / 1e3)
        if not args.fast:   # the plain kernels use the exact arithmetic
            assert np.allclose(llp.cpu().numpy(), loglik[:Fp], rtol=1e-12), "plain path disagrees"
        plain = {"value": plain_value, "unit": UNIT, "filters_timed": Fp,
                 "ratio_batched_over_plain": value / world / plain_value}

    # ---- accuracy: the 64 log-likelihoods against the exact Kalman value ----
    kalman_err = loglik_error(loglik, kalman_loglik(st.ys, LG_A, np.eye(2), LG_Q, LG_R, np.zeros(2)))

    # ---- the same workload with PPF_F_FAST (SFU special functions) --------
    fast = None
    if rank == 0 and not args.fast and not args.skip_fast:
        import ctypes

        dfa = _ffi.PfilterDesc()
        ctypes.memmove(ctypes.addressof(dfa), bytes(d), ctypes.sizeof(d))
        dfa.flags = d.flags | _ffi.F_FAST
        llf = torch.zeros(NSEED, dtype=torch.float64, device=dev)
        dfa.loglik = _ffi.ptr(llf)

        def step_fast():
            _ffi.check(_ffi.LIB.ppf_pfilter(dfa, stream.cuda_stream), "ppf_pfilter (fast)")

        for _ in range(args.warmup):
            step_fast()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as fclk:
            f0.record(stream)
            for _ in range(args.steps):
                step_fast()
            f1.record(stream)
            torch.cuda.synchronize()
        fms = f0.elapsed_time(f1) / args.steps
        _ffi.profile_begin()
        step_fast()
        fprof = _ffi.profile_end()
        f_rp = fprof["resample_propagate"][0] / fprof["resample_propagate"][1]
        f_ach = RESPROP_BYTES * J * NSEED / (f_rp / 1e3) / 1e9
        fast = {"arithmetic": "fast (PPF_F_FAST: SFU Box-Muller and weight exponential, contraction)",
                "value": NSEED * J * T / (fms / 1e3), "unit": UNIT, "ms_per_step": fms,
                "roofline": {"kernel": "k_resprop_fast", "avg_launch_ms": f_rp, "achieved": f_ach,
                             "peak": peak, "unit": "GB/s", "frac": f_ach / peak},
                "sum_kernel_avg_ms": fprof["weight_sum"][0] / fprof["weight_sum"][1],
                "clocks": fclk.summary(),
                "loglik_err_vs_kalman": loglik_error(llf.cpu().numpy(), kalman_err["kalman"])}
        if plain is not None:
            fast["ratio_over_plain"] = fast["value"] / plain["value"]

    # ---- MOP-alpha value + gradient (the metric's second half) ------------
    mop = None
    if rank == 0 and not args.skip_mop:
        mop = mop_block(args)

    # ---- CPU baseline (rank 0, N=1) ---------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        nthreads = os.cpu_count() or 1
        v, dt, Fc, Ts = cpu_baseline(nthreads, Tsample=args.cpu_t)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"{Fc} seeds x J={J} x first {Ts} observations ({dt:.1f} s of CPU work)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": headline_config(world),
            "path": "stream", "cuda_graph": bool(args.graph),
            "arithmetic": "fast (PPF_F_FAST)" if args.fast else "exact (bit-identical with the C oracle)",
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "api": "pypomp_b200.functional.pfilter"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": RESPROP_TRAFFIC_PER_PARTICLE * J * NSEED,
                         "kernel": "k_resprop (resample + propagate)",
                         "algorithmic_bytes_per_particle": RESPROP_BYTES,
                         "avg_launch_ms": rp_avg, "peak_source": peak_kind,
                         "sum_kernel_avg_ms": sum_avg,
                         "step_bytes_per_particle_step": RESPROP_BYTES + SUM_BYTES,
                         "kernel_timing": "CUDA events around each launch of one extra step run "
                                          "without the graph; the two kernels' averages add up "
                                          "to a few per cent more than the graph-replayed step"},
            "cpu_baseline": cpu,
            "plain": plain,
            "clocks": clk.summary(),
            "gpu_launches": launches_per_step * args.steps,
            "loglik_err_vs_kalman": kalman_err,
            "fast": fast,
            "mop": mop,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# The other configurations (one JSON line each; not the headline line)
# ---------------------------------------------------------------------------

def _timed(fn, steps, warmup, stream):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, clk.summary()


def _line(args, workload, value, ms, extra):
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": {"workload": workload}}
    line.update(extra)
    print(json.dumps(line))


def run_c1(args):
    """LG 2-D, T=50, J=1000, one filter (resident path); the spread over 256 seeds
    is reported (the Kalman comparison lives in the tests)."""
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import functional as F

    m = pp.LG(T=50, Q=LG_Q, R=LG_R, key=0)
    st = m.to_struct()
    th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    stream = torch.cuda.current_stream()
    out = {}

    def fn():
        out["r"] = F.run_pfilter(st, th, np.array([1], np.uint64), 1000, path="resident", return_torch=True)

    ms, clk = _timed(fn, args.steps, args.warmup, stream)
    reps = F.run_pfilter(st, np.repeat(th, 256, 0), np.arange(256, dtype=np.uint64), 1000, path="resident")
    ll = reps["loglik"]
    err = loglik_error(ll, kalman_loglik(st.ys, LG_A, np.eye(2), LG_Q, LG_R, np.zeros(2)))
    _line(args, "LG 2-D pfilter, T=50, J=1000, one filter, resident path",
          1000 * 50 / (ms / 1e3), ms,
          {"e2e": {"value": 1000 * 50 / (ms / 1e3), "unit": UNIT, "api": "functional.run_pfilter",
                   "h2d_bytes_per_step": int(st.ys.nbytes + th.nbytes + 8), "d2h_bytes_per_step": 0},
           "loglik_err_vs_kalman": err, "clocks": clk, "roofline": None,
           "note": "one CTA; latency bound, no HBM traffic to speak of"})


def mop_block(args, steps=None, warmup=None):
    """SV MOP-alpha value + gradient, T=2000, J=65536, alpha=0.97, one parameter
    set: particle-steps/s over whole value+gradient calls (device-resident
    inputs, one call = forward filter + adjoint sweep), per-kernel GB/s from
    CUDA events around each launch (launched without the graph, which adds a
    few per cent per launch), and the roofline of the whole call at the
    algorithmic bytes of its kernels."""
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from pypomp_b200.functional import MopCall

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    Jm, Tm = 65536, 2000
    m = pp.SV(T=Tm, key=0)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(np.float32)
    call = MopCall(st, th, np.array([1], np.uint64), Jm, 0.97)
    if args.graph:
        call.d.flags |= _ffi.F_GRAPH
    stream = torch.cuda.current_stream()
    ms, clk = _timed(lambda: call.forward(grad=True), steps, warmup, stream)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in call.out.items()}
    _ffi.profile_begin()
    call.forward(grad=True)
    prof = _ffi.profile_end()
    value = Jm * Tm / (ms / 1e3)
    # algorithmic bytes per particle-step of each MOP kernel kind (SV, dx = 2):
    # forward resample+propagate 24 + ancestor 4 + first-child offset 4; sums 4;
    # recompute 8 + 4 + 8; adjoint 8 (x) + 4 (anc) + 4 (offset) + 12 (adjoint in)
    # + 12 (adjoint out).  The persistent form records its forward (sums and
    # resample+propagate of every step) as one launch and its adjoint sweep
    # (recompute and adjoint) as another.  Every kind touches each of the
    # J x T particle-steps once, so its GB/s is bytes x J x T / its total time.
    persistent = "mop_recompute" not in prof
    bytes_kind = {"resample_propagate": 32, "weight_sum": 4, "mop_forward": 36, "mop_recompute": 20,
                  "mop_adjoint": 60 if persistent else 40}
    peak, peak_kind = peaks()
    kern = {}
    for k, (tms, n) in prof.items():
        if n:
            e = {"launches": n, "total_ms": tms, "avg_ms": tms / n}
            if k in bytes_kind:
                e["GBps"] = bytes_kind[k] * Jm * Tm / (tms / 1e3) / 1e9
            kern[k] = e
    call_bytes = 92 * Jm * Tm
    return {"workload": "SV MOP-alpha value+grad, T=2000, J=65536, alpha=0.97, one parameter set",
            "value": value, "unit": UNIT, "ms_per_call": ms, "steps": steps, "warmup": warmup,
            "cuda_graph": bool(args.graph), "form": "persistent" if persistent else "per-step launches",
            "kernels": kern, "clocks": clk,
            "roofline": {"bound": "hbm", "achieved": call_bytes / (ms / 1e3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": call_bytes / (ms / 1e3) / 1e9 / peak,
                         "algorithmic_bytes_per_particle_step": 92, "peak_source": peak_kind,
                         "basis": "whole value+grad call"},
            "value_out": float(res["value"][0]), "grad_out": res["grad"][0].tolist(),
            "grad_finite": bool(np.all(np.isfinite(res["grad"])))}


def run_c3(args):
    """SV MOP-alpha value + gradient: T=2000, J=65536, alpha=0.97, one parameter set."""
    b = mop_block(args)
    _line(args, b["workload"], b["value"], b["ms_per_call"],
          {"e2e": None, "clocks": b["clocks"], "kernels": b["kernels"], "roofline": b["roofline"],
           "value_out": b["value_out"], "grad_out": b["grad_out"], "grad_finite": b["grad_finite"]})


def run_c4(args):
    """Ricker profile grid: 32 x 32 (log r, sigma) x J=16384, T=500, one launch."""
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from pypomp_b200 import functional as F

    Jr, Tr = 16384, 500
    m = pp.Ricker(T=Tr, key=0)
    st = m.to_struct()
    lr = np.linspace(3.0, 4.6, 32)
    sg = np.linspace(0.05, 0.8, 32)
    grid = np.array([[math.exp(a), b, 10.0, 7.0] for a in lr for b in sg], np.float32)
    Fg = grid.shape[0]
    stream = torch.cuda.current_stream()
    seeds = np.arange(Fg, dtype=np.uint64)
    res = {}
    for path in ("resident", "stream"):
        ms, clk = _timed(lambda: F.run_pfilter(st, grid, seeds, Jr, path=path, return_torch=True),
                         args.steps, args.warmup, stream)
        res[path] = (ms, clk)
    best = min(res, key=lambda k: res[k][0])
    ms, clk = res[best]
    value = Fg * Jr * Tr / (ms / 1e3)
    # the plain one-filter-at-a-time kernels on two of the grid points (the
    # same results, one filter after the other)
    Fp = 2
    pms, _ = _timed(lambda: F.run_pfilter(st, grid[:Fp], seeds[:Fp], Jr, path="plain", return_torch=True),
                    1, 1, stream)
    plain_value = Fp * Jr * Tr / (pms / 1e3)
    _line(args, "Ricker 32x32 (log r, sigma) grid x J=16384, T=500", value, ms,
          {"e2e": {"value": value, "unit": UNIT, "api": "functional.run_pfilter (host inputs)",
                   "h2d_bytes_per_step": int(grid.nbytes + st.ys.nbytes + seeds.nbytes),
                   "d2h_bytes_per_step": 0},
           "clocks": clk, "path": best,
           "paths_ms": {k: v[0] for k, v in res.items()},
           "plain": {"value": plain_value, "unit": UNIT, "filters_timed": Fp,
                     "ratio_batched_over_plain": value / plain_value},
           "roofline": {"bound": "issue", "achieved": None, "peak": None, "unit": None, "frac": None,
                        "traffic": None,
                        "note": "resident path keeps each swarm in shared memory for all T: "
                                "no HBM claim; HBM-equivalent 24 B/particle-step = "
                                f"{24 * value / 1e9:.0f} GB/s"}})


def run_c5(args):
    """Panel IF2 then MOP training on 128 Ricker units of uneven length.

    T_u ~ U{50..800}, log r_u ~ N(3.8, 0.2^2), shared sigma = 0.3, phi = 10,
    J = 8192, rw sd 0.02 with geometric cooling 0.5.  The job is M = 100 IF2
    iterations then 50 gradient steps; the bench times ``--steps`` of each
    (after ``--warmup`` untimed ones) and reports particle-steps/s, where one
    IF2 iteration or one training step processes sum(T_u) x J particle-steps.
    """
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.optim import Adam, LearningRate, RWSigma

    rng = np.random.default_rng(0)
    U, Jp = 128, 8192
    T_u = rng.integers(50, 801, size=U)
    logr = rng.normal(3.8, 0.2, size=U)
    units = {f"unit{u}": pp.Ricker(T=int(T_u[u]), r=math.exp(logr[u]), key=1000 + u) for u in range(U)}
    names = list(units)
    import pandas as pd

    shared = pd.DataFrame({"shared": [0.3, 10.0]}, index=["sigma", "phi"])
    spec = pd.DataFrame([np.exp(logr), np.full(U, 7.0)], index=["r", "N_0"], columns=names)
    pan = pp.PanelPomp(units, pp.PanelParameters({"shared": shared, "unit_specific": spec}))
    st = pan.to_struct()
    rw = RWSigma({n: 0.02 for n in pan.canonical_param_names}).geometric_cooling(0.5)
    sh = np.repeat(pan.theta.shared_array()[:, None, :], Jp, axis=1)
    un = np.repeat(pan.theta.unit_array(names)[:, None], Jp, axis=1)
    steps_units = int(T_u.sum()) * Jp
    stream = torch.cuda.current_stream()

    def timed(fn, n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        fn(n)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), time.perf_counter() - t0

    with ClockSampler(torch.cuda.current_device()) as clk:
        F.panel_mif(st, sh, un, rw, max(args.warmup, 1), Jp, np.array([1], np.uint64))
        mif_ms, mif_wall = timed(lambda n: F.panel_mif(st, sh, un, rw, n, Jp, np.array([2], np.uint64)),
                                 args.steps)
        F.panel_mif(st, sh, un, rw, max(args.warmup, 1), Jp, np.array([1], np.uint64), mode="parallel")
        par_ms, par_wall = timed(lambda n: F.panel_mif(st, sh, un, rw, n, Jp, np.array([2], np.uint64),
                                                       mode="parallel"), args.steps)
        eta = LearningRate({n: 0.01 for n in pan.canonical_param_names})
        s0, u0 = pan.theta.shared_array(), pan.theta.unit_array(names)
        F.panel_train(st, s0, u0, Jp, Adam(), max(args.warmup, 1), eta, 0.97, np.array([3], np.uint64),
                      chunk_size=U)
        tr_ms, tr_wall = timed(lambda n: F.panel_train(st, s0, u0, Jp, Adam(), n, eta, 0.97,
                                                        np.array([4], np.uint64), chunk_size=U), args.steps)
    # per unit: is the MOP gradient at the starting parameters finite?
    est_all = np.stack([m_.spec.to_est(m_.theta.to_array(m_.canonical_param_names))[0]
                        for m_ in units.values()])[None].astype(np.float32)
    pm = F.panel_mop(st, est_all, Jp, 0.97, np.arange(U, dtype=np.uint64)[None] + 77, grad=True)
    finite_u = np.all(np.isfinite(pm["grad"][0]), axis=-1)
    mif_rate = steps_units * args.steps / (mif_ms / 1e3)
    par_rate = steps_units * args.steps / (par_ms / 1e3)
    tr_rate = steps_units * args.steps / (tr_ms / 1e3)
    job_s = 100 * mif_ms / args.steps / 1e3 + 50 * tr_ms / args.steps / 1e3
    _line(args, "Ricker panel: 128 units, T_u in [50, 800], J=8192; IF2 then MOP train",
          mif_rate, mif_ms / args.steps,
          {"e2e": {"value": mif_rate, "unit": UNIT, "api": "functional.panel_mif (host inputs)",
                   "h2d_bytes_per_step": int(sh.nbytes + un.nbytes + st.ys.nbytes), "d2h_bytes_per_step": 0},
           "train": {"value": tr_rate, "unit": UNIT, "ms_per_step": tr_ms / args.steps,
                     "api": "functional.panel_train, chunk_size=U (one MOP call per step)",
                     "grad_finite_units": int(finite_u.sum()), "units": U,
                     "grad_finite_by_T_u": {"T_u<=150": int(finite_u[T_u <= 150].sum()),
                                            "of": int((T_u <= 150).sum()),
                                            "T_u>150": int(finite_u[T_u > 150].sum()),
                                            "of_long": int((T_u > 150).sum())},
                     "valid": bool(finite_u.all()),
                     "note": "the speed of the MOP calls only: along chaotic Ricker trajectories "
                             "(log r near 3.8) the pathwise MOP gradient overflows float32 on long "
                             "series, and the update then propagates NaN as the reference's would"},
           "mif_parallel": {"value": par_rate, "unit": UNIT, "ms_per_iteration": par_ms / args.steps,
                            "api": "functional.panel_mif(mode='parallel'): all 128 units in one batched "
                                   "perturbed-filter call per iteration, shared swarm recombined "
                                   "(not the reference's unit-by-unit semantics)"},
           "sum_T_u": int(T_u.sum()), "full_job_seconds_estimate": job_s,
           "full_job_seconds_estimate_parallel": 100 * par_ms / args.steps / 1e3 + 50 * tr_ms / args.steps / 1e3,
           "wall_s": {"mif": mif_wall, "mif_parallel": par_wall, "train": tr_wall}, "clocks": clk.summary(),
           "roofline": None,
           "note": "IF2 visits the units one after another (the shared swarm carries from unit to unit), "
                   "so each perturbed filter runs J=8192 particles = 4 tiles: launch- and latency-bound"})


def run_sim(args):
    """Simulation (ppf_simulate): LG 2-D, 4 parameter sets x 65536 replicates x
    T = 1000 (X 2.1 GB + Y 2.1 GB written per step, larger than L2), plus the
    Ricker model (Poisson draws) on the same shape as a second figure."""
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from pypomp_b200 import functional as F

    Fs, nsim, Ts = 4, 65536, 1000
    m = pp.LG(T=Ts, Q=LG_Q, R=LG_R, key=0)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names).astype(np.float32), Fs, 0)
    keys = np.arange(1, Fs + 1, dtype=np.uint64)
    stream = torch.cuda.current_stream()
    out = {}

    def fn():
        out["xy"] = F.simulate(st, th, nsim, keys, return_torch=True)

    ms, clk = _timed(fn, args.steps, args.warmup, stream)
    torch.cuda.synchronize()
    _ffi.profile_begin()
    fn()
    prof = _ffi.profile_end()
    k_ms, k_n = prof["simulate"]
    steps = Fs * nsim * Ts
    value = steps / (ms / 1e3)
    bytes_per_step = (2 + 2) * 4              # X (dx = 2) and Y (dy = 2) written, float32
    achieved = bytes_per_step * steps / (k_ms / k_n / 1e3) / 1e9
    peak, peak_kind = peaks()
    # end to end: host parameters in, both arrays back to host memory
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        X, Y = F.simulate(st, th, nsim, keys)
    e2e_s = (time.perf_counter() - t0) / max(1, args.steps // 2)
    rk = pp.Ricker(T=Ts, key=0)
    rth = np.repeat(rk.theta.to_array(rk.canonical_param_names).astype(np.float32), Fs, 0)
    rms, _ = _timed(lambda: F.simulate(rk.to_struct(), rth, nsim, keys, return_torch=True),
                    args.steps, args.warmup, stream)
    cpu = {}
    if not args.skip_cpu:
        from oracle import cora

        t0 = time.perf_counter()
        cora.simulate(1, 2, 2, th[:1], 256, Ts, keys[:1])
        cs = time.perf_counter() - t0
        cpu = {"value": 256 * Ts / cs, "unit": "trajectory-steps/s", "cores": 1, "kind": "port",
               "sample": "1 parameter set x 256 replicates x T=1000, oracle/ppf_oracle.c single thread"}
    print(json.dumps({
        "metric": "trajectory-steps/s (simulate)", "value": value, "unit": "trajectory-steps/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "LG 2-D simulate, 4 parameter sets x 65536 replicates x T=1000",
                   "l2": "outputs (4.2 GB per step) larger than L2"},
        "e2e": {"value": steps / e2e_s, "unit": "trajectory-steps/s", "api": "functional.simulate",
                "h2d_bytes_per_step": int(th.nbytes + keys.nbytes),
                "d2h_bytes_per_step": int(4 * Fs * nsim * ((Ts + 1) * 2 + Ts * 2))},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": SIM_TRAFFIC_PER_TRAJ_STEP * steps, "kernel": "k_simulate",
                     "peak_source": peak_kind},
        "ricker": {"value": steps / (rms / 1e3), "ms_per_step": rms, "unit": "trajectory-steps/s"},
        "cpu_baseline": cpu or None, "clocks": clk, "gpu_launches": k_n * args.steps}))


def run_pmcmc(args):
    """PMCMC: 8 chains of the Ricker model (T = 500, J = 4096), adaptive random
    walk; every iteration filters all chains in one batched launch replayed
    from a CUDA graph.  Reports particle-steps/s over whole iterations (host
    proposal and accept step included) and iterations/s."""
    import pypomp_b200 as pp
    from pypomp_b200 import functional as F
    from pypomp_b200.proposals import MVNRWAdaptive

    n, Jc, Tc = 8, 4096, 500
    m = pp.Ricker(T=Tc, key=0)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names), n, 0)
    prop = MVNRWAdaptive(rw_sd={"r": 0.02, "sigma": 0.02, "phi": 0.02}, scale_start=20, shape_start=20)
    keys = np.arange(1, n + 1, dtype=np.uint64)
    F.pmcmc(st, th, prop, max(args.warmup, 3), Jc, keys)          # warm-up: capture and first replays
    Mi = max(20, 10 * args.steps)
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        ll, lp, tr, acc = F.pmcmc(st, th, prop, Mi, Jc, keys)
        wall = time.perf_counter() - t0
    value = n * Jc * Tc * (Mi + 1) / wall
    print(json.dumps({
        "metric": "particle-steps/s (pmcmc)", "value": value, "unit": "particle-steps/s", "n_gpus": 1,
        "steps": Mi, "warmup": max(args.warmup, 3), "ms_per_step": wall / (Mi + 1) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "Ricker PMCMC, 8 chains x J=4096 x T=500, adaptive MVN random walk"},
        "e2e": {"value": value, "unit": "particle-steps/s", "api": "functional.pmcmc (host loop)",
                "h2d_bytes_per_step": int(n * (4 * 4 + 8)), "d2h_bytes_per_step": int(8 * n)},
        "iterations_per_s": (Mi + 1) / wall, "acceptance": (acc / Mi).tolist(),
        "roofline": None, "clocks": clk.summary(),
        "note": "wall clock of whole iterations; the filters run on the cluster path"}))


def run_profile_case(args):
    """A small case of the same kernels for ncu captures: the headline model
    and J, 24 seeds (state 2 x 24 x 262144 x 12 B = 151 MB, larger than L2),
    the first 12 observations, one call (``--fast``: the PPF_F_FAST kernels).
    ``--config sim`` and ``--config c5`` give small cases of the simulation
    and cluster-path kernels; ``c3`` the persistent MOP forward and adjoint
    (SV, T = 200, J = 65536); ``c4`` the shared-memory-resident filter (64
    Ricker filters, J = 16384, T = 50; ``--path stream`` for the streaming
    kernels on the same filters); ``plain`` the one-filter baseline
    kernels (LG 2-D, J = 262144, T = 12); ``if2`` the streaming IF2 kernels
    (128 Ricker filters, J = 8192, T = 50, as one iteration of the packed
    panel IF2); ``mopsteps`` the per-step MOP kernels (8 LG 2-D filters,
    J = 131072, T = 20, persistent forms off); ``wide`` the wide LG's streaming
    kernels (4 LG 9 x 9 filters, J = 262144, T = 6)."""
    import math

    import torch

    from pypomp_b200 import functional as F

    import pypomp_b200 as pp

    if args.config == "c3":
        m = pp.SV(T=200, key=0)
        th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(np.float32)
        r = F.run_mop(m.to_struct(), th, np.array([1], np.uint64), 65536, 0.97, grad=True)
        print("profile case MOP", r["value"], r["grad"])
        return
    if args.config == "mopsteps":
        m = pp.LG(T=20, Q=LG_Q, R=LG_R, key=0)
        th = m.spec.to_est(np.repeat(m.theta.to_array(m.canonical_param_names), 8, axis=0)).astype(np.float32)
        r = F.run_mop(m.to_struct(), th, np.arange(8, dtype=np.uint64), 131072, 0.97, grad=True, persistent=False)
        print("profile case MOP per-step", r["value"][:2])
        return
    if args.config == "wide":
        m = pp.LG(T=6, A=0.9 * np.eye(9), C=np.eye(9) + 0.1, Q=np.eye(9) * 0.05, R=np.eye(9) * 0.2 + 0.02, key=0)
        th = np.repeat(m.theta.to_array(m.canonical_param_names), 4, axis=0).astype(np.float32)
        r = F.run_pfilter(m.to_struct(), th, np.arange(4, dtype=np.uint64), 262144, path="stream")
        print("profile case wide LG", r["loglik"][:2])
        return
    if args.config == "c4":
        m = pp.Ricker(T=50, key=0)
        grid = np.array([[math.exp(a), b, 10.0, 7.0] for a in np.linspace(3.0, 4.6, 8)
                         for b in np.linspace(0.05, 0.8, 8)], np.float32)
        path = args.path or "resident"
        r = F.run_pfilter(m.to_struct(), grid, np.arange(64, dtype=np.uint64), 16384, path=path)
        print("profile case", path, r["loglik"][:2])
        return
    if args.config == "plain":
        m = workload()
        st = m.to_struct()
        st.ys = st.ys[:12]
        th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
        r = F.run_pfilter(st, th, np.array([3], np.uint64), J, path="plain")
        print("profile case plain", r["loglik"])
        return
    if args.config == "if2":
        m = pp.Ricker(T=50, key=0)
        st = m.to_struct()
        est = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(np.float32)
        swarm = torch.from_numpy(np.ascontiguousarray(np.repeat(est[:, :, None], 8192, axis=2).repeat(128, 0))).cuda()
        sig = np.full(4, 0.02, np.float32)
        r = F.run_perfilter(st, swarm, np.arange(128, dtype=np.uint64), 8192, sig, sig, np.full(50, 0.5, np.float32),
                            0.5, stream_only=True)
        torch.cuda.synchronize()
        print("profile case IF2", float(r["loglik"][0]))
        return

    if args.config == "sim":
        # k_simulate: LG 2-D, one parameter set x 65536 replicates x T = 200
        # (outputs 2 x 65536 x 201 x 8 B = 211 MB, larger than L2)
        m = pp.LG(T=200, Q=LG_Q, R=LG_R, key=0)
        th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
        X, Y = F.simulate(m.to_struct(), th, 65536, np.array([1], np.uint64), return_torch=True)
        torch.cuda.synchronize()
        print("profile case simulate", float(X[0, 0, -1, 0]))
        return
    if args.config == "c5":
        # k_cluster: first the pfilter variant on 4 Ricker filters (J = 8192,
        # T = 500), then the IF2 variant on one unit filter as in the panel IF2
        # job (same J and T, rw sd 0.02)
        m = pp.Ricker(T=500, key=0)
        st = m.to_struct()
        th = m.theta.to_array(m.canonical_param_names).astype(np.float32)
        out = F.run_pfilter(st, np.repeat(th, 4, axis=0), np.arange(4, dtype=np.uint64), 8192, path="cluster")
        est = m.spec.to_est(th).astype(np.float32)
        swarm = torch.from_numpy(np.ascontiguousarray(np.repeat(est[:, :, None], 8192, axis=2))).cuda()
        sig = np.full(4, 0.02, np.float32)
        res = F.run_perfilter(st, swarm, np.array([7], np.uint64), 8192, sig, sig, np.full(500, 0.5, np.float32), 0.5)
        torch.cuda.synchronize()
        print("profile case cluster logLik", out["loglik"][:2], float(res["loglik"][0]))
        return
    m = workload()
    st = m.to_struct()
    st.ys = st.ys[:12]
    th = np.repeat(m.theta.to_array(m.canonical_param_names), 24, axis=0).astype(np.float32)
    out = F.run_pfilter(st, th, np.arange(24, dtype=np.uint64), J, path=args.path or "stream", fast=args.fast)
    torch.cuda.synchronize()
    print("profile case logLik", out["loglik"][:2])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-t", type=int, default=40)
    ap.add_argument("--ref-t", type=int, default=50,
                    help="observations per step of the reference arm's sample")
    ap.add_argument("--skip-mop", action="store_true", help="leave the MOP value+grad block out")
    ap.add_argument("--skip-fast", action="store_true", help="leave the PPF_F_FAST block out")
    ap.add_argument("--fast", action="store_true",
                    help="PPF_F_FAST kernels (hardware special functions; statistically, not bitwise, "
                         "equal to the exact arithmetic)")
    ap.add_argument("--profile-case", action="store_true",
                    help="run one small call of the same kernels (for ncu) and exit")
    ap.add_argument("--path", default=None,
                    help="filter path of a --profile-case (default: stream; resident for c4)")
    ap.add_argument("--tile", type=int, default=0, help="stream-path tile (0 = automatic)")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch the step loop directly instead of replaying it as a CUDA graph")
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "sim", "pmcmc", "plain", "if2", "mopsteps",
                                                   "wide"],
                    help="c2 (default) is the headline line; c1/c3/c4/c5/sim/pmcmc print their own lines; "
                         "plain, if2, mopsteps and wide are --profile-case cases")
    args = ap.parse_args()
    if args.config in ("plain", "if2", "mopsteps", "wide") and not args.profile_case:
        ap.error(f"--config {args.config} is a --profile-case case")
    if args.config != "c2" and args.impl == "ours" and not args.profile_case:
        {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5, "sim": run_sim, "pmcmc": run_pmcmc}[args.config](args)
        return
    if args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
