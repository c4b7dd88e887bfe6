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
restatement of the same algorithm with every host thread, on a bounded sample
of the workload, and reports the same metric.
"""

from __future__ import annotations

import argparse
import json
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
# algorithmic bytes per particle of the resample+propagate kernel (LG, dx=2):
# read parent log-weight 4 + parent state 8, write child state 8 + log-weight 4
RESPROP_BYTES = 24
SUM_BYTES = 4


def workload():
    import pypomp_b200 as pp

    m = pp.LG(T=T, Q=LG_Q, R=LG_R, key=0)
    return m


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
    """C restatement (oracle) on the host's cores, bounded sample of the workload."""
    from oracle import cora

    m = workload()
    st = m.to_struct()
    th = m.theta.to_array(m.canonical_param_names)
    F = F or nthreads
    t0 = time.perf_counter()
    cora.pfilter(1, 2, 2, np.repeat(th, F, 0), st.ys[:Tsample], J,
                 seeds=np.arange(F, dtype=np.uint64), nthreads=nthreads)
    dt = time.perf_counter() - t0
    return F * J * Tsample / dt, dt, F, Tsample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt, F, Ts = cpu_baseline(nthreads, Tsample=10, F=nthreads)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = f"{nthreads} of the 64 seeds x J={J} x first 10 of T={T} observations per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": NSEED * J * T / value * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "LG 2-D pfilter, T=1000, J=262144, 64 seeds (configs[1])",
                   "model": "LG", "global_batch": NSEED, "seq_len": T, "particles": J},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": sample,
                         "note": "reference JAX CPU path unavailable (jax not installed); "
                                 "C restatement of the same algorithm, all host threads"},
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
    seeds = (np.arange(NSEED, dtype=np.uint64) + np.uint64(1000 * rank))

    # ---- device-resident inputs, one descriptor, C-ABI calls -------------
    ys_d = torch.from_numpy(np.ascontiguousarray(st.ys)).to(dev)
    th_d = torch.from_numpy(th).to(dev)
    seeds_d = torch.from_numpy(seeds.view(np.int64).copy()).to(dev)
    ll_d = torch.zeros(NSEED, dtype=torch.float64, device=dev)
    d = _ffi.PfilterDesc()
    d.model = m.spec.ffi_model()
    d.J, d.F, d.T, d.U = J, NSEED, T, 1
    d.path = _ffi.PATH_STREAM
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
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    units_per_step = NSEED * J * T * world
    value = units_per_step * args.steps / (ms_max / 1e3)
    loglik = ll_d.cpu().numpy()
    launches_per_step = 1 + 2 * T

    # ---- per-kernel durations (CUDA events around each launch) -----------
    torch.cuda.synchronize()
    _ffi.profile_begin()
    step()
    prof = _ffi.profile_end()
    rp_ms, rp_n = prof["resample_propagate"]
    sum_ms, sum_n = prof["sum_lookback"]
    peak, peak_kind = peaks()
    rp_avg = rp_ms / rp_n
    achieved = RESPROP_BYTES * J * NSEED / (rp_avg / 1e3) / 1e9
    sum_avg = sum_ms / sum_n

    # ---- end to end through the public API (host inputs) -----------------
    struct = m.to_struct()
    thetas_host = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    keys_host = seeds.reshape(1, NSEED)
    F.pfilter(struct, thetas_host, J, keys_host)  # warm (allocator, module)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        out = F.pfilter(struct, thetas_host, J, keys_host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = units_per_step * e2e_steps / float(e2e_t.item())
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
        assert np.allclose(llp.cpu().numpy(), loglik[:Fp], rtol=1e-12), "plain path disagrees"
        plain = {"value": plain_value, "unit": UNIT, "filters_timed": Fp,
                 "ratio_batched_over_plain": value / world / plain_value}

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
            "config": {"workload": "LG 2-D pfilter, T=1000, J=262144, 64 seeds per GPU (configs[1])",
                       "model": "LG", "global_batch": NSEED * world, "seq_len": T, "particles": J,
                       "parallelism": f"replicas{world}", "path": "stream",
                       "l2": "inputs larger than L2 (state 2x64x262144x12 B = 403 MB per step)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "api": "pypomp_b200.functional.pfilter"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_resprop (resample + propagate)",
                         "algorithmic_bytes_per_particle": RESPROP_BYTES,
                         "avg_launch_ms": rp_avg, "peak_source": peak_kind,
                         "sum_kernel_avg_ms": sum_avg,
                         "step_bytes_per_particle_step": RESPROP_BYTES + SUM_BYTES},
            "cpu_baseline": cpu,
            "plain": plain,
            "clocks": clk.summary(),
            "gpu_launches": launches_per_step * args.steps,
            "loglik_mean": float(np.mean(loglik)),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_profile_case(args):
    """A small case of the same kernels for ncu captures: the headline model
    and J, 24 seeds (state 2 x 24 x 262144 x 12 B = 151 MB, larger than L2),
    the first 12 observations, one call."""
    import torch

    from pypomp_b200 import functional as F

    m = workload()
    st = m.to_struct()
    st.ys = st.ys[:12]
    th = np.repeat(m.theta.to_array(m.canonical_param_names), 24, axis=0).astype(np.float32)
    out = F.run_pfilter(st, th, np.arange(24, dtype=np.uint64), J, path=args.path)
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
    ap.add_argument("--profile-case", action="store_true",
                    help="run one small call of the same kernels (for ncu) and exit")
    ap.add_argument("--path", default="stream")
    args = ap.parse_args()
    if args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
