"""The reference arm of bench.py on the CPU.

``bench.py --impl reference`` times the CPU implementation of the path (the C
restatement, since the reference's JAX path cannot be installed) on the same
metric, unit and config as the CUDA arm, and prints one JSON line whose
``ms_per_step`` is the time of the sample it actually ran.  It builds its
inputs without the product package, so the CUDA library is never loaded in
that process.  Under a multi-rank launch only rank 0 works and prints; the
other ranks exit 0.
"""

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


_WRAP = ("import runpy, sys; sys.argv = ['bench.py'] + sys.argv[1:]; "
         "runpy.run_path('bench.py', run_name='__main__'); "
         "maps = open('/proc/self/maps').read(); "
         "print('LOADED', 'pypomp_b200' in sys.modules, 'libppf.so' in maps)")


def _run(env_extra, *extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "-c", _WRAP, "--impl", "reference", "--steps", "1", "--warmup", "3",
                           "--ref-t", "8", *extra],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    sys.path.insert(0, str(ROOT))
    import bench

    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"] == bench.headline_config(1)
    # ms_per_step is the sample actually timed: one seed per thread over 8 observations
    cb = d["cpu_baseline"]
    assert abs(d["value"] * d["ms_per_step"] / 1e3 - cb["cores"] * bench.J * 8) < 1e-6 * d["value"]
    assert "LOADED False False" in r.stdout
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_inputs_equal_the_product_workload():
    """oracle/workloads.py rebuilds the headline LG data and parameters exactly."""
    sys.path.insert(0, str(ROOT))
    import numpy as np

    import bench
    from oracle.workloads import headline_lg

    m = bench.workload()
    th, ys = headline_lg(bench.T, seed=0)
    assert np.array_equal(m.to_struct().ys, ys)
    assert np.array_equal(m.theta.to_array(m.canonical_param_names).astype(np.float32)[0], th)


def test_bench_kalman_equals_the_oracle_kalman():
    sys.path.insert(0, str(ROOT))
    import numpy as np

    import bench
    from oracle import kalman
    from oracle.workloads import headline_lg

    th, ys = headline_lg(200, seed=3)
    A, C, Q, R, X0 = kalman.lg_matrices(th.astype(np.float64), 2, 2)
    want = kalman.kalman_loglik(ys, A, C, Q, R, X0)
    got = bench.kalman_loglik(ys, bench.LG_A, np.eye(2), bench.LG_Q, bench.LG_R, np.zeros(2))
    assert abs(got - want) < 1e-5 * abs(want)
    err = bench.loglik_error(np.full(4, got) + np.array([0.01, -0.01, 0.02, -0.02]), got)
    assert err["rel_err"] < 1e-4 and err["n_filters"] == 4
