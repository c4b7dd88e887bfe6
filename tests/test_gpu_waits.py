"""Bounded device-side waits give up with PPF_ETIMEOUT and leave the context usable.

The resampling kernel waits on the bulk copies of its parent rows, and the
persistent MOP kernels wait on each other's per-step words and at grid
barriers; each wait is bounded.  ``ppf_debug_set_wait_limit(0)`` makes every such
wait give up at its first check, on a many-tile case (8 filters x 128 tiles
of 2048 particles).  The call must come back promptly with PPF_ETIMEOUT from
``ppf_workspace_status``, and, with the limit restored, the next call on the
same workspace must agree bit for bit with the C oracle.  Nothing here faults
or hangs the GPU: a wait that gives up only sets the workspace's error word
(and still drains its own bulk copy before the kernel goes on).
"""

import time

import numpy as np
import pytest

from oracle import cora

pytestmark = pytest.mark.gpu
f32 = np.float32


def _setup(J, F, T):
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from tests.conftest import LG2_Q, LG2_R

    m = pp.LG(T=T, Q=LG2_Q, R=LG2_R, key=5)
    st = m.to_struct()
    th = np.repeat(m.theta.to_array(m.canonical_param_names), F, axis=0).astype(f32)
    seeds = np.arange(F, dtype=np.uint64) + 40
    dev = torch.device("cuda", 0)
    keep = {
        "ys": torch.from_numpy(np.ascontiguousarray(st.ys)).to(dev),
        "theta": torch.from_numpy(th).to(dev),
        "seeds": torch.from_numpy(seeds.view(np.int64).copy()).to(dev),
        "loglik": torch.zeros(F, dtype=torch.float64, device=dev),
        "anc": torch.zeros(F, T, J, dtype=torch.int32, device=dev),
    }
    d = _ffi.PfilterDesc()
    d.model = m.spec.ffi_model()
    d.J, d.F, d.T, d.U = J, F, T, 1
    d.path, d.tile = _ffi.PATH_STREAM, 2048
    d.flags = _ffi.F_SAVE_ANC
    d.theta, d.ys, d.seeds = _ffi.ptr(keep["theta"]), _ffi.ptr(keep["ys"]), _ffi.ptr(keep["seeds"])
    d.loglik, d.anc = _ffi.ptr(keep["loglik"]), _ffi.ptr(keep["anc"])
    ws = torch.empty(_ffi.LIB.ppf_pfilter_workspace_bytes(d), dtype=torch.uint8, device=dev)
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    keep["ws"] = ws
    return d, keep, st, th, seeds


def test_wait_limit_zero_times_out_promptly_then_recovers():
    import torch

    from pypomp_b200 import _ffi

    J, F, T = 262144, 8, 6
    d, keep, st, th, seeds = _setup(J, F, T)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    prev = _ffi.LIB.ppf_debug_set_wait_limit(0)
    try:
        t0 = time.perf_counter()
        assert _ffi.LIB.ppf_pfilter(d, stream) == _ffi.PPF_OK      # launches are fine
        status = _ffi.LIB.ppf_workspace_status(d.workspace, stream)
        dt = time.perf_counter() - t0
    finally:
        _ffi.LIB.ppf_debug_set_wait_limit(-1)
    assert prev == 1 << 22
    assert status == _ffi.PPF_ETIMEOUT, _ffi.error_string(status)
    assert dt < 10.0, dt
    assert _ffi.LIB.ppf_debug_set_wait_limit(-1) == 1 << 22
    # the same workspace, default limit: a normal call, bit for bit the oracle's
    assert _ffi.LIB.ppf_pfilter(d, stream) == _ffi.PPF_OK
    assert _ffi.LIB.ppf_workspace_status(d.workspace, stream) == _ffi.PPF_OK
    want = cora.pfilter(1, 2, 2, th, st.ys, J, seeds=seeds, anc=True, nthreads=8)
    assert np.array_equal(keep["anc"].cpu().numpy(), want["anc"])
    np.testing.assert_allclose(keep["loglik"].cpu().numpy(), want["loglik"], rtol=1e-12)


def test_persistent_mop_barriers_time_out_promptly_then_recover():
    """The persistent MOP forward and adjoint wait at grid barriers; with the
    limit at 0 every waiting CTA gives up at once, sets the abort word so the
    others stop at their next barrier, and the call reports PPF_ETIMEOUT.  The
    next call (the control words are cleared per call) is correct again."""
    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from pypomp_b200 import functional as F

    m = pp.SV(T=300, key=2)
    st = m.to_struct()
    th = m.spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    seeds = np.array([9], np.uint64)
    want = F.run_mop(st, th, seeds, 65536, 0.97, grad=True, persistent=False)
    prev = _ffi.LIB.ppf_debug_set_wait_limit(0)
    try:
        t0 = time.perf_counter()
        with pytest.raises(RuntimeError, match="timed out"):
            F.run_mop(st, th, seeds, 65536, 0.97, grad=True, persistent=True)
        dt = time.perf_counter() - t0
    finally:
        _ffi.LIB.ppf_debug_set_wait_limit(-1)
    assert prev == 1 << 22 and dt < 10.0, dt
    got = F.run_mop(st, th, seeds, 65536, 0.97, grad=True, persistent=True)
    assert np.array_equal(got["value"], want["value"])
    np.testing.assert_allclose(got["grad"], want["grad"], rtol=1e-9)
