"""The C-ABI library loads and exports every symbol include/*.h declares (CPU)."""

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        # only extern "C" function declarations of the public ABI (ppf_*)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(ppf_\w+)\s*\(", text, re.M):
            syms.add(m.group(1))
    return syms


def test_library_exports_declared_symbols():
    from pypomp_b200 import _ffi

    out = subprocess.run(["nm", "-D", "--defined-only", _ffi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(ppf_\w+)", out))
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    missing = declared - exported
    assert not missing, f"declared but not exported: {missing}"
    assert set(_ffi.EXPORTED) <= exported


def test_error_strings_and_version():
    from pypomp_b200 import _ffi

    assert _ffi.error_string(_ffi.PPF_OK) == "ok"
    assert "timed out" in _ffi.error_string(_ffi.PPF_ETIMEOUT)
    assert "sm_100a" in _ffi.version()


def test_workspace_size_is_host_only():
    from pypomp_b200 import _ffi

    d = _ffi.PfilterDesc()
    d.model = _ffi.PpfModel(_ffi.MODEL_LG, 2, 2, 16, 0.0, 0)
    d.J, d.F, d.T, d.U = 262144, 64, 1000, 1
    d.path = _ffi.PATH_STREAM
    n = _ffi.LIB.ppf_pfilter_workspace_bytes(d)
    # X and W double-buffered: 2 * 64 * 262144 * (2 + 1) * 4 bytes, the run
    # prefixes (8 bytes per 4 particles), plus control
    assert n >= 2 * 64 * 262144 * 12 + 64 * 262144 * 2
    assert n < 2 * 64 * 262144 * 12 + 64 * 262144 * 2 + (1 << 24)


def test_validation_messages_without_gpu(lg2d):
    from pypomp_b200 import functional as F

    with pytest.raises(ValueError, match="J should be greater than 0"):
        lg2d.pfilter(J=0, key=1)
    st = lg2d.to_struct()
    th = lg2d.theta.to_array(lg2d.canonical_param_names)
    with pytest.raises((ValueError, RuntimeError)):
        F.run_pfilter(st, th, np.array([1], np.uint64), 0)


def test_simulate_validation_without_gpu():
    """ppf_simulate rejects bad descriptors before touching the device."""
    from pypomp_b200 import _ffi

    d = _ffi.SimulateDesc()
    d.model = _ffi.PpfModel(_ffi.MODEL_RICKER, 1, 1, 4, 0.0, 0)
    d.F, d.nsim, d.T = 0, 10, 5
    assert _ffi.LIB.ppf_simulate(d, None) == _ffi.PPF_EINVAL
    d.F, d.nsim = 1, 0
    assert _ffi.LIB.ppf_simulate(d, None) == _ffi.PPF_EINVAL
    d.nsim = 10
    assert _ffi.LIB.ppf_simulate(d, None) == _ffi.PPF_EINVAL      # null pointers
    d.model = _ffi.PpfModel(_ffi.MODEL_RICKER, 1, 1, 3, 0.0, 0)   # wrong parameter count
    assert _ffi.LIB.ppf_simulate(d, None) == _ffi.PPF_EINVAL


def test_wait_limit_hook_is_host_only():
    """ppf_debug_set_wait_limit only changes a host-side setting (no GPU work):
    it returns the previous limit, restores the default for negative values
    and clamps larger ones to it."""
    from pypomp_b200 import _ffi

    default = 1 << 22
    assert _ffi.LIB.ppf_debug_set_wait_limit(5) == default
    assert _ffi.LIB.ppf_debug_set_wait_limit(1 << 40) == 5
    assert _ffi.LIB.ppf_debug_set_wait_limit(-1) == default
    assert _ffi.LIB.ppf_debug_set_wait_limit(-1) == default


def test_dpop_descriptor_validation_without_gpu():
    """ppf_mop with PPF_F_DPOP refuses a process-weight index outside the
    state before touching the device; the descriptor carries the index after
    the workspace fields, as include/ppf.h declares it."""
    import ctypes

    from pypomp_b200 import _ffi

    assert _ffi.MopDesc.process_weight_index.offset == _ffi.MopDesc.ws_bytes.offset + ctypes.sizeof(ctypes.c_size_t)
    d = _ffi.MopDesc()
    d.model = _ffi.PpfModel(_ffi.MODEL_LG, 2, 2, 16, 0.0, 0)
    d.J, d.F, d.T, d.U = 100, 1, 5, 1
    d.alpha = 0.5
    buf = (ctypes.c_float * 64)()
    d.theta = d.ys = d.value = ctypes.addressof(buf)
    d.seeds = ctypes.addressof(buf)
    d.flags = _ffi.F_DPOP
    for bad in (-1, 2, 7):
        d.process_weight_index = bad
        assert _ffi.LIB.ppf_mop(d, None) == _ffi.PPF_EINVAL
        assert _ffi.LIB.ppf_mop_backward(d, None, None) == _ffi.PPF_EINVAL
