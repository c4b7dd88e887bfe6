"""ctypes binding of libppf.so (the C ABI declared in ``include/ppf.h``).

This is the seam where pypomp's jitted XLA programs are replaced: the
functional layer builds a descriptor of device pointers (torch tensors are
used only to own device memory and to name the stream) and calls the CUDA
library.  There is no CPU fallback: importing this module on a machine where
the library was not built raises ``ImportError``, and calling it without a
CUDA device raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libppf.so"

PPF_OK, PPF_EINVAL, PPF_ECUDA, PPF_ETIMEOUT, PPF_EUNSUPPORTED, PPF_EINTERNAL, PPF_ESCRATCH = 0, 1, 2, 3, 4, 5, 6
NOALLOC_SCRATCH_BYTES = 16 << 20
PPF_MAX_J = 1 << 21
MODEL_LG, MODEL_SV, MODEL_RICKER = 1, 2, 3

F_CLL = 1 << 0
F_ESS = 1 << 1
F_FMEAN = 1 << 2
F_PMEAN = 1 << 3
F_INJECT = 1 << 4
F_SAVE_ANC = 1 << 5
F_SAVE_W = 1 << 6
F_EST = 1 << 7
F_NATURAL = 1 << 8
F_GRAPH = 1 << 9
F_NO_PERSIST = 1 << 11
F_FAST = 1 << 12
F_DPOP = 1 << 13
F_NO_CLUSTER = 1 << 10

PATH_AUTO, PATH_PLAIN, PATH_STREAM, PATH_RESIDENT, PATH_CLUSTER = 0, 1, 2, 3, 4
PATHS = {"auto": PATH_AUTO, "plain": PATH_PLAIN, "stream": PATH_STREAM, "resident": PATH_RESIDENT,
         "cluster": PATH_CLUSTER}

# Every extern "C" symbol include/*.h declares; tests check the library exports them.
EXPORTED = (
    "ppf_pfilter_workspace_bytes",
    "ppf_pfilter",
    "ppf_mop_workspace_bytes",
    "ppf_mop",
    "ppf_mop_backward",
    "ppf_perfilter_workspace_bytes",
    "ppf_perfilter",
    "ppf_autotune",
    "ppf_workspace_status",
    "ppf_pfilter_noalloc",
    "ppf_simulate",
    "ppf_profile_begin",
    "ppf_debug_set_wait_limit",
    "ppf_profile_end",
    "ppf_error_string",
    "ppf_version",
)

_vp = ctypes.c_void_p


class PpfModel(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("dx", ctypes.c_int32),
        ("dy", ctypes.c_int32),
        ("n_params", ctypes.c_int32),
        ("dt", ctypes.c_float),
        ("reserved", ctypes.c_int32),
    ]


class PfilterDesc(ctypes.Structure):
    _fields_ = [
        ("model", PpfModel),
        ("J", ctypes.c_int32),
        ("F", ctypes.c_int32),
        ("T", ctypes.c_int32),
        ("U", ctypes.c_int32),
        ("path", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("thresh", ctypes.c_float),
        ("tile", ctypes.c_int32),
        ("theta", _vp),
        ("ys", _vp),
        ("ycon", _vp),
        ("unit", _vp),
        ("T_u", _vp),
        ("seeds", _vp),
        ("inj_z0", _vp),
        ("inj_z", _vp),
        ("inj_u", _vp),
        ("loglik", _vp),
        ("cll", _vp),
        ("ess", _vp),
        ("fmean", _vp),
        ("pmean", _vp),
        ("anc", _vp),
        ("logw", _vp),
        ("workspace", _vp),
        ("ws_bytes", ctypes.c_size_t),
    ]


class MopDesc(ctypes.Structure):
    _fields_ = [
        ("model", PpfModel),
        ("J", ctypes.c_int32),
        ("F", ctypes.c_int32),
        ("T", ctypes.c_int32),
        ("U", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("alpha", ctypes.c_float),
        ("ckpt_every", ctypes.c_int32),
        ("theta", _vp),
        ("ys", _vp),
        ("ycon", _vp),
        ("unit", _vp),
        ("T_u", _vp),
        ("seeds", _vp),
        ("inj_z0", _vp),
        ("inj_z", _vp),
        ("inj_u", _vp),
        ("value", _vp),
        ("grad", _vp),
        ("anc", _vp),
        ("workspace", _vp),
        ("ws_bytes", ctypes.c_size_t),
        ("process_weight_index", ctypes.c_int32),
    ]


class PerfilterDesc(ctypes.Structure):
    _fields_ = [
        ("model", PpfModel),
        ("J", ctypes.c_int32),
        ("F", ctypes.c_int32),
        ("T", ctypes.c_int32),
        ("U", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("thresh", ctypes.c_float),
        ("swarm_in", _vp),
        ("swarm_out", _vp),
        ("rw_sig", _vp),
        ("rw_sig0", _vp),
        ("cool", _vp),
        ("cool0", _vp),
        ("ys", _vp),
        ("ycon", _vp),
        ("unit", _vp),
        ("T_u", _vp),
        ("seeds", _vp),
        ("inj_zp0", _vp),
        ("inj_zp", _vp),
        ("inj_z0", _vp),
        ("inj_z", _vp),
        ("inj_u", _vp),
        ("loglik", _vp),
        ("cll", _vp),
        ("anc", _vp),
        ("workspace", _vp),
        ("ws_bytes", ctypes.c_size_t),
    ]


class SimulateDesc(ctypes.Structure):
    _fields_ = [
        ("model", PpfModel),
        ("F", ctypes.c_int32),
        ("nsim", ctypes.c_int32),
        ("T", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("theta", _vp),
        ("seeds", _vp),
        ("X", _vp),
        ("Y", _vp),
    ]


class PpfError(RuntimeError):
    """A non-zero return code from libppf.so."""

    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {error_string(code)} (code {code})")


def _load():
    if not _LIB_PATH.exists():
        raise ImportError(
            f"libppf.so not found at {_LIB_PATH}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` "
            "(the CUDA library is required: there is no CPU fallback)"
        )
    lib = ctypes.CDLL(str(_LIB_PATH))
    lib.ppf_pfilter_workspace_bytes.argtypes = [ctypes.POINTER(PfilterDesc)]
    lib.ppf_pfilter_workspace_bytes.restype = ctypes.c_size_t
    lib.ppf_pfilter.argtypes = [ctypes.POINTER(PfilterDesc), _vp]
    lib.ppf_pfilter.restype = ctypes.c_int
    lib.ppf_mop_workspace_bytes.argtypes = [ctypes.POINTER(MopDesc)]
    lib.ppf_mop_workspace_bytes.restype = ctypes.c_size_t
    lib.ppf_mop.argtypes = [ctypes.POINTER(MopDesc), _vp]
    lib.ppf_mop.restype = ctypes.c_int
    lib.ppf_mop_backward.argtypes = [ctypes.POINTER(MopDesc), _vp, _vp]
    lib.ppf_mop_backward.restype = ctypes.c_int
    lib.ppf_perfilter_workspace_bytes.argtypes = [ctypes.POINTER(PerfilterDesc)]
    lib.ppf_perfilter_workspace_bytes.restype = ctypes.c_size_t
    lib.ppf_perfilter.argtypes = [ctypes.POINTER(PerfilterDesc), _vp]
    lib.ppf_perfilter.restype = ctypes.c_int
    lib.ppf_pfilter_noalloc.argtypes = [ctypes.POINTER(PfilterDesc), _vp]
    lib.ppf_pfilter_noalloc.restype = ctypes.c_int
    lib.ppf_autotune.argtypes = [ctypes.POINTER(PfilterDesc), _vp, ctypes.POINTER(ctypes.c_int)]
    lib.ppf_autotune.restype = ctypes.c_int
    lib.ppf_simulate.argtypes = [ctypes.POINTER(SimulateDesc), _vp]
    lib.ppf_simulate.restype = ctypes.c_int
    lib.ppf_workspace_status.argtypes = [_vp, _vp]
    lib.ppf_workspace_status.restype = ctypes.c_int
    lib.ppf_debug_set_wait_limit.argtypes = [ctypes.c_longlong]
    lib.ppf_debug_set_wait_limit.restype = ctypes.c_longlong
    lib.ppf_profile_begin.argtypes = []
    lib.ppf_profile_begin.restype = ctypes.c_int
    lib.ppf_profile_end.argtypes = [_vp, _vp, ctypes.c_int]
    lib.ppf_profile_end.restype = ctypes.c_int
    lib.ppf_error_string.argtypes = [ctypes.c_int]
    lib.ppf_error_string.restype = ctypes.c_char_p
    lib.ppf_version.argtypes = []
    lib.ppf_version.restype = ctypes.c_char_p
    return lib


LIB = _load()
LIB_PATH = str(_LIB_PATH)


KIND_NAMES = ("init", "weight_sum", "resample_propagate", "resident", "plain_step",
              "mop_forward", "mop_recompute", "mop_adjoint", "if2", "cluster", "simulate")


def profile_begin() -> None:
    check(LIB.ppf_profile_begin(), "ppf_profile_begin")


def profile_end() -> dict:
    """{kind name: (total ms, launches)} for the calls since profile_begin()."""
    import numpy as np

    ms = np.zeros(16, np.float64)
    cnt = np.zeros(16, np.int32)
    check(LIB.ppf_profile_end(ms.ctypes.data, cnt.ctypes.data, 16), "ppf_profile_end")
    return {KIND_NAMES[i]: (float(ms[i]), int(cnt[i])) for i in range(len(KIND_NAMES)) if cnt[i]}


def error_string(code: int) -> str:
    return LIB.ppf_error_string(int(code)).decode()


def version() -> str:
    return LIB.ppf_version().decode()


def check(code: int, what: str) -> None:
    if code != PPF_OK:
        raise PpfError(code, what)


def ptr(t) -> int:
    """Device pointer of a torch tensor (or 0 for None)."""
    if t is None:
        return 0
    return int(t.data_ptr())


def require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError(
            "pypomp_b200 runs its particle filters only on a CUDA device (sm_100a); "
            "no CUDA device is visible"
        )
    return torch


def env_path() -> int:
    """Execution path override from PYPOMP_B200_PATH (auto/plain/stream/resident)."""
    return PATHS[os.environ.get("PYPOMP_B200_PATH", "auto").lower()]
