"""ppf_pfilter_noalloc: the filter for callers that cannot allocate (GPU).

Some callers of the library cannot hand it a device workspace -- a host runtime
that owns the device memory pool, or plugin code that may not call the CUDA
allocator -- so ppf_pfilter_noalloc runs the batched filter on a fixed scratch
array compiled into the library.  This file checks, through the C ABI, that two
calls in a row give the same results as the ordinary ppf_pfilter with a
caller-provided workspace (the tolerance of the other parity tests), also with
PPF_F_GRAPH set (the flag is ignored: a cached graph would need driver-side
allocations), that a request larger than the fixed scratch is refused with
PPF_ESCRATCH before any GPU work, and that a call on a stream being captured
into a CUDA graph is refused (the call waits for its stream, which a capture
cannot record).  It is collected last on purpose and also passes alone.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _desc(torch, spec, ys, theta, seeds, J, T, path, flags=0):
    from pypomp_b200 import _ffi

    dev = torch.device("cuda", 0)
    keep = {
        "ys": torch.from_numpy(np.ascontiguousarray(ys[None], dtype=np.float32)).to(dev),
        "theta": torch.from_numpy(np.ascontiguousarray(theta, dtype=np.float32)).to(dev),
        "seeds": torch.from_numpy(np.asarray(seeds, dtype=np.uint64).view(np.int64).copy()).to(dev),
    }
    F = theta.shape[0]
    keep["loglik"] = torch.zeros(F, dtype=torch.float64, device=dev)
    keep["cll"] = torch.zeros(F, T, dtype=torch.float64, device=dev)
    keep["anc"] = torch.zeros(F, T, J, dtype=torch.int32, device=dev)
    d = _ffi.PfilterDesc()
    d.model = spec.ffi_model()
    d.J, d.F, d.T, d.U = J, F, T, 1
    d.path = path
    d.flags = flags | _ffi.F_CLL | _ffi.F_SAVE_ANC
    d.theta, d.ys, d.seeds = _ffi.ptr(keep["theta"]), _ffi.ptr(keep["ys"]), _ffi.ptr(keep["seeds"])
    d.loglik, d.cll, d.anc = _ffi.ptr(keep["loglik"]), _ffi.ptr(keep["cll"]), _ffi.ptr(keep["anc"])
    return d, keep


@pytest.mark.parametrize("path,graph", [("stream", False), ("resident", False), ("stream", True)])
def test_noalloc_matches_workspace_entry_point(path, graph):
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from tests.conftest import LG2_Q, LG2_R

    m = pp.LG(T=20, Q=LG2_Q, R=LG2_R, key=4)
    st = m.to_struct()
    theta = np.repeat(m.theta.to_array(m.canonical_param_names), 4, axis=0).astype(np.float32)
    theta[1:, 0] *= np.float32(0.97)
    seeds = np.array([1, 2, 3, 4], np.uint64)
    J, T = (4096, 20) if path == "stream" else (1000, 20)
    stream = torch.cuda.current_stream().cuda_stream

    d, keep = _desc(torch, m.spec, st.ys, theta, seeds, J, T, _ffi.PATHS[path])
    ws = torch.empty(_ffi.LIB.ppf_pfilter_workspace_bytes(d), dtype=torch.uint8, device="cuda")
    d.workspace, d.ws_bytes = _ffi.ptr(ws), ws.numel()
    _ffi.check(_ffi.LIB.ppf_pfilter(d, stream), "ppf_pfilter")
    _ffi.check(_ffi.LIB.ppf_workspace_status(d.workspace, stream), "ppf_pfilter")
    want = {k: keep[k].cpu().numpy() for k in ("loglik", "cll", "anc")}

    for call in range(2):
        d2, keep2 = _desc(torch, m.spec, st.ys, theta, seeds, J, T, _ffi.PATHS[path],
                          flags=_ffi.F_GRAPH if graph else 0)
        assert _ffi.LIB.ppf_pfilter_noalloc(d2, stream) == _ffi.PPF_OK
        got = {k: keep2[k].cpu().numpy() for k in ("loglik", "cll", "anc")}
        np.testing.assert_allclose(got["loglik"], want["loglik"], rtol=1e-12, err_msg=f"call {call}")
        np.testing.assert_allclose(got["cll"], want["cll"], rtol=1e-12, atol=1e-12, err_msg=f"call {call}")
        assert np.array_equal(got["anc"], want["anc"]), f"call {call}"


def test_noalloc_refuses_requests_beyond_its_scratch():
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from tests.conftest import LG2_Q, LG2_R

    m = pp.LG(T=5, Q=LG2_Q, R=LG2_R, key=4)
    st = m.to_struct()
    J, F = 262144, 64
    theta = np.repeat(m.theta.to_array(m.canonical_param_names), F, axis=0).astype(np.float32)
    d, keep = _desc(torch, m.spec, st.ys, theta, np.arange(F, dtype=np.uint64), J, 5, _ffi.PATH_STREAM)
    assert _ffi.LIB.ppf_pfilter_workspace_bytes(d) > _ffi.NOALLOC_SCRATCH_BYTES
    stream = torch.cuda.current_stream().cuda_stream
    assert _ffi.LIB.ppf_pfilter_noalloc(d, stream) == _ffi.PPF_ESCRATCH
    assert "scratch" in _ffi.error_string(_ffi.PPF_ESCRATCH)


def test_noalloc_refuses_a_capturing_stream():
    import torch

    import pypomp_b200 as pp
    from pypomp_b200 import _ffi
    from tests.conftest import LG2_Q, LG2_R

    m = pp.LG(T=5, Q=LG2_Q, R=LG2_R, key=4)
    st = m.to_struct()
    theta = m.theta.to_array(m.canonical_param_names).astype(np.float32)
    d, keep = _desc(torch, m.spec, st.ys, theta, np.array([1], np.uint64), 1024, 5, _ffi.PATH_STREAM)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        g.capture_begin()
        try:
            rc = _ffi.LIB.ppf_pfilter_noalloc(d, side.cuda_stream)
            keep["loglik"].add_(0.0)      # something to capture
        finally:
            g.capture_end()
    assert rc == _ffi.PPF_EUNSUPPORTED
    # the stream and the library are usable afterwards
    assert _ffi.LIB.ppf_pfilter_noalloc(d, torch.cuda.current_stream().cuda_stream) == _ffi.PPF_OK
    del g
