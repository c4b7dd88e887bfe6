"""The FP64 MOP-alpha surrogate (oracle/mop_fp64.py) against the C oracle's
float32 surrogate on the same injected normals and frozen ancestors (CPU):
the values agree to float32 accuracy and, on a short series where float32
difference quotients are still accurate, the central differences agree."""

import numpy as np

from oracle import cora
from oracle.mop_fp64 import central_differences, sv_surrogate

f32 = np.float32


def test_fp64_surrogate_matches_c_oracle_on_sv():
    import pypomp_b200 as pp

    T, J, alpha = 30, 512, 0.97
    m = pp.SV(T=T, key=1)
    st = m.to_struct()
    spec = m.spec
    th = spec.to_est(m.theta.to_array(m.canonical_param_names)).astype(f32)
    rng = np.random.default_rng(3)
    z = rng.standard_normal((1, T, J, 1)).astype(f32)
    u = rng.random((1, T)).astype(f32)
    inj = {"z0": np.zeros((1, J, 1), f32), "z": z, "u": u}
    fwd = cora.pfilter(spec.kind, 2, 1, th, st.ys, J, est=True, mop=True, anc=True, inject=inj, dt=spec.dt)
    anc = fwd["anc"]
    c_val, c_m0 = cora.mop_surrogate(spec.kind, 2, 1, th, st.ys, J, alpha, anc, inject=inj, dt=spec.dt)
    v64, m0 = sv_surrogate(th[0], st.ys, spec.dt, z[0, :, :, 0], anc[0], alpha)
    assert abs(v64 - c_val[0]) <= 1e-5 * abs(c_val[0])
    np.testing.assert_allclose(m0, c_m0[0], rtol=1e-4, atol=1e-4)
    g64 = central_differences(lambda t: sv_surrogate(t, st.ys, spec.dt, z[0, :, :, 0], anc[0], alpha, m0)[0],
                              th[0].astype(np.float64))
    h = 1e-3
    g32 = np.zeros(th.shape[1])
    for p in range(th.shape[1]):
        tp, tm = th.copy(), th.copy()
        tp[0, p] += f32(h)
        tm[0, p] -= f32(h)
        vp, _ = cora.mop_surrogate(spec.kind, 2, 1, tp, st.ys, J, alpha, anc, c_m0, inject=inj, dt=spec.dt)
        vm, _ = cora.mop_surrogate(spec.kind, 2, 1, tm, st.ys, J, alpha, anc, c_m0, inject=inj, dt=spec.dt)
        g32[p] = (vp[0] - vm[0]) / (float(tp[0, p]) - float(tm[0, p]))
    assert np.linalg.norm(g64 - g32) <= 2e-3 * np.linalg.norm(g64), (g64, g32)
