"""Generate the committed golden fixtures under tests/golden/.

Run from the repository root (needs the reference checkout only to read its
regression CSVs; the GPU tests read only the files written here):

    python tests/golden/make_fixtures.py /path/to/reference-checkout

Writes
  ref_values.json  the reference's locked regression values, read from
                   tests/test_regression/*/*.csv of the reference checkout
                   (pfilter logLik, per-step diagnostics, MOP value, simulate)
  ref_lg1d.npz     the reference's 1-D LG data set (``LG(A=[[0.9]], T=4,
                   key=jax.random.key(0))``, tests/test_regression/conftest.py:23)
                   regenerated through oracle/jaxrng.py, plus the exact
                   normals and uniforms the reference draws for each locked
                   filter run (replayed key trees), for noise-injection runs;
                   ``mif_*`` / ``mift_*`` hold the draws of the locked mif runs
                   (perturbation normals too) and their monitors; ``ppf_*``,
                   ``pmif_*``, ``ptrain_*`` those of the locked panel runs
"""

from __future__ import annotations

import csv
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import jaxrng as jr  # noqa: E402
from oracle import refpath as rp  # noqa: E402

OUT = Path(__file__).resolve().parent
f32 = np.float32

# LG(A=[[0.9]]) natural-scale theta in canonical order A11, C11, Q11, R11, X0_1
# (default Q = 1/100 -> chol 0.1; default R = 1/10 -> chol sqrt(0.1)).
THETA_LG1D = np.array([0.9, 1.0, 0.1, np.sqrt(0.1), 0.0], dtype=f32)


def _read_csv(path: Path) -> dict:
    with open(path) as fh:
        rows = list(csv.reader(fh))
    header = rows[0][1:]
    cols = {h: [] for h in header}
    for r in rows[1:]:
        for h, v in zip(header, r[1:]):
            if v != "":
                cols[h].append(float(v))
    return cols


def main(ref_root: Path):
    reg = ref_root / "tests" / "test_regression"
    values = {
        "pfilter": _read_csv(reg / "test_pfilter_regression" / "test_pfilter_regression.csv"),
        "pfilter_diagnostics": _read_csv(reg / "test_pfilter_regression" / "test_pfilter_diagnostics_regression.csv"),
        "mop": _read_csv(reg / "test_mop_regression" / "test_mop_regression.csv"),
        "simulate": _read_csv(reg / "test_simulate_regression" / "test_simulate_regression.csv"),
        "mif": _read_csv(reg / "test_mif_regression" / "test_mif_regression.csv"),
        "mif_full_trace": _read_csv(reg / "test_mif_regression" / "test_mif_full_trace_regression.csv"),
        "train": _read_csv(reg / "test_train_regression" / "test_train_regression.csv"),
        "dpop": _read_csv(reg / "test_dpop_regression" / "test_dpop_regression.csv"),
        "dpop_train": _read_csv(reg / "test_dpop_train_regression" / "test_dpop_train_regression.csv"),
        "panel_pfilter": _read_csv(reg / "test_panel_pfilter_regression" / "test_panel_pfilter_regression.csv"),
        "panel_mif": _read_csv(reg / "test_panel_mif_regression" / "test_panel_mif_regression.csv"),
        "panel_train": _read_csv(reg / "test_panel_train_regression" / "test_panel_train_regression.csv"),
        "tolerance": {"atol": 1e-6, "rtol": 1e-4},
        "source": "pypomp 0.4.10.2 tests/test_regression (tolerance: tests/test_regression/conftest.py:118-125)",
    }
    (OUT / "ref_values.json").write_text(json.dumps(values, indent=1))

    # Data: Pomp.simulate(key=key(0)) inside LG(...)
    X, Y = rp.pomp_simulate_data("LG", THETA_LG1D, 4, jr.key(0))
    ys = Y.astype(f32)
    J = 12
    arrays = {"theta": THETA_LG1D, "ys": ys}
    # pfilter regression: keys = split(key(20260811), 1)
    k = jr.split(jr.key(20260811), 1)[0]
    rec = rp.RecordingNoise(rp.JaxKeyNoise(k, J, 1, 1))
    rp.pfilter("LG", THETA_LG1D, ys, J, rec)
    z0, z, u = rec.arrays()
    arrays.update(pf_z0=z0, pf_z=z, pf_u=u)
    # diagnostics: thetas (theta0, 1.05 theta0), keys = split(key(20260812), 2)
    ks = jr.split(jr.key(20260812), 2)
    thetas = np.stack([THETA_LG1D, (THETA_LG1D * f32(1.05)).astype(f32)])
    zz0, zz, uu = [], [], []
    for r in range(2):
        rec = rp.RecordingNoise(rp.JaxKeyNoise(ks[r], J, 1, 1))
        rp.pfilter("LG", thetas[r], ys, J, rec, diagnostics=True)
        a, b, c = rec.arrays()
        zz0.append(a); zz.append(b); uu.append(c)
    arrays.update(diag_theta=thetas, diag_z0=np.stack(zz0), diag_z=np.stack(zz), diag_u=np.stack(uu))
    # mop regression: keys = split(key(20260811), 1), alpha 0.5, theta0 read as estimation scale
    k = jr.split(jr.key(20260811), 1)[0]
    rec = rp.RecordingNoise(rp.JaxKeyNoise(k, J, 1, 1))
    rp.mop("LG", THETA_LG1D, ys, J, 0.5, rec)
    z0, z, u = rec.arrays()
    arrays.update(mop_z0=z0, mop_z=z, mop_u=u)
    # mif regression (test_mif_regression.py): uniform rw sd 0.02, geometric
    # cooling 0.5, thresh 0; 1 replicate M=3 without monitors, and 2 replicates
    # (theta0, 1.05 theta0) M=4 with one monitor
    sig = np.full(5, 0.02, f32)
    sig0 = np.zeros(5, f32)
    k = jr.split(jr.key(20260811), 1)[0]
    _, _, _, draws = rp.mif("LG", THETA_LG1D, ys, J, 3, sig, sig0, mif_cooling, k, 0)
    for key in ("zp0", "zp", "z0", "z", "u"):
        arrays[f"mif_{key}"] = np.stack([d["perfilter"][key] for d in draws])          # (M, ...)
    ks = jr.split(jr.key(20260812), 2)
    reps = [rp.mif("LG", thetas[r], ys, J, 4, sig, sig0, mif_cooling, ks[r], 1)[3] for r in range(2)]
    for key in ("zp0", "zp", "z0", "z", "u"):
        arrays[f"mift_{key}"] = np.stack([np.stack([d["perfilter"][key] for d in reps[r]]) for r in range(2)])
        if key in ("z0", "z", "u"):
            arrays[f"mift_mon_{key}"] = np.stack([np.stack([d["monitors"][0][key] for d in reps[r]])
                                                  for r in range(2)])                # (2, M, ...)
    # panel of two LG units (tests/test_regression/conftest.py:61-110): unit 2's
    # data from key(1); identity host transform; shared A11, C11; unit Q11, R11, X0_1
    _, Y2 = rp.pomp_simulate_data("LG", THETA_LG1D, 4, jr.key(1))
    ys2 = Y2.astype(f32)
    arrays["panel_ys2"] = ys2
    pkey = jr.key(20260811)
    _, pdraws = rp.panel_pfilter("LG", np.stack([THETA_LG1D, THETA_LG1D]), [ys, ys2], J, jr.split(pkey, 2))
    for key in ("z0", "z", "u"):
        arrays[f"ppf_{key}"] = np.stack([d[key] for d in pdraws])                       # (U, ...)
    _, _, mdraws = rp.panel_mif("LG", THETA_LG1D[:2], np.stack([THETA_LG1D[2:]] * 2), [ys, ys2], J, 3, sig,
                                sig0, mif_cooling, jr.split(pkey, 1)[0], host_identity=True)
    for key in ("zp0", "zp", "z0", "z", "u"):
        arrays[f"pmif_{key}"] = np.stack([np.stack([d["perfilter"][key] for d in dm]) for dm in mdraws])  # (M, U, ...)
    # panel train: keys split(key, n_reps * M * U) -> (M, U); each a MOP key tree
    tkeys = jr.split(pkey, 3 * 2)
    tz0, tz, tu = [], [], []
    for i in range(6):
        rec = rp.RecordingNoise(rp.JaxKeyNoise(tkeys[i], J, 1, 1))
        rp.mop("LG", THETA_LG1D, ys, J, 0.97, rec)
        a, b, c = rec.arrays()
        tz0.append(a); tz.append(b); tu.append(c)
    arrays["ptrain_z0"] = np.stack(tz0).reshape((3, 2) + tz0[0].shape)
    arrays["ptrain_z"] = np.stack(tz).reshape((3, 2) + tz[0].shape)
    arrays["ptrain_u"] = np.stack(tu).reshape((3, 2) + tu[0].shape)
    np.savez(OUT / "ref_lg1d.npz", **arrays)


def mif_cooling(nt, m, ntimes):
    """Geometric cooling with a = 0.5 in float32 (``rw_sigma.py:193-224``)."""
    frac = f32(f32(nt) / f32(ntimes) + f32(m))
    return f32(f32(0.5 ** (1.0 / 50.0)) ** frac)



if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py /path/to/reference-checkout")
    main(Path(sys.argv[1]))
