"""The mixed-precision form (FP32 bond loop, FP64 integration and
reductions) against the plain FP64 form on the same scene: the north-star
gates, written out —

* wall reaction (the compressive test's reference definition and the contact
  reaction on the moving wall) within 1e-3 relative of the FP64 history,
  normalised by the largest FP64 value;
* damage fraction (nodes with Z >= 1, broken-bond fraction) within 1e-3;
* positions within 1e-3 of the largest displacement.
"""
import numpy as np
import pytest

from peridem_b200 import scene as scn

pytestmark = pytest.mark.gpu


def _run(sc, prec, steps):
    from peridem_b200.model import GpuDEMModel
    m = GpuDEMModel(sc, precision=prec, build_neighbors=True, compute_mx=True)
    try:
        m.integrate_begin()
        m.integrate_step(steps)
        m.sync()
        out = {k: m.field(k) for k in ("x", "u", "Z", "bonds")}
        out["hist"] = m.history()
        out["sc"] = m.scalars()
    finally:
        m.close()
    return out


def test_mixed_matches_fp64_on_compression():
    from peridem_b200.model import PREC_FP64, PREC_MIXED
    h = 1e-3 / 8
    spec = scn.compressive_2d(n_particles=12, r_range=(1e-3, 1.3e-3), h_div=8, width=10e-3,
                              seed=7, gap=1.02 * h, wall_speed=-2.0, nt=3000)
    sc = scn.build_scene(spec)
    a = _run(sc, PREC_FP64, 3000)
    b = _run(sc, PREC_MIXED, 3000)
    ha, hb = a["hist"], b["hist"]
    assert ha.shape == hb.shape and len(ha) > 10
    for col, name in ((2, "reaction"), (3, "contact reaction")):
        den = max(np.max(np.abs(ha[:, col])), 1e-300)
        err = np.max(np.abs(ha[:, col] - hb[:, col])) / den
        print(f"{name}: max |fp64| {den:.4e}, rel err {err:.3e}")
        assert err <= 1e-3, name
    assert np.max(np.abs(ha[:, 3])) > 0, "the wall never touched the packing"
    za, zb = a["Z"], b["Z"]
    dfrac = abs(np.mean(za >= 1.0) - np.mean(zb >= 1.0))
    bfrac = abs(np.mean(a["bonds"]) - np.mean(b["bonds"]))
    assert dfrac <= 1e-3 and bfrac <= 1e-3, (dfrac, bfrac)
    du = np.max(np.abs(a["u"] - b["u"])) / max(np.max(np.abs(a["u"])), 1e-300)
    print(f"displacement rel err {du:.3e}")
    assert du <= 1e-3
