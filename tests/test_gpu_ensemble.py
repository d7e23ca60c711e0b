"""Batched ensemble: independent compression scenes of uneven size merged
into one model (one bond-loop launch over every scene's tiles, one contact
pass, one graph per step) against each scene run alone.

Each scene of the ensemble must follow its own single-scene run: the
displacement field and the per-scene compressive-test records (wall
displacement, reaction, contact reaction).  The two runs differ only in the
order of floating-point sums inside the contact candidate lists and in the
rebuild schedule (the ensemble rebuilds on its fastest scene), so the FP64
form is held to 1e-9 relative and the mixed form to 1e-6.
"""
import numpy as np
import pytest

from peridem_b200 import scene as scn

pytestmark = pytest.mark.gpu

STEPS = 2000


def _specs():
    return scn.ensemble_specs(n_scenes=3, seed=5, n_range=(5, 14), h_div_range=(4, 6),
                              speed_range=(2.0, 4.0), nt=STEPS)


def _run(sc, prec, graph):
    from peridem_b200.model import GpuDEMModel
    m = GpuDEMModel(sc, precision=prec, build_neighbors=True, compute_mx=True)
    try:
        m.integrate_begin()
        m.integrate_step(STEPS, graph_steps=1 if graph else 0)
        m.sync()
        hist = [m.scene_history(k) for k in range(sc.n_scenes)] if sc.n_scenes > 1 else [m.history()]
        return m.field("u"), hist
    finally:
        m.close()


@pytest.mark.parametrize("prec_name,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_ensemble_matches_single_scenes(prec_name, tol):
    from peridem_b200.model import PREC_FP64, PREC_MIXED
    prec = PREC_FP64 if prec_name == "fp64" else PREC_MIXED
    scenes = [scn.build_scene(s) for s in _specs()]
    ens = scn.merge_scenes(scenes)
    assert ens.n_scenes == 3 and len({s.n_nodes for s in scenes}) == 3
    ue, he = _run(ens, prec, graph=True)
    touched = 0
    for k, sc in enumerate(scenes):
        us, hs = _run(sc, prec, graph=False)
        n0 = int(ens.p_start[ens.scene_poff[k]])
        du = ue[n0:n0 + sc.n_nodes] - us
        den = max(float(np.max(np.abs(us))), 1e-300)
        eu = float(np.max(np.abs(du))) / den
        h1, h2 = he[k], hs[0]
        assert h1.shape == h2.shape and len(h1) > 0, (h1.shape, h2.shape)
        line = f"scene {k}: nodes {sc.n_nodes} u rel {eu:.2e}"
        for col, name in ((1, "wall disp"), (2, "reaction"), (3, "contact reaction")):
            d = max(float(np.max(np.abs(h2[:, col]))), 1e-300)
            e = float(np.max(np.abs(h1[:, col] - h2[:, col]))) / d
            line += f" | {name} max {d:.3e} rel {e:.2e}"
            assert e <= tol, (k, name, e)
        assert np.array_equal(h1[:, 0], h2[:, 0])
        print(line)
        assert eu <= tol
        touched += float(np.max(np.abs(h2[:, 3]))) > 0
    assert touched >= 2, "the walls did not reach the packings"
