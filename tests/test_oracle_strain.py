"""Quadrature-point strain and stress of linear triangles (the Strain_Stress
output, fe::getCurrentQuadPoints / fe::getStrainStress): the NumPy
restatement in oracle/fe_strain.py against fixtures the reference itself
produced (tests/golden/strain_tri.npz, from oracle/_ref/ref_strain), bit for
bit, for quadrature orders 1 and 2 in plane strain and plane stress; and,
where the reference's driver is built here, the fixtures against a fresh run
of it."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(HERE, "golden"), os.path.join(os.path.dirname(HERE), "oracle")]

import fe_strain  # noqa: E402
from peridem_b200 import fe  # noqa: E402

G = np.load(os.path.join(HERE, "golden", "strain_tri.npz"))


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ps", [0, 1])
def test_restatement_matches_reference_fixtures(order, ps):
    nu, lam, mu = G["material"]
    conn = G["conn"]
    m = len(conn)
    xq, e, s = fe_strain.strain_stress_tri(G["xref"], G["u"], conn, fe.tri_points(order), np.full(m, nu),
                                           np.full(m, lam), np.full(m, mu), np.full(m, ps, dtype=bool))
    k = f"o{order}_ps{ps}"
    assert np.array_equal(xq, G[k + "_xq"])
    assert np.array_equal(e, G[k + "_strain"])
    assert np.array_equal(s, G[k + "_stress"])
    if order == 1:  # three entries per element, the one-point rule fills the first
        assert not np.any(G[k + "_strain"].reshape(m, 3, 6)[:, 1:])


def test_fixture_mesh_is_the_two_particle_scene():
    import make_strain_golden as mk
    from peridem_b200 import scene as scn
    sc = scn.build_scene(mk.scene_spec())
    assert np.array_equal(np.asarray(sc.xref), G["xref"])
    assert np.array_equal(mk.mesh(sc), G["conn"])
    assert np.array_equal(mk.displacement(G["xref"]), G["u"])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_strain")),
                    reason="reference strain driver not built")
def test_fixtures_reproduce_with_the_reference():
    import make_strain_golden as mk
    nu, lam, mu = G["material"]
    xq, e, s = mk.run_reference(G["xref"], G["u"], G["conn"], 2, 1, nu, lam, mu)
    assert np.array_equal(xq, G["o2_ps1_xq"]) and np.array_equal(e, G["o2_ps1_strain"])
    assert np.array_equal(s, G["o2_ps1_stress"])


GT = np.load(os.path.join(HERE, "golden", "strain_tet.npz"))


def test_tet_restatement_matches_reference_fixtures():
    nu, lam, mu = GT["material"]
    m = len(GT["conn"])
    xq, e, s = fe_strain.strain_stress_tet(GT["xref"], GT["u"], GT["conn"], np.full(m, lam), np.full(m, mu))
    assert np.array_equal(xq, GT["o1_xq"])
    assert np.array_equal(e, GT["o1_strain"])
    assert np.array_equal(s, GT["o1_stress"])


def test_tet_fixture_mesh_is_the_column_scene():
    import make_strain_golden as mk
    from peridem_b200 import scene as scn
    spec = mk.scene_spec_3d()
    sc = scn.build_scene(spec)
    assert np.array_equal(np.asarray(sc.xref), GT["xref"])
    assert np.array_equal(mk.mesh_3d(sc, spec), GT["conn"])
