"""pdgpu_strain_stress_tri / _tet (the Strain_Stress output on the GPU)
against the reference's own fe::getCurrentQuadPoints / fe::getStrainStress:
bit for bit with tests/golden/strain_tri.npz (made by the reference from the
same two-particle scene's nodes and displacement; orders 1 and 2, plane
strain and plane stress) and strain_tet.npz (a two-sphere column's
tetrahedra, the one-point rule); argument checks on the host."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(HERE, "golden")]

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(HERE, "golden", "strain_tri.npz"))


def _model():
    import make_strain_golden as mk
    from peridem_b200 import scene as scn
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    sc = scn.build_scene(mk.scene_spec())
    m = GpuDEMModel(sc, precision=PREC_FP64, build_neighbors=True, compute_mx=True)
    m.set_field("u", G["u"])
    return m


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ps", [0, 1])
def test_strain_stress_matches_reference(order, ps):
    nu, lam, mu = G["material"]
    m = _model()
    try:
        xq, e, s = m.strain_stress_tri(G["conn"], order, nu, lam, mu, ps)
    finally:
        m.close()
    k = f"o{order}_ps{ps}"
    assert np.array_equal(xq, G[k + "_xq"]), float(np.max(np.abs(xq - G[k + "_xq"])))
    assert np.array_equal(e, G[k + "_strain"]), float(np.max(np.abs(e - G[k + "_strain"])))
    assert np.array_equal(s, G[k + "_stress"]), float(np.max(np.abs(s - G[k + "_stress"])))


def test_strain_stress_refuses_bad_arguments():
    from peridem_b200 import api
    m = _model()
    try:
        bad = np.array(G["conn"])
        bad[3, 1] = 10 ** 6
        with pytest.raises(api.PdgpuError):
            m.strain_stress_tri(bad, 1, 0.25, 1.0, 1.0, 0)
        with pytest.raises(ValueError):
            m.strain_stress_tri(G["conn"], 3, 0.25, 1.0, 1.0, 0)
    finally:
        m.close()


GT = np.load(os.path.join(HERE, "golden", "strain_tet.npz"))


def test_tet_strain_stress_matches_reference():
    import make_strain_golden as mk
    from peridem_b200 import scene as scn
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    nu, lam, mu = GT["material"]
    sc = scn.build_scene(mk.scene_spec_3d())
    m = GpuDEMModel(sc, precision=PREC_FP64, build_neighbors=True, compute_mx=True)
    try:
        m.set_field("u", GT["u"])
        xq, e, s = m.strain_stress_tet(GT["conn"], nu, lam, mu)
    finally:
        m.close()
    assert np.array_equal(xq, GT["o1_xq"]), float(np.max(np.abs(xq - GT["o1_xq"])))
    assert np.array_equal(e, GT["o1_strain"]), float(np.max(np.abs(e - GT["o1_strain"])))
    assert np.array_equal(s, GT["o1_stress"]), float(np.max(np.abs(s - GT["o1_stress"])))


def test_strain_vtu_holds_the_arrays(tmp_path):
    """pdgpu_write_strain_vtu: the quadrature points as points, Strain and
    Stress with components xx..xy, TIME (VtkParticleWriter::appendStrainStress)."""
    from test_gpu_output import _read
    nu, lam, mu = G["material"]
    m = _model()
    try:
        xq, e, s = m.strain_stress_tri(G["conn"], 2, nu, lam, mu, 1)
        path = str(tmp_path / "output_strain_0.vtu")
        m.write_strain_vtu(path, xq, e, s)
    finally:
        m.close()
    root, arrays = _read(path)
    assert np.array_equal(arrays["Points"], xq)
    assert np.array_equal(arrays["Strain"], e) and np.array_equal(arrays["Stress"], s)
    da = [d for d in root.iter("DataArray") if d.get("Name") == "Strain"][0]
    assert [da.get(f"ComponentName{k}") for k in range(6)] == ["xx", "yy", "zz", "yz", "xz", "xy"]
    assert arrays["TIME"].shape == (1, 1)
