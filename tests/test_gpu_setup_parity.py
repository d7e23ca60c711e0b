"""The device-side set-up the benchmark and every mixed-precision,
ensemble and surrogate run use, pinned against the reference:

* pdgpu_build_pd_neighbors (cell-list search on the GPU) against the
  reference's kd-tree lists of DEMModel::updatePeridynamicNeighborlist
  (demModel.cpp:1659-1694): the same SET per node, exactly (the reference's
  rows are in kd-tree order, the device's ascending);
* pdgpu_compute_mx (material::computeStateMx, materialUtil.cpp:21-73)
  against the reference's d_mX: bit for bit when it sums over the
  reference's own list order (one thread per node, list order, no FMA), and
  within MX_TOL relative over the device's ascending rows (a different sum
  order of ~30 positive terms);
* the same two at the benchmark's size (502 particles, 339 280 nodes) and on
  a 3-D packing, against the C oracle's brute-force search and m_x, which
  tests/test_oracle.py pins to the reference's own lists and m_x.
"""
import numpy as np
import pytest

import golden_io
import pdoracle
import refrun
import scenarios
from peridem_b200 import scene as scn

pytestmark = pytest.mark.gpu

MX_TOL = 1e-13


def _check_lists_and_mx(tag, init):
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    sc = refrun.scene_from_dump(init)
    ref_sets = refrun.csr_sets(init["pd_rowptr"], init["pd_col"])
    # device-built lists and m_x over them
    m = GpuDEMModel(sc, precision=PREC_FP64, build_neighbors=True, compute_mx=True)
    try:
        rp, col = m.pd_neighbors()
        mx_dev = m.field("mX")
        m.sync()
    finally:
        m.close()
    got = refrun.csr_sets(rp, col)
    bad = [i for i in ref_sets if got[i] != ref_sets[i]]
    assert not bad, f"{tag}: neighbour sets differ at {len(bad)} nodes, e.g. {bad[:5]}"
    for i in range(sc.n_nodes):
        row = col[rp[i]:rp[i + 1]]
        assert np.all(row[1:] > row[:-1]), f"{tag}: row {i} not ascending"
    mx_ref = init["mX"]
    e = float(np.max(np.abs(mx_dev - mx_ref) / np.abs(mx_ref)))
    assert e <= MX_TOL, f"{tag}: m_x over the device's lists differs by {e:.2e} (tol {MX_TOL:.0e})"
    # the reference's lists uploaded, m_x computed on the device
    m = GpuDEMModel(sc, precision=PREC_FP64, compute_mx=True)
    try:
        mx_same_order = m.field("mX")
    finally:
        m.close()
    nd = int(np.sum(mx_same_order != mx_ref))
    assert nd == 0, f"{tag}: m_x over the reference's list order differs at {nd} nodes " \
                    f"(max rel {float(np.max(np.abs(mx_same_order - mx_ref) / np.abs(mx_ref))):.2e})"
    print(f"{tag}: {sc.n_nodes} nodes, {len(col)} bonds, sets equal; m_x bit-exact in list order, "
          f"{e:.1e} over ascending rows")


@pytest.mark.parametrize("name", golden_io.names())
def test_device_neighbor_lists_and_mx_match_golden(name):
    init, _ = golden_io.load(name)
    _check_lists_and_mx(name, init)


@pytest.mark.skipif(not refrun.have_reference(), reason="reference binary not built")
@pytest.mark.parametrize("case", list(scenarios.CASES))
def test_device_neighbor_lists_and_mx_match_reference_live(case, tmp_path):
    factory, _, _ = scenarios.CASES[case]
    scn.write_deck(factory(), str(tmp_path))
    init, _ = refrun.run_reference(str(tmp_path), 0, [])
    _check_lists_and_mx(case, init)


def _check_against_oracle(tag, sc):
    from peridem_b200.model import GpuDEMModel, PREC_MIXED
    rp_o, col_o = pdoracle.build_pd_neighbors(sc)      # node order = ascending rows
    m = GpuDEMModel(sc, precision=PREC_MIXED, build_neighbors=True, compute_mx=True)
    try:
        rp, col = m.pd_neighbors()
        mx = m.field("mX")
    finally:
        m.close()
    assert np.array_equal(rp, rp_o), f"{tag}: row offsets differ"
    assert np.array_equal(col, col_o), f"{tag}: columns differ"
    sc.pd_rowptr, sc.pd_col = rp_o, col_o
    mx_o = pdoracle.compute_mx(sc)
    nd = int(np.sum(mx != mx_o))
    assert nd == 0, f"{tag}: m_x differs from the oracle's at {nd} nodes"
    print(f"{tag}: {sc.n_nodes} nodes, {len(col)} bonds: lists and m_x equal the oracle's")


def test_device_neighbor_lists_and_mx_at_benchmark_size():
    """The benchmark scene itself: 502 discs and hexagons, h = R/15."""
    _check_against_oracle("compressive_502", scn.build_scene(scn.compressive_2d()))


def test_device_neighbor_lists_and_mx_3d_packing():
    sc = scn.build_scene(scn.column_3d(n_spheres=27, median_r=1e-3, sigma=0.2, h_div=6,
                                       box=(8e-3, 8e-3, 12e-3), seed=4, nt=10, wall_h=6e-4))
    _check_against_oracle("column_27", sc)
