"""GPU parity against the reference itself: the reference's DEMModel
(oracle/_ref/peridem_ref, compiled here from the reference's own sources)
sets a scene up and steps it; the FP64 CUDA path starts from the same
ModelData (same neighbour-list order) and must reproduce:

* forces f after the integrate() prelude and after each checked step:
  max|f_gpu - f_ref| <= 1e-11 * max|f_ref| (the 1e-12 target plus headroom
  for summation order: lanes of a node sum in a tree, the reference in list
  order; RNP's exp() differs by at most an ulp);
* u, v, x to 1e-10 normwise;
* bond-broken flags and contact candidate sets: identical;
* contact-search control (update interval, counter, radius): identical;
* damage Z to 1e-5 relative (the reference's running max uses its own
  relative-epsilon comparison, so it can stop up to 1e-5 below the maximum).
"""
import os

import numpy as np
import pytest

import refrun
import scenarios
from peridem_b200 import scene as scn

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refrun.have_reference(),
                                 reason="reference binary oracle/_ref/peridem_ref not built")]

F_TOL = 1e-11
KIN_TOL = 1e-10
Z_TOL = 2e-5


def _model(init):
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    sc = refrun.scene_from_dump(init)
    return sc, GpuDEMModel(sc, precision=PREC_FP64)


def _searching_nodes(init):
    N = int(init["N"][0])
    out = []
    for p in range(int(init["Np"][0])):
        if init["p_type"][p] == 0 and init["p_computeForce"][p] and not init["p_allDofsConstrained"][p]:
            out.extend(range(int(init["p_globStart"][p]), int(init["p_globEnd"][p])))
    return [i for i in out if i < N]


def _compare(tag, m, ref, init, chaotic=False):
    N = int(init["N"][0])
    f = m.field("f")
    fr = ref["f"].reshape(N, 3)
    ef = refrun.rel_err(f, fr)
    eu = refrun.rel_err(m.field("u"), ref["u"].reshape(N, 3), floor=1e-30)
    ev = refrun.rel_err(m.field("v"), ref["v"].reshape(N, 3), floor=1e-30)
    ex = refrun.rel_err(m.field("x") - init["xRef"].reshape(N, 3),
                        ref["x"].reshape(N, 3) - init["xRef"].reshape(N, 3), floor=1e-30)
    bonds = m.field("bonds")
    nb = int(np.sum(bonds != ref["bond_state"]))
    z = m.field("Z")
    zr = ref["Z"]
    ez = float(np.max(np.abs(z - zr) / np.maximum(np.abs(zr), 1e-6))) if zr.size else 0.0
    msg = f"{tag}: f {ef:.2e} u {eu:.2e} v {ev:.2e} x {ex:.2e} bonds-diff {nb} Z {ez:.2e}"
    print(msg)
    assert nb == 0, msg
    assert ef <= F_TOL, msg
    assert eu <= KIN_TOL and ev <= KIN_TOL and ex <= KIN_TOL, msg
    assert ez <= Z_TOL, msg
    sc = m.scalars()
    if int(init["is_multi"][0]):
        assert sc["contact_update_interval"] == int(ref["contNeighUpdateInterval"][0]), (tag, sc)
        assert sc["contact_counter"] == int(ref["contNeighTimestepCounter"][0]), (tag, sc)
        assert sc["contact_search_radius"] == float(ref["contNeighSearchRadius"][0]), (tag, sc)
        rp, col = m.contact_lists()
        nodes = _searching_nodes(init)
        got = refrun.csr_sets(rp, col, nodes)
        exp = refrun.csr_sets(ref["c_rowptr"], ref["c_col"], nodes)
        bad = [i for i in nodes if got[i] != exp[i]]
        assert not bad, f"{tag}: contact candidate sets differ at {len(bad)} nodes, e.g. {bad[:5]}"
    if int(init["test"][0]) == 2 and int(ref["n"][0]) % int(init["dtTestOut"][0]) == 0:
        assert abs(sc["reaction"] - float(ref["reaction"][0])) <= 1e-12 * max(1.0, abs(float(ref["reaction"][0]))), (tag, sc)


@pytest.mark.parametrize("case", [c for c in scenarios.CASES if c != "two_particle_pmb_impact"])
def test_fp64_matches_reference(case, tmp_path):
    factory, steps, dump_steps = scenarios.CASES[case]
    spec = factory()
    scn.write_deck(spec, str(tmp_path))
    init, dumps = refrun.run_reference(str(tmp_path), steps, dump_steps)
    _, m = _model(init)
    try:
        m.integrate_begin()
        _compare(f"{case} n=0", m, init, init)
        n = 0
        for k in sorted(dumps):
            m.integrate_step(k - n)
            n = k
            m.sync()
            _compare(f"{case} n={k}", m, dumps[k], init)
    finally:
        m.close()


def test_fp64_fracture_onset_matches_reference(tmp_path):
    """PMB impact: bonds break within the first steps; until the broken-bond
    contact makes the motion chaotic the broken sets must agree exactly."""
    factory, _, _ = scenarios.CASES["two_particle_pmb_impact"]
    spec = factory()
    scn.write_deck(spec, str(tmp_path))
    steps = list(range(1, 31))
    init, dumps = refrun.run_reference(str(tmp_path), 30, steps)
    _, m = _model(init)
    broke = 0
    try:
        m.integrate_begin()
        n = 0
        for k in steps:
            m.integrate_step(k - n)
            n = k
            m.sync()
            b = m.field("bonds")
            assert np.array_equal(b, dumps[k]["bond_state"]), f"bond sets differ at step {k}"
            broke = int(b.sum())
    finally:
        m.close()
    assert broke > 0, "scenario should break bonds within 30 steps"


def test_fp64_graph_replay_matches_stream(tmp_path):
    """The CUDA-graph replay runs the same kernels as the stream path."""
    factory, _, _ = scenarios.CASES["compressive_small"]
    spec = factory()
    scn.write_deck(spec, str(tmp_path))
    init, _ = refrun.run_reference(str(tmp_path), 1, [1])
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    sc = refrun.scene_from_dump(init)
    a = GpuDEMModel(sc, precision=PREC_FP64)
    b = GpuDEMModel(sc, precision=PREC_FP64)
    try:
        a.integrate_begin()
        b.integrate_begin()
        a.integrate_step(120)
        b.integrate_step(120, graph_steps=40)
        a.sync()
        b.sync()
        for fld in ("x", "v", "f"):
            assert np.array_equal(a.field(fld), b.field(fld)), fld
    finally:
        a.close()
        b.close()
