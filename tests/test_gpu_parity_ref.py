"""GPU parity against the reference itself: the reference's DEMModel
(oracle/_ref/peridem_ref, compiled here from the reference's own sources)
sets a scene up and steps it; the FP64 CUDA path starts from the same
ModelData (same neighbour-list order) and must reproduce its state at every
dump step within the tolerances of tests/parity.py (forces to 1e-12 after
the prelude and the first step, 1e-10 later; bond flags and contact sets
exactly).  The scenes cover the four bond laws, the three influence
functions, both time schemes, every displacement and force boundary
condition time function with the spatial factors, 2-D and 3-D.
"""
import numpy as np
import pytest

import parity
import refrun
import scenarios
from peridem_b200 import scene as scn

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refrun.have_reference(),
                                 reason="reference binary oracle/_ref/peridem_ref not built")]


@pytest.mark.parametrize("case", [c for c in scenarios.CASES if c != "two_particle_pmb_impact"])
def test_fp64_matches_reference(case, tmp_path):
    factory, steps, dump_steps = scenarios.CASES[case]
    spec = factory()
    scn.write_deck(spec, str(tmp_path))
    init, dumps = refrun.run_reference(str(tmp_path), steps, dump_steps)
    _, m = parity.model(init)
    try:
        m.integrate_begin()
        parity.compare(f"{case} n=0", m, init, init, 0)
        n = 0
        for k in sorted(dumps):
            m.integrate_step(k - n)
            n = k
            m.sync()
            parity.compare(f"{case} n={k}", m, dumps[k], init, k)
    finally:
        m.close()


def test_fp64_fracture_onset_matches_reference(tmp_path):
    """PMB impact: bonds break within the first steps; until the broken-bond
    contact makes the motion chaotic the broken sets must agree exactly, and
    over the first ten steps the PMB forces too (1e-12 at the first step,
    1e-11 after)."""
    factory, _, _ = scenarios.CASES["two_particle_pmb_impact"]
    spec = factory()
    scn.write_deck(spec, str(tmp_path))
    steps = list(range(1, 31))
    init, dumps = refrun.run_reference(str(tmp_path), 30, steps)
    _, m = parity.model(init)
    broke = 0
    try:
        m.integrate_begin()
        parity.compare("pmb n=0", m, init, init, 0)
        n = 0
        for k in steps:
            m.integrate_step(k - n)
            n = k
            m.sync()
            b = m.field("bonds")
            assert np.array_equal(b, dumps[k]["bond_state"]), f"bond sets differ at step {k}"
            if k <= 10:
                parity.compare(f"pmb n={k}", m, dumps[k], init, k)
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
    from peridem_b200.model import GpuDEMModel, PREC_FP64  # noqa: F811
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
