"""The FP64 CUDA path against every golden fixture the reference wrote
(tests/golden, made by tests/golden/make_golden.py from the reference's own
DEMModel): RNP, PMB with fracture, PD state, PD elastic with velocity
Verlet, a compressive scene with walls, and 3-D PD state and RNP spheres in
a box under a piston.  Starting from the reference's init state (its own
neighbour-list order), the state after the integrate() prelude and at every
stored step must match within the tolerances of tests/parity.py.  No
reference binary is needed: the fixtures travel with the tests.

The PMB impact breaks bonds within its first steps; once broken-bond contact
makes the motion chaotic (after step 10) only the number of broken bonds is
compared, as tests/test_oracle.py does for the C restatement.
"""
import pytest

import golden_io
import parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_io.names())
def test_fp64_matches_golden(name):
    init, steps = golden_io.load(name)
    _, m = parity.model(init)
    try:
        m.integrate_begin()
        parity.compare(f"{name} n=0", m, init, init, 0)
        n = 0
        for k in sorted(steps):
            m.integrate_step(k - n)
            n = k
            m.sync()
            ref = steps[k]
            if name == "tp6_pmb_impact" and k > 10:
                got, exp = int(m.field("bonds").sum()), int(ref["bond_state"].sum())
                assert abs(got - exp) <= 2, f"{name} n={k}: broken bonds {got} vs {exp}"
                continue
            parity.compare(f"{name} n={k}", m, ref, init, k)
    finally:
        m.close()
