"""Regenerates the golden fixtures in this directory from the reference
itself: each scene deck is run by oracle/_ref/peridem_ref (the reference's
own DEMModel compiled from its sources) and the init state plus the states
after selected steps are stored as compressed npz.

    python tests/golden/make_golden.py [name ...]   (needs oracle/_ref/peridem_ref;
                                                     all cases when no name is given)

ORACLE TEST INFRASTRUCTURE: fixtures pin the oracle restatement; they are
never inputs of the product path.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import refrun  # noqa: E402
from peridem_b200 import scene  # noqa: E402

R = 1e-3
STEP_KEYS = ["n", "time", "x", "u", "v", "f", "Z", "vMag", "thetaX", "bond_state", "c_rowptr",
             "c_col", "contNeighUpdateInterval", "contNeighSearchRadius",
             "contNeighTimestepCounter", "maxVelocity", "reaction", "wall_penetration",
             "pen_dist", "max_y"]


def cases():
    # the committed fixtures were made from decks whose particle meshes list
    # their nodes in grid order (first index slowest)
    saved = scene.MESH_ORDER
    scene.MESH_ORDER = "grid"
    try:
        return _cases()
    finally:
        scene.MESH_ORDER = saved


def _cases():
    out = {}
    out["tp6_rnp"] = (scene.two_particle(h_div=6, radius=R, material="RNPBond", v0=-1.0,
                                         gap=0.02 * R / 6, nt=150), 150, [1, 25, 75, 150])
    out["tp6_pmb_impact"] = (scene.two_particle(h_div=6, radius=R, material="PMBBond", v0=-40.0,
                                                gap=0.01 * R / 6, nt=30), 30, [1, 5, 10, 20, 30])
    out["tp6_state"] = (scene.two_particle(h_div=6, radius=R, material="PDState", v0=-2.0,
                                           gap=0.02 * R / 6, nt=120), 120, [1, 40, 120])
    s = scene.two_particle(h_div=6, radius=R, material="PDElasticBond", v0=-1.0, gap=0.02 * R / 6,
                           nt=80)
    s.time_scheme = "velocity_verlet"
    out["tp6_pdelastic_verlet"] = (s, 80, [1, 40, 80])
    h = R / 4
    out["cmp6_rnp"] = (scene.compressive_2d(n_particles=6, r_range=(R, 1.2 * R), h_div=4,
                                            width=8e-3, seed=5, gap=1.02 * h, wall_speed=-3.0,
                                            nt=200, search_interval=10), 200, [1, 50, 200])
    # 3-D: two PD-state spheres in a box under a piston (walls meshed coarser
    # than the spheres to keep the fixture small)
    out["col3_state"] = (scene.column_3d(n_spheres=2, median_r=R, sigma=0.0, h_div=4,
                                         box=(3e-3, 3e-3, 6e-3), seed=1, material="PDState",
                                         piston_speed=-2.0, nt=150, wall_h=5e-4), 150, [1, 150])
    out["col3_rnp"] = (scene.column_3d(n_spheres=2, median_r=R, sigma=0.0, h_div=4,
                                       box=(3e-3, 3e-3, 6e-3), seed=2, material="RNPBond",
                                       piston_speed=-2.0, nt=150, wall_h=5e-4), 150, [1, 150])
    return out


def main(only=()):
    if not refrun.have_reference():
        sys.exit("oracle/_ref/peridem_ref is not built (make -C oracle ref)")
    for name, (spec, steps, dsteps) in cases().items():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as d:
            scene.write_deck(spec, d)
            init, dumps = refrun.run_reference(d, steps, dsteps)
        arrays = {f"init/{k}": v for k, v in init.items()}
        for n, dd in dumps.items():
            for k in STEP_KEYS:
                arrays[f"step{n}/{k}"] = dd[k]
        arrays["meta/steps"] = np.array(sorted(dumps))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **arrays)
        print(name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:])
