"""Loads the golden fixtures (tests/golden/*.npz) written by
tests/golden/make_golden.py from the reference's own runs."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The scene fixtures (strain_*.npz hold the strain/stress fixtures of
    tests/golden/make_strain_golden.py instead)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("strain_"))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    init = {k[5:]: z[k] for k in z.files if k.startswith("init/")}
    steps = {}
    for n in z["meta/steps"]:
        pre = f"step{int(n)}/"
        steps[int(n)] = {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}
    return init, steps
