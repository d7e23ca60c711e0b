"""Test helpers: run the reference (oracle/_ref/peridem_ref) on a scene deck
and load its dumps; compare GPU state against them.

ORACLE TEST INFRASTRUCTURE: the reference binary and its dumps are the
checker, never the thing measured.
"""
import os
import subprocess

import numpy as np

from refdump import read_dump, scene_from_dump  # noqa: F401  (oracle/)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "peridem_ref")


def have_reference() -> bool:
    return os.path.exists(REF_BIN)


def run_reference(deck_dir: str, steps: int, dump_steps, threads: int = 1, timeout: int = 900):
    """Run the reference on deck_dir/deck.yaml; return (init dump, {n: dump})."""
    deck_dir = os.path.abspath(deck_dir)
    out = os.path.join(deck_dir, "dump")
    os.makedirs(out, exist_ok=True)
    cmd = [REF_BIN, "-i", "deck.yaml", "-nThreads", str(threads), "-dump", out,
           "-steps", str(steps), "-dumpSteps", ",".join(str(s) for s in dump_steps)]
    r = subprocess.run(cmd, cwd=deck_dir, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}")
    init = read_dump(os.path.join(out, "init.bin"))
    dumps = {n: read_dump(os.path.join(out, f"step_{n}.bin")) for n in dump_steps if n <= steps}
    return init, dumps


def rel_err(a, b, floor=0.0):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(float(np.max(np.abs(b))) if b.size else 0.0, floor)
    if den == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b))) / den


def csr_sets(rowptr, col, rows=None):
    rowptr = np.asarray(rowptr, dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    rows = range(len(rowptr) - 1) if rows is None else rows
    return {int(i): frozenset(col[rowptr[i]:rowptr[i + 1]].tolist()) for i in rows}


def bonds_by_pair(rowptr, col, state):
    """bond state keyed by (i, j), independent of list order"""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    out = {}
    for i in range(len(rowptr) - 1):
        for k in range(rowptr[i], rowptr[i + 1]):
            out[(i, int(col[k]))] = int(state[k])
    return out
