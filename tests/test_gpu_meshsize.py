"""pdgpu_mesh_size, util::computeMeshSize (geom.cpp:578-604) on the device,
against the reference: bit for bit with the mesh sizes the reference's own
BaseParticle computed for every golden fixture (d_h of each particle, walls
included), with the scene builder's exact restatement on the benchmark's
502-particle scene and a 3-D packing, and with a literal transcription of
the reference's O(n^2) scan on random clouds whose record chains are long.
"""
import ctypes

import numpy as np
import pytest

import golden_io
from peridem_b200 import scene as scn

pytestmark = pytest.mark.gpu


def _device(x, starts, ends):
    from peridem_b200 import api
    L = api.lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    s = np.ascontiguousarray(starts, dtype=np.int64)
    e = np.ascontiguousarray(ends, dtype=np.int64)
    h = np.zeros(len(s))
    P = ctypes.POINTER
    rc = L.pdgpu_mesh_size(0, x.ctypes.data_as(P(ctypes.c_double)), len(x), s.ctypes.data_as(P(ctypes.c_int64)),
                           e.ctypes.data_as(P(ctypes.c_int64)), len(s), h.ctypes.data_as(P(ctypes.c_double)))
    assert rc == 0
    return h


def _literal(x):
    """The reference's loop, pair by pair."""
    def is_less(a, b):
        return (b - a) > max(abs(a), abs(b)) * 1e-5
    n = len(x)
    if n < 2:
        return 0.0
    g = float(np.sqrt(np.sum((x[0] - x[1]) ** 2)))
    for i in range(n):
        d = np.sqrt((x[i, 0] - x[:, 0]) ** 2 + (x[i, 1] - x[:, 1]) ** 2 + (x[i, 2] - x[:, 2]) ** 2)
        for j in range(n):
            if i != j and is_less(float(d[j]), g):
                g = float(d[j])
    return g


@pytest.mark.parametrize("name", golden_io.names())
def test_mesh_size_matches_reference_particles(name):
    init, _ = golden_io.load(name)
    N = int(init["N"][0])
    h = _device(init["xRef"].reshape(N, 3), init["p_globStart"], init["p_globEnd"])
    assert np.array_equal(h, init["p_h"]), np.max(np.abs(h - init["p_h"]))


def test_mesh_size_at_benchmark_size_and_in_3d():
    for spec in (scn.compressive_2d(n_particles=502, packing="deposit"),
                 scn.column_3d(n_spheres=27, median_r=1e-3, sigma=0.2, h_div=6, box=(8e-3, 8e-3, 12e-3),
                               seed=4, nt=10, wall_h=6e-4)):
        sc = scn.build_scene(spec)
        h = _device(sc.xref, sc.p_start, sc.p_end)
        want = np.array([scn.mesh_size(sc.xref[sc.p_start[p]:sc.p_end[p]]) for p in range(sc.n_particles)])
        assert np.array_equal(h, want), float(np.max(np.abs(h - want)))
        assert np.array_equal(h, np.asarray(sc.p_h)), "the scene's own mesh sizes"


def test_mesh_size_follows_long_record_chains():
    rng = np.random.default_rng(5)
    clouds = []
    for k in range(6):
        n = int(rng.integers(2, 160))
        c = rng.uniform(0, 1e-3, size=(n, 3))
        if k % 2:
            c[:, 2] = 0.0
        if k == 3:  # near-ties within the relative epsilon
            c = np.repeat(c[:1], n, axis=0) + np.arange(n)[:, None] * np.array([1e-4, 0, 0]) * (1 + 1e-7 * rng.standard_normal((n, 1)))
        clouds.append(c)
    x = np.concatenate(clouds)
    ends = np.cumsum([len(c) for c in clouds])
    starts = np.concatenate([[0], ends[:-1]])
    h = _device(x, starts, ends)
    want = np.array([_literal(c) for c in clouds])
    assert np.array_equal(h, want), (h, want)
