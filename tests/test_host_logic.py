"""Host-side logic without a GPU: the surrogate's body-frame transforms and
basis completion, the scene builder's sequential record chain, the
autotuner's search order, the bench's workload descriptions and its
layout-independent algorithmic byte count, the early stop of the
surrogate's snapshot collection (solver faked) and the safety margin of the
damping pass's FP32 pair pre-filter."""
import numpy as np
import pytest

from peridem_b200 import scene as scn


def _scene():
    return scn.build_scene(scn.compressive_2d(n_particles=6, r_range=(1e-3, 1.3e-3), h_div=6, width=8e-3,
                                              seed=3))


def test_body_frame_inverts_placement():
    from peridem_b200 import surrogate as sg
    sc = _scene()
    rng = np.random.default_rng(0)
    u = np.zeros((sc.n_nodes, 3))
    rows = {}
    for p in range(sc.n_particles):
        if sc.p_type[p] != 0:
            continue
        n = int(sc.p_end[p] - sc.p_start[p])
        rows[p] = rng.standard_normal(2 * n) * 1e-6
        sg._place(sc, u, p, rows[p])
    for p, ub in rows.items():
        # forces: a pure rotation back
        assert np.allclose(sg.body_frame(sc, u, p, relative=False), ub * sc.p_scale[p], rtol=0, atol=1e-18)
        # displacements: relative to the centre node, over the scale
        c = int(sc.p_center[p] - sc.p_start[p])
        rel = (ub.reshape(-1, 2) - ub.reshape(-1, 2)[c]).reshape(-1)
        assert np.allclose(sg.body_frame(sc, u, p, relative=True), rel, rtol=0, atol=1e-18)


def test_reference_coords_are_the_unrotated_mesh():
    from peridem_b200 import surrogate as sg
    sc = _scene()
    zs = sg.surrogate_zones(sc)
    assert zs  # discs and hexagons share one mesh each
    for z in zs:
        ps = sg._zone_particles(sc, z)
        X0 = sg.reference_coords(sc, ps[0])
        for p in ps[1:]:
            assert np.allclose(sg.reference_coords(sc, p), X0, rtol=0, atol=1e-12)


def test_complete_basis_is_orthonormal():
    from peridem_b200 import surrogate as sg
    sc = _scene()
    X = sg.reference_coords(sc, sg._zone_particles(sc, sg.surrogate_zones(sc)[0])[0])
    rng = np.random.default_rng(1)
    traj = np.linalg.qr(rng.standard_normal((2 * len(X), 5)))[0]
    B = sg.complete_basis(traj, X)
    assert B.shape == (2 * len(X), sg.RANK)
    assert np.allclose(B.T @ B, np.eye(sg.RANK), atol=1e-10)
    # the trajectory modes come first and span the same space
    assert np.allclose(np.abs(np.diag(traj.T @ B[:, :5])), 1.0, atol=1e-10)
    # constant translations are in the span (lowest-degree polynomials)
    t = np.tile([1.0, 0.0], len(X))
    t /= np.linalg.norm(t)
    assert np.linalg.norm(B @ (B.T @ t) - t) < 1e-10


def test_record_chain_matches_a_literal_scan():
    rng = np.random.default_rng(2)

    def literal(vals, g):
        idx = -1
        for k, v in enumerate(vals):
            if (g - v) > max(abs(v), abs(g)) * 1e-5:
                g, idx = float(v), k
        return idx, g

    for t in range(300):
        n = int(rng.integers(0, 200))
        if t % 3 == 0:   # near-ties within the tolerance
            vals = 1.0 + 1e-6 * rng.standard_normal(n)
        elif t % 3 == 1:  # repeated lattice distances
            vals = np.repeat(rng.uniform(0, 1, size=n // 4 + 1), 4)[:n]
        else:
            vals = np.abs(rng.standard_normal(n))
        g = float(rng.uniform(0, 2))
        assert scn._record_chain(vals, g) == literal(vals, g)


def test_autotune_descends_then_tries_skins(monkeypatch):
    from peridem_b200 import autotune as at
    from peridem_b200.model import PREC_MIXED
    sc = _scene()
    sc.search_factor = 5.0
    cost = {(1, 256, 5.0): 1.0, (4, 128, 5.0): 0.9, (1, 128, 5.0): 1.2, (4, 256, 5.0): 1.1,
            (4, 128, 2.0): 0.8, (4, 128, 3.0): 0.95}
    seen = []

    def fake(scene, precision, pd_lanes, tile_nodes, steps, warmup, device=0, contact_lanes=0, state=None):
        key = (pd_lanes, tile_nodes, float(scene.search_factor))
        seen.append(key)
        return cost.get(key, 2.0)

    monkeypatch.setattr(at, "time_candidate", fake)
    ch = at.autotune(sc, PREC_MIXED, lanes=(1, 4), tiles=(128, 256), skins=(2.0, 3.0, 5.0))
    assert (ch.pd_lanes, ch.tile_nodes, ch.search_factor) == (4, 128, 2.0)
    assert ch.ms_per_step == pytest.approx(0.8)
    # lanes x tiles on the scene's own skin first, then the other skins with the best pair
    assert seen[:4] == [(1, 128, 5.0), (1, 256, 5.0), (4, 128, 5.0), (4, 256, 5.0)]
    assert seen[4:] == [(4, 128, 2.0), (4, 128, 3.0)]
    assert sc.search_factor == 5.0  # the caller's scene is not modified
    assert len(ch.table) == 6


@pytest.mark.parametrize("workload", ["compressive", "ensemble", "column3d", "surrogate"])
def test_bench_describes_every_workload(workload):
    import argparse
    import bench
    args = argparse.Namespace(workload=workload, particles=502, scenes=256, spheres=4096, precision="mixed",
                              graph_steps=1, pd_lanes=0, tile_nodes=0, seed=0, prerun=20000)
    cfg = bench.workload_config(args, None)
    assert cfg["workload"] and cfg["precision"] == "mixed" and "l2" in cfg
    spec = bench.workload_spec(args)
    assert spec.dim in (2, 3)


def test_snapshot_collection_stops_when_no_particle_is_below_the_gate(monkeypatch):
    from peridem_b200 import model as mdl
    from peridem_b200 import surrogate as sg
    sc = _scene()
    zones = sg.surrogate_zones(sc)
    state = {"n": 0, "steps": []}

    class Fake:
        def __init__(self, scene, **kw):
            self.n = scene.n_nodes

        def integrate_begin(self):
            pass

        def integrate_step(self, k, graph_steps=0):
            state["n"] += k
            state["steps"].append(k)

        def field(self, name):
            if name == "Z":  # every particle past the gate from step 120 on
                return np.full(self.n, 0.9 if state["n"] >= 120 else 0.1, dtype=np.float32)
            if name == "bonds":
                return np.zeros(8, dtype=np.uint8)
            return np.zeros((self.n, 3))

        def set_field(self, name, values):
            pass

        def compute_pd_forces(self):
            pass

        def close(self):
            pass

    monkeypatch.setattr(mdl, "GpuDEMModel", Fake)
    monkeypatch.setattr(sg, "_probe", lambda s: Fake(s))
    snap = sg.collect_snapshots(sc, steps=400, every=40, fscale=np.ones(sc.n_particles), zones=zones)
    assert state["steps"] == [40, 40, 40]  # stopped at the first snapshot with nothing to record
    for z in zones:
        assert len(snap.u[z]) == 2 * len(sg._zone_particles(sc, z))


@pytest.mark.parametrize("dim", [2, 3])
def test_bench_algorithmic_bytes_are_layout_independent(dim):
    """Per bond a 32-bit index and the broken bit; per active node FP64 (or,
    in the mixed form, FP32) coordinates and displacement, FP64 volume, row
    offset and force, FP32 damage."""
    import bench

    class S:
        pass

    sc = S()
    sc.dim, sc.n_nodes, sc.n_particles = dim, 5, 2
    sc.p_compute_force, sc.p_start, sc.p_end = [1, 0], [0, 3], [3, 5]
    sc.pd_rowptr = np.array([0, 2, 5, 6, 8, 9])
    sc.p_material = [0, 0]
    b64, u64 = bench.algorithmic_bytes("pd_force", sc, "fp64")
    b32, u32 = bench.algorithmic_bytes("pd_force_mixed", sc, "mixed")
    assert u64["bonds"] == u32["bonds"] == 6 and u64["nodes"] == u32["nodes"] == 3
    assert u64["bytes_per_bond"] == u32["bytes_per_bond"] == 4.125
    assert u64["bytes_per_node"] == 8 * dim * 3 + 8 + 8 + 4
    assert u32["bytes_per_node"] == 4 * dim * 2 + 8 + 8 + 8 * dim + 4
    assert b32 == 6 * 4.125 + 3 * u32["bytes_per_node"]


@pytest.mark.parametrize("kind", ["RNPBond", "PMBBond", "PDElasticBond", "PDState"])
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("inf_type", [0, 1, 2])
def test_library_deck_constants_equal_the_scene_builder_and_reference(kind, dim, inf_type):
    """pdgpu_material_constants / pdgpu_influence_params (host functions of
    the library, for bindings that hold only the decks) give the same bits as
    the scene builder's restatement, which tests/test_scene.py pins to the
    reference's own init."""
    import ctypes
    from peridem_b200 import api
    from peridem_b200.model import MATERIAL_CODES
    L = api.lib()
    m = scn.elastic_material(kind, 2.0e9)
    m.influence_type = inf_type
    t, inf = scn.influence_params(m, dim)
    out = (ctypes.c_double * 2)()
    assert L.pdgpu_influence_params(inf_type, 0, None, dim, out) == 0
    assert (t, float(inf[0]), float(inf[1])) == (inf_type, out[0], out[1])
    for horizon in (3e-4, 1.234567e-4):
        code, mat, Kp = scn.material_constants(m, dim, horizon, t, inf)
        deck = api.MaterialDeck(law=MATERIAL_CODES[kind], irreversible=1 if m.irreversible else 0, E=m.E, K=m.K,
                                G=m.G, nu=m.nu, Gc=m.Gc, check_sc_factor=m.check_sc_factor)
        got = (ctypes.c_double * 6)()
        kb = ctypes.c_double()
        ip = (ctypes.c_double * 2)(*inf)
        assert L.pdgpu_material_constants(ctypes.byref(deck), dim, horizon, t, ip, got, ctypes.byref(kb)) == 0
        assert list(got) == [float(v) for v in mat], (kind, dim, inf_type)
        assert kb.value == Kp


def test_library_deck_constants_equal_the_reference_dump():
    """The reference's own constants (dumped from its materials) for the
    golden scenes: RNP, PMB, PD elastic and PD state, 2-D and 3-D."""
    import ctypes
    import golden_io
    from peridem_b200 import api
    L = api.lib()
    kinds = {"tp6_rnp": "RNPBond", "tp6_pmb_impact": "PMBBond", "tp6_state": "PDState",
             "tp6_pdelastic_verlet": "PDElasticBond", "col3_state": "PDState", "col3_rnp": "RNPBond"}
    for name, kind in kinds.items():
        init, _ = golden_io.load(name)
        dim = int(init["dim"][0])
        Np = int(init["Np"][0])
        mp = init["p_mat_params"].reshape(Np, 8)
        ip = (ctypes.c_double * 2)(*[float(v) for v in init["inf_params"][:2]])
        for p in range(Np):
            if int(init["p_type"][p]) != 0:
                continue
            deck = api.MaterialDeck(law=int(init["p_mat_type"][p]), irreversible=1, E=-1.0, K=-1.0, G=-1.0,
                                    nu=-1.0, Gc=500.0, check_sc_factor=1.0)
            E = 2.0e9 if name.startswith("tp6") else 5.0e9
            deck.E, deck.K = E, E / (3.0 * (1.0 - 2.0 * 0.25))
            got = (ctypes.c_double * 6)()
            rc = L.pdgpu_material_constants(ctypes.byref(deck), dim, float(init["p_horizon"][p]),
                                            int(init["inf_type"][0]), ip, got, None)
            assert rc == 0
            n = {0: 6, 1: 2, 2: 1, 3: 3}[int(init["p_mat_type"][p])]
            assert list(got)[:n] == [float(v) for v in mp[p, :n]], (name, kind, p)


def test_damping_fp32_prefilter_never_rejects_a_pair_the_fp64_test_passes():
    """The particle-damping pair search first tests FP32 copies of the
    centres and bounding radii, d2 > 1.17 (R_i + R_j + 1.01 rc_max)^2, and
    only the pairs it keeps reach the FP64 test of the one-particle form,
    d2 > 1.0625 reach_max^2 (then the exact contact test).  Restated here in
    NumPy with the kernel's FP32 operation order, over random pairs in a box
    far from the origin (where rounding the coordinates to FP32 costs the
    most) and pairs placed right at the FP64 threshold: no pair the FP64
    test keeps is rejected by the FP32 one."""
    rng = np.random.default_rng(5)
    n = 200000
    f32 = np.float32
    ri = rng.uniform(0.8e-3, 1.6e-3, n)
    rj = rng.uniform(0.8e-3, 1.6e-3, n)
    rc = 1.01 * 2.0e-4
    reach = rj + ri + rc
    ci = rng.uniform(-0.1, 0.1, (n, 3)) + 0.5          # centres around 0.5 m
    # half the pairs just inside the FP64 threshold, half anywhere nearby
    d = np.where(rng.random(n) < 0.5, np.sqrt(1.0625) * reach * (1 - 1e-12),
                 rng.uniform(0.0, 1.5, n) * reach)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    cj = ci + d[:, None] * u
    dx = cj - ci
    keep64 = ~((dx * dx).sum(1) > 1.0625 * reach * reach)
    e = cj.astype(f32) - ci.astype(f32)
    d2f = (e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1]) + e[:, 2] * e[:, 2]
    rmf = (rj.astype(f32) + ri.astype(f32)) + f32(rc)
    keep32 = ~(d2f > f32(1.17) * rmf * rmf)
    assert keep64.sum() > n // 3
    assert not np.any(keep64 & ~keep32)
