"""Host side of batched ensembles (no GPU): scene generation, merging and
the mesh-size scan the scene builder follows."""
import numpy as np

from peridem_b200 import scene as scn


def test_mesh_size_matches_full_scan():
    rng = np.random.default_rng(0)
    for trial in range(40):
        hd = int(rng.integers(4, 16))
        nodes, _ = (scn.disc_mesh if trial % 2 else scn.hexagon_mesh)(1e-3, 1e-3 / hd)
        x = np.array([rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05), 0.0]) + \
            rng.uniform(0.7, 1.6) * scn._rotate_z(np.asarray(nodes, float), rng.uniform(0, 6.3))
        if trial % 5 == 0:  # irregular spacing
            x[:, :2] += rng.normal(scale=2e-6, size=(len(x), 2))
        assert scn.mesh_size(x) == scn.mesh_size_scan(x)


def test_merge_keeps_scenes_apart_and_tables_block_diagonal():
    specs = scn.ensemble_specs(n_scenes=3, seed=2, n_range=(4, 9), h_div_range=(4, 6))
    assert len({s.dt for s in specs}) == 1
    scenes = [scn.build_scene(s) for s in specs]
    ens = scn.merge_scenes(scenes)
    assert ens.n_nodes == sum(s.n_nodes for s in scenes)
    assert ens.n_particles == sum(s.n_particles for s in scenes)
    assert list(ens.scene_poff) == list(np.cumsum([0] + [s.n_particles for s in scenes]))
    nz = ens.n_zones
    rc = ens.c_rc.reshape(nz, nz)
    z0 = 0
    boxes = []
    for k, s in enumerate(scenes):
        blk = rc[z0:z0 + s.n_zones, z0:z0 + s.n_zones]
        assert np.array_equal(blk, s.c_rc.reshape(s.n_zones, s.n_zones))
        off = np.delete(rc[z0:z0 + s.n_zones], np.s_[z0:z0 + s.n_zones], axis=1)
        assert not off.any()
        p0, p1 = ens.scene_poff[k], ens.scene_poff[k + 1]
        n0 = ens.p_start[p0]
        assert np.array_equal(ens.p_zone[p0:p1], s.p_zone + z0)
        assert np.array_equal(ens.p_start[p0:p1] - n0, s.p_start)
        assert ens.scene_walls[k] == s.test_wall + p0
        x = ens.xref[n0:n0 + s.n_nodes]
        # the same geometry, shifted
        shift = x[0] - s.xref[0]
        assert np.allclose(x - shift, s.xref, rtol=0, atol=1e-12)
        boxes.append((x.min(axis=0), x.max(axis=0)))
        z0 += s.n_zones
    reach = ens.search_factor * ens.max_contact_r
    for a in range(len(boxes)):
        for b in range(a + 1, len(boxes)):
            gap = np.maximum(boxes[b][0] - boxes[a][1], boxes[a][0] - boxes[b][1])
            assert np.max(gap[:2]) > 2 * reach
    # one moving-wall set per scene, on that scene's wall nodes only
    assert len(ens.ubc) == len(scenes)
    for k, b in enumerate(ens.ubc):
        assert b.sparse and list(b.particle_sel) == [ens.scene_walls[k]]
        w = ens.scene_walls[k]
        assert set(b.node_sel) == set(range(ens.p_start[w], ens.p_end[w]))
