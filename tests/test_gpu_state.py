"""State snapshots (pdgpu_save_state / pdgpu_load_state): a restart that
keeps the bond-broken bits and everything else a step reads.  A model loaded
from a snapshot taken at step k must continue exactly as the saved model
does (bit for bit: positions, velocities, forces, bond bits, damage, contact
lists and control, compressive-test history), in both precisions, with
bonds already broken and with contact.  The portable part of the file
(header, util::Point arrays, broken bonds as node pairs) is read back here
without the library.
"""
import os
import struct

import numpy as np
import pytest

import golden_io
import refrun

pytestmark = pytest.mark.gpu

HEADER = struct.Struct("<8s15q d 2q 2d q")  # SnapHeader of pdgpu_runtime.cu


def _read_portable(path):
    with open(path, "rb") as fh:
        raw = fh.read(HEADER.size)
        v = HEADER.unpack(raw)
        keys = ("magic", "dim", "n_nodes", "n_bonds", "n_particles", "stride", "n_broken", "n_words",
                "entries", "wp_cap", "history", "n_scenes", "scene_hist_cap", "surrogate",
                "multi_particle", "step")
        h = dict(zip(keys, v[:16]))
        h["time"] = v[16]
        h["contact_interval"], h["contact_counter"] = v[17], v[18]
        h["contact_radius"], h["max_velocity"] = v[19], v[20]
        h["ctrl_bytes"] = v[21]
        N = h["n_nodes"]
        xuv = np.frombuffer(fh.read(9 * N * 8), dtype=np.float64).reshape(3, N, 3)
        pairs = np.frombuffer(fh.read(16 * h["n_broken"]), dtype=np.uint64).reshape(-1, 2)
    return h, xuv, pairs


def _state(m):
    out = {k: m.field(k) for k in ("x", "u", "v", "f", "Z", "bonds", "vMag")}
    sc = m.scalars()
    out["scalars"] = {k: sc[k] for k in ("n", "time", "contact_update_interval", "contact_counter",
                                         "contact_search_radius", "contact_entries", "broken_bonds",
                                         "reaction", "contact_reaction")}
    if m.scene.multi_particle:
        out["contact"] = m.contact_lists()
    if m.scene.test == 2:
        out["history"] = m.history()
    return out


def _same(tag, a, b):
    for k in a:
        if k == "scalars":
            assert a[k] == b[k], (tag, a[k], b[k])
        elif k == "contact":
            assert np.array_equal(a[k][0], b[k][0]) and np.array_equal(a[k][1], b[k][1]), (tag, k)
        else:
            assert np.array_equal(a[k], b[k]), (tag, k, float(np.max(np.abs(
                a[k].astype(np.float64) - b[k].astype(np.float64)))))


CASES = [("cmp6_rnp", 60, 140), ("tp6_pmb_impact", 30, 20), ("col3_state", 50, 100)]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name,k1,k2", CASES)
def test_snapshot_continues_exactly(name, k1, k2, prec, tmp_path):
    from peridem_b200.model import GpuDEMModel, PREC_FP64, PREC_MIXED
    p = PREC_FP64 if prec == "fp64" else PREC_MIXED
    init, _ = golden_io.load(name)
    sc = refrun.scene_from_dump(init)
    path = str(tmp_path / "state.pdsnap")
    a = GpuDEMModel(sc, precision=p)
    try:
        a.integrate_begin()
        a.integrate_step(k1)
        a.sync()
        a.save_state(path)
        saved = _state(a)
        a.integrate_step(k2)
        a.sync()
        want = _state(a)
    finally:
        a.close()
    b = GpuDEMModel(sc, precision=p)
    try:
        b.load_state(path)
        _same(f"{name} {prec} after load", saved, _state(b))
        b.integrate_step(k2)
        b.sync()
        _same(f"{name} {prec} after {k2} more steps", want, _state(b))
    finally:
        b.close()
    # the portable part, read without the library
    h, xuv, pairs = _read_portable(path)
    assert h["magic"] == b"PDSNAP01" and h["step"] == k1 == saved["scalars"]["n"]
    assert h["time"] == saved["scalars"]["time"]
    assert h["contact_interval"] == saved["scalars"]["contact_update_interval"]
    for q, k in enumerate(("x", "u", "v")):
        assert np.array_equal(xuv[q], saved[k]), k
    rp = np.asarray(sc.pd_rowptr, dtype=np.int64)
    col = np.asarray(sc.pd_col, dtype=np.int64)
    broken = {(int(i), int(col[kk])) for i in range(sc.n_nodes) for kk in range(rp[i], rp[i + 1])
              if saved["bonds"][kk]}
    assert {(int(i), int(j)) for i, j in pairs} == broken
    if name == "tp6_pmb_impact":
        assert len(broken) > 0, "the snapshot should carry broken bonds"


def test_fp64_model_continues_from_a_mixed_snapshot(tmp_path):
    from peridem_b200.model import GpuDEMModel, PREC_FP64, PREC_MIXED
    init, _ = golden_io.load("cmp6_rnp")
    sc = refrun.scene_from_dump(init)
    path = str(tmp_path / "mixed.pdsnap")
    a = GpuDEMModel(sc, precision=PREC_MIXED)
    try:
        a.integrate_begin()
        a.integrate_step(50)
        a.save_state(path)
        saved = _state(a)
    finally:
        a.close()
    b = GpuDEMModel(sc, precision=PREC_FP64)
    try:
        b.load_state(path)
        got = _state(b)
        for k in ("x", "u", "v", "bonds"):
            assert np.array_equal(got[k], saved[k]), k
        b.integrate_step(20)
        b.sync()
        assert b.scalars()["n"] == 70
    finally:
        b.close()


def test_snapshot_of_another_scene_is_refused(tmp_path):
    from peridem_b200 import api
    from peridem_b200.model import GpuDEMModel
    path = str(tmp_path / "a.pdsnap")
    sa = refrun.scene_from_dump(golden_io.load("tp6_rnp")[0])
    sb = refrun.scene_from_dump(golden_io.load("cmp6_rnp")[0])
    a = GpuDEMModel(sa)
    try:
        a.integrate_begin()
        a.integrate_step(3)
        a.save_state(path)
    finally:
        a.close()
    b = GpuDEMModel(sb)
    try:
        if sb.n_nodes == sa.n_nodes and sb.n_bonds == sa.n_bonds:
            pytest.skip("the two fixtures have the same sizes")
        with pytest.raises(api.PdgpuError):
            b.load_state(path)
        with open(path, "wb") as fh:
            fh.write(b"not a snapshot")
        with pytest.raises(api.PdgpuError):
            b.load_state(path)
    finally:
        b.close()
    assert os.path.exists(path)
