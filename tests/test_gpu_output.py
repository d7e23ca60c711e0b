"""VTU output and restart (DEMModel::output / DEMModel::restart).

* the file is VTK XML UnstructuredGrid with the reference's array names,
  its points are the current positions and its arrays the model's fields;
* a run restarted from the file written at step n continues as the
  uninterrupted run: after another m steps the FP64 displacement and
  velocity fields agree to 1e-10 (the restart restores x, u, v, as the
  reference's does; no bond breaks in this scene).  They are not
  bit-identical: like the reference, the restart sets the time to n dt,
  while the uninterrupted run has summed dt n times, so the moving wall's
  prescribed displacement differs in its last bits (observed: 1e-12 in u,
  3e-12 in v after 1 000 contact steps).
"""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from peridem_b200 import scene as scn

pytestmark = pytest.mark.gpu

TAGS = ("Displacement", "Velocity", "Force", "Force_Density", "Damage_Z", "Particle_ID", "Zone_ID",
        "Fixity", "Nodal_Volume")


def _scene():
    h = 1e-3 / 8
    return scn.build_scene(scn.compressive_2d(n_particles=12, r_range=(1e-3, 1.3e-3), h_div=8, width=10e-3,
                                              seed=7, gap=1.02 * h, wall_speed=-2.0, nt=3000))


def _model(sc):
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    return GpuDEMModel(sc, precision=PREC_FP64, build_neighbors=True, compute_mx=True)


def _read(path):
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">')
    root = ET.fromstring(head.decode() + "</VTKFile>")
    base = rest.index(b"_") + 1
    arrays = {}
    for da in root.iter("DataArray"):
        off = int(da.get("offset"))
        nb = int(np.frombuffer(rest[base + off:base + off + 8], dtype=np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[da.get("type")]
        a = np.frombuffer(rest[base + off + 8:base + off + 8 + nb], dtype=dt)
        arrays[da.get("Name")] = a.reshape(-1, int(da.get("NumberOfComponents", "1")))
    return root, arrays


def test_vtu_holds_the_model_state(tmp_path):
    sc = _scene()
    m = _model(sc)
    try:
        m.integrate_begin()
        m.integrate_step(200)
        path = str(tmp_path / "output_1.vtu")
        m.write_vtu(path, TAGS)
        x, u, v, f = (m.field(k) for k in ("x", "u", "v", "f"))
        Z = m.field("Z")
        t = m.scalars()["time"]
    finally:
        m.close()
    root, arr = _read(path)
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfPoints")) == sc.n_nodes and int(piece.get("NumberOfCells")) == 0
    assert arr["TIME"][0, 0] == t
    assert np.array_equal(arr["Points"], x)
    assert np.array_equal(arr["Displacement"], u) and np.array_equal(arr["Velocity"], v)
    assert np.array_equal(arr["Force_Density"], f)
    assert np.allclose(arr["Force"], f * sc.vol[:, None], rtol=1e-15, atol=0)
    assert np.array_equal(arr["Damage_Z"][:, 0], Z.astype(np.float64))
    assert np.array_equal(arr["Particle_ID"][:, 0], sc.ptid.astype(np.float64))
    assert np.array_equal(arr["Zone_ID"][:, 0], sc.p_zone[sc.ptid.astype(np.int64)].astype(np.float64))
    assert np.array_equal(arr["Nodal_Volume"][:, 0], sc.vol)
    assert set(arr) == {"TIME", "Points", "connectivity", "offsets", "types"} | set(TAGS)


def test_restart_continues_the_run(tmp_path):
    sc = _scene()
    n, m_steps = 1000, 1000
    a = _model(sc)
    try:
        a.integrate_begin()
        a.integrate_step(n)
        path = str(tmp_path / "restart.vtu")
        a.write_vtu(path, ("Displacement", "Velocity"))
        a.integrate_step(m_steps)
        ua, va, ha = a.field("u"), a.field("v"), a.history()
        ta = a.scalars()["time"]
    finally:
        a.close()
    b = _model(sc)
    try:
        b.restart(path, n)
        b.integrate_begin()
        b.integrate_step(m_steps)
        ub, vb = b.field("u"), b.field("v")
        tb = b.scalars()["time"]
        sb = b.scalars()
    finally:
        b.close()
    eu = float(np.max(np.abs(ua - ub))) / float(np.max(np.abs(ua)))
    ev = float(np.max(np.abs(va - vb))) / float(np.max(np.abs(va)))
    print(f"restart at {n}: after {m_steps} more steps u rel {eu:.2e}, v rel {ev:.2e}; step {sb['n']}")
    assert sb["n"] == n + m_steps and abs(ta - tb) <= 1e-12 * ta
    assert float(np.max(np.abs(ha[:, 3]))) > 0, "the wall never touched the packing"
    assert eu <= 1e-10 and ev <= 1e-10


def test_async_output_writes_the_state_of_its_call(tmp_path):
    """pdgpu_write_vtu_async: the file holds the state as of the call, byte
    for byte what pdgpu_write_vtu writes then, although steps run while it
    is written."""
    sc = _scene()
    m = _model(sc)
    try:
        m.integrate_begin()
        m.integrate_step(30)
        a, b = str(tmp_path / "sync.vtu"), str(tmp_path / "async.vtu")
        m.write_vtu(a)
        m.write_vtu_async(b)
        m.integrate_step(50)   # issued while the file is written
        m.output_wait()
        assert open(a, "rb").read() == open(b, "rb").read()
        # a second call waits for nothing left over and writes the newer state
        c = str(tmp_path / "async2.vtu")
        m.write_vtu_async(c)
        m.output_wait()
        m.sync()
        d = str(tmp_path / "sync2.vtu")
        m.write_vtu(d)
        assert open(c, "rb").read() == open(d, "rb").read()
        assert open(a, "rb").read() != open(c, "rb").read()
    finally:
        m.close()
