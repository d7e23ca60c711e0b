"""Regenerates tests/golden/strain_tri.npz: quadrature-point strain and
stress of linear triangle meshes computed by the reference itself
(oracle/_ref/ref_strain: fe::getCurrentQuadPoints and fe::getStrainStress
compiled from the reference's sources) for quadrature orders 1 and 2 (the
orders whose rules fit the three entries per element the reference
stores), in plane strain and plane stress.

    python tests/golden/make_strain_golden.py   (needs oracle/_ref/ref_strain)

The mesh: the nodes of scene.two_particle(h_div=6) (two discs, R = 1 mm,
h = R/6), each particle's grid squares split into two triangles (global
node ids), displaced by a smooth field plus noise (up to ~1e-5 m, so that
the reference's u + dN/dx sums mix both magnitudes); nu = 0.25 and the
Lame constants of E = 2 GPa.  The GPU test builds the same scene, so the
device reads the same reference coordinates.  tests/golden/strain_tet.npz:
the same for the linear tetrahedra of a two-sphere column (six per grid
cube of each sphere's mesh, h = R/4), the one-point rule.

ORACLE TEST INFRASTRUCTURE: fixtures pin the oracle restatement and the
device kernel; they are never inputs of the product path.
"""
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT]

from peridem_b200 import fe, scene  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "ref_strain")


def run_reference(xref, u, conn, order, plane_strain, nu, lam, mu):
    conn = np.asarray(conn)
    tet = conn.shape[1] == 4
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<7q", 3 if tet else 2, len(xref), len(conn), conn.shape[1],
                                fe.VTK_TETRA if tet else fe.VTK_TRIANGLE, order, int(plane_strain)))
            f.write(struct.pack("<3d", nu, lam, mu))
            f.write(np.ascontiguousarray(xref, dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(u, dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(conn, dtype="<i8").tobytes())
        subprocess.run([BIN, fin, fout], check=True)
        raw = open(fout, "rb").read()
    n = struct.unpack_from("<q", raw, 0)[0]
    a = np.frombuffer(raw, dtype="<f8", offset=8)
    return a[:3 * n].reshape(n, 3), a[3 * n:9 * n].reshape(n, 6), a[9 * n:15 * n].reshape(n, 6)


def scene_spec():
    return scene.two_particle(h_div=6, radius=1e-3, material="RNPBond", nt=10)


def mesh(sc):
    """Triangles of every particle of a built scene: global connectivity."""
    h = 1e-3 / 6
    conn = []
    for p in range(sc.n_particles):
        a, b, c = int(sc.p_start[p]), int(sc.p_end[p]), int(sc.p_center[p])
        conn.append(a + fe.grid_triangles(sc.xref[a:b] - sc.xref[c], h))
    return np.concatenate(conn)


def scene_spec_3d():
    return scene.column_3d(n_spheres=2, median_r=2e-3, sigma=0.1, h_div=4, box=(6e-3, 6e-3, 12e-3), seed=3,
                           nt=10, wall_h=1e-3, wall_layers=1.0)


def mesh_3d(sc, spec):
    """Tetrahedra of every sphere: connectivity from the zone's reference mesh
    (grid-aligned), offset to each sphere's first node."""
    z = spec.zones[0]
    h = z.geom_params[0] / 4
    local = fe.grid_tetrahedra(np.asarray(z.mesh_nodes), h)
    conn = [int(sc.p_start[p]) + local for p in range(sc.n_particles) if sc.p_type[p] == 0]
    return np.concatenate(conn)


def displacement(x):
    rng = np.random.default_rng(11)
    u = np.zeros_like(x)
    u[:, 0] = 1e-5 * np.sin(900.0 * x[:, 1]) + 2e-6 * rng.standard_normal(len(x))
    u[:, 1] = -8e-6 * np.cos(700.0 * x[:, 0]) + 2e-6 * rng.standard_normal(len(x))
    return u


def main():
    E, nu = 2.0e9, 0.25
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    sc = scene.build_scene(scene_spec())
    x = np.asarray(sc.xref, dtype=np.float64)
    u = displacement(x)
    conn = mesh(sc)
    out = {"xref": x, "u": u, "conn": conn, "material": np.array([nu, lam, mu])}
    for order in (1, 2):
        for ps in (0, 1):
            xq, e, s = run_reference(x, u, conn, order, ps, nu, lam, mu)
            key = f"o{order}_ps{ps}"
            out[key + "_xq"], out[key + "_strain"], out[key + "_stress"] = xq, e, s
    np.savez_compressed(os.path.join(HERE, "strain_tri.npz"), **out)
    spec = scene_spec_3d()
    sc = scene.build_scene(spec)
    x = np.asarray(sc.xref, dtype=np.float64)
    u = displacement(x)
    u[:, 2] = 6e-6 * np.sin(500.0 * x[:, 0] + 300.0 * x[:, 1])
    conn = mesh_3d(sc, spec)
    xq, e, s = run_reference(x, u, conn, 1, 0, nu, lam, mu)
    np.savez_compressed(os.path.join(HERE, "strain_tet.npz"), xref=x, u=u, conn=conn, material=np.array([nu, lam, mu]),
                        o1_xq=xq, o1_strain=e, o1_stress=s)


if __name__ == "__main__":
    main()
