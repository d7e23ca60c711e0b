"""Synthetic PeriDEM scenes: reference-particle meshes, particle packings,
walls, and the input decks PeriDEM reads.

Two outputs from one scene description:

* ``write_deck(spec, directory)`` writes the YAML deck, CSV meshes and the
  particle-location CSV in the formats the reference reads
  (src/inp/input.cpp:189-1395, src/rw/reader.cpp:16-57 and 101-123), so the
  reference's own ``DEMModel::init`` can set the scene up.
* ``build_scene(spec)`` performs the same set-up directly in numpy and returns
  a :class:`peridem_b200.model.Scene` ready for the device, for workloads too
  large to set up through the reference.  It restates the reference's
  ``DEMModel::init`` steps (src/model/dem/demModel.cpp:109-266): particle
  creation by transform (src/particle/baseParticle.cpp:122-143,
  particleTransform.h:96-100), mesh size and horizon
  (baseParticle.cpp:146-154), material constants (material.h:541-620 RNP,
  919-997 PMB, 1257-1305 PD elastic, 1579-1700 PD state), internal contact
  (baseParticle.cpp:175-179), contact set-up (demModel.cpp:1531-1600) and
  fixity (particleULoading.cpp:90-113).

Synthetic inputs stand in for the reference's gmsh-built example scenes:
meshes are uniform square / cubic grids clipped to the shape, nodal volume
h^d, as the reference's finite-difference CSV meshes allow.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# reference-particle meshes (local coordinates, centred on the origin)
# ---------------------------------------------------------------------------


# Node order of the particle meshes: "grid" (the first index slowest; the
# default) or "morton" (Z-order of the grid indices, so that any run of
# consecutive nodes is a compact patch).  The reference reads the nodes in
# the deck's order, so both sides see the same numbering either way.  The
# bond loop stages each tile's neighbour window as one interval of node
# indices; in Z-order a tile's spatial neighbourhood falls on scattered index
# ranges, so that interval grows: measured on B200, the 2-D compressive
# test's bond loop 35.4 -> 38.1 us and a 256-sphere 3-D column's PD state
# pre-pass and bond loop 505 -> 928 us and 392 -> 777 us with "morton".
MESH_ORDER = "grid"


def _grid(n: int, dim: int) -> np.ndarray:
    r = np.arange(-n, n + 1, dtype=np.int64)
    if dim == 2:
        a, b = np.meshgrid(r, r, indexing="ij")
        return np.stack([a.ravel(), b.ravel()], axis=1)
    a, b, c = np.meshgrid(r, r, r, indexing="ij")
    return np.stack([a.ravel(), b.ravel(), c.ravel()], axis=1)


def _ordered(ij: np.ndarray) -> np.ndarray:
    """The grid points ij (integer indices) in MESH_ORDER: for "morton", by
    the interleaved bits of the shifted indices (x the lowest bit, then y,
    then z)."""
    if MESH_ORDER == "grid" or len(ij) == 0:
        return ij
    if MESH_ORDER != "morton":
        raise ValueError(f"unknown mesh order {MESH_ORDER!r}")
    u = (ij - ij.min(axis=0)).astype(np.uint64)
    dim = ij.shape[1]
    code = np.zeros(len(ij), dtype=np.uint64)
    for b in range(21):
        for d in range(dim):
            code |= ((u[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(dim * b + d)
    return ij[np.argsort(code, kind="stable")]


def disc_mesh(radius: float, h: float) -> Tuple[np.ndarray, np.ndarray]:
    """Square-grid nodes (spacing h) inside a disc; returns (nodes[n,3], vol[n])."""
    n = int(math.floor(radius / h + 1e-9))
    ij = _grid(n, 2)
    keep = (ij[:, 0] ** 2 + ij[:, 1] ** 2) <= (radius / h) ** 2 * (1 + 1e-12)
    ij = _ordered(ij[keep])
    x = np.zeros((len(ij), 3))
    x[:, :2] = ij * h
    return x, np.full(len(ij), h * h)


def hexagon_mesh(radius: float, h: float) -> Tuple[np.ndarray, np.ndarray]:
    """Square-grid nodes inside a regular hexagon of circumradius ``radius``
    with a vertex on the +x axis (the reference's hexagon with axis (1,0,0))."""
    n = int(math.floor(radius / h + 1e-9))
    ij = _grid(n, 2)
    x = ij[:, 0] * h
    y = ij[:, 1] * h
    s3 = math.sqrt(3.0)
    tol = 1e-12 * radius
    keep = (np.abs(y) <= 0.5 * s3 * radius + tol) & (
        s3 * np.abs(x) + np.abs(y) <= s3 * radius + tol)
    ij = _ordered(ij[keep])
    pts = np.zeros((len(ij), 3))
    pts[:, 0] = ij[:, 0] * h
    pts[:, 1] = ij[:, 1] * h
    return pts, np.full(len(pts), h * h)


def sphere_mesh(radius: float, h: float) -> Tuple[np.ndarray, np.ndarray]:
    """Cubic-grid nodes (spacing h) inside a ball."""
    n = int(math.floor(radius / h + 1e-9))
    ijk = _grid(n, 3)
    keep = (ijk ** 2).sum(axis=1) <= (radius / h) ** 2 * (1 + 1e-12)
    return _ordered(ijk[keep]) * h + 0.0, np.full(int(keep.sum()), h ** 3)


def box_mesh(lo: Sequence[float], hi: Sequence[float], h: float, dim: int,
             hole_lo: Optional[Sequence[float]] = None,
             hole_hi: Optional[Sequence[float]] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Grid nodes filling the box [lo, hi] (minus an optional open hole)."""
    axes = []
    for d in range(dim):
        m = int(math.floor((hi[d] - lo[d]) / h + 1e-9))
        axes.append(lo[d] + h * np.arange(m + 1))
    mesh = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([m.ravel() for m in mesh], axis=1)
    if hole_lo is not None:
        inside = np.ones(len(pts), dtype=bool)
        for d in range(dim):
            inside &= (pts[:, d] > hole_lo[d]) & (pts[:, d] < hole_hi[d])
        pts = pts[~inside]
    x = np.zeros((len(pts), 3))
    x[:, :dim] = pts
    return x, np.full(len(pts), h ** dim)


# ---------------------------------------------------------------------------
# scene description
# ---------------------------------------------------------------------------


@dataclass
class MaterialSpec:
    """One zone's material deck (keys of src/inp/input.cpp:1048-1180)."""
    kind: str = "RNPBond"            # RNPBond | PMBBond | PDElasticBond | PDState
    density: float = 1200.0
    E: float = -1.0
    K: float = -1.0
    G: float = -1.0
    nu: float = -1.0
    Gc: float = -1.0
    horizon_mesh_ratio: float = 3.0
    influence_type: int = 1
    check_sc_factor: float = 1.0
    irreversible: bool = True


@dataclass
class ContactSpec:
    """One zone pair's contact deck (src/inp/input.cpp:665-833)."""
    radius_factor: float = 0.95
    kn: float = 0.0                  # Kn before Kn_Factor
    kn_factor: float = 1.0
    epsilon: float = 0.95
    friction_on: bool = False
    friction_coeff: float = 0.5
    damping_on: bool = True
    betan_factor: float = 100.0


@dataclass
class ZoneSpec:
    name: str                        # circle | hexagon | sphere | rectangle | cuboid | ...
    is_wall: bool
    geom_type: str
    geom_params: List[float]
    mesh_nodes: np.ndarray           # local reference mesh [n,3]
    mesh_vol: np.ndarray
    material: MaterialSpec
    all_dofs_constrained: bool = False
    # particles of this zone: (centre[3], radius, orientation); walls use none
    sites: List[Tuple[Tuple[float, float, float], float, float]] = field(default_factory=list)


@dataclass
class BCSpec:
    particles: List[int]
    directions: List[int]            # 1-based, as in the deck
    time_fn: str = "constant"
    time_params: List[float] = field(default_factory=lambda: [0.0])
    spatial_fn: str = "constant"
    spatial_params: List[float] = field(default_factory=list)
    zero: bool = False


@dataclass
class SceneSpec:
    name: str
    dim: int
    dt: float
    nt: int
    zones: List[ZoneSpec]
    contact: Dict[Tuple[int, int], ContactSpec]
    container: Tuple[List[float], List[float]]
    gravity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    search_factor: float = 5.0
    search_interval: int = 40
    test_name: str = ""
    compressive_wall: int = 0
    compressive_dir: int = 2
    test_output_interval: int = 10
    ubc: List[BCSpec] = field(default_factory=list)
    fbc: List[BCSpec] = field(default_factory=list)
    ic_velocity: Optional[Tuple[float, float, float]] = None
    ic_particles: List[int] = field(default_factory=list)
    time_scheme: str = "central_difference"
    seed: int = 0

    @property
    def num_particles(self) -> int:
        return sum(len(z.sites) if not z.is_wall else 1 for z in self.zones)


def elastic_material(kind: str, E: float, Gc: float = 500.0, density: float = 1200.0,
                     nu: float = 0.25) -> MaterialSpec:
    """Material deck with Young's and bulk modulus both given: the reference's
    contact set-up needs K in the deck (demModel.cpp:1559-1565); the bond
    laws derive their constants from E (material.h:584-586), and PD state
    takes (E, K) as its elastic pair (material.h:1592-1616)."""
    K = E / (3.0 * (1.0 - 2.0 * nu))
    return MaterialSpec(kind=kind, density=density, E=E, K=K, Gc=Gc)


# ---------------------------------------------------------------------------
# deck writer (formats read by the reference)
# ---------------------------------------------------------------------------


def _f(v: float) -> str:
    return repr(float(v))


def _flist(v: Sequence[float]) -> str:
    return "[" + ", ".join(_f(x) for x in v) + "]"


def write_deck(spec: SceneSpec, directory: str, threads_note: str = "") -> str:
    """Write deck.yaml + meshes + particle CSV under ``directory``; return the
    YAML path.  Output is switched off (``Perform_Out: false``)."""
    os.makedirs(directory, exist_ok=True)
    L = []
    w = L.append
    w("Model:")
    w(f"  Dimension: {spec.dim}")
    w("  Discretization_Type:")
    w("    Spatial: finite_difference")
    w(f"    Time: {spec.time_scheme}")
    w(f"  Final_Time: {_f(spec.dt * spec.nt)}")
    w(f"  Time_Steps: {spec.nt}")
    w(f"  Seed: {spec.seed}")
    w("Container:")
    w("  Geometry:")
    w("    Type: " + ("rectangle" if spec.dim == 2 else "cuboid"))
    lo, hi = spec.container
    w("    Parameters: " + _flist(list(lo) + list(hi)))
    nz = len(spec.zones)
    w("Zone:")
    w(f"  Zones: {nz}")
    for z, zs in enumerate(spec.zones):
        w(f"  Zone_{z + 1}:")
        w(f"    Is_Wall: {'true' if zs.is_wall else 'false'}")
    w("Particle:")
    if spec.test_name:
        w(f"  Test_Name: {spec.test_name}")
    if spec.test_name == "compressive_test":
        w("  Compressive_Test:")
        w(f"    Particle_Id: {spec.compressive_wall}")
        w(f"    Particle_Force_Direction: {spec.compressive_dir}")
    for z, zs in enumerate(spec.zones):
        w(f"  Zone_{z + 1}:")
        if zs.is_wall:
            w("    Is_Wall: true")
        w(f"    Type: {zs.geom_type}")
        w("    Parameters: " + _flist(zs.geom_params))
        if zs.is_wall:
            w(f"    All_Dofs_Constrained: {'true' if zs.all_dofs_constrained else 'false'}")
            w("    Create_Particle_Using_ParticleZone_GeomObject: true")
        elif zs.all_dofs_constrained:
            w("    All_Dofs_Constrained: true")
    w("Particle_Generation:")
    w("  From_File: particle_locations.csv")
    w("  File_Data_Type: loc_rad_orient")
    w("Mesh:")
    for z, zs in enumerate(spec.zones):
        w(f"  Zone_{z + 1}:")
        w(f"    File: mesh_zone_{z + 1}.csv")
    w("Contact:")
    for i in range(nz):
        for j in range(i, nz):
            c = spec.contact[(i, j)]
            w(f"  Zone_{i + 1}{j + 1}:")
            w(f"    Contact_Radius_Factor: {_f(c.radius_factor)}")
            if not c.damping_on:
                w("    Damping_On: false")
            if not c.friction_on:
                w("    Friction_On: false")
            w(f"    Kn: {_f(c.kn)}")
            w(f"    Epsilon: {_f(c.epsilon)}")
            w(f"    Friction_Coeff: {_f(c.friction_coeff)}")
            w(f"    Kn_Factor: {_f(c.kn_factor)}")
            w(f"    Beta_n_Factor: {_f(c.betan_factor)}")
    w("Neighbor:")
    w("  Update_Criteria: simple_all")
    w(f"  Search_Factor: {_f(spec.search_factor)}")
    w(f"  Search_Interval: {spec.search_interval}")
    w("Material:")
    for z, zs in enumerate(spec.zones):
        m = zs.material
        w(f"  Zone_{z + 1}:")
        w(f"    Type: {m.kind}")
        w(f"    Horizon_Mesh_Ratio: {_f(m.horizon_mesh_ratio)}")
        w(f"    Density: {_f(m.density)}")
        w("    Compute_From_Classical: true")
        for key, val in (("E", m.E), ("K", m.K), ("G", m.G), ("Poisson_Ratio", m.nu), ("Gc", m.Gc)):
            if val > 0:
                w(f"    {key}: {_f(val)}")
        w("    Influence_Function:")
        w(f"      Type: {m.influence_type}")
        if m.kind == "RNPBond":
            w("    Bond_Potential:")
            w(f"      Check_Sc_Factor: {_f(m.check_sc_factor)}")
            w(f"      Irreversible_Bond_Fracture: {'true' if m.irreversible else 'false'}")
    if any(g != 0.0 for g in spec.gravity) or spec.fbc:
        w("Force_BC:")
        if any(g != 0.0 for g in spec.gravity):
            w("  Gravity: " + _flist(spec.gravity))
        if spec.fbc:
            _write_bc_sets(w, spec.fbc)
    if spec.ubc:
        w("Displacement_BC:")
        _write_bc_sets(w, spec.ubc)
    if spec.ic_velocity is not None:
        w("IC:")
        w("  Constant_Velocity:")
        w("    Velocity_Vector: " + _flist(spec.ic_velocity))
        w("    Particle_List: [" + ", ".join(str(p) for p in spec.ic_particles) + "]")
    w("Output:")
    w("  Path: ./")
    w("  Tags:")
    w("    - Displacement")
    w(f"  Output_Interval: {max(1, spec.nt)}")
    w("  Perform_FE_Out: false")
    w("  Perform_Out: false")
    w(f"  Test_Output_Interval: {spec.test_output_interval}")
    w("  Debug: 0")
    w("  Tag_PP: 0")
    path = os.path.join(directory, "deck.yaml")
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")

    # meshes
    for z, zs in enumerate(spec.zones):
        with open(os.path.join(directory, f"mesh_zone_{z + 1}.csv"), "w") as fh:
            if spec.dim == 2:
                fh.write("id,x,y,volume\n")
                for i, (p, v) in enumerate(zip(zs.mesh_nodes, zs.mesh_vol)):
                    fh.write(f"{i},{_f(p[0])},{_f(p[1])},{_f(v)}\n")
            else:
                fh.write("id,x,y,z,volume\n")
                for i, (p, v) in enumerate(zip(zs.mesh_nodes, zs.mesh_vol)):
                    fh.write(f"{i},{_f(p[0])},{_f(p[1])},{_f(p[2])},{_f(v)}\n")
    with open(os.path.join(directory, "particle_locations.csv"), "w") as fh:
        fh.write("i, x, y, z, r, o\n")
        for z, zs in enumerate(spec.zones):
            if zs.is_wall:
                continue
            for (c, r, o) in zs.sites:
                fh.write(f"{z}, {_f(c[0])}, {_f(c[1])}, {_f(c[2])}, {_f(r)}, {_f(o)}\n")
    return path


def _write_bc_sets(w, sets: List[BCSpec]) -> None:
    w(f"  Sets: {len(sets)}")
    for s, bc in enumerate(sets):
        w(f"  Set_{s + 1}:")
        w("    Particle_List: [" + ", ".join(str(p) for p in bc.particles) + "]")
        w("    Direction: [" + ",".join(str(d) for d in bc.directions) + "]")
        if bc.zero:
            w("    Zero_Displacement: true")
        else:
            w("    Time_Function:")
            w(f"      Type: {bc.time_fn}")
            w("      Parameters:")
            for p in bc.time_params:
                w(f"        - {_f(p)}")
            w("    Spatial_Function:")
            w(f"      Type: {bc.spatial_fn}")
            if bc.spatial_params:
                w("      Parameters:")
                for p in bc.spatial_params:
                    w(f"        - {_f(p)}")


# ---------------------------------------------------------------------------
# named workloads
# ---------------------------------------------------------------------------


def stable_dt(E: float, density: float, h: float, courant: float = 0.2) -> float:
    """Explicit step for a bond-based PD body of Young's modulus E, mesh size
    h, horizon 3h: dt = courant * h / sqrt(E / rho).  The linearised bond
    stiffness of RNP/PMB on a square grid gives omega_max*dt ~ 2.5 * h/c-units,
    so courant = 0.2 keeps omega_max*dt near 0.5 (the limit is 2)."""
    return courant * h / math.sqrt(E / density)


def stable_kn(density: float, node_volume: float, dt: float, omega_dt: float = 0.3) -> float:
    """Contact stiffness Kn whose node-pair penalty spring has omega*dt =
    omega_dt.  A pair inside the contact radius feels the force density
    Kn*(R - Rc)*vol_j (demModel.cpp:895-899), so omega^2 = Kn*vol_j/rho; the
    bulk-modulus choice 18K/(pi eps^5) of the reference's examples is
    thousands of times stiffer than an explicit step of 5e-8..1e-7 s allows
    for E = 2 GPa at these mesh sizes."""
    return density * (omega_dt / dt) ** 2 / node_volume


def _all_pairs(nz: int, c: ContactSpec) -> Dict[Tuple[int, int], ContactSpec]:
    return {(i, j): c for i in range(nz) for j in range(i, nz)}


def two_particle(h_div: int = 10, radius: float = 1e-3, material: str = "RNPBond",
                 nt: int = 20000, dt: Optional[float] = None, v0: float = -0.1,
                 gap: Optional[float] = None) -> SceneSpec:
    """Two discs of radius R, square-grid nodes h = R/h_div, horizon 3h; the
    top disc starts at v0 under gravity; the bottom disc's force is off
    (test name two_particle, demModel.cpp:218-220)."""
    h = radius / h_div
    nodes, vol = disc_mesh(radius, h)
    mat = elastic_material(material, 2.0e9)
    dt = stable_dt(2.0e9, 1200.0, h) if dt is None else dt
    kn = stable_kn(1200.0, h * h, dt)
    gap = 0.5 * h if gap is None else gap
    sites = [((radius, radius, 0.0), radius, 0.0),
             ((radius, 3.0 * radius + 0.95 * h + gap, 0.0), radius, 0.0)]
    z = ZoneSpec("disc", False, "circle", [radius, 0.0, 0.0, 0.0], nodes, vol, mat, sites=sites)
    c = ContactSpec(radius_factor=0.95, kn=kn, kn_factor=1.0, epsilon=0.7,
                    friction_on=True, friction_coeff=0.5, damping_on=True, betan_factor=1.0)
    return SceneSpec(name=f"two_particle_h{h_div}", dim=2, dt=dt, nt=nt, zones=[z],
                     contact=_all_pairs(1, c),
                     container=([0.0, 0.0, 0.0], [2 * radius, 4 * radius + 2 * h, 0.0]),
                     gravity=(0.0, -10.0, 0.0), search_factor=5.0, search_interval=40,
                     test_name="two_particle", test_output_interval=10,
                     ic_velocity=(0.0, v0, 0.0), ic_particles=[1])


def deposit_2d(offsets: Sequence[np.ndarray], x_lim: Tuple[float, float], floor: np.ndarray, gap: float,
               rng: np.random.Generator, trials: int = 8) -> np.ndarray:
    """Seeded ballistic deposition of rigid node sets: body k (node offsets
    [n_k, 2] from its centre, already rotated and scaled) falls straight down
    at a random x (of `trials` draws, the one where it comes to rest lowest)
    until one of its nodes comes within `gap` of a node below it: of the
    floor nodes `floor` [m, 2] or of a body placed before it.  Every node
    keeps `gap` from the side walls' inner node columns x_lim = (x_left,
    x_right).  No two nodes of different bodies start closer than `gap`,
    and every body rests on the floor or on a body below it, at a clearance
    of at most gap (1 + 1/64).

    The heights come from an upper envelope of the placed nodes over bins
    gap/64 wide (per bin its highest node), tested at the widened clearance
    gap (1 + 1/64): a node lower in the same bin, at most one bin width
    aside, cannot stop the body higher than the bin's top node does, so
    the clearance is never below `gap`.  Returns the centres [n, 2]."""
    w = gap / 64.0
    ge = gap + w
    x0 = x_lim[0]
    nb = int(math.ceil((x_lim[1] - x0) / w)) + 1
    top_y = np.full(nb, -np.inf)
    top_x = np.zeros(nb)

    def add(pts):
        b = np.clip(((pts[:, 0] - x0) / w).astype(np.int64), 0, nb - 1)
        order = np.lexsort((pts[:, 1], b))
        b, y, x = b[order], pts[order, 1], pts[order, 0]
        last = np.r_[b[1:] != b[:-1], True]          # the highest node of each bin
        b, y, x = b[last], y[last], x[last]
        up = y > top_y[b]
        top_y[b[up]] = y[up]
        top_x[b[up]] = x[up]

    add(np.asarray(floor, dtype=np.float64))
    m = int(math.ceil(ge / w)) + 1
    span = np.arange(-m, m + 1)
    cen = np.zeros((len(offsets), 2))
    for k, off in enumerate(offsets):
        off = np.asarray(off, dtype=np.float64)
        lo = x_lim[0] + gap - float(off[:, 0].min())
        hi = x_lim[1] - gap - float(off[:, 0].max())
        if hi < lo:
            raise ValueError("box too narrow for one particle")
        xs = rng.uniform(lo, hi, size=trials)
        xa = xs[:, None] + off[None, :, 0]                      # [trials, nodes]
        bins = np.clip(((xa - x0) / w).astype(np.int64)[..., None] + span, 0, nb - 1)
        dx = top_x[bins] - xa[..., None]
        ty = top_y[bins]
        ok = (np.abs(dx) < ge) & np.isfinite(ty)
        lift = np.where(ok, ty - off[None, :, 1, None] + np.sqrt(np.maximum(ge * ge - dx * dx, 0.0)), -np.inf)
        ys = lift.reshape(trials, -1).max(axis=1)
        t = int(np.argmin(ys))                                  # the lowest rest (first on ties)
        best_x, best_y = float(xs[t]), float(ys[t])
        cen[k] = (best_x, best_y)
        add(cen[k] + off)
    return cen


def compressive_2d(n_particles: int = 502, r_range: Tuple[float, float] = (1e-3, 1.5e-3),
                   h_div: int = 15, width: float = 40e-3, seed: int = 0,
                   material: str = "RNPBond", wall_speed: float = -0.1,
                   dt: Optional[float] = None, nt: int = 50000, gravity: float = -10.0,
                   search_factor: float = 5.0, search_interval: int = 40,
                   friction: bool = True, gap: Optional[float] = None,
                   jitter: float = 0.5, packing: str = "lattice",
                   contact_omega_dt: float = 0.3) -> SceneSpec:
    """2-D compression: discs and hexagons (50/50) inside a fixed frame,
    pressed by a top wall moving at ``wall_speed``.  One reference mesh per
    shape at h = R_ref/h_div, scaled per particle, so every particle has the
    same node count.

    packing "lattice": a jittered triangular lattice; ``gap`` is the
    clearance between lattice neighbours of maximal radius and between the
    packing and the walls (default 1.05 h_min, just beyond the contact
    radius 0.95 h_min, so nothing starts in contact).

    packing "deposit": ballistic deposition (``deposit_2d``) of the
    particles' own nodes at clearance ``gap`` (default 0.96 h_min, just
    beyond the contact radius 0.95 h_min): each particle falls until one of
    its nodes comes within ``gap`` of a node of the floor or of a particle
    below it, so every particle rests on a support, the wall's load reaches
    the floor through chains of supports, and the packing closes its
    remaining clearances (each support's at most gap (1 + 1/64), under
    3 % of h beyond the contact radius) early in the run under gravity.  No node pair of
    two bodies starts inside the contact radius (contacts open as the
    packing settles and the wall presses instead of as preloaded penalty
    springs).  The top wall starts ``gap`` above the highest node.

    With the lattice the top wall starts ``gap`` above the highest particle.

    The contact stiffness Kn is ``scene.stable_kn`` at omega dt =
    ``contact_omega_dt`` for a node pair of the smallest mesh size."""
    rng = np.random.default_rng(seed)
    r_ref = r_range[0]
    h_ref = r_ref / h_div
    disc_n, disc_v = disc_mesh(r_ref, h_ref)
    hex_n, hex_v = hexagon_mesh(r_ref, h_ref)
    radii = rng.uniform(r_range[0], r_range[1], size=n_particles)
    orients = rng.uniform(0.0, 2.0 * math.pi, size=n_particles)
    shapes = np.arange(n_particles) % 2          # 0 disc, 1 hexagon
    rng.shuffle(shapes)
    h_min = r_range[0] / h_div
    if packing not in ("lattice", "deposit"):
        raise ValueError(f"unknown packing {packing!r}")
    gap = (1.05 if packing == "lattice" else 0.96) * h_min if gap is None else gap
    dt = stable_dt(2.0e9, 1200.0, h_min) if dt is None else dt
    spacing = 2.0 * r_range[1] + gap
    # triangular-lattice slots; odd rows shift by half a spacing and drop the
    # slots that would leave the box, so no two lattice neighbours are closer
    # than `spacing`
    dy = spacing * math.sqrt(3.0) / 2.0
    t_wall = 3.0 * h_min                          # wall thickness
    slots = []
    row = 0
    while len(slots) < n_particles:
        x = gap + 0.5 * spacing + (0.5 * spacing if row % 2 else 0.0)
        cy = gap + r_range[1] + row * dy
        while x + 0.5 * spacing <= width + 1e-12 and len(slots) < n_particles:
            slots.append((x, cy))
            x += spacing
        row += 1
        if row > 100000:
            raise ValueError("box too narrow for one particle")
    sites_by_shape = {0: [], 1: []}
    top = 0.0
    if packing == "deposit":
        # the frame's floor nodes and inner wall columns, as built below
        # (they do not depend on the frame's height)
        probe, _ = box_mesh([-t_wall, -t_wall], [width + t_wall, 4.0 * t_wall + 2.0 * h_min], h_min, 2,
                            hole_lo=[0.5 * h_min, 0.5 * h_min], hole_hi=[width - 0.5 * h_min, 1.0])
        side = probe[:, 1] > 0.5 * h_min
        x_lim = (float(probe[side & (probe[:, 0] < 0.5 * width), 0].max()),
                 float(probe[side & (probe[:, 0] > 0.5 * width), 0].min()))
        floor = probe[~side][:, :2]
        meshes = {0: _csv_array(disc_n), 1: _csv_array(hex_n)}
        offsets = []
        for p in range(n_particles):
            scale = csv_float(_f(radii[p])) / r_ref
            rot = _rotate_z(meshes[int(shapes[p])], csv_float(_f(orients[p])))
            offsets.append(scale * rot[:, :2])
        cen = deposit_2d(offsets, x_lim, floor, gap, rng)
    for p in range(n_particles):
        if packing == "deposit":
            cx, cy = float(cen[p, 0]), float(cen[p, 1])
        else:
            cx, cy = slots[p]
            room = max(0.0, spacing - 2.0 * radii[p] - gap)
            jx, jy = rng.uniform(-0.5, 0.5, size=2) * room * jitter
            jy = max(jy, -(cy - radii[p] - gap))
            cx, cy = cx + jx, cy + jy
        sites_by_shape[int(shapes[p])].append(((cx, cy, 0.0), float(radii[p]), float(orients[p])))
        if packing == "deposit":
            top = max(top, cy + float(offsets[p][:, 1].max()))
        else:
            top = max(top, cy + radii[p])
    height = top + gap
    mat = elastic_material(material, 2.0e9)
    zones = [
        ZoneSpec("disc", False, "circle", [r_ref, 0.0, 0.0, 0.0], disc_n, disc_v, mat,
                 sites=sites_by_shape[0]),
        ZoneSpec("hexagon", False, "hexagon", [r_ref, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0], hex_n, hex_v,
                 mat, sites=sites_by_shape[1]),
    ]
    # fixed frame (left, right, bottom) and moving top bar, walls meshed at h_min
    lo = [-t_wall, -t_wall]
    hi = [width + t_wall, height + 2.0 * t_wall]
    frame_n, frame_v = box_mesh([lo[0], lo[1]], [hi[0], hi[1]], h_min, 2,
                                hole_lo=[0.5 * h_min, 0.5 * h_min],
                                hole_hi=[width - 0.5 * h_min, hi[1] + 1.0])
    bar_lo = [h_min, height]
    bar_hi = [width - h_min, height + t_wall]
    bar_n, bar_v = box_mesh(bar_lo, bar_hi, h_min, 2)
    wall_mat = elastic_material(material, 2.0e9)
    zones.append(ZoneSpec("frame", True, "rectangle", [lo[0], lo[1], 0.0, hi[0], hi[1], 0.0],
                          frame_n, frame_v, wall_mat, all_dofs_constrained=True))
    zones.append(ZoneSpec("top_wall", True, "rectangle",
                          [bar_lo[0], bar_lo[1], 0.0, bar_hi[0], bar_hi[1], 0.0],
                          bar_n, bar_v, wall_mat, all_dofs_constrained=True))
    kn = stable_kn(1200.0, h_min * h_min, dt, contact_omega_dt)
    c = ContactSpec(radius_factor=0.95, kn=kn, kn_factor=1.0, epsilon=0.7,
                    friction_on=friction, friction_coeff=0.5, damping_on=True, betan_factor=1.0)
    wall_fixed, wall_moving = n_particles, n_particles + 1
    ubc = [BCSpec(particles=[wall_fixed], directions=[1, 2], zero=True),
           BCSpec(particles=[wall_moving], directions=[2], time_fn="linear",
                  time_params=[wall_speed])]
    return SceneSpec(name=f"compressive_{n_particles}", dim=2, dt=dt, nt=nt, zones=zones,
                     contact=_all_pairs(4, c),
                     container=([lo[0], lo[1], 0.0], [hi[0], hi[1], 0.0]),
                     gravity=(0.0, gravity, 0.0), search_factor=search_factor,
                     search_interval=search_interval, test_name="compressive_test",
                     compressive_wall=wall_moving, compressive_dir=2, test_output_interval=10,
                     ubc=ubc, seed=seed)


def column_3d(n_spheres: int = 4096, median_r: float = 1e-3, sigma: float = 0.2,
              h_div: int = 10, box: Tuple[float, float, float] = (20e-3, 20e-3, 60e-3),
              seed: int = 0, material: str = "PDState", piston_speed: float = -0.05,
              dt: Optional[float] = None, nt: int = 5000, footprint: Optional[Tuple[int, int]] = None,
              wall_h: Optional[float] = None, wall_layers: float = 3.0) -> SceneSpec:
    """3-D granular column: spheres with lognormal radii on a jittered cubic
    lattice inside a fixed box, a piston on top moving at ``piston_speed``.
    The lattice is as wide as ``box`` allows (or ``footprint`` = (nx, ny)
    sites per layer) and as tall as the spheres need; the box and piston are
    meshed at ``wall_h`` (default: the smallest sphere's h) with walls
    ``wall_layers`` mesh sizes thick."""
    rng = np.random.default_rng(seed)
    r_ref = median_r
    h_ref = r_ref / h_div
    s_n, s_v = sphere_mesh(r_ref, h_ref)
    radii = np.clip(median_r * np.exp(sigma * rng.standard_normal(n_spheres)), 0.6 * median_r,
                    1.6 * median_r)
    h_min = float(radii.min()) / h_div
    dt = stable_dt(5.0e9, 1200.0, h_min) if dt is None else dt
    spacing = 2.0 * float(radii.max()) + 2.0 * h_min
    nx = max(1, int(math.floor(box[0] / spacing)))
    ny = max(1, int(math.floor(box[1] / spacing)))
    if footprint is not None:
        nx, ny = footprint
    sites = []
    for p in range(n_spheres):
        layer, rem = divmod(p, nx * ny)
        iy, ix = divmod(rem, nx)
        c = (0.5 * spacing + ix * spacing, 0.5 * spacing + iy * spacing,
             0.5 * spacing + layer * spacing)
        j = rng.uniform(-0.5, 0.5, size=3) * (spacing - 2 * radii[p] - 1.5 * h_min) * 0.5
        sites.append(((c[0] + j[0], c[1] + j[1], c[2] + j[2]), float(radii[p]), 0.0))
    height = (int(math.ceil(n_spheres / (nx * ny)))) * spacing
    mat = elastic_material(material, 5.0e9)
    hw = h_min if wall_h is None else wall_h
    t = wall_layers * hw
    W = (nx * spacing, ny * spacing)
    lo = [-t - h_min, -t - h_min, -t - h_min]
    hi = [W[0] + t + h_min, W[1] + t + h_min, height + 2 * t]
    box_n, box_v = box_mesh(lo, hi, hw, 3, hole_lo=[-0.5 * h_min, -0.5 * h_min, -0.5 * h_min],
                            hole_hi=[W[0] + 0.5 * h_min, W[1] + 0.5 * h_min, hi[2] + 1.0])
    pis_n, pis_v = box_mesh([0.5 * h_min, 0.5 * h_min, height], [W[0] - 0.5 * h_min,
                                                                 W[1] - 0.5 * h_min, height + t],
                            hw, 3)
    zones = [ZoneSpec("sphere", False, "sphere", [r_ref, 0.0, 0.0, 0.0], s_n, s_v, mat, sites=sites),
             ZoneSpec("box", True, "cuboid", lo + hi, box_n, box_v, mat, all_dofs_constrained=True),
             ZoneSpec("piston", True, "cuboid",
                      [0.5 * h_min, 0.5 * h_min, height, W[0] - 0.5 * h_min, W[1] - 0.5 * h_min,
                       height + t], pis_n, pis_v, mat, all_dofs_constrained=True)]
    kn = stable_kn(1200.0, h_min ** 3, dt)
    c = ContactSpec(radius_factor=0.95, kn=kn, kn_factor=1.0, epsilon=0.7, friction_on=True,
                    friction_coeff=0.5, damping_on=True, betan_factor=1.0)
    ubc = [BCSpec(particles=[n_spheres], directions=[1, 2, 3], zero=True),
           BCSpec(particles=[n_spheres + 1], directions=[3], time_fn="linear",
                  time_params=[piston_speed])]
    return SceneSpec(name=f"column_{n_spheres}", dim=3, dt=dt, nt=nt, zones=zones,
                     contact=_all_pairs(3, c), container=(lo, hi), gravity=(0.0, 0.0, -10.0),
                     search_factor=5.0, search_interval=40, test_name="compressive_test",
                     compressive_wall=n_spheres + 1, compressive_dir=3, test_output_interval=10,
                     ubc=ubc, seed=seed)


# ---------------------------------------------------------------------------
# direct set-up (DEMModel::init restated)
# ---------------------------------------------------------------------------


def csv_float(text: str) -> float:
    """The reference's CSV number parser (external/csv/csv.h:964-1024,
    fast-cpp-csv-parser): digit accumulation and repeated multiplication, not
    correctly rounded.  Meshes and particle locations pass through it, so the
    direct set-up parses the same strings the same way."""
    col = text.strip()
    neg = False
    p = 0
    if col[p:p + 1] == "-":
        neg = True
        p += 1
    elif col[p:p + 1] == "+":
        p += 1
    x = 0.0
    while p < len(col) and col[p].isdigit():
        x = x * 10
        x = x + float(ord(col[p]) - 48)
        p += 1
    if p < len(col) and col[p] in ".,":
        p += 1
        pos = 1.0
        while p < len(col) and col[p].isdigit():
            pos = pos / 10
            y = ord(col[p]) - 48
            p += 1
            x = x + y * pos
    if p < len(col) and col[p] in "eE":
        p += 1
        e = int(col[p:])
        if e != 0:
            if e < 0:
                base = 0.1
                e = -e
            else:
                base = 10.0
            while e != 1:
                if (e & 1) == 0:
                    base = base * base
                    e >>= 1
                else:
                    x = x * base
                    e -= 1
            x = x * base
    return -x if neg else x


def _csv_array(a: np.ndarray) -> np.ndarray:
    """csv_float(_f(v)) elementwise, evaluated once per distinct value (mesh
    coordinates repeat along every lattice line)."""
    a = np.asarray(a, dtype=np.float64)
    uniq, inv = np.unique(a, return_inverse=True)
    return np.array([csv_float(_f(v)) for v in uniq])[inv].reshape(a.shape)


def _csvv(v: float) -> float:
    return csv_float(_f(v))


def _is_less(a: float, b: float) -> bool:
    return (b - a) > (max(abs(a), abs(b)) * 1.0e-5)


def _is_greater(a: float, b: float) -> bool:
    return (a - b) > (max(abs(a), abs(b)) * 1.0e-5)


def _record_chain(values: np.ndarray, guess: float):
    """Scan non-negative ``values`` in order, replacing the running guess by
    every value that is util::isLess than it; returns (index of the last
    replacement or -1, final guess).  A replacement lies below the guess by
    more than the relative tolerance, hence below every value skipped since
    the previous one: it is a strict new running minimum.  So only the
    positions where the running minimum falls are tested, in order."""
    values = np.asarray(values, dtype=np.float64)
    if len(values) == 0:
        return -1, guess
    prev = np.concatenate(([np.inf], np.minimum.accumulate(values)[:-1]))
    idx = -1
    for k in np.nonzero(values < prev)[0]:
        v = float(values[k])
        if (guess - v) > max(abs(v), abs(guess)) * 1.0e-5:
            guess, idx = v, int(k)
    return idx, guess


def mesh_size(x: np.ndarray) -> float:
    """util::computeMeshSize (src/util/geom.cpp:578-603): scan i, j in
    order, keep the first distance that is isLess than the running guess.

    The guess starts at |x0 - x1| and only ever moves to a smaller distance,
    so only pairs closer than |x0 - x1| can change it: those are found with a
    k-d tree, their distances recomputed with the scan's own arithmetic, and
    the scan's sequence of replacements replayed over them in (i, j) order.
    Same result as the full scan (mesh_size_scan), in O(n log n)."""
    n = len(x)
    if n < 2:
        return 0.0
    try:
        from scipy.spatial import cKDTree
    except ImportError:  # pragma: no cover
        return mesh_size_scan(x)
    x = np.asarray(x, dtype=np.float64)
    guess = float(np.sqrt(((x[0] - x[1]) ** 2).sum(axis=-1)))
    # row 0 in full: afterwards the guess is within the tolerance of node 0's
    # nearest-neighbour distance, which bounds every later replacement
    d = x[0] - x
    row0 = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    row0[0] = np.inf
    _, guess = _record_chain(row0, guess)
    pairs = cKDTree(x).query_pairs(guess * (1.0 + 1e-9) + 1e-300, output_type="ndarray")
    if len(pairs) == 0:
        return guess
    i = np.concatenate([pairs[:, 0], pairs[:, 1]])
    j = np.concatenate([pairs[:, 1], pairs[:, 0]])
    keep = i > 0
    i, j = i[keep], j[keep]
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    d = x[i] - x[j]
    dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    _, guess = _record_chain(dist, guess)
    return guess


def mesh_size_scan(x: np.ndarray) -> float:
    """The full O(n^2) scan of util::computeMeshSize."""
    n = len(x)
    if n < 2:
        return 0.0
    guess = float(np.sqrt(((x[0] - x[1]) ** 2).sum(axis=-1)))
    for i in range(n):
        d = x[i] - x
        dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        dist[i] = np.inf
        start = 0
        while True:
            thr = dist[start:]
            cand = (guess - thr) > (np.maximum(np.abs(thr), abs(guess)) * 1.0e-5)
            if not cand.any():
                break
            k = int(np.argmax(cand)) + start
            guess = float(dist[k])
            start = k + 1
    return guess


def _moment(inf_type: int, params: np.ndarray, i: int) -> float:
    """BaseInfluenceFn::getMoment (influenceFn.cpp:25-27, 59-61, 90-121)."""
    if inf_type == 0:
        return params[0] / float(i + 1)
    if inf_type == 1:
        return (params[0] / float(i + 1)) + (params[1] / float(i + 2))
    a, b = params
    sq1, sq2 = math.sqrt(b), math.sqrt(math.pi)
    if i == 0:
        return 0.5 * a * sq1 * sq2 * math.erf(1. / sq1)
    if i == 1:
        return 0.5 * a * b * (1. - math.exp(-1. / b))
    if i == 2:
        return 0.5 * a * b * sq1 * (0.5 * sq2 * math.erf(1. / sq1) - (1. / sq1) * math.exp(-1. / b))
    return 0.5 * a * b * b * (1. - (1. + 1. / b) * math.exp(-1. / b))


def influence_params(m: MaterialSpec, dim: int) -> Tuple[int, np.ndarray]:
    """Default influence-function constants (influenceFn.cpp:14-84)."""
    t = m.influence_type
    if t == 0:
        return 0, np.array([float(dim + 1), 0.0])
    if t == 1:
        a0 = {1: 6., 2: 12., 3: 20.}[dim]
        return 1, np.array([a0, -a0])
    b = 0.2
    if dim == 1:
        a = 2. / (b * (1. - math.exp(-1. / b)))
    elif dim == 2:
        a = (4.0 / b) * 1.0 / (math.sqrt(math.pi * b) * math.erf(1.0 / math.sqrt(b))
                               - 2.0 * math.exp(-1.0 / b))
    else:
        a = (2.0 / b) * 1.0 / (b - (b + 1.) * math.exp(-1.0 / b))
    return 2, np.array([a, b])


def material_constants(m: MaterialSpec, dim: int, horizon: float, inf_type: int,
                       inf: np.ndarray) -> Tuple[int, np.ndarray, float]:
    """Bond-law constants and the bulk modulus that BaseParticle uses for the
    internal contact stiffness (baseParticle.cpp:156-179): RnpMaterial
    (material.h:541-620, 461-489), PmbMaterial (:919-997, 846-871),
    PdElastic (:1257-1305, 1189-1210), PdState (:1579-1700, 1504-1530)."""
    E, K, G, nu, Gc = m.E, m.K, m.G, m.nu, m.Gc
    mat = np.zeros(6)
    toK = lambda E_, nu_: E_ / (3. * (1. - 2. * nu_))
    toLambdaE = lambda E_, nu_: E_ * nu_ / ((1. + nu_) * (1. - 2. * nu_))
    toGE = lambda E_, nu_: E_ / (2. * (1. + nu_))
    toELambda = lambda l_, nu_: l_ * (1. + nu_) * (1. - 2. * nu_) / nu_
    code = MATERIAL_CODE[m.kind]
    if code in (0, 1, 2):
        nu = 0.25
        if E > 0.:
            K = toK(E, nu)
        if K > 0. and E < 0.:
            E = K * (3. * (1. - 2. * nu))
        lam = toLambdaE(E, nu)
        M = _moment(inf_type, inf, dim)
        if code == 0:
            if dim == 2:
                C = math.pi * Gc / (4. * M)
                beta = 4. * lam / (C * M)
                inv = math.pow(horizon, 3) * math.pi
            else:
                C = 2. * Gc / (3. * M)
                beta = 5. * lam / (C * M)
                inv = math.pow(horizon, 4) * 4. * math.pi / 3.
            mat[:] = [C, beta, math.sqrt(0.5 / beta), inv, m.check_sc_factor,
                      1.0 if m.irreversible else 0.0]
            lam2 = C * M * beta / 4. if dim == 2 else C * M * beta / 5.
            Kp = toK(toELambda(lam2, 0.25), 0.25)
        elif code == 1:
            if dim == 2:
                c = 24.0 * E / (math.pi * math.pow(horizon, 3.0) * (1. - nu))
            else:
                c = 24.0 * lam / (math.pi * math.pow(horizon, 3.0))
            s0 = math.sqrt(5.0 * math.pi * Gc / (9.0 * E * horizon))
            mat[:2] = [c, s0]
            lam2 = c * (math.pi * math.pow(horizon, 3.0)) / 24.0
            Kp = toK(toELambda(lam2, 0.25), 0.25)
        else:
            c = 24.0 * lam / (math.pi * math.pow(horizon, 3.0))
            mat[0] = c
            lam2 = c * (math.pi * math.pow(horizon, 3.0)) / 24.0
            Kp = toK(toELambda(lam2, 0.25), 0.25)
        return code, mat, Kp
    # PD state: exactly two of E, K, G, nu
    fE, fK, fG, fnu = E > 0, K > 0, G > 0, nu > 0
    if not fnu:
        if fE and fG:
            nu = (0.5 * E / G) - 1.
        if fE and fK:
            nu = (3. * K - E) / (6. * K)
        if fG and fK:
            nu = (3. * K - 2. * G) / (2. * (3. * K + G))
    if not fE:
        if fK:
            E = K * (3. * (1. - 2. * nu))
        if fG:
            E = 2. * G * (1. + nu)
    if not fK:
        K = toK(E, nu)
    if not fG:
        G = toGE(E, nu)
    d = (3. * G + math.pow(3. / 4., 4) * (K - 5. * G / 3.)) * horizon
    s0 = math.sqrt(Gc / d)
    mat[:3] = [K, G, s0]
    return 3, mat, K


MATERIAL_CODE = {"RNPBond": 0, "PMBBond": 1, "PDElasticBond": 2, "PDState": 3}
TIME_CODE = {"constant": 0, "linear": 1, "quadratic": 2, "sin": 3, "rotation": 4,
             "linear_step": 5, "linear_slow_fast": 6}
SPATIAL_CODE = {"constant": 0, "hat_x": 1, "hat_y": 2, "sin_x": 3, "sin_y": 4, "linear_x": 5,
                "linear_y": 6}


def _rotate_z(v: np.ndarray, theta: float) -> np.ndarray:
    """util::rotate about (0,0,1) (transformation.cpp:67-79), in its
    evaluation order: (1-ct)(p.n) n + ct p + st (n x p)."""
    ct, st = math.cos(theta), math.sin(theta)
    pdn = v[:, 0] * 0.0 + v[:, 1] * 0.0 + v[:, 2] * 1.0
    a = (1. - ct) * pdn
    nx = 0.0 * v[:, 2] - 1.0 * v[:, 1]
    ny = 1.0 * v[:, 0] - 0.0 * v[:, 2]
    nz = 0.0 * v[:, 1] - 0.0 * v[:, 0]
    out = np.empty_like(v)
    out[:, 0] = (a * 0.0 + ct * v[:, 0]) + st * nx
    out[:, 1] = (a * 0.0 + ct * v[:, 1]) + st * ny
    out[:, 2] = (a * 1.0 + ct * v[:, 2]) + st * nz
    return out


def _bounding_radius(geom_type: str, params: List[float]) -> float:
    """GeomObject::boundingRadius: circle/sphere/hexagon radius, half the
    rectangle diagonal, the full cuboid diagonal (geomObjects.h:855, 1693)."""
    if geom_type in ("circle", "sphere", "hexagon"):
        return params[0]
    L = [params[3 + q] - params[q] for q in range(3)]
    if geom_type == "cuboid":
        return math.sqrt(math.pow(L[0], 2) + math.pow(L[1], 2) + math.pow(L[2], 2))
    return 0.5 * math.sqrt(math.pow(L[0], 2) + math.pow(L[1], 2))


def build_scene(spec: SceneSpec):
    """The ModelData the reference's DEMModel::init would produce for
    ``spec`` (same transforms, mesh sizes, constants and selections).  The
    peridynamic neighbour lists and m_x are left to the device
    (GpuDEMModel(build_neighbors=True, compute_mx=True)) or the oracle."""
    from .model import Scene, BCSet
    dim = spec.dim
    xs, vols, pts = [], [], []
    parts = []
    zone_K = []
    inf_type, inf = influence_params(spec.zones[0].material, dim)
    # the first particle's material fixes the influence function
    # (material.h:273-288); particles are created zone by zone
    for z, zs in enumerate(spec.zones):
        zone_K.append(zs.material.K)
        local = _csv_array(zs.mesh_nodes) if len(zs.mesh_nodes) else zs.mesh_nodes
        local[:, 2] = local[:, 2] if dim == 3 else 0.0
        lvol = _csv_array(zs.mesh_vol)
        # RefParticle centre node: closest to the geometry centre
        # (refParticle.cpp:27-36)
        gc = np.zeros(3) if not zs.is_wall else (
            0.5 * (np.array(zs.geom_params[:3]) + np.array(zs.geom_params[3:6])))
        dd = np.sqrt(((gc - local) ** 2).sum(axis=1))
        center, best = _record_chain(dd, _bounding_radius(zs.geom_type, zs.geom_params))
        center = max(center, 0)
        if zs.is_wall:
            sites = [(None, None, None)]
        else:
            sites = zs.sites
        rep_r = zs.geom_params[0]
        for (c, r, o) in sites:
            scale, oo = 1.0, 0.0
            if zs.is_wall:
                xg = local.copy()
                vg = lvol.copy()
                bound = _bounding_radius(zs.geom_type, zs.geom_params)
            else:
                cc = np.array([csv_float(_f(c[0])), csv_float(_f(c[1])), csv_float(_f(c[2]))])
                rr, oo = csv_float(_f(r)), csv_float(_f(o))
                scale = rr / rep_r
                rot = _rotate_z(local, oo)
                xg = cc + scale * rot
                vg = lvol * math.pow(scale, dim)
                bound = rr
            pid = len(parts)
            start = sum(len(a) for a in xs)
            xs.append(xg)
            vols.append(vg)
            pts.append(np.full(len(xg), pid, dtype=np.uint64))
            h = mesh_size(xg)
            horizon = zs.material.horizon_mesh_ratio * h
            code, mat, Kp = material_constants(zs.material, dim, horizon, inf_type, inf)
            parts.append(dict(start=start, end=start + len(xg), center=start + center,
                              type=1 if zs.is_wall else 0, zone=z,
                              all_fixed=1 if zs.all_dofs_constrained else 0,
                              compute_force=0 if zs.all_dofs_constrained else 1,
                              material=code, horizon=horizon, h=h,
                              density=zs.material.density, rc=0.95 * h, scale=scale, orient=oo,
                              kn=(18. / (math.pi * math.pow(horizon, 5))) * Kp,
                              bound_r=bound, mat=mat))
    if spec.test_name == "two_particle":
        parts[0]["compute_force"] = 0  # demModel.cpp:218-220
    xref = np.concatenate(xs)
    vol = np.concatenate(vols)
    ptid = np.concatenate(pts)
    N, Np = len(xref), len(parts)
    P = {k: np.array([p[k] for p in parts]) for k in parts[0] if k != "mat"}
    pmat = np.stack([p["mat"] for p in parts])
    # contact (DEMModel::setupContact, demModel.cpp:1531-1600)
    nz = len(spec.zones)
    hmin = hmax = None
    for p in parts:
        if hmin is None:
            hmin = hmax = p["h"]
        if _is_greater(hmin, p["h"]):
            hmin = p["h"]
        if _is_greater(p["h"], hmax):
            hmax = p["h"]
    crc = np.zeros((nz, nz)); ckn = np.zeros((nz, nz)); cmu = np.zeros((nz, nz))
    cbn = np.zeros((nz, nz)); cka = np.zeros((nz, nz))
    maxr = 0.0
    for i in range(nz):
        for j in range(nz):
            c = spec.contact[(min(i, j), max(i, j))]
            crc[i, j] = c.radius_factor * hmin
            maxr = max(maxr, crc[i, j])
            cka[i, j] = 2. * zone_K[i] * zone_K[j] / (zone_K[i] + zone_K[j])
            ckn[i, j] = c.kn * c.kn_factor
            bf = c.betan_factor if c.damping_on else 0.0
            le = math.log(c.epsilon)
            cbn[i, j] = bf * (-2. * le * math.sqrt(1. / (math.pi * math.pi + le * le)))
            cmu[i, j] = c.friction_coeff if c.friction_on else 0.0
    # boundary conditions: particle-list selections (particleULoading.cpp:38-88)
    fix = np.zeros(N, dtype=np.uint8)

    def mk(bcs, disp):
        out = []
        for b in bcs:
            psel = np.zeros(Np, dtype=np.uint8)
            psel[b.particles] = 1
            nsel = np.zeros(N, dtype=np.uint8)
            for p in b.particles:
                nsel[parts[p]["start"]:parts[p]["end"]] = 1
            mask = 0
            for d in b.directions:
                mask |= 1 << (d - 1)
            if disp:
                for p in b.particles:
                    fix[parts[p]["start"]:parts[p]["end"]] |= np.uint8(mask)
            tp = np.zeros(4)
            if not b.zero:
                tp[:len(b.time_params)] = b.time_params
            sp = np.zeros(2)
            sp[:len(b.spatial_params)] = b.spatial_params
            box = np.zeros((Np, 6))
            tcode = TIME_CODE.get(b.time_fn, 99) if not b.zero else 99
            out.append(BCSet(time_fn=tcode, spatial_fn=SPATIAL_CODE.get(b.spatial_fn, 0),
                             dir_mask=mask, zero=b.zero, time_params=tp, spatial_params=sp,
                             particle_sel=psel, node_sel=nsel, particle_box=box))
        return out

    ubc = mk(spec.ubc, True)
    fbc = mk(spec.fbc, False)
    T = float(_f(spec.dt * spec.nt))
    dt = T / spec.nt   # input.cpp:281
    test = {"two_particle": 1, "compressive_test": 2}.get(spec.test_name, 0)
    return Scene(
        dim=dim, dt=dt, nt=spec.nt, xref=xref, vol=vol, fix=fix, ptid=ptid,
        p_start=P["start"], p_end=P["end"], p_center=P["center"], p_type=P["type"],
        p_zone=P["zone"], p_compute_force=P["compute_force"], p_all_fixed=P["all_fixed"],
        p_material=P["material"], p_horizon=P["horizon"], p_h=P["h"], p_density=P["density"],
        p_rc=P["rc"], p_kn=P["kn"], p_bound_r=P["bound_r"], p_mat=pmat,
        p_scale=P["scale"].astype(float), p_orient=P["orient"].astype(float),
        inf_type=inf_type, inf_params=inf, gravity=np.array(spec.gravity, dtype=float),
        time_scheme=1 if spec.time_scheme == "velocity_verlet" else 0,
        multi_particle=True, n_zones=nz, c_rc=crc.ravel(), c_kn=ckn.ravel(),
        c_mu=cmu.ravel(), c_betan=cbn.ravel(), c_kappa=cka.ravel(), max_contact_r=maxr,
        search_factor=spec.search_factor, search_interval=spec.search_interval,
        test=test, test_wall=spec.compressive_wall if test == 2 else 0,
        test_dir=spec.compressive_dir - 1 if test == 2 else 0,
        test_interval=spec.test_output_interval,
        x=xref.copy(), u=np.zeros_like(xref), v=np.zeros_like(xref),
        ubc=ubc, fbc=fbc,
        ic_velocity=np.array(spec.ic_velocity) if spec.ic_velocity is not None else None,
        ic_particles=np.array(spec.ic_particles, dtype=np.uint64), name=spec.name)


# ---------------------------------------------------------------------------
# batched ensembles
# ---------------------------------------------------------------------------
def ensemble_specs(n_scenes: int = 256, seed: int = 0, n_range: Tuple[int, int] = (20, 200),
                   r_range: Tuple[float, float] = (0.8e-3, 1.6e-3), h_div_range: Tuple[int, int] = (8, 16),
                   speed_range: Tuple[float, float] = (0.05, 0.2), material: str = "RNPBond",
                   nt: int = 20000, search_factor: float = 5.0) -> List[SceneSpec]:
    """Independent 2-D compression scenes of uneven size: per scene a
    particle count U[n_range], a mesh h = R / U{h_div_range}, a top-wall
    speed U[speed_range] and its own packing seed; discs and hexagons with
    radii U[r_range].  Every scene takes the smallest stable step of the set,
    so that they can advance together."""
    rng = np.random.default_rng(seed)
    picks = []
    for s in range(n_scenes):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        hd = int(rng.integers(h_div_range[0], h_div_range[1] + 1))
        v = float(rng.uniform(*speed_range))
        picks.append((n, hd, v))
    dt = min(stable_dt(2.0e9, 1200.0, r_range[0] / hd) for _, hd, _ in picks)
    spacing = 2.0 * r_range[1] + 1.05 * r_range[0] / h_div_range[0]
    specs = []
    for s, (n, hd, v) in enumerate(picks):
        width = math.ceil(math.sqrt(n)) * spacing
        specs.append(compressive_2d(n_particles=n, r_range=r_range, h_div=hd, width=width,
                                    seed=seed * 100003 + s, material=material, wall_speed=-v, dt=dt, nt=nt,
                                    search_factor=search_factor))
    return specs


def merge_scenes(scenes, pad: Optional[float] = None):
    """One model of independent scenes laid out on a grid, each shifted so
    that no contact candidate can join two scenes (``pad`` between their
    bounding boxes; default 4 search radii plus 2 mm).  Zones are renumbered
    per scene and the contact table is block-diagonal (no contact between
    scenes); the scenes' displacement BCs become sparse sets; particle
    offsets and test walls go to the ensemble tables (pdgpu_set_scenes).
    All scenes must share dt, influence function, time scheme, gravity and
    search parameters.  Zero-displacement sets are left out: the reference
    applies them through particle 0 only, which in these scenes is never a
    wall."""
    from .model import Scene, BCSet
    s0 = scenes[0]
    for sc in scenes:
        if (sc.dt != s0.dt or sc.inf_type != s0.inf_type or np.any(sc.inf_params != s0.inf_params)
                or sc.time_scheme != s0.time_scheme or np.any(sc.gravity != s0.gravity)
                or sc.search_factor != s0.search_factor or sc.search_interval != s0.search_interval
                or sc.dim != s0.dim or sc.test_dir != s0.test_dir or sc.test_interval != s0.test_interval):
            raise ValueError("scenes of an ensemble must share dt, influence, scheme, gravity, search and test")
        if sc.ic_velocity is not None and len(sc.ic_particles):
            raise ValueError("initial-velocity sets are not merged")
    dim = s0.dim
    max_rc = max(sc.max_contact_r for sc in scenes)
    if pad is None:
        pad = 4.0 * s0.search_factor * max_rc + 2e-3
    ext = [(sc.xref.min(axis=0), sc.xref.max(axis=0)) for sc in scenes]
    cw = max(hi[0] - lo[0] for lo, hi in ext) + pad
    ch = max(hi[1] - lo[1] for lo, hi in ext) + pad
    cols = int(math.ceil(math.sqrt(len(scenes))))
    xs, xr, vol, fix, ptid = [], [], [], [], []
    P = {k: [] for k in ("p_start", "p_end", "p_center", "p_type", "p_zone", "p_compute_force",
                         "p_all_fixed", "p_material", "p_horizon", "p_h", "p_density", "p_rc", "p_kn",
                         "p_bound_r", "p_mat", "p_scale", "p_orient")}
    nz_tot = sum(sc.n_zones for sc in scenes)
    tabs = {k: np.zeros((nz_tot, nz_tot)) for k in ("c_rc", "c_kn", "c_mu", "c_betan", "c_kappa")}
    ubc, poff, walls = [], [0], []
    n_off = p_off = z_off = 0
    for k, sc in enumerate(scenes):
        lo, _ = ext[k]
        shift = np.zeros(3)
        shift[0] = (k % cols) * cw - lo[0]
        shift[1] = (k // cols) * ch - lo[1]
        xr.append(sc.xref + shift)
        xs.append((sc.x if sc.x is not None else sc.xref) + shift)
        vol.append(sc.vol)
        fix.append(sc.fix)
        ptid.append(np.asarray(sc.ptid, dtype=np.uint64) + np.uint64(p_off))
        for key in P:
            a = getattr(sc, key)
            if key in ("p_start", "p_end", "p_center"):
                a = np.asarray(a) + n_off
            elif key == "p_zone":
                a = np.asarray(a) + z_off
            P[key].append(np.asarray(a))
        nz = sc.n_zones
        for key in tabs:
            tabs[key][z_off:z_off + nz, z_off:z_off + nz] = np.asarray(getattr(sc, key)).reshape(nz, nz)
        for b in sc.ubc:
            if b.zero:
                continue
            sel = np.nonzero(b.particle_sel)[0]
            nodes = np.nonzero(b.node_sel)[0]
            ubc.append(BCSet(time_fn=b.time_fn, spatial_fn=b.spatial_fn, dir_mask=b.dir_mask, zero=False,
                             time_params=b.time_params, spatial_params=b.spatial_params,
                             particle_sel=sel + p_off, node_sel=nodes + n_off,
                             particle_box=np.zeros((0, 6)), sparse=True))
        walls.append(int(sc.test_wall) + p_off if sc.test == 2 else -1)
        n_off += sc.n_nodes
        p_off += sc.n_particles
        z_off += nz
        poff.append(p_off)
    Np = p_off
    for b in ubc:
        b.particle_box = np.zeros((Np, 6))
    cat = lambda key: np.concatenate(P[key]) if key != "p_mat" else np.concatenate(P[key], axis=0)
    xref = np.concatenate(xr)
    return Scene(
        dim=dim, dt=s0.dt, nt=s0.nt, xref=xref, vol=np.concatenate(vol), fix=np.concatenate(fix),
        ptid=np.concatenate(ptid),
        **{key: cat(key) for key in P},
        inf_type=s0.inf_type, inf_params=s0.inf_params, gravity=s0.gravity, time_scheme=s0.time_scheme,
        multi_particle=True, n_zones=nz_tot, **{key: tabs[key].ravel() for key in tabs},
        max_contact_r=max_rc, search_factor=s0.search_factor, search_interval=s0.search_interval,
        test=0, test_wall=0, test_dir=s0.test_dir, test_interval=s0.test_interval,
        x=np.concatenate(xs), u=np.zeros_like(xref), v=np.zeros_like(xref), ubc=ubc, fbc=[],
        ic_velocity=None, ic_particles=np.zeros(0, dtype=np.uint64), name=f"ensemble_{len(scenes)}",
        scene_poff=np.array(poff, dtype=np.int64), scene_walls=np.array(walls, dtype=np.int64))


def build_scenes(specs: Sequence[SceneSpec], workers: int = 0) -> list:
    """build_scene over many specs, in a pool of spawned processes (the
    set-up is per-particle host work: transforms, mesh sizes, constants)."""
    if workers == 1 or len(specs) < 4:
        return [build_scene(s) for s in specs]
    import concurrent.futures as cf
    import multiprocessing as mp
    n = workers or min(len(specs), os.cpu_count() or 1, 64)
    with cf.ProcessPoolExecutor(max_workers=n, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(build_scene, specs, chunksize=max(1, len(specs) // (4 * n))))
