"""Host-side model: the scene data a ``DEMModel`` holds after ``init()`` and
the GPU model that steps it through the C ABI (``include/pdgpu.h``).

``GpuDEMModel`` mirrors the step methods of the reference's
``model::DEMModel`` (src/model/dem/demModel.h:74-233): ``init`` uploads
ModelData, ``integrate_begin`` is the prelude of ``DEMModel::integrate``
(demModel.cpp:268-283) and ``integrate_step`` is ``DEMModel::integrateStep``
plus the test post-processing of the integrate loop (:285-324).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import api

# bond laws, influence functions, BC function codes (include/pdgpu.h)
MAT_RNP, MAT_PMB, MAT_PDELASTIC, MAT_PDSTATE = 0, 1, 2, 3
MATERIAL_CODES = {"RNPBond": MAT_RNP, "PMBBond": MAT_PMB, "PDElasticBond": MAT_PDELASTIC,
                  "PDState": MAT_PDSTATE}
TEST_NONE, TEST_TWO_PARTICLE, TEST_COMPRESSIVE = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
FIELD = {"x": 0, "u": 1, "v": 2, "f": 3, "Z": 4, "vMag": 5, "theta": 6, "mX": 7, "bonds": 8,
         "fix": 9}


@dataclass
class BCSet:
    """One boundary-condition set with its node / particle selection."""
    time_fn: int
    spatial_fn: int
    dir_mask: int
    zero: bool
    time_params: np.ndarray        # 4
    spatial_params: np.ndarray     # 2
    particle_sel: np.ndarray       # uint8 [Np] (sparse: selected particle ids)
    node_sel: np.ndarray           # uint8 [N] (sparse: selected node ids)
    particle_box: np.ndarray       # float64 [Np, 6]
    sparse: bool = False           # selections given as index lists (merged scenes)


@dataclass
class Scene:
    """ModelData of one scene after ``DEMModel::init`` (arrays in the
    reference's layouts: points as [N, 3] float64, ids as uint64)."""
    dim: int
    dt: float
    nt: int
    xref: np.ndarray
    vol: np.ndarray
    fix: np.ndarray
    ptid: np.ndarray
    # particles [Np]
    p_start: np.ndarray
    p_end: np.ndarray
    p_center: np.ndarray
    p_type: np.ndarray
    p_zone: np.ndarray
    p_compute_force: np.ndarray
    p_all_fixed: np.ndarray
    p_material: np.ndarray
    p_horizon: np.ndarray
    p_h: np.ndarray
    p_density: np.ndarray
    p_rc: np.ndarray
    p_kn: np.ndarray
    p_bound_r: np.ndarray
    p_mat: np.ndarray               # [Np, 6]
    inf_type: int
    inf_params: np.ndarray          # 2
    gravity: np.ndarray = field(default_factory=lambda: np.zeros(3))
    time_scheme: int = 0
    multi_particle: bool = True
    n_zones: int = 0
    c_rc: Optional[np.ndarray] = None
    c_kn: Optional[np.ndarray] = None
    c_mu: Optional[np.ndarray] = None
    c_betan: Optional[np.ndarray] = None
    c_kappa: Optional[np.ndarray] = None
    max_contact_r: float = 0.0
    search_factor: float = 1.0
    search_interval: int = 1
    test: int = TEST_NONE
    test_wall: int = 0
    test_dir: int = 0
    test_interval: int = 1
    x: Optional[np.ndarray] = None
    u: Optional[np.ndarray] = None
    v: Optional[np.ndarray] = None
    mx: Optional[np.ndarray] = None
    pd_rowptr: Optional[np.ndarray] = None
    pd_col: Optional[np.ndarray] = None
    bond_state: Optional[np.ndarray] = None
    ubc: List[BCSet] = field(default_factory=list)
    fbc: List[BCSet] = field(default_factory=list)
    ic_velocity: Optional[np.ndarray] = None
    ic_particles: Optional[np.ndarray] = None
    name: str = "scene"
    # per particle: size relative to its zone's reference mesh and rotation
    # about z (set by the scene builder; used by the learned surrogate)
    p_scale: Optional[np.ndarray] = None
    p_orient: Optional[np.ndarray] = None
    # batched ensemble (scene.merge_scenes): particle offsets of the scenes
    # (CSR, n_scenes + 1) and each scene's test wall (-1: none)
    scene_poff: Optional[np.ndarray] = None
    scene_walls: Optional[np.ndarray] = None

    @property
    def n_scenes(self) -> int:
        return 1 if self.scene_poff is None else len(self.scene_poff) - 1

    @property
    def n_nodes(self) -> int:
        return int(self.xref.shape[0])

    @property
    def n_particles(self) -> int:
        return int(self.p_start.shape[0])

    @property
    def n_bonds(self) -> int:
        return int(self.pd_rowptr[-1]) if self.pd_rowptr is not None else 0


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class GpuDEMModel:
    """A scene on one B200, stepped by the sm_100a kernels of libpdgpu.

    precision: PREC_FP64 (the drop-in form) or PREC_MIXED (FP32 bond loop).
    build_neighbors: build the peridynamic neighbour lists on the device
    instead of uploading ``scene.pd_rowptr/pd_col``; compute_mx likewise for
    the weighted volume.
    """

    def __init__(self, scene: Scene, precision: int = PREC_FP64, device: int = 0,
                 build_neighbors: bool = False, compute_mx: bool = False,
                 contact_capacity: int = 0, wall_pair_capacity: int = 0,
                 pd_lanes: int = 0, tile_nodes: int = 0, bond_scheme: int = 0,
                 contact_lanes: int = 0, contact_ctas: int = 0):
        self.lib = api.lib()
        self.scene = scene
        desc = api.Desc()
        desc.dim = scene.dim
        desc.time_scheme = scene.time_scheme
        desc.precision = precision
        desc.device = device
        desc.dt = scene.dt
        for q in range(3):
            desc.gravity[q] = float(scene.gravity[q])
        desc.multi_particle = 1 if scene.multi_particle else 0
        desc.test = scene.test
        desc.test_wall = scene.test_wall
        desc.test_dir = scene.test_dir
        desc.test_interval = scene.test_interval
        desc.search_factor = scene.search_factor
        desc.search_interval = scene.search_interval
        desc.max_contact_r = scene.max_contact_r
        desc.contact_capacity = contact_capacity
        desc.wall_pair_capacity = wall_pair_capacity
        ctx = ctypes.c_void_p()
        rc = self.lib.pdgpu_create(ctypes.byref(desc), ctypes.byref(ctx))
        if rc != 0:
            msg = ctypes.create_string_buffer(256)
            self.lib.pdgpu_device_check(device, msg, 256)
            raise api.PdgpuError(rc, f"pdgpu_create failed: {msg.value.decode()}")
        self.ctx = ctx
        self.precision = precision
        self._closed = False
        if pd_lanes:
            api.set_lanes(self, pd_lanes)
        if tile_nodes:
            self._check(self.lib.pdgpu_set_tile_nodes(self.ctx, tile_nodes))
        if bond_scheme:
            self._check(self.lib.pdgpu_set_bond_scheme(self.ctx, bond_scheme))
        if contact_lanes:
            api.set_lanes(self, 0, contact_lanes)
        if contact_ctas:
            self._check(self.lib.pdgpu_set_contact_grid(self.ctx, contact_ctas))
        self._upload(build_neighbors, compute_mx)

    # ---- DEMModel::init: upload ModelData -----------------------------------
    def _upload(self, build_neighbors: bool, compute_mx: bool) -> None:
        s, L, c = self.scene, self.lib, self.ctx
        N = s.n_nodes
        self._keep = []
        xref = _f64(s.xref)
        x = _f64(s.x) if s.x is not None else xref
        u = _f64(s.u) if s.u is not None else np.zeros_like(xref)
        v = _f64(s.v) if s.v is not None else np.zeros_like(xref)
        vol = _f64(s.vol)
        fix = np.ascontiguousarray(s.fix, dtype=np.uint8)
        pt = np.ascontiguousarray(s.ptid, dtype=np.uint64)
        self._check(L.pdgpu_upload_nodes(c, N, _ptr(xref, ctypes.c_double), _ptr(x, ctypes.c_double),
                                         _ptr(u, ctypes.c_double), _ptr(v, ctypes.c_double),
                                         _ptr(vol, ctypes.c_double), _ptr(fix, ctypes.c_uint8),
                                         _ptr(pt, ctypes.c_uint64)))
        Np = s.n_particles
        parts = (api.Particle * Np)()
        for k in range(Np):
            P = parts[k]
            P.glob_start = int(s.p_start[k])
            P.glob_end = int(s.p_end[k])
            P.center_node = int(s.p_center[k])
            P.type = int(s.p_type[k])
            P.zone = int(s.p_zone[k])
            P.compute_force = int(s.p_compute_force[k])
            P.all_dofs_constrained = int(s.p_all_fixed[k])
            P.material = int(s.p_material[k])
            P.horizon = float(s.p_horizon[k])
            P.h = float(s.p_h[k])
            P.density = float(s.p_density[k])
            P.rc = float(s.p_rc[k])
            P.kn = float(s.p_kn[k])
            P.bound_r = float(s.p_bound_r[k])
            for q in range(6):
                P.mat[q] = float(s.p_mat[k, q])
        self._check(L.pdgpu_upload_particles(c, Np, parts))
        if s.scene_poff is not None:
            po = np.ascontiguousarray(s.scene_poff, dtype=np.int64)
            tw = np.ascontiguousarray(s.scene_walls, dtype=np.int64)
            self._check(L.pdgpu_set_scenes(c, len(po) - 1, _ptr(po, ctypes.c_int64), _ptr(tw, ctypes.c_int64)))
        ip = (ctypes.c_double * 2)(*[float(a) for a in s.inf_params[:2]])
        self._check(L.pdgpu_set_influence(c, int(s.inf_type), ip))
        if s.multi_particle:
            arrs = [_f64(a) for a in (s.c_rc, s.c_kn, s.c_mu, s.c_betan, s.c_kappa)]
            self._check(L.pdgpu_upload_contact(c, int(s.n_zones),
                                               *[_ptr(a, ctypes.c_double) for a in arrs]))
        if build_neighbors:
            self._check(L.pdgpu_build_pd_neighbors(c))
        else:
            rp = np.ascontiguousarray(s.pd_rowptr, dtype=np.uint64)
            col = np.ascontiguousarray(s.pd_col, dtype=np.uint64)
            bs = None
            if s.bond_state is not None:
                bs = np.ascontiguousarray(s.bond_state, dtype=np.uint8)
            self._check(L.pdgpu_upload_pd_neighbors(
                c, _ptr(rp, ctypes.c_uint64), _ptr(col, ctypes.c_uint64),
                _ptr(bs, ctypes.c_uint8) if bs is not None else None))
        if compute_mx or s.mx is None:
            self._check(L.pdgpu_compute_mx(c))
        else:
            mx = _f64(s.mx)
            self._check(L.pdgpu_upload_mx(c, _ptr(mx, ctypes.c_double)))
        for sets, fn in ((s.ubc, L.pdgpu_add_displacement_bc), (s.fbc, L.pdgpu_add_force_bc)):
            for b in sets:
                bc = api.BcSet()
                bc.time_fn = b.time_fn
                bc.spatial_fn = b.spatial_fn
                bc.dir_mask = b.dir_mask
                bc.zero = 1 if b.zero else 0
                for q in range(4):
                    bc.time_params[q] = float(b.time_params[q]) if q < len(b.time_params) else 0.0
                for q in range(2):
                    bc.spatial_params[q] = (float(b.spatial_params[q])
                                            if q < len(b.spatial_params) else 0.0)
                if b.sparse:
                    ps = np.zeros(Np, dtype=np.uint8)
                    ps[np.asarray(b.particle_sel, dtype=np.int64)] = 1
                    ns = np.zeros(N, dtype=np.uint8)
                    ns[np.asarray(b.node_sel, dtype=np.int64)] = 1
                else:
                    ps = np.ascontiguousarray(b.particle_sel, dtype=np.uint8)
                    ns = np.ascontiguousarray(b.node_sel, dtype=np.uint8)
                bx = _f64(b.particle_box).reshape(-1)
                self._check(fn(c, ctypes.byref(bc), _ptr(ps, ctypes.c_uint8),
                               _ptr(ns, ctypes.c_uint8), _ptr(bx, ctypes.c_double)))
        if s.ic_velocity is not None:
            icv = (ctypes.c_double * 3)(*[float(a) for a in s.ic_velocity])
            pl = np.ascontiguousarray(s.ic_particles, dtype=np.uint64)
            self._check(L.pdgpu_set_initial_condition(c, icv, _ptr(pl, ctypes.c_uint64), len(pl)))
        if s.multi_particle:
            self._check(L.pdgpu_init_contact(c))

    # ---- DEMModel::integrate / integrateStep ----------------------------------
    def integrate_begin(self) -> None:
        self._check(self.lib.pdgpu_integrate_begin(self.ctx))

    def integrate_step(self, nsteps: int = 1, graph_steps: int = 0) -> None:
        if graph_steps:
            self._check(self.lib.pdgpu_step_graph(self.ctx, nsteps, graph_steps))
        else:
            self._check(self.lib.pdgpu_step(self.ctx, nsteps))

    def sync(self) -> None:
        self._check(self.lib.pdgpu_sync(self.ctx))

    # ---- fields ---------------------------------------------------------------
    def field(self, name: str) -> np.ndarray:
        N = self.scene.n_nodes
        f = FIELD[name]
        if name in ("x", "u", "v", "f"):
            out = np.empty((N, 3), dtype=np.float64)
        elif name == "Z":
            out = np.empty(N, dtype=np.float32)
        elif name in ("vMag", "theta", "mX"):
            out = np.empty(N, dtype=np.float64)
        elif name == "fix":
            out = np.empty(N, dtype=np.uint8)
        else:
            nb = ctypes.c_int64()
            self._check(self.lib.pdgpu_num_bonds(self.ctx, ctypes.byref(nb)))
            out = np.empty(nb.value, dtype=np.uint8)
        self._check(self.lib.pdgpu_download(self.ctx, f, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def scalars(self) -> Dict[str, float]:
        sc = api.Scalars()
        self._check(self.lib.pdgpu_get_scalars(self.ctx, ctypes.byref(sc)))
        return {k: getattr(sc, k) for k, _ in api.Scalars._fields_}

    def history(self) -> np.ndarray:
        cnt = ctypes.c_int64()
        self._check(self.lib.pdgpu_get_history(self.ctx, None, None, None, None, 0, ctypes.byref(cnt)))
        n = cnt.value
        cols = [np.empty(n) for _ in range(4)]
        self._check(self.lib.pdgpu_get_history(self.ctx, *[_ptr(c, ctypes.c_double) for c in cols],
                                                n, ctypes.byref(cnt)))
        return np.stack(cols, axis=1)

    def contact_lists(self):
        N = self.scene.n_nodes
        rp = np.empty(N + 1, dtype=np.uint64)
        self._check(self.lib.pdgpu_download_contact(self.ctx, _ptr(rp, ctypes.c_uint64), None))
        col = np.empty(int(rp[-1]), dtype=np.uint64)
        self._check(self.lib.pdgpu_download_contact(self.ctx, _ptr(rp, ctypes.c_uint64),
                                                    _ptr(col, ctypes.c_uint64)))
        return rp, col

    def pd_neighbors(self):
        N = self.scene.n_nodes
        nb = ctypes.c_int64()
        self._check(self.lib.pdgpu_num_bonds(self.ctx, ctypes.byref(nb)))
        rp = np.empty(N + 1, dtype=np.uint64)
        col = np.empty(nb.value, dtype=np.uint64)
        self._check(self.lib.pdgpu_download_pd_neighbors(self.ctx, _ptr(rp, ctypes.c_uint64),
                                                         _ptr(col, ctypes.c_uint64)))
        return rp, col

    def step_kernel_count(self) -> int:
        n = ctypes.c_int64()
        self._check(self.lib.pdgpu_step_kernel_count(self.ctx, ctypes.byref(n)))
        return n.value

    def stream_handle(self) -> int:
        p = ctypes.c_void_p()
        self._check(self.lib.pdgpu_get_stream(self.ctx, ctypes.byref(p)))
        return p.value or 0

    def enable_timing(self, on: bool = True) -> None:
        self._check(self.lib.pdgpu_enable_timing(self.ctx, 1 if on else 0))

    def kernel_times(self) -> Dict[str, tuple]:
        names = (ctypes.c_char_p * 64)()
        ms = (ctypes.c_double * 64)()
        cnt = (ctypes.c_int64 * 64)()
        n = ctypes.c_int32()
        self._check(self.lib.pdgpu_kernel_times(self.ctx, 64, names, ms, cnt, ctypes.byref(n)))
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(n.value)}

    def set_field(self, name: str, values: np.ndarray) -> None:
        """Overwrite x, u, v ([N, 3] float64) or the bond state ("bonds",
        uint8 per bond, 1 = broken) (pdgpu_upload_field)."""
        if name == "bonds":
            a = np.ascontiguousarray(values, dtype=np.uint8)
            ptr = a.ctypes.data_as(ctypes.c_void_p)
        else:
            a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.scene.n_nodes, 3)
            ptr = a.ctypes.data_as(ctypes.c_void_p)
        self._check(self.lib.pdgpu_upload_field(self.ctx, FIELD[name], ptr))

    def write_vtu(self, path: str, tags=("Displacement", "Velocity", "Force", "Force_Density", "Damage_Z",
                                         "Particle_ID", "Zone_ID", "Fixity", "Nodal_Volume")) -> None:
        """DEMModel::output: the current state as a .vtu file (pdgpu_write_vtu)."""
        self._check(self.lib.pdgpu_write_vtu(self.ctx, path.encode(), ",".join(tags).encode()))

    def strain_stress_tri(self, conn: np.ndarray, order: int, nu, lam, mu, plane_strain):
        """Quadrature-point strain and stress of linear triangles (2-D) from the
        current displacement (pdgpu_strain_stress_tri): conn [m, 3] global
        node ids, quadrature order 1 or 2, per-element (or scalar) nu,
        lambda, mu and plane-strain flag.  Returns xq [3 m, 3], strain and
        stress [3 m, 6] (xx, yy, zz, yz, xz, xy), three entries per element
        as the reference stores them."""
        from . import fe
        conn = np.ascontiguousarray(conn, dtype=np.int64).reshape(-1, 3)
        m = len(conn)
        pts = np.ascontiguousarray(fe.tri_points(order))
        arr = [np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (m,))) for a in (nu, lam, mu)]
        ps = np.ascontiguousarray(np.broadcast_to(np.asarray(plane_strain, dtype=np.uint8), (m,)))
        xq = np.zeros((3 * m, 3))
        strain = np.zeros((3 * m, 6))
        stress = np.zeros((3 * m, 6))
        self._check(self.lib.pdgpu_strain_stress_tri(
            self.ctx, m, _ptr(conn, ctypes.c_int64), len(pts), _ptr(pts, ctypes.c_double),
            *(_ptr(a, ctypes.c_double) for a in arr), _ptr(ps, ctypes.c_uint8),
            _ptr(xq, ctypes.c_double), _ptr(strain, ctypes.c_double), _ptr(stress, ctypes.c_double)))
        return xq, strain, stress

    def strain_stress_tet(self, conn: np.ndarray, nu, lam, mu):
        """Quadrature-point strain and stress of linear tetrahedra (3-D) from
        the current displacement, one-point rule (pdgpu_strain_stress_tet):
        conn [m, 4]; returns xq [3 m, 3], strain and stress [3 m, 6]."""
        conn = np.ascontiguousarray(conn, dtype=np.int64).reshape(-1, 4)
        m = len(conn)
        arr = [np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (m,))) for a in (nu, lam, mu)]
        xq = np.zeros((3 * m, 3))
        strain = np.zeros((3 * m, 6))
        stress = np.zeros((3 * m, 6))
        self._check(self.lib.pdgpu_strain_stress_tet(
            self.ctx, m, _ptr(conn, ctypes.c_int64), *(_ptr(a, ctypes.c_double) for a in arr),
            _ptr(xq, ctypes.c_double), _ptr(strain, ctypes.c_double), _ptr(stress, ctypes.c_double)))
        return xq, strain, stress

    def write_strain_vtu(self, path: str, xq: np.ndarray, strain: np.ndarray, stress: np.ndarray) -> None:
        """output_strain_<n>.vtu as VtkParticleWriter::appendStrainStress writes
        it (pdgpu_write_strain_vtu), from strain_stress_tri/_tet results."""
        xq, strain, stress = (np.ascontiguousarray(a, dtype=np.float64) for a in (xq, strain, stress))
        self._check(self.lib.pdgpu_write_strain_vtu(self.ctx, path.encode(), len(xq), _ptr(xq, ctypes.c_double),
                                                    _ptr(strain, ctypes.c_double), _ptr(stress, ctypes.c_double)))

    def rebuild_phases(self, on: Optional[bool] = None) -> List[int]:
        """Phase clock of the contact-list rebuild (pdgpu_enable_rebuild_phases /
        pdgpu_rebuild_phases): with `on` given, switch recording; returns the
        latest rebuild's marks (GPU global timer, ns)."""
        if on is not None:
            self._check(self.lib.pdgpu_enable_rebuild_phases(self.ctx, 1 if on else 0))
        buf = (ctypes.c_int64 * 16)()
        n = ctypes.c_int32()
        self._check(self.lib.pdgpu_rebuild_phases(self.ctx, buf, 16, ctypes.byref(n)))
        return list(buf[:n.value])

    def bond_scheme(self) -> int:
        """Mixed bond loop: 0 every bond from both ends, node order; 1 symmetric
        bond visits (2-D); 2 every bond from both ends, nodes longest row first."""
        v = ctypes.c_int32()
        self._check(self.lib.pdgpu_bond_scheme(self.ctx, ctypes.byref(v)))
        return v.value

    def save_state(self, path: str) -> None:
        """Snapshot of the whole step state, bond bits included (pdgpu_save_state)."""
        self._check(self.lib.pdgpu_save_state(self.ctx, path.encode()))

    def load_state(self, path: str) -> None:
        """Continue from a snapshot of the same scene; in place of
        integrate_begin (pdgpu_load_state)."""
        self._check(self.lib.pdgpu_load_state(self.ctx, path.encode()))

    def write_vtu_async(self, path: str, tags=("Displacement", "Velocity", "Force", "Force_Density", "Damage_Z",
                                              "Particle_ID", "Zone_ID", "Fixity", "Nodal_Volume")) -> None:
        """write_vtu of the state as of now, written while later steps run
        (pdgpu_write_vtu_async); output_wait() finishes it."""
        self._check(self.lib.pdgpu_write_vtu_async(self.ctx, path.encode(), ",".join(tags).encode()))

    def output_wait(self) -> None:
        self._check(self.lib.pdgpu_output_wait(self.ctx))

    def restart(self, path: str, step: int) -> None:
        """DEMModel::restart from a file of write_vtu; before integrate_begin."""
        self._check(self.lib.pdgpu_restart(self.ctx, path.encode(), int(step)))

    def scene_history(self, scene: int) -> np.ndarray:
        """Compressive-test records of one scene of an ensemble: rows of
        (time, wall displacement, reaction, contact reaction)."""
        cnt = ctypes.c_int64()
        self._check(self.lib.pdgpu_get_scene_history(self.ctx, scene, None, None, None, None, 0,
                                                     ctypes.byref(cnt)))
        n = cnt.value
        cols = [np.empty(n) for _ in range(4)]
        self._check(self.lib.pdgpu_get_scene_history(self.ctx, scene, *[_ptr(c, ctypes.c_double) for c in cols],
                                                     n, ctypes.byref(cnt)))
        return np.stack(cols, axis=1)

    def surrogate_stats(self):
        """(particles on the learned surrogate now, particles it covers,
        particle-steps on the surrogate so far, particle-steps covered)."""
        v = [ctypes.c_int64() for _ in range(4)]
        self._check(self.lib.pdgpu_surrogate_stats(self.ctx, *(ctypes.byref(x) for x in v)))
        return tuple(x.value for x in v)

    def surrogate_errors(self) -> np.ndarray:
        """The last check step per particle: (sum |f_s - f|^2, sum |f|^2),
        an (n_particles, 2) array."""
        out = np.zeros((self.scene.n_particles, 2), dtype=np.float64)
        self._check(self.lib.pdgpu_surrogate_errors(self.ctx, _ptr(out, ctypes.c_double), out.size))
        return out

    def compute_pd_forces(self) -> None:
        """DEMModel::computePeridynamicForces alone on the current state
        (pdgpu_compute_pd_forces): peridynamic f and Z, bonds may break."""
        self._check(self.lib.pdgpu_compute_pd_forces(self.ctx))

    def step_host(self, u: np.ndarray, v: np.ndarray, x: np.ndarray, f: np.ndarray,
                  nsteps: int = 1) -> None:
        """One reference-facing step on host buffers (pdgpu_step_host)."""
        self._check(self.lib.pdgpu_step_host(self.ctx, _ptr(u, ctypes.c_double),
                                             _ptr(v, ctypes.c_double), _ptr(x, ctypes.c_double),
                                             _ptr(f, ctypes.c_double), nsteps, None))

    # ---- lifetime ---------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.pdgpu_last_error(self.ctx, buf, 512)
            raise api.PdgpuError(rc, buf.value.decode())

    def close(self) -> None:
        if not self._closed:
            self.lib.pdgpu_destroy(self.ctx)
            self._closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
