"""ctypes wrapper of the C oracle (oracle/pdoracle.c).

ORACLE TEST INFRASTRUCTURE ONLY: imported by tests, the smoke check and
the benchmark's CPU-baseline leg; never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libpdoracle.so")

P = ctypes.POINTER
c_d, c_i32, c_i64, c_u8, c_u64 = ctypes.c_double, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint8, ctypes.c_uint64


class PoBc(ctypes.Structure):
    _fields_ = [("time_fn", c_i32), ("spatial_fn", c_i32), ("dir_mask", c_i32), ("zero", c_i32),
                ("time_params", c_d * 4), ("spatial_params", c_d * 2),
                ("particle_sel", P(c_u8)), ("node_sel", P(c_u8)), ("particle_box", P(c_d))]


class PoScene(ctypes.Structure):
    _fields_ = [("dim", c_i32), ("time_scheme", c_i32), ("multi_particle", c_i32), ("test", c_i32),
                ("dt", c_d), ("gravity", c_d * 3), ("n_nodes", c_i64), ("n_particles", c_i64),
                ("xref", P(c_d)), ("vol", P(c_d)), ("fix", P(c_u8)), ("ptid", P(c_u64)),
                ("p_start", P(c_i64)), ("p_end", P(c_i64)), ("p_center", P(c_i64)),
                ("p_type", P(c_i32)), ("p_zone", P(c_i32)), ("p_compute_force", P(c_i32)),
                ("p_all_fixed", P(c_i32)), ("p_material", P(c_i32)),
                ("p_horizon", P(c_d)), ("p_h", P(c_d)), ("p_density", P(c_d)), ("p_rc", P(c_d)),
                ("p_kn", P(c_d)), ("p_bound_r", P(c_d)), ("p_mat", P(c_d)),
                ("inf_type", c_i32), ("inf_params", c_d * 2),
                ("n_zones", c_i32), ("c_rc", P(c_d)), ("c_kn", P(c_d)), ("c_mu", P(c_d)),
                ("c_betan", P(c_d)), ("c_kappa", P(c_d)),
                ("max_contact_r", c_d), ("search_factor", c_d), ("search_interval", c_i64),
                ("test_wall", c_i64), ("test_interval", c_i64), ("test_dir", c_i32),
                ("pd_rowptr", P(c_u64)), ("pd_col", P(c_u64)), ("mx", P(c_d)),
                ("n_ubc", c_i32), ("n_fbc", c_i32), ("ubc", P(PoBc)), ("fbc", P(PoBc)),
                ("ic_active", c_i32), ("ic_v", c_d * 3), ("ic_particle", P(c_u8))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.po_create.restype = vp
        L.po_create.argtypes = [P(PoScene)]
        for name in ("po_destroy", "po_integrate_begin"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        L.po_step.argtypes = [vp, c_i64]
        L.po_step.restype = None
        for name, rt in (("po_x", P(c_d)), ("po_u", P(c_d)), ("po_v", P(c_d)), ("po_f", P(c_d)),
                         ("po_Z", P(ctypes.c_float)), ("po_theta", P(c_d)), ("po_vmag", P(c_d)),
                         ("po_bonds", P(c_u8)), ("po_n", c_i64), ("po_time", c_d),
                         ("po_contact_entries", c_i64)):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = rt
        L.po_contact_state.argtypes = [vp, P(c_i64), P(c_i64), P(c_d), P(c_d)]
        L.po_contact_state.restype = None
        L.po_contact_lists.argtypes = [vp, P(c_u64), P(c_u64)]
        L.po_contact_lists.restype = None
        L.po_test_values.argtypes = [vp, P(c_d), P(c_d), P(c_d), P(c_d), P(c_d)]
        L.po_test_values.restype = None
        L.po_count_pd_neighbors.argtypes = [P(PoScene)]
        L.po_count_pd_neighbors.restype = c_i64
        L.po_build_pd_neighbors.argtypes = [P(PoScene), P(c_u64), P(c_u64)]
        L.po_build_pd_neighbors.restype = None
        L.po_compute_mx.argtypes = [P(PoScene), P(c_d)]
        L.po_compute_mx.restype = None
        _lib = L
    return _lib


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class _SceneStruct:
    """Keeps the numpy arrays a PoScene points into alive."""

    def __init__(self, sc):
        k = self.keep = []

        def ptr(a, dt, ct):
            a = _arr(a, dt)
            k.append(a)
            return a.ctypes.data_as(P(ct))

        s = PoScene()
        s.dim, s.time_scheme = sc.dim, sc.time_scheme
        s.multi_particle, s.test = int(sc.multi_particle), sc.test
        s.dt = sc.dt
        for q in range(3):
            s.gravity[q] = float(sc.gravity[q])
        s.n_nodes, s.n_particles = sc.n_nodes, sc.n_particles
        s.xref = ptr(sc.xref, np.float64, c_d)
        s.vol = ptr(sc.vol, np.float64, c_d)
        s.fix = ptr(sc.fix, np.uint8, c_u8)
        s.ptid = ptr(sc.ptid, np.uint64, c_u64)
        s.p_start = ptr(sc.p_start, np.int64, c_i64)
        s.p_end = ptr(sc.p_end, np.int64, c_i64)
        s.p_center = ptr(sc.p_center, np.int64, c_i64)
        for name in ("p_type", "p_zone", "p_compute_force", "p_all_fixed", "p_material"):
            setattr(s, name, ptr(getattr(sc, name), np.int32, c_i32))
        for name in ("p_horizon", "p_h", "p_density", "p_rc", "p_kn", "p_bound_r"):
            setattr(s, name, ptr(getattr(sc, name), np.float64, c_d))
        s.p_mat = ptr(np.asarray(sc.p_mat).reshape(-1, 6), np.float64, c_d)
        s.inf_type = int(sc.inf_type)
        s.inf_params[0], s.inf_params[1] = float(sc.inf_params[0]), float(sc.inf_params[1])
        if sc.multi_particle:
            s.n_zones = int(sc.n_zones)
            for name in ("c_rc", "c_kn", "c_mu", "c_betan", "c_kappa"):
                setattr(s, name, ptr(getattr(sc, name), np.float64, c_d))
        s.max_contact_r, s.search_factor = sc.max_contact_r, sc.search_factor
        s.search_interval = sc.search_interval
        s.test_wall, s.test_interval, s.test_dir = sc.test_wall, sc.test_interval, sc.test_dir
        if sc.pd_rowptr is not None:
            s.pd_rowptr = ptr(sc.pd_rowptr, np.uint64, c_u64)
            s.pd_col = ptr(sc.pd_col, np.uint64, c_u64)
        if sc.mx is not None:
            s.mx = ptr(sc.mx, np.float64, c_d)
        for attr, nattr, sets in (("ubc", "n_ubc", sc.ubc), ("fbc", "n_fbc", sc.fbc)):
            arr = (PoBc * max(1, len(sets)))()
            for k2, b in enumerate(sets):
                arr[k2].time_fn, arr[k2].spatial_fn = b.time_fn, b.spatial_fn
                arr[k2].dir_mask, arr[k2].zero = b.dir_mask, int(b.zero)
                for q in range(4):
                    arr[k2].time_params[q] = float(b.time_params[q]) if q < len(b.time_params) else 0.0
                for q in range(2):
                    arr[k2].spatial_params[q] = (float(b.spatial_params[q])
                                                 if q < len(b.spatial_params) else 0.0)
                arr[k2].particle_sel = ptr(b.particle_sel, np.uint8, c_u8)
                arr[k2].node_sel = ptr(b.node_sel, np.uint8, c_u8)
                arr[k2].particle_box = ptr(np.asarray(b.particle_box).reshape(-1), np.float64, c_d)
            k.append(arr)
            setattr(s, attr, ctypes.cast(arr, P(PoBc)))
            setattr(s, nattr, len(sets))
        if sc.ic_velocity is not None:
            s.ic_active = 1
            for q in range(3):
                s.ic_v[q] = float(sc.ic_velocity[q])
            sel = np.zeros(sc.n_particles, dtype=np.uint8)
            sel[np.asarray(sc.ic_particles, dtype=np.int64)] = 1
            s.ic_particle = ptr(sel, np.uint8, c_u8)
        self.s = s


def build_pd_neighbors(sc):
    """(rowptr, col) of the reference's peridynamic neighbour sets, node order."""
    st = _SceneStruct(sc)
    L = lib()
    B = L.po_count_pd_neighbors(ctypes.byref(st.s))
    rp = np.zeros(sc.n_nodes + 1, dtype=np.uint64)
    col = np.zeros(max(B, 1), dtype=np.uint64)
    L.po_build_pd_neighbors(ctypes.byref(st.s), rp.ctypes.data_as(P(c_u64)), col.ctypes.data_as(P(c_u64)))
    return rp, col[:B]


def compute_mx(sc):
    st = _SceneStruct(sc)
    mx = np.zeros(sc.n_nodes)
    lib().po_compute_mx(ctypes.byref(st.s), mx.ctypes.data_as(P(c_d)))
    return mx


class Oracle:
    """The reference's step restated in C; same interface as GpuDEMModel
    for the parts tests compare."""

    def __init__(self, sc):
        if sc.pd_rowptr is None:
            sc.pd_rowptr, sc.pd_col = build_pd_neighbors(sc)
        if sc.mx is None:
            sc.mx = compute_mx(sc)
        self.sc = sc
        self._st = _SceneStruct(sc)
        self.L = lib()
        self.m = self.L.po_create(ctypes.byref(self._st.s))

    def integrate_begin(self):
        self.L.po_integrate_begin(self.m)

    def step(self, n=1):
        self.L.po_step(self.m, n)

    def field(self, name):
        N, B = self.sc.n_nodes, self.sc.n_bonds
        g = {"x": (self.L.po_x, (N, 3)), "u": (self.L.po_u, (N, 3)), "v": (self.L.po_v, (N, 3)),
             "f": (self.L.po_f, (N, 3)), "Z": (self.L.po_Z, (N,)), "theta": (self.L.po_theta, (N,)),
             "vMag": (self.L.po_vmag, (N,)), "bonds": (self.L.po_bonds, (B,))}[name]
        ptr = g[0](self.m)
        return np.ctypeslib.as_array(ptr, shape=g[1]).copy()

    def contact_state(self):
        a, b, r, v = c_i64(), c_i64(), c_d(), c_d()
        self.L.po_contact_state(self.m, ctypes.byref(a), ctypes.byref(b), ctypes.byref(r), ctypes.byref(v))
        return {"interval": a.value, "counter": b.value, "radius": r.value, "max_velocity": v.value}

    def contact_lists(self):
        E = self.L.po_contact_entries(self.m)
        rp = np.zeros(self.sc.n_nodes + 1, dtype=np.uint64)
        col = np.zeros(max(E, 1), dtype=np.uint64)
        self.L.po_contact_lists(self.m, rp.ctypes.data_as(P(c_u64)), col.ctypes.data_as(P(c_u64)))
        return rp, col[:E]

    def test_values(self):
        vals = [c_d() for _ in range(5)]
        self.L.po_test_values(self.m, *[ctypes.byref(v) for v in vals])
        return dict(zip(("reaction", "penetration", "contact_reaction", "pen_dist", "max_y"),
                        [v.value for v in vals]))

    @property
    def n(self):
        return self.L.po_n(self.m)

    def close(self):
        if self.m:
            self.L.po_destroy(self.m)
            self.m = None

    def __del__(self):
        self.close()
