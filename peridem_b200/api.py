"""ctypes binding of libpdgpu (include/pdgpu.h).

The product path has no fallback: importing the binding without a built
library, or creating a context without a B200, raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpdgpu.so")

_lib = None


class PdgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pdgpu error {code}: {msg}")
        self.code = code


c_i32, c_i64, c_d, c_u8, c_u64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_uint8, ctypes.c_uint64
P = ctypes.POINTER
c_vp = ctypes.c_void_p


class Desc(ctypes.Structure):
    _fields_ = [("dim", c_i32), ("time_scheme", c_i32), ("precision", c_i32), ("device", c_i32),
                ("dt", c_d), ("gravity", c_d * 3), ("multi_particle", c_i32), ("test", c_i32),
                ("test_wall", c_i64), ("test_dir", c_i32), ("pad0", c_i32), ("test_interval", c_i64),
                ("search_factor", c_d), ("search_interval", c_i64), ("max_contact_r", c_d),
                ("contact_capacity", c_i64), ("wall_pair_capacity", c_i64)]


class Particle(ctypes.Structure):
    _fields_ = [("glob_start", c_i64), ("glob_end", c_i64), ("center_node", c_i64),
                ("type", c_i32), ("zone", c_i32), ("compute_force", c_i32),
                ("all_dofs_constrained", c_i32), ("material", c_i32), ("pad0", c_i32),
                ("horizon", c_d), ("h", c_d), ("density", c_d), ("rc", c_d), ("kn", c_d),
                ("bound_r", c_d), ("mat", c_d * 6)]


class MaterialDeck(ctypes.Structure):
    _fields_ = [("law", ctypes.c_int32), ("irreversible", ctypes.c_int32), ("E", ctypes.c_double),
                ("K", ctypes.c_double), ("G", ctypes.c_double), ("nu", ctypes.c_double),
                ("Gc", ctypes.c_double), ("check_sc_factor", ctypes.c_double)]


class BcSet(ctypes.Structure):
    _fields_ = [("time_fn", c_i32), ("spatial_fn", c_i32), ("dir_mask", c_i32), ("zero", c_i32),
                ("time_params", c_d * 4), ("spatial_params", c_d * 2)]


class Scalars(ctypes.Structure):
    _fields_ = [("n", c_i64), ("time", c_d), ("reaction", c_d), ("contact_reaction", c_d),
                ("wall_penetration", c_d), ("max_velocity", c_d), ("contact_search_radius", c_d),
                ("contact_update_interval", c_i64), ("contact_counter", c_i64),
                ("contact_updates", c_i64), ("contact_entries", c_i64), ("broken_bonds", c_i64),
                ("pen_dist", c_d), ("max_y", c_d), ("contact_area_radius", c_d)]


# every entry point of include/pdgpu.h with its argument types
SIGNATURES = {
    "pdgpu_device_check": [c_i32, ctypes.c_char_p, ctypes.c_size_t],
    "pdgpu_create": [P(Desc), P(c_vp)],
    "pdgpu_destroy": [c_vp],
    "pdgpu_last_error": [c_vp, ctypes.c_char_p, ctypes.c_size_t],
    "pdgpu_upload_nodes": [c_vp, c_i64, P(c_d), P(c_d), P(c_d), P(c_d), P(c_d), P(c_u8), P(c_u64)],
    "pdgpu_upload_particles": [c_vp, c_i64, P(Particle)],
    "pdgpu_set_influence": [c_vp, c_i32, P(c_d)],
    "pdgpu_upload_contact": [c_vp, c_i32, P(c_d), P(c_d), P(c_d), P(c_d), P(c_d)],
    "pdgpu_upload_pd_neighbors": [c_vp, P(c_u64), P(c_u64), P(c_u8)],
    "pdgpu_save_state": [c_vp, ctypes.c_char_p],
    "pdgpu_write_vtu_async": [c_vp, ctypes.c_char_p, ctypes.c_char_p],
    "pdgpu_output_wait": [c_vp],
    "pdgpu_mesh_size": [c_i32, P(c_d), c_i64, P(c_i64), P(c_i64), c_i64, P(c_d)],
    "pdgpu_influence_params": [c_i32, c_i32, P(c_d), c_i32, P(c_d)],
    "pdgpu_material_constants": [P(MaterialDeck), c_i32, c_d, c_i32, P(c_d), P(c_d), P(c_d)],
    "pdgpu_set_bond_scheme": [c_vp, c_i32],
    "pdgpu_set_contact_grid": [c_vp, c_i32],
    "pdgpu_bond_scheme": [c_vp, P(c_i32)],
    "pdgpu_load_state": [c_vp, ctypes.c_char_p],
    "pdgpu_build_pd_neighbors": [c_vp],
    "pdgpu_upload_mx": [c_vp, P(c_d)],
    "pdgpu_compute_mx": [c_vp],
    "pdgpu_add_displacement_bc": [c_vp, P(BcSet), P(c_u8), P(c_u8), P(c_d)],
    "pdgpu_add_force_bc": [c_vp, P(BcSet), P(c_u8), P(c_u8), P(c_d)],
    "pdgpu_set_initial_condition": [c_vp, P(c_d), P(c_u64), c_i64],
    "pdgpu_init_contact": [c_vp],
    "pdgpu_integrate_begin": [c_vp],
    "pdgpu_step": [c_vp, c_i64],
    "pdgpu_step_graph": [c_vp, c_i64, c_i32],
    "pdgpu_sync": [c_vp],
    "pdgpu_step_kernel_count": [c_vp, P(c_i64)],
    "pdgpu_download": [c_vp, c_i32, c_vp],
    "pdgpu_upload_field": [c_vp, c_i32, c_vp],
    "pdgpu_step_host": [c_vp, P(c_d), P(c_d), P(c_d), P(c_d), c_i64, P(Scalars)],
    "pdgpu_get_scalars": [c_vp, P(Scalars)],
    "pdgpu_get_history": [c_vp, P(c_d), P(c_d), P(c_d), P(c_d), c_i64, P(c_i64)],
    "pdgpu_download_contact": [c_vp, P(c_u64), P(c_u64)],
    "pdgpu_num_bonds": [c_vp, P(c_i64)],
    "pdgpu_download_pd_neighbors": [c_vp, P(c_u64), P(c_u64)],
    "pdgpu_set_tuning": [c_vp, c_i32, c_i32],
    "pdgpu_get_stream": [c_vp, P(c_vp)],
    "pdgpu_enable_timing": [c_vp, c_i32],
    "pdgpu_kernel_times": [c_vp, c_i32, P(ctypes.c_char_p), P(c_d), P(c_i64), P(c_i32)],
    "pdgpu_strain_stress_tri": [c_vp, c_i64, P(c_i64), c_i32, P(c_d), P(c_d), P(c_d), P(c_d), P(ctypes.c_uint8),
                                P(c_d), P(c_d), P(c_d)],
    "pdgpu_strain_stress_tet": [c_vp, c_i64, P(c_i64), P(c_d), P(c_d), P(c_d), P(c_d), P(c_d), P(c_d)],
    "pdgpu_write_strain_vtu": [c_vp, ctypes.c_char_p, c_i64, P(c_d), P(c_d), P(c_d)],
    "pdgpu_enable_rebuild_phases": [c_vp, c_i32],
    "pdgpu_rebuild_phases": [c_vp, P(c_i64), c_i32, P(c_i32)],
    "pdgpu_compute_pd_forces": [c_vp],
    "pdgpu_set_tile_nodes": [c_vp, c_i32],
    "pdgpu_tc_gemm": [c_vp, c_i32, c_vp, c_i32, c_i32, c_i32, c_i32, c_vp, c_i32, c_vp, c_vp, c_i32,
                      c_vp, c_vp],
    "pdgpu_build_neighbors_noalloc": [c_vp, c_vp, c_vp, c_i64, c_i32, c_vp, c_vp, c_i64, P(c_i64),
                                      c_vp, ctypes.c_char_p, ctypes.c_size_t],
    "pdgpu_write_vtu": [c_vp, ctypes.c_char_p, ctypes.c_char_p],
    "pdgpu_restart": [c_vp, ctypes.c_char_p, c_i64],
    "pdgpu_set_scenes": [c_vp, c_i32, P(c_i64), P(c_i64)],
    "pdgpu_get_scene_history": [c_vp, c_i32, P(c_d), P(c_d), P(c_d), P(c_d), c_i64, P(c_i64)],
    "pdgpu_set_surrogate_chain": [c_vp, c_i32],
    "pdgpu_set_surrogate": [c_vp, c_i32, c_vp, P(c_d), P(c_d), P(c_d), P(c_d), c_i32, c_d, c_d, c_i32],
    "pdgpu_surrogate_stats": [c_vp, P(c_i64), P(c_i64), P(c_i64), P(c_i64)],
    "pdgpu_surrogate_errors": [c_vp, P(c_d), c_i64],
    "pdgpu_sur_mse_grad": [c_vp, c_vp, c_i64, ctypes.c_float, c_vp, c_vp, c_vp, c_vp],
    "pdgpu_sur_tanh_back": [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp],
    "pdgpu_sur_colsum": [c_vp, c_i32, c_i32, c_vp, c_vp],
    "pdgpu_sur_transpose": [c_vp, c_i32, c_i32, c_vp, c_vp],
    "pdgpu_sur_adam": [c_vp, c_vp, c_vp, c_vp, c_i64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                       ctypes.c_float, c_i32, c_vp, c_vp],
}


class SurShape(ctypes.Structure):
    """pdgpu_sur_shape: one reference shape of the learned surrogate."""
    _fields_ = [("zone", c_i32), ("n_nodes", c_i32),
                ("phi_t", P(ctypes.c_float)), ("psi", P(ctypes.c_float)),
                ("w1", P(ctypes.c_float)), ("b1", P(ctypes.c_float)),
                ("w2", P(ctypes.c_float)), ("b2", P(ctypes.c_float)),
                ("w3", P(ctypes.c_float)), ("b3", P(ctypes.c_float))]


def lib(path: str = LIB_PATH):
    """Load libpdgpu.so (built in-tree by peridem_b200.build); raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libpdgpu.so not built ({path}); run python -m peridem_b200.build")
    L = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = None if name == "pdgpu_destroy" else c_i32
    _lib = L
    return L


def set_lanes(model, pd_lanes: int = 0, contact_lanes: int = 0) -> None:
    model._check(model.lib.pdgpu_set_tuning(model.ctx, pd_lanes, contact_lanes))
