"""ctypes binding of libb200dem.so (the C ABI declared in include/b200dem.h).

There is no CPU fallback: importing a solver without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb200dem.so")

DEM_OK = 0
ERR = {
    0x001: "DEM_ERR_INVALID", 0x002: "DEM_ERR_CUDA", 0x004: "DEM_ERR_CONTACT_OVERFLOW",
    0x008: "DEM_ERR_NEIGHBOR_OVERFLOW", 0x010: "DEM_ERR_NAN", 0x020: "DEM_ERR_TIMEOUT",
    0x040: "DEM_ERR_BOND_OVERFLOW", 0x080: "DEM_ERR_NOMEM", 0x100: "DEM_ERR_UNSUPPORTED",
    0x200: "DEM_ERR_MESH_OVERFLOW",
}
DEM_ERR_CONTACT_OVERFLOW = 0x004
DEM_ERR_TIMEOUT = 0x020

# enum dem_field
F = {name: k for k, name in enumerate(
    ["x", "u", "omega", "force", "torque", "m", "rho", "rad", "I", "E", "nu", "G", "tng_idx", "tng_ss_x",
     "tng_ss_y", "tng_ss_z", "tng_count", "tng_sw_x", "tng_sw_y", "tng_sw_z", "fix", "ext_force", "scene"])}
W = {name: k for k, name in enumerate(["x", "u", "omega", "normal", "E", "nu", "G"])}
DEM_FP64, DEM_MIXED = 0, 1


class ForceParams(C.Structure):
    _fields_ = [("cor_pp", C.c_double), ("cor_pw", C.c_double), ("mu_pp", C.c_double), ("mu_pw", C.c_double),
                ("quirks", C.c_uint)]


class SolverParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("delta", C.c_double), ("skin", C.c_double), ("rebuild_every_step", C.c_int),
                ("precision", C.c_int), ("gravity", C.c_double * 3), ("max_neighbors", C.c_int),
                ("steps_per_launch", C.c_int), ("stream_block", C.c_int), ("contact_lanes", C.c_int),
                ("stream_split", C.c_int), ("dense_form", C.c_int), ("scene_kernel", C.c_int),
                ("launch_overlap", C.c_int), ("cooperative_loop", C.c_int)]


class SceneParams(C.Structure):
    _fields_ = [("cor_pp", C.c_double), ("cor_pw", C.c_double), ("mu_pp", C.c_double), ("mu_pw", C.c_double)]


class BondParams(C.Structure):
    _fields_ = [("quirks", C.c_uint), ("beta", C.c_double), ("radius_factor", C.c_double), ("kn", C.c_double),
                ("kt", C.c_double), ("break_strain", C.c_double)]


BFIELD = {name: k for k, name in enumerate(
    ["idx", "init_len", "count", "ft_x", "ft_y", "ft_z", "mn_x", "mn_y", "mn_z", "mt_x", "mt_y", "mt_z", "broken"])}


class RunStats(C.Structure):
    _fields_ = [("steps", C.c_long), ("rebuilds", C.c_long), ("max_neighbors", C.c_int),
                ("neighbor_capacity", C.c_int), ("status", C.c_int), ("disp_bound", C.c_double),
                ("launches", C.c_long), ("graph_ms", C.c_double), ("graph_steps", C.c_long),
                ("launch_overlap", C.c_int), ("cooperative_loop", C.c_int)]


class NnRows(C.Structure):
    _fields_ = [("data", C.c_void_p), ("index", C.c_void_p), ("width", C.c_int)]


class NnMlp(C.Structure):
    _fields_ = [("kin", C.c_int), ("nout", C.c_int), ("w1t", C.c_void_p), ("w1", C.c_void_p), ("b1", C.c_void_p),
                ("w2t", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p)]


class SurrogateParams(C.Structure):
    _fields_ = [("radius_graph", C.c_double), ("steps_per_stride", C.c_int), ("dt", C.c_double),
                ("sigma_d", C.c_double), ("sigma_a", C.c_double), ("r_mean", C.c_double), ("r_std", C.c_double),
                ("nwalls", C.c_int), ("wall_x", (C.c_double * 3) * 4), ("wall_n", (C.c_double * 3) * 4),
                ("wall_clip", C.c_double), ("gravity", C.c_double * 3), ("max_overlap", C.c_double),
                ("energy_tol", C.c_double), ("max_nodes", C.c_int), ("max_frames", C.c_int),
                ("project_iters", C.c_int), ("project_allow", C.c_double)]


class RolloutStats(C.Structure):
    _fields_ = [("strides_network", C.c_long), ("strides_dem", C.c_long), ("fallback_overlap", C.c_long),
                ("fallback_energy", C.c_long), ("max_overlap_seen", C.c_double)]


class DemError(RuntimeError):
    pass


_lib = None

_VP = C.c_void_p
_PROTOS = {
    "dem_version": ([], C.c_int),
    "dem_ctx_create": ([C.c_int, C.POINTER(_VP)], C.c_int),
    "dem_ctx_destroy": ([_VP], C.c_int),
    "dem_ctx_sync": ([_VP], C.c_int),
    "dem_last_error": ([_VP], C.c_char_p),
    "dem_particles_create": ([_VP, C.c_int, C.c_int, C.c_int, C.POINTER(_VP)], C.c_int),
    "dem_particles_destroy": ([_VP], C.c_int),
    "dem_particles_set": ([_VP, C.c_int, _VP, C.c_long], C.c_int),
    "dem_particles_get": ([_VP, C.c_int, _VP, C.c_long], C.c_int),
    "dem_particles_size": ([_VP], C.c_int),
    "dem_walls_create": ([_VP, C.c_int, C.POINTER(_VP)], C.c_int),
    "dem_walls_destroy": ([_VP], C.c_int),
    "dem_walls_set": ([_VP, C.c_int, _VP, C.c_long], C.c_int),
    "dem_solver_create": ([_VP, _VP, _VP, C.POINTER(ForceParams), C.POINTER(SolverParams), C.POINTER(_VP)],
                          C.c_int),
    "dem_solver_destroy": ([_VP], C.c_int),
    "dem_solver_run": ([_VP, C.c_int], C.c_int),
    "dem_solver_stats": ([_VP, C.POINTER(RunStats)], C.c_int),
    "dem_solver_wall_positions": ([_VP, _VP, C.c_long], C.c_int),
    "dem_solver_set_mesh": ([_VP, _VP, C.c_int, C.c_double, C.c_double, C.c_double, _VP, C.c_int], C.c_int),
    "dem_solver_mesh_translation": ([_VP, _VP], C.c_int),
    "dem_solver_profile": ([_VP, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "dem_ctx_stream": ([_VP], C.c_void_p),
    "dem_stage1": ([_VP], C.c_int),
    "dem_stage2": ([_VP], C.c_int),
    "dem_stage3": ([_VP], C.c_int),
    "dem_build_neighbors": ([_VP], C.c_int),
    "dem_solver_rebuild": ([_VP], C.c_int),
    "dem_solver_set_timestep": ([_VP, C.c_double], C.c_int),
    "dem_compute_force": ([_VP], C.c_int),
    "dem_neighbors_get": ([_VP, _VP, _VP, C.POINTER(C.c_long)], C.c_int),
    "dem_energy": ([_VP, C.POINTER(C.c_double)], C.c_int),
    "dem_solver_set_scenes": ([_VP, _VP, C.c_int, C.c_int], C.c_int),
    "dem_bonds_create": ([_VP, C.c_int, C.POINTER(BondParams), C.POINTER(_VP)], C.c_int),
    "dem_bonds_destroy": ([_VP], C.c_int),
    "dem_bonds_setup": ([_VP, C.c_double, C.c_double], C.c_int),
    "dem_bonds_get": ([_VP, C.c_int, _VP, C.c_long], C.c_int),
    "dem_bonds_broken": ([_VP, C.POINTER(C.c_long)], C.c_int),
    "dem_bonded_run": ([_VP, C.c_int], C.c_int),
    "dem_bonds_set": ([_VP, C.c_int, _VP, C.c_long], C.c_int),
    "dem_bonded_reset": ([_VP], C.c_int),
    "dem_apply_external_force": ([_VP], C.c_int),
    "dem_bonded_force": ([_VP, C.c_double], C.c_int),
    "dem_apply_boundary_conditions": ([_VP], C.c_int),
    "dem_neighbor_list_noalloc": ([_VP, _VP, C.c_int, C.c_double, C.c_double, C.c_int, _VP, _VP, _VP], C.c_int),
    "dem_nn_mlp_forward": ([_VP, C.POINTER(NnMlp), C.c_long, C.POINTER(NnRows), C.c_int, _VP, _VP, _VP, _VP],
                           C.c_int),
    "dem_nn_mlp_backward": ([_VP, C.POINTER(NnMlp), C.c_long, C.POINTER(NnRows), C.c_int, _VP, _VP, _VP, _VP, _VP,
                             _VP, _VP, _VP], C.c_int),
    "dem_nn_edge_forward": ([_VP, C.c_long, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.c_int], C.c_int),
    "dem_nn_status": ([_VP, C.POINTER(C.c_int)], C.c_int),
    "dem_nn_debug_waits": ([_VP, C.c_int, C.c_int], C.c_int),
    "dem_solver_debug_stream_waits": ([_VP, C.c_int, C.c_int], C.c_int),
    "dem_particles_get_device": ([_VP, C.c_int, _VP, C.c_long], C.c_int),
    "dem_particles_clear_contacts": ([_VP], C.c_int),
    "dem_particles_clear_forces": ([_VP], C.c_int),
    "dem_checkpoint_save": ([_VP, C.c_char_p], C.c_int),
    "dem_checkpoint_load": ([_VP, C.c_char_p], C.c_int),
    "dem_surrogate_create": ([_VP, C.POINTER(SurrogateParams), C.POINTER(_VP)], C.c_int),
    "dem_surrogate_destroy": ([_VP], C.c_int),
    "dem_surrogate_num_params": ([_VP], C.c_long),
    "dem_surrogate_get_params": ([_VP, _VP, C.c_long], C.c_int),
    "dem_surrogate_set_params": ([_VP, _VP, C.c_long], C.c_int),
    "dem_surrogate_init_params": ([_VP, C.c_ulonglong], C.c_int),
    "dem_surrogate_loss_grad": ([_VP, C.c_int, _VP, _VP, _VP, _VP, _VP, C.c_int, C.c_double, C.c_ulonglong,
                                 C.POINTER(C.c_double), _VP], C.c_int),
    "dem_surrogate_train_step": ([_VP, C.c_int, _VP, _VP, _VP, _VP, _VP, C.c_int, C.c_double, C.c_ulonglong,
                                  C.c_double, C.POINTER(C.c_double)], C.c_int),
    "dem_surrogate_predict": ([_VP, C.c_int, _VP, _VP, _VP, _VP, C.c_int, _VP], C.c_int),
    "dem_surrogate_rollout": ([_VP, _VP, C.c_int, C.c_int, C.POINTER(RolloutStats)], C.c_int),
}
NOALLOC_MAX_PARTICLES = 32768
NOALLOC_MAX_NEIGHBORS = 128


def exported_symbols():
    """Names the C ABI header declares (checked against the library's exports)."""
    return sorted(_PROTOS)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DemError("libb200dem.so is not built (run __graft_entry__.build() or make -C cabanadem_b200/csrc); "
                           "there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _PROTOS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(st, ctx=None, what="", allow=0):
    if st & ~allow:
        msg = ", ".join(v for k, v in ERR.items() if st & k) or str(st)
        detail = ""
        if ctx is not None:
            try:
                detail = lib().dem_last_error(ctx).decode()
            except Exception:
                pass
        raise DemError(f"{what}: {msg} {detail}".strip())
    return st
