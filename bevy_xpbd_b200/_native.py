"""ctypes binding of libxpbd_cuda.so (the C ABI declared in include/xpbd_cuda.h).

The library is built in-tree by bevy_xpbd_b200/build.py. There is no fallback: if the shared library is missing or
cannot be loaded, importing the solver raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxpbd_cuda.so")

XPBD_OK = 0
STATUS_NAMES = {
    -1: "XPBD_ERR_INVALID_ARGUMENT", -2: "XPBD_ERR_CUDA", -3: "XPBD_ERR_OUT_OF_MEMORY", -4: "XPBD_ERR_UNSUPPORTED",
    -5: "XPBD_ERR_STATE", -6: "XPBD_ERR_DEVICE_NONFINITE", -7: "XPBD_ERR_BARRIER_TIMEOUT", -8: "XPBD_ERR_INDEX_RANGE",
    -9: "XPBD_ERR_CAPACITY", -10: "XPBD_ERR_NO_DEVICE",
}
ERR_BARRIER_TIMEOUT = -7
ERR_DEVICE_NONFINITE = -6
ERR_INVALID_ARGUMENT = -1
ERR_STATE = -5
ERR_INDEX_RANGE = -8
ERR_UNSUPPORTED = -4

EXPORTED = [
    "xpbd_create", "xpbd_destroy", "xpbd_default_opts", "xpbd_set_stream", "xpbd_add_cloth", "xpbd_commit",
    "xpbd_set_params", "xpbd_step", "xpbd_step_params", "xpbd_substep", "xpbd_sync", "xpbd_read_positions",
    "xpbd_read_velocities", "xpbd_write_state", "xpbd_reset", "xpbd_read_lambda", "xpbd_strain_residual",
    "xpbd_get_stats", "xpbd_get_coloring", "xpbd_autotune", "xpbd_collision_keys", "xpbd_collision_pairs",
    "xpbd_radix_sort_scratch_bytes", "xpbd_radix_sort_pairs", "xpbd_hash_keys", "xpbd_last_error",
    "xpbd_status_string", "xpbd_debug_force_barrier_timeout", "xpbd_color_constraints",
    "xpbd_radix_sort_pairs_noalloc", "xpbd_set_warm_lambda", "xpbd_mlp_init", "xpbd_mlp_set_params",
    "xpbd_mlp_get_params", "xpbd_mlp_collect", "xpbd_mlp_dataset_size", "xpbd_mlp_dataset_read",
    "xpbd_mlp_fit_normalization", "xpbd_mlp_train", "xpbd_mlp_eval", "xpbd_mlp_gradients", "xpbd_mlp_predict_lambda",
    "xpbd_converge_history", "xpbd_converge_cloth_iterations", "xpbd_selftest_division",
    "xpbd_mlp_minibatch_gradients", "xpbd_mlp_apply_gradients", "xpbd_set_triangles", "xpbd_read_normals",
    "xpbd_mesh_grid_hanging", "xpbd_mesh_from_obj", "xpbd_mesh_from_triangles", "xpbd_mesh_sizes", "xpbd_mesh_get",
    "xpbd_mesh_free", "xpbd_set_cloth_grab", "xpbd_set_cloth_wind", "xpbd_color_constraints_device_scratch_bytes",
    "xpbd_color_constraints_device", "xpbd_neighbor_table_device_scratch_bytes", "xpbd_neighbor_table_device",
]
MLP_PARAMS = 4865
MLP_NORM = 20
MLP_FEATURES = 9
NOALLOC_SORT_MAX_KEYS = 1 << 18
ERR_CAPACITY = -9


class TimeStepParams(C.Structure):
    _fields_ = [
        ("dt", C.c_float), ("inv_dt", C.c_float), ("jacobi_omega", C.c_float), ("inner_iterations", C.c_uint32),
        ("gravity", C.c_float * 3), ("grab_idx", C.c_int32), ("grab_active", C.c_uint32),
        ("grab_target", C.c_float * 3), ("grab_stiffness", C.c_float), ("linear_drag_per_sec", C.c_float),
    ]


class SolverOpts(C.Structure):
    _fields_ = [
        ("solver", C.c_uint32), ("relaxation", C.c_uint32), ("lambda_mode", C.c_uint32), ("substeps", C.c_uint32),
        ("collision", C.c_uint32), ("collision_every_n_substeps", C.c_uint32), ("thickness", C.c_float),
        ("coll_scale", C.c_float), ("hash_cell", C.c_float), ("hash_table_bits", C.c_uint32),
        ("ring_depth", C.c_uint32), ("ground_enabled", C.c_uint32), ("ground_y", C.c_float),
        ("use_graphs", C.c_uint32), ("barrier_timeout_ms", C.c_float), ("block_threads", C.c_uint32),
        ("blocks_per_sm", C.c_uint32), ("warm_start", C.c_uint32), ("cluster_ctas", C.c_uint32),
        ("jacobi_kernel", C.c_uint32), ("tolerance", C.c_float), ("gs_strips", C.c_uint32),
        ("reserved", C.c_uint32 * 2),
    ]


class ClothDesc(C.Structure):
    _fields_ = [
        ("num_particles", C.c_uint32), ("positions", C.c_void_p), ("velocities", C.c_void_p),
        ("inv_mass", C.c_void_p), ("rest_positions", C.c_void_p), ("num_constraints", C.c_uint32),
        ("constraint_i", C.c_void_p), ("constraint_j", C.c_void_p), ("rest_len", C.c_void_p),
        ("compliance", C.c_void_p), ("constraint_type", C.c_void_p), ("order", C.c_uint32),
        ("batch_offsets", C.c_void_p), ("batch_count", C.c_uint32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("frames", C.c_uint64), ("substeps", C.c_uint64), ("num_particles", C.c_uint32),
        ("num_constraints", C.c_uint32), ("num_cloths", C.c_uint32), ("num_colors", C.c_uint32),
        ("grid_blocks", C.c_uint32), ("block_threads", C.c_uint32), ("graph_captured", C.c_uint32),
        ("cooperative_launch", C.c_uint32), ("kernel_launches", C.c_uint64), ("warm_start_fallbacks", C.c_uint64),
        ("collision_pairs", C.c_uint64), ("solver_kernel", C.c_uint32), ("cluster_ctas", C.c_uint32),
        ("converge_iterations", C.c_uint64), ("converge_substeps", C.c_uint64),
        ("converge_max_iterations", C.c_uint32), ("pad", C.c_uint32),
    ]


_lib = None


def load():
    """Loads the in-tree CUDA library (raises if it is absent — there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m bevy_xpbd_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, I, U = C.c_void_p, C.c_int, C.c_uint32
    sig = {
        "xpbd_create": (I, [C.POINTER(C.c_void_p), I]),
        "xpbd_destroy": (None, [P]),
        "xpbd_default_opts": (None, [C.POINTER(SolverOpts)]),
        "xpbd_set_stream": (I, [P, P]),
        "xpbd_add_cloth": (I, [P, C.POINTER(ClothDesc), C.POINTER(U)]),
        "xpbd_commit": (I, [P]),
        "xpbd_set_params": (I, [P, C.POINTER(TimeStepParams), C.POINTER(SolverOpts)]),
        "xpbd_step": (I, [P, U]),
        "xpbd_step_params": (I, [P, C.POINTER(TimeStepParams), U]),
        "xpbd_substep": (I, [P, U]),
        "xpbd_sync": (I, [P]),
        "xpbd_read_positions": (I, [P, U, P]),
        "xpbd_read_velocities": (I, [P, U, P]),
        "xpbd_write_state": (I, [P, U, P, P]),
        "xpbd_reset": (I, [P]),
        "xpbd_read_lambda": (I, [P, U, P]),
        "xpbd_strain_residual": (I, [P, U, C.POINTER(C.c_float)]),
        "xpbd_get_stats": (I, [P, C.POINTER(Stats)]),
        "xpbd_get_coloring": (I, [P, U, P, P, C.POINTER(U)]),
        "xpbd_autotune": (I, [P, U, C.POINTER(SolverOpts)]),
        "xpbd_collision_keys": (I, [P, P, P, P]),
        "xpbd_collision_pairs": (I, [P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
        "xpbd_radix_sort_scratch_bytes": (C.c_size_t, [U]),
        "xpbd_radix_sort_pairs": (I, [P, P, P, P, U, U, P, C.c_size_t, P]),
        "xpbd_hash_keys": (I, [P, U, C.c_float, U, P, P]),
        "xpbd_last_error": (C.c_char_p, [P]),
        "xpbd_status_string": (C.c_char_p, [I]),
        "xpbd_debug_force_barrier_timeout": (I, [P, C.c_float]),
        "xpbd_color_constraints": (I, [U, U, P, P, U, P, P, C.POINTER(U)]),
        "xpbd_radix_sort_pairs_noalloc": (I, [P, P, P, P, U, U, P]),
        "xpbd_color_constraints_device_scratch_bytes": (C.c_size_t, [U, U, U]),
        "xpbd_color_constraints_device": (I, [U, U, P, P, U, U, P, P, P, P, C.POINTER(U), P, C.c_size_t, P]),
        "xpbd_neighbor_table_device_scratch_bytes": (C.c_size_t, [U, U]),
        "xpbd_neighbor_table_device": (I, [U, U, P, P, P, P, P, P, C.c_size_t, P]),
        "xpbd_set_warm_lambda": (I, [P, U, P]),
        "xpbd_mlp_init": (I, [P, C.c_uint64, U]),
        "xpbd_mlp_set_params": (I, [P, P, P]),
        "xpbd_mlp_get_params": (I, [P, P, P]),
        "xpbd_mlp_collect": (I, [P, U, U]),
        "xpbd_mlp_dataset_size": (I, [P, C.POINTER(U)]),
        "xpbd_mlp_dataset_read": (I, [P, U, P, P, C.POINTER(U)]),
        "xpbd_mlp_fit_normalization": (I, [P]),
        "xpbd_mlp_train": (I, [P, U, U, C.c_float, C.c_uint64, P]),
        "xpbd_mlp_eval": (I, [P, P, U, P]),
        "xpbd_mlp_gradients": (I, [P, P, P, U, P, P]),
        "xpbd_mlp_predict_lambda": (I, [P, U, P]),
        "xpbd_converge_history": (I, [P, P, U, C.POINTER(U)]),
        "xpbd_converge_cloth_iterations": (I, [P, P]),
        "xpbd_selftest_division": (I, [I, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
        "xpbd_mlp_minibatch_gradients": (I, [P, U, C.c_uint64, P, P]),
        "xpbd_mlp_apply_gradients": (I, [P, P, C.c_float, C.c_float]),
        "xpbd_set_triangles": (I, [P, U, U, P]),
        "xpbd_read_normals": (I, [P, U, P]),
        "xpbd_mesh_grid_hanging": (I, [U, U, C.c_float, C.POINTER(C.c_void_p)]),
        "xpbd_mesh_from_obj": (I, [C.c_char_p, C.POINTER(C.c_void_p)]),
        "xpbd_mesh_from_triangles": (I, [U, P, U, P, U, P, P, P, P, C.POINTER(C.c_void_p)]),
        "xpbd_mesh_sizes": (I, [P, C.POINTER(U), C.POINTER(U), C.POINTER(U), C.POINTER(U)]),
        "xpbd_mesh_get": (I, [P, P, P, P, P, P, P, P, P]),
        "xpbd_mesh_free": (None, [P]),
        "xpbd_set_cloth_grab": (I, [P, U, C.c_int32, P, C.c_float]),
        "xpbd_set_cloth_wind": (I, [P, U, P, C.c_float]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class XpbdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
