"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, as the checker.
The product (package bevy_xpbd_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_oracle

_lib = None
_variant = "serial"


def select(variant: str):
    """'serial' (checker, the reference's loop order) or 'omp' (OpenMP build, used only as the timed CPU baseline;
    it parallelises loops whose iterations are independent, so results are identical)."""
    global _lib, _variant
    if variant not in ("serial", "omp"):
        raise ValueError(variant)
    if variant != _variant:
        _variant = variant
        _lib = None


class OracleParams(C.Structure):
    """Layout of oracle::Params (xpbd_oracle.hpp): XpbdCpuTimeStepParams (xpbd_cpu.rs:11-26) + modes."""
    _fields_ = [
        ("dt", C.c_float), ("inv_dt", C.c_float), ("jacobi_omega", C.c_float), ("inner_iterations", C.c_uint32),
        ("gravity", C.c_float * 3), ("grab_idx", C.c_int32), ("grab_active", C.c_uint32),
        ("grab_target", C.c_float * 3), ("grab_stiffness", C.c_float), ("linear_drag_per_sec", C.c_float),
        ("solver", C.c_uint32), ("relaxation", C.c_uint32), ("lambda_mode", C.c_uint32),
        ("collision", C.c_uint32), ("thickness", C.c_float), ("coll_scale", C.c_float),
        ("hash_cell", C.c_float), ("ground_enabled", C.c_uint32), ("ground_y", C.c_float), ("damp", C.c_float),
        ("tolerance", C.c_float), ("warm_start", C.c_uint32), ("wind", C.c_float * 3), ("wind_drag", C.c_float),
    ]


def lib():
    global _lib
    if _lib is None:
        name = "liboracle.so" if _variant == "serial" else "liboracle_omp.so"
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), name)
        if not os.path.exists(path):
            build_oracle.build()
        L = C.CDLL(path)
        P = C.c_void_p
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.oracle_mesh_grid_hanging.restype = P
        L.oracle_mesh_grid_hanging.argtypes = [C.c_uint32, C.c_uint32, C.c_float]
        L.oracle_mesh_parse_obj.restype = P
        L.oracle_mesh_parse_obj.argtypes = [C.c_char_p]
        L.oracle_mesh_free.argtypes = [P]
        L.oracle_mesh_sizes.argtypes = [P, u32p]
        L.oracle_mesh_get.argtypes = [P] + [C.c_void_p] * 14
        L.oracle_partition.restype = C.c_uint32
        L.oracle_partition.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, C.c_int, u32p, u32p, u32p]
        L.oracle_build_csr.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, u32p, u32p, u32p]
        L.oracle_sim_create.restype = P
        L.oracle_sim_create.argtypes = [C.c_int, C.c_uint32, f32p, C.c_void_p, f32p, C.c_void_p,
                                        C.c_uint32, u32p, u32p, f32p, f32p, C.c_void_p]
        L.oracle_sim_free.argtypes = [P]
        L.oracle_sim_set_params.argtypes = [P, C.POINTER(OracleParams)]
        L.oracle_sim_substeps.argtypes = [P, C.c_uint32, C.c_int]
        L.oracle_sim_get.argtypes = [P, C.c_void_p, C.c_void_p]
        L.oracle_sim_set_state.argtypes = [P, C.c_void_p, C.c_void_p]
        L.oracle_sim_get_lambda.argtypes = [P, f64p]
        L.oracle_sim_set_warm_lambda.argtypes = [P, C.c_void_p]
        L.oracle_sim_strain_residual.restype = C.c_double
        L.oracle_sim_strain_residual.argtypes = [P]
        L.oracle_sim_collision_pairs_last.restype = C.c_uint64
        L.oracle_sim_collision_pairs_last.argtypes = [P]
        L.oracle_self_collision_resolve.argtypes = [C.c_uint32, f32p, f32p, f32p, C.c_float, C.c_float]
        L.oracle_hash_keys.argtypes = [C.c_uint32, f32p, C.c_float, C.c_uint32, u32p]
        L.oracle_stable_radix_sort.argtypes = [C.c_uint32, u32p, u32p, C.c_int]
        L.oracle_sim_collision_pairs.restype = C.c_uint64
        L.oracle_sim_collision_pairs.argtypes = [P, u32p, C.c_uint64]
        L.oracle_sim_set_batches.argtypes = [P, C.c_void_p, C.c_uint32]
        L.oracle_threads.restype = C.c_int
        L.oracle_sim_substeps_converge.argtypes = [P, C.c_uint32, C.c_void_p, C.c_void_p]
        L.oracle_sim_predicted.argtypes = [P, f64p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleMesh:
    """ClothMeshData (mesh_prep.rs:103-131) produced by the restated builders."""

    def __init__(self, handle):
        L = lib()
        sz = np.zeros(5, np.uint32)
        L.oracle_mesh_sizes(handle, sz)
        n, e, ni, nb, nn = (int(v) for v in sz)
        self.num_particles = n
        self.positions = np.zeros((n, 3), np.float32)
        self.rest_positions = np.zeros((n, 3), np.float32)
        self.inv_mass = np.zeros(n, np.float32)
        self.indices = np.zeros(ni, np.uint32)
        self.constraint_i = np.zeros(e, np.uint32)
        self.constraint_j = np.zeros(e, np.uint32)
        self.constraint_rest_len = np.zeros(e, np.float32)
        self.constraint_compliance = np.zeros(e, np.float32)
        self.constraint_batch_offsets = np.zeros(nb + 1, np.uint32)
        self.constraint_batch_count = nb
        self.neighbor_offsets = np.zeros(n + 1, np.uint32)
        self.neighbor_other = np.zeros(nn, np.uint32)
        self.neighbor_constraint_id = np.zeros(nn, np.uint32)
        self.neighbor_rest_len = np.zeros(nn, np.float32)
        self.neighbor_compliance = np.zeros(nn, np.float32)
        L.oracle_mesh_get(handle, *[_ptr(a) for a in (
            self.positions, self.rest_positions, self.inv_mass, self.indices, self.constraint_i, self.constraint_j,
            self.constraint_rest_len, self.constraint_compliance, self.constraint_batch_offsets,
            self.neighbor_offsets, self.neighbor_other, self.neighbor_constraint_id, self.neighbor_rest_len,
            self.neighbor_compliance)])
        L.oracle_mesh_free(handle)


def grid_cloth_hanging(quad_cols: int, quad_rows: int, cell_size: float) -> OracleMesh:
    """mesh_prep.rs:363-406."""
    return OracleMesh(lib().oracle_mesh_grid_hanging(quad_cols, quad_rows, cell_size))


def parse_welded_obj(text: str) -> OracleMesh:
    """mesh_prep.rs:223-357."""
    return OracleMesh(lib().oracle_mesh_parse_obj(text.encode()))


def partition(n: int, ci, cj, order_by_index: bool = False):
    """partition_constraints_for_gs_batches (mesh_prep.rs:153-221): (perm, colors, batch offsets)."""
    ci = np.ascontiguousarray(ci, np.uint32)
    cj = np.ascontiguousarray(cj, np.uint32)
    e = len(ci)
    perm = np.zeros(e, np.uint32)
    colors = np.zeros(e, np.uint32)
    offs = np.zeros(e + 2, np.uint32)
    nb = lib().oracle_partition(n, e, ci, cj, int(order_by_index), perm, colors, offs)
    return perm, colors, offs[: nb + 1].copy()


def build_csr(n: int, ci, cj):
    """Neighbour CSR cursor scatter, mesh_prep.rs:588-635: (offsets, other, constraint id)."""
    ci = np.ascontiguousarray(ci, np.uint32)
    cj = np.ascontiguousarray(cj, np.uint32)
    off = np.zeros(n + 1, np.uint32)
    other = np.zeros(2 * len(ci), np.uint32)
    eid = np.zeros(2 * len(ci), np.uint32)
    lib().oracle_build_csr(n, len(ci), ci, cj, off, other, eid)
    return off, other, eid


def make_params(p: dict) -> OracleParams:
    o = OracleParams()
    for k, v in p.items():
        if k in ("gravity", "grab_target", "wind"):
            getattr(o, k)[:] = [float(x) for x in v]
        elif hasattr(o, k):
            setattr(o, k, v)
    return o


class OracleSim:
    """Single cloth, FP32 (fp64=False: the reference's arithmetic) or FP64 accuracy build."""

    def __init__(self, x, inv_mass, ci, cj, rest, comp, v=None, rest_pos=None, ctype=None, fp64=False):
        L = self.L = lib()
        self.n = len(inv_mass)
        self.e = len(ci)
        keep = [np.ascontiguousarray(x, np.float32).reshape(-1), np.ascontiguousarray(inv_mass, np.float32),
                np.ascontiguousarray(ci, np.uint32), np.ascontiguousarray(cj, np.uint32),
                np.ascontiguousarray(rest, np.float32), np.ascontiguousarray(comp, np.float32)]
        vv = None if v is None else np.ascontiguousarray(v, np.float32).reshape(-1)
        rp = None if rest_pos is None else np.ascontiguousarray(rest_pos, np.float32).reshape(-1)
        ct = None if ctype is None else np.ascontiguousarray(ctype, np.uint32)
        self.h = L.oracle_sim_create(int(fp64), self.n, keep[0], _ptr(vv), keep[1], _ptr(rp), self.e, keep[2],
                                     keep[3], keep[4], keep[5], _ptr(ct))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_sim_free(self.h)
            self.h = None

    def set_params(self, params: dict):
        self._p = make_params(params)
        self.L.oracle_sim_set_params(self.h, C.byref(self._p))

    def substeps(self, count: int, brute_force: bool = False):
        self.L.oracle_sim_substeps(self.h, count, int(brute_force))

    def substeps_converge(self, count: int):
        """Convergence solve (extension); returns (update passes, fallback flag) per substep."""
        it = np.zeros(count, np.uint32)
        fb = np.zeros(count, np.uint32)
        self.L.oracle_sim_substeps_converge(self.h, count, _ptr(it), _ptr(fb))
        return it, fb

    def state(self):
        x = np.zeros((self.n, 3), np.float64)
        v = np.zeros((self.n, 3), np.float64)
        self.L.oracle_sim_get(self.h, _ptr(x), _ptr(v))
        return x, v

    def set_state(self, x=None, v=None):
        xx = None if x is None else np.ascontiguousarray(x, np.float32).reshape(-1)
        vv = None if v is None else np.ascontiguousarray(v, np.float32).reshape(-1)
        self.L.oracle_sim_set_state(self.h, _ptr(xx), _ptr(vv))

    def predicted(self):
        """Positions after the next substep's prediction step (xpbd_cpu.rs:251-260), state unchanged."""
        out = np.zeros((self.n, 3), np.float64)
        self.L.oracle_sim_predicted(self.h, out.reshape(-1))
        return out

    def lambdas(self):
        out = np.zeros(self.e, np.float64)
        self.L.oracle_sim_get_lambda(self.h, out)
        return out

    def set_warm_lambda(self, lam):
        self._warm = None if lam is None else np.ascontiguousarray(lam, np.float32)
        self.L.oracle_sim_set_warm_lambda(self.h, _ptr(self._warm))

    def set_batches(self, offsets):
        """Color-batch offsets of the (batch-sorted) constraints: lets the OpenMP build sweep a batch in parallel."""
        self._batches = np.ascontiguousarray(offsets, np.uint32)
        self.L.oracle_sim_set_batches(self.h, _ptr(self._batches), len(self._batches) - 1)

    def strain_residual(self) -> float:
        return float(self.L.oracle_sim_strain_residual(self.h))

    def collision_pairs(self, cap: int = 1 << 22):
        buf = np.zeros(2 * cap, np.uint32)
        cnt = int(self.L.oracle_sim_collision_pairs(self.h, buf, cap))
        if cnt > cap:
            return self.collision_pairs(cnt)
        return buf[: 2 * cnt].reshape(-1, 2).copy()


def threads() -> int:
    return int(lib().oracle_threads())


def self_collision_resolve(x, inv_mass, rest_pos, thickness, coll_scale):
    """xpbd_cpu.rs:67-137 (FP32, returns the new positions)."""
    xx = np.ascontiguousarray(x, np.float32).copy().reshape(-1)
    lib().oracle_self_collision_resolve(len(inv_mass), xx, np.ascontiguousarray(inv_mass, np.float32),
                                        np.ascontiguousarray(rest_pos, np.float32).reshape(-1), thickness,
                                        coll_scale)
    return xx.reshape(-1, 3)


def hash_keys(x, inv_cell: float, table_bits: int):
    x = np.ascontiguousarray(x, np.float32).reshape(-1)
    keys = np.zeros(len(x) // 3, np.uint32)
    lib().oracle_hash_keys(len(keys), x, inv_cell, table_bits, keys)
    return keys


def stable_radix_sort(keys, vals, passes: int = 4):
    k = np.ascontiguousarray(keys, np.uint32).copy()
    v = np.ascontiguousarray(vals, np.uint32).copy()
    lib().oracle_stable_radix_sort(len(k), k, v, passes)
    return k, v
