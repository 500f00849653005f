"""Cloth meshes — the crate's `ClothMeshData` builders (src/mesh_prep.rs) over the C ABI.

    mesh = grid_cloth_hanging(24, 18, 0.045)          # or parse_welded_obj(text), finalize_cloth_mesh(...)
    plugin.add_mesh(mesh)                             # constraints already batch-sorted (ORDER_PRESORTED)

Fields (host arrays): positions, rest_positions, inv_mass, indices (triangles), constraint_i, constraint_j,
constraint_rest_len, constraint_compliance (greedy-colored batch order), constraint_batch_offsets.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import XpbdError

DEFAULT_STRETCH_COMPLIANCE = np.float32(2e-8)   # mesh_prep.rs:93
DEFAULT_BEND_COMPLIANCE = np.float32(3.8)       # mesh_prep.rs:89
DEFAULT_SKIP2_COMPLIANCE = np.float32(2.5e-8)   # mesh_prep.rs:97
DEFAULT_CROSS_DIAG_COMPLIANCE = np.float32(6e-9)  # mesh_prep.rs:101


class ClothMeshData:
    """mesh_prep.rs:103-131 (the render attributes normals/uvs are not kept: vertex normals come from the solver)."""

    def __init__(self, handle):
        L = N.load()
        nv, nt, ne, nb = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        L.xpbd_mesh_sizes(handle, C.byref(nv), C.byref(nt), C.byref(ne), C.byref(nb))
        n, t, e, b = nv.value, nt.value, ne.value, nb.value
        self.positions = np.zeros((n, 3), np.float32)
        self.inv_mass = np.zeros(n, np.float32)
        self.indices = np.zeros(3 * t, np.uint32)
        self.constraint_i = np.zeros(e, np.uint32)
        self.constraint_j = np.zeros(e, np.uint32)
        self.constraint_rest_len = np.zeros(e, np.float32)
        self.constraint_compliance = np.zeros(e, np.float32)
        self.constraint_batch_offsets = np.zeros(b + 1, np.uint32)
        arrs = [self.positions, self.inv_mass, self.indices, self.constraint_i, self.constraint_j,
                self.constraint_rest_len, self.constraint_compliance, self.constraint_batch_offsets]
        L.xpbd_mesh_get(handle, *[a.ctypes.data_as(C.c_void_p) for a in arrs])
        L.xpbd_mesh_free(handle)
        self.rest_positions = self.positions.copy()
        self.num_particles = n
        self.num_distance_constraints = e
        self.constraint_batch_count = b

    def to_spec_arrays(self) -> dict:
        """Keyword arguments of ClothComputePlugin.add_cloth (as ClothMeshData::to_sim_config hands them over)."""
        from .plugin import ORDER_PRESORTED
        return dict(positions=self.positions, inv_mass=self.inv_mass, constraint_i=self.constraint_i,
                    constraint_j=self.constraint_j, rest_len=self.constraint_rest_len,
                    compliance=self.constraint_compliance, rest_positions=self.rest_positions,
                    order=ORDER_PRESORTED, batch_offsets=self.constraint_batch_offsets)


def _build(status: int, handle: C.c_void_p) -> ClothMeshData:
    if status != N.XPBD_OK:
        raise XpbdError(status, "mesh build failed")
    return ClothMeshData(handle)


def grid_cloth_hanging(quad_cols: int, quad_rows: int, cell_size: float) -> ClothMeshData:
    h = C.c_void_p()
    return _build(N.load().xpbd_mesh_grid_hanging(quad_cols, quad_rows, C.c_float(cell_size), C.byref(h)), h)


def parse_welded_obj(obj_text: str) -> ClothMeshData:
    h = C.c_void_p()
    return _build(N.load().xpbd_mesh_from_obj(obj_text.encode(), C.byref(h)), h)


def finalize_cloth_mesh(positions, indices, extra_constraints=()) -> ClothMeshData:
    """extra_constraints: iterable of (i, j, rest, compliance)."""
    x = np.ascontiguousarray(positions, np.float32).reshape(-1)
    t = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    ex = list(extra_constraints)
    ei = np.ascontiguousarray([c[0] for c in ex], np.uint32)
    ej = np.ascontiguousarray([c[1] for c in ex], np.uint32)
    er = np.ascontiguousarray([c[2] for c in ex], np.float32)
    ec = np.ascontiguousarray([c[3] for c in ex], np.float32)
    h = C.c_void_p()
    p = [a.ctypes.data_as(C.c_void_p) for a in (x, t, ei, ej, er, ec)]
    st = N.load().xpbd_mesh_from_triangles(x.size // 3, p[0], t.size // 3, p[1], len(ex), p[2], p[3], p[4], p[5],
                                           C.byref(h))
    return _build(st, h)
