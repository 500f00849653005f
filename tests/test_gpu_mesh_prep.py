"""Mesh preparation on the GPU against the host path and the oracle, bit for bit.

xpbd_color_constraints_device must give exactly the coloring of partition_constraints_for_gs_batches
(mesh_prep.rs:153-221) — the oracle's restatement and the library's host coloring — on sheets, the reference's
hanging grid, batches of cloths colored in one call, and random graphs with repeated constraints and hubs of more than
64 colors. xpbd_neighbor_table_device must give the cursor-scatter table of finalize_cloth_mesh (mesh_prep.rs:588-635).
"""
import ctypes as C

import numpy as np
import pytest

from bevy_xpbd_b200 import _native as N
from bevy_xpbd_b200 import mesh as M
from bevy_xpbd_b200 import workloads as wl
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

REF, INDEX = 0, 1


def _vp(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def color_device(n, ci, cj, order=REF, cloths=None):
    """cloths: None = one graph (schedule over the whole grid); a list of constraint offsets = one CTA per cloth."""
    import torch
    L = N.load()
    e = len(ci)
    dci, dcj = _dev(torch, ci), _dev(torch, cj)
    perm = torch.empty(max(e, 1), dtype=torch.int32, device="cuda")
    colors = torch.empty(max(e, 1), dtype=torch.int32, device="cuda")
    offs = torch.empty(e + 2, dtype=torch.int32, device="cuda")
    nc = 0 if cloths is None else len(cloths) - 1
    coff = np.ascontiguousarray(cloths if cloths is not None else [0], np.uint32)
    nbytes = L.xpbd_color_constraints_device_scratch_bytes(n, e, nc)
    scratch = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    bc = C.c_uint32()
    st = L.xpbd_color_constraints_device(n, e, _vp(dci), _vp(dcj), order, nc, coff.ctypes.data if nc else None,
                                         _vp(perm), _vp(colors), _vp(offs), C.byref(bc), _vp(scratch), nbytes,
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st, _host(perm)[:e], _host(colors)[:e], _host(offs)[: bc.value + 1], bc.value


def color_host(n, ci, cj, order=REF):
    L = N.load()
    e = len(ci)
    ci = np.ascontiguousarray(ci, np.uint32)
    cj = np.ascontiguousarray(cj, np.uint32)
    perm = np.zeros(max(e, 1), np.uint32)
    offs = np.zeros(e + 2, np.uint32)
    bc = C.c_uint32()
    st = L.xpbd_color_constraints(n, e, ci.ctypes.data, cj.ctypes.data, order, perm.ctypes.data, offs.ctypes.data,
                                  C.byref(bc))
    assert st == 0
    return perm[:e], offs[: bc.value + 1], bc.value


def check_coloring(n, ci, cj, order=REF):
    """Both schedules — over the whole grid, and the graph as one cloth of its own CTA — against host and oracle."""
    hperm, hoffs, hnb = color_host(n, ci, cj, order)
    operm, ocolors, ooffs = orc.partition(n, ci, cj, order == INDEX)
    for cloths in (None, [0, len(ci)]):
        st, perm, colors, offs, nb = color_device(n, ci, cj, order, cloths)
        assert st == 0
        assert nb == hnb == len(ooffs) - 1
        assert np.array_equal(perm, hperm) and np.array_equal(perm, operm)
        assert np.array_equal(offs, hoffs) and np.array_equal(offs, ooffs)
        assert np.array_equal(colors[perm], ocolors)
    return hnb


@pytest.mark.parametrize("side", [2, 3, 32, 256])
def test_sheet_coloring_matches_oracle(side):
    ci, cj, _ = wl.sheet_constraints(side)
    nb = check_coloring(side * side, ci, cj)
    assert nb >= 1


def test_index_order_coloring_matches_oracle():
    ci, cj, _ = wl.sheet_constraints(48)
    check_coloring(48 * 48, ci, cj, INDEX)


def test_hanging_grid_coloring_matches_oracle():
    mesh = M.grid_cloth_hanging(20, 30, 0.05)
    # the built mesh holds its constraints in batch order already; recolor a shuffled copy of them
    rng = np.random.default_rng(5)
    p = rng.permutation(len(mesh.constraint_i))
    check_coloring(mesh.num_particles, mesh.constraint_i[p], mesh.constraint_j[p])


@pytest.mark.parametrize("per_cloth", [False, True], ids=["grid", "cta_per_cloth"])
def test_batch_coloring_equals_per_cloth_coloring(per_cloth):
    specs = wl.config3_batch()[:24]
    offs_v = np.cumsum([0] + [s.num_particles for s in specs])
    ci = np.concatenate([s.constraint_i + o for s, o in zip(specs, offs_v)]).astype(np.uint32)
    cj = np.concatenate([s.constraint_j + o for s, o in zip(specs, offs_v)]).astype(np.uint32)
    eoff = np.cumsum([0] + [s.num_constraints for s in specs])
    st, perm, colors, offs, nb = color_device(int(offs_v[-1]), ci, cj, cloths=list(eoff) if per_cloth else None)
    assert st == 0
    for k, s in enumerate(specs):
        operm, ocolors, _ = orc.partition(s.num_particles, s.constraint_i, s.constraint_j)
        mine = colors[eoff[k]:eoff[k + 1]]
        assert np.array_equal(mine[operm], ocolors), f"cloth {k}"
    # perm is color-major across the batch, (color, global index) inside a color
    key = colors[perm].astype(np.uint64) << np.uint64(32) | perm.astype(np.uint64)
    assert np.all(np.diff(key) > 0)
    assert np.array_equal(offs, np.searchsorted(colors[perm], np.arange(nb + 1), side="left"))


def test_random_graphs_with_repeats_and_hubs():
    rng = np.random.default_rng(7)
    for trial in range(6):
        n = int(rng.integers(2, 400))
        e = int(rng.integers(1, 3000))
        ci = rng.integers(0, n, e).astype(np.uint32)
        cj = rng.integers(0, n, e).astype(np.uint32)
        cj = np.where(cj == ci, (ci + 1) % n, cj).astype(np.uint32)
        if trial % 2 == 0:  # a hub at particle 0 with more than 64 constraints: colors beyond one 64-bit window
            m = min(e, 150)
            ci[:m] = 0
            cj[:m] = np.maximum(cj[:m], 1)
        check_coloring(n, ci, cj)


def test_coloring_edge_cases():
    st, perm, colors, offs, nb = color_device(5, np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert st == 0 and nb == 1 and list(offs) == [0, 0]
    st, *_ = color_device(4, np.array([0, 1], np.uint32), np.array([1, 4], np.uint32))
    assert st == N.ERR_INDEX_RANGE
    st, *_ = color_device(4, np.array([0, 2], np.uint32), np.array([1, 2], np.uint32))
    assert st == N.ERR_INDEX_RANGE
    # too little scratch is refused before any work
    import torch
    L = N.load()
    ci, cj = _dev(torch, [0]), _dev(torch, [1])
    perm = torch.empty(1, dtype=torch.int32, device="cuda")
    offs = torch.empty(2, dtype=torch.int32, device="cuda")
    scratch = torch.empty(256, dtype=torch.uint8, device="cuda")
    bc = C.c_uint32()
    assert L.xpbd_color_constraints_device(2, 1, _vp(ci), _vp(cj), REF, 0, None, _vp(perm), None, _vp(offs),
                                           C.byref(bc), _vp(scratch), 256, None) == N.ERR_INVALID_ARGUMENT
    # cloth ranges that do not cover the constraints, or that decrease, are refused
    ci3, cj3 = np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32)
    assert color_device(4, ci3, cj3, cloths=[0, 2])[0] == N.ERR_INVALID_ARGUMENT
    assert color_device(4, ci3, cj3, cloths=[0, 2, 1, 3])[0] == N.ERR_INVALID_ARGUMENT
    # two "cloths" that share particle 1 (and 2): refused, nothing colored out of range
    assert color_device(4, ci3, cj3, cloths=[0, 1, 3])[0] == N.ERR_INVALID_ARGUMENT
    # the same constraints as one cloth are fine
    assert color_device(4, ci3, cj3, cloths=[0, 3])[0] == 0


def neighbor_table_device(n, ci, cj):
    import torch
    L = N.load()
    e = len(ci)
    dci, dcj = _dev(torch, ci), _dev(torch, cj)
    row = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    other = torch.empty(max(2 * e, 1), dtype=torch.int32, device="cuda")
    eid = torch.empty(max(2 * e, 1), dtype=torch.int32, device="cuda")
    nbytes = L.xpbd_neighbor_table_device_scratch_bytes(n, e)
    scratch = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    st = L.xpbd_neighbor_table_device(n, e, _vp(dci), _vp(dcj), _vp(row), _vp(other), _vp(eid), _vp(scratch),
                                      nbytes, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st, _host(row), _host(other)[: 2 * e], _host(eid)[: 2 * e]


@pytest.mark.parametrize("side", [3, 64, 300])
def test_neighbor_table_matches_oracle(side):
    ci, cj, _ = wl.sheet_constraints(side)
    n = side * side
    perm, _, _ = orc.partition(n, ci, cj)
    si, sj = ci[perm].astype(np.uint32), cj[perm].astype(np.uint32)
    st, row, other, eid = neighbor_table_device(n, si, sj)
    assert st == 0
    oo, ooth, oeid = orc.build_csr(n, si, sj)
    assert np.array_equal(row, oo) and np.array_equal(other, ooth) and np.array_equal(eid, oeid)


def test_neighbor_table_random_and_edge_cases():
    rng = np.random.default_rng(3)
    n, e = 1000, 5000
    ci = rng.integers(0, n, e).astype(np.uint32)
    cj = rng.integers(0, n, e).astype(np.uint32)
    st, row, other, eid = neighbor_table_device(n, ci, cj)
    assert st == 0
    oo, ooth, oeid = orc.build_csr(n, ci, cj)
    assert np.array_equal(row, oo) and np.array_equal(other, ooth) and np.array_equal(eid, oeid)
    st, row, _, _ = neighbor_table_device(7, np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert st == 0 and not row.any()
    st, *_ = neighbor_table_device(3, np.array([0], np.uint32), np.array([3], np.uint32))
    assert st == N.ERR_INDEX_RANGE
