"""CPU-only checks of the product's host side: the C-ABI library loads and exports every declared symbol, the host
coloring is bit-identical to the restated reference coloring, and the workload generators have the documented
shapes. No CUDA device is used."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from bevy_xpbd_b200 import _native as N
from bevy_xpbd_b200 import workloads as wl
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "xpbd_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xpbd_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = N.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(N.EXPORTED) == names


def color(n, ci, cj, order=0):
    L = N.load()
    ci = np.ascontiguousarray(ci, np.uint32)
    cj = np.ascontiguousarray(cj, np.uint32)
    perm = np.zeros(len(ci), np.uint32)
    offs = np.zeros(len(ci) + 2, np.uint32)
    nb = C.c_uint32()
    st = L.xpbd_color_constraints(n, len(ci), ci.ctypes.data_as(C.c_void_p), cj.ctypes.data_as(C.c_void_p), order,
                                  perm.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), C.byref(nb))
    assert st == 0
    return perm, offs[: nb.value + 1]


def _random_graph(seed, n=400, e=2500):
    rng = np.random.default_rng(seed)
    ci = rng.integers(0, n, e)
    cj = rng.integers(0, n, e)
    keep = ci != cj
    return n, ci[keep].astype(np.uint32), cj[keep].astype(np.uint32)


CASES = {
    "sheet32": lambda: (32 * 32,) + wl.sheet_constraints(32)[:2],
    "sheet77": lambda: (77 * 77,) + wl.sheet_constraints(77)[:2],
    "hanging16": lambda: (lambda m: (m.num_particles, m.constraint_i, m.constraint_j))(
        orc.grid_cloth_hanging(16, 16, 0.045)),
    "random_multigraph": lambda: _random_graph(7),
    "dense_star": lambda: (70, np.zeros(69, np.uint32), np.arange(1, 70, dtype=np.uint32)),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("order", [0, 1], ids=["reference_order", "index_order"])
def test_host_coloring_bit_exact_vs_reference(case, order):
    """partition_constraints_for_gs_batches (mesh_prep.rs:153-221): identical permutation and batch offsets."""
    n, ci, cj = CASES[case]()
    perm, offs = color(n, ci, cj, order)
    operm, _, ooffs = orc.partition(n, ci, cj, order_by_index=bool(order))
    assert np.array_equal(perm, operm)
    assert np.array_equal(offs, ooffs)


def test_coloring_is_valid_edge_coloring():
    n, ci, cj = _random_graph(3)
    perm, offs = color(n, ci, cj)
    for b in range(len(offs) - 1):
        seg = perm[offs[b]:offs[b + 1]]
        v = np.concatenate([ci[seg], cj[seg]])
        assert len(np.unique(v)) == len(v)


def test_color_constraints_rejects_bad_indices():
    L = N.load()
    ci = np.array([0, 5], np.uint32)
    cj = np.array([1, 1], np.uint32)
    perm = np.zeros(2, np.uint32)
    offs = np.zeros(3, np.uint32)
    nb = C.c_uint32()
    st = L.xpbd_color_constraints(3, 2, ci.ctypes.data_as(C.c_void_p), cj.ctypes.data_as(C.c_void_p), 0,
                                  perm.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), C.byref(nb))
    assert st == N.ERR_INDEX_RANGE


def test_device_coloring_validates_cloth_ranges_before_any_device_work():
    """The GPU coloring checks its host arguments first: cloth ranges that do not start at 0, do not end at the
    constraint count, or decrease are refused before any CUDA call (the device pointers are never touched)."""
    L = N.load()
    fake = C.c_void_p(0x1000)  # never dereferenced: the call returns before using it
    nb = C.c_uint32()
    n, e = 10, 6
    for bad in ([0, 4], [1, 3, 6], [0, 4, 3, 6], [0, 7]):
        offs = np.array(bad, np.uint32)
        st = L.xpbd_color_constraints_device(n, e, fake, fake, 0, len(bad) - 1, offs.ctypes.data, fake, None, fake,
                                             C.byref(nb), fake, 1 << 30, None)
        assert st == N.ERR_INVALID_ARGUMENT, bad
    st = L.xpbd_color_constraints_device(n, e, fake, fake, 7, 0, None, fake, None, fake, C.byref(nb), fake, 1 << 30,
                                         None)
    assert st == N.ERR_INVALID_ARGUMENT  # unknown order
    # scratch grows with the constraints and (a little) with the cloth count
    a = L.xpbd_color_constraints_device_scratch_bytes(1000, 5000, 0)
    b = L.xpbd_color_constraints_device_scratch_bytes(1000, 5000, 100)
    assert 5000 * 48 < a < b


@pytest.mark.parametrize("s", [3, 4, 16, 32, 256])
def test_sheet_constraint_count(s):
    ci, cj, ct = wl.sheet_constraints(s)
    assert len(ci) == 6 * s * s - 10 * s + 2
    assert np.all(ci != cj)
    assert (ct == 0).sum() == 2 * s * (s - 1) and (ct == 1).sum() == 2 * (s - 1) ** 2


def test_sheet_geometry_and_pins():
    sp = wl.config0_sheet()
    assert sp.num_particles == 1024 and sp.num_constraints == 5826
    assert np.isclose(sp.rest_len[0], 1.0 / 31.0, rtol=1e-6)
    assert (sp.inv_mass == 0).sum() == 2 and np.all(sp.inv_mass[sp.inv_mass > 0] == 100.0)
    assert np.max(np.abs(sp.positions - sp.rest_positions)) <= 1e-3 + 1e-7
    top = wl.config1_sheet()
    assert (top.inv_mass == 0).sum() == 256 and top.num_constraints == 390658


def test_batch_generator_is_seeded():
    a = wl.config3_batch(seed=5, count=8)
    b = wl.config3_batch(seed=5, count=8)
    assert [c.side for c in a] == [c.side for c in b]
    assert all(np.array_equal(x.positions, y.positions) for x, y in zip(a, b))
    assert all(16 <= c.side <= 192 for c in a)


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "bevy_xpbd_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "from oracle" not in text and "xpbd_oracle" not in text, f


def test_bench_reports_committed_traffic_only_for_the_full_launch():
    """The committed ncu traffic per launch is of the full single-GPU workload: a sample of c3's cloths or a rank's
    shard of them launches less work and must not be reported with it; single-sheet replicas launch the same."""
    import bench
    assert bench.make_workload("c3", 0, 1)["full_launch"]
    assert not bench.make_workload("c3", 0, 1, c3_cloths=8)["full_launch"]
    assert not bench.make_workload("c3", 1, 2)["full_launch"]
    assert bench.make_workload("c0", 1, 2)["full_launch"]


def test_sort_entry_points_refuse_overlap_and_oversize_before_touching_the_device():
    """Argument checks of both sort entry points run on the host before any CUDA call (no device here): overlapping
    output arrays, and more keys than the stated maximums."""
    L = N.load()
    n = 1000
    base = 1 << 40  # fake device addresses: never dereferenced, the checks return first
    ki, vi, ko, vo = base, base + 4 * n, base + 8 * n, base + 12 * n
    big = L.xpbd_radix_sort_scratch_bytes(n)
    assert big > 0
    P = C.c_void_p
    for a, b, c, d in [(ki, vi, ko, ko), (ki, vi, ki, vo), (ki, vi, vi, vo), (ki, vi, ko, ki), (ki, vi, ko, vi),
                       (ki, vi, ko, ko + 4 * n - 4), (ki, vi, vi - 4, vo)]:
        assert L.xpbd_radix_sort_pairs(P(a), P(b), P(c), P(d), n, 4, P(base + (1 << 30)), big, None) == \
            N.ERR_INVALID_ARGUMENT
        assert L.xpbd_radix_sort_pairs_noalloc(P(a), P(b), P(c), P(d), n, 4, None) == N.ERR_INVALID_ARGUMENT
    assert L.xpbd_radix_sort_scratch_bytes((1 << 31) + 1) == 0
    far = [base + k * (1 << 36) for k in range(4)]  # disjoint for any n below 2^34
    assert L.xpbd_radix_sort_pairs(*map(P, far), (1 << 31) + 1, 4, P(base), 1 << 40, None) == -9
    assert L.xpbd_radix_sort_pairs_noalloc(*map(P, far), (1 << 18) + 1, 4, None) == -9
