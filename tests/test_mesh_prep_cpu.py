"""The schedule of the GPU coloring (xpbd_color_constraints_device), emulated on the CPU, against the oracle's
partition_constraints_for_gs_batches (mesh_prep.rs:153-221).

The device colors constraints in Jones–Plassmann rounds whose priority is the reference's processing rank: a
constraint is colored, with the smallest color its earlier-ranked neighbours leave free, once all of them are colored.
This file checks that claim in plain Python on small graphs — the same colors as the sequential greedy — and that the
number of rounds grows with a sheet's side, not with its area.
"""
import numpy as np
import pytest

from bevy_xpbd_b200 import workloads as wl
from oracle import oracle as orc


def processing_rank(n, ci, cj):
    """Rank in the order (max endpoint degree desc, min endpoint, max endpoint, index) — mesh_prep.rs:172-177."""
    deg = np.bincount(ci, minlength=n) + np.bincount(cj, minlength=n)
    d = np.maximum(deg[ci], deg[cj])
    order = np.lexsort((np.arange(len(ci)), np.maximum(ci, cj), np.minimum(ci, cj), -d))
    rank = np.empty(len(ci), np.int64)
    rank[order] = np.arange(len(ci))
    return rank


def jones_plassmann(n, ci, cj):
    """Round-by-round emulation of the device kernel: (colors per input constraint, rounds)."""
    e = len(ci)
    rank = processing_rank(n, ci, cj)
    rows = [[] for _ in range(n)]
    for k in range(e):
        rows[ci[k]].append(k)
        rows[cj[k]].append(k)
    slots = [[f for p in (ci[k], cj[k]) for f in rows[p] if f != k] for k in range(e)]
    pending = [sum(rank[f] < rank[k] for f in slots[k]) for k in range(e)]
    color = [-1] * e
    frontier = [k for k in range(e) if pending[k] == 0]
    rounds = 0
    while frontier:
        rounds += 1
        nxt = []
        for k in frontier:
            used = {color[f] for f in slots[k] if rank[f] < rank[k]}
            assert -1 not in used
            c = 0
            while c in used:
                c += 1
            color[k] = c
        for k in frontier:
            for f in slots[k]:
                if rank[f] > rank[k]:
                    pending[f] -= 1
                    if pending[f] == 0:
                        nxt.append(f)
        frontier = nxt
    assert min(color) >= 0
    return np.array(color, np.uint32), rounds


def _check(n, ci, cj):
    colors, rounds = jones_plassmann(n, ci, cj)
    perm, ocolors, offs = orc.partition(n, ci, cj)
    assert np.array_equal(colors[perm], ocolors)
    # (color, index) order is a stable sort by color
    assert np.array_equal(np.argsort(colors, kind="stable"), perm)
    return rounds


@pytest.mark.parametrize("side", [2, 5, 12])
def test_schedule_colors_sheets_like_the_greedy(side):
    ci, cj, _ = wl.sheet_constraints(side)
    _check(side * side, ci.astype(np.int64), cj.astype(np.int64))


def test_schedule_colors_random_graphs_like_the_greedy():
    rng = np.random.default_rng(17)
    for _ in range(8):
        n = int(rng.integers(2, 60))
        e = int(rng.integers(1, 300))
        ci = rng.integers(0, n, e)
        cj = rng.integers(0, n, e)
        cj = np.where(cj == ci, (ci + 1) % n, cj)
        _check(n, ci, cj)


def test_rounds_grow_with_the_side():
    r = []
    for side in (8, 16):
        ci, cj, _ = wl.sheet_constraints(side)
        r.append(_check(side * side, ci.astype(np.int64), cj.astype(np.int64)))
    # about 10 rounds per vertex of the side: doubling the side doubles the rounds, not quadruples them
    assert r[1] < 3 * r[0]
