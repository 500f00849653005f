"""The reference's own input fixture, assets/cloth.obj (copied to tests/golden/cloth.obj by make_golden.py), through
`parse_welded_obj` (src/mesh_prep.rs:223-357) in the product's host code (C ABI) and in the oracle.

The reference cannot be built here, so the expected structure is derived from its source:
  * the file is a 21 x 31 vertex grid of 600 quads ("v/vt/vn" corners shared between quads, so welding keeps 651
    vertices); each quad becomes the fan (v0,v1,v2) + (v0,v2,v3) -> 1,200 triangles (:314-326);
  * constraint order [triangle edges, hinge bends, extras] (:575-585): unique triangle edges 20x31 + 21x30 + 600
    diagonals = 1,850 at the stretch compliance 2e-8 (:93); one hinge bend per interior edge, 1,850 - 100 boundary
    edges = 1,750 at 3.8 (:89); skip-2 braces 31x19 + 21x29 = 1,198 at 2.5e-8 (:97); one cross diagonal v1-v3 per
    quad, 600 at 6e-9 (:101) -> 5,398;
  * every vertex at the maximum y (0.75, the top row of 21) is pinned (:558-568);
  * inverse mass = sum over incident triangles of 1/area/3 (:541-554): triangle area 0.00125 m^2, so an interior
    vertex (6 triangles) gets 6 x 266.67 = 1,600.
"""
import os

import numpy as np

from bevy_xpbd_b200 import mesh as M
from oracle import oracle as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cloth.obj")
FIELDS = ["positions", "inv_mass", "indices", "constraint_i", "constraint_j", "constraint_rest_len",
          "constraint_compliance", "constraint_batch_offsets"]


def _text():
    with open(GOLDEN) as f:
        return f.read()


def test_reference_cloth_obj_product_equals_oracle_bit_for_bit():
    a = M.parse_welded_obj(_text())
    b = orc.parse_welded_obj(_text())
    for f in FIELDS:
        x, y = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
        assert x.shape == y.shape, f
        assert np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                              y.view(np.uint32) if y.dtype == np.float32 else y), f


def test_reference_cloth_obj_structure_from_the_reference_source():
    m = M.parse_welded_obj(_text())
    assert m.num_particles == 651
    assert len(m.indices) == 3 * 1200
    top = m.positions[:, 1] == np.float32(0.75)
    assert top.sum() == 21
    assert np.array_equal(m.inv_mass == 0, top)
    assert len(m.constraint_i) == 5398
    comp, counts = np.unique(m.constraint_compliance, return_counts=True)
    by = dict(zip(comp.tolist(), counts.tolist()))
    assert by == {float(np.float32(2e-8)): 1850, float(np.float32(3.8)): 1750, float(np.float32(2.5e-8)): 1198,
                  float(np.float32(6e-9)): 600}
    # rest lengths: grid edges 0.05, diagonals / cross diagonals / bends over a diagonal sqrt(2)*0.05, skip-2 0.1,
    # bends over a grid edge sqrt(0.05^2 + 0.1^2)
    rl = np.round(m.constraint_rest_len.astype(np.float64), 5)
    vals, cnt = np.unique(rl, return_counts=True)
    assert np.allclose(vals, [0.05, 0.07071, 0.1, 0.1118], atol=1e-5)
    assert cnt.tolist() == [1250, 1800, 1198, 1150]
    # interior vertices: six triangles of area 0.00125 each
    interior = (np.abs(m.positions[:, 0]) < 0.49) & (np.abs(m.positions[:, 1]) < 0.74)
    assert interior.sum() == 19 * 29
    assert np.allclose(m.inv_mass[interior], 1600.0, rtol=1e-5)
    # greedy coloring: batches cover every constraint once and are particle-disjoint
    off = m.constraint_batch_offsets
    assert off[0] == 0 and off[-1] == 5398 and np.all(np.diff(off) > 0)
    for b in range(len(off) - 1):
        used = np.concatenate([m.constraint_i[off[b]:off[b + 1]], m.constraint_j[off[b]:off[b + 1]]])
        assert len(np.unique(used)) == len(used)
