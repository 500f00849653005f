"""Vertex-normal oracle (cloth_sim_jacobi.wgsl:492-547) on hand-computed cases, and the sheet triangulation."""
import numpy as np

from bevy_xpbd_b200 import workloads as wl
from oracle import normals_oracle as NO


def test_flat_sheet_normals_point_up():
    s = 5
    sp = wl.make_sheet(s, 1.0, 1.0, "none", jitter=0.0, seed=0)
    n = NO.vertex_normals(sp.positions, wl.sheet_triangles(s))
    np.testing.assert_allclose(n, np.tile([0.0, 1.0, 0.0], (s * s, 1)), atol=1e-6)


def test_fixed_point_truncation_and_isolated_vertex():
    # one triangle with cross product (0, 0, 0.5): 0.5 * 33333 = 16666.5 -> 16666 -> 16666 / 33333
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [5, 5, 5]], np.float32)
    n = NO.vertex_normals(x, [[0, 1, 2]])
    assert np.array_equal(n[:3], np.tile(np.float32([0, 0, 1]), (3, 1)))
    assert np.array_equal(n[3], np.float32([0, 1, 0]))          # no triangle: the reference's fallback
    q = NO._fixed(np.float32([0.5, -0.5, 1e30, np.nan]))
    assert list(q) == [16666, -16666, 2**31 - 1, 0]


def test_sheet_triangles_cover_each_quad_once():
    t = wl.sheet_triangles(4)
    assert t.shape == (2 * 9, 3)
    assert t.max() == 15 and len({tuple(sorted(r)) for r in t}) == 18
