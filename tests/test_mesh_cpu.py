"""The product's cloth mesh builders (bevy_xpbd_b200.mesh over the C ABI, host code) against the oracle's
restatement of src/mesh_prep.rs, array for array and bit for bit: grid_cloth_hanging, parse_welded_obj (synthetic OBJ
texts: a Blender-style quad grid, fans, odd index tokens), finalize_cloth_mesh with extra constraints."""
import numpy as np
import pytest

from bevy_xpbd_b200 import mesh as M
from oracle import oracle as orc

FIELDS = ["positions", "inv_mass", "indices", "constraint_i", "constraint_j", "constraint_rest_len",
          "constraint_compliance", "constraint_batch_offsets"]


def _same(a, b):
    for f in FIELDS:
        x, y = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
        assert x.shape == y.shape, f
        assert np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                              y.view(np.uint32) if y.dtype == np.float32 else y), f


@pytest.mark.parametrize("cols,rows,cell", [(16, 16, 0.045), (24, 18, 0.045), (1, 1, 0.5), (7, 3, 0.1)])
def test_grid_cloth_hanging_matches_oracle(cols, rows, cell):
    _same(M.grid_cloth_hanging(cols, rows, cell), orc.grid_cloth_hanging(cols, rows, cell))


def _quad_grid_obj(cols, rows, h, seed=0):
    """A Blender-style export of a cols × rows vertex grid in XY: v / vt lines, quads with v/vt corners."""
    rng = np.random.default_rng(seed)
    lines = ["# synthetic grid"]
    for r in range(rows):
        for c in range(cols):
            lines.append(f"v {c * h - 0.5:.6f} {r * h:.6f} {rng.uniform(-1e-3, 1e-3):.6f}")
    for r in range(rows):
        for c in range(cols):
            lines.append(f"vt {c / (cols - 1):.4f} {r / (rows - 1):.4f}")
    for r in range(rows - 1):
        for c in range(cols - 1):
            a = r * cols + c + 1
            b, cc, d = a + 1, a + cols + 1, a + cols
            lines.append(f"f {a}/{a} {b}/{b} {cc}/{cc} {d}/{d}")
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("text", [
    _quad_grid_obj(21, 31, 0.05),
    _quad_grid_obj(5, 4, 0.1, seed=2),
    "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nf 1/1 2/2 3/3\n",
    # pentagon fan, a quad with different uv corners (unwelded), an index token with '+', a too-short face
    "v 0 0 0\nv 1 0 0\nv 1.5 1 0\nv 0.5 1.6 0\nv -0.5 1 0\nv 2 2 1\nvt 0 0\nvt 1 1\n"
    "f 1 2 3 4 5\nf 2/1 6/2 3/1 +3/2\nf 1 2\n# comment\n   \nf 4/1/1 5/2/1 6\n",
])
def test_parse_welded_obj_matches_oracle(text):
    _same(M.parse_welded_obj(text), orc.parse_welded_obj(text))


def test_finalize_with_extras_and_pins():
    m0 = M.grid_cloth_hanging(6, 5, 0.1)
    extras = [(0, 14, 0.3, 1e-6), (3, 20, 0.25, 0.0)]
    m = M.finalize_cloth_mesh(m0.positions, m0.indices, extras)
    assert m.constraint_batch_offsets[-1] == len(m.constraint_i)
    top = m.positions[:, 1].max()
    assert np.array_equal(m.inv_mass == 0, m.positions[:, 1] >= top - np.float32(1e-5))
    pairs = {(int(i), int(j)) for i, j in zip(m.constraint_i, m.constraint_j)}
    assert (0, 14) in pairs and (3, 20) in pairs
    # batches are particle-disjoint (greedy coloring)
    for b in range(len(m.constraint_batch_offsets) - 1):
        s, e = m.constraint_batch_offsets[b], m.constraint_batch_offsets[b + 1]
        used = np.concatenate([m.constraint_i[s:e], m.constraint_j[s:e]])
        assert len(np.unique(used)) == len(used)


def test_mesh_input_errors():
    with pytest.raises(Exception):
        M.grid_cloth_hanging(0, 3, 0.1)
    with pytest.raises(Exception):
        M.finalize_cloth_mesh(np.zeros((3, 3)), [[0, 1, 5]])
