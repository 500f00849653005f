"""Vertex normals through the C ABI against the oracle restatement of accumulate_normals + finalize_normals
(cloth_sim_jacobi.wgsl:492-547), bit-exact, on the GPU's own positions after a few frames: the reference hanging grid
(its triangle list from the mesh builder) and a jittered sheet batched in one context."""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from oracle import normals_oracle as NO
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_vertex_normals_bit_exact():
    m = orc.grid_cloth_hanging(16, 16, 0.045)
    sp = wl.make_sheet(40, 1.0, 1.0, "corners", seed=3)
    plug = P.ClothComputePlugin(0)
    plug.add_cloth(m.positions, m.inv_mass, m.constraint_i, m.constraint_j, m.constraint_rest_len,
                   m.constraint_compliance, rest_positions=m.rest_positions, order=P.ORDER_PRESORTED,
                   batch_offsets=m.constraint_batch_offsets)
    plug.add_spec(sp)
    plug.set_triangles(0, m.indices)
    plug.set_triangles(1, wl.sheet_triangles(40))
    plug.commit()
    prm = P.ClothSimUniforms().substep_params()
    prm.grab_active = False
    plug.set_params(prm, P.ClothSimConfig(solve_substeps=P.SUBSTEPS))
    for frames in (0, 3):
        if frames:
            plug.step(frames=frames)
        for cloth, tris in ((0, m.indices), (1, wl.sheet_triangles(40))):
            x = plug.positions(cloth)
            n_gpu = plug.normals(cloth)
            n_ref = NO.vertex_normals(x, tris)
            assert np.array_equal(n_gpu.view(np.uint32), n_ref.view(np.uint32)), (frames, cloth)
    assert np.all(np.abs(np.linalg.norm(n_gpu, axis=1) - 1.0) < 1e-5)
    mat = P.ClothMaterialPlugin(plug)
    assert np.array_equal(mat.render_normals(1), n_gpu)


def test_normals_need_triangles():
    sp = wl.make_sheet(8, 1.0, 1.0, "corners", seed=3)
    plug = P.ClothComputePlugin(0)
    plug.add_spec(sp)
    with pytest.raises(P.XpbdError):
        plug.set_triangles(0, [[0, 1, 64]])      # index out of range
    plug.commit()
    with pytest.raises(P.XpbdError):
        plug.normals(0)


def test_mesh_builder_to_solver_and_normals():
    """A mesh from the product's builder (grid_cloth_hanging) through add_mesh — batch order and triangles included —
    steps exactly like the oracle fed the oracle's own mesh, and its normals match the oracle's."""
    from bevy_xpbd_b200 import mesh as M
    m = M.grid_cloth_hanging(16, 16, 0.045)
    ref = orc.grid_cloth_hanging(16, 16, 0.045)
    plug = P.ClothComputePlugin(0)
    plug.add_mesh(m)
    plug.commit()
    u = P.ClothSimUniforms(solver=P.SOLVER_JACOBI)
    prm = u.substep_params()
    prm.grab_active = False
    plug.set_params(prm, P.ClothSimConfig(solver=P.SOLVER_JACOBI, solve_substeps=P.SUBSTEPS))
    plug.step(frames=2)
    s = orc.OracleSim(ref.positions, ref.inv_mass, ref.constraint_i, ref.constraint_j, ref.constraint_rest_len,
                      ref.constraint_compliance, rest_pos=ref.rest_positions)
    d = prm.as_dict()
    d.update(grab_active=0, solver=P.SOLVER_JACOBI)
    s.set_params(d)
    s.substeps(2 * P.SUBSTEPS)
    x = plug.positions(0)
    assert np.array_equal(x.astype(np.float64), s.state()[0])
    assert np.array_equal(plug.normals(0).view(np.uint32), NO.vertex_normals(x, ref.indices).view(np.uint32))
