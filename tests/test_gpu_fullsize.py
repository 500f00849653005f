"""Parity at the benchmark configurations' full sizes, and on the reference's own input fixture.

Every comparison is bit for bit against the CPU oracle (the FP32 restatement of src/xpbd_cpu.rs); the 1e-5 x rest
edge bar is asserted as well. The oracle runs on its OpenMP build here (bit-identical to the serial build,
tests/test_oracle_omp_cpu.py) so that the full sizes finish in seconds.

  * assets/cloth.obj (tests/golden/cloth.obj) parsed by parse_welded_obj, stepped with ClothSimUniforms::default()
    (36 substeps x 22 iterations, omega 0.32 / 1.0, drag 1.25) for two frames on both solvers, and one frame with the
    reference's self collision (xpbd_frame_with_self_collision, xpbd_cpu.rs:646-722).
  * 256x256 sheet, colored Gauss-Seidel, damping 0.01, 10 x 10, 120 frames (positions and velocities); the error
    of both against the FP64 oracle is recorded.
  * 256 seeded cloths of 16..192 vertices a side, plain Jacobi with degree-averaged corrections, two frames, every
    cloth against its own oracle run.
  * 512x512 sheet with self collision (2 mm thickness, 4 mm hash cells, 2^20 table, 2-ring filter, ground plane):
    hash keys, stable sorted order and pair list at a folded state lying on the ground whose layers are in contact,
    then 20 frames of the contact-heavy trajectory (about 1e5 colliding pairs throughout).
"""
import os

import numpy as np
import pytest

from bevy_xpbd_b200 import mesh as M
from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import folded_state, gpu_sim, max_abs, oracle_sim, params_for

pytestmark = pytest.mark.gpu

GOLDEN_OBJ = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cloth.obj")


def _cfg(**kw):
    c = P.ClothSimConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("solver,frames,collision", [
    (P.SOLVER_JACOBI, 2, P.COLLISION_NONE), (P.SOLVER_GAUSS_SEIDEL, 2, P.COLLISION_NONE),
    (P.SOLVER_JACOBI, 1, P.COLLISION_REST_FILTER), (P.SOLVER_GAUSS_SEIDEL, 1, P.COLLISION_REST_FILTER)],
    ids=["jacobi", "gauss_seidel", "jacobi_self_collision", "gauss_seidel_self_collision"])
def test_reference_cloth_obj_default_uniforms_bit_exact(solver, frames, collision):
    with open(GOLDEN_OBJ) as f:
        mesh = M.parse_welded_obj(f.read())
    assert mesh.num_particles == 651
    u = P.ClothSimUniforms(solver=solver)
    prm = u.substep_params()
    prm.grab_active = False
    cfg = _cfg(solver=solver, solve_substeps=P.SUBSTEPS, collision=collision, thickness=u.thickness,
               coll_scale=u.coll_scale, hash_cell=u.thickness)
    plug = P.ClothComputePlugin(0)
    plug.add_mesh(mesh)
    plug.commit()
    plug.set_params(prm, cfg)
    plug.step(frames=frames)
    s = orc.OracleSim(mesh.positions, mesh.inv_mass, mesh.constraint_i, mesh.constraint_j, mesh.constraint_rest_len,
                      mesh.constraint_compliance, rest_pos=mesh.rest_positions)
    d = prm.as_dict()
    d.update(grab_active=0, solver=solver, collision=collision, thickness=u.thickness, coll_scale=u.coll_scale,
             hash_cell=u.thickness)
    s.set_params(d)
    s.substeps(P.SUBSTEPS * frames, brute_force=True)
    xg = plug.positions()
    xo, vo = s.state()
    assert np.all(np.isfinite(xg))
    assert max_abs(xg, xo) <= 1e-5 * 0.05
    assert max_abs(xg, xo) == 0.0
    assert max_abs(plug.velocities(), vo) == 0.0
    # the hanging sheet settles under gravity (it starts close to rest: tens of microns in two frames); the pinned
    # top row does not move
    moved = np.linalg.norm(xg - mesh.positions, axis=1)
    assert moved[mesh.inv_mass > 0].max() > 5e-6 and moved[mesh.inv_mass == 0].max() == 0.0


def test_config1_full_size_gauss_seidel_120_frames_bit_exact(record_property):
    sp = wl.config1_sheet()
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=120)
    xg, vg = plug.positions(), plug.velocities()
    o = oracle_sim(sp, prm, cfg, omp=True)
    o.substeps(1200)
    xo, vo = o.state()
    d = max_abs(xg, xo)
    record_property("max_abs_gpu_vs_fp32", d)
    o64 = oracle_sim(sp, prm, cfg, fp64=True, omp=True)
    o64.substeps(1200)
    x64, _ = o64.state()
    record_property("max_abs_gpu_vs_fp64", max_abs(xg, x64))
    record_property("max_abs_fp32_vs_fp64", max_abs(xo, x64))
    assert d <= 1e-5 * float(sp.rest_len[0])
    assert d == 0.0 and max_abs(vg, vo) == 0.0
    assert np.array_equal(xg[sp.inv_mass == 0], sp.positions[sp.inv_mass == 0])


@pytest.fixture(scope="module")
def c3_batch():
    return wl.config3_batch()


def test_config3_full_batch_two_frames_bit_exact(c3_batch, record_property):
    specs = c3_batch
    assert len(specs) == 256
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    plug = gpu_sim(specs, prm, cfg)
    record_property("solver_kernel", plug.stats()["solver_kernel"])
    plug.step(frames=2)
    worst = 0.0
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg, omp=True)
        o.substeps(20)
        xo, vo = o.state()
        d = max_abs(plug.positions(k), xo)
        worst = max(worst, d, max_abs(plug.velocities(k), vo))
        assert d == 0.0, k
    record_property("max_abs_worst_cloth", worst)
    assert worst == 0.0


def test_config2_full_sheet_folded_keys_sort_pairs_and_20_contact_frames(record_property):
    sp = wl.config2_sheet()
    assert sp.num_particles == 512 * 512
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
               collision=P.COLLISION_RING_FILTER, thickness=0.002, coll_scale=0.38, hash_cell=0.004,
               hash_table_bits=20, ring_depth=2, ground_enabled=True, ground_y=0.0)
    plug = gpu_sim(sp, prm, cfg)
    # folded in half and lying on the ground: the lower half 1 mm above the plane, the upper half 1.5 mm above it
    # (closer than the 2 mm thickness everywhere); gravity keeps pressing the layers together, so contacts persist
    xf = folded_state(sp, gap=0.0015)
    xf[:, 1] -= np.float32(0.999)
    vf = np.zeros_like(xf)
    plug.write_state(xf, vf)
    x = plug.positions()
    assert np.array_equal(x, xf)
    keys, skeys, svals = plug.collision_keys()
    inv_cell = float(np.float32(1.0) / np.float32(cfg.hash_cell))
    okeys = orc.hash_keys(x, inv_cell, cfg.hash_table_bits)
    assert np.array_equal(keys, okeys)
    ok, ov = orc.stable_radix_sort(okeys, np.arange(len(okeys), dtype=np.uint32), 4)
    assert np.array_equal(skeys, ok) and np.array_equal(svals, ov)
    o = oracle_sim(sp, prm, cfg, omp=True)
    o.set_state(xf, vf)
    pairs = plug.collision_pairs()
    opairs = o.collision_pairs()
    record_property("pairs_folded", int(len(pairs)))
    assert len(pairs) > 100_000
    assert np.array_equal(pairs, opairs)
    for chunk in range(4):  # 20 frames, compared every 5
        plug.step(frames=5)
        o.substeps(50)
        xo, vo = o.state()
        assert max_abs(plug.positions(), xo) == 0.0, chunk
        assert max_abs(plug.velocities(), vo) == 0.0, chunk
    still = plug.collision_pairs()
    record_property("pairs_after_20_frames", int(len(still)))
    assert len(still) > 10_000
    assert np.array_equal(still, o.collision_pairs())
