"""Parity of the CUDA path (through the C ABI) with the CPU oracle of xpbd_cpu.rs on the same seeded inputs.

Tolerance: positions after the stated frames must satisfy max |Δx| <= 1e-5 × rest edge length (the stated bar); the
kernels mirror the FP32 operation order of the reference, so the observed difference is 0 (bit-exact) and the
tests assert that too. Integer outputs (coloring, hash keys, sorted order, pair lists) must be identical.
"""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import folded_state, gpu_sim, max_abs, oracle_sim, params_for

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    c = P.ClothSimConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def test_config0_jacobi_120_frames_bit_exact(record_property):
    """32x32 sheet, plain Jacobi with degree-averaged corrections, 10x10, 120 frames vs the FP32 oracle; the error of
    both against the FP64 oracle is recorded."""
    sp = wl.config0_sheet()
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=120)
    xg = plug.positions()
    o32 = oracle_sim(sp, prm, cfg)
    o32.substeps(1200)
    x32, _ = o32.state()
    o64 = oracle_sim(sp, prm, cfg, fp64=True)
    o64.substeps(1200)
    x64, _ = o64.state()
    rest_edge = float(sp.rest_len[0])
    d = max_abs(xg, x32)
    record_property("max_abs_gpu_vs_fp32", d)
    record_property("max_abs_gpu_vs_fp64", max_abs(xg, x64))
    record_property("max_abs_fp32_vs_fp64", max_abs(x32, x64))
    assert d <= 1e-5 * rest_edge
    assert d == 0.0
    assert np.all(np.isfinite(xg))
    # pinned corners did not move
    assert np.array_equal(xg[sp.inv_mass == 0], sp.positions[sp.inv_mass == 0])


def _hanging_mesh_gpu_and_oracle(solver, frames=1, collision=0):
    m = orc.grid_cloth_hanging(16, 16, 0.045)
    u = P.ClothSimUniforms(solver=solver)
    prm = u.substep_params()
    prm.grab_active = False
    cfg = _cfg(solver=solver, solve_substeps=P.SUBSTEPS, collision=collision, thickness=0.04, coll_scale=0.38,
               hash_cell=0.04)
    plug = P.ClothComputePlugin(0)
    plug.add_cloth(m.positions, m.inv_mass, m.constraint_i, m.constraint_j, m.constraint_rest_len,
                   m.constraint_compliance, rest_positions=m.rest_positions, order=P.ORDER_PRESORTED,
                   batch_offsets=m.constraint_batch_offsets)
    plug.commit()
    plug.set_params(prm, cfg)
    plug.step(frames=frames)
    s = orc.OracleSim(m.positions, m.inv_mass, m.constraint_i, m.constraint_j, m.constraint_rest_len,
                      m.constraint_compliance, rest_pos=m.rest_positions)
    d = prm.as_dict()
    d.update(grab_active=0, solver=solver, collision=collision, thickness=0.04, coll_scale=0.38, hash_cell=0.04)
    s.set_params(d)
    s.substeps(P.SUBSTEPS * frames, brute_force=True)
    return m, plug.positions(), s.state()[0], plug


@pytest.mark.parametrize("solver", [P.SOLVER_JACOBI, P.SOLVER_GAUSS_SEIDEL], ids=["jacobi", "gauss_seidel"])
def test_reference_hanging_grid_defaults_bit_exact(solver):
    """grid_cloth_hanging(16,16,0.045) with ClothSimUniforms::default() (ω=0.32 Jacobi / 1.0 GS, λ cleared per inner
    iteration, 36 substeps × 22 iterations, drag 1.25), two frames, constraint order as finalize_cloth_mesh gives."""
    m, xg, xo, _ = _hanging_mesh_gpu_and_oracle(solver, frames=2)
    assert max_abs(xg, xo) == 0.0


@pytest.mark.parametrize("solver", [P.SOLVER_JACOBI, P.SOLVER_GAUSS_SEIDEL], ids=["jacobi", "gauss_seidel"])
def test_reference_hanging_grid_with_self_collision_bit_exact(solver):
    """xpbd_frame_with_self_collision (xpbd_cpu.rs:646-722; test :1075-1128): collision every substep, the GPU's
    hashed 27-cell query against the reference's all-pairs loop."""
    m, xg, xo, plug = _hanging_mesh_gpu_and_oracle(solver, frames=1, collision=P.COLLISION_REST_FILTER)
    assert np.all(np.isfinite(xg))
    assert max_abs(xg, xo) == 0.0


def test_pins_hold_and_extent_15_frames_gpu():
    """xpbd_cpu.rs:857-913 and :976-1034 through the CUDA path."""
    m = orc.grid_cloth_hanging(16, 16, 0.045)
    prm = P.ClothSimUniforms().substep_params()
    prm.grab_active = False
    plug = P.ClothComputePlugin(0)
    plug.add_cloth(m.positions, m.inv_mass, m.constraint_i, m.constraint_j, m.constraint_rest_len,
                   m.constraint_compliance, order=P.ORDER_PRESORTED, batch_offsets=m.constraint_batch_offsets)
    plug.commit()
    plug.set_params(prm, _cfg(solve_substeps=P.SUBSTEPS))
    plug.step(frames=1)
    x = plug.positions()
    pinned = m.inv_mass <= 0
    assert np.all(np.linalg.norm(x[pinned] - m.positions[pinned], axis=1) < 1e-4)
    plug.step(frames=14)
    x = plug.positions()
    ext = x[~pinned].max(0) - x[~pinned].min(0)
    assert ext[0] > 0.18 and ext[1] > 0.04


def test_gs_sheet_damped_bit_exact():
    """Colored Gauss–Seidel on a 64x64 sheet with the top edge pinned and damping 0.01 (config-1 setup, smaller)."""
    sp = wl.make_sheet(64, 2.0, 1.0, "top_edge", seed=11)
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=10)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(100)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0
    assert max_abs(plug.velocities(), o.state()[1]) == 0.0


@pytest.mark.parametrize("solver", [P.SOLVER_JACOBI, P.SOLVER_GAUSS_SEIDEL], ids=["jacobi", "gauss_seidel"])
def test_lambda_per_substep_mode_bit_exact(solver):
    """Extension mode: λ accumulated over a substep's iterations (standard XPBD), λ read back per constraint."""
    sp = wl.make_sheet(40, 1.0, 1.0, "corners", seed=4, stretch_comp=1e-7)
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=solver, relaxation=P.RELAX_AVERAGE if solver == 0 else P.RELAX_OMEGA,
               lambda_mode=P.LAMBDA_PER_SUBSTEP, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=12)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(120)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0
    perm, _, _ = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j)
    lam_o = np.empty(sp.num_constraints)
    lam_o[perm] = o.lambdas()
    lam_g = plug.lambdas(0)
    both_pinned = (sp.inv_mass[sp.constraint_i] == 0) & (sp.inv_mass[sp.constraint_j] == 0)
    assert np.array_equal(lam_g[~both_pinned].astype(np.float64), lam_o[~both_pinned])


def test_batched_uneven_cloths_bit_exact():
    """Several cloths of uneven sizes packed into one launch: each equals its own oracle run."""
    specs = wl.config3_batch(seed=9, count=6, side_lo=12, side_hi=40)
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    plug = gpu_sim(specs, prm, cfg)
    plug.step(frames=8)
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        o.substeps(80)
        assert max_abs(plug.positions(k), o.state()[0]) == 0.0, k
    cfg.solver = P.SOLVER_GAUSS_SEIDEL
    cfg.relaxation = P.RELAX_OMEGA
    plug2 = gpu_sim(specs, prm, cfg)
    plug2.step(frames=5)
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        o.substeps(50)
        assert max_abs(plug2.positions(k), o.state()[0]) == 0.0, k


def test_collision_two_particle_known_answer():
    """xpbd_cpu.rs:1036-1047 through the CUDA substep (no gravity, no constraints): distance 0.015 becomes 0.01975."""
    x = np.array([[0, 0, 0], [0.015, 0, 0]], np.float32)
    rest = np.array([[0, 0, 0], [0.1, 0, 0]], np.float32)
    plug = P.ClothComputePlugin(0)
    plug.add_cloth(x, np.ones(2, np.float32), np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float32),
                   np.zeros(0, np.float32), rest_positions=rest)
    plug.commit()
    prm = params_for(1, 0, 1.0, gravity=(0.0, 0.0, 0.0))
    plug.set_params(prm, _cfg(solve_substeps=1, collision=P.COLLISION_REST_FILTER, thickness=0.04, coll_scale=0.38,
                              hash_cell=0.04))
    plug.step(frames=1)
    out = plug.positions()
    assert abs(np.linalg.norm(out[1] - out[0]) - 0.01975) < 1e-7
    ref = orc.self_collision_resolve(x, np.ones(2, np.float32), rest, 0.04, 0.38)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("offset,thickness", [((0.0, 0.0, 0.0), 0.03), ((1000.0, -37.5, 250.0), 0.03),
                                              ((-3.3, 0.7, -0.01), 0.02)])
def test_collision_cell_reach_keeps_pairs_across_faces_edges_corners(offset, thickness):
    """The 27-cell query leaves out cells beyond the narrow phase's reach. Pairs just inside the reach whose
    particles sit a hair on either side of cell faces, along face, edge and corner directions, near the origin and at
    large coordinates: the pair list equals the oracle's and one substep equals the oracle's all-pairs loop."""
    cell = 0.04
    rng = np.random.default_rng(11)
    m = 1500
    hair = rng.choice([0.0, 1e-7, 1e-6, 1e-4, 0.3 * cell], (m, 3)) * rng.choice([-1.0, 1.0], (m, 3))
    base = rng.integers(-12, 12, (m, 3)) * cell + hair
    axis = np.eye(3)[rng.integers(0, 3, m)] * rng.choice([-1.0, 1.0], (m, 1))
    edge = rng.choice([-1.0, 0.0, 1.0], (m, 3))
    edge[np.all(edge == 0, axis=1), 0] = 1.0
    rand = rng.normal(size=(m, 3))
    kind = rng.integers(0, 3, m)[:, None]
    dirs = np.where(kind == 0, axis, np.where(kind == 1, edge, rand))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    dist = thickness * (1.0 - rng.choice([1e-6, 1e-4, 1e-2, 0.3], m))
    x = (np.concatenate([base, base + dirs * dist[:, None]]) + np.asarray(offset)).astype(np.float32)
    n = len(x)
    g = np.arange(n)
    rest = np.stack([g % 64, (g // 64) % 64, g // 4096], axis=1).astype(np.float32)  # rest distances >= 1
    e0 = np.zeros(0, np.uint32)
    spec = wl.ClothSpec(x, np.ones(n, np.float32), e0, e0, np.zeros(0, np.float32), np.zeros(0, np.float32), e0,
                        rest)
    prm = params_for(1, 0, 1.0, gravity=(0.0, 0.0, 0.0))
    cfg = _cfg(solve_substeps=1, collision=P.COLLISION_REST_FILTER, thickness=thickness, coll_scale=0.38,
               hash_cell=cell)
    plug = gpu_sim(spec, prm, cfg)
    o = oracle_sim(spec, prm, cfg)
    pairs = plug.collision_pairs()
    assert len(pairs) > m // 2
    assert np.array_equal(pairs, o.collision_pairs())
    plug.step(frames=1)
    o.substeps(1, brute_force=True)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


def _folding_sheet(side=48, frames=40):
    sp = wl.config2_sheet(seed=2, side=side)
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
               collision=P.COLLISION_RING_FILTER, thickness=0.05, coll_scale=0.38, hash_cell=0.1,
               hash_table_bits=20, ring_depth=2, ground_enabled=True, ground_y=0.0)
    return sp, prm, cfg


def test_self_collision_ring_filter_trajectory_bit_exact():
    """Falling, folding sheet with ground plane and 2-ring filtered self collision: the whole trajectory matches."""
    sp, prm, cfg = _folding_sheet(40)
    plug = gpu_sim(sp, prm, cfg)
    o = oracle_sim(sp, prm, cfg)
    for _ in range(4):
        plug.step(frames=10)
        o.substeps(100)
        assert max_abs(plug.positions(), o.state()[0]) == 0.0
    assert plug.positions()[:, 1].min() >= 0.0


def test_hash_keys_sorted_order_and_pairs_bit_exact():
    """Spatial hash keys, stable 8-bit-digit LSD radix sort and the collision pair list of a folded sheet, then the
    collision-heavy trajectory from that state. The GPU sorts only the passes that cover the table's bits; the oracle
    runs all four, whose extra passes over all-zero digits leave the order unchanged."""
    sp, prm, cfg = _folding_sheet(64)
    plug = gpu_sim(sp, prm, cfg)
    xf = folded_state(sp)
    plug.write_state(xf, np.zeros_like(xf))
    x = plug.positions()
    assert np.array_equal(x, xf)
    keys, skeys, svals = plug.collision_keys()
    inv_cell = float(np.float32(1.0) / np.float32(cfg.hash_cell))
    okeys = orc.hash_keys(x, inv_cell, cfg.hash_table_bits)
    assert np.array_equal(keys, okeys)
    ok, ov = orc.stable_radix_sort(okeys, np.arange(len(okeys), dtype=np.uint32), 4)
    assert np.array_equal(skeys, ok) and np.array_equal(svals, ov)
    assert np.array_equal(svals, np.argsort(okeys, kind="stable").astype(np.uint32))
    pairs = plug.collision_pairs()
    o = oracle_sim(sp, prm, cfg)
    o.set_state(x, np.zeros_like(x))
    opairs = o.collision_pairs()
    assert len(pairs) > 1000
    assert np.array_equal(pairs, opairs)
    # trajectory with many contacts
    plug.step(frames=5)
    o.substeps(50)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


def test_radix_sort_primitive_matches_stable_argsort():
    import torch
    import ctypes as C
    from bevy_xpbd_b200 import _native as N
    L = N.load()
    rng = np.random.default_rng(0)
    # (n, key bound, passes): the 8-bit passes cover the keys' bits; 300k and 2M keys give 147 and 977 tiles, so the
    # scan over the (digit, tile) counts runs over two and eight 32768-value chunks.
    for n, hi, passes in [(1, 5, 4), (1000, 7, 1), (300_000, 1 << 20, 3), (70_001, 1 << 32, 4),
                          (2_000_000, 1 << 16, 2), (262_144, 1 << 20, 3), (131_071, 1 << 24, 3)]:
        keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
        kin = torch.from_numpy(keys.view(np.int32)).cuda()
        vin = torch.arange(n, dtype=torch.int32, device="cuda")
        kout = torch.empty_like(kin)
        vout = torch.empty_like(vin)
        nbytes = L.xpbd_radix_sort_scratch_bytes(n)
        scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        st = L.xpbd_radix_sort_pairs(C.c_void_p(kin.data_ptr()), C.c_void_p(vin.data_ptr()),
                                     C.c_void_p(kout.data_ptr()), C.c_void_p(vout.data_ptr()), n, passes,
                                     C.c_void_p(scratch.data_ptr()), nbytes,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0
        torch.cuda.synchronize()
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(vout.cpu().numpy().astype(np.int64), order)
        assert np.array_equal(kout.cpu().numpy().view(np.uint32), keys[order])


def test_substep_graph_and_autotune_do_not_change_results():
    sp = wl.make_sheet(48, 1.0, 1.0, "corners", seed=3)
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    a = gpu_sim(sp, prm, cfg)
    a.step(frames=3)
    cfg2 = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, use_graphs=False)
    b = gpu_sim(sp, prm, cfg2)
    b.substep(30)
    assert max_abs(a.positions(), b.positions()) == 0.0
    c = gpu_sim(sp, prm, cfg)
    c.autotune(frames=1)
    c.step(frames=3)
    assert max_abs(a.positions(), c.positions()) == 0.0


def test_strain_residual_matches_oracle():
    sp = wl.config0_sheet()
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=5)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(50)
    assert abs(plug.strain_residual() - o.strain_residual()) <= 1e-6 * max(1.0, o.strain_residual())


def test_full_size_config1_gauss_seidel_properties():
    """256x256 colored GS (config 1 sizes): finite, pins hold, coloring identical to the reference algorithm."""
    sp = wl.config1_sheet()
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=3)
    x = plug.positions()
    assert np.all(np.isfinite(x))
    assert np.array_equal(x[sp.inv_mass == 0], sp.positions[sp.inv_mass == 0])
    perm, offs = plug.coloring(0)
    operm, _, ooffs = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j)
    assert np.array_equal(perm, operm) and np.array_equal(offs, ooffs)


@pytest.mark.parametrize("cluster", [1, 8, 16], ids=["grid_barrier", "cluster8", "cluster16"])
def test_gauss_seidel_execution_paths_bit_exact(cluster):
    """Both Gauss–Seidel executions — the grid-wide persistent kernel and the thread-block-cluster kernel with
    the state in distributed shared memory — give the reference result, with and without a collision pass."""
    sp = wl.make_sheet(72, 2.0, 1.0, "top_edge", seed=5)
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10, cluster_ctas=cluster)
    plug = gpu_sim(sp, prm, cfg)
    st = plug.stats()
    if cluster > 1:
        assert st["grid_blocks"] == cluster
    assert st["solver_kernel"] == (3 if cluster > 1 else 1)  # the requested execution ran
    plug.step(frames=6)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(60)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0
    cfg2 = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10, cluster_ctas=cluster,
                collision=P.COLLISION_RING_FILTER, thickness=0.03, hash_cell=0.06, ground_enabled=True)
    plug2 = gpu_sim(sp, prm, cfg2)
    plug2.step(frames=4)
    o2 = oracle_sim(sp, prm, cfg2)
    o2.substeps(40)
    assert max_abs(plug2.positions(), o2.state()[0]) == 0.0


@pytest.mark.parametrize("kernel", [1, 2, 3, 4], ids=["warp_tiles", "spatial_patches", "thread_rows",
                                                     "cloth_resident"])
@pytest.mark.parametrize("lam", [P.LAMBDA_RESET_PER_ITERATION, P.LAMBDA_PER_SUBSTEP], ids=["lambda_reset", "lambda_substep"])
def test_jacobi_execution_paths_bit_exact(kernel, lam):
    """Every Jacobi execution — warp tiles over the neighbour table, shared-memory spatial patches that solve each
    constraint once, thread per particle over the incidence table — gives the reference result on a batch of uneven
    cloths, in both λ modes."""
    specs = wl.config3_batch(seed=13, count=5, side_lo=20, side_hi=70)
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, lambda_mode=lam, solve_substeps=10,
               jacobi_kernel=kernel)
    plug = gpu_sim(specs, prm, cfg)
    plug.step(frames=6)
    # the requested execution ran: kernel ids 0 warp tiles, 2 spatial patches, 5 thread per particle, 7 cloth-resident
    # (λ cleared per pass only; with λ kept over the substep the thread-per-particle kernel runs instead)
    want = {1: 0, 2: 2, 3: 5, 4: 7 if lam == P.LAMBDA_RESET_PER_ITERATION else 5}[kernel]
    assert plug.stats()["solver_kernel"] == want
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        o.substeps(60)
        assert max_abs(plug.positions(k), o.state()[0]) == 0.0, k
        if lam == P.LAMBDA_PER_SUBSTEP:
            perm, _, _ = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j)
            lam_o = np.empty(sp.num_constraints)
            lam_o[perm] = o.lambdas()
            both = (sp.inv_mass[sp.constraint_i] == 0) & (sp.inv_mass[sp.constraint_j] == 0)
            assert np.array_equal(plug.lambdas(k)[~both].astype(np.float64), lam_o[~both]), k


@pytest.mark.parametrize("where", ["pinned", "free"])
def test_row_kernel_coordinates_outside_fast_division_range_bit_exact(where):
    """The row kernel divides by a constraint's length through one shared reciprocal when every position of a pass has
    all coordinates 0 or in [2^-37, 2^58], and by the ordinary division otherwise (decided per pass on the GPU).
    Coordinates of 1e-13 on a pinned particle (every pass takes the exact path) or on free particles (the first
    passes do) give the reference result as well."""
    sp = wl.make_sheet(24, 1.0, 1.0, "corners", seed=21)
    x = sp.positions.copy()
    idx = np.flatnonzero(sp.inv_mass == 0)[:1] if where == "pinned" else np.array([30, 31, 57, 300])
    x[idx, 0] = np.float32(1e-13)
    x[idx[-1], 2] = np.float32(-3e-20)
    sp.positions = x
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=3)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=3)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(30)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


@pytest.mark.parametrize("where", ["pinned", "free"])
def test_cluster_gs_coordinates_outside_fast_division_range_bit_exact(where):
    """The cluster Gauss–Seidel kernel takes the shared-reciprocal division per constraint when its operands pass
    the range test and the ordinary division otherwise: coordinates of 1e-13 and -3e-20 give the reference result."""
    sp = wl.make_sheet(64, 2.0, 1.0, "top_edge", seed=22)
    x = sp.positions.copy()
    idx = np.flatnonzero(sp.inv_mass == 0)[:1] if where == "pinned" else np.array([700, 701, 1500, 3000])
    x[idx, 0] = np.float32(1e-13)
    x[idx[-1], 2] = np.float32(-3e-20)
    sp.positions = x
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10, cluster_ctas=16)
    plug = gpu_sim(sp, prm, cfg)
    assert plug.stats()["cluster_ctas"] == 16
    plug.step(frames=2)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(20)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


@pytest.mark.parametrize("solver,kernel,lam", [
    (P.SOLVER_JACOBI, 3, P.LAMBDA_RESET_PER_ITERATION), (P.SOLVER_JACOBI, 1, P.LAMBDA_RESET_PER_ITERATION),
    (P.SOLVER_JACOBI, 4, P.LAMBDA_RESET_PER_ITERATION), (P.SOLVER_JACOBI, 3, P.LAMBDA_PER_SUBSTEP),
    (P.SOLVER_GAUSS_SEIDEL, 0, P.LAMBDA_RESET_PER_ITERATION)],
    ids=["rows", "warp_tiles", "cloth_resident", "rows_lambda_substep", "gauss_seidel"])
def test_any_number_of_compliance_values_bit_exact(solver, kernel, lam):
    """A cloth whose every constraint has its own compliance (the reference packs an f32 compliance per constraint,
    cloth_jacobi.rs:95-111): more than the 16 values a cloth's palette names, so the incidences carry their own."""
    rng = np.random.default_rng(31)
    specs = [wl.make_sheet(36, 1.0, 1.0, "corners", seed=32), wl.make_sheet(20, 1.0, 1.0, "top_edge", seed=33)]
    specs[0].compliance = (10.0 ** rng.uniform(-9, -3, specs[0].num_constraints)).astype(np.float32)
    assert len(np.unique(specs[0].compliance)) > 16
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=solver, relaxation=P.RELAX_AVERAGE if solver == P.SOLVER_JACOBI else P.RELAX_OMEGA,
               lambda_mode=lam, solve_substeps=10, jacobi_kernel=kernel)
    plug = gpu_sim(specs, prm, cfg)
    plug.step(frames=3)
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        o.substeps(30)
        assert max_abs(plug.positions(k), o.state()[0]) == 0.0, k


@pytest.mark.parametrize("solver,kernel,cluster", [
    (P.SOLVER_JACOBI, 3, 0), (P.SOLVER_JACOBI, 5, 0), (P.SOLVER_JACOBI, 4, 0),
    (P.SOLVER_GAUSS_SEIDEL, 0, 16), (P.SOLVER_GAUSS_SEIDEL, 0, 1)],
    ids=["rows", "small_batch", "cloth_resident", "gs_cluster", "gs_grid"])
def test_tiny_inverse_mass_next_to_a_pin_bit_exact(solver, kernel, cluster):
    """A free particle of inverse mass 1e-9 beside a pinned corner: the stretch constraint between them has a w sum
    below 1e-8, which the reference skips (xpbd_cpu.rs:174-178, :369-372). Such an input also turns off the kernels'
    shortcut that assumes every free particle's inverse mass is at least 1e-8, so the general terms run."""
    sp = wl.make_sheet(24, 1.0, 1.0, "corners", seed=41)
    w = sp.inv_mass.copy()
    corner = int(np.flatnonzero(w == 0)[0])
    nbrs = np.concatenate([sp.constraint_j[sp.constraint_i == corner], sp.constraint_i[sp.constraint_j == corner]])
    heavy = int(nbrs[0])
    w[heavy] = np.float32(1e-9)
    sp.inv_mass = w
    pair = ((sp.constraint_i == corner) & (sp.constraint_j == heavy)) | \
           ((sp.constraint_i == heavy) & (sp.constraint_j == corner))
    comp = sp.compliance.copy()
    comp[pair] = 0.0
    sp.compliance = comp
    prm = params_for(10, 10, 1.0 if solver == P.SOLVER_JACOBI else 0.9)
    cfg = _cfg(solver=solver, relaxation=P.RELAX_AVERAGE if solver == P.SOLVER_JACOBI else P.RELAX_OMEGA,
               solve_substeps=10, jacobi_kernel=kernel, cluster_ctas=cluster)
    plug = gpu_sim(sp, prm, cfg)
    plug.step(frames=2)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(20)
    xo, vo = o.state()
    assert max_abs(plug.positions(), xo) == 0.0
    assert max_abs(plug.velocities(), vo) == 0.0
