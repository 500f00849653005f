"""The cloth-resident Jacobi kernel (jacobi_kernel 4, kernel id 7: each cloth in the shared memory of one CTA or of a
thread-block cluster for a whole frame, each constraint solved once per pass, colors summed in order) against the
CPU oracle of xpbd_cpu.rs, bit for bit: every launch class (single CTAs of 256 / 512 / 1024 threads, clusters of
2, 4, 8 and 16 CTAs), both relaxations, per-cloth grabs, no-iteration substeps, single substeps, and the fallback to the
thread-per-particle kernel when a cloth's color batches share a particle."""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from tests.helpers import gpu_sim, max_abs, oracle_sim, params_for

pytestmark = pytest.mark.gpu

CLOTH = 7  # kernel id of the cloth-resident kernel
ROWS = 5   # thread per particle


def _cfg(**kw):
    c = P.ClothSimConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


# sides whose particle counts land in every launch class: <= 1,760 / 3,520 / 7,168 particles on one CTA, then
# clusters of 2 (<= 14,336), 4 (<= 28,672), 8 (<= 57,344) and 16 (<= 65,536) CTAs
SIDES = [12, 41, 42, 59, 60, 84, 85, 119, 120, 169, 170, 239, 240, 256]


@pytest.fixture(scope="module")
def mixed_batch():
    rng = np.random.default_rng(5)
    specs = []
    for k, s in enumerate(SIDES):
        specs.append(wl.make_sheet(s, 1.0, 1.0, "corners" if k % 2 else "top_edge", seed=40 + k,
                                   stretch_comp=float(10 ** rng.uniform(-8, -3))))
    return specs


@pytest.mark.parametrize("relax", [P.RELAX_AVERAGE, P.RELAX_OMEGA], ids=["average", "omega"])
def test_cloth_kernel_every_launch_class_bit_exact(mixed_batch, relax):
    prm = params_for(10, 10, 1.0 if relax == P.RELAX_AVERAGE else 0.32)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=relax, solve_substeps=10, jacobi_kernel=4)
    plug = gpu_sim(mixed_batch, prm, cfg)
    st = plug.stats()
    assert st["solver_kernel"] == CLOTH
    assert st["cluster_ctas"] == 16
    plug.step(frames=2)
    for k, sp in enumerate(mixed_batch):
        o = oracle_sim(sp, prm, cfg, omp=True)
        o.substeps(20)
        xo, vo = o.state()
        assert max_abs(plug.positions(k), xo) == 0.0, (k, sp.side)
        assert max_abs(plug.velocities(k), vo) == 0.0, (k, sp.side)


def test_cloth_kernel_matches_the_thread_per_particle_kernel():
    specs = wl.config3_batch(seed=21, count=12, side_lo=16, side_hi=100)
    prm = params_for(10, 10, 1.0)
    a = gpu_sim(specs, prm, _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
                                 jacobi_kernel=4))
    b = gpu_sim(specs, prm, _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
                                 jacobi_kernel=3))
    assert a.stats()["solver_kernel"] == CLOTH and b.stats()["solver_kernel"] == ROWS
    a.step(frames=4)
    b.step(frames=4)
    assert max_abs(a.positions(), b.positions()) == 0.0
    assert max_abs(a.velocities(), b.velocities()) == 0.0


def test_cloth_kernel_grabs_drag_gravity_and_substep_api_bit_exact():
    sp = wl.make_sheet(70, 1.0, 1.0, "corners", seed=23)
    prm = params_for(10, 10, 1.0, drag=1.25, gravity=(0.3, -9.81, -0.2))
    prm.grab_idx, prm.grab_active, prm.grab_target, prm.grab_stiffness = 2000, True, (0.1, 0.8, 0.2), 0.28
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=4)
    plug = gpu_sim(sp, prm, cfg)
    assert plug.stats()["solver_kernel"] == CLOTH
    plug.set_cloth_grab(0, 3000, (-0.2, 0.9, 0.1), 0.45)
    plug.step(frames=2)
    plug.substep(3)  # single substeps (no graph)
    # against the thread-per-particle kernel, whose per-cloth grab is checked against the oracle in test_gpu_grab.py
    ref = gpu_sim(sp, prm, _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
                                jacobi_kernel=3))
    ref.set_cloth_grab(0, 3000, (-0.2, 0.9, 0.1), 0.45)
    ref.step(frames=2)
    ref.substep(3)
    assert max_abs(plug.positions(), ref.positions()) == 0.0
    assert max_abs(plug.velocities(), ref.velocities()) == 0.0


def test_cloth_kernel_context_grab_against_oracle():
    sp = wl.make_sheet(48, 1.0, 1.0, "top_edge", seed=24)
    prm = params_for(10, 10, 1.0, drag=0.5)
    prm.grab_idx, prm.grab_active, prm.grab_target, prm.grab_stiffness = 1500, True, (0.1, 0.8, 0.2), 0.28
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=4)
    plug = gpu_sim(sp, prm, cfg)
    assert plug.stats()["solver_kernel"] == CLOTH
    plug.step(frames=3)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(30)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


def test_cloth_kernel_zero_iterations_bit_exact():
    sp = wl.make_sheet(30, 1.0, 1.0, "corners", seed=25)
    prm = params_for(10, 0, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=4)
    plug = gpu_sim(sp, prm, cfg)
    assert plug.stats()["solver_kernel"] == CLOTH
    plug.step(frames=2)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(20)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


def test_cloth_kernel_refuses_batches_that_share_a_particle():
    """Presorted constraints whose batches are not particle-disjoint: the summation order of the cloth-resident
    kernel would differ from the neighbour-table order, so the schedule keeps the thread-per-particle kernel."""
    sp = wl.make_sheet(20, 1.0, 1.0, "corners", seed=26)
    e = sp.num_constraints
    plug = P.ClothComputePlugin(0)
    plug.add_cloth(sp.positions, sp.inv_mass, sp.constraint_i, sp.constraint_j, sp.rest_len, sp.compliance,
                   order=P.ORDER_PRESORTED, batch_offsets=np.array([0, e // 2, e], np.uint32))
    plug.commit()
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=4)
    plug.set_params(prm, cfg)
    assert plug.stats()["solver_kernel"] == ROWS
    plug.step(frames=1)
    from oracle import oracle as orc
    from tests.helpers import oracle_params
    o = orc.OracleSim(sp.positions, sp.inv_mass, sp.constraint_i, sp.constraint_j, sp.rest_len, sp.compliance)
    o.set_params(oracle_params(prm, cfg))
    o.substeps(10)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


SMALL = 8  # kernel id of the single-cluster small-batch kernel


@pytest.mark.parametrize("relax", [P.RELAX_AVERAGE, P.RELAX_OMEGA], ids=["average", "omega"])
def test_small_batch_kernel_bit_exact(relax):
    """A few small cloths in one cluster (thread per incidence, one cluster barrier per pass) against the oracle."""
    specs = [wl.make_sheet(s, 1.0, 1.0, "corners" if k % 2 else "top_edge", seed=60 + k)
             for k, s in enumerate([32, 17, 9, 40])]
    prm = params_for(10, 10, 1.0 if relax == P.RELAX_AVERAGE else 0.32, drag=0.3)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=relax, solve_substeps=10, jacobi_kernel=5)
    plug = gpu_sim(specs, prm, cfg)
    assert plug.stats()["solver_kernel"] == SMALL
    plug.step(frames=3)
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        o.substeps(30)
        xo, vo = o.state()
        assert max_abs(plug.positions(k), xo) == 0.0, k
        assert max_abs(plug.velocities(k), vo) == 0.0, k


@pytest.mark.parametrize("iters", [0, 1, 3], ids=["no_pass", "one_pass", "three_passes"])
def test_small_batch_kernel_odd_pass_counts_and_grab(iters):
    """Odd pass counts alternate the two position buffers across substeps; a context grab pulls one vertex."""
    sp = wl.make_sheet(32, 1.0, 1.0, "corners", seed=64)
    prm = params_for(10, iters, 1.0)
    prm.grab_idx, prm.grab_active, prm.grab_target, prm.grab_stiffness = 700, True, (0.2, 0.7, 0.1), 0.28
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    plug = gpu_sim(sp, prm, cfg)
    assert plug.stats()["solver_kernel"] == SMALL  # the default for a 1,024-particle sheet
    plug.step(frames=2)
    plug.substep(3)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(23)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


@pytest.mark.parametrize("kernel", [5, 3], ids=["small_batch", "thread_rows"])
def test_repeated_constraints_between_one_pair_bit_exact(kernel):
    """Several constraints joining the same two particles (different rest lengths and compliances, in both endpoint
    orders), inside one CTA of the small-batch cluster and across two: each row lists them in table order, and the
    small-batch kernel pairs the k-th of one row with the k-th of the other when it solves a constraint once for both
    endpoints."""
    sp = wl.make_sheet(24, 1.0, 1.0, "corners", seed=71)
    rng = np.random.default_rng(72)
    pick = rng.choice(sp.num_constraints, 40, replace=False)
    extra_i = sp.constraint_i[pick].copy()
    extra_j = sp.constraint_j[pick].copy()
    flip = rng.random(40) < 0.5
    extra_i[flip], extra_j[flip] = sp.constraint_j[pick][flip], sp.constraint_i[pick][flip]
    # a particle of row 1 joined twice more to one of row 20 (different CTAs of the cluster)
    extra_i = np.concatenate([extra_i, np.array([30, 485], np.uint32)])
    extra_j = np.concatenate([extra_j, np.array([485, 30], np.uint32)])
    n_extra = len(extra_i)
    sp.constraint_i = np.concatenate([sp.constraint_i, extra_i]).astype(np.uint32)
    sp.constraint_j = np.concatenate([sp.constraint_j, extra_j]).astype(np.uint32)
    rest = np.linalg.norm(sp.rest_positions[extra_i].astype(np.float64) - sp.rest_positions[extra_j], axis=1)
    sp.rest_len = np.concatenate([sp.rest_len, (rest * rng.uniform(0.9, 1.1, n_extra)).astype(np.float32)])
    sp.compliance = np.concatenate([sp.compliance, (10.0 ** rng.uniform(-8, -4, n_extra)).astype(np.float32)])
    sp.constraint_type = np.concatenate([sp.constraint_type, np.zeros(n_extra, np.uint32)])
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=kernel)
    plug = gpu_sim(sp, prm, cfg)
    assert plug.stats()["solver_kernel"] == (SMALL if kernel == 5 else ROWS)
    plug.step(frames=2)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(20)
    xo, vo = o.state()
    assert max_abs(plug.positions(), xo) == 0.0
    assert max_abs(plug.velocities(), vo) == 0.0


def test_small_batch_kernel_eight_cta_cluster_bit_exact():
    """The small-batch kernel on a cluster of 8 CTAs (128 particles per CTA here): the same records, pairing of
    rank-internal constraints and row updates as on 16, with a different split of the sheet."""
    sp = wl.make_sheet(32, 1.0, 1.0, "corners", seed=73)
    prm = params_for(10, 10, 1.0, drag=0.2)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10, jacobi_kernel=5,
               cluster_ctas=8)
    plug = gpu_sim(sp, prm, cfg)
    st = plug.stats()
    assert st["solver_kernel"] == SMALL and st["cluster_ctas"] == 8
    plug.step(frames=3)
    o = oracle_sim(sp, prm, cfg)
    o.substeps(30)
    xo, vo = o.state()
    assert max_abs(plug.positions(), xo) == 0.0
    assert max_abs(plug.velocities(), vo) == 0.0
