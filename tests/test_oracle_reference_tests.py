"""The reference's own tests for this path, ported onto the CPU oracle (pins the oracle).

Each test names the Rust test it restates (src/xpbd_cpu.rs:751-1128, src/cloth_compute.rs:1528-1577) and uses
the same inputs: `grid_cloth_hanging(16, 16, 0.045)`, `ClothSimUniforms::default()` (cloth_compute.rs:204-243)
and `SUBSTEPS` = 36 substeps per frame (cloth_compute.rs:59). Both solver features are exercised (Jacobi =
`solver-jacobi`, GS = `solver-gauss-seidel`).
"""
import numpy as np
import pytest

from oracle import oracle as orc

SUBSTEPS = 36
INNER_ITERS = 22


def default_params(solver: int) -> dict:
    """ClothSimUniforms::default() turned into XpbdCpuTimeStepParams like `substep_params` (xpbd_cpu.rs:735-749)."""
    sdt = np.float32(np.float32(1.0 / 60.0) / np.float32(SUBSTEPS))
    return dict(dt=float(sdt), inv_dt=float(np.float32(1.0) / sdt),
                jacobi_omega=0.32 if solver == 0 else 1.0, inner_iterations=INNER_ITERS,
                gravity=(0.0, -9.81, 0.0), grab_idx=-1, grab_active=0, grab_target=(0.0, 0.0, 0.0),
                grab_stiffness=0.28 if solver == 0 else 0.45, linear_drag_per_sec=1.25, solver=solver,
                thickness=0.04, coll_scale=0.38, hash_cell=0.04)


def sim_from_mesh(m, params, fp64=False):
    s = orc.OracleSim(m.positions, m.inv_mass, m.constraint_i, m.constraint_j, m.constraint_rest_len,
                      m.constraint_compliance, rest_pos=m.rest_positions, fp64=fp64)
    s.set_params(params)
    return s


@pytest.fixture(scope="module")
def cloth():
    return orc.grid_cloth_hanging(16, 16, 0.045)


SOLVERS = [pytest.param(0, id="jacobi"), pytest.param(1, id="gauss_seidel")]


def test_cloth_mesh_inv_mass_and_neighbors_sane(cloth):
    """xpbd_cpu.rs:751-757."""
    assert np.all(np.isfinite(cloth.inv_mass))


@pytest.mark.parametrize("solver", SOLVERS)
def test_cpu_xpbd_cloth_one_frame_integrator_only_stays_finite(cloth, solver):
    """xpbd_cpu.rs:759-807: jacobi_omega = 0, one frame."""
    p = default_params(solver)
    p["jacobi_omega"] = 0.0
    s = sim_from_mesh(cloth, p)
    s.substeps(SUBSTEPS)
    x, _ = s.state()
    assert np.all(np.isfinite(x))


@pytest.mark.parametrize("solver", SOLVERS)
def test_cpu_xpbd_cloth_one_frame_full_solver_stays_finite(cloth, solver):
    """xpbd_cpu.rs:809-855."""
    s = sim_from_mesh(cloth, default_params(solver))
    s.substeps(SUBSTEPS)
    x, _ = s.state()
    assert np.all(np.isfinite(x))


@pytest.mark.parametrize("solver", SOLVERS)
def test_cpu_xpbd_pins_hold_rest_positions(cloth, solver):
    """xpbd_cpu.rs:857-913: pinned particles stay within 1e-4 of rest after one frame."""
    p = default_params(solver)
    p.update(grab_idx=-1, grab_active=0, grab_stiffness=0.0)
    s = sim_from_mesh(cloth, p)
    s.substeps(SUBSTEPS)
    x, _ = s.state()
    pinned = cloth.inv_mass <= 0
    assert pinned.sum() == 17
    assert np.all(np.linalg.norm(x[pinned] - cloth.positions[pinned], axis=1) < 1e-4)


@pytest.mark.parametrize("solver", SOLVERS)
def test_cpu_xpbd_single_triangle_one_frame_finite(solver):
    """xpbd_cpu.rs:915-974: single welded OBJ triangle, gravity (-1,-2,0.5)."""
    obj = "\nv 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nf 1/1 2/2 3/3\n"
    m = orc.parse_welded_obj(obj)
    assert m.num_particles == 3
    p = default_params(solver)
    p.update(gravity=(-1.0, -2.0, 0.5), grab_active=0)
    s = sim_from_mesh(m, p)
    s.substeps(SUBSTEPS)
    x, _ = s.state()
    assert np.all(np.isfinite(x))


@pytest.mark.parametrize("solver", SOLVERS)
def test_cpu_xpbd_cloth_15_frames_extent_stays_reasonable(cloth, solver):
    """xpbd_cpu.rs:976-1034: AABB of free particles after 15 frames has ext.x > 0.18 and ext.y > 0.04."""
    p = default_params(solver)
    p["grab_active"] = 0
    s = sim_from_mesh(cloth, p)
    s.substeps(15 * SUBSTEPS)
    x, _ = s.state()
    free = cloth.inv_mass > 0
    ext = x[free].max(0) - x[free].min(0)
    assert ext[0] > 0.18 and ext[1] > 0.04, ext


def _two_particles(w0, x1):
    inv_mass = np.array([w0, 1.0], np.float32)
    rest = np.array([[0, 0, 0], [0.1, 0, 0]], np.float32)
    sim = np.array([[0, 0, 0], [x1, 0, 0]], np.float32)
    return inv_mass, rest, sim


def test_cpu_self_collision_pair_separates_when_penetrating():
    """xpbd_cpu.rs:1036-1047, plus the known answer derivable from its inputs: corr = (0.04-0.015)*0.5*0.38,
    split equally, so the new distance is 0.015 + 0.0095 = 0.01975."""
    w, rest, sim = _two_particles(1.0, 0.015)
    d0 = np.linalg.norm(sim[1] - sim[0])
    out = orc.self_collision_resolve(sim, w, rest, 0.04, 0.38)
    d1 = np.linalg.norm(out[1] - out[0])
    assert d1 > d0 + 1e-4
    assert abs(d1 - 0.01975) < 1e-7
    assert abs(out[0, 0] - (-0.002375)) < 1e-8 and abs(out[1, 0] - 0.017375) < 1e-8


def test_cpu_self_collision_skips_when_world_separation_exceeds_rest():
    """xpbd_cpu.rs:1049-1060: untouched bit for bit."""
    w, rest, sim = _two_particles(1.0, 0.15)
    out = orc.self_collision_resolve(sim, w, rest, 0.04, 0.38)
    assert np.array_equal(out, sim)


def test_cpu_self_collision_pinned_neighbor_takes_no_delta():
    """xpbd_cpu.rs:1062-1073."""
    w, rest, sim = _two_particles(0.0, 0.015)
    out = orc.self_collision_resolve(sim, w, rest, 0.04, 0.38)
    assert np.array_equal(out[0], sim[0])
    assert out[1, 0] > 0.015


@pytest.mark.parametrize("solver", SOLVERS)
def test_cpu_xpbd_cloth_one_frame_with_self_collision_stays_finite(cloth, solver):
    """xpbd_cpu.rs:1075-1128 (all-pairs collision every substep)."""
    p = default_params(solver)
    p["collision"] = 1
    s = sim_from_mesh(cloth, p)
    s.substeps(SUBSTEPS, brute_force=True)
    x, _ = s.state()
    assert np.all(np.isfinite(x))


def test_cloth_neighbor_and_tri_indices_in_range():
    """cloth_compute.rs:1528-1548."""
    m = orc.grid_cloth_hanging(12, 10, 0.05)
    assert np.all(m.neighbor_other < m.num_particles)
    assert np.all(m.indices < m.num_particles)


def test_cloth_neighbor_slices_match_constraints():
    """cloth_compute.rs:1550-1577."""
    m = orc.grid_cloth_hanging(10, 8, 0.05)
    edges = {(min(a, b), max(a, b)) for a, b in zip(m.constraint_i.tolist(), m.constraint_j.tolist())}
    for i in range(m.num_particles):
        for k in range(m.neighbor_offsets[i], m.neighbor_offsets[i + 1]):
            j = int(m.neighbor_other[k])
            assert (min(i, j), max(i, j)) in edges


def test_grid_mesh_structure_matches_reference_builder():
    """grid_cloth_hanging(16,16,0.045): counts follow mesh_prep.rs:363-406 — 17x17 vertices; 3*16*16+16+16 triangle
    edges; hinge bends; 2*17*15 skip-2 braces; 16*16 cross diagonals; coloring yields a valid edge coloring whose
    batches are contiguous and ordered."""
    m = orc.grid_cloth_hanging(16, 16, 0.045)
    n = 17 * 17
    assert m.num_particles == n
    tri_edges = 16 * 17 * 2 + 16 * 16
    bends = 3 * 16 * 16 - 16 - 16  # one per interior triangle edge
    skip2 = 2 * 17 * 15
    cross = 16 * 16
    assert len(m.constraint_i) == tri_edges + bends + skip2 + cross
    offs = m.constraint_batch_offsets
    assert offs[0] == 0 and offs[-1] == len(m.constraint_i)
    for b in range(m.constraint_batch_count):
        seg_i = m.constraint_i[offs[b]:offs[b + 1]]
        seg_j = m.constraint_j[offs[b]:offs[b + 1]]
        verts = np.concatenate([seg_i, seg_j])
        assert len(np.unique(verts)) == len(verts), "batch shares a particle"
    # top row pinned (mesh_prep.rs:558-568), area inverse mass elsewhere
    top = np.isclose(m.positions[:, 1], m.positions[:, 1].max())
    assert np.all(m.inv_mass[top] == 0) and np.all(m.inv_mass[~top] > 0)


def test_oracle_fp32_vs_fp64_small_drift(cloth):
    """The FP32 oracle stays close to its FP64 build over one frame (sanity of the templated restatement)."""
    p = default_params(0)
    a = sim_from_mesh(cloth, p)
    b = sim_from_mesh(cloth, p, fp64=True)
    a.substeps(SUBSTEPS)
    b.substeps(SUBSTEPS)
    xa, _ = a.state()
    xb, _ = b.state()
    assert np.max(np.abs(xa - xb)) < 1e-4


@pytest.mark.parametrize("solver", SOLVERS)
def test_oracle_openmp_build_matches_serial(solver):
    """The OpenMP build (timed CPU baseline only) gives the serial checker's result bit for bit."""
    from bevy_xpbd_b200 import workloads as wl
    sp = wl.make_sheet(48, 1.0, 1.0, "top_edge", seed=2)
    perm, _, offs = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j)
    p = default_params(solver)
    p.update(relaxation=1 if solver == 0 else 0, inner_iterations=10)
    out = []
    for variant in ("serial", "omp"):
        orc.select(variant)
        try:
            s = orc.OracleSim(sp.positions, sp.inv_mass, sp.constraint_i[perm], sp.constraint_j[perm],
                              sp.rest_len[perm], sp.compliance[perm])
            s.set_params(p)
            if variant == "omp":
                s.set_batches(offs)
            s.substeps(20)
            out.append(s.state()[0])
            del s
        finally:
            orc.select("serial")
    assert np.array_equal(out[0], out[1])
