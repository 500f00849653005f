"""Host-side mirror of the reference plugin interface for the cloth substep, over the C ABI.

Names follow the Rust crate `bevy_softbody`:
  XpbdCpuTimeStepParams  — solver parameter struct (src/xpbd_cpu.rs:11-26)
  ClothSimUniforms       — per-frame uniforms with the reference defaults (src/cloth_compute.rs:181-243)
  ClothSimConfig         — solver configuration (src/cloth_compute.rs:140-179) + extension modes
  ClothComputePlugin     — owns the simulation (src/cloth_compute.rs:443-479); `step(params)` is the headless entry
  ClothMaterialPlugin    — headless stand-in of the render material (src/cloth_material.rs:40-49): it exposes the
                           simulated positions as a host array instead of a GPU vertex buffer (no graphics stack).
Errors raise XpbdError carrying the library status code; the reference panics or returns silently instead
(cloth_compute.rs:1189, :1219-1228).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields

import numpy as np

from . import _native as N
from ._native import XpbdError

SUBSTEPS = 36          # cloth_compute.rs:59
INNER_ITERS = 22       # cloth_compute.rs:61
REFERENCE_FRAME_DELTA_SECS = np.float32(1.0) / np.float32(60.0)  # cloth_compute.rs:65
THICKNESS = 0.04       # cloth_compute.rs:72
DEFAULT_COLL_SCALE = 0.38
DEFAULT_LINEAR_AIR_DRAG_PER_SEC = 1.25
JACOBI_DEFAULT_OMEGA = 0.32  # cloth_jacobi.rs:946-948

SOLVER_JACOBI, SOLVER_GAUSS_SEIDEL = 0, 1
RELAX_OMEGA, RELAX_AVERAGE = 0, 1
LAMBDA_RESET_PER_ITERATION, LAMBDA_PER_SUBSTEP = 0, 1
COLLISION_NONE, COLLISION_REST_FILTER, COLLISION_RING_FILTER = 0, 1, 2
ORDER_COLOR_REFERENCE, ORDER_COLOR_INDEX, ORDER_PRESORTED = 0, 1, 2
WARM_NONE, WARM_LEARNED, WARM_GIVEN, WARM_PREVIOUS = 0, 1, 2, 3
ALL = 0xFFFFFFFF


@dataclass
class XpbdCpuTimeStepParams:
    """src/xpbd_cpu.rs:11-26."""
    dt: float
    inv_dt: float
    jacobi_omega: float
    inner_iterations: int
    gravity: tuple = (0.0, -9.81, 0.0)
    grab_idx: int = -1
    grab_active: bool = False
    grab_target: tuple = (0.0, 0.0, 0.0)
    grab_stiffness: float = 0.0
    linear_drag_per_sec: float = 0.0

    def to_c(self) -> N.TimeStepParams:
        p = N.TimeStepParams()
        p.dt, p.inv_dt, p.jacobi_omega = self.dt, self.inv_dt, self.jacobi_omega
        p.inner_iterations = int(self.inner_iterations)
        p.gravity[:] = [float(v) for v in self.gravity]
        p.grab_idx, p.grab_active = int(self.grab_idx), int(bool(self.grab_active))
        p.grab_target[:] = [float(v) for v in self.grab_target]
        p.grab_stiffness, p.linear_drag_per_sec = self.grab_stiffness, self.linear_drag_per_sec
        return p

    def as_dict(self) -> dict:
        return {f.name: getattr(self, f.name) for f in fields(self)}


@dataclass
class ClothSimUniforms:
    """ClothSimUniforms::default() (cloth_compute.rs:204-243) for the chosen solver feature."""
    solver: int = SOLVER_JACOBI
    dt: float = float(np.float32(REFERENCE_FRAME_DELTA_SECS / np.float32(SUBSTEPS)))
    inner_iterations: int = INNER_ITERS
    thickness: float = THICKNESS
    coll_scale: float = DEFAULT_COLL_SCALE
    gravity: tuple = (0.0, -9.81, 0.0)
    grab_target: tuple = (0.0, 0.0, 0.0)
    grab_idx: int = -1
    grab_active: int = 0
    linear_drag_per_sec: float = DEFAULT_LINEAR_AIR_DRAG_PER_SEC
    jacobi_omega: float | None = None
    grab_stiffness: float | None = None

    def __post_init__(self):
        if self.jacobi_omega is None:
            self.jacobi_omega = JACOBI_DEFAULT_OMEGA if self.solver == SOLVER_JACOBI else 1.0
        if self.grab_stiffness is None:
            self.grab_stiffness = 0.28 if self.solver == SOLVER_JACOBI else 0.45

    @property
    def inv_dt(self) -> float:
        return float(np.float32(1.0) / np.float32(self.dt))

    def substep_params(self) -> XpbdCpuTimeStepParams:
        """`substep_params` of the reference tests (xpbd_cpu.rs:735-749)."""
        return XpbdCpuTimeStepParams(self.dt, self.inv_dt, self.jacobi_omega, self.inner_iterations, self.gravity,
                                     self.grab_idx, bool(self.grab_active), self.grab_target, self.grab_stiffness,
                                     self.linear_drag_per_sec)


@dataclass
class ClothSimConfig:
    """Solver configuration: ClothSimConfig (cloth_compute.rs:140-179) solve_* fields, the collision uniforms, and
    the extension modes. Defaults are the reference's (xpbd_default_opts)."""
    solver: int = SOLVER_JACOBI
    relaxation: int = RELAX_OMEGA
    lambda_mode: int = LAMBDA_RESET_PER_ITERATION
    solve_substeps: int = SUBSTEPS
    collision: int = COLLISION_NONE
    collision_every_n_substeps: int = 1
    thickness: float = THICKNESS
    coll_scale: float = DEFAULT_COLL_SCALE
    hash_cell: float = THICKNESS
    hash_table_bits: int = 20
    ring_depth: int = 2
    ground_enabled: bool = False
    ground_y: float = 0.0
    use_graphs: bool = True
    barrier_timeout_ms: float = 2000.0
    block_threads: int = 0
    blocks_per_sm: int = 0
    warm_start: int = WARM_NONE
    cluster_ctas: int = 0
    jacobi_kernel: int = 0
    tolerance: float = 0.0
    gs_strips: int = 0

    def to_c(self) -> N.SolverOpts:
        o = N.SolverOpts()
        o.solver, o.relaxation, o.lambda_mode = self.solver, self.relaxation, self.lambda_mode
        o.substeps, o.collision = self.solve_substeps, self.collision
        o.collision_every_n_substeps = self.collision_every_n_substeps
        o.thickness, o.coll_scale, o.hash_cell = self.thickness, self.coll_scale, self.hash_cell
        o.hash_table_bits, o.ring_depth = self.hash_table_bits, self.ring_depth
        o.ground_enabled, o.ground_y = int(self.ground_enabled), self.ground_y
        o.use_graphs, o.barrier_timeout_ms = int(self.use_graphs), self.barrier_timeout_ms
        o.block_threads, o.blocks_per_sm, o.warm_start = self.block_threads, self.blocks_per_sm, int(self.warm_start)
        o.cluster_ctas = self.cluster_ctas
        o.jacobi_kernel = self.jacobi_kernel
        o.tolerance = self.tolerance
        o.gs_strips = self.gs_strips
        return o


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, np.float32)
    return a.reshape(shape) if shape is not None else a


def _u32(a):
    return np.ascontiguousarray(a, np.uint32)


def mlp_scale_change(params, norm, factor: float):
    """Parameters of the warm-start network whose predicted change of the multiplier is `factor` times the given one's.

    The network predicts, standardised, the change of t = λ·(wi + wj + α̃)/rest over the previous substep:
    λ0 = (y·tstd + tmean + t_prev)·rest/(wi + wj + α̃), with y linear in the output layer (w3, b3). Scaling w3, b3 and
    tmean by `factor` scales the change y·tstd + tmean and nothing else: factor 1 is the network as trained, 0 the
    previous substep's multiplier. A factor below 1 shrinks the prediction toward the previous multiplier, which lowers
    the worst-constraint error that the convergence test is bound by; choose it on the training cloths."""
    p = np.array(params, np.float32, copy=True)
    n = np.array(norm, np.float32, copy=True)
    w3 = N.MLP_PARAMS - 65  # w3[64] then b3 at the end of the parameter vector
    p[w3:] *= np.float32(factor)
    n[18] *= np.float32(factor)
    return p, n


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class ClothComputePlugin:
    """A batch of cloths simulated on one GPU (ClothComputePlugin + init_cloth_sim + run_cloth_sim)."""

    def __init__(self, device: int = 0):
        self._L = N.load()
        h = C.c_void_p()
        st = self._L.xpbd_create(C.byref(h), device)
        if st != N.XPBD_OK:
            raise XpbdError(st, "xpbd_create failed (no usable CUDA device?)")
        self._h = h
        self._cloths = []  # (num_particles, num_constraints)
        self.config = ClothSimConfig()
        self.params: XpbdCpuTimeStepParams | None = None
        self._keep = []

    # ---- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._L.xpbd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str = ""):
        if st != N.XPBD_OK:
            msg = self._L.xpbd_last_error(self._h).decode() if self._h else what
            raise XpbdError(st, msg or what)

    def set_stream(self, stream_handle: int | None):
        self._check(self._L.xpbd_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    # ---- building
    def add_cloth(self, positions, inv_mass, constraint_i, constraint_j, rest_len, compliance, velocities=None,
                  rest_positions=None, constraint_type=None, order=ORDER_COLOR_REFERENCE, batch_offsets=None) -> int:
        pos = _f32(positions).reshape(-1)
        w = _f32(inv_mass)
        ci, cj = _u32(constraint_i), _u32(constraint_j)
        rl, cp = _f32(rest_len), _f32(compliance)
        vel = None if velocities is None else _f32(velocities).reshape(-1)
        rp = None if rest_positions is None else _f32(rest_positions).reshape(-1)
        ct = None if constraint_type is None else _u32(constraint_type)
        bo = None if batch_offsets is None else _u32(batch_offsets)
        d = N.ClothDesc()
        d.num_particles = len(w)
        d.positions, d.velocities, d.inv_mass, d.rest_positions = _ptr(pos), _ptr(vel), _ptr(w), _ptr(rp)
        d.num_constraints = len(ci)
        d.constraint_i, d.constraint_j, d.rest_len, d.compliance = _ptr(ci), _ptr(cj), _ptr(rl), _ptr(cp)
        d.constraint_type, d.order = _ptr(ct), order
        d.batch_offsets, d.batch_count = _ptr(bo), 0 if bo is None else len(bo) - 1
        cid = C.c_uint32()
        self._check(self._L.xpbd_add_cloth(self._h, C.byref(d), C.byref(cid)))
        self._cloths.append((len(w), len(ci)))
        return cid.value

    def add_spec(self, spec, order=ORDER_COLOR_REFERENCE) -> int:
        """Adds a workloads.ClothSpec."""
        return self.add_cloth(spec.positions, spec.inv_mass, spec.constraint_i, spec.constraint_j, spec.rest_len,
                              spec.compliance, spec.velocities, spec.rest_positions, spec.constraint_type, order)

    def add_mesh(self, mesh) -> int:
        """A ClothMeshData (bevy_xpbd_b200.mesh) with its batch order and render triangles."""
        cid = self.add_cloth(**mesh.to_spec_arrays())
        if len(mesh.indices):
            self.set_triangles(cid, mesh.indices)
        return cid

    def set_cloth_grab(self, cloth: int, vertex: int | None, target=(0.0, 0.0, 0.0), stiffness: float = 0.0):
        """Grab one vertex of a cloth (None releases it): pulled toward `target` after each prediction."""
        t = np.ascontiguousarray(target, np.float32)
        self._check(self._L.xpbd_set_cloth_grab(self._h, cloth, -1 if vertex is None else int(vertex), _ptr(t),
                                                C.c_float(stiffness)))

    def set_cloth_wind(self, cloth: int, velocity=(0.0, 0.0, 0.0), drag: float = 0.0):
        """Wind on a cloth (extension): after gravity, v += (velocity - v) * (drag * dt); drag 0 turns it off."""
        w = np.ascontiguousarray(velocity, np.float32)
        self._check(self._L.xpbd_set_cloth_wind(self._h, cloth, _ptr(w), C.c_float(drag)))

    def set_triangles(self, cloth: int, tri_indices):
        """Render triangles (local vertex indices, 3 per triangle) of a cloth, for `normals`."""
        t = _u32(tri_indices).reshape(-1)
        self._check(self._L.xpbd_set_triangles(self._h, cloth, t.size // 3, _ptr(t)))

    def normals(self, cloth: int = 0) -> np.ndarray:
        """Vertex normals of the current positions (accumulate_normals + finalize_normals)."""
        out = np.empty((self._cloths[cloth][0], 3), np.float32)
        self._check(self._L.xpbd_read_normals(self._h, cloth, _ptr(out)))
        return out

    def commit(self):
        self._check(self._L.xpbd_commit(self._h))

    @property
    def num_particles(self) -> int:
        return sum(n for n, _ in self._cloths)

    def cloth_size(self, cloth: int) -> tuple[int, int]:
        return self._cloths[cloth]

    # ---- per frame
    def set_params(self, params: XpbdCpuTimeStepParams, config: ClothSimConfig | None = None):
        if config is not None:
            self.config = config
        self.params = params
        self._cp = params.to_c()
        self._co = self.config.to_c()
        self._check(self._L.xpbd_set_params(self._h, C.byref(self._cp), C.byref(self._co)))

    def step(self, params: XpbdCpuTimeStepParams | None = None, frames: int = 1):
        """Headless step(params): enqueue `frames` frames (asynchronous; positions() synchronises)."""
        if params is not None:
            self._cp = params.to_c()
            self.params = params
            self._check(self._L.xpbd_step_params(self._h, C.byref(self._cp), frames))
        else:
            self._check(self._L.xpbd_step(self._h, frames))

    def substep(self, count: int = 1):
        self._check(self._L.xpbd_substep(self._h, count))

    def sync(self):
        self._check(self._L.xpbd_sync(self._h))

    # ---- state
    def _n(self, cloth):
        return self.num_particles if cloth is None else self._cloths[cloth][0]

    def positions(self, cloth: int | None = None) -> np.ndarray:
        out = np.empty((self._n(cloth), 3), np.float32)
        self._check(self._L.xpbd_read_positions(self._h, ALL if cloth is None else cloth, _ptr(out)))
        return out

    def positions_into(self, out: np.ndarray, cloth: int | None = None):
        self._check(self._L.xpbd_read_positions(self._h, ALL if cloth is None else cloth, _ptr(out)))

    def velocities(self, cloth: int | None = None) -> np.ndarray:
        out = np.empty((self._n(cloth), 3), np.float32)
        self._check(self._L.xpbd_read_velocities(self._h, ALL if cloth is None else cloth, _ptr(out)))
        return out

    def write_state(self, positions=None, velocities=None, cloth: int | None = None):
        p = None if positions is None else _f32(positions).reshape(-1)
        v = None if velocities is None else _f32(velocities).reshape(-1)
        self._check(self._L.xpbd_write_state(self._h, ALL if cloth is None else cloth, _ptr(p), _ptr(v)))

    def reset(self):
        self._check(self._L.xpbd_reset(self._h))

    def lambdas(self, cloth: int = 0) -> np.ndarray:
        out = np.empty(self._cloths[cloth][1], np.float32)
        self._check(self._L.xpbd_read_lambda(self._h, cloth, _ptr(out)))
        return out

    def set_warm_lambda(self, lambda0, cloth: int = 0):
        """λ0 per constraint (input order) for the WARM_GIVEN start of the convergence solve."""
        self._warm = _f32(lambda0)
        self._check(self._L.xpbd_set_warm_lambda(self._h, cloth, _ptr(self._warm)))

    def converge_history(self, max_count: int = 4096) -> np.ndarray:
        """Max residual |C + α̃λ|/rest before each update pass of the most recent convergence-solve substep."""
        out = np.zeros(max_count, np.float32)
        c = C.c_uint32(0)
        self._check(self._L.xpbd_converge_history(self._h, _ptr(out), max_count, C.byref(c)))
        return out[: min(int(c.value), max_count)]

    def converge_cloth_iterations(self) -> np.ndarray:
        """Update passes each cloth took in the most recent convergence-solve substep."""
        out = np.zeros(len(self._cloths), np.uint32)
        self._check(self._L.xpbd_converge_cloth_iterations(self._h, _ptr(out)))
        return out

    # ---- learned warm start (extension) ------------------------------------------------------------------------
    def mlp_init(self, seed: int = 0, capacity: int = 1 << 20):
        """Allocates the warm-start MLP (seeded initialisation) and room for `capacity` training samples."""
        self._check(self._L.xpbd_mlp_init(self._h, seed, capacity))

    def mlp_params(self) -> tuple[np.ndarray, np.ndarray]:
        """(fp32 parameters [w1 64x9, b1, w2 64x64, b2, w3, b3], normalisation [fmean 9, fstd 9, tmean, tstd])."""
        p = np.zeros(N.MLP_PARAMS, np.float32)
        n = np.zeros(N.MLP_NORM, np.float32)
        self._check(self._L.xpbd_mlp_get_params(self._h, _ptr(p), _ptr(n)))
        return p, n

    def mlp_set_params(self, params, norm=None):
        p = _f32(params)
        n = None if norm is None else _f32(norm)
        self._check(self._L.xpbd_mlp_set_params(self._h, _ptr(p), None if n is None else _ptr(n)))

    def mlp_predict_lambda(self, cloth: int = 0) -> np.ndarray:
        """λ0 the learned warm start gives the next substep (input order); the state is unchanged."""
        n_con = self.cloth_size(cloth)[1]
        out = np.zeros(n_con, np.float32)
        self._check(self._L.xpbd_mlp_predict_lambda(self._h, cloth, _ptr(out)))
        return out

    def mlp_collect(self, substeps: int, stride: int = 1) -> int:
        """Runs `substeps` convergence-solve substeps as configured and stores (features, final λ target) samples."""
        self._check(self._L.xpbd_mlp_collect(self._h, substeps, stride))
        c = C.c_uint32(0)
        self._check(self._L.xpbd_mlp_dataset_size(self._h, C.byref(c)))
        return int(c.value)

    def mlp_dataset(self, max_rows: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        c = C.c_uint32(0)
        self._check(self._L.xpbd_mlp_dataset_size(self._h, C.byref(c)))
        n = int(c.value) if max_rows is None else min(int(c.value), max_rows)
        f = np.zeros((n, N.MLP_FEATURES), np.float32)
        t = np.zeros(n, np.float32)
        rows = C.c_uint32(0)
        self._check(self._L.xpbd_mlp_dataset_read(self._h, n, _ptr(f), _ptr(t), C.byref(rows)))
        return f[: rows.value], t[: rows.value]

    def mlp_fit_normalization(self):
        self._check(self._L.xpbd_mlp_fit_normalization(self._h))

    def mlp_train(self, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(steps, np.float32)
        self._check(self._L.xpbd_mlp_train(self._h, steps, batch, C.c_float(lr), seed, _ptr(losses)))
        return losses

    def mlp_minibatch_gradients(self, batch: int, seed: int, grads_ptr: int, loss_ptr: int):
        """Asynchronous: gradient of a seeded minibatch into the device buffer at grads_ptr (4,865 floats)."""
        self._check(self._L.xpbd_mlp_minibatch_gradients(self._h, batch, seed, C.c_void_p(grads_ptr),
                                                         C.c_void_p(loss_ptr)))

    def mlp_apply_gradients(self, grads_ptr: int, scale: float, lr: float):
        """Asynchronous: one Adam step with the device gradient at grads_ptr times `scale`."""
        self._check(self._L.xpbd_mlp_apply_gradients(self._h, C.c_void_p(grads_ptr), C.c_float(scale),
                                                     C.c_float(lr)))

    def mlp_eval(self, features) -> np.ndarray:
        f = _f32(features)
        n = f.size // N.MLP_FEATURES
        out = np.zeros(n, np.float32)
        self._check(self._L.xpbd_mlp_eval(self._h, _ptr(f), n, _ptr(out)))
        return out

    def mlp_gradients(self, features, targets) -> tuple[np.ndarray, float]:
        f = _f32(features)
        t = _f32(targets)
        g = np.zeros(N.MLP_PARAMS, np.float32)
        loss = C.c_float(0)
        self._check(self._L.xpbd_mlp_gradients(self._h, _ptr(f), _ptr(t), t.size, _ptr(g), C.byref(loss)))
        return g, float(loss.value)

    def strain_residual(self, cloth: int | None = None) -> float:
        v = C.c_float()
        self._check(self._L.xpbd_strain_residual(self._h, ALL if cloth is None else cloth, C.byref(v)))
        return v.value

    def coloring(self, cloth: int = 0):
        nb = C.c_uint32()
        self._check(self._L.xpbd_get_coloring(self._h, cloth, None, None, C.byref(nb)))
        perm = np.empty(self._cloths[cloth][1], np.uint32)
        offs = np.empty(nb.value + 1, np.uint32)
        self._check(self._L.xpbd_get_coloring(self._h, cloth, _ptr(perm), _ptr(offs), C.byref(nb)))
        return perm, offs

    def stats(self) -> dict:
        s = N.Stats()
        self._check(self._L.xpbd_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in N.Stats._fields_}

    def autotune(self, frames: int = 3) -> ClothSimConfig:
        o = N.SolverOpts()
        self._check(self._L.xpbd_autotune(self._h, frames, C.byref(o)))
        self.config.block_threads, self.config.blocks_per_sm = o.block_threads, o.blocks_per_sm
        self.config.cluster_ctas = o.cluster_ctas
        self.config.jacobi_kernel = o.jacobi_kernel
        self.config.gs_strips = o.gs_strips
        return self.config

    # ---- collision introspection
    def collision_keys(self):
        n = self.num_particles
        k, sk, sv = (np.empty(n, np.uint32) for _ in range(3))
        self._check(self._L.xpbd_collision_keys(self._h, _ptr(k), _ptr(sk), _ptr(sv)))
        return k, sk, sv

    def collision_pairs(self, cap: int | None = None) -> np.ndarray:
        cnt = C.c_uint64()
        self._check(self._L.xpbd_collision_pairs(self._h, None, 0, C.byref(cnt)))
        total = cnt.value if cap is None else min(cap, cnt.value)
        out = np.empty((total, 2), np.uint32)
        if total:
            self._check(self._L.xpbd_collision_pairs(self._h, _ptr(out), total, C.byref(cnt)))
        return out

    def debug_force_barrier_timeout(self, timeout_ms: float) -> int:
        """Runs one launch whose first grid barrier can never complete; returns the status (expected -7)."""
        return self._L.xpbd_debug_force_barrier_timeout(self._h, timeout_ms)


class ClothMaterialPlugin:
    """Headless stand-in of ClothMaterialPlugin / ClothMatExt (cloth_material.rs:14-49): the render material read the
    simulated positions from GPU storage buffers; here they are read back as an (N,3) array."""

    def __init__(self, compute: ClothComputePlugin):
        self.compute = compute

    def render_positions(self, cloth: int | None = None) -> np.ndarray:
        return self.compute.positions(cloth)

    def render_normals(self, cloth: int = 0) -> np.ndarray:
        """render_normals of the reference (finalize_normals, cloth_sim_jacobi.wgsl:528-547)."""
        return self.compute.normals(cloth)
