"""Seeded synthetic cloth workloads with the shapes, sizes and value distributions of the benchmark sheets.

No public dataset is involved: every workload is a procedural square sheet. A sheet of `s` x `s` vertices has
vertex (r, c) at index r*s + c, lying in the xz plane (x along columns, z along rows) at height `y0`, centred on
the origin. Constraint generation order (which fixes the greedy coloring input order):

  stretch  type 0: horizontal grid edges (r,c)-(r,c+1) row-major, then vertical (r,c)-(r+1,c) row-major
  shear    type 1: per cell row-major, diagonal (r,c)-(r+1,c+1) then anti-diagonal (r,c+1)-(r+1,c)
  bend     type 2: distance-2 pairs (r,c)-(r,c+2) row-major, then (r,c)-(r+2,c) row-major

so E = 2s(s-1) + 2(s-1)^2 + 2s(s-2) = 6s^2 - 10s + 2. Rest lengths come from the unjittered grid (FP32
length of the difference); the initial state is jittered by a seeded uniform offset per component.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

STRETCH, SHEAR, BEND = 0, 1, 2


@dataclass
class ClothSpec:
    """Host arrays of one cloth, the inputs of `xpbd_add_cloth`."""
    positions: np.ndarray        # (N,3) float32 initial state
    inv_mass: np.ndarray         # (N,) float32, 0 = pinned
    constraint_i: np.ndarray     # (E,) uint32
    constraint_j: np.ndarray     # (E,) uint32
    rest_len: np.ndarray         # (E,) float32
    compliance: np.ndarray       # (E,) float32
    constraint_type: np.ndarray  # (E,) uint32
    rest_positions: np.ndarray   # (N,3) float32
    velocities: np.ndarray | None = None
    side: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def num_particles(self) -> int:
        return int(self.inv_mass.shape[0])

    @property
    def num_constraints(self) -> int:
        return int(self.constraint_i.shape[0])


def sheet_constraints(s: int):
    """(ci, cj, type) of an s x s sheet in the documented generation order."""
    idx = np.arange(s * s, dtype=np.uint32).reshape(s, s)
    parts_i, parts_j, parts_t = [], [], []

    def add(a, b, t):
        parts_i.append(a.reshape(-1))
        parts_j.append(b.reshape(-1))
        parts_t.append(np.full(a.size, t, np.uint32))

    add(idx[:, :-1], idx[:, 1:], STRETCH)
    add(idx[:-1, :], idx[1:, :], STRETCH)
    d_i = idx[:-1, :-1]
    d_j = idx[1:, 1:]
    a_i = idx[:-1, 1:]
    a_j = idx[1:, :-1]
    add(np.stack([d_i, a_i], -1), np.stack([d_j, a_j], -1), SHEAR)
    add(idx[:, :-2], idx[:, 2:], BEND)
    add(idx[:-2, :], idx[2:, :], BEND)
    return np.concatenate(parts_i), np.concatenate(parts_j), np.concatenate(parts_t)


def _f32_len(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    d = (a - b).astype(np.float32)
    return np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32)


def make_sheet(s: int, side_m: float = 1.0, y0: float = 1.0, pins: str = "corners", mass: float = 0.01,
               jitter: float = 1e-3, seed: int = 0, stretch_comp: float = 0.0, shear_comp: float = 1e-6,
               bend_comp: float = 1e-4, velocity: np.ndarray | None = None) -> ClothSpec:
    """One sheet. pins: 'corners' (the two row-0 corners), 'top_edge' (all of row 0) or 'none'."""
    h = side_m / (s - 1)
    r, c = np.meshgrid(np.arange(s), np.arange(s), indexing="ij")
    rest64 = np.stack([c * h - 0.5 * side_m, np.full_like(r, y0, dtype=np.float64), r * h - 0.5 * side_m],
                      -1).reshape(-1, 3).astype(np.float64)
    rest = rest64.astype(np.float32)
    rng = np.random.default_rng(seed)
    pos = (rest64 + (rng.uniform(-jitter, jitter, rest64.shape) if jitter > 0 else 0.0)).astype(np.float32)
    w = np.full(s * s, np.float32(1.0 / mass), np.float32)
    if pins == "corners":
        w[0] = 0.0
        w[s - 1] = 0.0
    elif pins == "top_edge":
        w[:s] = 0.0
    elif pins != "none":
        raise ValueError(pins)
    ci, cj, ct = sheet_constraints(s)
    rl = _f32_len(rest[ci], rest[cj])
    comp = np.where(ct == STRETCH, stretch_comp, np.where(ct == SHEAR, shear_comp, bend_comp)).astype(np.float32)
    return ClothSpec(pos, w, ci, cj, rl, comp, ct, rest, velocity, side=s,
                     meta=dict(side_m=side_m, pins=pins, seed=seed, stretch_comp=stretch_comp))


def fourier_velocity(s: int, modes: int = 4, amplitude: float = 0.5, seed: int = 0) -> np.ndarray:
    """Smooth seeded random velocity field on an s x s sheet: a sum of `modes` plane waves in the sheet's (u,v)
    parameterisation with random integer wave vectors (1..3 per axis), phases and 3-D directions, scaled so the
    largest speed equals `amplitude`."""
    rng = np.random.default_rng(seed)
    u, v = np.meshgrid(np.linspace(0, 1, s), np.linspace(0, 1, s), indexing="ij")
    vel = np.zeros((s, s, 3))
    for _ in range(modes):
        k = rng.integers(1, 4, size=2)
        phase = rng.uniform(0, 2 * np.pi)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        vel += np.sin(2 * np.pi * (k[0] * u + k[1] * v) + phase)[..., None] * d
    vel *= amplitude / np.max(np.linalg.norm(vel, axis=-1))
    return vel.reshape(-1, 3).astype(np.float32)


# -------------------------------------------------------------------------------------------- benchmark sheets
FRAME_DT = np.float32(1.0) / np.float32(60.0)


def substep_dt(substeps: int) -> tuple[np.float32, np.float32]:
    """Per-substep dt and 1/dt in FP32, as `REFERENCE_FRAME_DELTA_SECS / s` (cloth_compute.rs:438-439)."""
    dt = np.float32(FRAME_DT / np.float32(substeps))
    return dt, np.float32(np.float32(1.0) / dt)


def config0_sheet(seed: int = 0) -> ClothSpec:
    """32x32 sheet, 1 m, two corners pinned, plain Jacobi with degree-averaged corrections."""
    return make_sheet(32, 1.0, 1.0, "corners", seed=seed)


def config1_sheet(seed: int = 1) -> ClothSpec:
    """256x256 sheet, 2 m, whole top edge pinned, colored Gauss-Seidel, damping 0.01."""
    return make_sheet(256, 2.0, 1.0, "top_edge", seed=seed)


def config2_sheet(seed: int = 2, side: int = 512) -> ClothSpec:
    """512x512 sheet, 2 m, unpinned, 1 m above the ground, folding under a smooth random velocity field."""
    vel = fourier_velocity(side, 4, 0.5, seed)
    return make_sheet(side, 2.0, 1.0, "none", jitter=0.0, seed=seed, velocity=vel)


def sheet_triangles(s: int) -> np.ndarray:
    """Two render triangles per quad of an s×s sheet (vertex r*s + c), counter-clockwise seen from +y."""
    r, c = np.meshgrid(np.arange(s - 1), np.arange(s - 1), indexing="ij")
    i = (r * s + c).ravel()
    t = np.stack([np.stack([i, i + s, i + 1], 1), np.stack([i + 1, i + s, i + s + 1], 1)], 1)
    return t.reshape(-1, 3).astype(np.uint32)


def config3_batch(seed: int = 3, count: int = 256, side_lo: int = 16, side_hi: int = 192) -> list[ClothSpec]:
    """`count` square cloths, side uniform in [side_lo, side_hi] vertices, random pin pattern and log-uniform
    stretch compliance in [1e-8, 1e-3]; shear and bend as config 0."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(side_lo, side_hi + 1, size=count)
    pins = rng.integers(0, 2, size=count)
    comps = 10.0 ** rng.uniform(-8.0, -3.0, size=count)
    return [make_sheet(int(s), 1.0, 1.0, "corners" if p == 0 else "top_edge", seed=seed * 100003 + k,
                       stretch_comp=float(cmp)) for k, (s, p, cmp) in enumerate(zip(sides, pins, comps))]


def solver_params(substeps: int = 10, iterations: int = 10, omega: float = 1.0, drag: float = 0.0) -> dict:
    dt, inv_dt = substep_dt(substeps)
    return dict(dt=float(dt), inv_dt=float(inv_dt), jacobi_omega=omega, inner_iterations=iterations,
                gravity=(0.0, -9.81, 0.0), grab_idx=-1, grab_active=0, grab_target=(0.0, 0.0, 0.0),
                grab_stiffness=0.0, linear_drag_per_sec=drag)
