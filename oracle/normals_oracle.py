"""CPU oracle of the vertex normals — test infrastructure only (imported by tests/, never by the product).

Restates accumulate_normals / finalize_normals (src/shaders/cloth_sim_jacobi.wgsl:492-547) in float32 numpy:
per triangle (p0, p1, p2) the cross product c = cross(p1 - p0, p2 - p0), each component rounded per operation with
no fused multiply-add (x = e0.y·e1.z − e0.z·e1.y, ...), scaled by 33333 and truncated toward zero to i32 (saturating,
NaN → 0); the three vertices sum these integers with i32 wrap-around; then n = f32(sum) / 33333 and, when
|n| = sqrt((x² + y²) + z²) > 1e-8, n / |n| per component, else (0, 1, 0).

The shader's integer sums are exact, so that part is pinned by construction; its float steps are WGSL operations
whose rounding (and fusing) is up to the GPU compiler, so ulp-level parity with a wgpu run is unpinned — the CUDA
kernel is held to this restatement bit for bit.
"""
from __future__ import annotations

import numpy as np

FIX = np.float32(33333.0)


def _fixed(c):
    c = (np.asarray(c, np.float32) * FIX).astype(np.float64)
    c = np.where(np.isnan(c), 0.0, c)
    return np.clip(np.trunc(c), -2.0**31, 2.0**31 - 1).astype(np.int64)  # toward zero, saturating


def vertex_normals(x, tris) -> np.ndarray:
    f32 = np.float32
    x = np.asarray(x, f32).reshape(-1, 3)
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    p0, p1, p2 = x[t[:, 0]], x[t[:, 1]], x[t[:, 2]]
    e0 = p1 - p0
    e1 = p2 - p0
    c = np.stack([e0[:, 1] * e1[:, 2] - e0[:, 2] * e1[:, 1],
                  e0[:, 2] * e1[:, 0] - e0[:, 0] * e1[:, 2],
                  e0[:, 0] * e1[:, 1] - e0[:, 1] * e1[:, 0]], axis=1).astype(f32)
    q = _fixed(c)
    acc = np.zeros((len(x), 3), np.int64)
    for k in range(3):
        np.add.at(acc, t[:, k], q)
    acc = ((acc + 2**31) % 2**32 - 2**31).astype(np.int64)  # i32 wrap-around
    n = acc.astype(f32) / FIX
    ln = np.sqrt((n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]).astype(f32)
    out = np.zeros_like(n)
    good = ln > f32(1e-8)
    out[good] = n[good] / ln[good, None]
    out[~good] = np.array([0.0, 1.0, 0.0], f32)
    return out
