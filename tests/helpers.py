"""Shared test helpers: run the same seeded cloth through the CUDA path (C ABI) and through the CPU oracle."""
from __future__ import annotations

import numpy as np

from bevy_xpbd_b200 import plugin as P
from oracle import oracle as orc


def oracle_params(params: P.XpbdCpuTimeStepParams, cfg: P.ClothSimConfig) -> dict:
    d = params.as_dict()
    d["grab_active"] = int(bool(d["grab_active"]))
    d.update(solver=cfg.solver, relaxation=cfg.relaxation, lambda_mode=cfg.lambda_mode, collision=cfg.collision,
             thickness=cfg.thickness, coll_scale=cfg.coll_scale, hash_cell=cfg.hash_cell,
             ground_enabled=int(cfg.ground_enabled), ground_y=cfg.ground_y, tolerance=cfg.tolerance,
             warm_start=int(cfg.warm_start != 0))
    return d


def oracle_sim(spec, params, cfg, fp64=False, order_by_index=False, omp=False):
    """Oracle fed the batch-sorted constraints (as finalize_cloth_mesh hands them to the solver). omp=True builds it
    on the OpenMP library (independent loops and each color batch in parallel; bit-identical to the serial build,
    tests/test_host_cpu.py), for the full-size comparisons."""
    perm, _, offs = orc.partition(spec.num_particles, spec.constraint_i, spec.constraint_j, order_by_index)
    if omp:
        orc.select("omp")
    try:
        s = orc.OracleSim(spec.positions, spec.inv_mass, spec.constraint_i[perm], spec.constraint_j[perm],
                          spec.rest_len[perm], spec.compliance[perm], v=spec.velocities,
                          rest_pos=spec.rest_positions, ctype=spec.constraint_type[perm], fp64=fp64)
    finally:
        if omp:
            orc.select("serial")
    s.set_params(oracle_params(params, cfg))
    if omp:
        s.set_batches(offs)
    return s


def gpu_sim(specs, params, cfg, order=P.ORDER_COLOR_REFERENCE):
    plug = P.ClothComputePlugin(0)
    for sp in (specs if isinstance(specs, list) else [specs]):
        plug.add_spec(sp, order)
    plug.commit()
    plug.set_params(params, cfg)
    return plug


def params_for(substeps=10, iterations=10, omega=1.0, drag=0.0, gravity=(0.0, -9.81, 0.0)):
    dt = np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(substeps)
    dt = np.float32(dt)
    return P.XpbdCpuTimeStepParams(float(dt), float(np.float32(1.0) / dt), omega, iterations, gravity,
                                   linear_drag_per_sec=drag)


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


def folded_state(sp, gap=0.03):
    """The sheet folded in half along its middle row: the upper half lies `gap` above the lower half."""
    s = sp.side
    x = sp.positions.reshape(s, s, 3).astype(np.float64).copy()
    zf = x[s // 2, 0, 2]
    x[s // 2:, :, 2] = 2 * zf - x[s // 2:, :, 2]
    x[s // 2:, :, 1] += gap
    return x.reshape(-1, 3).astype(np.float32)
