"""The OpenMP build of the oracle (oracle/liboracle_omp.so) gives the serial build's results bit for bit.

The full-size GPU comparisons use the OpenMP build as their checker, so that 256x256 x 120 frames, the 256-cloth batch
and the 512x512 collision sheet finish in seconds: its parallel loops are the reference's independent ones (per
constraint, per particle, per color batch of the Gauss-Seidel sweep, per particle of the hashed collision query), so
each value is computed by the same operations in the same order.
"""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from tests.helpers import folded_state, oracle_sim, params_for


def _cfg(**kw):
    c = P.ClothSimConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


CASES = [
    ("jacobi_avg", lambda: wl.make_sheet(40, 1.0, 1.0, "corners", seed=7, stretch_comp=1e-7),
     dict(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE), 30, 0.0),
    ("gauss_seidel", lambda: wl.make_sheet(48, 2.0, 1.0, "top_edge", seed=8),
     dict(solver=P.SOLVER_GAUSS_SEIDEL), 30, 0.01),
    ("collision", lambda: wl.config2_sheet(seed=2, side=40),
     dict(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, collision=P.COLLISION_RING_FILTER, thickness=0.05,
          coll_scale=0.38, hash_cell=0.1, hash_table_bits=20, ring_depth=2, ground_enabled=True, ground_y=0.0),
     100, 0.0),
]


@pytest.mark.parametrize("name,make,kw,substeps,drag", CASES, ids=[c[0] for c in CASES])
def test_openmp_oracle_equals_serial_oracle(name, make, kw, substeps, drag):
    sp = make()
    prm = params_for(10, 10, 1.0, drag=drag)
    cfg = _cfg(solve_substeps=10, **kw)
    a = oracle_sim(sp, prm, cfg)
    b = oracle_sim(sp, prm, cfg, omp=True)
    if kw.get("collision"):  # start folded so that the layers collide
        xf = folded_state(sp)
        for s in (a, b):
            s.set_state(xf, np.zeros_like(xf))
        assert len(a.collision_pairs()) > 500
    a.substeps(substeps)
    b.substeps(substeps)
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    if kw.get("collision"):
        assert np.array_equal(a.collision_pairs(), b.collision_pairs())


def test_oracle_wind_changes_only_the_windy_run():
    """The wind extension of the oracle's predict: off (drag 0) leaves the reference result, on moves the sheet."""
    from tests.helpers import oracle_params
    sp = wl.make_sheet(12, 1.0, 1.0, "top_edge", seed=3)
    prm = params_for(10, 10, 1.0)
    cfg = _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    a = oracle_sim(sp, prm, cfg)
    b = oracle_sim(sp, prm, cfg)
    c = oracle_sim(sp, prm, cfg)
    d = oracle_params(prm, cfg)
    b.set_params(dict(d, wind=(4.0, 0.0, 0.0), wind_drag=0.0))
    c.set_params(dict(d, wind=(4.0, 0.0, 0.0), wind_drag=1.0))
    for s in (a, b, c):
        s.substeps(20)
    assert np.array_equal(a.state()[0], b.state()[0])
    assert np.abs(a.state()[0] - c.state()[0]).max() > 1e-4
    assert c.state()[0][:, 0].mean() > a.state()[0][:, 0].mean()
