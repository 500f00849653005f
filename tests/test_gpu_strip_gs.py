"""Colored Gauss–Seidel over several thread-block clusters (kernel id 9, `gs_strips`): particles joined to another
strip by a constraint live in global memory and are ordered across clusters by per-CTA step flags. Bit for bit
against the CPU oracle of xpbd_cpu.rs (colors are particle-disjoint, so the sweep equals the sequential one)."""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from tests.helpers import gpu_sim, max_abs, oracle_params, oracle_sim, params_for

pytestmark = pytest.mark.gpu

STRIPS = 9  # kernel id


def _cfg(**kw):
    c = P.ClothSimConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("side,strips,cluster,frames", [(256, 8, 8, 6), (96, 4, 8, 6), (256, 4, 16, 3),
                                                        (130, 2, 16, 5)],
                         ids=["256_8x8", "96_4x8", "256_4x16", "130_2x16"])
def test_strip_gauss_seidel_bit_exact(side, strips, cluster, frames):
    sp = wl.make_sheet(side, 2.0, 1.0, "top_edge", seed=80 + side)
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10, gs_strips=strips, cluster_ctas=cluster)
    plug = gpu_sim(sp, prm, cfg)
    st = plug.stats()
    assert st["solver_kernel"] == STRIPS and st["grid_blocks"] == strips * cluster
    plug.step(frames=frames)
    o = oracle_sim(sp, prm, cfg, omp=True)
    o.substeps(10 * frames)
    xo, vo = o.state()
    assert max_abs(plug.positions(), xo) == 0.0
    assert max_abs(plug.velocities(), vo) == 0.0
    plug.step(frames=1)  # a later launch starts from the step flags the previous one left
    o.substeps(10)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


def test_strip_gauss_seidel_batch_wind_grab_and_substeps():
    specs = [wl.make_sheet(s, 1.0, 1.0, "corners" if k % 2 else "top_edge", seed=90 + k)
             for k, s in enumerate([90, 40, 120, 64])]
    prm = params_for(10, 10, 1.0, drag=0.2)
    prm.grab_idx, prm.grab_active, prm.grab_target, prm.grab_stiffness = 3000, True, (0.2, 0.8, 0.0), 0.45
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10, gs_strips=4, cluster_ctas=16)
    plug = gpu_sim(specs, prm, cfg)
    assert plug.stats()["solver_kernel"] == STRIPS
    plug.set_cloth_wind(2, (2.0, 0.0, 1.0), 1.5)
    plug.step(frames=3)
    plug.substep(4)
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        d = oracle_params(prm, cfg)
        if k != 0:
            d.update(grab_active=0)  # the context grab names a vertex of the first cloth
        if k == 2:
            d.update(wind=(2.0, 0.0, 1.0), wind_drag=1.5)
        o.set_params(d)
        o.substeps(34)
        assert max_abs(plug.positions(k), o.state()[0]) == 0.0, k


def test_strips_fall_back_when_the_shape_does_not_fit():
    sp = wl.make_sheet(12, 1.0, 1.0, "top_edge", seed=3)
    prm = params_for(10, 10, 1.0)
    plug = gpu_sim(sp, prm, _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10, gs_strips=8))
    assert plug.stats()["solver_kernel"] != STRIPS
    plug.step(frames=1)
    o = oracle_sim(sp, prm, _cfg(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10))
    o.substeps(10)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0
