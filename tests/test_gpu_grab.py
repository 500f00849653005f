"""Per-cloth kinematic grabs (extension of the reference's single mouse grab, xpbd_cpu.rs:56-63): each cloth of a
batch follows the oracle run of that cloth alone with the same grab, bit for bit, on the Jacobi and Gauss–Seidel
paths; releasing a grab returns the cloth to the ungrabbed oracle."""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from tests.helpers import max_abs, oracle_params, oracle_sim, params_for

pytestmark = pytest.mark.gpu

GRABS = {0: (5, (0.1, 1.4, 0.2), 0.28), 2: (17, (-0.3, 0.6, 0.4), 0.45)}


def _cfg(**kw):
    c = P.ClothSimConfig(solve_substeps=10)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("cfg", [
    _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, jacobi_kernel=3),
    _cfg(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, jacobi_kernel=2),
    _cfg(solver=P.SOLVER_GAUSS_SEIDEL, cluster_ctas=1),
], ids=["jacobi_rows", "jacobi_patches", "gs_grid"])
def test_per_cloth_grabs_bit_exact(cfg):
    specs = [wl.make_sheet(20, 1.0, 1.0, "top_edge", seed=1), wl.make_sheet(24, 1.0, 1.0, "corners", seed=2),
             wl.make_sheet(16, 1.0, 1.0, "top_edge", seed=3)]
    prm = params_for(10, 10, 1.0, drag=0.01)
    plug = P.ClothComputePlugin(0)
    for sp in specs:
        plug.add_spec(sp)
    plug.commit()
    plug.set_params(prm, cfg)
    for c, (v, t, k) in GRABS.items():
        plug.set_cloth_grab(c, v, t, k)
    plug.step(frames=3)
    oracles = []
    for c, sp in enumerate(specs):
        p = params_for(10, 10, 1.0, drag=0.01)
        if c in GRABS:
            v, t, k = GRABS[c]
            p.grab_idx, p.grab_active, p.grab_target, p.grab_stiffness = v, True, t, k
        o = oracle_sim(sp, p, cfg)
        o.substeps(30)
        oracles.append(o)
        assert max_abs(plug.positions(c), o.state()[0]) == 0.0, c
    plug.set_cloth_grab(0, None)
    plug.step(frames=1)
    for c, (sp, o) in enumerate(zip(specs, oracles)):
        if c == 0:
            o.set_params(oracle_params(prm, cfg))
        o.substeps(10)
        assert max_abs(plug.positions(c), o.state()[0]) == 0.0, c


def test_cluster_gs_grab_bit_exact():
    sp = wl.make_sheet(64, 2.0, 1.0, "top_edge", seed=4)
    prm = params_for(10, 10, 1.0, drag=0.01)
    cfg = _cfg(solver=P.SOLVER_GAUSS_SEIDEL, cluster_ctas=16)
    plug = P.ClothComputePlugin(0)
    plug.add_spec(sp)
    plug.commit()
    plug.set_params(prm, cfg)
    assert plug.stats()["cluster_ctas"] == 16
    plug.set_cloth_grab(0, 2000, (0.3, 1.2, 0.5), 0.45)
    plug.step(frames=2)
    p = params_for(10, 10, 1.0, drag=0.01)
    p.grab_idx, p.grab_active, p.grab_target, p.grab_stiffness = 2000, True, (0.3, 1.2, 0.5), 0.45
    o = oracle_sim(sp, p, cfg)
    o.substeps(20)
    assert max_abs(plug.positions(), o.state()[0]) == 0.0


def test_grab_argument_errors():
    sp = wl.make_sheet(8, 1.0, 1.0, "corners", seed=3)
    plug = P.ClothComputePlugin(0)
    plug.add_spec(sp)
    plug.commit()
    with pytest.raises(P.XpbdError):
        plug.set_cloth_grab(0, 64, (0, 0, 0), 0.3)
    with pytest.raises(P.XpbdError):
        plug.set_cloth_grab(1, 3, (0, 0, 0), 0.3)
