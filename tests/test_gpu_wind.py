"""Per-cloth wind (extension, used to generate the warm-start training data): after gravity, the predicted velocity
relaxes toward the wind velocity, v += (wind - v) * (drag * dt). Every solver execution against the oracle, which
applies the same step in its predict_particle (xpbd_cpu.rs:38-65 plus the wind line), bit for bit."""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from tests.helpers import gpu_sim, max_abs, oracle_params, oracle_sim, params_for

pytestmark = pytest.mark.gpu

WIND = [(3.0, 0.0, -1.5), (0.0, 0.0, 0.0), (-1.0, 0.5, 4.0)]
DRAG = [0.8, 0.0, 2.5]


def _cfg(**kw):
    c = P.ClothSimConfig()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("solver,kernel,cluster", [
    (P.SOLVER_JACOBI, 4, 0), (P.SOLVER_JACOBI, 3, 0), (P.SOLVER_JACOBI, 5, 0), (P.SOLVER_GAUSS_SEIDEL, 0, 8),
    (P.SOLVER_GAUSS_SEIDEL, 0, 1)],
    ids=["cloth_resident", "rows", "small_batch", "gs_cluster", "gs_grid"])
def test_per_cloth_wind_bit_exact(solver, kernel, cluster):
    specs = [wl.make_sheet(s, 1.0, 1.0, "top_edge", seed=70 + k) for k, s in enumerate([30, 24, 18])]
    prm = params_for(10, 10, 1.0, drag=0.2)
    cfg = _cfg(solver=solver, relaxation=P.RELAX_AVERAGE if solver == P.SOLVER_JACOBI else P.RELAX_OMEGA,
               solve_substeps=10, jacobi_kernel=kernel, cluster_ctas=cluster)
    plug = gpu_sim(specs, prm, cfg)
    want = {(P.SOLVER_JACOBI, 4): 7, (P.SOLVER_JACOBI, 3): 5, (P.SOLVER_JACOBI, 5): 8}
    if solver == P.SOLVER_JACOBI:
        assert plug.stats()["solver_kernel"] == want[(solver, kernel)]
    for k in range(3):
        plug.set_cloth_wind(k, WIND[k], DRAG[k])
    plug.step(frames=4)
    for k, sp in enumerate(specs):
        o = oracle_sim(sp, prm, cfg)
        prm_o = oracle_params(prm, cfg)
        prm_o.update(wind=WIND[k], wind_drag=DRAG[k])
        o.set_params(prm_o)
        o.substeps(40)
        xo, vo = o.state()
        assert max_abs(plug.positions(k), xo) == 0.0, k
        assert max_abs(plug.velocities(k), vo) == 0.0, k
    # the wind moved the sheets it blows on
    calm = gpu_sim(specs, prm, cfg)
    calm.step(frames=4)
    assert max_abs(plug.positions(0), calm.positions(0)) > 1e-3
    assert max_abs(plug.positions(1), calm.positions(1)) == 0.0
