"""Failure detection on the GPU without faulting it: bounded waits and host-injected bad state."""
import numpy as np
import pytest

from bevy_xpbd_b200 import _native as N
from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from tests.helpers import gpu_sim, params_for

pytestmark = pytest.mark.gpu


def _plug(solver=P.SOLVER_JACOBI, **kw):
    sp = wl.make_sheet(kw.pop("side", 24), 1.0, 1.0, "corners", seed=1)
    cfg = P.ClothSimConfig(solver=solver, relaxation=P.RELAX_AVERAGE if solver == 0 else P.RELAX_OMEGA,
                           solve_substeps=10, **kw)
    return sp, gpu_sim(sp, params_for(10, 10, 1.0), cfg)


@pytest.mark.parametrize("solver,kw", [(P.SOLVER_JACOBI, dict(jacobi_kernel=3)), (P.SOLVER_GAUSS_SEIDEL, {}),
                                       (P.SOLVER_GAUSS_SEIDEL, dict(side=128, gs_strips=4, cluster_ctas=16))],
                         ids=["jacobi_rows", "gauss_seidel", "gauss_seidel_strips"])
def test_grid_barrier_wait_times_out_and_context_recovers(solver, kw):
    """A launch whose wait can never complete — the grid barrier expects one block more than exists, or one strip CTA
    starts from a step count its neighbours never reach: the wait ends after 20 ms with XPBD_ERR_BARRIER_TIMEOUT,
    and the context keeps working afterwards."""
    sp, plug = _plug(solver, **kw)
    if kw.get("gs_strips"):
        assert plug.stats()["solver_kernel"] == 9
    st = plug.debug_force_barrier_timeout(20.0)
    assert st == N.ERR_BARRIER_TIMEOUT, plug._L.xpbd_last_error(plug._h).decode()
    plug.reset()
    plug.step(frames=2)
    x = plug.positions()
    assert np.all(np.isfinite(x))


def test_nonfinite_state_is_reported():
    """A NaN written through the C ABI is caught on the device and reported as XPBD_ERR_DEVICE_NONFINITE."""
    sp, plug = _plug()
    x = sp.positions.copy()
    x[100, 1] = np.nan
    plug.write_state(x)
    plug.step(frames=1)
    with pytest.raises(N.XpbdError) as e:
        plug.positions()
    assert e.value.status == N.ERR_DEVICE_NONFINITE
    plug.reset()
    plug.step(frames=1)
    assert np.all(np.isfinite(plug.positions()))


def test_invalid_inputs_rejected_before_launch():
    plug = P.ClothComputePlugin(0)
    x = np.zeros((3, 3), np.float32)
    with pytest.raises(N.XpbdError) as e:
        plug.add_cloth(x, np.ones(3, np.float32), [0], [7], [1.0], [0.0])
    assert e.value.status == N.ERR_INDEX_RANGE
    with pytest.raises(N.XpbdError) as e:
        plug.step(frames=1)
    assert e.value.status == N.ERR_STATE
