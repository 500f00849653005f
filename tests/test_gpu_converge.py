"""Convergence solve (extension: Jacobi iterated until the max pre-update constraint residual |C + α̃λ|/rest is at or
below the tolerance, λ kept across the iterations of a substep) through the C ABI against the oracle's
substep_converge: positions bit-exact, the same number of update passes per substep, the same warm-start fallbacks."""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import gpu_sim, max_abs, oracle_sim, params_for

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    # 2e-2 on this sheet: early substeps stop after a few passes, later ones need tens (a mix the parity must cover)
    c = P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=4, tolerance=2e-2)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _sheet():
    sp = wl.make_sheet(24, 1.0, 1.0, "top_edge", seed=5)
    return sp, params_for(4, 160, 1.0, drag=0.01)


def _perm(sp):
    perm, _, _ = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j, False)
    return perm


def test_converge_plain_bit_exact():
    sp, prm = _sheet()
    cfg = _cfg()
    plug = gpu_sim(sp, prm, cfg)
    o = oracle_sim(sp, prm, cfg)
    its = []
    for frame in range(3):
        plug.step(frames=1)
        it, fb = o.substeps_converge(cfg.solve_substeps)
        its += [int(k) for k in it]
        assert max_abs(plug.positions(), o.state()[0]) == 0.0, frame
        assert max_abs(plug.velocities(), o.state()[1]) == 0.0, frame
    st = plug.stats()
    assert st["converge_substeps"] == 12
    assert st["converge_iterations"] == sum(its)
    assert st["converge_max_iterations"] == max(its)
    assert min(its) < max(its) < prm.inner_iterations   # early exits of different lengths
    # λ after the last substep, input order
    perm = _perm(sp)
    lam_o = np.zeros(len(perm))
    lam_o[perm] = o.lambdas()
    assert np.array_equal(plug.lambdas().astype(np.float64), lam_o)


def test_converge_given_warm_start_bit_exact_and_fallback():
    sp, prm = _sheet()
    perm = _perm(sp)
    cfg = _cfg(warm_start=P.WARM_GIVEN)
    # a good λ0: the converged λ of a first plain substep from the same state, slightly off
    probe = oracle_sim(sp, prm, _cfg())
    probe.substeps_converge(1)
    good = (probe.lambdas() * 0.9).astype(np.float32)     # oracle (batch) order
    for lam0_o, expect_fallback in ((good, 0), (np.full_like(good, 5.0), 1)):
        plug = gpu_sim(sp, prm, cfg)
        lam0_in = np.zeros_like(lam0_o)
        lam0_in[perm] = lam0_o
        plug.set_warm_lambda(lam0_in)
        o = oracle_sim(sp, prm, cfg)
        o.set_warm_lambda(lam0_o)
        plug.substep(1)
        it, fb = o.substeps_converge(1)
        assert int(fb[0]) == expect_fallback
        assert plug.stats()["warm_start_fallbacks"] == expect_fallback
        assert plug.stats()["converge_iterations"] == int(it[0])
        assert max_abs(plug.positions(), o.state()[0]) == 0.0


def test_converge_previous_lambda_warm_start_bit_exact():
    sp, prm = _sheet()
    perm = _perm(sp)
    cfg = _cfg(warm_start=P.WARM_PREVIOUS)
    plug = gpu_sim(sp, prm, cfg)
    o = oracle_sim(sp, prm, cfg)
    o.set_warm_lambda(np.zeros(len(perm), np.float32))
    its, fbs = [], []
    for s in range(8):
        plug.substep(1)
        it, fb = o.substeps_converge(1)
        its.append(int(it[0]))
        fbs.append(int(fb[0]))
        o.set_warm_lambda(o.lambdas().astype(np.float32))
        assert max_abs(plug.positions(), o.state()[0]) == 0.0, s
    st = plug.stats()
    assert st["converge_iterations"] == sum(its)
    assert st["warm_start_fallbacks"] == sum(fbs)


def test_converge_rejects_unsupported_modes():
    sp, prm = _sheet()
    plug = gpu_sim(sp, prm, _cfg())
    with pytest.raises(P.XpbdError):
        plug.set_params(prm, _cfg(solver=P.SOLVER_GAUSS_SEIDEL))
    with pytest.raises(P.XpbdError):
        plug.set_params(prm, _cfg(collision=P.COLLISION_REST_FILTER))
    with pytest.raises(P.XpbdError):       # learned start without a network
        plug.set_params(prm, _cfg(warm_start=P.WARM_LEARNED))


def test_converge_batched_cloths_stop_independently():
    """Three cloths in one context: each takes the passes it takes alone (per-cloth early exit), bit-exact."""
    specs = [wl.make_sheet(s, 1.0, 1.0, "top_edge", seed=5 + s) for s in (12, 24, 16)]
    prm = params_for(4, 160, 1.0, drag=0.01)
    for warm in (P.WARM_NONE, P.WARM_PREVIOUS):
        cfg = _cfg(warm_start=warm)
        plug = gpu_sim(specs, prm, cfg)
        oracles = [oracle_sim(sp, prm, cfg) for sp in specs]
        if warm:
            for sp, o in zip(specs, oracles):
                o.set_warm_lambda(np.zeros(len(sp.constraint_i), np.float32))
        tot, seen = 0, set()
        for s in range(8):
            plug.substep(1)
            per = plug.converge_cloth_iterations()
            for c, o in enumerate(oracles):
                it, _ = o.substeps_converge(1)
                if warm:
                    o.set_warm_lambda(o.lambdas().astype(np.float32))
                assert int(per[c]) == int(it[0]), (warm, s, c)
                tot += int(it[0])
                seen.add(int(it[0]))
                assert max_abs(plug.positions(c), o.state()[0]) == 0.0, (warm, s, c)
        st = plug.stats()
        assert st["converge_iterations"] == tot
        assert st["converge_substeps"] == 8 * len(specs)
        assert len(seen) > 2          # the cloths stopped after different numbers of passes
