"""Learned λ warm start (extension) through the C ABI against the numpy oracle of the network (oracle/mlp_oracle.py)
and the C++ oracle of the convergence solve.

Tolerances (the network runs on BF16 tensor-core tiles with FP32 accumulation; the oracle emulates every bfloat16
rounding point and accumulates in FP64, so what remains is accumulation order, the device's fast exp and rare
one-ulp bfloat16 flips of a hidden activation):
* forward: max |y_gpu - y_oracle| <= 2e-2 · max(1, std(y)), mean <= 1e-3 · max(1, std(y));
* gradients: per parameter block ||g_gpu - g_oracle|| <= 2e-2 · ||g_oracle|| (the device also rounds dz to bf16);
* features: FP32 restatement, rtol 1e-5 (FMA contraction on the device), the one-hot / pin flags exact;
* the learned solve itself: bit-exact against the oracle run with the same λ0 (WARM_GIVEN path of the oracle).
"""
import numpy as np
import pytest

from bevy_xpbd_b200 import plugin as P
from bevy_xpbd_b200 import workloads as wl
from oracle import mlp_oracle as MO
from oracle import oracle as orc
from tests.helpers import gpu_sim, max_abs, oracle_sim, params_for

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    c = P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=4, tolerance=1e-4)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _sheet(s=24, seed=5):
    sp = wl.make_sheet(s, 1.0, 1.0, "top_edge", seed=seed)
    return sp, params_for(4, 160, 1.0, drag=0.01)


def _perm(sp):
    perm, _, _ = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j, False)
    return perm


def _random_features(rng, n):
    f = rng.normal(size=(n, 9)).astype(np.float32)
    f[:, 5:8] = 0.0
    f[np.arange(n), 5 + rng.integers(0, 3, n)] = 1.0
    f[:, 8] = (rng.random(n) < 0.1).astype(np.float32)
    return f


def _random_norm(rng):
    nm = np.zeros(20, np.float32)
    nm[:5] = rng.normal(size=5) * 0.1
    nm[9:14] = 0.5 + rng.random(5)
    nm[5:9] = 0.0
    nm[14:18] = 1.0
    nm[18], nm[19] = 0.1, 2.0
    return nm


def test_mlp_init_layout():
    sp, prm = _sheet(16)
    plug = gpu_sim(sp, prm, _cfg())
    plug.mlp_init(seed=3, capacity=1024)
    p, nm = plug.mlp_params()
    w1, b1, w2, b2, w3, b3 = MO.unpack(p)
    assert p.shape == (MO.N_PARAMS,)
    assert np.all(np.abs(w1) <= 1 / 3 + 1e-6) and np.abs(w1).max() > 0.2
    assert np.all(np.abs(w2) <= 1 / 8 + 1e-6) and np.all(np.abs(w3) <= 1 / 8 + 1e-6)
    assert not b1.any() and not b2.any() and b3 == 0.0
    assert np.array_equal(nm[9:18], np.ones(9, np.float32)) and nm[19] == 1.0
    plug.mlp_init(seed=3, capacity=1024)
    assert np.array_equal(plug.mlp_params()[0], p)            # seeded


@pytest.mark.parametrize("n", [1, 16, 1001])
def test_mlp_forward_matches_oracle(n):
    rng = np.random.default_rng(n)
    sp, prm = _sheet(16)
    plug = gpu_sim(sp, prm, _cfg())
    plug.mlp_init(seed=1, capacity=16)
    params = (rng.normal(size=MO.N_PARAMS) * 0.3).astype(np.float32)
    norm = _random_norm(rng)
    plug.mlp_set_params(params, norm)
    f = _random_features(rng, n)
    y = plug.mlp_eval(f)
    y_ref = MO.forward(params, norm, f)
    scale = max(1.0, float(np.std(y_ref)) if n > 1 else abs(float(y_ref[0])))
    err = np.abs(y.astype(np.float64) - y_ref)
    assert err.max() <= 2e-2 * scale
    assert err.mean() <= 1e-3 * scale


def test_mlp_gradients_match_oracle():
    rng = np.random.default_rng(7)
    sp, prm = _sheet(16)
    plug = gpu_sim(sp, prm, _cfg())
    plug.mlp_init(seed=2, capacity=16)
    p, _ = plug.mlp_params()
    norm = _random_norm(rng)
    plug.mlp_set_params(p, norm)
    f = _random_features(rng, 515)
    t = (rng.normal(size=515) * 2.0 + 0.1).astype(np.float32)
    g, loss = plug.mlp_gradients(f, t)
    g_ref, loss_ref = MO.gradients(p, norm, f, t)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    blocks = {"w1": (0, 576), "b1": (576, 640), "w2": (640, 4736), "b2": (4736, 4800), "w3": (4800, 4864),
              "b3": (4864, 4865)}
    for name, (a, b) in blocks.items():
        ref = g_ref[a:b]
        assert np.linalg.norm(g[a:b] - ref) <= 2e-2 * np.linalg.norm(ref) + 1e-9, name


def test_collect_features_targets_match_oracle():
    sp, prm = _sheet(20)
    cfg = _cfg()
    perm = _perm(sp)
    E = len(sp.constraint_i)
    plug = gpu_sim(sp, prm, cfg)
    plug.mlp_init(seed=1, capacity=4 * E)
    o = oracle_sim(sp, prm, cfg)
    lam_prev = np.zeros(E, np.float32)
    feats, tgts = [], []
    for _ in range(2):
        pred = o.predicted()
        v = o.state()[1]
        feats.append(MO.features(pred, v, sp.constraint_i, sp.constraint_j, sp.rest_len, sp.compliance,
                                 sp.constraint_type, sp.inv_mass, lam_prev, prm.dt, prm.inv_dt))
        plug.mlp_collect(1, stride=1)
        o.substeps_converge(1)
        lam = np.zeros(E, np.float32)
        lam[perm] = o.lambdas()
        tgts.append(MO.targets(lam, sp.rest_len, sp.compliance, sp.inv_mass, sp.constraint_i, sp.constraint_j,
                               prm.inv_dt))
        lam_prev = lam
        assert max_abs(plug.positions(), o.state()[0]) == 0.0     # collection runs the plain convergence solve
    f, t = plug.mlp_dataset()
    assert f.shape == (2 * E, 9)
    fr = np.concatenate(feats)
    tr = np.concatenate(tgts)
    np.testing.assert_array_equal(f[:, 5:], fr[:, 5:])
    np.testing.assert_array_equal(f[:, 4], fr[:, 4])
    # f0: |xi - xj| may differ by an ulp (FMA contraction of the squared length on the device) → 4 ulp / rest
    ratio = float((1.0 + np.abs(fr[:, 0])).max())
    np.testing.assert_allclose(f[:, 0], fr[:, 0], rtol=0, atol=4 * np.finfo(np.float32).eps * ratio)
    for k in range(1, 4):
        sc = max(1e-6, float(np.abs(fr[:, k]).max()))
        np.testing.assert_allclose(f[:, k], fr[:, k], rtol=1e-5, atol=2e-6 * sc, err_msg=f"feature {k}")
    np.testing.assert_allclose(t, tr, rtol=1e-5, atol=1e-6 * float(np.abs(tr).max()))
    # stride sampling: every 3rd constraint, offsets rotating per substep
    plug2 = gpu_sim(sp, prm, cfg)
    plug2.mlp_init(seed=1, capacity=4 * E)
    plug2.mlp_collect(1, stride=3)
    f2, _ = plug2.mlp_dataset()
    np.testing.assert_array_equal(f2, f[: E][0::3])


def _trained(sp, prm, cfg, substeps=24, steps=400, seed=11):
    plug = gpu_sim(sp, prm, cfg)
    plug.mlp_init(seed=seed, capacity=1 << 18)
    plug.mlp_collect(substeps, stride=1)
    plug.mlp_fit_normalization()
    losses = plug.mlp_train(steps, batch=2048, lr=2e-3, seed=seed)
    return plug, losses


def test_adam_step_matches_oracle():
    sp, prm = _sheet(16)
    cfg = _cfg()
    plug = gpu_sim(sp, prm, cfg)
    plug.mlp_init(seed=4, capacity=1 << 14)
    n = plug.mlp_collect(2, stride=1)
    plug.mlp_fit_normalization()
    f, t = plug.mlp_dataset()
    p0, norm = plug.mlp_params()
    lr = 1e-3
    losses = plug.mlp_train(1, batch=512, lr=lr, seed=9)
    p1, _ = plug.mlp_params()
    idx = MO.xorshift_indices(9, 512, n)
    g_ref, loss_ref = MO.gradients(p0, norm, f[idx], t[idx])
    assert abs(losses[0] - loss_ref) <= 1e-3 * max(loss_ref, 1e-6)
    p1_ref, _, _ = MO.adam(p0, np.zeros_like(p0), np.zeros_like(p0), g_ref, 1, lr)
    big = np.abs(g_ref) > 1e-2 * np.abs(g_ref).max()
    assert big.sum() > 100
    np.testing.assert_allclose(p1[big], p1_ref[big], atol=1e-5 * lr * 100)


def test_learned_warm_start_bit_exact_against_oracle_with_same_lambda0():
    sp, prm = _sheet(24)
    cfg = _cfg()
    perm = _perm(sp)
    plug, losses = _trained(sp, prm, cfg, substeps=8, steps=100)
    assert np.all(np.isfinite(losses))
    plug.set_params(prm, _cfg(warm_start=P.WARM_LEARNED))
    o = oracle_sim(sp, prm, _cfg(warm_start=P.WARM_GIVEN))
    x, v = plug.positions(), plug.velocities()
    o.set_state(x, v)
    st0 = plug.stats()
    its, fbs = 0, 0
    for s in range(4):
        lam0 = plug.mlp_predict_lambda()
        assert np.all(np.isfinite(lam0))
        o.set_warm_lambda(lam0[perm])
        plug.substep(1)
        it, fb = o.substeps_converge(1)
        its += int(it[0])
        fbs += int(fb[0])
        assert max_abs(plug.positions(), o.state()[0]) == 0.0, s
        assert max_abs(plug.velocities(), o.state()[1]) == 0.0, s
    st = plug.stats()
    assert st["converge_iterations"] - st0["converge_iterations"] == its
    assert st["warm_start_fallbacks"] - st0["warm_start_fallbacks"] == fbs


def test_learned_warm_start_reduces_iterations(record_property):
    """Train on one batch of config-3 cloths (varied stiffness), then run a different batch plain, previous-λ and learned
    from the same initial state. The learned start needs fewer update passes per cloth-substep than the plain start.
    Against the previous substep's λ — the method the network extends (it is one of its inputs, and the network
    predicts the change over it) — the gain is recorded (passes_gain_over_previous) and the learned start, its predicted
    change shrunk by 0.15 toward the previous multiplier, must not take more passes than previous-λ plus 5 %: on these
    cloths the network adds little to what that input carries."""
    cap = 1024
    prm = params_for(10, cap, 1.0, drag=0.01)
    cfg = _cfg(solve_substeps=10)
    train = wl.config3_batch(seed=31, count=48, side_lo=16, side_hi=96)
    test = wl.config3_batch(seed=32, count=48, side_lo=16, side_hi=96)
    plug = gpu_sim(train, prm, cfg)
    plug.mlp_init(seed=11, capacity=1 << 21)
    plug.mlp_collect(40, stride=28)
    plug.mlp_fit_normalization()
    losses = np.concatenate([plug.mlp_train(1500, batch=4096, lr=2e-3, seed=11),
                             plug.mlp_train(500, batch=4096, lr=3e-4, seed=12)])
    assert np.all(np.isfinite(losses))
    assert losses[-200:].mean() < losses[:20].mean()      # per-batch losses are heavy-tailed: compare means
    params, norm = P.mlp_scale_change(*plug.mlp_params(), 0.15)  # the change shrunk as the bench chooses it
    runs = {}
    for name, warm in (("plain", P.WARM_NONE), ("previous", P.WARM_PREVIOUS), ("learned", P.WARM_LEARNED)):
        q = gpu_sim(test, prm, cfg)
        q.mlp_init(seed=0, capacity=16)
        q.mlp_set_params(params, norm)
        q.set_params(prm, _cfg(solve_substeps=10, warm_start=warm))
        q.step(frames=2)
        st = q.stats()
        runs[name] = st["converge_iterations"] / st["converge_substeps"]
        record_property(f"passes_per_cloth_substep_{name}", runs[name])
    record_property("passes_gain_over_previous", runs["previous"] / runs["learned"])
    record_property("passes_gain_over_plain", runs["plain"] / runs["learned"])
    assert runs["learned"] < runs["plain"]
    assert runs["learned"] <= 1.05 * runs["previous"]


def test_data_parallel_training_step_matches_oracle():
    """The two-call step used for multi-GPU training (minibatch gradient into a caller buffer, then Adam with the
    scaled buffer), run through bevy_xpbd_b200.mlp_train on one GPU, against the oracle's gradient and Adam."""
    from bevy_xpbd_b200 import mlp_train
    sp, prm = _sheet(16)
    plug = gpu_sim(sp, prm, _cfg())
    plug.mlp_init(seed=4, capacity=1 << 14)
    n = plug.mlp_collect(2, stride=1)
    p0 = plug.mlp_params()[0]
    lr = 1e-3
    losses = mlp_train.train_on_gpus(plug, steps=1, batch=512, lr=lr, seed=5)
    p1, norm = plug.mlp_params()
    f, t = plug.mlp_dataset()
    idx = MO.xorshift_indices(mlp_train.minibatch_seed(5, 0, 0), 512, n)
    g_ref, loss_ref = MO.gradients(p0, norm, f[idx], t[idx])
    assert abs(losses[0] - loss_ref) <= 1e-3 * max(loss_ref, 1e-6)
    p1_ref, _, _ = MO.adam(p0, np.zeros_like(p0), np.zeros_like(p0), g_ref, 1, lr)
    big = np.abs(g_ref) > 1e-2 * np.abs(g_ref).max()
    assert big.sum() > 100
    np.testing.assert_allclose(p1[big], p1_ref[big], atol=1e-5 * lr * 100)
