"""Pins of the warm-start MLP oracle on CPU: its bfloat16 rounding against torch's, its analytic gradient against
central finite differences of the FP64 network, and the feature restatement on a hand-computed constraint."""
import numpy as np
import torch

from oracle import mlp_oracle as MO


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=20000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 20000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, -3.5e-39, 3.0e38], np.float32)])
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(MO.bf16(x), ref)


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    p = (rng.normal(size=MO.N_PARAMS) * 0.2).astype(np.float64)
    nm = np.zeros(MO.N_NORM)
    nm[9:18] = 1.0
    nm[19] = 1.0
    f = rng.normal(size=(37, 9))
    t = rng.normal(size=37).astype(np.float32).astype(np.float64)
    g, loss = MO.gradients(p, nm, f, t, rounding=False)

    d = (t.astype(np.float32) - f[:, 1].astype(np.float32)).astype(np.float64)   # the learned change t - f1

    def L(q):
        y = MO.forward(q, nm, f, rounding=False)
        return float(np.mean((y - d) ** 2))

    assert abs(L(p) - loss) < 1e-12
    for k in list(rng.integers(0, MO.N_PARAMS, 40)) + [0, 580, 700, 4750, 4810, 4864]:
        h = 1e-6
        q1, q2 = p.copy(), p.copy()
        q1[k] += h
        q2[k] -= h
        fd = (L(q1) - L(q2)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), k


def test_features_hand_computed():
    pred = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.1]], np.float32)
    vel = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, -1.0]], np.float32)
    f = MO.features(pred, vel, [0], [1], [1.0], [1e-6], [1], [1.0, 0.0], [2.0], 0.01, 100.0)
    # strain 0.1, λprev·(1 + 0 + 1e-6·1e4)/1, ((vi-vj)·(pi-pj)/|pi-pj|)·dt/rest = (2·-1.1/1.1)·0.01
    np.testing.assert_allclose(f[0, :5], [0.1, 2.0 * 1.01, -0.02, -6.0, 1.0], rtol=1e-5)
    assert list(f[0, 5:]) == [0.0, 1.0, 0.0, 1.0]
    t = MO.targets([3.0], [1.0], [1e-6], [1.0, 0.0], [0], [1], 100.0)
    np.testing.assert_allclose(t, [3.0 * 1.01], rtol=1e-6)


def test_scaled_change_scales_the_predicted_change():
    """mlp_scale_change: the change y·tstd + tmean that the network adds to the previous multiplier scales by the
    factor (exactly for a power of two, where the fp32 parameters scale without rounding)."""
    from bevy_xpbd_b200.plugin import mlp_scale_change
    rng = np.random.default_rng(4)
    p = (rng.normal(size=MO.N_PARAMS) * 0.2).astype(np.float32)
    nm = np.concatenate([rng.normal(size=9), np.abs(rng.normal(size=9)) + 0.5, [0.3, 1.7]]).astype(np.float32)
    f = rng.normal(size=(50, MO.N_FEATURES)).astype(np.float32)

    def change(pp, nn):
        return MO.forward(pp, nn, f, rounding=False) * float(nn[19]) + float(nn[18])

    base = change(p, nm)
    for factor, tol in ((0.5, 0.0), (0.0, 0.0), (0.35, 1e-6)):
        p2, n2 = mlp_scale_change(p, nm, factor)
        assert np.array_equal(p2[:-65], p[:-65]) and np.array_equal(n2[:18], nm[:18]) and n2[19] == nm[19]
        np.testing.assert_allclose(change(p2, n2), factor * base, rtol=tol, atol=tol)
