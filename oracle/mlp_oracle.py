"""CPU oracle of the learned λ warm start — test infrastructure only (imported by tests/, never by the product).

The reference has no learned component (the warm start is an extension of the convergence solve), so this oracle is
pinned by construction rather than by reference vectors: it restates, in numpy, the network the CUDA kernels run —

* features of constraint e = (i, j) at the predicted positions p of a substep (float32, as computed on the device):
  f0 = (|pi - pj| - rest)/rest, f1 = λprev·(wi + wj + α̃)/rest, f2 = ((vi - vj)·n̂)·dt/rest,
  f3 = log10(max(α, 1e-12)), f4 = rest, f5..f7 = one-hot constraint type (stretch, shear, bend), f8 = pinned endpoint;
* target t = λ·(wi + wj + α̃)/rest (λ the converged multiplier of the substep); the network predicts the change
  t - f1 over the previous substep, standardised: λ0 = (y·tstd + tmean + f1)·rest/(wi + wj + α̃);
* forward 9→64→64→1 with SiLU, the device's rounding points emulated: standardised inputs, weights and both hidden
  activations rounded to bfloat16 (round to nearest even), products accumulated in float64 here (fp32 on the
  tensor cores — the remaining difference is accumulation order and the device's fast exp);
* backward: float64 gradients of mean((y - (t - f1 - tmean)/tstd)^2) through the same emulated forward, the rounding points
  taken as identity (the device additionally rounds dz2 and dz1 to bfloat16 for its weight-gradient tiles);
* Adam (β1 0.9, β2 0.999, ε 1e-8, bias-corrected) on the fp32 master parameters.

Parameter layout (fp32, 4865 values): w1[64][9], b1[64], w2[64][64], b2[64], w3[64], b3.
Normalisation (20 values): feature mean[9], std[9], target mean, std; only f0..f4 are standardised.
"""
from __future__ import annotations

import numpy as np

N_PARAMS = 4865
N_NORM = 20
N_FEATURES = 9


def bf16(x) -> np.ndarray:
    """float32 → bfloat16 (round to nearest, ties to even) → float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def unpack(params):
    p = np.asarray(params, np.float64)
    w1 = p[0:576].reshape(64, 9)
    b1 = p[576:640]
    w2 = p[640:4736].reshape(64, 64)
    b2 = p[4736:4800]
    w3 = p[4800:4864]
    b3 = p[4864]
    return w1, b1, w2, b2, w3, b3


def pack(w1, b1, w2, b2, w3, b3) -> np.ndarray:
    return np.concatenate([np.ravel(w1), b1, np.ravel(w2), b2, w3, [b3]]).astype(np.float64)


def standardize(features, norm) -> np.ndarray:
    f = np.array(features, np.float32).reshape(-1, N_FEATURES)
    nm = np.asarray(norm, np.float32)
    f[:, :5] = (f[:, :5] - nm[:5]) / nm[9:14]
    return f


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, norm, features, keep=False, rounding=True):
    """Standardised prediction y per feature row (float64); keep=True also returns the intermediates.
    rounding=False drops the bfloat16 rounding points (an exact FP64 network, for finite-difference checks)."""
    w1, b1, w2, b2, w3, b3 = (np.asarray(a, np.float64) for a in unpack(params))
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    x = np.asarray(r(standardize(features, norm)), np.float64)
    z1 = x @ np.asarray(r(w1), np.float64).T + b1
    h1 = np.asarray(r(_silu(z1)), np.float64)
    z2 = h1 @ np.asarray(r(w2), np.float64).T + b2
    h2 = np.asarray(r(_silu(z2)), np.float64)
    y = h2 @ np.asarray(r(w3), np.float64) + float(b3)
    if keep:
        return y, dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2)
    return y


def gradients(params, norm, features, targets, rounding=True):
    """(gradient[4865] float64, loss) of mean((y - (t - f1 - tmean)/tstd)^2), f1 the raw feature 1."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    nm = np.asarray(norm, np.float32)
    y, k = forward(params, norm, features, keep=True, rounding=rounding)
    f1 = np.asarray(features, np.float32).reshape(-1, N_FEATURES)[:, 1]
    t = (np.asarray(targets, np.float32) - f1 - nm[18]) / nm[19]
    e = y - t.astype(np.float64)
    n = len(e)
    dy = 2.0 * e / n
    gw3 = dy @ k["h2"]
    gb3 = dy.sum()
    dz2 = dy[:, None] * np.asarray(r(w3), np.float64)[None, :] * _dsilu(k["z2"])
    gb2 = dz2.sum(0)
    gw2 = dz2.T @ k["h1"]
    dh1 = dz2 @ np.asarray(r(w2), np.float64)
    dz1 = dh1 * _dsilu(k["z1"])
    gb1 = dz1.sum(0)
    gw1 = dz1.T @ k["x"]
    return pack(gw1, gb1, gw2, gb2, gw3, gb3), float(np.mean(e * e))


def adam(params, m1, m2, grads, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One bias-corrected Adam step (float32, as on the device); returns (params, m1, m2)."""
    p = np.asarray(params, np.float32)
    g = np.asarray(grads, np.float32)
    a = np.float32(beta1) * m1 + np.float32(1 - beta1) * g
    b = np.float32(beta2) * m2 + np.float32(1 - beta2) * g * g
    bc1 = np.float32(1 - beta1 ** step)
    bc2 = np.float32(1 - beta2 ** step)
    p = p - np.float32(lr) * (a / bc1) / (np.sqrt(b / bc2) + np.float32(eps))
    return p.astype(np.float32), a.astype(np.float32), b.astype(np.float32)


def features(pred, vel, ci, cj, rest, comp, ctype, inv_mass, lam_prev, dt, inv_dt):
    """Raw features (n_constraints x 9, float32) at predicted positions `pred` with pre-substep velocities `vel`;
    dt and inv_dt are the substep's parameters as given (α̃ = α·inv_dt², cloth_compute.rs:325)."""
    f32 = np.float32
    pred = np.asarray(pred, f32).reshape(-1, 3)
    vel = np.asarray(vel, f32).reshape(-1, 3)
    ci = np.asarray(ci, np.int64)
    cj = np.asarray(cj, np.int64)
    rest = np.asarray(rest, f32)
    comp = np.asarray(comp, f32)
    w = np.asarray(inv_mass, f32)
    dt = f32(dt)
    inv_dt = f32(inv_dt)
    g = pred[ci] - pred[cj]
    ln = np.sqrt((g * g).sum(1, dtype=f32)).astype(f32)
    inv = np.where(ln > f32(1e-8), f32(1.0) / np.maximum(ln, f32(1e-30)), f32(0.0)).astype(f32)
    alpha_t = comp * (inv_dt * inv_dt)
    denom = w[ci] + w[cj] + alpha_t
    out = np.zeros((len(ci), N_FEATURES), f32)
    out[:, 0] = (ln - rest) / rest
    out[:, 1] = np.asarray(lam_prev, f32) * denom / rest
    out[:, 2] = ((vel[ci] - vel[cj]) * g).sum(1, dtype=f32) * inv * dt / rest
    out[:, 3] = np.log10(np.maximum(comp, f32(1e-12)))
    out[:, 4] = rest
    ct = np.minimum(np.asarray(ctype, np.int64), 2)
    out[np.arange(len(ci)), 5 + ct] = 1.0
    out[:, 8] = ((w[ci] <= 0) | (w[cj] <= 0)).astype(f32)
    return out


def warm_lambda(params, norm, features, scale):
    """λ0 = (y·tstd + tmean + f1)·scale, scale = rest/(wi + wj + α̃)."""
    nm = np.asarray(norm, np.float32)
    y = forward(params, norm, features)
    f1 = np.asarray(features, np.float32).reshape(-1, N_FEATURES)[:, 1]
    return (y * nm[19] + nm[18] + f1) * np.asarray(scale, np.float64)


def targets(lam, rest, comp, inv_mass, ci, cj, inv_dt):
    """t = λ·(wi + wj + α̃)/rest (float32)."""
    f32 = np.float32
    w = np.asarray(inv_mass, f32)
    inv_dt = f32(inv_dt)
    denom = w[np.asarray(ci)] + w[np.asarray(cj)] + np.asarray(comp, f32) * (inv_dt * inv_dt)
    return (np.asarray(lam, f32) * denom / np.asarray(rest, f32)).astype(f32)


def xorshift_indices(seed: int, count: int, n: int) -> np.ndarray:
    """Minibatch row indices drawn the way xpbd_mlp_train draws them (xorshift64, z % n)."""
    mask = (1 << 64) - 1
    z = (seed ^ 0xD1B54A32D192ED03) & mask
    out = np.zeros(count, np.int64)
    for k in range(count):
        z ^= (z << 13) & mask
        z ^= z >> 7
        z ^= (z << 17) & mask
        out[k] = z % n
    return out
