"""CPU oracle of the learned warm-start MLP (test infrastructure only).

Restates warpsph_b200/csrc/sph_mlp.cu in numpy: 8 -> 64 -> 64 -> 64 -> 1 with ReLU,
mean-squared-error gradient, Adam.  With ``bf16=True`` the operands that the GPU feeds
to its BF16 tensor-core GEMMs are rounded to BF16 (round to nearest even) at the same
points as the kernels (features, W1..W3, the hidden activations that enter the next
layer, and the dZ operands of the weight- and data-gradient GEMMs) and everything else
is computed in float64; with ``bf16=False`` the network is plain float64 (used for the
finite-difference check of the gradient formulas).

Parameter vector layout (float32): W1[64][8] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4[1].
"""
from __future__ import annotations

import numpy as np

IN, HID = 8, 64
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)), ("b3", (HID,)),
         ("w4", (HID,)), ("b4", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def bf16(a):
    """float32 -> nearest-even bfloat16, returned as float32 (finite inputs)."""
    a = np.ascontiguousarray(np.asarray(a, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float32).reshape(-1) for name, _ in SIZES]).astype(np.float32)


def init_params(seed=0):
    """He-uniform weights, zero biases (the initialisation warpsph_b200.learned uses)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SIZES:
        if name.startswith("b"):
            d[name] = np.zeros(shape, np.float32)
        else:
            fan_in = shape[1] if len(shape) == 2 else HID
            lim = np.sqrt(6.0 / fan_in)
            d[name] = rng.uniform(-lim, lim, size=shape).astype(np.float32)
    return pack(d)


def _r(a, on):
    return bf16(a).astype(np.float64) if on else np.asarray(a, np.float64)


def forward(theta, x, bf=True):
    P = unpack(theta)
    xb = _r(x, bf)
    z1 = xb @ _r(P["W1"], bf).T + P["b1"]
    h1 = np.maximum(z1, 0.0)
    h1b = _r(h1, bf)
    z2 = h1b @ _r(P["W2"], bf).T + P["b2"]
    h2 = np.maximum(z2, 0.0)
    h2b = _r(h2, bf)
    z3 = h2b @ _r(P["W3"], bf).T + P["b3"]
    h3 = np.maximum(z3, 0.0)
    y = h3 @ P["w4"] + P["b4"][0]
    return y, dict(xb=xb, h1b=h1b, h2b=h2b, h3=h3)


def grad(theta, x, target, bf=True):
    """(grad vector float64, loss = sum (y - t)^2) of the mean squared error."""
    P = unpack(theta)
    n = x.shape[0]
    y, c = forward(theta, x, bf)
    e = y - np.asarray(target, np.float64)
    dy = 2.0 * e / n
    g = {"w4": dy @ c["h3"], "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, P["w4"]) * (c["h3"] > 0)
    g["b3"] = dz3.sum(0)
    dz3b = _r(dz3, bf)
    g["W3"] = dz3b.T @ c["h2b"]
    dz2 = (dz3b @ _r(P["W3"], bf)) * (c["h2b"] > 0)
    g["b2"] = dz2.sum(0)
    dz2b = _r(dz2, bf)
    g["W2"] = dz2b.T @ c["h1b"]
    dz1 = (dz2b @ _r(P["W2"], bf)) * (c["h1b"] > 0)
    g["b1"] = dz1.sum(0)
    g["W1"] = _r(dz1, bf).T @ c["xb"]
    flat = np.concatenate([np.asarray(g[name], np.float64).reshape(-1) for name, _ in SIZES])
    return flat, float((e * e).sum())


def adam(theta, g, m1, m2, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One bias-corrected Adam step in float32 (returns new theta, m1, m2)."""
    f = np.float32
    g = np.asarray(g, f)
    m1 = (f(beta1) * m1 + f(1 - beta1) * g).astype(f)
    m2 = (f(beta2) * m2 + f(1 - beta2) * g * g).astype(f)
    c1, c2 = f(1 - beta1 ** step), f(1 - beta2 ** step)
    theta = (theta - f(lr) * (m1 / c1) / (np.sqrt(m2 / c2) + f(eps))).astype(f)
    return theta, m1, m2
