"""Radiance-cache network restated in numpy — TEST INFRASTRUCTURE ONLY.

This module is the checker for libpt's radiance-cache kernels
(pbrt-renderer-_b200/csrc/pt_cache.cu, pt_cache.cuh): only the tests import
it.  The reference has no radiance cache, so there is no reference file to
cite; the network follows Müller et al. 2021 ("Real-time Neural Radiance
Caching for Path Tracing") as the library states it:

* encoding: position in box units, sin/cos(2^j pi p) for j = 0..5, direction,
  normal, roughness, albedo, a constant 1, zero padding (64 features);
* 5 hidden layers of 64 with ReLU and no biases, 16 linear outputs (0..2 used);
* BF16 operands (round to nearest even), FP32 accumulation — emulated here by
  rounding operands to BF16 and summing exactly in float64;
* loss sum_c (y_c - t_c)^2 / (y_c^2 + 0.01), denominator held constant;
  output gradient 2 (y - t) / (y^2 + 0.01) rounded to BF16, hidden-layer
  gradients dZ_{l-1} = BF16(dZ_l . W_l * [A_l > 0]);
* Adam (beta1 0.9, beta2 0.99, eps 1e-8) on the mean gradient over 3 n terms.
"""

from __future__ import annotations

import numpy as np

IN, WIDTH, OUT, LAYERS = 64, 64, 16, 6
PARAMS = 5 * WIDTH * IN + OUT * WIDTH


def rows(l):
    return WIDTH if l < 5 else OUT


def split(w):
    """Canonical parameter vector -> list of [out][in] matrices."""
    out, o = [], 0
    for l in range(LAYERS):
        r = rows(l)
        out.append(np.asarray(w[o:o + r * IN], np.float64).reshape(r, IN))
        o += r * IN
    return out


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    out = np.where(np.isfinite(a), out, a)
    return out.astype(np.float64)


def fp32(x):
    """Round to float32, returned as float64."""
    return np.asarray(x, np.float32).astype(np.float64)


def encode(records, bmin, bmax):
    """records: n x 16 floats -> n x 64 features (float64)."""
    r = np.asarray(records, np.float64).reshape(-1, 16)
    bmin = np.asarray(bmin, np.float64)
    ext = np.asarray(bmax, np.float64) - bmin
    inv = np.where(ext > 0, 1.0 / np.where(ext > 0, ext, 1.0), 1.0)
    # the kernels compute (x - min) * (1 / extent) in float32
    p = ((r[:, 0:3].astype(np.float32) - bmin.astype(np.float32)) * inv.astype(np.float32)).astype(np.float64)
    f = np.zeros((len(r), IN))
    f[:, 0:3] = p
    for j in range(6):
        for a in range(3):
            x = np.pi * p[:, a] * (1 << j)
            f[:, 3 + 6 * j + 2 * a] = np.sin(x)
            f[:, 4 + 6 * j + 2 * a] = np.cos(x)
    f[:, 39:42] = r[:, 4:7]
    f[:, 42:45] = r[:, 8:11]
    f[:, 45] = r[:, 3]
    f[:, 46:49] = r[:, 12:15]
    f[:, 49] = 1.0
    return f


def forward(w, features):
    """Activations A_0..A_5 (BF16-rounded) and the FP32-accumulated outputs."""
    W = [bf16(m) for m in split(w)]
    A = [bf16(features)]
    for l in range(5):
        z = A[-1] @ W[l].T
        A.append(bf16(np.maximum(z, 0.0)))
    y = fp32(A[-1] @ W[5].T)
    return A, y


def infer(w, features):
    return forward(w, features)[1][:, :3]


def gradient(w, features, targets):
    """Summed parameter gradient (canonical layout) and loss sum."""
    W = [bf16(m) for m in split(w)]
    A, y = forward(w, features)
    t = np.asarray(targets, np.float64).reshape(-1, 3)
    d = y[:, :3] - t
    den = fp32(y[:, :3] ** 2 + 0.01)
    loss = float(np.sum(d * d / den))
    g = np.zeros((len(y), OUT))
    g[:, :3] = 2.0 * d / den
    dz = bf16(g)
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = dz.T @ A[l]
        if l > 0:
            da = dz @ W[l]
            dz = bf16(np.where(A[l] > 0, da, 0.0))
    return np.concatenate([gm.reshape(-1) for gm in grads]), loss


def adam(w, m, v, grad_sum, n, step, lr, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step in float32 as the kernel takes it; returns (w, m, v)."""
    f = np.float32
    g = (np.asarray(grad_sum, f) * f(1.0 / (3.0 * n))).astype(f)
    m = (f(b1) * m + f(1 - b1) * g).astype(f)
    v = (f(b2) * v + f(1 - b2) * g * g).astype(f)
    bc1, bc2 = f(1 - b1 ** step), f(1 - b2 ** step)
    w = (w - f(lr) * (m / bc1) / (np.sqrt(v / bc2) + f(eps))).astype(f)
    return w, m, v


def constant_weights(c):
    """Weights whose network outputs the constant c (3 values, exact in BF16)
    for every input: feature 49 (the constant 1) carried through unit 0."""
    w = np.zeros(PARAMS, np.float32)
    mats = []
    for l in range(LAYERS):
        mats.append(np.zeros((rows(l), IN), np.float32))
    mats[0][0, 49] = 1.0
    for l in range(1, 5):
        mats[l][0, 0] = 1.0
    mats[5][:3, 0] = c
    o = 0
    for mtx in mats:
        w[o:o + mtx.size] = mtx.reshape(-1)
        o += mtx.size
    return w
