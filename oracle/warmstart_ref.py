"""CPU reference of the learned warm-start network (test infrastructure only).

The warm start has no counterpart in the reference project, so there is no
upstream algorithm to restate: this module restates the network that
taremincloth_b200/csrc/warmstart.cuh computes, in numpy, as the checker for
its forward and backward kernels.  Only tests may import it.

Network (per vertex i, neighbours N(i) from an adjacency CSR; FS, YS the
normalizer stored after the weights, not trained):
    X0 = bf16(bf16(features) * FS)           16
    H0 = bf16(SiLU(X0 W0 + b0))              64
    X1 = [H0_i, bf16(mean_{j in N(i)} H0_j)] 128
    H1 = bf16(SiLU(X1 W1 + b1))              64
    X2 = [H1_i, bf16(mean H1_j)]             128
    H2 = bf16(SiLU(X2 W2 + b2))              64
    Y  = H2 bf16(W3) + b3                    3
    loss = sum_i mask_i |Y_i - T_i / YS|^2 / (3 n)
Weights are used as bf16, biases as fp32.  The backward pass treats the bf16
roundings of activations as identity (straight-through) and rounds dZ to bf16
before the weight and input gradient products, as the kernels do.  With
``round_bf16=False`` and float64 every rounding is dropped, which gives the
exact gradient of the smooth function (checked against finite differences).
"""
from __future__ import annotations

import numpy as np

PARAM_COUNT = 17812
LAYOUT = (("W0", 0, (16, 64)), ("b0", 1024, (64,)), ("W1", 1088, (128, 64)), ("b1", 9280, (64,)),
          ("W2", 9344, (128, 64)), ("b2", 17536, (64,)), ("W3", 17600, (64, 3)), ("b3", 17792, (3,)))
# the normalizer (not trained): per-feature input scales and the output scale
NORM_LAYOUT = (("fscale", 17795, (16,)), ("yscale", 17811, (1,)))


def bf16(x):
    """Round float32 to the nearest bfloat16 (ties to even), kept as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(blob, dtype=np.float32):
    blob = np.asarray(blob, dtype).ravel()
    return {name: blob[off:off + int(np.prod(shape))].reshape(shape) for name, off, shape in LAYOUT + NORM_LAYOUT}


def pack(params):
    """Blob of the named arrays; a missing entry is zero (the gradient of the
    normalizer, which is not trained)."""
    out = np.zeros(PARAM_COUNT, np.float64)
    for name, off, shape in LAYOUT + NORM_LAYOUT:
        if name in params:
            out[off:off + int(np.prod(shape))] = np.asarray(params[name]).ravel()
    return out


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _mean_neighbours(h, adj_off, adj_idx, dt):
    n = h.shape[0]
    deg = np.diff(adj_off).astype(np.int64)
    rows = np.repeat(np.arange(n), deg)
    acc = np.zeros_like(h, dtype=dt)
    np.add.at(acc, rows, h[adj_idx].astype(dt))
    inv = np.where(deg > 0, (1.0 / np.maximum(deg, 1)).astype(dt), dt(0))
    return acc * inv[:, None]


def forward_backward(feat, adj_off, adj_idx, target, mask, blob, round_bf16=True, dtype=np.float32):
    """(loss, gradient blob, y) of the network on one graph."""
    dt = np.dtype(dtype).type
    R = (lambda a: bf16(a)) if round_bf16 else (lambda a: np.asarray(a, dt))
    adj_off = np.asarray(adj_off, np.int64)
    adj_idx = np.asarray(adj_idx, np.int64)
    n = feat.shape[0]
    P = unpack(blob, np.float64 if dtype == np.float64 else np.float32)
    W = [R(P["W0"]).astype(dt), R(P["W1"]).astype(dt), R(P["W2"]).astype(dt)]
    B = [P["b0"].astype(dt), P["b1"].astype(dt), P["b2"].astype(dt)]
    W3 = R(P["W3"]).astype(dt)
    b3 = P["b3"].astype(dt)
    ys = P["yscale"].astype(dt)[0]
    ys = ys if ys > 0 else dt(1)
    X = [R(R(feat).astype(dt) * P["fscale"].astype(dt)).astype(dt)]
    Z, H = [], []
    for layer in range(3):
        if layer > 0:
            hp = H[-1]
            X.append(np.concatenate([hp, R(_mean_neighbours(hp, adj_off, adj_idx, dt)).astype(dt)], axis=1))
        z = (X[layer].astype(np.float64) @ W[layer].astype(np.float64)).astype(dt) + B[layer]
        Z.append(z)
        H.append(R(_silu(z)).astype(dt))
    y = (H[2].astype(np.float64) @ W3.astype(np.float64)).astype(dt) + b3
    m = np.asarray(mask, dt).reshape(n, 1)
    d = (y - np.asarray(target, dt).reshape(n, 3) / ys) * m
    loss = float(np.sum(d.astype(np.float64) ** 2) / (3.0 * n))
    dy = (2.0 * d / (3.0 * n)).astype(dt)
    g = {"W3": H[2].astype(np.float64).T @ dy, "b3": dy.sum(0, dtype=np.float64)}
    dh = (dy.astype(np.float64) @ W3.astype(np.float64).T).astype(dt)
    deg = np.diff(adj_off).astype(np.int64)
    for layer in (2, 1, 0):
        dz = (dh * _silu_grad(Z[layer])).astype(dt)
        g[f"b{layer}"] = dz.sum(0, dtype=np.float64)
        dzr = R(dz).astype(np.float64)
        g[f"W{layer}"] = X[layer].astype(np.float64).T @ dzr
        if layer == 0:
            break
        dx = (dzr @ W[layer].astype(np.float64).T).astype(dt)
        # the mean's transpose: vertex j receives dX_i[64:] / deg(i) from each i with j in N(i)
        share = np.zeros((n, 64), np.float64)
        rows = np.repeat(np.arange(n), deg)
        scale = (1.0 / np.maximum(deg, 1))[rows]
        np.add.at(share, adj_idx, dx[rows, 64:].astype(np.float64) * scale[:, None])
        dh = (dx[:, :64].astype(np.float64) + share).astype(dt)
    return loss, pack(g), y


def grid_graph(w, h):
    """Adjacency CSR of a w x h grid with both diagonals (symmetric, sorted)."""
    nb = [[] for _ in range(w * h)]
    for r in range(h):
        for c in range(w):
            for dr in (-1, 0, 1):
                for dc in (-1, 0, 1):
                    if (dr or dc) and 0 <= r + dr < h and 0 <= c + dc < w:
                        nb[r * w + c].append((r + dr) * w + c + dc)
    off = np.zeros(w * h + 1, np.uint32)
    off[1:] = np.cumsum([len(x) for x in nb])
    idx = np.asarray([j for x in nb for j in sorted(x)], np.uint32)
    return off, idx


def random_params(rng, scale_head=1.0):
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases, and a
    normalizer of scales in [0.5, 2]."""
    blob = np.zeros(PARAM_COUNT, np.float32)
    for name, off, shape in LAYOUT:
        k = int(np.prod(shape))
        fan_in = shape[0] if len(shape) == 2 else 4.0
        sc = 1.0 / np.sqrt(fan_in) * (scale_head if name == "W3" else 1.0)
        blob[off:off + k] = rng.uniform(-sc, sc, k).astype(np.float32)
    for name, off, shape in NORM_LAYOUT:
        k = int(np.prod(shape))
        blob[off:off + k] = rng.uniform(0.5, 2.0, k).astype(np.float32)
    return blob
