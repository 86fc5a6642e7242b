"""Learned warm start helpers (new; no counterpart in the reference).

``mlp_grad`` runs the warm-start network's forward and backward kernels on
one graph and returns the loss, the parameter gradients and the outputs.
``plain_residual`` measures the plain solver's RMS constraint residual after
every substep, whose percentile is the threshold the warm start is judged
against.  ``fit`` records plain-solver
snapshots, trains on them and leaves the network in the simulator.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

PARAM_COUNT = 17812
# (name, offset, shape) of the fp32 parameter blob
LAYOUT = (("W0", 0, (16, 64)), ("b0", 1024, (64,)), ("W1", 1088, (128, 64)), ("b1", 9280, (64,)),
          ("W2", 9344, (128, 64)), ("b2", 17536, (64,)), ("W3", 17600, (64, 3)), ("b3", 17792, (3,)))
# the normalizer (not trained): per-feature input scales and the output scale
NORM_LAYOUT = (("fscale", 17795, (16,)), ("yscale", 17811, (1,)))


def unpack(blob):
    blob = np.asarray(blob, np.float32).ravel()
    if blob.size != PARAM_COUNT:
        raise ValueError(f"parameter blob must hold {PARAM_COUNT} floats")
    return {name: blob[off:off + int(np.prod(shape))].reshape(shape) for name, off, shape in LAYOUT + NORM_LAYOUT}


def pack(params):
    """Blob of the named arrays; a missing normalizer entry is the identity (1)."""
    out = np.zeros(PARAM_COUNT, np.float32)
    for name, off, shape in LAYOUT + NORM_LAYOUT:
        k = int(np.prod(shape))
        out[off:off + k] = np.asarray(params[name], np.float32).ravel() if name in params else 1.0
    return out


def mlp_grad(feat, adj_off, adj_idx, target, mask, params, device=0, with_inference=False):
    """(loss, grads blob, y) of the network on one graph, computed on the GPU;
    with_inference adds the outputs of the fused inference kernels."""
    L = _lib.load()
    feat = np.ascontiguousarray(feat, np.float32)
    n = feat.shape[0]
    if feat.shape != (n, 16):
        raise ValueError("feat must have shape (n, 16)")
    adj_off = np.ascontiguousarray(adj_off, np.uint32)
    adj_idx = np.ascontiguousarray(adj_idx, np.uint32)
    target = np.ascontiguousarray(target, np.float32).reshape(n, 3)
    mask = np.ascontiguousarray(mask, np.float32).reshape(n)
    params = np.ascontiguousarray(params, np.float32).ravel()
    if adj_off.size != n + 1 or params.size != PARAM_COUNT:
        raise ValueError("adj_off must hold n + 1 entries and params PARAM_COUNT floats")
    loss = C.c_float()
    grads = np.zeros(PARAM_COUNT, np.float32)
    y = np.zeros((n, 3), np.float32)
    yi = np.zeros((n, 3), np.float32) if with_inference else None
    p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    _lib.check(L.tc_mlp_grad(n, p(feat), p(adj_off), p(adj_idx), p(target), p(mask), p(params), C.byref(loss),
                             p(grads), p(y), p(yi), int(device)))
    return (loss.value, grads, y, yi) if with_inference else (loss.value, grads, y)


def plain_residual(sim, dt, substeps, frames, percentile=90.0):
    """The plain solver's RMS constraint residual |C + alpha~ lambda| over all
    distance and bending constraints, measured after every substep of
    `frames` frames (each substep stepped on its own, dt / substeps), as the
    given percentile of those values: the level the warm-started substep is
    judged against after each substep.  Advances the simulation."""
    c = sim.get_counts()
    nd, nb = c["nd"], c["nb"]
    sim.set_residual_tracking(True)
    vals = []
    try:
        for _ in range(frames * substeps):
            sim.step(dt / substeps, 1)
            r = sim.get_residuals()
            ss = nd * r["dist_rms_total"] ** 2 + nb * r["bend_rms_total"] ** 2
            vals.append(float(np.sqrt(ss / max(nd + nb, 1))))
    finally:
        sim.set_residual_tracking(False)
    return float(np.percentile(vals, percentile))


def plain_residual_ratio(sim, dt, substeps, frames, percentile=90.0):
    """The plain solver's final / predicted residual ratio (RMS |C + alpha~
    lambda| after the iterations over RMS |C| of the predicted positions),
    per substep over `frames` frames (each substep stepped on its own), as
    the given percentile: the ratio of a relative warm-start threshold.
    Advances the simulation."""
    c = sim.get_counts()
    nd, nb = c["nd"], c["nb"]
    sim.set_residual_tracking(True)
    vals = []
    try:
        for _ in range(frames * substeps):
            sim.step(dt / substeps, 1)
            r = sim.get_residuals()
            ss = nd * r["dist_rms_total"] ** 2 + nb * r["bend_rms_total"] ** 2
            r0 = sim.get_predicted_residual()
            if r0 > 0.0:
                vals.append(float(np.sqrt(ss / max(nd + nb, 1))) / r0)
    finally:
        sim.set_residual_tracking(False)
    return float(np.percentile(vals, percentile)) if vals else float("inf")


def fit(sim, dt, substeps, frames, every=1, capacity=None, epochs=60, lr=2e-3, seed=0):
    """Record plain-solver snapshots over `frames` frames, then train.
    Returns (snapshots, first-epoch loss, last-epoch loss)."""
    cap = capacity if capacity is not None else max(1, frames * substeps // every)
    sim.ws_record(cap, every)
    for _ in range(frames):
        sim.step(dt, substeps)
        if sim.ws_recorded() >= cap:
            break
    got = sim.ws_recorded()
    sim.ws_record(0, 1)
    l0, l1 = sim.ws_train(epochs, lr, seed)
    return got, l0, l1
