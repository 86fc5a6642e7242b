"""Learned warm start on the GPU.

* The tensor-core forward/backward kernels against the numpy reference of
  the network (loss, outputs, every parameter gradient; bf16 rounding points
  emulated, tolerance 2e-2 of each tensor's norm).
* With an all-zero network the warm-started substep is the plain solver:
  threshold +inf gives the bits of (iterations - k) plain iterations,
  threshold -1 (always fall back) the bits of the full iteration count.
* Trained on plain-solver snapshots (the first training fits the feature
  and output normalizer), the network lowers the RMS constraint residual
  that (iterations - k) iterations leave, against no warm start.
"""
import numpy as np
import pytest

from oracle import warmstart_ref as W
from taremincloth_b200 import ClothSimulator, scenes, warmstart

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("seed", [0, 1])
def test_mlp_grad_matches_reference(seed):
    rng = np.random.default_rng(seed)
    off, idx = W.grid_graph(20, 21)  # 420 vertices: 7 tiles of 64 rows, the last one ragged
    n = 420
    feat = rng.normal(0, 1, (n, 16)).astype(np.float32)
    target = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    mask = (rng.random(n) > 0.1).astype(np.float32)
    blob = W.random_params(rng)
    loss_g, grad_g, y_g, y_inf = warmstart.mlp_grad(feat, off, idx, target, mask, blob, with_inference=True)
    loss_r, grad_r, y_r = W.forward_backward(feat, off, idx, target, mask, blob)
    assert abs(loss_g - loss_r) <= 1e-3 * abs(loss_r)
    assert _nrel(y_g, y_r) <= 5e-3
    assert _nrel(y_inf, y_r) <= 5e-3  # fused inference head
    for name, o, shape in W.LAYOUT:
        k = int(np.prod(shape))
        e = _nrel(grad_g[o:o + k], grad_r[o:o + k])
        assert e <= 2e-2, (name, e)


def test_mlp_inference_large_graph_matches_reference():
    """Inference on a large graph (persistent layer kernels, many tiles per
    block): outputs against the numpy reference on a 259 x 255 grid graph
    (66,045 vertices, a ragged last tile)."""
    rng = np.random.default_rng(5)
    off, idx = W.grid_graph(259, 255)
    n = 259 * 255
    feat = rng.normal(0, 1, (n, 16)).astype(np.float32)
    target = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    mask = np.ones(n, np.float32)
    blob = W.random_params(rng)
    _, _, _, y_inf = warmstart.mlp_grad(feat, off, idx, target, mask, blob, with_inference=True)
    _, _, y_r = W.forward_backward(feat, off, idx, target, mask, blob)
    assert _nrel(y_inf, y_r) <= 5e-3


def test_tcgen05_inference_matches_mma_sync():
    """The warm start's message-passing layers on tcgen05 (TMEM accumulator,
    the default) against the warp-level mma.sync kernels: same rounding
    points, so one warm-started substep of config 1 with a random network
    agrees to fp32 summation order (and the network does move vertices)."""
    sc = scenes.config1()
    rng = np.random.default_rng(11)
    blob = W.random_params(rng)
    a, b, c = _scene_sims(sc, 3)
    for s, kind in ((a, 0), (b, 1)):
        s.ws_set_params(blob)
        s.ws_set_kernel(kind)
        s.ws_enable(2, float("inf"))
    for s in (a, b, c):
        s.step(sc["dt"] / sc["substeps"], 1)
    xa, xb, xc = (_state(s)[0] for s in (a, b, c))
    ext = float(np.linalg.norm(xc.max(0) - xc.min(0)))
    assert np.abs(xa - xc).max() > 1e-4 * ext  # the network moved the cloth
    assert np.abs(xa - xb).max() <= 1e-5 * ext, np.abs(xa - xb).max() / ext


def _state(sim):
    x, _, v = sim.get_state()
    return x.copy(), v.copy()


def _restore(sim, st):
    sim.set_positions_and_velocities(st[0], st[1])


def _scene_sims(scene, n_sims):
    return [scenes.build(ClothSimulator, scene) for _ in range(n_sims)]


@pytest.mark.parametrize("which", ["config1", "config2_small"])
def test_zero_network_is_the_plain_solver(which):
    sc = scenes.config1() if which == "config1" else scenes.config2(n=24, subdiv=2)
    it, k = sc["iterations"], 2
    a, b, c, d = _scene_sims(sc, 4)
    zeros = np.zeros(warmstart.PARAM_COUNT, np.float32)
    for s in (a, c):
        s.ws_set_params(zeros)
    a.ws_enable(k, float("inf"))
    b.set_solver_iterations(it - k)
    c.ws_enable(k, -1.0)
    frames = 3
    for _ in range(frames):
        for s in (a, b, c, d):
            s.step(sc["dt"], sc["substeps"])
    xa, xb, xc, xd = (_state(s)[0] for s in (a, b, c, d))
    assert np.array_equal(xa, xb)
    assert np.array_equal(xc, xd)
    st_a, st_c = a.ws_stats(), c.ws_stats()
    assert st_a["substeps"] == st_c["substeps"] == frames * sc["substeps"]
    assert st_a["fallbacks"] == 0 and st_c["fallbacks"] == frames * sc["substeps"]
    assert st_a["last_residual"] > 0.0


@pytest.mark.parametrize("mode", ["absolute", "relative"])
@pytest.mark.parametrize("which", ["config1", "config2_small"])
def test_per_colour_warm_start_matches_persistent(which, mode):
    """The per-colour launch mode (residual check on the device, fallback
    iterations gated by its flag) gives the bits of the persistent solver,
    with a threshold (absolute, or relative to the residual of the predicted
    positions) that some substeps miss and others meet."""
    sc = scenes.config1() if which == "config1" else scenes.config2(n=24, subdiv=2)
    dt, sub, k = sc["dt"], sc["substeps"], 2
    a, b = _scene_sims(sc, 2)
    b.set_launch_config(False)
    rng = np.random.default_rng(7)
    blob = W.random_params(rng, scale_head=0.05)
    probe = scenes.build(ClothSimulator, sc)
    probe.ws_set_params(blob)
    probe.ws_enable(k, float("inf"))
    if mode == "relative":
        probe.ws_set_relative_threshold(1e6)  # stats give 1e6 x the predicted residual
    res = []
    for _ in range(2 * sub):
        probe.step(dt / sub, 1)
        st = probe.ws_stats()
        if mode == "absolute":
            res.append(st["last_residual"])
        elif st["threshold"] > 0.0:  # a rigidly moving cloth has a zero predicted residual
            res.append(st["last_residual"] / (st["threshold"] / 1e6))
    assert res
    thr = float(np.median(res))
    for s in (a, b):
        s.ws_set_params(blob)
        if mode == "relative":
            s.ws_enable(k, float("inf"))
            s.ws_set_relative_threshold(thr)
        else:
            s.ws_enable(k, thr)
    for _ in range(3):
        for s in (a, b):
            s.step(dt, sub)
    sa, sb = a.ws_stats(), b.ws_stats()
    assert sa == sb, (sa, sb)
    assert 0 < sa["fallbacks"] < sa["substeps"], sa
    assert np.array_equal(_state(a)[0], _state(b)[0])
    assert np.array_equal(_state(a)[1], _state(b)[1])


def test_plain_residual_ratio():
    """The plain solver's final / predicted residual ratio is a positive
    finite number (on the pinned 64x64 sheet about 1: five Gauss-Seidel
    iterations hardly move its global RMS residual)."""
    sc = scenes.config1()
    s = scenes.build(ClothSimulator, sc)
    s.step(sc["dt"], sc["substeps"])
    r = warmstart.plain_residual_ratio(s, sc["dt"], sc["substeps"], 1)
    assert 0.0 < r < 4.0, r


def test_invalid_warm_start_arguments():
    sc = scenes.config1()
    s = scenes.build(ClothSimulator, sc)
    with pytest.raises(ValueError):
        s.ws_enable(sc["iterations"], 1.0)  # k must leave at least one plain iteration
    with pytest.raises(ValueError):
        s.ws_enable(0, 1.0)
    with pytest.raises(ValueError):
        s.ws_set_params(np.zeros(10, np.float32))
    with pytest.raises(ValueError):
        s.ws_train(10, 1e-3)  # nothing recorded


def test_trained_warm_start_gains_over_no_warm_start():
    sc = scenes.config1()
    dt, sub, it, k = sc["dt"], sc["substeps"], sc["iterations"], 2
    s = scenes.build(ClothSimulator, sc)
    for _ in range(4):
        s.step(dt, sub)
    got, l0, l1 = warmstart.fit(s, dt, sub, frames=10, every=2, epochs=60, lr=2e-3, seed=0)
    assert got == 50
    assert l1 < 0.5 * l0, (l0, l1)
    trained = s.ws_params()
    # the first training fitted the normalizer: motion features (about 1e-3
    # of the edge length) are scaled up, the bias and free-flag inputs stay 1
    P = warmstart.unpack(trained)
    assert P["fscale"][0] > 10.0 and P["fscale"][15] == 1.0 and P["fscale"][14] == 1.0, P["fscale"]
    assert 0.0 < P["yscale"][0] < 0.1, P["yscale"]
    start = _state(s)

    def run(params, enable):
        _restore(s, start)
        if enable:
            s.ws_set_params(params)
            s.ws_enable(k, float("inf"))
        else:
            s.ws_disable()
        s.step(dt, sub)
        out = _state(s)[0].astype(np.float64)
        res = s.ws_stats()["last_residual"] if enable else None
        s.ws_disable()
        return out, res

    full, _ = run(None, False)
    x_zero, r_zero = run(np.zeros_like(trained), True)
    x_ws, r_ws = run(trained, True)
    e_zero = float(np.sqrt(np.mean((x_zero - full) ** 2)))
    e_ws = float(np.sqrt(np.mean((x_ws - full) ** 2)))
    print(f"after {it - k} of {it} iterations: RMS residual no warm start {r_zero:.3e}, learned {r_ws:.3e}; "
          f"rms distance to the {it}-iteration positions {e_zero:.3e} vs {e_ws:.3e}")
    assert r_ws < r_zero
    # a loaded network keeps its normalizer through further training
    s.ws_set_params(trained)
    warmstart.fit(s, dt, sub, frames=1, every=5, epochs=1, lr=1e-4, seed=1)
    P2 = warmstart.unpack(s.ws_params())
    assert np.array_equal(P2["fscale"], P["fscale"]) and np.array_equal(P2["yscale"], P["yscale"])
