"""CPU checks of the warm-start network's reference (the checker of the GPU
training kernels): its backward pass against central finite differences of
its own forward in float64, and the parameter-blob layout."""
import numpy as np
import pytest

from oracle import warmstart_ref as W


def _case(seed, w=4, h=3):
    rng = np.random.default_rng(seed)
    off, idx = W.grid_graph(w, h)
    n = w * h
    feat = rng.normal(0, 1, (n, 16))
    target = rng.normal(0, 0.5, (n, 3))
    mask = (rng.random(n) > 0.2).astype(np.float64)
    blob = W.random_params(rng).astype(np.float64)
    return feat, off, idx, target, mask, blob


@pytest.mark.parametrize("seed", [0, 1])
def test_reference_backward_matches_finite_differences(seed):
    feat, off, idx, target, mask, blob = _case(seed)
    loss, grad, _ = W.forward_backward(feat, off, idx, target, mask, blob, round_bf16=False, dtype=np.float64)
    rng = np.random.default_rng(100 + seed)
    # every bias entry and a sample of each weight matrix
    picks = []
    for name, o, shape in W.LAYOUT:
        k = int(np.prod(shape))
        picks += list(o + rng.choice(k, size=min(k, 12), replace=False))
    eps = 1e-6
    for p in picks:
        b1, b2 = blob.copy(), blob.copy()
        b1[p] += eps
        b2[p] -= eps
        l1 = W.forward_backward(feat, off, idx, target, mask, b1, round_bf16=False, dtype=np.float64)[0]
        l2 = W.forward_backward(feat, off, idx, target, mask, b2, round_bf16=False, dtype=np.float64)[0]
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - grad[p]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (p, fd, grad[p])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3, 65504.0], np.float32)
    r = W.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1.0); 1 + 1.5 * 2^-8 rounds up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8
    assert (W.bf16(r) == r).all()


def test_blob_layout_roundtrip():
    rng = np.random.default_rng(3)
    blob = W.random_params(rng)
    assert blob.size == W.PARAM_COUNT
    assert np.array_equal(W.pack(W.unpack(blob)).astype(np.float32), blob)
    from taremincloth_b200 import warmstart as host
    assert host.PARAM_COUNT == W.PARAM_COUNT and host.LAYOUT == W.LAYOUT and host.NORM_LAYOUT == W.NORM_LAYOUT
    assert np.array_equal(host.pack(host.unpack(blob)), blob)
