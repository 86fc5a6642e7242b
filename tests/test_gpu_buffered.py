"""Buffered readback (dispatch.rs:1293-1408, lib.rs:1845-1881) on the GPU:
frames stepped into the 8-slot device ring give, at one fetch, the bits of
the same frames stepped and read one at a time; past 8 frames the last slot
holds the newest frame; fetch, clear_frame_buffer and reset empty the ring.
A fetch feeds the last frame's displacement to the auto-coupling decision,
as the reference's does."""
import numpy as np
import pytest

from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu


def _frames(sc, k):
    s = scenes.build(ClothSimulator, sc)
    out = []
    for _ in range(k):
        s.step(sc["dt"], sc["substeps"])
        x = np.empty(len(sc["positions"]) * 3, np.float32)
        s.get_positions(x)
        out.append(x)
    return out


def test_buffered_frames_match_stepped_frames():
    sc = scenes.config1()
    n3 = len(sc["positions"]) * 3
    ref = _frames(sc, 10)
    s = scenes.build(ClothSimulator, sc)
    assert [s.step_buffered(sc["dt"], sc["substeps"]) for _ in range(3)] == [1, 2, 3]
    assert s.get_buffered_frame_count() == 3
    out = np.zeros(8 * n3, np.float32)
    assert s.fetch_buffered_positions(out) == 3
    for k in range(3):
        assert np.array_equal(out[k * n3:(k + 1) * n3], ref[k])
    assert s.get_buffered_frame_count() == 0
    assert s.fetch_buffered_positions(out) == 0
    # A fetch feeds the last frame's displacement to the auto-coupled
    # collider decision (update_feedback_from_floats, dispatch.rs:1397-1400),
    # which plain frames do not; so frames 4..10 are checked against a
    # simulator that fetched the same way and then stepped plainly.
    t = scenes.build(ClothSimulator, sc)
    for _ in range(3):
        t.step_buffered(sc["dt"], sc["substeps"])
    t.fetch_buffered_positions(np.zeros(8 * n3, np.float32))
    ref2 = []
    for _ in range(7):
        t.step(sc["dt"], sc["substeps"])
        x = np.empty(n3, np.float32)
        t.get_positions(x)
        ref2.append(x)
    counts = [s.step_buffered(sc["dt"], sc["substeps"]) for _ in range(7)]
    assert counts == list(range(1, 8))
    assert s.fetch_buffered_positions(out) == 7
    for k in range(7):
        assert np.array_equal(out[k * n3:(k + 1) * n3], ref2[k])


def test_buffered_ring_overflow_keeps_newest_in_last_slot():
    sc = scenes.config1()
    n3 = len(sc["positions"]) * 3
    ref = _frames(sc, 10)
    s = scenes.build(ClothSimulator, sc)
    counts = [s.step_buffered(sc["dt"], sc["substeps"]) for _ in range(10)]
    assert counts == [1, 2, 3, 4, 5, 6, 7, 8, 8, 8]
    out = np.zeros(8 * n3, np.float32)
    assert s.fetch_buffered_positions(out) == 8
    for k in range(7):
        assert np.array_equal(out[k * n3:(k + 1) * n3], ref[k])
    assert np.array_equal(out[7 * n3:], ref[9])


def test_clear_and_reset_empty_the_ring():
    sc = scenes.config1()
    s = scenes.build(ClothSimulator, sc)
    s.step_buffered(sc["dt"], sc["substeps"])
    s.step_buffered(sc["dt"], sc["substeps"])
    s.clear_frame_buffer()
    assert s.get_buffered_frame_count() == 0
    s.step_buffered(sc["dt"], sc["substeps"])
    s.reset()
    assert s.get_buffered_frame_count() == 0
    with pytest.raises(ValueError):
        s.fetch_buffered_positions(np.zeros(4, np.float64))
