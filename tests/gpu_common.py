"""Shared helpers for the GPU parity tests."""
import numpy as np


def extent(pos):
    p = np.asarray(pos, np.float64)
    return float(np.linalg.norm(p.max(0) - p.min(0)))


def compare_frames(prod, orc, frames, dt, substeps, ext, tol_rel=1e-5):
    """Step both simulators frame by frame; return per-frame max |dx| / extent
    and the fraction of bit-identical coordinates."""
    worst, same = [], []
    for _ in range(frames):
        prod.step(dt, substeps)
        orc.step(dt, substeps)
        xg, _, vg = prod.get_state()
        xo, _, vo = orc.get_state()
        d = np.abs(xg.astype(np.float64) - xo.astype(np.float64)).max() / ext
        worst.append(float(d))
        same.append(float(np.mean(xg == xo)))
    return np.asarray(worst), np.asarray(same)
