"""Autotuner for a simulator's launch shape and, on request, its hash cell.

Launch shape (results never change, only speed):
* the launch-per-colour path at each tile size (threads per block of the
  per-colour constraint launches: 128, 256, 512),
* the persistent solver at every blocks-per-SM value the occupancy allows,
* for batched instances without self-collision, the cluster solver (one
  thread-block cluster per bin of instances) and the staged cluster solver
  (the same bins, vertex records in the clusters' shared memory).
Each candidate is timed over a few frames with CUDA events; the simulation
state is restored after every trial and the fastest is kept.

Hash cell (tune_cell=True): the cell is a physics setting, because the
self-collision passes only see neighbours within one cell.  Candidate cells
are kept only when, from the same state, one frame's positions stay within
`cell_tol` x the cloth extent of the reference cell's frame and the final
constraint residual is no larger than `res_tol` x the reference cell's; the
reference formula (the parity setting) is kept otherwise.
"""
from __future__ import annotations

import numpy as np


def _time(sim, dt, substeps, frames):
    sim.step(dt, substeps)  # record the graph
    t = 0.0
    for _ in range(frames):
        sim.step(dt, substeps)
        t += sim.last_frame_ms()
    return t / frames


def _residual(sim, dt, substeps):
    sim.set_residual_tracking(True)
    sim.step(dt, substeps)
    r = sim.get_residuals()
    sim.set_residual_tracking(False)
    return float(r["dist_rms_total"] + r["bend_rms_total"])


def tune_cell(sim, dt, substeps, cells, frames=2, cell_tol=1e-4, res_tol=1.0):
    """Try hash cells (absolute sizes) against the reference cell; returns the
    kept cell (None = reference) and every trial with its timing, position
    deviation and residual."""
    x, _, v = sim.get_state()
    x, v = x.copy(), v.copy()
    ext = float(np.linalg.norm(x.max(0) - x.min(0))) or 1.0
    sim.set_hash_cell_size(None)
    ref_ms = _time(sim, dt, substeps, frames)
    sim.set_positions_and_velocities(x, v)
    ref_res = _residual(sim, dt, substeps)
    ref_x = sim.get_state()[0].astype(np.float64)
    trials = [dict(cell=None, ms=ref_ms, deviation=0.0, residual=ref_res, accepted=True)]
    best = (ref_ms, None)
    for c in cells:
        sim.set_hash_cell_size(c)
        sim.set_positions_and_velocities(x, v)
        ms = _time(sim, dt, substeps, frames)
        sim.set_positions_and_velocities(x, v)
        res = _residual(sim, dt, substeps)
        dev = float(np.abs(sim.get_state()[0].astype(np.float64) - ref_x).max()) / ext
        ok = dev <= cell_tol and res <= res_tol * ref_res
        trials.append(dict(cell=float(c), ms=ms, deviation=dev, residual=res, accepted=ok))
        if ok and ms < best[0]:
            best = (ms, float(c))
    sim.set_hash_cell_size(best[1])
    sim.set_positions_and_velocities(x, v)
    return best[1], trials


def autotune(sim, dt, substeps, frames=3, verbose=False, tune_cell_sizes=None):
    x, _, v = sim.get_state()
    x, v = x.copy(), v.copy()
    max_per_sm, _ = sim.get_launch_limits()
    trials = [(False, 0, b) for b in (128, 256, 512)]
    trials += [(True, b, 256) for b in range(1, min(max_per_sm, 4) + 1)]
    for mode in (2, 3):  # cluster solver, staged cluster solver
        try:
            sim.set_launch_config(mode, 1)
            trials.append((mode, 0, 256))
        except ValueError:
            pass
    results = []
    for persistent, bps, block in trials:
        sim.set_launch_config(persistent, bps if persistent is True else 1)
        sim.set_launch_block(block)
        ms = _time(sim, dt, substeps, frames)
        results.append((ms, persistent, bps, block))
        sim.set_positions_and_velocities(x, v)
        if verbose:
            print(f"persistent={persistent} blocks/SM={bps} block={block}: {ms:.3f} ms/frame")
    best = min(results, key=lambda r: r[0])
    sim.set_launch_config(best[1], best[2] if best[1] is True else 1)
    sim.set_launch_block(best[3])
    out = dict(ms_per_frame=best[0], persistent=best[1], blocks_per_sm=best[2], block=best[3],
               trials=[dict(ms=r[0], persistent=r[1], blocks_per_sm=r[2], block=r[3]) for r in results])
    if tune_cell_sizes:
        cell, ctrials = tune_cell(sim, dt, substeps, tune_cell_sizes)
        out["hash_cell"] = cell
        out["hash_cell_trials"] = ctrials
    return out
