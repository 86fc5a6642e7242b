"""Autotuner for the launch shape of a simulator.

Tries the launch-per-colour path, the persistent solver at every
blocks-per-SM value the occupancy allows and, for batched instances without
self-collision, the cluster solver (one thread-block cluster per bin of
instances) and the staged cluster solver (the same bins, vertex records in
the clusters' shared memory); times a few frames of each with CUDA events, keeps the fastest
and restores the simulation state after every trial (the settings never
change results, only speed).

The spatial-hash cell size is a physics parameter (neighbours beyond one cell
are never seen), so it is not tuned here.
"""
from __future__ import annotations

import numpy as np


def autotune(sim, dt, substeps, frames=3, verbose=False):
    x, _, v = sim.get_state()
    x, v = x.copy(), v.copy()
    max_per_sm, _ = sim.get_launch_limits()
    trials = [(False, 0)] + [(True, b) for b in range(1, min(max_per_sm, 4) + 1)]
    for mode in (2, 3):  # cluster solver, staged cluster solver
        try:
            sim.set_launch_config(mode, 1)
            trials.append((mode, 0))
        except ValueError:
            pass
    results = []
    for persistent, bps in trials:
        sim.set_launch_config(persistent, bps if persistent is True else 1)
        sim.step(dt, substeps)  # record the graph
        t = 0.0
        for _ in range(frames):
            sim.step(dt, substeps)
            t += sim.last_frame_ms()
        results.append((t / frames, persistent, bps))
        sim.set_positions_and_velocities(x, v)
        if verbose:
            print(f"persistent={persistent} blocks/SM={bps}: {t / frames:.3f} ms/frame")
    best = min(results, key=lambda r: r[0])
    sim.set_launch_config(best[1], best[2] if best[1] is True else 1)
    return dict(ms_per_frame=best[0], persistent=best[1], blocks_per_sm=best[2],
                trials=[dict(ms=r[0], persistent=r[1], blocks_per_sm=r[2]) for r in results])
