"""Oracle frames of the config-2 scene at sizes the oracle cannot finish on
the GPU host within a test run, written to tests/golden/oracle_frames.npz:

  full_f1      the full scene (two 256 x 256 sheets, 131,072 vertices, on the
               subdivision-5 icosphere, self-collision on), committed
               positions after one frame (20 substeps x 4 iterations)
  mid_f{1,10,20,30}  two 128 x 128 sheets on the same icosphere, frames 1,
               10, 20 and 30 (600 substeps)

Inputs are the seeded scenes of taremincloth_b200/scenes.py; the oracle is
oracle/tcloth_oracle.c (OpenMP over all host threads).  Run from the
repository root:
    python tests/golden/make_oracle_frames.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from taremincloth_b200 import scenes  # noqa: E402


def main():
    out = {}
    t0 = time.time()
    sc = scenes.config2()
    o = scenes.build(oracle.OracleSim, sc)
    o.step(sc["dt"], sc["substeps"])
    out["full_f1"] = o.get_state()[0]
    print(f"full frame 1: {time.time() - t0:.0f} s", flush=True)
    sc = scenes.config2(n=128)
    o = scenes.build(oracle.OracleSim, sc)
    for f in range(1, 31):
        o.step(sc["dt"], sc["substeps"])
        if f in (1, 10, 20, 30):
            out[f"mid_f{f}"] = o.get_state()[0]
            print(f"128 x 128 frame {f}: {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "oracle_frames.npz"), **out)


if __name__ == "__main__":
    main()
