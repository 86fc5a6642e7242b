"""Adaptive substep / iteration rules (dispatch.rs:477-607) through the pure
evaluator of the C ABI, restating the reference's known-answer tests
(crates/cloth_core/src/simulation/tests.rs:905-1060): a 3-vertex triangle,
5 cm edges, thickness 5 mm (CFL margin 5 mm), dt = 0.016."""
import ctypes as C

import numpy as np

from taremincloth_b200 import _lib


def _eval(dt=0.016, requested=20, enabled=1, mn=4, mx=64, base=20, prev=0, char_len=0.01, thick=0.005,
          g=(0.0, 0.0, -9.81), disp=0.0, ext=0.0, strain_on=1, tol=0.008, strain=0.0, comp=1, iters=2, hops=10,
          iter_sub=0):
    L = _lib.load()
    a = np.array([enabled, mn, mx, base, prev, char_len, thick, *g, disp, ext, strain_on, tol, strain, comp, iters,
                  hops], np.float32)
    out = np.zeros(2, np.uint32)
    _lib.check(L.tc_adaptive_eval(dt, requested, iter_sub, a.ctypes.data_as(C.c_void_p),
                                  out.ctypes.data_as(C.c_void_p)))
    return int(out[0]), int(out[1])


def test_cfl_and_gravity_floor():
    assert _eval(prev=4, disp=0.0)[0] == 4            # at rest: min_substeps
    assert _eval(prev=4, disp=0.20)[0] == 40          # 20 cm over a 5 mm margin: emergency jump to 40
    assert _eval(mx=25, prev=20, disp=0.20)[0] == 25  # capped by max_substeps
    assert _eval(mx=25, prev=25, disp=0.0)[0] == 23   # falls by at most 2 per frame


def test_hysteresis_deadband_and_rate_limit():
    assert _eval(prev=10, disp=0.055)[0] == 10        # target 11: within the +-1 dead band
    assert _eval(prev=10, disp=0.07)[0] == 14         # target 14 > 4 x margin: emergency, immediate
    assert _eval(prev=10, disp=0.019, strain_on=0)[0] == 8  # target 4: down by 2
    assert _eval(prev=0, disp=0.03)[0] == 6           # no history: the target itself
    assert _eval(enabled=0, requested=0)[0] == 20     # off: base substeps when none requested
    assert _eval(enabled=0, requested=7)[0] == 7


def test_strain_driven_iterations_and_substeps():
    assert _eval(strain=0.002, iters=2, iter_sub=4)[1] == 5   # 20 solves / 4 substeps
    assert _eval(strain=0.016, iters=2, iter_sub=4)[1] == 8   # boosted to 40 solves, capped at max(2*4, 8)
    assert _eval(strain=0.016, iters=4, iter_sub=4)[1] > 5
    assert _eval(prev=4, disp=0.0, strain=0.016)[0] >= 6                         # strain floor on substeps
    assert _eval(prev=4, disp=0.0, strain=0.016, strain_on=0)[0] == 4            # strain control off
    assert _eval(enabled=0, iters=3)[1] == 3                                     # off: iterations unchanged
