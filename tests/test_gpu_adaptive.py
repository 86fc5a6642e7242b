"""Adaptive substeps and iterations on the GPU (simulation/tests.rs:951-1000
restated) and the GPU feedback against a host reduction of the same
positions: the maximum per-axis displacement over a frame and the P95
tensile strain of every (nd // 2048)-th distance constraint (exact)."""
import numpy as np
import pytest

from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu
F = np.float32


def _tri(z=1.0):
    pos = np.array([[0.0, 0.0, z], [0.05, 0.0, z], [0.0, 0.05, z]], F)
    return ClothSimulator(pos, np.array([[0, 1], [1, 2], [2, 0]], np.uint32))


def test_step_loop():
    s = _tri()
    s.set_gravity(0.0, 0.0, -9.81)
    s.set_adaptive_substep_options(True, 4, 40)
    assert s.step(0.016, 10) == 4  # at rest before the first feedback
    for _ in range(10):
        eff = s.step(0.016, 10)
        assert 4 <= eff <= 40 and eff == s.get_effective_substeps()


def test_history_on_option_updates():
    s = _tri()
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_adaptive_substep_options(True, 4, 40)
    s.note_external_displacement(0.2)
    assert s.step(1.0 / 60.0, 0) == 40
    s.set_adaptive_substep_options(True, 4, 18)  # still on: history kept, clamped to the new range
    assert s.get_effective_substeps() == 18
    s.set_adaptive_substep_options(False, 4, 40)
    assert s.get_effective_substeps() == 0
    s.note_external_displacement(0.5)
    s.set_adaptive_substep_options(True, 4, 40)  # the displacement noted while off is dropped
    assert s.get_effective_substeps() == 0
    s.step(1.0 / 60.0, 0)
    assert s.get_effective_substeps() == 4


def test_external_displacement_boosts_substeps():
    s = _tri()
    s.set_gravity(0.0, 0.0, 0.0)
    s.set_adaptive_substep_options(True, 4, 64)
    s.step(1.0 / 60.0, 0)
    s.note_external_displacement(0.2)  # 20 cm over a 5 mm CFL margin: 40
    assert s.step(1.0 / 60.0, 0) == 40


def _p95(v):
    v = np.sort(v[v > 0])
    if not len(v):
        return 0.0
    return float(v[min(int(np.float32(len(v)) * np.float32(0.95)), len(v) - 1)])


def test_gpu_feedback_matches_host_reduction():
    sc = scenes.config1()
    s = scenes.build(ClothSimulator, sc)
    s.set_adaptive_substep_options(True, 4, 64)
    col = s.get_coloring()
    ids, rest0 = col["dist_v"], col["dist_par"][:, 0].copy()
    nd = len(ids)
    stride = max(nd // 2048, 1)
    acc = F(0)
    for r in rest0:  # the host's sequential float sum
        acc = F(acc + r)
    avg = F(acc / F(nd))
    min_ref = np.float32(max(np.float32(0.5) * avg, np.float32(0.002)))
    prev = s.get_state()[0].copy()
    for f in range(4):
        s.step(sc["dt"], 0)
        x = s.get_state()[0]
        disp = float(np.max(np.abs(x - prev)))
        prev = x.copy()
        st = s._adaptive()
        assert st[3] == np.float32(disp)
        k = np.arange(0, nd, stride)
        a, b = x[ids[k, 0]], x[ids[k, 1]]
        d = (a - b).astype(F)
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        l0 = rest0[k]
        ok = (l0 > F(1e-6)) & (d2 > l0 * l0)
        strain = np.where(ok, (np.sqrt(d2) - l0) / np.maximum(l0, min_ref), F(-1)).astype(F)
        assert st[2] == np.float32(_p95(strain)), (f, st[2], _p95(strain))
    assert s.get_effective_solver_iterations() >= sc["iterations"]
