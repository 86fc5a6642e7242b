"""Self-collision and edge-edge substep interval gating (dispatch.rs:105-114)
against the oracle on a reduced config 2 (two 24^2 sheets, icosphere 2,
self-collision on), on both solver paths.  Tolerance 1e-5 of the extent;
measured bit-exact."""
import pytest

from gpu_common import compare_frames, extent
from taremincloth_b200 import ClothSimulator, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("persistent", [True, False])
@pytest.mark.parametrize("sc_iv,ee_iv", [(3, 2), (1, 0), (4, 1)])
def test_interval_gating_matches_oracle(oracle_lib, persistent, sc_iv, ee_iv):
    sc = scenes.config2(n=24, subdiv=2)
    g = scenes.build(ClothSimulator, sc)
    o = scenes.build(oracle_lib.OracleSim, sc)
    g.set_persistent_solver(persistent)
    for s in (g, o):
        s.set_self_collision_substep_interval(sc_iv)
        s.set_self_collision_ee_substep_interval(ee_iv)
    assert g.get_self_collision_substep_interval() == sc_iv
    assert g.get_self_collision_ee_substep_interval() == ee_iv
    worst, same = compare_frames(g, o, 6, sc["dt"], sc["substeps"], extent(sc["positions"]))
    assert worst.max() <= 1e-5, worst
    assert same[-1] == 1.0
