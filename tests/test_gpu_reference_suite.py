"""The reference's own Python tests, unchanged, against the drop-in module.

oracle/stage_reference_tests.py copies tests/regression/test_single_step_exact.py,
tests/regression/test_golden_regression.py, tests/core/test_pair_caching.py
and tests/core/test_self_collision_symmetry.py (with the package files and
golden fixtures they read) from a reference checkout into oracle/_ref/suite;
__graft_entry__.build() stages them where the checkout is present.  They run
here in a child pytest with the repository root on PYTHONPATH, so that their
``import taremin_cloth_core`` loads this library.

Every test must pass except the one whose bound this path misses by
construction: case 2's 15 mm all-frame bound
(test_golden_regression.py:170), which the oracle misses too (19.3 mm at
frame 25; tests/test_oracle_golden.py shows that a one-ulp input change
moves the trajectory as far after contact).
"""
import os
import subprocess
import sys
import xml.etree.ElementTree as ET

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITE = os.path.join(ROOT, "oracle", "_ref", "suite")
FILES = ["tests/regression/test_single_step_exact.py", "tests/regression/test_golden_regression.py",
         "tests/core/test_pair_caching.py", "tests/core/test_self_collision_symmetry.py"]
EXPECTED_FAIL = {"test_case2_plane_sphere_regression": "Case 2 max vertex diverged"}


def test_reference_suite_unchanged(tmp_path):
    if not os.path.isdir(os.path.join(SUITE, "tests")):
        pytest.skip("reference tests not staged (oracle/stage_reference_tests.py needs a reference checkout)")
    xml = tmp_path / "suite.xml"
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([ROOT, os.environ.get("PYTHONPATH", "")]))
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", f"--junitxml={xml}",
                        "--rootdir", SUITE, *FILES], cwd=SUITE, env=env, capture_output=True, text=True,
                       timeout=1800)
    cases = ET.parse(xml).getroot().iter("testcase")
    passed, failed, skipped = [], {}, []
    for c in cases:
        name = c.get("name")
        bad = c.find("failure") if c.find("failure") is not None else c.find("error")
        if bad is not None:
            failed[name] = (bad.get("message") or "") + (bad.text or "")
        elif c.find("skipped") is not None:
            skipped.append(name)
        else:
            passed.append(name)
    assert not skipped, skipped
    assert set(failed) <= set(EXPECTED_FAIL), {k: v[:400] for k, v in failed.items()} or r.stdout[-2000:]
    for name, why in EXPECTED_FAIL.items():
        if name in failed:
            assert why in failed[name], failed[name][:400]
    assert len(passed) >= 15, (passed, r.stdout[-2000:])
