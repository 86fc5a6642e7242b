"""Stages the reference's own Python tests for the drop-in module, unchanged.

Copies, from a reference checkout, the test files that exercise the XPBD
substep through ``taremin_cloth_core`` (with the package ``__init__`` files
they import and the golden fixtures they read) into ``oracle/_ref/suite``,
keeping the reference's layout so their path logic works as written:

    tests/__init__.py, tests/regression/__init__.py, tests/core/__init__.py
    tests/regression/test_single_step_exact.py
    tests/regression/test_golden_regression.py
    tests/core/test_pair_caching.py
    tests/core/test_self_collision_symmetry.py
    tests/fixtures/golden_master/*.npz

The staged copy is test input, like the compiled reference under
``oracle/_ref``: it is not part of this repository's history.  Run it with
the repository root on PYTHONPATH so that ``import taremin_cloth_core``
resolves to the drop-in module (tests/test_gpu_reference_suite.py does).

    python oracle/stage_reference_tests.py <reference checkout root>
"""
import glob
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SUITE = os.path.join(HERE, "_ref", "suite")
FILES = ["tests/__init__.py", "tests/regression/__init__.py", "tests/core/__init__.py",
         "tests/regression/test_single_step_exact.py", "tests/regression/test_golden_regression.py",
         "tests/core/test_pair_caching.py", "tests/core/test_self_collision_symmetry.py"]


def stage(ref_root):
    for rel in FILES + [os.path.relpath(p, ref_root) for p in
                        sorted(glob.glob(os.path.join(ref_root, "tests", "fixtures", "golden_master", "*.npz")))]:
        dst = os.path.join(SUITE, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        shutil.copyfile(os.path.join(ref_root, rel), dst)
    os.makedirs(os.path.join(SUITE, "python"), exist_ok=True)
    return SUITE


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: stage_reference_tests.py <reference checkout root>")
    print(stage(sys.argv[1]))
