"""Copies the reference's golden-master vectors into tests/golden/.

Run once in a container where the reference checkout is mounted, giving
the checkout's root:
    python tests/golden/make_fixtures.py <reference checkout>
The files are the reference's own fixtures
(tests/fixtures/golden_master/*.npz): initial positions, edges, faces,
inverse masses and 26 frames produced by the reference GPU solver, plus the
one-frame step_case{1,2,3}_f1.npz pairs.  They are data, copied verbatim.
"""
import os
import shutil
import sys

NAMES = ["case1_cloth_body.npz", "case2_plane_sphere.npz", "case3_multi_collider.npz",
         "case4_self_collision_drape.npz", "step_case1_f1.npz", "step_case2_f1.npz",
         "step_case3_f1.npz"]


def main(ref_root):
    src = os.path.join(ref_root, "tests", "fixtures", "golden_master")
    dst = os.path.dirname(os.path.abspath(__file__))
    for n in NAMES:
        shutil.copyfile(os.path.join(src, n), os.path.join(dst, n))
        print("copied", n)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <reference checkout root>")
    main(sys.argv[1])
