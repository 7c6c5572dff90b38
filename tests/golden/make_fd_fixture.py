"""Generates tests/golden/fd_smooth.npz: float64 central finite differences (h = 1e-4)
of msplat's training loss (L1 + 0.2 (1 - SSIM)) with respect to every parameter of
the two smooth 64-Gaussian, 32 x 32 scenes of tests/smooth_scenes.py (colour without
and with view dependence).

    python tests/golden/make_fd_fixture.py

The loss is evaluated by tests/fp64_reference.py (a float64 restatement of the
reference's projection, compositing and loss). The means are not differentiated in
the view-dependent scene: like the reference (tests/gradcheck.cpp:344), the backward
does not carry the SH view direction's dependence on the mean.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from fp64_reference import finite_differences  # noqa: E402
from parity_util import BACKGROUND  # noqa: E402
from smooth_scenes import smooth_scene  # noqa: E402


def main():
    out = {}
    for vd in (False, True):
        g, cam, gt = smooth_scene(view_dependent=vd)
        fd = finite_differences(g.arrays(), cam, BACKGROUND, gt, 0.2, 3, h=1e-4, chunk=256,
                                skip=(0,) if vd else ())
        for name, a in zip(("means", "scales", "quats", "dc", "rest", "opacities"), fd):
            out[f"{'vd' if vd else 'flat'}_{name}"] = a.astype(np.float64)
    np.savez_compressed(os.path.join(HERE, "fd_smooth.npz"), **out)
    print("fd_smooth.npz", os.path.getsize(os.path.join(HERE, "fd_smooth.npz")), "bytes")


if __name__ == "__main__":
    main()
