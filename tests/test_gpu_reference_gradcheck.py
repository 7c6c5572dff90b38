"""The reference's own gradient check on this backend.

tests/gradcheck.cpp of the reference runs five training-step gradient checks against
central finite differences through the backend contract (core/metal/bindings.h): L1,
SSIM, L1 + SSIM, view-dependent colour, and the prior-guided step with depth / sky /
fill priors, a learned sky and exposure (gradients of the Gaussians, the exposure
parameters and the sky texels). It is linked against this library through
msplat_street_b200/integration/bindings_cuda.cpp, the bindings.h implementation over
the C-ABI, at build time where the reference sources are present; the binary runs
here without them.
"""
import os
import subprocess

import pytest

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "msplat_street_b200", "_build",
                   "gradcheck_cuda")

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(BIN), reason="gradcheck_cuda not built (needs the reference sources)")
def test_reference_gradcheck_passes_on_this_backend():
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out
    assert out.strip().endswith("OK"), out
    # every run reports its checked gradients; none may mismatch
    runs = [line for line in out.splitlines() if "gradients match" in line]
    assert len(runs) == 5, out
    for line in runs:
        got, total = line.split("gradients match")[0].split()[-1].split("/")
        assert got == total, line
