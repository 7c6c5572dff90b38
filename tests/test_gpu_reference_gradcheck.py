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


TRAIN_BIN = os.path.join(os.path.dirname(BIN), "train_bindings")


@pytest.mark.skipif(not os.path.exists(TRAIN_BIN), reason="train_bindings not built (needs the reference headers)")
def test_training_through_bindings_h_with_host_tensors():
    """integration/train_bindings.cpp trains the small plain config through bindings.h
    with host tensors, as the reference's Model / CLI hold them: every call stages its
    tensors through the persistent device buffers and back. It must run, report its
    throughput, and its loss must fall from the first steps to the last. The same
    training from C++ through the C-ABI with device-resident tensors (mode c_abi) ends
    at the same loss: the staging only moves bytes."""
    import json
    first = subprocess.run([TRAIN_BIN, "2", "0"], capture_output=True, text=True, timeout=300)
    last = subprocess.run([TRAIN_BIN, "150", "0"], capture_output=True, text=True, timeout=300)
    direct = subprocess.run([TRAIN_BIN, "150", "0", "c_abi"], capture_output=True, text=True, timeout=300)
    for r in (first, last, direct):
        assert r.returncode == 0, r.stdout + r.stderr
    a = json.loads(first.stdout.strip().splitlines()[-1])
    b = json.loads(last.stdout.strip().splitlines()[-1])
    c = json.loads(direct.stdout.strip().splitlines()[-1])
    assert b["iters_per_s"] > 0 and b["steps"] == 150
    assert b["final_loss"] < a["final_loss"], (a, b)
    assert c["mode"] == "c_abi" and c["final_loss"] == b["final_loss"], (b, c)
