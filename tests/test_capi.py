"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU
needed: nothing here launches a kernel), and argument errors come back as status
codes with messages, as the reference's exceptions do."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from msplat_street_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(msplat_cuda_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("msplat_cuda_render", "msplat_cuda_train_step", "msplat_cuda_sync", "msplat_cuda_alloc",
                     "msplat_cuda_copy_buffer", "msplat_cuda_cleanup"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.msplat_cuda_version() >= 100


def test_argument_errors_are_status_codes():
    lib = _lib.lib()
    ctx = C.c_void_p()
    assert lib.msplat_cuda_ctx_create(C.byref(ctx)) == 0
    vm = np.eye(4, dtype=np.float32)
    cp = np.zeros(3, np.float32)
    bg = np.zeros(3, np.float32)
    out = C.c_void_p()
    # tile bounds that do not match the image: rejected before any GPU work
    st = lib.msplat_cuda_render(ctx, 0, None, None, 1.0, None, vm.ctypes.data, vm.ctypes.data, 1.0, 1.0, 0.0, 0.0,
                                32, 32, 3, 2, 0.01, 0, 0, cp.ctypes.data, None, None, None, bg.ctypes.data,
                                C.byref(out))
    assert st == 1
    assert b"tile bounds" in lib.msplat_cuda_last_error()
    with pytest.raises(ValueError):
        _lib.check(st)
    st = lib.msplat_cuda_ctx_set_option(ctx, b"no_such_option", 1)
    assert st == 1 and b"unknown option" in lib.msplat_cuda_last_error()
    lib.msplat_cuda_ctx_destroy(ctx)


# the reference checkout: MSPLAT_REFERENCE_ROOT, else a `reference` directory beside the repository
REF = os.environ.get("MSPLAT_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "core", "metal", "bindings.h")),
                    reason="reference headers not present here")
def test_bindings_shim_links_the_reference_gradcheck():
    """integration/bindings_cuda.cpp implements every bindings.h function the
    reference's callers use: its own gradient check links against it unchanged."""
    from msplat_street_b200 import build
    path = build.build_reference_gradcheck(REF)
    assert os.path.exists(path) and os.access(path, os.X_OK)
