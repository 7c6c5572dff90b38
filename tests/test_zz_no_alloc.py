"""The allocation-free radix sort, msplat_cuda_radix_sort_static (needs a GPU).

Some callers may not allocate GPU memory at the moment they sort: a serving process
whose HBM is fully committed to resident scenes, a render loop that cannot take the
device-wide synchronisation cudaMalloc / cudaFree imply, a plugin host that forbids
libraries to allocate. They use this variant, whose scratch is one fixed array in
device memory instead of buffers grown on demand in a context.

This test calls it through the C-ABI, twice in a row (the array keeps the previous
call's contents between calls), and checks each result against the context-based
msplat_cuda_radix_sort on the same keys -- bit for bit, the bar of every sort test
here -- and against NumPy's stable argsort. It also checks that a size beyond the
array's capacity is refused with a message. This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from msplat_street_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20  # MSPLAT_STATIC_SORT_MAX_KEYS in include/msplat_cuda.h


def _context_sort(keys: np.ndarray, bits: int):
    lib = _lib.lib()
    ctx = C.c_void_p()
    _lib.check(lib.msplat_cuda_ctx_create(C.byref(ctx)))
    try:
        _lib.check(lib.msplat_cuda_ctx_set_stream(ctx, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        k = torch.from_numpy(keys.view(np.int64)).cuda()
        v = torch.arange(keys.size, dtype=torch.int32, device="cuda")
        _lib.check(lib.msplat_cuda_radix_sort(ctx, C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), keys.size,
                                              bits))
        torch.cuda.synchronize()
        return k.cpu().numpy().view(np.uint64), v.cpu().numpy()
    finally:
        lib.msplat_cuda_ctx_destroy(ctx)


def _static_sort(keys: np.ndarray, bits: int):
    lib = _lib.lib()
    k = torch.from_numpy(keys.view(np.int64)).cuda()
    v = torch.arange(keys.size, dtype=torch.int32, device="cuda")
    _lib.check(lib.msplat_cuda_radix_sort_static(C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                                 C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), keys.size, bits))
    torch.cuda.synchronize()
    return k.cpu().numpy().view(np.uint64), v.cpu().numpy()


@pytest.mark.parametrize("n,bits,hi", [(1000, 32, 2 ** 30), (300_001, 43, 2 ** 43), (MAX_KEYS, 64, 2 ** 63)])
def test_static_sort_matches_context_sort_on_two_calls(n, bits, hi):
    rng = np.random.default_rng(n + bits)
    for call in range(2):  # two calls in a row, different keys each time
        keys = rng.integers(0, hi, n, dtype=np.uint64)
        want_k, want_v = _context_sort(keys, bits)
        got_k, got_v = _static_sort(keys, bits)
        np.testing.assert_array_equal(got_k, want_k, err_msg=f"call {call}")
        np.testing.assert_array_equal(got_v, want_v, err_msg=f"call {call}")
        mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(2 ** 64 - 1)
        np.testing.assert_array_equal(got_v, np.argsort(keys & mask, kind="stable"), err_msg=f"call {call}")


def test_static_sort_allocates_no_device_memory():
    """After a first call (which looks up the array's address), a 2^20-key sort leaves
    the device's free memory where it was; the context sort of the same keys grows
    about 13 MB of scratch in its context."""
    n = MAX_KEYS
    keys = np.random.default_rng(1).integers(0, 2 ** 63, n, dtype=np.uint64)
    k = torch.from_numpy(keys.view(np.int64)).cuda()
    v = torch.arange(n, dtype=torch.int32, device="cuda")
    lib = _lib.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.msplat_cuda_radix_sort_static(st, C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), n, 64))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        _lib.check(lib.msplat_cuda_radix_sort_static(st, C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), n, 64))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_static_sort_refuses_more_keys_than_its_array_holds():
    lib = _lib.lib()
    n = MAX_KEYS + 1
    k = torch.zeros(n, dtype=torch.int64, device="cuda")
    v = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = lib.msplat_cuda_radix_sort_static(None, C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), n, 32)
    assert st == 3
    assert b"exceed the static scratch capacity" in lib.msplat_cuda_last_error()
