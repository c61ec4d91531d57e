"""The allocation-free sort entry point, rt_radix_sort_pairs_static.

It exists for callers that cannot allocate device memory where they sort: a
plug-in whose host application owns every device allocation and only hands it
the buffers it works on, or a frame loop that cannot afford cudaMalloc and
cudaFree, which may synchronize the device. Its scratch is an array inside the
library, so this test checks, through the C ABI, that two calls in a row give
exactly the keys and values of the scratch-taking entry point
rt_radix_sort_pairs (integer outputs: exact), that the second call is not
disturbed by what the first left in the shared array, and that sizes above the
stated maximum are refused. This file is collected last so that a failure here
comes after every other test has run.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "rt_core.h")


def _max_n():
    m = re.search(r"#define RT_STATIC_SORT_MAX_N \(1u << (\d+)\)", open(HEADER).read())
    return 1 << int(m.group(1))


def _sort_with_scratch(lib, torch, keys, vals, bits, init):
    n = keys.numel()
    nb = C.c_size_t(0)
    assert lib.rt_sort_scratch_bytes(n, C.byref(nb)) == 0
    scratch = torch.empty(max(nb.value, 256), dtype=torch.uint8, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.rt_radix_sort_pairs(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()), n, bits, int(init),
                                   C.c_void_p(scratch.data_ptr()), scratch.numel(), st) == 0


def _sort_static(lib, torch, keys, vals, bits, init):
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.rt_radix_sort_pairs_static(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()), keys.numel(), bits,
                                          int(init), st)


def test_static_sort_matches_scratch_sort_twice():
    import torch
    from cudart_b200 import _abi
    lib = _abi.lib()
    lib.rt_radix_sort_pairs_static.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
    lib.rt_radix_sort_pairs_static.restype = C.c_int
    max_n = _max_n()
    assert max_n >= 1 << 20
    rng = np.random.default_rng(2024)
    # two different calls in a row: a large one, then a smaller one with other
    # digits, so that a stale scratch would show up in the second result
    for n, bits, init in ((max_n, 32, True), (300007, 21, False)):
        keys = rng.integers(0, 1 << bits, n, dtype=np.int64).astype(np.uint32).view(np.int32)
        vals = rng.integers(0, 1 << 31, n, dtype=np.int64).astype(np.int32)
        k_ref = torch.from_numpy(keys.copy()).cuda()
        v_ref = torch.from_numpy(vals.copy()).cuda()
        k_new = k_ref.clone()
        v_new = v_ref.clone()
        _sort_with_scratch(lib, torch, k_ref, v_ref, bits, init)
        assert _sort_static(lib, torch, k_new, v_new, bits, init) == 0
        torch.cuda.synchronize()
        assert torch.equal(k_new, k_ref)
        assert torch.equal(v_new, v_ref)


def test_static_sort_rejects_oversize():
    import torch
    from cudart_b200 import _abi
    lib = _abi.lib()
    lib.rt_radix_sort_pairs_static.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
    max_n = _max_n()
    k = torch.zeros(8, dtype=torch.int32, device="cuda")
    # the size check comes before any access, so small buffers are never touched
    status = lib.rt_radix_sort_pairs_static(C.c_void_p(k.data_ptr()), C.c_void_p(k.data_ptr()), max_n + 1, 32, 0, None)
    assert status == 5  # RT_ERR_CAPACITY
    assert lib.rt_status_string(status) == b"capacity exceeded"


def test_static_sort_sizes_that_skip_the_scratch():
    """Sizes whose sort never touches the shared array: one key (only the values may be set) and up to one
    4096-key tile (a single-block sort in shared memory), plus 4097 keys, the first size that uses the array;
    each compared exactly with rt_radix_sort_pairs."""
    import torch
    from cudart_b200 import _abi
    lib = _abi.lib()
    lib.rt_radix_sort_pairs_static.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
    lib.rt_radix_sort_pairs_static.restype = C.c_int
    rng = np.random.default_rng(7)
    for n, bits, init in ((1, 32, True), (1, 32, False), (4096, 32, True), (4096, 8, False), (4097, 21, True), (4097, 32, False)):
        keys = rng.integers(0, 1 << bits, n, dtype=np.int64).astype(np.uint32).view(np.int32)
        vals = rng.integers(1, 1 << 31, n, dtype=np.int64).astype(np.int32)  # nonzero: an unset value would show
        k_ref = torch.from_numpy(keys.copy()).cuda()
        v_ref = torch.from_numpy(vals.copy()).cuda()
        k_new, v_new = k_ref.clone(), v_ref.clone()
        _sort_with_scratch(lib, torch, k_ref, v_ref, bits, init)
        assert _sort_static(lib, torch, k_new, v_new, bits, init) == 0
        torch.cuda.synchronize()
        assert torch.equal(k_new, k_ref), (n, bits, init)
        assert torch.equal(v_new, v_ref), (n, bits, init)
        if init:
            assert torch.equal(torch.sort(v_new.long()).values, torch.arange(n, device="cuda")), (n, bits)
