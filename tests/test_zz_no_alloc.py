"""The scan entry point that allocates nothing (b3_prefix_scan_u32_static).

It exists for callers that cannot call cudaMalloc, such as an engine that
owns all GPU memory through its own pool or a real-time loop that must
never allocate: its scratch is a fixed device array inside the library.
This test calls it through the C ABI twice in a row (the shared array keeps
the previous call's contents, which each call must clear) and checks both
results, element for element, against the allocating b3_prefix_scan_u32.
The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from experiments_b200 import b3

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def test_static_scan_matches_allocating_scan_twice(ctx):
    lib = b3.load()
    rng = np.random.default_rng(2024)
    # two calls of different sizes; the second is smaller so stale tile
    # status from the first call would corrupt it if it were not cleared
    for n in (3000017, 1000003):
        x = rng.integers(0, 1000, n).astype(np.uint32)
        src = _dev(x)
        ref = _dev(np.zeros(n, np.uint32))
        out = _dev(np.full(n, 0xFFFFFFFF, np.uint32))
        dsum = _dev(np.zeros(1, np.uint32))
        # the error flag comes back 0 after a valid scan (set to 7 first so a
        # call that never writes it would show)
        derr = _dev(np.full(1, 7, np.uint32))
        total_ref = b3.PrefixScan(ctx).execute(src, ref)
        rc = lib.b3_prefix_scan_u32_static(C.c_void_p(src.data_ptr()), C.c_void_p(out.data_ptr()), n,
                                           C.c_void_p(dsum.data_ptr()), C.c_void_p(derr.data_ptr()), None)
        assert rc == 0, lib.b3_last_error()
        torch.cuda.synchronize()
        assert int(derr.cpu().numpy()[0]) == 0
        got = out.cpu().numpy().view(np.uint32)
        want = ref.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want)
        assert int(dsum.cpu().numpy().view(np.uint32)[0]) == total_ref == int(x.astype(np.uint64).sum())


def test_static_scan_rejects_oversized_input(ctx):
    lib = b3.load()
    rc = lib.b3_prefix_scan_u32_static(C.c_void_p(16), C.c_void_p(16), (1 << 24) + 1, None, None, None)
    assert rc == 3  # B3_ERR_CAPACITY, nothing launched
    assert b"exceeds the static limit" in lib.b3_last_error()
