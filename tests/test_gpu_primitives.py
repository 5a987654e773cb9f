"""GPU primitives (fill, prefix scan, radix sort, bound search) against
numpy, after the reference's primitive tests
(opencl/primitives/AdlTest/main.cpp: fillIntTest :68-109, boundSearchTest
:129-228, prefixScanTest :232-273, radixSortTest :277-325)."""
import numpy as np
import pytest
import torch

from experiments_b200 import b3

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


SORT_CASES = [(0, 8), (1, 8), (2, 1), (5, 8), (255, 4), (4095, 13), (4096, 18), (4097, 24), (65536, 8),
              (100003, 32), (1 << 20, 20), (3000017, 26)]


@pytest.mark.parametrize("n,bits", SORT_CASES)
def test_radix_sort_kv_is_stable_sort(ctx, n, bits):
    rng = np.random.default_rng(1000 + n + bits)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    vals = rng.permutation(n).astype(np.uint32)
    dk, dv = _dev(keys), _dev(vals)
    b3.RadixSort32(ctx).execute(dk, dv, key_bits=bits)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(_host(dk), keys[order])
    assert np.array_equal(_host(dv), vals[order])


@pytest.mark.parametrize("dist", ["few", "sorted", "reversed", "constant"])
def test_radix_sort_distributions(ctx, dist):
    n = 200001
    rng = np.random.default_rng(7)
    if dist == "few":
        keys = rng.integers(0, 3, n).astype(np.uint32) * 77777
    elif dist == "sorted":
        keys = np.sort(rng.integers(0, 1 << 24, n)).astype(np.uint32)
    elif dist == "reversed":
        keys = np.sort(rng.integers(0, 1 << 24, n))[::-1].astype(np.uint32)
    else:
        keys = np.full(n, 123456, np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = _dev(keys), _dev(vals)
    b3.RadixSort32(ctx).execute(dk, dv, key_bits=24)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(_host(dk), keys[order])
    assert np.array_equal(_host(dv), vals[order])


def test_radix_sort_keys_only(ctx):
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 32, 1 << 18, dtype=np.uint64).astype(np.uint32)
    dk = _dev(keys)
    b3.RadixSort32(ctx).execute(dk, None, key_bits=32)
    torch.cuda.synchronize()
    assert np.array_equal(_host(dk), np.sort(keys))


@pytest.mark.parametrize("n", [0, 1, 7, 4096, 4097, 1000003, 10000000])
def test_prefix_scan_exclusive(ctx, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 100, n).astype(np.uint32)
    src, dst = _dev(x), _dev(np.zeros(n, np.uint32))
    total = b3.PrefixScan(ctx).execute(src, dst)
    ref = np.concatenate([[0], np.cumsum(x.astype(np.uint64))[:-1]]).astype(np.uint32) if n else x
    assert np.array_equal(_host(dst), ref[:n])
    assert total == int(x.astype(np.uint64).sum())


def test_prefix_scan_all_ones_in_place(ctx):
    n = 524289  # one past the reference's 2,048 x 256 top-level limit
    x = np.ones(n, np.uint32)
    d = _dev(x)
    total = b3.PrefixScan(ctx).execute(d, d)
    assert total == n
    assert np.array_equal(_host(d), np.arange(n, dtype=np.uint32))


@pytest.mark.parametrize("n", [1, 100, 4096, 65537])
def test_bound_search(ctx, n):
    rng = np.random.default_rng(n)
    keys = np.sort(rng.integers(0, 256, n)).astype(np.uint32)
    dk = _dev(keys)
    nd = 256
    lo = _dev(np.full(nd, 0xFFFFFFFF, np.uint32))
    up = _dev(np.full(nd, 0xFFFFFFFF, np.uint32))
    cnt = _dev(np.zeros(nd, np.uint32))
    bs = b3.BoundSearch(ctx)
    bs.execute(dk, n, lo, nd, bs.LOWER)
    bs.execute(dk, n, up, nd, bs.UPPER)
    bs.execute(dk, n, cnt, nd, bs.COUNT)
    torch.cuda.synchronize()
    L, U, Cn = _host(lo), _host(up), _host(cnt)
    for k in range(nd):
        present = np.any(keys == k)
        if present:
            assert L[k] == np.searchsorted(keys, k, "left")
            assert U[k] == np.searchsorted(keys, k, "right")
            assert np.all(keys[L[k]:U[k]] == k)
        else:
            assert L[k] == 0xFFFFFFFF and U[k] == 0xFFFFFFFF
        assert Cn[k] == np.count_nonzero(keys == k)


def test_fill(ctx):
    d = _dev(np.zeros(1000, np.uint32))
    b3.Fill(ctx).execute(d, 0xDEADBEEF, n=500, offset=250)
    h = _host(d)
    assert np.all(h[250:750] == 0xDEADBEEF) and np.all(h[:250] == 0) and np.all(h[750:] == 0)
    d2 = torch.zeros((64, 2), dtype=torch.int32, device="cuda")
    b3.Fill(ctx).execute(d2, (7, -3), n=32, offset=16)
    h2 = d2.cpu().numpy()
    assert np.all(h2[16:48] == [7, -3]) and np.all(h2[:16] == 0) and np.all(h2[48:] == 0)


# --- the btSortData and out-of-place forms (BB/btRadixSort32CL.h:67-70,
# BB/btBoundSearchCL.h:60), each against the split-array form


@pytest.mark.parametrize("n,bits", [(2, 32), (4097, 32), (1000003, 32), (300000, 13), (70000, 8), (5, 4)])
def test_sortdata_sort_matches_split_form(ctx, n, bits):
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    kv = np.stack([keys, vals], 1).view(np.int32).copy()
    dkv = torch.from_numpy(kv).cuda()
    dk, dv = _dev(keys), _dev(vals)
    s = b3.RadixSort32(ctx)
    s.execute_sortdata(dkv, key_bits=bits)
    s.execute(dk, dv, key_bits=bits)
    torch.cuda.synchronize()
    out = dkv.cpu().numpy().view(np.uint32)
    assert np.array_equal(out[:, 0], _host(dk)) and np.array_equal(out[:, 1], _host(dv))
    # stable: the numpy stable order
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(out[:, 1], order.astype(np.uint32))


@pytest.mark.parametrize("n,bits,with_values", [(3, 32, True), (65537, 32, True), (500000, 24, True),
                                                (200000, 16, False), (9999, 7, True)])
def test_out_of_place_sort_leaves_inputs(ctx, n, bits, with_values):
    rng = np.random.default_rng(7 * n + bits)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    vals = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    ki, ko = _dev(keys), _dev(np.zeros(n, np.uint32))
    vi = _dev(vals) if with_values else None
    vo = _dev(np.zeros(n, np.uint32)) if with_values else None
    b3.RadixSort32(ctx).execute_out(ki, ko, vi, vo, key_bits=bits)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(_host(ko), keys[order])
    assert np.array_equal(_host(ki), keys)
    if with_values:
        assert np.array_equal(_host(vo), vals[order]) and np.array_equal(_host(vi), vals)


def test_out_of_place_sort_rejects_aliased_outputs(ctx):
    k = _dev(np.arange(10, dtype=np.uint32))
    with pytest.raises(b3.B3Error):
        b3.RadixSort32(ctx).execute_out(k, k)


@pytest.mark.parametrize("n", [1, 100, 4096, 65537])
def test_sortdata_bound_search(ctx, n):
    rng = np.random.default_rng(n + 11)
    keys = np.sort(rng.integers(1 if n == 100 else 0, 256, n)).astype(np.uint32)
    kv = np.stack([keys, np.arange(n, dtype=np.uint32)], 1).view(np.int32).copy()
    dkv = torch.from_numpy(kv).cuda()
    dk = _dev(keys)
    nd = 256
    bs = b3.BoundSearch(ctx)
    for mode in (bs.LOWER, bs.UPPER, bs.COUNT):
        a = _dev(np.full(nd, 0xFFFFFFFF, np.uint32))
        b = _dev(np.full(nd, 0xFFFFFFFF, np.uint32))
        bs.execute_sortdata(dkv, n, a, nd, mode)
        bs.execute(dk, n, b, nd, mode)
        torch.cuda.synchronize()
        A, B = _host(a), _host(b)
        if mode == bs.UPPER and keys[0] != 0:
            # SearchSortDataUpperKernel: upper bound of an absent key 0 is 0
            assert A[0] == 0
            A[0] = B[0]
        assert np.array_equal(A, B), mode
