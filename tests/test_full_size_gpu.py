"""The hot path at its full benchmark sizes (2^28 elements; 2^27 for the 64-bit and float
sorts), checked on the device through properties that do not depend on the size: a sort's
output is ordered, stable and a permutation of its input that carries the values along; a
scan agrees with an int64 / float64 cumulative sum modulo the element width; a compaction
equals torch's boolean selection; a reduction agrees with a float64 sum within the FP32
bound (relative 1e-5).  The CPU oracle checks the same kernels element by element at the
sizes it finishes in seconds (test_raw_kernels_gpu.py and the others); these tests add the
sizes where tile counts, look-back chains and 32-bit status words reach their limits.
All calls go through the library's C ABI on device buffers.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N28 = 1 << 28
N27 = 1 << 27
REL_TOL = 1e-5


@pytest.fixture(scope="module")
def N(cuda):
    from thrustrtc_b200 import _native
    return _native


def P(t):
    return ctypes.c_void_p(t.data_ptr())


def gen(seed):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return g


def rand_u32_as_i32(n, seed):
    """uniform 32-bit patterns in an int32 tensor (the bits are the uint32 keys)"""
    import torch
    x = torch.randint(0, 1 << 32, (n,), dtype=torch.int64, device="cuda", generator=gen(seed))
    return (x - (x >= (1 << 31)).to(torch.int64) * (1 << 32)).to(torch.int32)


def check_sorted_pairs(k0, k, v, key_u32, desc=False):
    """k ordered (stable: equal keys keep their value order), v a permutation, and, when k0
    is given, k == k0[v]"""
    import torch
    kk = (k.to(torch.int64) & 0xFFFFFFFF) if key_u32 else k
    if desc:
        assert bool((kk[1:] <= kk[:-1]).all())
    else:
        assert bool((kk[1:] >= kk[:-1]).all())
    perm = v.to(torch.int64)
    eq = kk[1:] == kk[:-1]
    assert bool((perm[1:][eq] > perm[:-1][eq]).all())
    assert int(torch.bincount(perm, minlength=k.numel()).max()) == 1
    if k0 is not None:
        assert torch.equal(k0[perm], k)


@pytest.mark.parametrize("desc", [False, True])
def test_sort_by_key_u32_pairs_2e28(N, desc):
    import torch
    k0 = rand_u32_as_i32(N28, 1 + desc)
    k, v = k0.clone(), torch.arange(N28, dtype=torch.int32, device="cuda")
    assert N.lib.trtc_raw_sort_by_key(5, P(k), P(v), 4, N28, int(desc), None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    check_sorted_pairs(k0, k, v, True, desc)


def test_sort_by_key_u32_pairs_past_2e30(N):
    # n >= 2^30: the digit passes switch to 64-bit look-back status words and positions; the
    # last tile is partial (its payloads take the per-element copies, the others the bulk copy)
    import torch
    n = (1 << 30) + 4099
    k0 = rand_u32_as_i32(n, 30)
    k, v = k0.clone(), torch.arange(n, dtype=torch.int32, device="cuda")
    assert N.lib.trtc_raw_sort_by_key(5, P(k), P(v), 4, n, 0, None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    check_sorted_pairs(k0, k, v, True)
    del k0, k, v
    torch.cuda.empty_cache()


def test_sort_u32_keys_narrow_range_2e28(N):
    # 1000 distinct keys: two of the four digit passes are skipped, the others carry long runs
    import torch
    k0 = torch.randint(0, 1000, (N28,), dtype=torch.int32, device="cuda", generator=gen(3))
    k = k0.clone()
    assert N.lib.trtc_raw_sort(5, P(k), N28, 0, None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    assert torch.equal(k, torch.sort(k0)[0])


def test_sort_by_key_i64_zipf_2e27(N):
    # Zipf(1.1) ranks over 2^20 distinct 64-bit keys sharing their upper 32 bits
    import torch
    u = torch.rand(N27, dtype=torch.float64, device="cuda", generator=gen(4))
    ranks = torch.arange(1, (1 << 20) + 1, dtype=torch.float64, device="cuda")
    cdf = torch.cumsum(ranks ** -1.1, 0)
    cdf /= cdf[-1].clone()
    r = torch.searchsorted(cdf, u).clamp_(max=(1 << 20) - 1) + 1
    k0 = 0x0123456700000000 + ((r * 0x9E3B1) & ((1 << 20) - 1))
    k, v = k0.clone(), torch.arange(N27, dtype=torch.int32, device="cuda")
    assert N.lib.trtc_raw_sort_by_key(6, P(k), P(v), 4, N27, 0, None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    check_sorted_pairs(k0, k, v, False)


def test_sort_by_key_f32_2e27(N):
    # normal floats with 1% -0.0 and 0.1% NaN.  The reference orders a float key x by
    # d(x) = its bits, or 2^32 minus its magnitude bits when the sign is set (so -0.0 and +0.0
    # are equal), taken relative to d(minimum element) modulo 2^32 (NaNs move that base); the
    # output starts at that base, so its rotated codes must be ascending and stable
    import torch
    g = gen(5)
    x = torch.randn(N27, dtype=torch.float32, device="cuda", generator=g)
    sel = torch.randint(0, 1000, (N27,), dtype=torch.int32, device="cuda", generator=g)
    x[sel < 10] = -0.0
    x[sel == 10] = float("nan")
    k0 = x.view(torch.int32).clone()
    k, v = k0.clone(), torch.arange(N27, dtype=torch.int32, device="cuda")
    assert N.lib.trtc_raw_sort_by_key(8, P(k), P(v), 4, N27, 0, None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    b = k.to(torch.int64) & 0xFFFFFFFF
    d = torch.where((b >> 31) == 1, (-(b & 0x7FFFFFFF)) & 0xFFFFFFFF, b)
    check_sorted_pairs(None, (d - d[0]) & 0xFFFFFFFF, v, False)  # codes ordered, stable, permutation
    assert torch.equal(k0[v.to(torch.int64)], k)


@pytest.mark.parametrize("excl", [False, True])
def test_scan_i32_2e28(N, excl):
    import torch
    x = torch.randint(-1000, 1001, (N28,), dtype=torch.int32, device="cuda", generator=gen(6))
    out = torch.empty_like(x)
    init = np.array([7], np.int32)
    ini = init.ctypes.data_as(ctypes.c_void_p) if excl else None
    assert N.lib.trtc_raw_scan(4, 0, int(excl), P(x), P(out), N28, ini, None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    ref = torch.cumsum(x, 0, dtype=torch.int64)
    if excl:
        ref = torch.cat([torch.zeros(1, dtype=torch.int64, device="cuda"), ref[:-1]]) + 7
    assert bool((((out.to(torch.int64) - ref) & 0xFFFFFFFF) == 0).all())  # equal modulo 2^32


def test_scan_max_u32_2e28(N):
    import torch
    x = rand_u32_as_i32(N28, 7)
    out = torch.empty_like(x)
    assert N.lib.trtc_raw_scan(5, 1, 0, P(x), P(out), N28, None, None) == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
    ref = torch.cummax(x.to(torch.int64) & 0xFFFFFFFF, 0)[0]
    assert torch.equal(out.to(torch.int64) & 0xFFFFFFFF, ref)


def test_reduce_f32_2e28(N):
    import torch
    x = torch.rand(N28, dtype=torch.float32, device="cuda", generator=gen(8))
    res = np.zeros(1, np.float32)
    for op, init in ((0, None), (1, -1.0), (2, 2.0)):  # Plus from 0; Maximum / Minimum past x's range
        iv = np.array([0.0 if init is None else init], np.float32)
        ini = None if init is None else iv.ctypes.data_as(ctypes.c_void_p)
        assert N.lib.trtc_raw_reduce(8, op, P(x), N28, ini, res.ctypes.data_as(ctypes.c_void_p), None) == 0
        if op == 0:
            exp = float(x.double().sum())
            assert abs(float(res[0]) - exp) <= REL_TOL * abs(exp), (float(res[0]), exp)
        else:
            assert float(res[0]) == float(x.max() if op == 1 else x.min())


def test_scan_by_key_f32_2e28(N):
    # runs of Geometric(1/32) length; integer-valued float values make every order of summation
    # exact, so the segmented scan must equal the float64 reference bit for bit
    import torch
    g = gen(9)
    heads = torch.rand(N28, device="cuda", generator=g) < (1.0 / 32.0)
    heads[0] = True
    keys = (torch.cumsum(heads, 0, dtype=torch.int64) - 1).to(torch.int32)
    vals = torch.randint(0, 16, (N28,), device="cuda", generator=g).to(torch.float32)
    out = torch.empty_like(vals)
    for excl in (False, True):
        assert N.lib.trtc_raw_scan_by_key(4, 8, int(excl), P(keys), P(vals), P(out), N28, None, None) == 0
        assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
        cs = torch.cumsum(vals.double(), 0)
        idx = torch.arange(N28, device="cuda")
        start = torch.cummax(torch.where(heads, idx, torch.zeros_like(idx)), 0)[0]
        ref = cs - (cs[start] - vals[start].double())
        if excl:
            ref = ref - vals.double()
        assert torch.equal(out.double(), ref)


def test_copy_if_functor_2e28(N):
    # the user Functor is compiled by NVRTC into the compaction kernel
    import torch
    import thrustrtc_b200 as trtc
    trtc.init()
    x = rand_u32_as_i32(N28, 10)
    dst = torch.empty_like(x)
    vin = trtc.DVVectorAdaptor("int32_t", N28, x.data_ptr())
    vout = trtc.DVVectorAdaptor("int32_t", N28, dst.data_ptr())
    c = trtc.Copy_If(vin, vout, trtc.Functor({}, ["x"], "        return (x & 1) != 0;\n"))
    sel = x[(x & 1) != 0]
    assert c == sel.numel() and torch.equal(dst[:c], sel)


def test_remove_and_unique_2e28(N):
    import torch
    x = torch.randint(0, 4, (N28,), dtype=torch.int32, device="cuda", generator=gen(11))
    out = torch.empty_like(x)
    val = np.array([2], np.int32)
    c = N.lib.trtc_raw_remove_copy(4, P(x), P(out), N28, val.ctypes.data_as(ctypes.c_void_p), None)
    sel = x[x != 2]
    assert c == sel.numel() and torch.equal(out[:c], sel)
    ref = torch.unique_consecutive(x)
    c = N.lib.trtc_raw_unique_copy(4, P(x), P(x), N28, None)  # in place
    assert c == ref.numel() and torch.equal(x[:c], ref)
