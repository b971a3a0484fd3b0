"""Parity of the ThrustRTC-shaped API (thrustrtc_b200 package -> C ABI -> CUDA) with the
oracle.  The small cases are the reference's own test programs (python/test/test_*.py,
cpp/test/test_*.cpp) with their outputs checked instead of printed; the larger ones are
seeded random inputs.  Integer results are bit-exact; float sums use rel. tol. 1e-5.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL_TOL = 1e-5


@pytest.fixture(scope="module")
def trtc(cuda):
    import thrustrtc_b200 as t
    t.init()
    return t


def is_even(trtc):
    return trtc.Functor({}, ["x"], "\n         return x % 2 == 0;\n")


# ---------------------------------------------------------------- docs + reference tests
def test_docs_golden(trtc):
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "docs_vectors.json")))
    v = trtc.device_vector_from_list(d["inclusive_scan"]["in"], "int32_t")
    trtc.Inclusive_Scan(v, v)
    assert v.to_host().tolist() == d["inclusive_scan"]["out"]
    v = trtc.device_vector_from_list(d["exclusive_scan"]["in"], "int32_t")
    trtc.Exclusive_Scan(v, v)
    assert v.to_host().tolist() == d["exclusive_scan"]["out"]
    v = trtc.device_vector_from_list(d["sort"]["in"], "int32_t")
    trtc.Sort(v)
    assert v.to_host().tolist() == d["sort"]["out"]
    v = trtc.device_vector_from_list(d["sort"]["in"], "int32_t")
    trtc.Sort(v, trtc.Greater())
    assert v.to_host().tolist() == d["sort_greater"]["out"]
    for case in ("sort_by_key_char", "sort_by_key_int"):
        c = d[case]
        k = trtc.device_vector_from_list(c["keys"], c["key_dtype"])
        val = trtc.device_vector_from_list(c["values"], c["value_dtype"])
        trtc.Sort_By_Key(k, val)
        assert k.to_host().tolist() == c["keys_out"] and val.to_host().tolist() == c["values_out"]


def test_reference_scan_program(trtc):
    # python/test/test_scan.py and cpp/test/test_scan.cpp
    data = [1, 0, 2, 2, 1, 3]
    mx = [-5, 0, 2, -3, 2, 4, 0, -1, 2, 8]
    a = np.array(data, np.int32)
    b = np.array(mx, np.int32)
    d = trtc.device_vector_from_list(data, "int32_t"); trtc.Inclusive_Scan(d, d)
    assert d.to_host().tolist() == O.scan(a).tolist()
    d = trtc.device_vector_from_list(mx, "int32_t"); trtc.Inclusive_Scan(d, d, trtc.Maximum())
    assert d.to_host().tolist() == O.scan(b, "Maximum").tolist()
    d = trtc.device_vector_from_list(data, "int32_t"); trtc.Exclusive_Scan(d, d)
    assert d.to_host().tolist() == O.scan(a, exclusive=True).tolist()
    d = trtc.device_vector_from_list(data, "int32_t"); trtc.Exclusive_Scan(d, d, trtc.DVInt32(4))
    assert d.to_host().tolist() == O.scan(a, exclusive=True, init=4).tolist()
    d = trtc.device_vector_from_list(mx, "int32_t"); trtc.Exclusive_Scan(d, d, trtc.DVInt32(1), trtc.Maximum())
    assert d.to_host().tolist() == O.scan(b, "Maximum", True, 1).tolist()
    # scan of a computed view: DVCounter(1), 1000 elements (cpp/test/test_scan.cpp:10-31)
    cnt = trtc.DVCounter(trtc.DVInt32(1), 1000)
    out = trtc.device_vector("int32_t", 1000)
    trtc.Inclusive_Scan(cnt, out)
    assert out.to_host().tolist() == O.scan(np.arange(1, 1001, dtype=np.int32)).tolist()
    trtc.Exclusive_Scan(cnt, out)
    assert out.to_host().tolist() == O.scan(np.arange(1, 1001, dtype=np.int32), exclusive=True).tolist()


def test_reference_transform_scan_and_reduce(trtc):
    data = [1, 0, 2, 2, 1, 3]
    d = trtc.device_vector_from_list(data, "int32_t")
    trtc.Transform_Inclusive_Scan(d, d, trtc.Negate(), trtc.Plus())
    assert d.to_host().tolist() == O.scan(-np.array(data, np.int32)).tolist()
    d = trtc.device_vector_from_list(data, "int32_t")
    trtc.Transform_Exclusive_Scan(d, d, trtc.Negate(), trtc.DVInt32(4), trtc.Plus())
    assert d.to_host().tolist() == O.scan(-np.array(data, np.int32), exclusive=True, init=4).tolist()
    d = trtc.device_vector_from_list([-1, 0, -2, -2, 1, -3], "int32_t")
    absolute = trtc.Functor({}, ["x"], "\n         return x<(decltype(x))0 ? -x : x;\n")
    assert trtc.Transform_Reduce(d, absolute, trtc.DVInt32(0), trtc.Maximum()) == 3


def test_reference_reduce_program(trtc):
    d = trtc.device_vector_from_list([1, 0, 2, 2, 1, 3], "int32_t")
    assert trtc.Reduce(d) == 9
    assert trtc.Reduce(d, trtc.DVInt32(1)) == 10
    assert trtc.Reduce(d, trtc.DVInt32(-1), trtc.Maximum()) == 3
    kin = trtc.device_vector_from_list([1, 3, 3, 3, 2, 2, 1], "int32_t")
    vin = trtc.device_vector_from_list([9, 8, 7, 6, 5, 4, 3], "int32_t")
    kout = trtc.device_vector("int32_t", 7)
    vout = trtc.device_vector("int32_t", 7)
    ek, ev = O.reduce_by_key(np.array([1, 3, 3, 3, 2, 2, 1]), np.array([9, 8, 7, 6, 5, 4, 3], np.int32))
    for args in ((), (trtc.EqualTo(),), (trtc.EqualTo(), trtc.Plus())):
        c = trtc.Reduce_By_Key(kin, vin, kout, vout, *args)
        assert kout.to_host(0, c).tolist() == ek.tolist() and vout.to_host(0, c).tolist() == ev.tolist()


def test_reference_copy_program(trtc):
    din = trtc.device_vector_from_list([10, 20, 30, 40, 50, 60, 70, 80], "int32_t")
    dout = trtc.device_vector("int32_t", 8)
    trtc.Copy(din, dout)
    assert dout.to_host().tolist() == [10, 20, 30, 40, 50, 60, 70, 80]
    din = trtc.device_vector_from_list([-2, 0, -1, 0, 1, 2], "int32_t")
    dout = trtc.device_vector("int32_t", 6)
    c = trtc.Copy_If(din, dout, is_even(trtc))
    assert dout.to_host(0, c).tolist() == [-2, 0, 0, 2]
    din = trtc.device_vector_from_list([0, 1, 2, 3, 4, 5], "int32_t")
    st = trtc.device_vector_from_list([-2, 0, -1, 0, 1, 2], "int32_t")
    c = trtc.Copy_If_Stencil(din, st, dout, is_even(trtc))
    assert dout.to_host(0, c).tolist() == [0, 1, 3, 5]


def test_reference_partition_program(trtc):
    ev = is_even(trtc)
    v = trtc.device_vector_from_list(list(range(1, 11)), "int32_t")
    c = trtc.Partition(v, ev)
    exp, ec = O.partition(np.arange(1, 11), np.arange(1, 11) % 2 == 0)
    assert c == ec and v.to_host().tolist() == exp.tolist()
    v = trtc.device_vector_from_list([0, 1] * 5, "int32_t")
    s = trtc.device_vector_from_list(list(range(1, 11)), "int32_t")
    c = trtc.Partition_Stencil(v, s, ev)
    exp, ec = O.partition(np.array([0, 1] * 5), np.arange(1, 11) % 2 == 0)
    assert c == ec and v.to_host().tolist() == exp.tolist()
    v = trtc.device_vector_from_list(list(range(1, 11)), "int32_t")
    t = trtc.device_vector("int32_t", 10)
    f = trtc.device_vector("int32_t", 10)
    c = trtc.Partition_Copy(v, t, f, ev)
    assert t.to_host(0, c).tolist() == [2, 4, 6, 8, 10] and f.to_host(0, 10 - c).tolist() == [1, 3, 5, 7, 9]
    s = trtc.device_vector_from_list([0, 1] * 5, "int32_t")
    c = trtc.Partition_Copy_Stencil(v, s, t, f, trtc.Identity())
    assert t.to_host(0, c).tolist() == [2, 4, 6, 8, 10] and f.to_host(0, 10 - c).tolist() == [1, 3, 5, 7, 9]


def test_reference_remove_program(trtc):
    v = trtc.device_vector_from_list([3, 1, 4, 1, 5, 9], "int32_t")
    c = trtc.Remove(v, trtc.DVInt32(1))
    assert v.to_host(0, c).tolist() == [3, 4, 5, 9]
    din = trtc.device_vector_from_list([-2, 0, -1, 0, 1, 2], "int32_t")
    dout = trtc.device_vector("int32_t", 6)
    c = trtc.Remove_Copy(din, dout, trtc.DVInt32(0))
    assert dout.to_host(0, c).tolist() == [-2, -1, 1, 2]
    v = trtc.device_vector_from_list([1, 4, 2, 8, 5, 7], "int32_t")
    c = trtc.Remove_If(v, is_even(trtc))
    assert v.to_host(0, c).tolist() == [1, 5, 7]
    c = trtc.Remove_Copy_If(din, dout, is_even(trtc))
    assert dout.to_host(0, c).tolist() == [-1, 1]
    v = trtc.device_vector_from_list([1, 4, 2, 8, 5, 7], "int32_t")
    st = trtc.device_vector_from_list([0, 1, 1, 1, 0, 0], "int32_t")
    c = trtc.Remove_If_Stencil(v, st, trtc.Identity())
    assert v.to_host(0, c).tolist() == [1, 5, 7]
    st = trtc.device_vector_from_list([1, 1, 0, 1, 0, 1], "int32_t")
    c = trtc.Remove_Copy_If_Stencil(din, st, dout, trtc.Identity())
    assert dout.to_host(0, c).tolist() == [-1, 1]


def test_reference_unique_program(trtc):
    base = [1, 3, 3, 3, 2, 2, 1]
    for args in ((), (trtc.EqualTo(),)):
        v = trtc.device_vector_from_list(base, "int32_t")
        c = trtc.Unique(v, *args)
        assert v.to_host(0, c).tolist() == [1, 3, 2, 1]
        din = trtc.device_vector_from_list(base, "int32_t")
        dout = trtc.device_vector("int32_t", 7)
        c = trtc.Unique_Copy(din, dout, *args)
        assert dout.to_host(0, c).tolist() == [1, 3, 2, 1]
        k = trtc.device_vector_from_list(base, "int32_t")
        val = trtc.device_vector_from_list([9, 8, 7, 6, 5, 4, 3], "int32_t")
        c = trtc.Unique_By_Key(k, val, *args)
        assert k.to_host(0, c).tolist() == [1, 3, 2, 1] and val.to_host(0, c).tolist() == [9, 8, 5, 3]
        ko = trtc.device_vector("int32_t", 7)
        vo = trtc.device_vector("int32_t", 7)
        k = trtc.device_vector_from_list(base, "int32_t")
        val = trtc.device_vector_from_list([9, 8, 7, 6, 5, 4, 3], "int32_t")
        c = trtc.Unique_By_Key_Copy(k, val, ko, vo, *args)
        assert ko.to_host(0, c).tolist() == [1, 3, 2, 1] and vo.to_host(0, c).tolist() == [9, 8, 5, 3]


def test_reference_scan_by_key_program(trtc):
    keys = np.array([0, 0, 0, 1, 1, 2, 3, 3, 3, 3], np.int32)
    ones = np.ones(10, np.int32)
    k = trtc.device_vector_from_numpy(keys)
    v = trtc.device_vector_from_numpy(ones); trtc.Inclusive_Scan_By_Key(k, v, v)
    assert v.to_host().tolist() == O.scan_by_key(keys, ones).tolist()
    v = trtc.device_vector_from_numpy(ones); trtc.Exclusive_Scan_By_Key(k, v, v)
    assert v.to_host().tolist() == O.scan_by_key(keys, ones, exclusive=True, init=0).tolist()
    v = trtc.device_vector_from_numpy(ones); trtc.Exclusive_Scan_By_Key(k, v, v, trtc.DVInt32(5))
    assert v.to_host().tolist() == O.scan_by_key(keys, ones, exclusive=True, init=5).tolist()
    v = trtc.device_vector_from_numpy(ones); trtc.Exclusive_Scan_By_Key(k, v, v, trtc.DVInt32(5), trtc.EqualTo())
    assert v.to_host().tolist() == O.scan_by_key(keys, ones, exclusive=True, init=5).tolist()
    # cpp/test/test_scan_by_key.cpp:8-24: 1000 elements in runs of 300
    kk = (np.arange(1000) // 300).astype(np.int32)
    vv = (np.arange(1000) % 300).astype(np.int32)
    k = trtc.device_vector_from_numpy(kk)
    v = trtc.device_vector_from_numpy(vv)
    trtc.Inclusive_Scan_By_Key(k, v, v)
    assert v.to_host().tolist() == O.scan_by_key(kk, vv).tolist()


# ---------------------------------------------------------------- larger seeded cases
def test_copy_if_user_functor_large(trtc):
    # C3c shape: int32 uniform over the full range, predicate (x & 1) != 0 as a user Functor
    rng = np.random.default_rng(1)
    for n in (1, 4095, 4097, 1 << 22):
        x = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32)
        d = trtc.device_vector_from_numpy(x)
        o = trtc.device_vector("int32_t", n)
        odd = trtc.Functor({}, ["x"], "        return (x & 1) != 0;\n")
        c = trtc.Copy_If(d, o, odd)
        exp = x[(x & 1) != 0]
        assert c == len(exp) and o.to_host(0, c).tolist() == exp.tolist()


def test_sort_user_comparator_merge_path(trtc):
    rng = np.random.default_rng(2)
    for n in (1, 3, 511, 512, 513, 5000, 70001):
        k = rng.integers(-50, 50, n).astype(np.int32)
        v = np.arange(n, dtype=np.int32)
        dk, dv = trtc.device_vector_from_numpy(k), trtc.device_vector_from_numpy(v)
        gt = trtc.Functor({}, ["a", "b"], "        return a > b;\n")
        trtc.Sort_By_Key(dk, dv, gt)
        p = O.sort_perm(k, descending=True)
        assert dk.to_host().tolist() == k[p].tolist() and dv.to_host().tolist() == v[p].tolist()


def test_sort_views_and_types(trtc):
    rng = np.random.default_rng(3)
    for dt, cls in ((np.float32, "float"), (np.int64, "int64_t"), (np.uint16, "uint16_t"), (np.float64, "double")):
        n = 100003
        x = (rng.standard_normal(n) * 1000).astype(dt)
        if dt in (np.float32, np.float64):
            x[::97] = np.nan
            x[::89] = -0.0
        d = trtc.device_vector_from_numpy(x)
        r = trtc.DVRange(d, 7, n - 5)  # a sub-range sorts in place
        trtc.Sort(r)
        exp = x.copy()
        exp[7:n - 5] = O.sort(x[7:n - 5])
        assert d.to_host().tobytes() == exp.tobytes(), cls
        d = trtc.device_vector_from_numpy(x)
        trtc.Sort(d, trtc.Greater())
        assert d.to_host().tobytes() == O.sort(x, True).tobytes(), cls


def test_min_element_and_empty_inputs(trtc):
    x = np.array([5, np.nan, 3, 0], np.float32)
    assert trtc.Min_Element(trtc.device_vector_from_numpy(x)) == O.min_element(x)
    d = trtc.device_vector_from_list([1, 2, 3], "int32_t")
    empty = trtc.DVRange(d, 1, 1)
    # the reference fails on empty sorts / scans / compactions and reduces without init
    with pytest.raises(SystemError):
        trtc.Sort(empty)
    with pytest.raises(SystemError):
        trtc.Inclusive_Scan(empty, d)
    with pytest.raises(SystemError):
        trtc.Reduce(empty)
    assert trtc.Reduce(empty, trtc.DVInt32(7)) == 7


def test_scan_float_and_views(trtc):
    rng = np.random.default_rng(4)
    n = 1 << 20
    x = rng.random(n).astype(np.float32)
    d = trtc.device_vector_from_numpy(x)
    o = trtc.device_vector("float", n)
    trtc.Inclusive_Scan(trtc.DVReverse(d), o)
    got = o.to_host().astype(np.float64)
    exp = O.scan_f64(x[::-1].copy())
    assert np.max(np.abs(got - exp) / np.maximum(np.abs(exp), 1e-30)) <= REL_TOL
    s = trtc.Reduce(d)
    assert abs(s - O.reduce_f64(x)) <= REL_TOL * O.reduce_f64(x)


def test_for_and_kernel(trtc):
    v = trtc.device_vector("int32_t", 1000)
    f = trtc.For(["vec"], "idx", "    vec[idx] = (int)idx * 3;\n")
    f.launch_n(1000, [v])
    assert v.to_host().tolist() == [3 * i for i in range(1000)]
    k = trtc.Kernel(["vec", "n"], "    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;\n"
                                   "    if (i < n) vec[i] = vec[i] + 1;\n")
    k.launch(4, 256, [v, trtc.DVUInt32(1000)])
    assert v.to_host().tolist() == [3 * i + 1 for i in range(1000)]


def test_compaction_alignment_and_extremes(trtc):
    # aligned full tiles (16-byte vector path), misaligned sub-ranges (element path), all / none kept
    rng = np.random.default_rng(12)
    n = 3 * 4096 + 1000
    x = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int64).astype(np.int32)
    d = trtc.device_vector_from_numpy(x)
    odd = trtc.Functor({}, ["x"], "        return (x & 1) != 0;\n")
    for off in (0, 1, 3, 4):
        src = trtc.DVRange(d, off, n)
        o = trtc.device_vector("int32_t", n)
        c = trtc.Copy_If(src, o, odd)
        xs = x[off:]
        exp = xs[(xs & 1) != 0]
        assert c == len(exp) and o.to_host(0, c).tolist() == exp.tolist(), off
    allk = trtc.Functor({}, ["x"], "        return true;\n")
    nonek = trtc.Functor({}, ["x"], "        return false;\n")
    o = trtc.device_vector("int32_t", n)
    assert trtc.Copy_If(d, o, allk) == n and o.to_host().tolist() == x.tolist()
    assert trtc.Copy_If(d, o, nonek) == 0
    r = trtc.device_vector("int32_t", n)
    c = trtc.Remove_Copy(d, r, trtc.DVInt32(int(x[5])))
    exp = x[x != x[5]]
    assert c == len(exp) and r.to_host(0, c).tolist() == exp.tolist()


def test_reference_binary_search_program(trtc):
    # python/test/test_binary_search.py inputs; expected values are numpy's searchsorted
    d_input = trtc.device_vector_from_list([0, 2, 5, 7, 8], "int32_t")
    a = np.array([0, 2, 5, 7, 8])
    qs = [0, 1, 2, 3, 8, 9]
    assert [trtc.Lower_Bound(d_input, trtc.DVInt32(q)) for q in qs] == np.searchsorted(a, qs, "left").tolist()
    assert [trtc.Upper_Bound(d_input, trtc.DVInt32(q)) for q in qs] == np.searchsorted(a, qs, "right").tolist()
    assert [trtc.Binary_Search(d_input, trtc.DVInt32(q)) for q in qs] == [q in a for q in qs]
    d_values = trtc.device_vector_from_list(qs, "int32_t")
    d_output = trtc.device_vector("int32_t", 6)
    trtc.Lower_Bound_V(d_input, d_values, d_output)
    assert d_output.to_host().tolist() == [0, 1, 1, 2, 4, 5]
    trtc.Upper_Bound_V(d_input, d_values, d_output)
    assert d_output.to_host().tolist() == [1, 1, 2, 2, 5, 5]
    trtc.Binary_Search_V(d_input, d_values, d_output)
    assert d_output.to_host().tolist() == [1, 0, 1, 0, 1, 0]


def test_vectorised_searches_large_and_comparator(trtc):
    rng = np.random.default_rng(21)
    a = np.sort(rng.integers(0, 10**6, 1 << 20)).astype(np.int64)
    q = rng.integers(-10, 10**6 + 10, 300001).astype(np.int64)
    da, dq = trtc.device_vector_from_numpy(a), trtc.device_vector_from_numpy(q)
    out = trtc.device_vector("uint64_t", len(q))
    trtc.Lower_Bound_V(da, dq, out)
    assert np.array_equal(out.to_host(), np.searchsorted(a, q, "left").astype(np.uint64))
    trtc.Upper_Bound_V(da, dq, out)
    assert np.array_equal(out.to_host(), np.searchsorted(a, q, "right").astype(np.uint64))
    found = trtc.device_vector("bool", len(q))
    trtc.Binary_Search_V(da, dq, found)
    assert np.array_equal(found.to_host().astype(bool), np.isin(q, a))
    # descending order with Greater
    d = a[::-1].copy()
    dd = trtc.device_vector_from_numpy(d)
    trtc.Lower_Bound_V(dd, dq, out, trtc.Greater())
    exp = len(d) - np.searchsorted(a, q, "right")
    assert np.array_equal(out.to_host(), exp.astype(np.uint64))
    assert trtc.Lower_Bound(dd, trtc.DVInt64(int(q[0])), trtc.Greater()) == int(exp[0])


@pytest.mark.parametrize("dtype,tname", [(np.int32, "int32_t"), (np.float32, "float"), (np.uint64, "uint64_t")])
def test_vectorised_searches_sample_edges(trtc, dtype, tname):
    # vectorised searches against numpy's searchsorted / isin: sizes around 2^13 and up to
    # 2^20 + 5, duplicate runs (1, 37 and 5000 equal keys), queries below the first and above
    # the last element, ascending (Less) and descending (Greater) views
    rng = np.random.default_rng(8)
    for n in [8191, 8192, 8193, 100003, (1 << 20) + 5]:
        for run in (1, 37, 5000):
            a = np.sort((np.arange(n) // run * 3 + rng.integers(0, 2, n)).astype(dtype))
            lo, hi = a[0], a[-1]
            q = np.concatenate([a[rng.integers(0, n, 3000)], rng.integers(int(lo) - 5 if lo > 5 else 0,
                                int(hi) + 6, 3000).astype(dtype),
                                np.array([lo, hi], dtype=dtype)])
            if dtype != np.uint64 or lo > 0:
                q = np.concatenate([q, np.array([lo - 1], dtype=dtype)])
            q = q.astype(dtype)
            da, dq = trtc.device_vector_from_numpy(a), trtc.device_vector_from_numpy(q)
            out = trtc.device_vector("uint64_t", len(q))
            trtc.Lower_Bound_V(da, dq, out)
            assert np.array_equal(out.to_host(), np.searchsorted(a, q, "left").astype(np.uint64)), (n, run)
            trtc.Upper_Bound_V(da, dq, out)
            assert np.array_equal(out.to_host(), np.searchsorted(a, q, "right").astype(np.uint64)), (n, run)
            found = trtc.device_vector("bool", len(q))
            trtc.Binary_Search_V(da, dq, found)
            assert np.array_equal(found.to_host().astype(bool), np.isin(q, a)), (n, run)
            d = a[::-1].copy()
            dd = trtc.device_vector_from_numpy(d)
            trtc.Lower_Bound_V(dd, dq, out, trtc.Greater())
            assert np.array_equal(out.to_host(), (n - np.searchsorted(a, q, "right")).astype(np.uint64)), (n, run)
            trtc.Upper_Bound_V(dd, dq, out, trtc.Greater())
            assert np.array_equal(out.to_host(), (n - np.searchsorted(a, q, "left")).astype(np.uint64)), (n, run)


def test_reference_zipped_program(trtc):
    # python/test/test_zipped.py with its outputs checked
    d_int_in = trtc.device_vector_from_list([0, 1, 2, 3, 4], "int32_t")
    d_float_in = trtc.device_vector_from_list([0.0, 10.0, 20.0, 30.0, 40.0], "float")
    d_int_out = trtc.device_vector("int32_t", 5)
    d_float_out = trtc.device_vector("float", 5)
    zipped_in = trtc.DVZipped([d_int_in, d_float_in], ["a", "b"])
    zipped_out = trtc.DVZipped([d_int_out, d_float_out], ["a", "b"])
    trtc.Copy(zipped_in, zipped_out)
    assert d_int_out.to_host().tolist() == [0, 1, 2, 3, 4]
    assert d_float_out.to_host().tolist() == [0.0, 10.0, 20.0, 30.0, 40.0]
    d_int_in = trtc.DVCounter(trtc.DVInt32(0), 5)
    d_float_in = trtc.DVTransform(d_int_in, "float", trtc.Functor({}, ["i"], "        return (float)i*10.0f +10.0f;\n"))
    zipped_in = trtc.DVZipped([d_int_in, d_float_in], ["a", "b"])
    trtc.Copy(zipped_in, zipped_out)
    assert d_int_out.to_host().tolist() == [0, 1, 2, 3, 4]
    assert d_float_out.to_host().tolist() == [10.0, 20.0, 30.0, 40.0, 50.0]
    const_in = trtc.DVConstant(trtc.DVTuple({"a": trtc.DVInt32(123), "b": trtc.DVFloat(456.0)}), 5)
    trtc.Copy(const_in, zipped_out)
    assert d_int_out.to_host().tolist() == [123] * 5
    assert d_float_out.to_host().tolist() == [456.0] * 5


def test_sort_by_key_zipped_payload_and_custom_vector(trtc):
    # k-means demo pattern: Sort_By_Key with a zipped (x, y) payload
    rng = np.random.default_rng(31)
    n = 100_003
    k = rng.integers(0, 97, n).astype(np.int32)
    x = rng.standard_normal(n).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    dk, dx, dy = (trtc.device_vector_from_numpy(a) for a in (k, x, y))
    trtc.Sort_By_Key(dk, trtc.DVZipped([dx, dy], ["x", "y"]))
    p = O.sort_perm(k)
    assert dk.to_host().tolist() == k[p].tolist()
    assert dx.to_host().tobytes() == x[p].tobytes() and dy.to_host().tobytes() == y[p].tobytes()
    # a read-only custom vector feeding a reduction and a scan
    src = trtc.device_vector_from_numpy(np.arange(1000, dtype=np.int32))
    cv = trtc.DVCustomVector({"src": src}, "idx", "        return src[idx] * 2;\n", "int32_t", 1000)
    assert trtc.Reduce(cv) == 2 * sum(range(1000))
    out = trtc.device_vector("int32_t", 1000)
    trtc.Inclusive_Scan(cv, out)
    assert out.to_host().tolist() == np.cumsum(2 * np.arange(1000)).tolist()


def test_cuda_array_interface_vectors(trtc):
    # DVCupyVector / DVNumbaVector adapt any CUDA Array Interface exporter (a torch tensor here)
    import torch
    x = torch.tensor([5, 3, 9, 1, 7], dtype=torch.int32, device="cuda")
    v = trtc.DVCupyVector(x)
    assert v.name_elem_cls() == "int32_t" and v.size() == 5
    trtc.Sort(v)
    torch.cuda.synchronize()
    assert x.cpu().tolist() == [1, 3, 5, 7, 9]
    y = torch.tensor([1.5, -2.0, 0.25], dtype=torch.float64, device="cuda")
    w = trtc.DVNumbaVector(y)
    assert trtc.Reduce(w) == -0.25


def test_inplace_compaction_large(trtc):
    # in-place forms on contiguous vectors go through a pool temporary (two-phase kernel + copy
    # back); a range of a vector takes the same route, a permuted view the one-pass kernel
    rng = np.random.default_rng(41)
    n = (3 << 20) + 11
    x = rng.integers(0, 1000, n).astype(np.int32)
    v = trtc.device_vector_from_numpy(x)
    c = trtc.Remove_If(v, is_even(trtc))
    assert c == int((x % 2 != 0).sum()) and np.array_equal(v.to_host(0, c), x[x % 2 != 0])
    y = np.repeat(rng.integers(0, 50, n // 4), 4)[: n - 100].astype(np.int32)
    w = trtc.device_vector_from_numpy(np.concatenate([np.zeros(100, np.int32), y]))
    c = trtc.Unique(w.range(100, 100 + len(y)), trtc.EqualTo())
    keep = np.concatenate([[True], y[1:] != y[:-1]])
    got = w.to_host(100, 100 + c)
    assert c == int(keep.sum()) and np.array_equal(got, y[keep])
    assert np.array_equal(w.to_host(0, 100), np.zeros(100, np.int32))  # outside the range: untouched
    z = np.arange(20000, dtype=np.int32)
    base = trtc.device_vector_from_numpy(z)
    rev = trtc.DVReverse(base)
    c = trtc.Remove_If(rev, is_even(trtc))  # reversed view: elements 19999, 19997, ... kept in order
    out = base.to_host()
    assert c == 10000 and np.array_equal(out[::-1][:c], z[::-1][z[::-1] % 2 != 0])


def test_vector_storage_reused_and_bounded(trtc):
    # DVVector storage comes from a pool of its own: a destroyed vector's memory serves the
    # next vector without a new mapping, and beyond 8 GiB of cached storage it goes back to
    # the device at the next synchronisation (as cudaFree would have returned it)
    import gc
    import torch
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    big = trtc.device_vector("int8_t", 24 << 30)
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 >= (16 << 30)  # storage cached by earlier tests' vectors may serve a part
    assert trtc.Count(big.range(0, 1 << 20), trtc.DVInt8(0)) == 1 << 20  # zero-filled
    del big
    gc.collect()
    torch.cuda.synchronize()
    free2 = torch.cuda.mem_get_info()[0]
    assert free2 - free1 >= (16 << 30) - (64 << 20)  # all but the 8 GiB cache went back
    assert free0 - free2 <= (8 << 30) + (64 << 20)
    x = np.arange(1 << 20, dtype=np.int32)
    for _ in range(3):  # create / destroy cycles keep their contents right
        v = trtc.device_vector_from_numpy(x)
        assert np.array_equal(v.to_host(), x)
        del v


def test_vector_pool_can_be_switched_off(cuda):
    # TRTC_VECTOR_POOL=0 (read once, at device initialisation) keeps one cudaMalloc per vector
    import subprocess
    import sys
    code = ("import numpy as np, thrustrtc_b200 as t; t.init(); x = np.arange(1000, dtype=np.int32); "
            "v = t.device_vector_from_numpy(x); assert np.array_equal(v.to_host(), x); "
            "t.Sort(v); assert t.Reduce(v) == int(x.sum()); del v; print('ok')")
    env = dict(os.environ, TRTC_VECTOR_POOL="0")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]
