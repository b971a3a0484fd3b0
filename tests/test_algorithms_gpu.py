"""Parity of the remaining reference algorithms (transformations, copying, counting,
searching, extrema, inner product, logical tests, merging) through the package -> C ABI ->
NVRTC kernels of trtc_misc.cuh.  The small cases are the reference's own python/test
programs with their printed values asserted (Thrust semantics, worked by hand); the large
ones are seeded random inputs checked against the oracle.  Integer and index results are
bit-exact; the float64 inner product is within REL_TOL of the oracle's sum."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL_TOL = 1e-12


@pytest.fixture(scope="module")
def trtc(cuda):
    import thrustrtc_b200 as t
    t.init()
    return t


def F(trtc, params, body):
    return trtc.Functor({}, params, "\n         " + body + "\n")


def host(v):
    return v.to_host().tolist()


# ---------------------------------------------------------------- python/test programs
def test_fill_sequence_tabulate(trtc):
    d = trtc.device_vector("int32_t", 5)
    trtc.Fill(d, trtc.DVInt32(123))
    assert host(d) == [123] * 5
    trtc.Fill(d.range(1, 3), trtc.DVInt32(456))
    assert host(d) == [123, 456, 456, 123, 123]
    d = trtc.device_vector("int32_t", 10)
    trtc.Sequence(d)
    assert host(d) == list(range(10))
    trtc.Sequence(d, trtc.DVInt32(1))
    assert host(d) == list(range(1, 11))
    trtc.Sequence(d, trtc.DVInt32(1), trtc.DVInt32(3))
    assert host(d) == [1 + 3 * i for i in range(10)]
    trtc.Sequence(d)
    trtc.Tabulate(d, trtc.Negate())
    assert host(d) == [-i for i in range(10)]
    f = trtc.device_vector("float", 7)
    trtc.Sequence(f, trtc.DVFloat(0.25), trtc.DVFloat(0.5))
    assert host(f) == [0.25 + 0.5 * i for i in range(7)]


def test_replace(trtc):
    neg = F(trtc, ["x"], "return x<0;")
    d = trtc.device_vector_from_list([1, 2, 3, 1, 2], "int32_t")
    trtc.Replace(d, trtc.DVInt32(1), trtc.DVInt32(99))
    assert host(d) == [99, 2, 3, 99, 2]
    d = trtc.device_vector_from_list([1, -2, 3, -4, 5], "int32_t")
    trtc.Replace_If(d, neg, trtc.DVInt32(0))
    assert host(d) == [1, 0, 3, 0, 5]
    i = trtc.device_vector_from_list([1, 2, 3, 1, 2], "int32_t")
    o = trtc.device_vector("int32_t", 5)
    trtc.Replace_Copy(i, o, trtc.DVInt32(1), trtc.DVInt32(99))
    assert host(o) == [99, 2, 3, 99, 2] and host(i) == [1, 2, 3, 1, 2]
    i = trtc.device_vector_from_list([1, -2, 3, -4, 5], "int32_t")
    trtc.Replace_Copy_If(i, o, neg, trtc.DVInt32(0))
    assert host(o) == [1, 0, 3, 0, 5]
    # old/new values converted to the element type first (replace.cpp:7)
    f = trtc.device_vector_from_list([1.0, 2.5, 1.0], "float")
    trtc.Replace(f, trtc.DVDouble(1.0), trtc.DVInt32(7))
    assert host(f) == [7.0, 2.5, 7.0]


def test_for_each(trtc):
    d = trtc.device_vector_from_list([1, 2, 3, 1, 2], "int32_t")
    cnt = trtc.device_vector_from_list([0], "int32_t")
    f = trtc.Functor({"cnt": cnt}, ["x"], "\n         atomicAdd(&cnt[0], x);\n")
    trtc.For_Each(d, f)
    assert host(cnt) == [9]


def test_adjacent_difference(trtc):
    i = trtc.device_vector_from_list([1, 2, 1, 2, 1, 2, 1, 2], "int32_t")
    o = trtc.device_vector("int32_t", 8)
    trtc.Adjacent_Difference(i, o)
    assert host(o) == [1, 1, -1, 1, -1, 1, -1, 1]
    trtc.Adjacent_Difference(i, o, trtc.Plus())
    assert host(o) == [1, 3, 3, 3, 3, 3, 3, 3]
    # in place, over many CTAs: reads come from a copy of the input
    x = np.random.default_rng(5).integers(-1000, 1000, 1 << 20).astype(np.int32)
    d = trtc.device_vector_from_numpy(x)
    trtc.Adjacent_Difference(d, d)
    assert np.array_equal(d.to_host(), O.adjacent_difference(x))


def test_transform(trtc):
    is_odd = F(trtc, ["x"], "return x % 2;")
    d = trtc.device_vector_from_list([-5, 0, 2, -3, 2, 4, 0, -1, 2, 8], "int32_t")
    trtc.Transform(d, d, trtc.Negate())
    assert host(d) == [5, 0, -2, 3, -2, -4, 0, 1, -2, -8]
    a = trtc.device_vector_from_list([-5, 0, 2, 3, 2, 4], "int32_t")
    b = trtc.device_vector_from_list([3, 6, -2, 1, 2, 3], "int32_t")
    o = trtc.device_vector("int32_t", 6)
    trtc.Transform_Binary(a, b, o, trtc.Plus())
    assert host(o) == [-2, 6, 0, 4, 4, 7]
    d = trtc.device_vector_from_list([-5, 0, 2, -3, 2, 4, 0, -1, 2, 8], "int32_t")
    trtc.Transform_If(d, d, trtc.Negate(), is_odd)
    assert host(d) == [5, 0, 2, 3, 2, 4, 0, 1, 2, 8]
    d = trtc.device_vector_from_list([-5, 0, 2, -3, 2, 4, 0, -1, 2, 8], "int32_t")
    st = trtc.device_vector_from_list([1, 0, 1, 0, 1, 0, 1, 0, 1, 0], "int32_t")
    trtc.Transform_If_Stencil(d, st, d, trtc.Negate(), trtc.Identity())
    assert host(d) == [5, 0, -2, -3, -2, 4, 0, -1, -2, 8]
    st = trtc.device_vector_from_list([1, 0, 1, 0, 1, 0], "int32_t")
    o = trtc.device_vector_from_list([-1] * 6, "int32_t")
    trtc.Transform_Binary_If_Stencil(a, b, st, o, trtc.Plus(), trtc.Identity())
    assert host(o) == [-2, -1, 0, -1, 4, -1]
    # computed input view -> range output
    o = trtc.device_vector_from_list([0] * 8, "int32_t")
    trtc.Transform(trtc.DVCounter(trtc.DVInt32(10), 4), o.range(2, 6), trtc.Negate())
    assert host(o) == [0, 0, -10, -11, -12, -13, 0, 0]


def test_gather_scatter_swap(trtc):
    even = F(trtc, ["x"], "return ((x % 2) == 0);")
    v = trtc.device_vector_from_list([1, 0, 1, 0, 1, 0, 1, 0, 1, 0], "int32_t")
    m = trtc.device_vector_from_list([0, 2, 4, 6, 8, 1, 3, 5, 7, 9], "int32_t")
    o = trtc.device_vector("int32_t", 10)
    trtc.Gather(m, v, o)
    assert host(o) == [1, 1, 1, 1, 1, 0, 0, 0, 0, 0]
    v = trtc.device_vector_from_list(list(range(10)), "int32_t")
    st = trtc.device_vector_from_list([1, 0, 1, 0, 1, 0, 1, 0, 1, 0], "int32_t")
    o = trtc.device_vector_from_list([7] * 10, "int32_t")
    trtc.Gather_If(m, st, v, o)
    assert host(o) == [0, 7, 4, 7, 8, 7, 3, 7, 7, 7]
    st = trtc.device_vector_from_list([0, 3, 4, 1, 4, 1, 2, 7, 8, 9], "int32_t")
    o = trtc.device_vector_from_list([7] * 10, "int32_t")
    trtc.Gather_If(m, st, v, o, even)
    assert host(o) == [0, 7, 4, 7, 8, 7, 3, 7, 7, 7]
    v = trtc.device_vector_from_list([1, 0, 1, 0, 1, 0, 1, 0, 1, 0], "int32_t")
    m = trtc.device_vector_from_list([0, 5, 1, 6, 2, 7, 3, 8, 4, 9], "int32_t")
    o = trtc.device_vector("int32_t", 10)
    trtc.Scatter(v, m, o)
    assert host(o) == [1, 1, 1, 1, 1, 0, 0, 0, 0, 0]
    V = trtc.device_vector_from_list([10, 20, 30, 40, 50, 60, 70, 80], "int32_t")
    M = trtc.device_vector_from_list([0, 5, 1, 6, 2, 7, 3, 4], "int32_t")
    S = trtc.device_vector_from_list([1, 0, 1, 0, 1, 0, 1, 0], "int32_t")
    D = trtc.device_vector_from_list([0] * 8, "int32_t")
    trtc.Scatter_If(V, M, S, D)
    assert host(D) == [10, 30, 50, 70, 0, 0, 0, 0]
    S = trtc.device_vector_from_list([2, 1, 2, 1, 2, 1, 2, 1], "int32_t")
    D = trtc.device_vector_from_list([0] * 8, "int32_t")
    trtc.Scatter_If(V, M, S, D, even)
    assert host(D) == [10, 30, 50, 70, 0, 0, 0, 0]
    a = trtc.device_vector_from_list([10, 20, 30, 40, 50, 60, 70, 80], "int32_t")
    b = trtc.device_vector_from_list([1000, 900, 800, 700, 600, 500, 400, 300], "int32_t")
    trtc.Swap(a, b)
    assert host(a) == [1000, 900, 800, 700, 600, 500, 400, 300]
    assert host(b) == [10, 20, 30, 40, 50, 60, 70, 80]
    # a random permutation, both directions
    rng = np.random.default_rng(6)
    n = 3 << 20
    x = rng.standard_normal(n).astype(np.float32)
    p = rng.permutation(n).astype(np.int32)
    dx, dp, do = trtc.device_vector_from_numpy(x), trtc.device_vector_from_numpy(p), trtc.device_vector("float", n)
    trtc.Gather(dp, dx, do)
    assert np.array_equal(do.to_host(), x[p])
    trtc.Scatter(dx, dp, do)
    exp = np.empty_like(x)
    exp[p] = x
    assert np.array_equal(do.to_host(), exp)


def test_count(trtc):
    d = trtc.device_vector("int32_t", 2000)
    trtc.Transform(trtc.DVCounter(trtc.DVInt32(0), 2000), d, F(trtc, ["x"], "return x % 100;"))
    assert trtc.Count(d, trtc.DVInt32(47)) == 20
    trtc.Sequence(d)
    assert trtc.Count_If(d, F(trtc, ["x"], "return (x % 100)==47;")) == 20
    rng = np.random.default_rng(7)
    x = rng.integers(0, 7, (5 << 20) + 3).astype(np.int64)
    dx = trtc.device_vector_from_numpy(x)
    assert trtc.Count(dx, trtc.DVInt64(3)) == int((x == 3).sum())
    assert trtc.Count_If(dx, F(trtc, ["x"], "return x > 4;")) == int((x > 4).sum())
    # the value converts to the element type first (count.cpp:6): 3.7 counts the 3s
    assert trtc.Count(dx, trtc.DVDouble(3.7)) == int((x == 3).sum())
    assert trtc.Count(d.range(0, 0), trtc.DVInt32(0)) == 0


def test_find_mismatch(trtc):
    d = trtc.device_vector_from_list([0, 5, 3, 7], "int32_t")
    assert trtc.Find(d, trtc.DVInt32(3)) == 2
    assert trtc.Find(d, trtc.DVInt32(5)) == 1
    assert trtc.Find(d, trtc.DVInt32(9)) is None
    assert trtc.Find_If(d, F(trtc, ["x"], "return x>4;")) == 1
    assert trtc.Find_If(d, F(trtc, ["x"], "return x>10;")) is None
    assert trtc.Find_If_Not(d, F(trtc, ["x"], "return x>4;")) == 0
    assert trtc.Find_If_Not(d, F(trtc, ["x"], "return x>10;")) == 0
    # no conversion of the value in find.cpp:6: 3.5 matches nothing in an int vector
    assert trtc.Find(d, trtc.DVDouble(3.5)) is None
    d1 = trtc.device_vector_from_list([0, 5, 3, 7], "int32_t")
    d2 = trtc.device_vector_from_list([0, 5, 8, 7], "int32_t")
    assert trtc.Mismatch(d1, d2) == 2
    assert trtc.Mismatch(d1, d2, trtc.EqualTo()) == 2
    assert trtc.Mismatch(d1, d1) is None
    # large: first hit far into the range, several hits (the smallest wins), none
    n = (7 << 20) + 5
    x = np.zeros(n, np.int32)
    for pos in (n - 1, 4 << 20, 12345):
        x[pos] = 9
        assert trtc.Find(trtc.device_vector_from_numpy(x), trtc.DVInt32(9)) == pos
    y = x.copy()
    y[(5 << 20) + 77] = 1
    y[(6 << 20)] = 2
    assert trtc.Mismatch(trtc.device_vector_from_numpy(x), trtc.device_vector_from_numpy(y)) == (5 << 20) + 77
    assert trtc.Find(d.range(0, 0), trtc.DVInt32(0)) is None


def test_equal_logical(trtc):
    m2 = trtc.Functor({}, ["x", "y"], "\n         return (x % 2) == (y % 2);\n")
    a = trtc.device_vector_from_list([3, 1, 4, 1, 5, 9, 3], "int32_t")
    b = trtc.device_vector_from_list([3, 1, 4, 2, 8, 5, 7], "int32_t")
    c = trtc.device_vector_from_list([3, 1, 4, 1, 5, 9, 3], "int32_t")
    assert trtc.Equal(a, b) is False and trtc.Equal(a, c) is True
    dx = trtc.device_vector_from_list([1, 2, 3, 4, 5, 6], "int32_t")
    dy = trtc.device_vector_from_list([7, 8, 9, 10, 11, 12], "int32_t")
    assert trtc.Equal(dx, dy, m2) is True
    ident = trtc.Identity()
    d = trtc.device_vector_from_list([True, True, False], "bool")
    assert [trtc.All_Of(d.range(0, 2), ident), trtc.All_Of(d.range(0, 3), ident),
            trtc.All_Of(d.range(0, 0), ident)] == [True, False, False]
    assert [trtc.Any_Of(d.range(0, 2), ident), trtc.Any_Of(d.range(0, 3), ident), trtc.Any_Of(d.range(2, 3), ident),
            trtc.Any_Of(d.range(0, 0), ident)] == [True, True, False, False]
    assert [trtc.None_Of(d.range(0, 2), ident), trtc.None_Of(d.range(0, 3), ident),
            trtc.None_Of(d.range(2, 3), ident), trtc.None_Of(d.range(0, 0), ident)] == [False, False, True, True]


def test_extrema(trtc):
    d = trtc.device_vector_from_list([1, 0, 2, 2, 1, 3], "int32_t")
    assert trtc.Min_Element(d) == 1 and trtc.Max_Element(d) == 5
    assert tuple(int(i) for i in trtc.MinMax_Element(d)) == (1, 5)
    rng = np.random.default_rng(8)
    for n in (1, 257, 65536 + 300, (3 << 20) + 1):
        x = rng.integers(0, 100, n).astype(np.float32)
        x[rng.integers(0, n, max(1, n // 100))] = np.nan  # NaN makes the tree order visible
        dx = trtc.device_vector_from_numpy(x)
        assert trtc.Max_Element(dx) == O.index_tree(x, maximum=True)
        assert trtc.Min_Element(dx, trtc.Less()) == O.index_tree(x)
        assert trtc.Max_Element(dx, trtc.Greater()) == O.index_tree(x, maximum=True, less=lambda a, b: a > b)
        lo, hi = trtc.MinMax_Element(dx, trtc.Greater())
        assert (int(lo), int(hi)) == (O.index_tree(x, less=lambda a, b: a > b),
                                      O.index_tree(x, maximum=True, less=lambda a, b: a > b))


def test_inner_product(trtc):
    a = trtc.device_vector_from_list([1.0, 2.0, 5.0], "float")
    b = trtc.device_vector_from_list([4.0, 1.0, 5.0], "float")
    assert trtc.Inner_Product(a, b, trtc.DVFloat(0.0)) == 31.0
    assert trtc.Inner_Product(a, b, trtc.DVFloat(0.0), trtc.Plus(), trtc.Multiplies()) == 31.0
    # mixed element types with the default product; int accumulation is exact
    i = trtc.device_vector_from_list([1, 2, 3], "int32_t")
    assert trtc.Inner_Product(i, a, trtc.DVDouble(0.5)) == 0.5 + 1.0 + 4.0 + 15.0
    rng = np.random.default_rng(9)
    x, y = rng.standard_normal(3 << 20), rng.standard_normal(3 << 20)
    got = trtc.Inner_Product(trtc.device_vector_from_numpy(x), trtc.device_vector_from_numpy(y), trtc.DVDouble(1.0))
    exact = 1.0 + float(np.dot(x, y))
    assert abs(got - exact) <= REL_TOL * (1.0 + float(np.abs(x * y).sum()))
    p = rng.integers(-50, 50, 1 << 20).astype(np.int64)
    q = rng.integers(-50, 50, 1 << 20).astype(np.int64)
    assert trtc.Inner_Product(trtc.device_vector_from_numpy(p), trtc.device_vector_from_numpy(q),
                              trtc.DVInt64(7)) == 7 + int(np.dot(p, q))
    assert trtc.Inner_Product(a.range(0, 0), b, trtc.DVFloat(2.5)) == 2.5


def test_sorted_partitioned(trtc):
    even = F(trtc, ["x"], "return ((x % 2) == 0);")
    d = trtc.device_vector_from_list([2, 4, 6, 8, 10, 1, 3, 5, 7, 9], "int32_t")
    assert trtc.Partition_Point(d, even) == 5
    assert trtc.Is_Partitioned(d, even) is True
    assert trtc.Is_Partitioned(trtc.device_vector_from_list(list(range(1, 11)), "int32_t"), even) is False
    d = trtc.device_vector_from_list([1, 4, 2, 8, 5, 7], "int32_t")
    assert trtc.Is_Sorted(d) is False
    trtc.Sort(d)
    assert trtc.Is_Sorted(d) is True
    d = trtc.device_vector_from_list([1, 4, 2, 8, 5, 7], "int32_t")
    assert trtc.Is_Sorted(d, trtc.Greater()) is False
    trtc.Sort(d, trtc.Greater())
    assert trtc.Is_Sorted(d, trtc.Greater()) is True
    assert trtc.Is_Sorted_Until(trtc.device_vector_from_list([0, 1, 2, 3, 0, 1, 2, 3], "int32_t")) == 4
    assert trtc.Is_Sorted_Until(trtc.device_vector_from_list([3, 2, 1, 0, 3, 2, 1, 0], "int32_t"),
                                trtc.Greater()) == 4
    empty = d.range(0, 0)
    assert trtc.Is_Sorted(empty) is True and trtc.Is_Sorted(d.range(0, 1)) is True
    assert trtc.Is_Sorted_Until(empty) == 0 and trtc.Is_Sorted_Until(d.range(0, 1)) == 1
    assert trtc.Is_Partitioned(empty, even) is True
    with pytest.raises(SystemError):
        trtc.Partition_Point(empty, even)
    # large: a sorted run broken deep inside, a long partitioned range
    n = (6 << 20) + 11
    x = np.sort(np.random.default_rng(10).integers(0, 1 << 30, n)).astype(np.int32)
    assert trtc.Is_Sorted_Until(trtc.device_vector_from_numpy(x)) == n
    x[(5 << 20) + 3] = -1
    dx = trtc.device_vector_from_numpy(x)
    assert trtc.Is_Sorted_Until(dx) == O.is_sorted_until(x) == (5 << 20) + 3
    assert trtc.Is_Sorted(dx) is False
    f = np.concatenate([np.zeros(4 << 20, np.int32), np.ones(n - (4 << 20), np.int32)])
    df = trtc.device_vector_from_numpy(f)
    assert trtc.Partition_Point(df, even) == 4 << 20
    assert trtc.Is_Partitioned(df, even) is True
    f[n - 2] = 0
    assert trtc.Is_Partitioned(trtc.device_vector_from_numpy(f), even) is O.is_partitioned(f % 2 == 0) is False


def test_merge(trtc):
    a = trtc.device_vector_from_list([1, 3, 5, 7, 9, 11], "int32_t")
    b = trtc.device_vector_from_list([1, 1, 2, 3, 5, 8, 13], "int32_t")
    o = trtc.device_vector("int32_t", 13)
    trtc.Merge(a, b, o)
    assert host(o) == [1, 1, 1, 2, 3, 3, 5, 5, 7, 8, 9, 11, 13]
    a = trtc.device_vector_from_list([11, 9, 7, 5, 3, 1], "int32_t")
    b = trtc.device_vector_from_list([13, 8, 5, 3, 2, 1, 1], "int32_t")
    trtc.Merge(a, b, o, trtc.Greater())
    assert host(o) == [13, 11, 9, 8, 7, 5, 5, 3, 3, 2, 1, 1, 1]
    k1 = trtc.device_vector_from_list([1, 3, 5, 7, 9, 11], "int32_t")
    v1 = trtc.device_vector_from_list([0] * 6, "int32_t")
    k2 = trtc.device_vector_from_list([1, 1, 2, 3, 5, 8, 13], "int32_t")
    v2 = trtc.device_vector_from_list([1] * 7, "int32_t")
    ko, vo = trtc.device_vector("int32_t", 13), trtc.device_vector("int32_t", 13)
    trtc.Merge_By_Key(k1, k2, v1, v2, ko, vo)
    assert host(ko) == [1, 1, 1, 2, 3, 3, 5, 5, 7, 8, 9, 11, 13]
    assert host(vo) == [0, 1, 1, 1, 0, 1, 0, 1, 0, 1, 0, 0, 1]
    k1 = trtc.device_vector_from_list([11, 9, 7, 5, 3, 1], "int32_t")
    k2 = trtc.device_vector_from_list([13, 8, 5, 3, 2, 1, 1], "int32_t")
    trtc.Merge_By_Key(k1, k2, v1, v2, ko, vo, trtc.Greater())
    assert host(ko) == [13, 11, 9, 8, 7, 5, 5, 3, 3, 2, 1, 1, 1]
    assert host(vo) == [1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 1, 1]
    # large, many duplicates, unequal lengths, and one empty side
    rng = np.random.default_rng(12)
    def dv(arr):  # empty inputs are empty ranges: the API refuses 0-size vectors
        return trtc.device_vector_from_numpy(arr) if len(arr) else trtc.device_vector("int32_t", 1).range(0, 0)

    for na, nb in ((3 << 20, (1 << 20) + 17), (0, 1000), (999, 0)):
        x = np.sort(rng.integers(0, 5000, na)).astype(np.int32)
        y = np.sort(rng.integers(0, 5000, nb)).astype(np.int32)
        vx = np.arange(na, dtype=np.int32)
        vy = -1 - np.arange(nb, dtype=np.int32)
        ek, ev = O.merge(x, y, vx, vy)
        ko, vo = trtc.device_vector("int32_t", na + nb), trtc.device_vector("int32_t", na + nb)
        trtc.Merge_By_Key(dv(x), dv(y), dv(vx), dv(vy), ko, vo)
        assert np.array_equal(ko.to_host(), ek) and np.array_equal(vo.to_host(), ev)


def test_fake_vector_programs(trtc):
    # python/test/test_constant.py, test_counter.py, test_discard.py, test_permutation.py,
    # test_range.py, test_reverse.py, test_transform_iter.py with their printed values asserted
    d = trtc.device_vector_from_list([3, 7, 2, 5], "int32_t")
    trtc.Transform_Binary(d, trtc.DVConstant(trtc.DVInt32(10)), d, trtc.Plus())
    assert host(d) == [13, 17, 12, 15]
    d = trtc.device_vector("int32_t", 10)
    trtc.Transform(trtc.DVCounter(trtc.DVInt32(5), 10), d, trtc.Negate())
    assert host(d) == [-5 - i for i in range(10)]
    trtc.Transform(trtc.DVCounter(trtc.DVInt32(5), 10), trtc.DVDiscard("int32_t"), trtc.Negate())  # no effect, no error
    vals = trtc.device_vector_from_list([10.0, 20.0, 30.0, 40.0, 50.0, 60.0, 70.0, 80.0], "float")
    idx = trtc.device_vector_from_list([2, 6, 1, 3], "int32_t")
    out = trtc.device_vector("float", 4)
    trtc.Transform(trtc.DVPermutation(vals, idx), out, trtc.Negate())
    assert host(out) == [-30.0, -70.0, -20.0, -40.0]
    din = trtc.device_vector_from_list([10, 20, 30, 40, 50, 60, 70, 80], "int32_t")
    dout = trtc.device_vector("int32_t", 4)
    trtc.Copy(din.range(2, 6), dout)
    assert host(dout) == [30, 40, 50, 60]
    din = trtc.device_vector_from_list([3, 7, 2, 5], "int32_t")
    trtc.Transform(trtc.DVReverse(din), dout, trtc.Negate())
    assert host(dout) == [-5, -2, -7, -3]
    sq = trtc.Functor({}, ["x"], "\n         return sqrtf(x);\n")
    f = trtc.device_vector_from_list([1.0, 4.0, 9.0, 16.0], "float")
    fo = trtc.device_vector("float", 4)
    trtc.Transform(trtc.DVTransform(f, "float", sq), fo, trtc.Negate())
    assert host(fo) == [-1.0, -2.0, -3.0, -4.0]


def test_multithread_program(trtc):
    # python/test/test_multithread.py: one For kernel launched from three host threads at once
    import threading
    darr = trtc.device_vector_from_numpy(np.array([1.0, 2.0, 3.0, 4.0, 5.0], dtype=np.float32))
    loop = trtc.For(["arr_in", "arr_out", "k"], "idx", "\n\tarr_out[idx] = arr_in[idx]*k;\n\t")
    results, errors = [], []

    def work():
        try:
            o = trtc.device_vector("float", 5)
            loop.launch_n(5, [darr, o, trtc.DVFloat(10.0)])
            results.append(o.to_host().tolist())
        except Exception as e:  # reported below
            errors.append(e)

    ts = [threading.Thread(target=work) for _ in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors and results == [[10.0, 20.0, 30.0, 40.0, 50.0]] * 3


def test_fft_program_fill(trtc):
    # python/test/test_fft.py: Fill of a complex64 device array adapted through the CUDA Array
    # Interface, then a library FFT of it (torch here in place of CuPy)
    import torch
    arr = torch.empty(4, dtype=torch.complex64, device="cuda")
    trtc.Fill(trtc.DVCupyVector(arr), trtc.DVComplex64(complex(1.0, 2.0)))
    torch.cuda.synchronize()
    assert arr.cpu().tolist() == [complex(1.0, 2.0)] * 4
    assert torch.fft.fft(arr).cpu().tolist() == [complex(4.0, 8.0), 0j, 0j, 0j]


def test_kernel_program_two_types(trtc):
    # python/test/test_trtc.py: one Kernel launched with float and with int32 arguments
    harr = np.array([1.0, 2.0, 3.0, 4.0, 5.0], dtype=np.float32)
    darr = trtc.device_vector_from_numpy(harr)
    assert darr.name_view_cls() == "VectorView<float>"
    darr2 = trtc.device_vector_from_numpy(np.array([6, 7, 8, 9, 10], dtype=np.int32))
    kernel = trtc.Kernel(["arr_in", "arr_out", "k"], """
    size_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= arr_in.size()) return;
    arr_out[idx] = arr_in[idx]*k;
    """)
    out = trtc.device_vector("float", 5)
    kernel.launch(1, 128, [darr, out, trtc.DVFloat(10.0)])
    assert host(out) == [10.0, 20.0, 30.0, 40.0, 50.0]
    out = trtc.device_vector("int32_t", 5)
    kernel.launch(1, 128, [darr2, out, trtc.DVInt32(5)])
    assert host(out) == [30, 35, 40, 45, 50]


def test_custom_vector_reduce_by_key_program(trtc):
    # python/test/test_custom_vector.py: keys and values computed on the fly, keys discarded
    darr = trtc.device_vector("int32_t", 2000)
    trtc.Sequence(darr)
    vals = trtc.DVCustomVector({"src": darr}, "idx", """
    unsigned group = idx / src.size();
    unsigned sub_idx = idx % src.size();
    return src[sub_idx] % (group+1) ==0 ? 1: 0;
""", "uint32_t", 20000)
    keys = trtc.DVCustomVector({"src": darr}, "idx", "\n\treturn idx / src.size();\n", "uint32_t", 20000)
    out = trtc.device_vector("uint32_t", 10)
    c = trtc.Reduce_By_Key(keys, vals, trtc.DVDiscard("uint32_t", 10), out)
    assert c == 10
    assert host(out) == [sum(1 for x in range(2000) if x % (g + 1) == 0) for g in range(10)]
