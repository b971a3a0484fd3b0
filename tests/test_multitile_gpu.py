"""Multi-tile parity of the compaction family, the by-key reductions and the transform scans.

Sizes straddle the kernels' tiles (4096 / 5120 / 8192 elements) and reach several thousand
tiles (2^22), so the decoupled look-back carries counts and offsets across tile boundaries:
the two-sided partition scatter (rejected elements at ``index - selected_before``), the
two-array tail compaction of Reduce_By_Key / Unique_By_Key, Copy_If_Stencil and both transform
scans.  Every result is compared byte for byte with the oracle
(partition.cpp:29-125, reduce.cpp:36-62, unique.cpp:37-72, copy.cpp:16-28,
transform_scan.cpp:4-16).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = (4097, 5121, (1 << 20) + 7, 1 << 22)
SELECT = ("none", "half", "all")


@pytest.fixture(scope="module")
def trtc(cuda):
    import thrustrtc_b200 as t
    t.init()
    return t


def _data(n, sel, seed):
    rng = np.random.default_rng(seed)
    x = rng.integers(-(1 << 30), 1 << 30, n).astype(np.int32)
    if sel == "all":
        x &= ~np.int32(1)
    elif sel == "none":
        x |= np.int32(1)
    return x


def _even(trtc):
    return trtc.Functor({}, ["x"], "\n         return x % 2 == 0;\n")


def _runs(n, seed, mean):
    rng = np.random.default_rng(seed)
    lens = rng.geometric(1.0 / mean, n)
    ids = np.repeat(np.arange(len(lens), dtype=np.int64), lens)[:n]
    return (ids * 7 % 1000).astype(np.int32)


def _eq(dev, exp, count=None):
    got = dev.to_host(0, count) if count is not None else dev.to_host()
    if count == 0:
        got = np.zeros(0, dtype=exp.dtype)
    assert got.dtype == exp.dtype and got.shape == exp.shape, (got.shape, exp.shape)
    bad = np.flatnonzero(got != exp)
    assert bad.size == 0, "first mismatch at %d of %d" % (bad[0], len(exp))


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("sel", SELECT)
def test_partition_forms(trtc, n, sel):
    ev = _even(trtc)
    x = _data(n, sel, n + len(sel))
    flags = (x % 2) == 0
    exp, ec = O.partition(x, flags)
    # Partition (in place)
    d = trtc.device_vector_from_numpy(x)
    c = trtc.Partition(d, ev)
    assert c == ec
    _eq(d, exp)
    # Partition_Stencil: the stencil decides, the values move
    st = _data(n, "half", n + 1)
    sf = (st % 2) == 0
    exp_s, ec_s = O.partition(x, sf)
    d = trtc.device_vector_from_numpy(x)
    c = trtc.Partition_Stencil(d, trtc.device_vector_from_numpy(st), ev)
    assert c == ec_s
    _eq(d, exp_s)
    # Partition_Copy and Partition_Copy_Stencil
    t, f = trtc.device_vector("int32_t", n), trtc.device_vector("int32_t", n)
    c = trtc.Partition_Copy(trtc.device_vector_from_numpy(x), t, f, ev)
    assert c == ec
    _eq(t, x[flags], c)
    _eq(f, x[~flags], n - c)
    c = trtc.Partition_Copy_Stencil(trtc.device_vector_from_numpy(x), trtc.device_vector_from_numpy(st), t, f, ev)
    assert c == ec_s
    _eq(t, x[sf], c)
    _eq(f, x[~sf], n - c)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("sel", SELECT)
def test_copy_if_stencil_and_remove_if_stencil(trtc, n, sel):
    ev = _even(trtc)
    x = _data(n, "half", n + 3)
    st = _data(n, sel, n + 4)
    sf = (st % 2) == 0
    out = trtc.device_vector("int32_t", n)
    c = trtc.Copy_If_Stencil(trtc.device_vector_from_numpy(x), trtc.device_vector_from_numpy(st), out, ev)
    assert c == int(sf.sum())
    _eq(out, O.copy_if(x, sf), c)
    d = trtc.device_vector_from_numpy(x)
    c = trtc.Remove_If_Stencil(d, trtc.device_vector_from_numpy(st), ev)
    assert c == int((~sf).sum())
    _eq(d, O.copy_if(x, ~sf), c)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("mean", (1, 6, 300))
def test_reduce_by_key_multi_tile(trtc, n, mean):
    k = _runs(n, n + mean, mean)
    rng = np.random.default_rng(mean)
    v = rng.integers(-1000, 1001, n).astype(np.int32)
    ek, ev = O.reduce_by_key(k, v)
    ko, vo = trtc.device_vector("int32_t", n), trtc.device_vector("int32_t", n)
    c = trtc.Reduce_By_Key(trtc.device_vector_from_numpy(k), trtc.device_vector_from_numpy(v), ko, vo)
    assert c == len(ek)
    _eq(ko, ek, c)
    _eq(vo, ev, c)
    # Maximum under an explicit EqualTo
    ek, ev = O.reduce_by_key(k, v, "Maximum")
    c = trtc.Reduce_By_Key(trtc.device_vector_from_numpy(k), trtc.device_vector_from_numpy(v), ko, vo,
                           trtc.EqualTo(), trtc.Maximum())
    assert c == len(ek)
    _eq(ko, ek, c)
    _eq(vo, ev, c)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("mean", (1, 6, 300))
def test_unique_by_key_multi_tile(trtc, n, mean):
    k = _runs(n, n + 2 * mean, mean)
    v = np.arange(n, dtype=np.int32)[::-1].copy()
    f = O.unique_flags(k)
    ek, ev = k[f], v[f]
    dk, dv = trtc.device_vector_from_numpy(k), trtc.device_vector_from_numpy(v)
    c = trtc.Unique_By_Key(dk, dv)
    assert c == len(ek)
    _eq(dk, ek, c)
    _eq(dv, ev, c)
    ko, vo = trtc.device_vector("int32_t", n), trtc.device_vector("int32_t", n)
    c = trtc.Unique_By_Key_Copy(trtc.device_vector_from_numpy(k), trtc.device_vector_from_numpy(v), ko, vo,
                                trtc.EqualTo())
    assert c == len(ek)
    _eq(ko, ek, c)
    _eq(vo, ev, c)


@pytest.mark.parametrize("n", SIZES)
def test_transform_scans_multi_tile(trtc, n):
    rng = np.random.default_rng(n)
    x = rng.integers(-1000, 1001, n).astype(np.int32)
    neg = (-x.astype(np.int64)).astype(np.int32)
    d = trtc.device_vector_from_numpy(x)
    o = trtc.device_vector("int32_t", n)
    trtc.Transform_Inclusive_Scan(d, o, trtc.Negate(), trtc.Plus())
    _eq(o, O.scan(neg))
    trtc.Transform_Exclusive_Scan(d, o, trtc.Negate(), trtc.DVInt32(3), trtc.Plus())
    _eq(o, O.scan(neg, exclusive=True, init=3))
    trtc.Transform_Inclusive_Scan(d, o, trtc.Negate(), trtc.Maximum())
    _eq(o, O.scan(neg, "Maximum"))
    # a user unary Functor and in place
    sq = trtc.Functor({}, ["x"], "        return x * 3 + 1;\n")
    d2 = trtc.device_vector_from_numpy(x)
    trtc.Transform_Exclusive_Scan(d2, d2, sq, trtc.DVInt32(-7), trtc.Plus())
    _eq(d2, O.scan((x * 3 + 1).astype(np.int32), exclusive=True, init=-7))
