"""Parity of the CUDA kernels (raw-pointer C ABI, include/trtc_raw.h) against the CPU oracle.

Integer / index / permutation results must be bit-exact; float sums and scans are compared
with the FP64 oracle at a relative tolerance of 1e-5 (the north-star FP32 bound).
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# tile edges of the sort (256 x 8 keys for 4-byte keys up to 2^18 keys, 256 x 20 beyond; 256 x 12
# for 8-byte keys), the switch between the two 4-byte tile sizes, and the scans (4096)
SIZES = [1, 2, 3, 255, 256, 257, 511, 512, 513, 2047, 2048, 2049, 3071, 3072, 3073, 4095, 4096, 4097, 5119, 5120,
         5121, 6145, 10241, 65537, 1 << 18, (1 << 18) + 1, 1 << 20 | 7]
NP_OF = {"int8_t": np.int8, "uint8_t": np.uint8, "int16_t": np.int16, "uint16_t": np.uint16,
         "int32_t": np.int32, "uint32_t": np.uint32, "int64_t": np.int64, "uint64_t": np.uint64,
         "float": np.float32, "double": np.float64}
REL_TOL = 1e-5


@pytest.fixture(scope="module")
def N(cuda):
    from thrustrtc_b200 import _native
    return _native


def dev(a):
    import torch
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a.view(np.uint8).copy()).cuda()
    return t


def host(t, dtype):
    return t.cpu().numpy().view(dtype)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def rand_keys(rng, name, n):
    dt = NP_OF[name]
    if name in ("float", "double"):
        x = rng.standard_normal(n).astype(dt)
        if n > 8:
            x[rng.integers(0, n, max(1, n // 50))] = -0.0
            x[rng.integers(0, n, max(1, n // 50))] = 0.0
            x[rng.integers(0, n, max(1, n // 10))] = x[rng.integers(0, n, max(1, n // 10))]
        return x
    info = np.iinfo(dt)
    return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)


@pytest.mark.parametrize("name", list(NP_OF))
@pytest.mark.parametrize("desc", [False, True])
def test_sort_keys(N, name, desc):
    rng = np.random.default_rng(1234)
    for n in SIZES:
        x = rand_keys(rng, name, n)
        d = dev(x)
        rc = N.lib.trtc_raw_sort(N.TYPE_CODES[name], ptr(d), n, int(desc), None)
        assert rc == 0, N.last_error()
        assert N.lib.trtc_raw_sync(None) == 0, N.last_error()
        got = host(d, NP_OF[name])
        exp = O.sort(x, desc)
        assert got.view(np.uint8).tobytes() == exp.view(np.uint8).tobytes(), (name, n, desc)


@pytest.mark.parametrize("name", ["uint32_t", "int32_t", "float", "int64_t", "double", "uint16_t"])
@pytest.mark.parametrize("vsize", [4, 8, 1, 12])
def test_sort_by_key(N, name, vsize):
    rng = np.random.default_rng(99)
    for n in [1, 5, 4097, 5121, 100003, 1 << 20]:
        k = rand_keys(rng, name, n)
        if vsize in (4, 8):
            v = np.arange(n, dtype=np.uint32 if vsize == 4 else np.uint64)
        else:
            v = rng.integers(0, 255, (n, vsize), dtype=np.uint8)
        dk, dv = dev(k), dev(v)
        for desc in (False, True):
            dk, dv = dev(k), dev(v)
            rc = N.lib.trtc_raw_sort_by_key(N.TYPE_CODES[name], ptr(dk), ptr(dv), vsize, n, int(desc), None)
            assert rc == 0, N.last_error()
            assert N.lib.trtc_raw_sync(None) == 0
            p = O.sort_perm(k, desc)
            assert host(dk, NP_OF[name]).tobytes() == k[p].tobytes()
            gv = host(dv, v.dtype).reshape(v.shape)
            assert gv.tobytes() == v[p].tobytes(), (name, n, vsize, desc)


@pytest.mark.parametrize("name", ["uint32_t", "float", "int64_t"])
@pytest.mark.parametrize("off", [0, 1, 2, 3])
def test_sort_by_key_payload_offsets(N, name, off):
    # 4-byte payloads of full tiles arrive by one bulk copy when the tile's payload address
    # is 16-byte aligned, else by per-element copies; payload views at element offsets 0..3
    # take both paths, and n leaves a partial last tile (per-element path) behind full ones
    rng = np.random.default_rng(31 + off)
    n = (1 << 20) + 4099
    k = rand_keys(rng, name, n)
    v = rng.integers(0, 2**32, n, dtype=np.uint32)
    dk = dev(k)
    vbuf = dev(np.concatenate([np.zeros(off, np.uint32), v]))
    vp = ctypes.c_void_p(vbuf.data_ptr() + 4 * off)
    rc = N.lib.trtc_raw_sort_by_key(N.TYPE_CODES[name], ptr(dk), vp, 4, n, 0, None)
    assert rc == 0, N.last_error()
    assert N.lib.trtc_raw_sync(None) == 0
    p = O.sort_perm(k, False)
    assert host(dk, NP_OF[name]).tobytes() == k[p].tobytes()
    gv = host(vbuf, np.uint32)
    assert gv[off:].tobytes() == v[p].tobytes(), (name, off)
    assert not gv[:off].any()  # the words before the view are untouched


def test_sort_float_nan_rotation(N):
    # NaN in a left slot of the Min_Element tree: the reference output is a rotation
    rng = np.random.default_rng(5)
    cases = [np.array([5, np.nan, 3, 0], np.float32)]
    for n in [300, 4097, 70000, 1 << 20]:
        x = rng.standard_normal(n).astype(np.float32)
        x[rng.integers(0, n, max(1, n // 100))] = np.nan
        x[rng.integers(0, n, max(1, n // 100))] = -0.0
        neg = np.array([0xFFC00000], dtype=np.uint32).view(np.float32)[0]
        x[rng.integers(0, n, 3)] = neg
        cases.append(x.copy())
        x[0] = np.nan
        cases.append(x.copy())
        y = x.astype(np.float64)
        cases.append(y)
    for x in cases:
        for desc in (False, True):
            d = dev(x)
            name = "float" if x.dtype == np.float32 else "double"
            assert N.lib.trtc_raw_sort(N.TYPE_CODES[name], ptr(d), len(x), int(desc), None) == 0
            assert N.lib.trtc_raw_sync(None) == 0
            assert host(d, x.dtype).tobytes() == O.sort(x, desc).tobytes(), (len(x), desc)


def test_sort_digit_skipping(N):
    # Zipf-like int64 keys with constant high bits (only 3 live digits) and odd pass counts
    rng = np.random.default_rng(7)
    n = 300001
    r = np.minimum(rng.zipf(1.1, n), 1 << 20) - 1
    k = (0x0123456700000000 + ((r * 0x9E3B1) % (1 << 20))).astype(np.int64)
    v = np.arange(n, dtype=np.int32)
    for keys in (k, k[:1000], (k & 0xFF) + 5, np.full(n, 42, np.int64), (k & 0xFFFF)):
        dk, dv = dev(keys), dev(v[: len(keys)])
        assert N.lib.trtc_raw_sort_by_key(6, ptr(dk), ptr(dv), 4, len(keys), 0, None) == 0
        assert N.lib.trtc_raw_sync(None) == 0
        p = O.sort_perm(keys)
        assert host(dk, np.int64).tobytes() == keys[p].tobytes()
        assert host(dv, np.int32).tobytes() == v[: len(keys)][p].tobytes()


def test_sort_reference_bigcases(N):
    # cpp/test/test_sort.cpp:82-168 self-checks: the shuffled 1..10000 sorts back
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "test_sort_cpp.npz"))
    d = dev(g["sort_in"])
    assert N.lib.trtc_raw_sort(4, ptr(d), 10000, 0, None) == 0
    assert (host(d, np.int32) == np.arange(1, 10001)).all()
    dk, dv = dev(g["sbk_keys"]), dev(g["sbk_values"])
    assert N.lib.trtc_raw_sort_by_key(4, ptr(dk), ptr(dv), 4, 10000, 0, None) == 0
    assert (host(dk, np.int32) == np.arange(1, 10001)).all()
    assert (host(dv, np.int32) == 10000 - np.arange(10000)).all()


@pytest.mark.parametrize("name", ["int32_t", "uint8_t", "float", "double", "int64_t"])
def test_min_element_tree(N, name):
    rng = np.random.default_rng(3)
    for n in [1, 2, 255, 256, 257, 65536, 65537, 1 << 20]:
        x = rand_keys(rng, name, n)
        if name in ("float", "double") and n > 4:
            x[rng.integers(0, n, max(1, n // 64))] = np.nan
        d = dev(x)
        got = N.lib.trtc_raw_min_element(N.TYPE_CODES[name], ptr(d), n, None)
        assert got == O.min_element(x), (name, n)


@pytest.mark.parametrize("name", ["int32_t", "uint32_t", "int64_t", "int8_t", "uint16_t"])
@pytest.mark.parametrize("op", ["Plus", "Maximum", "Minimum"])
def test_scan_int(N, name, op):
    rng = np.random.default_rng(11)
    for n in SIZES:
        x = rand_keys(rng, name, n)
        for excl in (False, True):
            init = NP_OF[name](3) if excl else None
            d = dev(x)
            out = dev(np.zeros_like(x))
            ini = np.array([init if init is not None else 0], dtype=NP_OF[name])
            rc = N.lib.trtc_raw_scan(N.TYPE_CODES[name], N.OP_CODES[op], int(excl), ptr(d), ptr(out), n,
                                     ini.ctypes.data_as(ctypes.c_void_p), None)
            assert rc == 0, N.last_error()
            exp = O.scan(x, op, excl, init)
            assert host(out, NP_OF[name]).tobytes() == exp.tobytes(), (name, op, n, excl)


def test_scan_inplace_exclusive(N):
    # docs/QuickStartGuide.md:1013-1019: exclusive scans may run in place
    rng = np.random.default_rng(12)
    for n in [6, 4096 * 3 + 5, 1 << 20]:
        x = rng.integers(-1000, 1001, n, dtype=np.int32)
        d = dev(x)
        zero = np.zeros(1, np.int32)
        assert N.lib.trtc_raw_scan(4, 0, 1, ptr(d), ptr(d), n, zero.ctypes.data_as(ctypes.c_void_p), None) == 0
        assert host(d, np.int32).tobytes() == O.scan(x, "Plus", True, 0).tobytes()


@pytest.mark.parametrize("name", ["float", "double"])
def test_scan_float(N, name):
    rng = np.random.default_rng(13)
    for n in [1, 1000, 4097, 1 << 20]:
        x = rng.random(n).astype(NP_OF[name])
        d, out = dev(x), dev(np.zeros_like(x))
        assert N.lib.trtc_raw_scan(N.TYPE_CODES[name], 0, 0, ptr(d), ptr(out), n, None, None) == 0
        got = host(out, NP_OF[name]).astype(np.float64)
        exp = O.scan_f64(x)
        rel = np.max(np.abs(got - exp) / np.maximum(np.abs(exp), 1e-30))
        assert rel <= REL_TOL, rel


@pytest.mark.parametrize("name", ["float", "int32_t", "uint32_t", "int64_t", "double", "int8_t"])
@pytest.mark.parametrize("op", ["Plus", "Maximum", "Minimum"])
def test_reduce(N, name, op):
    rng = np.random.default_rng(17)
    for n in [1, 3, 255, 4097, 1 << 20 | 3]:
        x = rng.random(n).astype(NP_OF[name]) if name in ("float", "double") else rand_keys(rng, name, n)
        d = dev(x)
        res = np.zeros(1, NP_OF[name])
        for init in (None, NP_OF[name](1)):
            ini = None if init is None else np.array([init], NP_OF[name])
            rc = N.lib.trtc_raw_reduce(N.TYPE_CODES[name], N.OP_CODES[op], ptr(d), n,
                                       None if ini is None else ini.ctypes.data_as(ctypes.c_void_p),
                                       res.ctypes.data_as(ctypes.c_void_p), None)
            assert rc == 0, N.last_error()
            if name in ("float", "double") and op == "Plus":
                exp = O.reduce_f64(x, init, op)
                assert abs(float(res[0]) - exp) <= REL_TOL * abs(exp), (n, res[0], exp)
            else:
                assert res[0] == O.reduce(x, init, op), (name, op, n)


@pytest.mark.parametrize("kname,vname", [("int32_t", "float"), ("int32_t", "int32_t"), ("int64_t", "int64_t"),
                                         ("int64_t", "float"), ("uint32_t", "double")])
def test_scan_by_key(N, kname, vname):
    rng = np.random.default_rng(23)
    for n in [1, 10, 1000, 4097, 1 << 20]:
        runs = rng.geometric(1 / 32, n)
        keys = np.repeat(np.arange(len(runs)), runs)[:n].astype(NP_OF[kname])
        vals = (rng.random(n) if vname in ("float", "double") else rng.integers(-1000, 1000, n)).astype(NP_OF[vname])
        for excl in (False, True):
            init = NP_OF[vname](5)
            dk, dv, do = dev(keys), dev(vals), dev(np.zeros_like(vals))
            ini = np.array([init], NP_OF[vname])
            rc = N.lib.trtc_raw_scan_by_key(N.TYPE_CODES[kname], N.TYPE_CODES[vname], int(excl), ptr(dk), ptr(dv),
                                            ptr(do), n, ini.ctypes.data_as(ctypes.c_void_p), None)
            assert rc == 0, N.last_error()
            got = host(do, NP_OF[vname])
            if vname in ("float", "double"):
                exp = O.scan_by_key(keys, vals, "Plus", excl, init if excl else None, f64=True)
                rel = np.max(np.abs(got - exp) / np.maximum(np.abs(exp), 1e-30))
                assert rel <= REL_TOL, rel
            else:
                exp = O.scan_by_key(keys, vals, "Plus", excl, init if excl else None)
                assert got.tobytes() == exp.tobytes(), (kname, vname, n, excl)


@pytest.mark.parametrize("kname,vname", [("int32_t", "int32_t"), ("int64_t", "int64_t")])
def test_scan_by_key_long_runs_inplace_unaligned(N, kname, vname):
    # segments spanning many tiles (the segmented look-back walks over head-free tiles),
    # a single segment, all heads, in-place output, and arrays shifted off 16-byte alignment
    rng = np.random.default_rng(31)
    n = (1 << 21) + 37
    cases = {
        "long runs": np.repeat(np.arange(40), rng.multinomial(n, [1 / 40] * 40)),
        "one segment": np.zeros(n, np.int64),
        "all heads": np.arange(n),
    }
    for label, kk in cases.items():
        keys = kk[:n].astype(NP_OF[kname])
        vals = rng.integers(-1000, 1000, n).astype(NP_OF[vname])
        for excl in (False, True):
            ini = np.array([7], NP_OF[vname])
            exp = O.scan_by_key(keys, vals, "Plus", excl, 7 if excl else None)
            for shift in (0, 1):
                dk = dev(np.concatenate([np.zeros(shift, keys.dtype), keys]))
                dv = dev(np.concatenate([np.zeros(shift, vals.dtype), vals]))
                esz = keys.dtype.itemsize
                kp = ctypes.c_void_p(dk.data_ptr() + shift * esz)
                vp = ctypes.c_void_p(dv.data_ptr() + shift * esz)
                rc = N.lib.trtc_raw_scan_by_key(N.TYPE_CODES[kname], N.TYPE_CODES[vname], int(excl), kp, vp, vp, n,
                                                ini.ctypes.data_as(ctypes.c_void_p), None)
                assert rc == 0, N.last_error()
                got = host(dv, NP_OF[vname])[shift:]
                assert got.tobytes() == exp.tobytes(), (label, excl, shift)


@pytest.mark.parametrize("name", ["int32_t", "float", "uint8_t", "int64_t"])
def test_remove_unique(N, name):
    rng = np.random.default_rng(29)
    for n in [1, 7, 4096, 4097, 1 << 20]:
        x = rng.integers(0, 5, n).astype(NP_OF[name])
        d, out = dev(x), dev(np.zeros_like(x))
        val = np.array([2], NP_OF[name])
        c = N.lib.trtc_raw_remove_copy(N.TYPE_CODES[name], ptr(d), ptr(out), n, val.ctypes.data_as(ctypes.c_void_p), None)
        exp = x[O.remove_flags(x, 2)]
        assert c == len(exp)
        assert host(out, NP_OF[name])[:c].tobytes() == exp.tobytes()
        # in place
        c = N.lib.trtc_raw_unique_copy(N.TYPE_CODES[name], ptr(d), ptr(d), n, None)
        exp = x[O.unique_flags(x)]
        assert c == len(exp)
        assert host(d, NP_OF[name])[:c].tobytes() == exp.tobytes()
