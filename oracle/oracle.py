"""CPU oracle for the ThrustRTC hot path -- TEST INFRASTRUCTURE ONLY.

This module restates, on the host, the results the reference library (fynv/ThrustRTC)
produces for sort / scan / scan_by_key / reduce / min_element (C++ in trtc_oracle.cpp,
loaded with ctypes), for the scan-based compaction family and for the remaining algorithms
(index trees of the extrema, merge ranks, first-index searches; numpy, below).  It is the
checker for the CUDA kernels of ``thrustrtc_b200``: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  Nothing in the product package imports or calls it.

Parity pins: the doc vectors of docs/QuickStartGuide.md:996-1095 and the self-checking
big cases of cpp/test/test_sort.cpp:82-168 (see tests/golden/), plus the key map and the
built-in operators of built_in.h:14-150,430-458, compiled from the reference's own header
by oracle/build_ref_probe.py into oracle/_ref/ where the reference tree is present.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "trtc_oracle.cpp")
LIB = os.path.join(HERE, "liboracle.so")

TYPE_CODES = {
    "int8_t": 0, "uint8_t": 1, "int16_t": 2, "uint16_t": 3, "int32_t": 4, "uint32_t": 5,
    "int64_t": 6, "uint64_t": 7, "float": 8, "double": 9,
}
NP_CODES = {
    np.dtype(np.int8): 0, np.dtype(np.uint8): 1, np.dtype(np.int16): 2, np.dtype(np.uint16): 3,
    np.dtype(np.int32): 4, np.dtype(np.uint32): 5, np.dtype(np.int64): 6, np.dtype(np.uint64): 7,
    np.dtype(np.float32): 8, np.dtype(np.float64): 9,
}
OPS = {"Plus": 0, "Maximum": 1, "Minimum": 2}


def build(force=False):
    """Compile trtc_oracle.cpp into oracle/liboracle.so (g++, -O2, std::thread)."""
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(SRC)):
        return LIB
    tmp = LIB + ".tmp"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", SRC, "-o", tmp])
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, u64, i = ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_int
        L.oracle_min_element.restype = u64
        L.oracle_min_element.argtypes = [i, vp, u64]
        for name in ("oracle_sort_perm", "oracle_sort_perm_bitsplit"):
            getattr(L, name).restype = i
            getattr(L, name).argtypes = [i, vp, u64, i, vp]
        L.oracle_keymap.argtypes = [i, vp, u64, vp]
        L.oracle_scan.argtypes = [i, i, i, vp, u64, vp, vp]
        L.oracle_scan_f64.argtypes = [i, i, i, vp, u64, vp, vp]
        L.oracle_scan_by_key.argtypes = [i, i, i, i, vp, vp, u64, vp, vp, vp]
        L.oracle_reduce.argtypes = [i, i, vp, u64, vp, vp]
        L.oracle_reduce_f64.argtypes = [i, i, vp, u64, vp, vp]
        L.oracle_reduce_tree.argtypes = [i, i, vp, u64, vp, vp]
        L.oracle_sort_pairs32.argtypes = [i, vp, vp, u64, i, i, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _scalar(dtype, v):
    if v is None:
        return None
    return np.array([v], dtype=dtype)


# ---------------------------------------------------------------- sort / min_element

def min_element(keys):
    """TRTC_Min_Element (extrema.cpp:5-13) with its exact 256-wide tree order."""
    keys = np.ascontiguousarray(keys)
    if len(keys) == 0:
        return 0
    return int(lib().oracle_min_element(NP_CODES[keys.dtype], _ptr(keys), len(keys)))


def keymap(keys):
    """d_u32 / d_u64 of built_in.h:430-458, as uint64."""
    keys = np.ascontiguousarray(keys)
    out = np.empty(len(keys), dtype=np.uint64)
    lib().oracle_keymap(NP_CODES[keys.dtype], _ptr(keys), len(keys), _ptr(out))
    return out


def sort_perm(keys, descending=False, literal=False):
    """Stable permutation the reference radix sort applies (internal/radix_sort.cpp)."""
    keys = np.ascontiguousarray(keys)
    perm = np.empty(len(keys), dtype=np.uint64)
    if len(keys):
        fn = lib().oracle_sort_perm_bitsplit if literal else lib().oracle_sort_perm
        fn(NP_CODES[keys.dtype], _ptr(keys), len(keys), 1 if descending else 0, _ptr(perm))
    return perm.astype(np.int64)


def sort(keys, descending=False):
    return np.ascontiguousarray(keys)[sort_perm(keys, descending)]


def sort_pairs32(keys, values, descending=False, threads=1):
    """Sort_By_Key of 32-bit keys with 32-bit values on `threads` host threads (same order as
    sort_by_key); the timed host baseline of the pair sort."""
    keys = np.ascontiguousarray(keys)
    values = np.ascontiguousarray(values)
    assert keys.dtype.itemsize == 4 and values.dtype.itemsize == 4 and len(values) == len(keys)
    ko, vo = np.empty_like(keys), np.empty_like(values)
    r = lib().oracle_sort_pairs32(NP_CODES[keys.dtype], _ptr(keys), _ptr(values), len(keys),
                                  1 if descending else 0, int(threads), _ptr(ko), _ptr(vo))
    if r != 0:
        raise ValueError("sort_pairs32: unsupported input")
    return ko, vo


def sort_by_key(keys, values, descending=False):
    """TRTC_Sort_By_Key: values beyond len(keys) stay in place (radix_sort.cpp:328-343)."""
    p = sort_perm(keys, descending)
    v = np.array(values, copy=True)
    v[: len(keys)] = np.asarray(values)[: len(keys)][p]
    return np.ascontiguousarray(keys)[p], v


# ---------------------------------------------------------------- scans

def scan(x, op="Plus", exclusive=False, init=None):
    """Inclusive / exclusive scan in the value type (scan.cpp:4-39)."""
    x = np.ascontiguousarray(x)
    out = np.empty_like(x)
    if exclusive and init is None:
        init = 0
    ini = _scalar(x.dtype, init)
    if len(x):
        lib().oracle_scan(NP_CODES[x.dtype], OPS[op], 1 if exclusive else 0, _ptr(x), len(x), _ptr(ini), _ptr(out))
    return out


def scan_f64(x, op="Plus", exclusive=False, init=None):
    x = np.ascontiguousarray(x)
    out = np.empty(len(x), dtype=np.float64)
    if exclusive and init is None:
        init = 0
    ini = _scalar(x.dtype, init)
    if len(x):
        lib().oracle_scan_f64(NP_CODES[x.dtype], OPS[op], 1 if exclusive else 0, _ptr(x), len(x), _ptr(ini), _ptr(out))
    return out


def scan_by_key(keys, vals, op="Plus", exclusive=False, init=None, f64=False):
    """Segmented scan, segments continue while key[i-1] == key[i] (scan_by_key.cpp:4-53)."""
    keys = np.ascontiguousarray(keys)
    vals = np.ascontiguousarray(vals)
    ini = _scalar(vals.dtype, init)
    out = np.empty(len(vals), dtype=np.float64 if f64 else vals.dtype)
    if len(vals):
        rc = lib().oracle_scan_by_key(NP_CODES[keys.dtype], NP_CODES[vals.dtype], OPS[op], 1 if exclusive else 0,
                                      _ptr(keys), _ptr(vals), len(vals), _ptr(ini),
                                      None if f64 else _ptr(out), _ptr(out) if f64 else None)
        assert rc == 0, "unsupported key/value types for the scan_by_key oracle"
    return out


# ---------------------------------------------------------------- reduce

def reduce(x, init=None, op="Plus"):
    """TRTC_Reduce in the value type (sequential fold; None for the n == 0 failure)."""
    x = np.ascontiguousarray(x)
    ini = _scalar(x.dtype, init)
    out = np.empty(1, dtype=x.dtype)
    rc = lib().oracle_reduce(NP_CODES[x.dtype], OPS[op], _ptr(x), len(x), _ptr(ini), _ptr(out))
    return None if rc else out[0]


def reduce_f64(x, init=None, op="Plus"):
    x = np.ascontiguousarray(x)
    ini = _scalar(x.dtype, init)
    out = np.empty(1, dtype=np.float64)
    rc = lib().oracle_reduce_f64(NP_CODES[x.dtype], OPS[op], _ptr(x), len(x), _ptr(ini), _ptr(out))
    return None if rc else float(out[0])


def reduce_tree(x, init=None, op="Plus"):
    """The reference's own association order (256-wide trees), for FP diagnostics."""
    x = np.ascontiguousarray(x)
    ini = _scalar(x.dtype, init)
    out = np.empty(1, dtype=x.dtype)
    rc = lib().oracle_reduce_tree(NP_CODES[x.dtype], OPS[op], _ptr(x), len(x), _ptr(ini), _ptr(out))
    return None if rc else out[0]


# ---------------------------------------------------------------- compaction (numpy)
# internal/general_copy_if.cpp:26-64: a stable compaction of the elements whose flag is 1.

def copy_if(x, flags):
    return np.asarray(x)[np.asarray(flags, dtype=bool)]


def remove_flags(x, value):
    """remove.cpp:5-19: keep src[idx] != value."""
    return np.asarray(x) != value


def unique_flags(x, eq=None):
    """unique.cpp:5-12,14-21: keep idx == 0 || !pred(src[idx], src[idx-1]) (default !=)."""
    x = np.asarray(x)
    f = np.ones(len(x), dtype=bool)
    if len(x) > 1:
        f[1:] = (x[1:] != x[:-1]) if eq is None else ~eq(x[1:], x[:-1])
    return f


def partition(x, flags):
    """partition.cpp:29-125: trues in order, then falses in order; returns (out, count)."""
    x = np.asarray(x)
    f = np.asarray(flags, dtype=bool)
    return np.concatenate([x[f], x[~f]]), int(f.sum())


def reduce_by_key(keys, vals, op="Plus"):
    """reduce.cpp:36-44: scan_by_key then copy_if of the segment tails."""
    keys = np.asarray(keys)
    s = scan_by_key(keys, vals, op)
    tail = np.ones(len(keys), dtype=bool)
    if len(keys) > 1:
        tail[:-1] = keys[:-1] != keys[1:]
    return keys[tail], s[tail]


# ---------------------------------------------------------------- remaining algorithms (numpy)

def index_tree(x, maximum=False, less=None):
    """Max/Min_Element (extrema.cpp:5-44) over internal/general_reduce.cpp:55-95: blocks of 256
    slots, s = 128..1, slot t takes op(h[t], h[t+s]) when t + s < L; rounds repeat on the
    block results.  max: comp(v[i1], v[i2]) ? i2 : i1; min: comp(v[i2], v[i1]) ? i2 : i1.
    `less(a, b)` is the elementwise comparison (default a < b, so NaN compares false)."""
    x = np.asarray(x)
    if len(x) == 0:
        return None
    if less is None:
        less = lambda a, b: a < b  # noqa: E731
    cur = np.arange(len(x), dtype=np.int64)
    first = True
    while first or len(cur) > 1:
        first = False
        m = len(cur)
        nb = (m + 255) // 256
        h = np.zeros(nb * 256, dtype=np.int64)
        h[:m] = cur
        h = h.reshape(nb, 256)
        L = np.minimum(256, m - np.arange(nb) * 256)[:, None]
        s = 128
        while s > 0:
            t = np.arange(s)[None, :]
            ok = (t + s) < L
            i1, i2 = h[:, :s], h[:, s:2 * s]
            take2 = less(x[i1], x[i2]) if maximum else less(x[i2], x[i1])
            h[:, :s] = np.where(ok & take2, i2, i1)
            s >>= 1
        cur = h[:, 0].copy()
    return int(cur[0])


def first_true(flags):
    """internal/general_find.cpp:4-42: the lowest index whose flag is set, else None."""
    idx = np.flatnonzero(np.asarray(flags, dtype=bool))
    return int(idx[0]) if len(idx) else None


def merge(a, b, va=None, vb=None, less=None):
    """merge.cpp:3-66: a[i] goes to i + lower_bound(b, a[i]), b[j] to j + upper_bound(a, b[j])
    under `less` (default <; pass lambda x, y: x > y for Greater).  Returns keys (, values)."""
    a, b = np.asarray(a), np.asarray(b)
    if less is None:
        pa = np.arange(len(a)) + np.searchsorted(b, a, side="left")
        pb = np.arange(len(b)) + np.searchsorted(a, b, side="right")
    else:
        pa = np.array([i + sum(1 for y in b if less(y, x)) for i, x in enumerate(a)], dtype=np.int64)
        pb = np.array([j + sum(1 for x in a if not less(y, x)) for j, y in enumerate(b)], dtype=np.int64)
    out = np.empty(len(a) + len(b), dtype=np.result_type(a, b))
    out[pa], out[pb] = a, b
    if va is None:
        return out
    vout = np.empty(len(a) + len(b), dtype=np.result_type(np.asarray(va), np.asarray(vb)))
    vout[pa], vout[pb] = va, vb
    return out, vout


def adjacent_difference(x):
    """adjacent_difference.cpp:3-13: out[0] = in[0], out[i] = in[i] - in[i-1] in the element type."""
    x = np.asarray(x)
    out = x.copy()
    if len(x) > 1:
        out[1:] = x[1:] - x[:-1]
    return out


def is_sorted_until(x, less=None):
    """sort.cpp:93-103: the first i >= 1 with comp(v[i], v[i-1]), else the size."""
    x = np.asarray(x)
    if len(x) < 2:
        return len(x)
    brk = (x[1:] < x[:-1]) if less is None else less(x[1:], x[:-1])
    i = first_true(brk)
    return len(x) if i is None else i + 1


def is_partitioned(flags):
    """partition.cpp:199-214: no true flag right after a false one (true when empty)."""
    f = np.asarray(flags, dtype=bool)
    return not bool(np.any(~f[:-1] & f[1:])) if len(f) > 1 else True
