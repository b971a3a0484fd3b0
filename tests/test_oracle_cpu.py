"""CPU checks of the oracle itself, against the reference's golden vectors.

Pins: docs/QuickStartGuide.md known answers (tests/golden/docs_vectors.json), the
self-checking big cases of cpp/test/test_sort.cpp (tests/golden/test_sort_cpp.npz), and
d_u32/d_u64 + Maximum/Minimum evaluated by the reference's own built_in.h compiled on the
CPU (tests/golden/builtin_h_probe.json).  Also cross-checks the oracle's fast sort against
its literal restatement of the 1-bit LSD split.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
NP = {"int32_t": np.int32, "int8_t": np.int8}


def _docs():
    with open(os.path.join(GOLD, "docs_vectors.json")) as f:
        return json.load(f)


def test_docs_scans():
    d = _docs()
    x = np.array(d["inclusive_scan"]["in"], np.int32)
    assert O.scan(x).tolist() == d["inclusive_scan"]["out"]
    x = np.array(d["exclusive_scan"]["in"], np.int32)
    assert O.scan(x, exclusive=True).tolist() == d["exclusive_scan"]["out"]


def test_docs_sorts():
    d = _docs()
    x = np.array(d["sort"]["in"], np.int32)
    assert O.sort(x).tolist() == d["sort"]["out"]
    assert O.sort(x, descending=True).tolist() == d["sort_greater"]["out"]
    for case in ("sort_by_key_char", "sort_by_key_int"):
        c = d[case]
        k, v = O.sort_by_key(np.array(c["keys"], NP[c["key_dtype"]]), np.array(c["values"], NP[c["value_dtype"]]))
        assert k.tolist() == c["keys_out"] and v.tolist() == c["values_out"]


def test_reference_test_sort_bigcases():
    g = np.load(os.path.join(GOLD, "test_sort_cpp.npz"))
    assert (O.sort(g["sort_in"]) == np.arange(1, 10001)).all()
    k, v = O.sort_by_key(g["sbk_keys"], g["sbk_values"])
    assert (k == np.arange(1, 10001)).all() and (v == 10000 - np.arange(10000)).all()


def test_keymap_matches_reference_header():
    with open(os.path.join(GOLD, "builtin_h_probe.json")) as f:
        p = json.load(f)
    bits = np.array([a for a, _ in p["f32"]], np.uint32)
    got = O.keymap(bits.view(np.float32)).astype(np.uint64)
    assert got.tolist() == [b for _, b in p["f32"]]
    # double: the CPU-compiled header agrees with the oracle except on negative NaNs, where
    # the oracle follows the reference as it runs on the GPU (next test)
    bits = np.array([int(a) for a, _ in p["f64"]], np.uint64)
    neg_nan = ((bits & np.uint64(0x7FFFFFFFFFFFFFFF)) > np.uint64(0x7FF0000000000000)) & (bits >> np.uint64(63) == 1)
    got = O.keymap(bits.view(np.float64))
    want = np.array([int(b) for _, b in p["f64"]], np.uint64)
    assert neg_nan.any() and (got[~neg_nan] == want[~neg_nan]).all()
    for row in p["ints"]:
        v = int(row[0])
        assert O.keymap(np.array([v], np.int64).astype(np.int8))[0] == row[1]
        assert O.keymap(np.array([v & 0xFF], np.uint8))[0] == row[2]
        assert O.keymap(np.array([v], np.int64).astype(np.int16))[0] == row[3]
        assert O.keymap(np.array([v & 0xFFFF], np.uint16))[0] == row[4]
        assert O.keymap(np.array([v], np.int64).astype(np.int32))[0] == row[5]
        assert O.keymap(np.array([v & 0xFFFFFFFF], np.uint32))[0] == row[6]
        assert O.keymap(np.array([v], np.int64))[0] == int(row[7])
        assert O.keymap(np.array([v % (1 << 64)], np.uint64))[0] == int(row[8])


def test_keymap_matches_reference_on_the_gpu():
    # d_u64 / d_u32 of built_in.h evaluated by the reference itself on a B200 (a TRTC_For kernel
    # compiled by NVRTC; tests/golden/make_ref_fixtures.py) on edge bit patterns: signed zeros,
    # denormals, infinities and NaNs of both signs, quiet and signalling, with payloads
    with open(os.path.join(GOLD, "ref_keymap_probe.json")) as f:
        p = json.load(f)
    for tag, ft, bt in (("f64", np.float64, np.uint64), ("f32", np.float32, np.uint32)):
        bits = np.array([int(e["bits"], 16) for e in p[tag]], bt)
        want = [int(e["key"], 16) for e in p[tag]]
        assert [int(x) for x in O.keymap(bits.view(ft))] == want, tag
        # the reference's own copy kernel keeps every bit pattern
        assert [int(e["after_copy"], 16) for e in p[tag]] == [int(b) for b in bits]


def test_maxmin_semantics_match_reference_header():
    with open(os.path.join(GOLD, "builtin_h_probe.json")) as f:
        p = json.load(f)
    for xb, yb, mx, mn in p["maxmin_f32"]:
        x, y = np.array([xb, yb], np.uint32).view(np.float32)
        # Maximum: x < y ? y : x ; Minimum: x > y ? y : x (built_in.h:23-39)
        a = y if x < y else x
        b = y if x > y else x
        assert np.array([a], np.float32).view(np.uint32)[0] == mx
        assert np.array([b], np.float32).view(np.uint32)[0] == mn
        # the oracle's scans/reductions use the same rule
        assert O.reduce(np.array([y], np.float32), x, "Maximum").view(np.uint32) == mx


@pytest.mark.parametrize("dt", [np.int8, np.uint8, np.int16, np.int32, np.uint32, np.int64, np.uint64,
                                np.float32, np.float64])
def test_fast_sort_equals_literal_bitsplit(dt):
    rng = np.random.default_rng(0)
    for n in (1, 2, 17, 300, 2000):
        if np.issubdtype(dt, np.floating):
            x = rng.standard_normal(n).astype(dt)
            x[rng.integers(0, n, max(1, n // 20))] = np.nan
            x[rng.integers(0, n, max(1, n // 20))] = -0.0
            if n > 3:
                x[0] = np.nan
        else:
            info = np.iinfo(dt)
            x = rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
        for desc in (False, True):
            assert (O.sort_perm(x, desc) == O.sort_perm(x, desc, literal=True)).all()


def test_min_element_tree_nan_selection():
    # a NaN in a left slot absorbs its subtree: [5, NaN, 3, 0] selects 3, not 0
    x = np.array([5, np.nan, 3, 0], np.float32)
    assert O.min_element(x) == 2
    # and the sorted output is the rotation that puts keys >= 3 first
    assert O.sort(x).tolist()[:2] == [3.0, 5.0] and np.isnan(O.sort(x)[2]) and O.sort(x)[3] == 0.0


def test_compaction_restatements():
    x = np.array([1, 3, 3, 3, 2, 2, 1], np.int32)
    assert x[O.unique_flags(x)].tolist() == [1, 3, 2, 1]
    assert x[O.remove_flags(x, 3)].tolist() == [1, 2, 2, 1]
    out, c = O.partition(np.arange(1, 11), np.arange(1, 11) % 2 == 0)
    assert out.tolist() == [2, 4, 6, 8, 10, 1, 3, 5, 7, 9] and c == 5
    k, v = O.reduce_by_key(x, np.array([9, 8, 7, 6, 5, 4, 3], np.int32))
    assert k.tolist() == [1, 3, 2, 1] and v.tolist() == [9, 21, 9, 3]


def test_remaining_algorithm_restatements():
    # the numpy index tree agrees with the C++ restatement of extrema.cpp (NaNs included)
    rng = np.random.default_rng(11)
    for n in (1, 255, 256, 257, 70000):
        x = rng.integers(0, 40, n).astype(np.float32)
        x[rng.integers(0, n, max(1, n // 50))] = np.nan
        assert O.index_tree(x) == O.min_element(x)
    # hand-worked cases of python/test/test_extrema.py, test_merge.py, test_sort.py,
    # test_partition.py, test_adjacent_difference.py (Thrust semantics)
    assert O.index_tree([1, 0, 2, 2, 1, 3]) == 1 and O.index_tree([1, 0, 2, 2, 1, 3], maximum=True) == 5
    assert O.merge([1, 3, 5, 7, 9, 11], [1, 1, 2, 3, 5, 8, 13]).tolist() == [1, 1, 1, 2, 3, 3, 5, 5, 7, 8, 9, 11, 13]
    k, v = O.merge([11, 9, 7, 5, 3, 1], [13, 8, 5, 3, 2, 1, 1], [0] * 6, [1] * 7, less=lambda a, b: a > b)
    assert k.tolist() == [13, 11, 9, 8, 7, 5, 5, 3, 3, 2, 1, 1, 1]
    assert v.tolist() == [1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 1, 1]
    assert O.is_sorted_until([0, 1, 2, 3, 0, 1, 2, 3]) == 4
    assert O.is_sorted_until([3, 2, 1, 0, 3, 2, 1, 0], less=lambda a, b: a > b) == 4
    assert O.is_partitioned(np.array([2, 4, 6, 8, 10, 1, 3, 5, 7, 9]) % 2 == 0)
    assert not O.is_partitioned(np.arange(1, 11) % 2 == 0)
    assert O.adjacent_difference(np.array([1, 2, 1, 2, 1, 2, 1, 2], np.int32)).tolist() == [1, 1, -1, 1, -1, 1, -1, 1]
    assert O.first_true([False, False]) is None and O.first_true([0, 1, 1]) == 1


def test_reference_hot_path_programs_hand_worked():
    # the inputs of python/test/test_scan.py, test_transform_scan.py, test_scan_by_key.py,
    # test_remove.py, test_sort.py and test_unique.py, with their printed values worked by
    # hand from Thrust's semantics (the programs print without expected outputs)
    i32 = lambda v: np.array(v, np.int32)
    a, m = i32([1, 0, 2, 2, 1, 3]), i32([-5, 0, 2, -3, 2, 4, 0, -1, 2, 8])
    assert O.scan(a).tolist() == [1, 1, 3, 5, 6, 9]
    assert O.scan(m, "Maximum").tolist() == [-5, 0, 2, 2, 2, 4, 4, 4, 4, 8]
    assert O.scan(a, exclusive=True).tolist() == [0, 1, 1, 3, 5, 6]
    assert O.scan(a, exclusive=True, init=4).tolist() == [4, 5, 5, 7, 9, 10]
    assert O.scan(m, "Maximum", True, 1).tolist() == [1, 1, 1, 2, 2, 2, 4, 4, 4, 4]
    assert O.scan(-a).tolist() == [-1, -1, -3, -5, -6, -9]
    assert O.scan(-a, exclusive=True, init=4).tolist() == [4, 3, 3, 1, -1, -2]
    k, ones = i32([0, 0, 0, 1, 1, 2, 3, 3, 3, 3]), i32([1] * 10)
    assert O.scan_by_key(k, ones).tolist() == [1, 2, 3, 1, 2, 1, 1, 2, 3, 4]
    assert O.scan_by_key(k, ones, exclusive=True).tolist() == [0, 1, 2, 0, 1, 0, 0, 1, 2, 3]
    assert O.scan_by_key(k, ones, exclusive=True, init=5).tolist() == [5, 6, 7, 5, 6, 5, 5, 6, 7, 8]
    x = i32([3, 1, 4, 1, 5, 9])
    assert x[O.remove_flags(x, 1)].tolist() == [3, 4, 5, 9]
    y = i32([-2, 0, -1, 0, 1, 2])
    assert y[O.remove_flags(y, 0)].tolist() == [-2, -1, 1, 2]
    assert O.copy_if(y, y % 2 != 0).tolist() == [-1, 1]
    z = i32([1, 4, 2, 8, 5, 7])
    assert O.copy_if(z, z % 2 != 0).tolist() == [1, 5, 7]
    assert O.copy_if(z, i32([0, 1, 1, 1, 0, 0]) == 0).tolist() == [1, 5, 7]
    assert O.sort(z).tolist() == [1, 2, 4, 5, 7, 8] and O.sort(z, True).tolist() == [8, 7, 5, 4, 2, 1]
    sk, sv = O.sort_by_key(z, i32([1, 2, 3, 4, 5, 6]))
    assert sk.tolist() == [1, 2, 4, 5, 7, 8] and sv.tolist() == [1, 3, 2, 5, 6, 4]
    sk, sv = O.sort_by_key(z, i32([1, 2, 3, 4, 5, 6]), True)
    assert sk.tolist() == [8, 7, 5, 4, 2, 1] and sv.tolist() == [4, 6, 5, 2, 3, 1]
    u, uv = i32([1, 3, 3, 3, 2, 2, 1]), i32([9, 8, 7, 6, 5, 4, 3])
    f = O.unique_flags(u)
    assert u[f].tolist() == [1, 3, 2, 1] and uv[f].tolist() == [9, 8, 5, 3]


@pytest.mark.parametrize("dt", [np.uint32, np.int32, np.float32])
def test_threaded_pair_sort_equals_the_oracle_order(dt):
    # the timed host baseline (packed key'|index words, parallel chunks, pairwise merges)
    # must produce exactly sort_by_key's order, whatever the thread count
    rng = np.random.default_rng(21)
    n = 100_003
    if dt == np.float32:
        x = rng.standard_normal(n).astype(dt)
        x[rng.integers(0, n, 500)] = -0.0
        x[rng.integers(0, n, 50)] = np.nan
        x[rng.integers(0, n, 2000)] = x[rng.integers(0, n, 2000)]
    else:
        x = rng.integers(0, 5000, n).astype(dt)  # many ties
    v = np.arange(n, dtype=np.uint32)
    for desc in (False, True):
        ek, ev = O.sort_by_key(x, v, desc)
        for threads in (1, 3, 4):
            k, vv = O.sort_pairs32(x, v, desc, threads)
            assert k.tobytes() == ek.tobytes() and vv.tobytes() == ev.tobytes(), (dt, desc, threads)


def test_oracle_forms_agree_where_the_arithmetic_is_exact():
    # integer-valued floats sum exactly in any order and width: the value-type scans, their
    # FP64 forms, the sequential fold and the reference's 256-wide reduction tree must agree,
    # and wrapping int32 sums must equal numpy's modulo-2^32 cumulative sums
    rng = np.random.default_rng(5)
    for n in (1, 255, 256, 257, 70_001):
        f = rng.integers(0, 16, n).astype(np.float32)
        assert O.scan(f).astype(np.float64).tolist() == O.scan_f64(f).tolist() == np.cumsum(f, dtype=np.float64).tolist()
        assert float(O.reduce(f)) == O.reduce_f64(f) == float(O.reduce_tree(f)) == float(f.sum(dtype=np.float64))
        k = np.repeat(np.arange(n), rng.integers(1, 5, n))[:n].astype(np.int32)
        assert O.scan_by_key(k, f).astype(np.float64).tolist() == O.scan_by_key(k, f, f64=True).tolist()
        i = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
        assert O.scan(i).tolist() == np.cumsum(i, dtype=np.int64).astype(np.int32).tolist()
        assert O.reduce(i) == O.reduce_tree(i) == np.int32(np.int64(i.sum(dtype=np.int64)).astype(np.int32))
