"""Batched segmented sort + exclusive scan (trtc_raw_segmented_sort_scan) against the oracle,
segment by segment: every segment must equal a stable Sort_By_Key of that segment alone and
the exclusive Plus scan (uint32 wrap-around) of its sorted values.  Bit-exact."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TC = {"uint32_t": 5, "int32_t": 4, "float": 8, "int64_t": 6, "uint64_t": 7}
NP = {"uint32_t": np.uint32, "int32_t": np.int32, "float": np.float32, "int64_t": np.int64, "uint64_t": np.uint64}


@pytest.fixture(scope="module")
def N(cuda):
    from thrustrtc_b200 import _native as N
    L = N.lib
    L.trtc_raw_segmented_workspace_bytes.restype = ctypes.c_ulonglong
    L.trtc_raw_segmented_workspace_bytes.argtypes = [ctypes.c_int, ctypes.c_ulonglong, ctypes.c_ulonglong]
    L.trtc_raw_segmented_sort_scan.restype = ctypes.c_int
    L.trtc_raw_segmented_sort_scan.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + \
        [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_void_p]
    L.trtc_raw_segmented_tuning_json.restype = ctypes.c_ulonglong
    L.trtc_raw_segmented_tuning_json.argtypes = [ctypes.c_char_p, ctypes.c_ulonglong]
    L.trtc_raw_segmented_tuning_load.restype = ctypes.c_int
    L.trtc_raw_segmented_tuning_load.argtypes = [ctypes.c_char_p]
    L.trtc_raw_segmented_autotune.restype = ctypes.c_int
    L.trtc_raw_segmented_autotune.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong,
                                              ctypes.c_ulonglong, ctypes.c_void_p]
    return N


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def make_lengths(rng, nseg, median, sigma, hi):
    z = rng.standard_normal(nseg)
    lens = np.clip(np.round(np.exp(np.log(median) + sigma * z)), 1, hi).astype(np.int64)
    return lens


def keys_for(rng, name, n):
    if name == "float":
        x = (rng.standard_normal(n) * 100).astype(np.float32)
        x[rng.integers(0, n, max(1, n // 50))] = -0.0
        x[rng.integers(0, n, max(1, n // 50))] = 0.0
        return x
    info = np.iinfo(NP[name])
    if rng.random() < 0.5:
        return rng.integers(info.min, info.max, n, dtype=NP[name], endpoint=True)
    return rng.integers(0, 50, n).astype(NP[name])  # many duplicates: stability matters


def expected(keys, vals, off, desc):
    ek, ev, es = keys.copy(), vals.copy(), np.zeros_like(vals)
    for i in range(len(off) - 1):
        a, b = off[i], off[i + 1]
        if a == b:
            continue
        k, v = O.sort_by_key(keys[a:b], vals[a:b], desc)
        ek[a:b], ev[a:b] = k, v
        c = np.cumsum(v.astype(np.uint64)) & 0xFFFFFFFF
        es[a:b] = np.concatenate([[0], c[:-1]]).astype(np.uint32)
    return ek, ev, es


def run(N, name, keys, vals, off, desc, stream=None):
    import torch
    n, nseg = len(keys), len(off) - 1
    tk = torch.from_numpy(keys.view(np.int32) if keys.dtype.itemsize == 4 else keys.view(np.int64)).cuda()
    tv = torch.from_numpy(vals.view(np.int32)).cuda()
    ts = torch.full_like(tv, -1)
    to = torch.from_numpy(off.astype(np.int64)).cuda()
    wsb = N.lib.trtc_raw_segmented_workspace_bytes(TC[name], n, nseg)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    rc = N.lib.trtc_raw_segmented_sort_scan(TC[name], _p(tk), _p(tv), _p(ts), _p(to), nseg, n, _p(ws), wsb,
                                            int(desc), stream)
    assert rc == 0, N.last_error()
    torch.cuda.synchronize()
    return (tk.cpu().numpy().view(keys.dtype), tv.cpu().numpy().view(np.uint32), ts.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("name", ["uint32_t", "int32_t", "float", "int64_t", "uint64_t"])
@pytest.mark.parametrize("desc", [False, True])
def test_segmented_matches_per_segment_sort_and_scan(N, name, desc):
    rng = np.random.default_rng(7 + 3 * int(desc) + len(name))
    lens = make_lengths(rng, 400, 64, 1.5, 20000)
    lens[:5] = [0, 1, 2, 2048, 4097]     # empty, single, tile edges of both configurations
    lens[5:8] = [4096, 4095, 12000]       # on-chip limit and a chunked segment
    lens[8:20] = [31, 32, 33, 255, 256, 257, 511, 512, 513, 300, 700, 3]  # one-warp limits (256 / 512 keys)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n = int(off[-1])
    keys = keys_for(rng, name, n)
    vals = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    gk, gv, gs = run(N, name, keys, vals, off, desc)
    ek, ev, es = expected(keys, vals, off, desc)
    assert gk.tobytes() == ek.tobytes()
    assert np.array_equal(gv, ev)
    assert np.array_equal(gs, es)


def test_segmented_autotune_and_repeat(N):
    import torch
    rng = np.random.default_rng(11)
    lens = make_lengths(rng, 3000, 256, 1.5, 1 << 20)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n = int(off[-1])
    to = torch.from_numpy(off).cuda()
    chosen = N.lib.trtc_raw_segmented_autotune(5, _p(to), len(lens), n, None)
    assert chosen in (8, 16), N.last_error()
    keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    ek, ev, es = expected(keys, vals, off, False)
    for _ in range(2):
        gk, gv, gs = run(N, "uint32_t", keys, vals, off, False)
        assert np.array_equal(gk, ek) and np.array_equal(gv, ev) and np.array_equal(gs, es)


def test_segmented_cuda_graph_replay(N):
    import torch
    rng = np.random.default_rng(5)
    lens = make_lengths(rng, 1000, 128, 1.5, 50000)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n, nseg = int(off[-1]), len(lens)
    keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    ek, ev, es = expected(keys, vals, off, False)
    k0 = torch.from_numpy(keys.view(np.int32)).cuda()
    v0 = torch.from_numpy(vals.view(np.int32)).cuda()
    tk, tv, ts = torch.empty_like(k0), torch.empty_like(v0), torch.empty_like(v0)
    to = torch.from_numpy(off).cuda()
    wsb = N.lib.trtc_raw_segmented_workspace_bytes(5, n, nseg)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()

    def step():
        tk.copy_(k0)
        tv.copy_(v0)
        rc = N.lib.trtc_raw_segmented_sort_scan(5, _p(tk), _p(tv), _p(ts), _p(to), nseg, n, _p(ws), wsb, 0,
                                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, N.last_error()

    with torch.cuda.stream(s):
        step()  # uncaptured first call sets the kernels up
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        step()
    for _ in range(2):
        ts.fill_(0)
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(tk.cpu().numpy().view(np.uint32), ek)
        assert np.array_equal(tv.cpu().numpy().view(np.uint32), ev)
        assert np.array_equal(ts.cpu().numpy().view(np.uint32), es)


@pytest.mark.parametrize("desc", [False, True])
def test_segmented_float_nan_rotation(N, desc):
    # Segments holding NaNs get the reference's Min_Element rotation (extrema.cpp:5-13), as a
    # Sort_By_Key call on the segment alone would: +NaN, -NaN, payload NaNs, NaN at the
    # segment's index 0 (the tree then selects it), NaN only past the first 256-block, and
    # segments of every class (one warp, on chip, global memory; > 65536 keys: three tree rounds).
    rng = np.random.default_rng(41 + int(desc))
    lens = np.array([1, 2, 5, 31, 33, 256, 257, 300, 513, 2047, 4096, 4097, 9000, 70000, 200, 1000, 3, 64],
                    dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n = int(off[-1])
    keys = (rng.standard_normal(n) * 10).astype(np.float32)
    keys[rng.integers(0, n, n // 40)] = -0.0
    bits = keys.view(np.uint32)
    pats = np.array([0x7FC00000, 0xFFC00000, 0x7FC00123, 0xFF800001], dtype=np.uint32)
    for i in range(len(lens)):
        a, b = off[i], off[i + 1]
        mode = i % 4
        if mode == 0:      # NaN at index 0 of the segment
            bits[a] = pats[i % len(pats)]
        elif mode == 1:    # NaNs scattered (may sit in left slots of the tree)
            for j in rng.integers(a, b, max(1, (b - a) // 50)):
                bits[j] = pats[int(j) % len(pats)]
        elif mode == 2 and b - a > 300:  # NaN only after the first 256-block
            bits[a + 280] = pats[1]
        # mode 3: no NaN
    vals = np.arange(n, dtype=np.uint32)
    gk, gv, gs = run(N, "float", keys, vals, off, desc)
    ek, ev, es = expected(keys, vals, off, desc)
    assert gk.tobytes() == ek.tobytes()
    assert np.array_equal(gv, ev)
    assert np.array_equal(gs, es)


SHAPES = [(8, 0), (8, 32), (16, 0), (16, 32)]


@pytest.mark.parametrize("items,warp_small", SHAPES)
@pytest.mark.parametrize("name", ["uint32_t", "float", "int64_t"])
def test_every_size_class_of_every_shape(N, items, warp_small, name):
    # a table forcing each shape; lengths on both sides of every class limit of that shape:
    # the bitonic warp class (<= 32), the radix warp class (<= 32 * items), the two- and
    # four-warp groups (<= 64 * items, <= 128 * items), the on-chip CTA class (<= 256 * items)
    # and the global-memory CTA class
    table = ('{"format": "thrustrtc_b200.segmented_tuning", "version": 1, "entries": '
             '[{"key_type": %d, "items": %d, "warp_small": %d}]}' % (TC[name], items, warp_small))
    old = ctypes.create_string_buffer(4096)
    N.lib.trtc_raw_segmented_tuning_json(old, 4096)
    assert N.lib.trtc_raw_segmented_tuning_load(table.encode()) == 0
    try:
        rng = np.random.default_rng(items + warp_small + len(name))
        lims = [1, 2, 31, 32, 33, 32 * items - 1, 32 * items, 32 * items + 1, 48 * items + 5, 64 * items - 1,
                64 * items, 64 * items + 1, 100 * items + 3, 128 * items - 1, 128 * items, 128 * items + 1,
                256 * items - 1, 256 * items, 256 * items + 1, 3 * 256 * items + 17]
        lims += [64 * items] * 9 + [128 * items - 7] * 5  # several groups of one class at once
        lens = np.array(lims + list(make_lengths(rng, 200, 40, 1.5, 6000)), dtype=np.int64)
        rng.shuffle(lens)
        off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        n = int(off[-1])
        keys = keys_for(rng, name, n)
        vals = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        for desc in (False, True):
            gk, gv, gs = run(N, name, keys, vals, off, desc)
            ek, ev, es = expected(keys, vals, off, desc)
            assert gk.tobytes() == ek.tobytes()
            assert np.array_equal(gv, ev)
            assert np.array_equal(gs, es)
    finally:
        N.lib.trtc_raw_segmented_tuning_load(old.value)
