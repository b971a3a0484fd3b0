"""Request server (include/trtc_server.h): a mix of Sort_By_Key, exclusive scan and reduce
requests of many sizes and element types, served with coalescing and overlap, must give each
request the same result as serving it alone, and the oracle's result (bit-exact for sorts and
integer work; float sums and scans of mixed-sign data within REL_TOL times the sum of the
magnitudes of the terms, the FP32 accumulation bound, of the FP64 oracle)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL_TOL = 1e-5
TYPES = {5: np.uint32, 6: np.int64, 8: np.float32}


@pytest.fixture(scope="module")
def L(cuda):
    from thrustrtc_b200 import _native as N
    L = N.lib
    L.trtc_server_create.restype = ctypes.c_void_p
    L.trtc_server_create.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.c_ulonglong]
    L.trtc_server_submit.restype = ctypes.c_longlong
    L.trtc_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_ulonglong]
    L.trtc_server_poll.restype = ctypes.c_int
    L.trtc_server_poll.argtypes = [ctypes.c_void_p]
    L.trtc_server_info.restype = ctypes.c_int
    L.trtc_server_info.argtypes = [ctypes.c_void_p, ctypes.c_longlong] + [ctypes.POINTER(ctypes.c_double)] * 3
    L.trtc_server_result.restype = ctypes.c_int
    L.trtc_server_result.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p]
    L.trtc_server_destroy.argtypes = [ctypes.c_void_p]
    return L


NAN_BITS = np.array([0x7FC00000, 0xFFC00000, 0x7FC00123], dtype=np.uint32)


def add_nans(rng, x):
    """NaNs (+, -, payload) in a float sort request; at index 0 in a third of the requests
    (the reference's Min_Element then selects the NaN and the sorted order is rotated)."""
    b = x.view(np.uint32)
    b[rng.integers(0, len(x), max(1, len(x) // 100))] = NAN_BITS[rng.integers(0, 3)]
    if rng.random() < 0.34:
        b[0] = NAN_BITS[rng.integers(0, 3)]


def make_requests(rng, count, lo_log2, hi_log2):
    reqs = []
    for _ in range(count):
        kind = rng.choice([0, 1, 2], p=[0.6, 0.25, 0.15])
        t = int(rng.choice(list(TYPES)))
        n = int(2 ** rng.uniform(lo_log2, hi_log2))
        dt = TYPES[t]
        if dt == np.float32:
            x = rng.standard_normal(n).astype(np.float32)
            if kind == 0 and rng.random() < 0.5:
                add_nans(rng, x)
        elif kind == 0:
            x = rng.integers(0, 1000, n).astype(dt)  # duplicates: stability matters
        else:
            x = rng.integers(-1000 if dt == np.int64 else 0, 1000, n).astype(dt)
        reqs.append((kind, t, x))
    return reqs


class Run:
    def __init__(self, L, reqs):
        import torch
        self.L, self.reqs = L, reqs
        self.k = [torch.from_numpy(x.view(np.int32) if x.dtype.itemsize == 4 else x.view(np.int64)).cuda()
                  for _, _, x in reqs]
        self.v = [torch.arange(len(x), dtype=torch.int32, device="cuda") if kind == 0 else None
                  for kind, _, x in reqs]
        self.o = [torch.empty_like(k) if kind == 1 else None for (kind, _, _), k in zip(reqs, self.k)]

    def submit(self, srv, i):
        kind, t, x = self.reqs[i]
        p = lambda a: ctypes.c_void_p(a.data_ptr()) if a is not None else None  # noqa: E731
        rid = self.L.trtc_server_submit(srv, kind, t, p(self.k[i]), p(self.v[i]), p(self.o[i]), len(x))
        assert rid > 0
        return rid

    def result(self, srv, i, rid):
        import torch
        torch.cuda.synchronize()
        kind, t, x = self.reqs[i]
        if kind == 0:
            return self.k[i].cpu().numpy().view(x.dtype), self.v[i].cpu().numpy()
        if kind == 1:
            return self.o[i].cpu().numpy().view(x.dtype)
        w = np.zeros(1, np.uint64)
        assert self.L.trtc_server_result(srv, rid, w.ctypes.data_as(ctypes.c_void_p)) == 0
        return w.view(np.uint8)[: x.dtype.itemsize].view(x.dtype)[0]


def drain(L, srv):
    while True:
        left = L.trtc_server_poll(srv)
        assert left >= 0
        if left == 0:
            return


def check_oracle(kind, x, got):
    if kind == 0:
        ek, ev = O.sort_by_key(x, np.arange(len(x), dtype=np.int32))
        assert got[0].tobytes() == ek.tobytes() and np.array_equal(got[1], ev)
    elif kind == 1:
        if x.dtype == np.float32:
            exp = O.scan_f64(x, exclusive=True, init=0.0)
            mag = np.concatenate([[0.0], np.cumsum(np.abs(x.astype(np.float64)))[:-1]])
            assert np.all(np.abs(got.astype(np.float64) - exp) <= REL_TOL * mag + 1e-30)
        else:
            assert np.array_equal(got, O.scan(x, exclusive=True, init=0))
    else:
        if x.dtype == np.float32:
            ref = O.reduce_f64(x)
            assert abs(float(got) - ref) <= REL_TOL * float(np.abs(x.astype(np.float64)).sum())
        else:
            assert got == O.reduce(x)


def test_server_mix_equals_alone_and_oracle(L):
    rng = np.random.default_rng(3)
    reqs = make_requests(rng, 240, 4, 18)
    srv = L.trtc_server_create(4 << 30, 4, 1 << 16)
    assert srv
    try:
        mix = Run(L, reqs)
        ids = [mix.submit(srv, i) for i in range(len(reqs))]
        drain(L, srv)
        got_mix = [mix.result(srv, i, rid) for i, rid in enumerate(ids)]
        for (kind, _, x), g in zip(reqs, got_mix):
            check_oracle(kind, x, g)
        # the same requests served one at a time
        alone = Run(L, reqs)
        for i in range(len(reqs)):
            rid = alone.submit(srv, i)
            drain(L, srv)
            g = alone.result(srv, i, rid)
            kind, _, x = reqs[i]
            if kind == 0:
                assert g[0].tobytes() == got_mix[i][0].tobytes() and np.array_equal(g[1], got_mix[i][1])
            elif x.dtype != np.float32:
                assert np.array_equal(np.asarray(g), np.asarray(got_mix[i]))
            else:
                check_oracle(kind, x, g)
    finally:
        L.trtc_server_destroy(srv)


def test_server_admission_budget(L):
    # a budget that fits one large sort at a time still serves everything, in order
    rng = np.random.default_rng(4)
    reqs = [(0, 5, rng.integers(0, 2**32, 1 << 20, dtype=np.uint64).astype(np.uint32)) for _ in range(6)]
    srv = L.trtc_server_create(24 << 20, 4, 1 << 16)
    try:
        run = Run(L, reqs)
        ids = [run.submit(srv, i) for i in range(len(reqs))]
        drain(L, srv)
        for i, rid in enumerate(ids):
            check_oracle(0, reqs[i][2], run.result(srv, i, rid))
    finally:
        L.trtc_server_destroy(srv)


def test_server_float_sorts_with_nan(L):
    # coalesced (segmented kernel) and plain float Sort_By_Key requests holding NaNs give the
    # order of the single-request call (the reference's Min_Element rotation included)
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(120):
        n = int(2 ** rng.uniform(4, 14)) if i < 110 else int(2 ** rng.uniform(17, 19))
        x = (rng.standard_normal(n) * 3).astype(np.float32)
        add_nans(rng, x)
        if i % 5 == 0:
            x.view(np.uint32)[0] = NAN_BITS[i % 3]
        reqs.append((0, 8, x))
    srv = L.trtc_server_create(4 << 30, 4, 1 << 16)
    assert srv
    try:
        run = Run(L, reqs)
        ids = [run.submit(srv, i) for i in range(len(reqs))]
        drain(L, srv)
        for i, rid in enumerate(ids):
            check_oracle(0, reqs[i][2], run.result(srv, i, rid))
    finally:
        L.trtc_server_destroy(srv)


def test_server_refuses_request_beyond_budget(L):
    # a request whose temporaries exceed the whole budget is refused at submission (-1 and a
    # message), nothing of it runs, and the server keeps serving requests that fit
    import torch
    from thrustrtc_b200 import _native as N
    srv = L.trtc_server_create(1 << 20, 2, 1 << 12)
    assert srv
    try:
        big = torch.arange(1 << 20, dtype=torch.int32, device="cuda")
        bigv = big.clone()
        p = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
        assert L.trtc_server_submit(srv, 0, 5, p(big), p(bigv), None, 1 << 20) == -1
        assert "budget" in N.last_error()
        torch.cuda.synchronize()
        assert torch.equal(big, bigv)
        rng = np.random.default_rng(6)
        reqs = [(0, 5, rng.integers(0, 2**32, 3000, dtype=np.uint64).astype(np.uint32))]
        run = Run(L, reqs)
        rid = run.submit(srv, 0)
        drain(L, srv)
        check_oracle(0, reqs[0][2], run.result(srv, 0, rid))
    finally:
        L.trtc_server_destroy(srv)
