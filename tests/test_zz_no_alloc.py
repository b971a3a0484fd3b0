"""trtc_raw_scan_noalloc (include/trtc_raw.h), the scan entry point that allocates nothing.

It exists for callers that cannot allocate device memory while they run: code inside a
memory-pool or allocator callback (an allocation there would re-enter the allocator), a
framework that has reserved the device's memory for its own allocator up front (a cudaMalloc
would fail), or a real-time loop that must not take cudaMalloc's device-wide synchronisation.  Its look-back scratch is a fixed array in the
library's static device memory, so it accepts 4-byte element types and n <= 2^28 only.

Checked through the C ABI against the existing entry point trtc_raw_scan (integer scans
bit-identical, float scans within REL_TOL: both run the same two-phase kernel, but a float
look-back may add tile totals in a different grouping from one run to the next) and against
the oracle, on two calls in a row that share the static scratch.  The file is named to be
collected last, so that a run stopping at the first failure has run every other test first;
it passes alone too.  TRTC_NOALLOC_EPOCH_LIMIT (read once, at the entry point's first call in
the process) makes the scratch's epoch wrap every few calls, so the clear-on-wrap path runs
here as well.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

os.environ.setdefault("TRTC_NOALLOC_EPOCH_LIMIT", "5")

pytestmark = pytest.mark.gpu
REL_TOL = 1e-5
MAX_N = 1 << 28


@pytest.fixture(scope="module")
def lib(cuda):
    from thrustrtc_b200 import _native as N
    L = N.lib
    L.trtc_raw_scan_noalloc.restype = ctypes.c_int
    L.trtc_raw_scan_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return L


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


OPS = {0: "Plus", 1: "Maximum", 2: "Minimum"}
CASES = [  # (type code, numpy dtype, op, exclusive, n)
    (4, np.int32, 0, 0, 1),
    (4, np.int32, 0, 0, 8193),
    (4, np.int32, 0, 1, 1_000_003),
    (5, np.uint32, 1, 0, 300_001),
    (4, np.int32, 2, 1, 65_536),
    (8, np.float32, 0, 0, 1_048_577),
    (8, np.float32, 1, 1, 77_777),
    (8, np.float32, 0, 1, 200_000),
]


def _input(rng, ndt, n):
    if ndt == np.float32:
        return rng.random(n).astype(np.float32) - np.float32(0.25), np.array([0.25], np.float32)
    return rng.integers(-1000, 1001, n).astype(ndt), np.array([7], ndt)


def _check_float(got, ref64, terms, init=0.0):
    # FP32 accumulation bound: REL_TOL times the running sum of the magnitudes (init included)
    mag = np.maximum(abs(init) + np.cumsum(np.abs(terms.astype(np.float64))), 1e-30)
    assert np.all(np.abs(got.astype(np.float64) - ref64) <= REL_TOL * mag)


@pytest.mark.parametrize("tc,ndt,op,excl,n", CASES)
def test_noalloc_matches_scan_and_oracle_twice(lib, tc, ndt, op, excl, n):
    import torch
    rng = np.random.default_rng(n + 17 * op + excl)
    x, init = _input(rng, ndt, n)
    xin = torch.from_numpy(x.view(np.int32)).cuda()
    ref = torch.empty_like(xin)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    ini = init.ctypes.data_as(ctypes.c_void_p) if excl else None
    assert lib.trtc_raw_scan(tc, op, excl, _p(xin), _p(ref), n, ini, None) == 0
    existing = ref.cpu().numpy().view(ndt)
    for _ in range(2):  # two calls in a row reuse the same static scratch
        out = torch.full_like(xin, -1)
        assert lib.trtc_raw_scan_noalloc(tc, op, excl, _p(xin), _p(out), n, ini, _p(status), None) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(ndt)
        assert int(status.item()) == 0
        if ndt == np.float32:
            if op == 0:
                ref64 = O.scan_f64(x, exclusive=bool(excl), init=float(init[0]) if excl else None)
                i0 = float(init[0]) if excl else 0.0
                _check_float(got, ref64, x, i0)
                _check_float(existing, ref64, x, i0)
                _check_float(got, existing.astype(np.float64), x, i0)
            else:  # Maximum / Minimum select elements: exact
                assert got.tobytes() == O.scan(x, OPS[op], bool(excl), init[0] if excl else None).tobytes()
                assert got.tobytes() == existing.tobytes()
        else:
            assert np.array_equal(got, existing)
            assert got.tobytes() == O.scan(x, OPS[op], bool(excl), init[0] if excl else None).tobytes()


@pytest.mark.parametrize("excl", [0, 1])
def test_noalloc_in_place(lib, excl):
    import torch
    n = 123_457
    x = torch.randint(-5, 6, (n,), dtype=torch.int32, device="cuda")
    x0 = x.cpu().numpy()
    init = np.array([-3], np.int32)
    ini = init.ctypes.data_as(ctypes.c_void_p) if excl else None
    for _ in range(2):
        y = torch.from_numpy(x0).cuda()
        assert lib.trtc_raw_scan_noalloc(4, 0, excl, _p(y), _p(y), n, ini, None, None) == 0
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == O.scan(x0, "Plus", bool(excl), -3 if excl else None).tobytes()


def test_noalloc_allocates_nothing_and_wraps_its_epoch(lib):
    # after a first call (one-time set-up), calls leave the device's free memory unchanged;
    # twelve calls in a row cross the shortened epoch wrap (and its clear) twice
    import torch
    n = 2_000_003
    x = torch.randint(-1000, 1001, (n,), dtype=torch.int32, device="cuda")
    out = torch.empty_like(x)
    expect = O.scan(x.cpu().numpy())
    assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(x), _p(out), n, None, None, None) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(12):
        out.fill_(-1)
        assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(x), _p(out), n, None, None, None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), expect)
    assert torch.cuda.mem_get_info()[0] == free0


@pytest.mark.parametrize("n", [MAX_N - 1, MAX_N])
def test_noalloc_largest_sizes(lib, n):
    # n = 2^28 fills every slot of the scratch; 2^28 - 1 leaves the last tile partial
    import torch
    x = torch.randint(-1000, 1001, (n,), dtype=torch.int32, device="cuda")
    ref = torch.empty_like(x)
    assert lib.trtc_raw_scan(4, 0, 0, _p(x), _p(ref), n, None, None) == 0
    for _ in range(2):
        out = torch.full_like(x, -1)
        assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(x), _p(out), n, None, None, None) == 0
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    # and against an independent int64 cumulative sum, wrapped to int32
    wrapped = torch.cumsum(x.to(torch.int64), 0).remainder_(1 << 32)
    wrapped = torch.where(wrapped >= (1 << 31), wrapped - (1 << 32), wrapped).to(torch.int32)
    assert torch.equal(out, wrapped)


def test_noalloc_rejects_beyond_max(lib):
    import torch
    from thrustrtc_b200 import _native as N
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    # rejected on the host before any launch: the buffer is never touched
    assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(buf), _p(buf), MAX_N + 1, None, None, None) == -1
    assert "exceeds the maximum of 268435456" in N.last_error()
    assert lib.trtc_raw_scan_noalloc(6, 0, 0, _p(buf), _p(buf), 16, None, None, None) == -1
    assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(buf), _p(buf), 0, None, None, None) == -1
    assert lib.trtc_raw_scan_noalloc(4, 3, 0, _p(buf), _p(buf), 16, None, None, None) == -1
    torch.cuda.synchronize()
    assert int(buf.abs().sum()) == 0
