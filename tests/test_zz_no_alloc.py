"""trtc_raw_scan_noalloc (include/trtc_raw.h) against trtc_raw_scan, through the C ABI.

Named to be collected last, so that it also runs after every other test has used the
library on the same device; it passes alone as well.  Integer scans must match exactly;
float scans within a relative 1e-5 (both entry points run the same kernel and tiling).
"""
import ctypes

import numpy as np
import pytest

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


CASES = [  # (type code, torch dtype, numpy dtype, op, exclusive, n)
    (4, "int32", np.int32, 0, 0, 1),
    (4, "int32", np.int32, 0, 0, 4097),
    (4, "int32", np.int32, 0, 1, 1_000_003),
    (5, "int32", np.uint32, 1, 0, 300_001),
    (4, "int32", np.int32, 2, 1, 65_536),
    (8, "float32", np.float32, 0, 0, 1_048_577),
    (8, "float32", np.float32, 1, 1, 77_777),
]


@pytest.mark.parametrize("tc,tdt,ndt,op,excl,n", CASES)
def test_noalloc_matches_scan_twice(lib, tc, tdt, ndt, op, excl, n):
    import torch
    rng = np.random.default_rng(n + 17 * op + excl)
    if ndt == np.float32:
        x = rng.random(n).astype(np.float32)
        init = np.array([0.25], np.float32)
    else:
        x = rng.integers(-1000, 1001, n).astype(ndt)
        init = np.array([7], ndt)
    xin = torch.from_numpy(x.view(np.int32) if ndt == np.uint32 else x).cuda()
    ref = torch.empty_like(xin)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    ini = init.ctypes.data_as(ctypes.c_void_p) if excl else None
    assert lib.trtc_raw_scan(tc, op, excl, _p(xin), _p(ref), n, ini, None) == 0
    expect = ref.cpu().numpy().view(ndt)
    for _ in range(2):  # two calls in a row reuse the same static scratch
        out = torch.full_like(xin, -1)
        assert lib.trtc_raw_scan_noalloc(tc, op, excl, _p(xin), _p(out), n, ini, _p(status), None) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(ndt)
        if ndt == np.float32:
            den = np.maximum(np.abs(expect.astype(np.float64)), 1e-30)
            assert np.max(np.abs(got.astype(np.float64) - expect) / den) <= REL_TOL
        else:
            assert np.array_equal(got, expect)
        assert int(status.item()) == 0


def test_noalloc_in_place(lib):
    import torch
    n = 123_457
    x = torch.randint(-5, 6, (n,), dtype=torch.int32, device="cuda")
    ref = torch.cumsum(x.to(torch.int64), 0).to(torch.int32)
    assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(x), _p(x), n, None, None, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(x, ref)


def test_noalloc_rejects_beyond_max(lib):
    import torch
    from thrustrtc_b200 import _native as N
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    # rejected on the host before any launch: the buffer is never touched
    assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(buf), _p(buf), MAX_N + 1, None, None, None) == -1
    assert "exceeds the maximum of 268435456" in N.last_error()
    assert lib.trtc_raw_scan_noalloc(6, 0, 0, _p(buf), _p(buf), 16, None, None, None) == -1
    assert lib.trtc_raw_scan_noalloc(4, 0, 0, _p(buf), _p(buf), 0, None, None, None) == -1
    torch.cuda.synchronize()
    assert int(buf.abs().sum()) == 0
