"""Failure paths, made on purpose without faulting, trapping or hanging the GPU.

* A bounded look-back wait that runs out: a test build of the two-phase scan in which one
  tile never publishes (trtc_test_scan_lookback_timeout).  The call must report the expired
  wait, and the next calls on the same stream must succeed with correct results.
* An allocation above the library's cap (trtc_set_alloc_limit): the op fails the way the
  reference's does when its cuMemAlloc fails (false / -1 / SystemError, DVVector.cpp:5-25,
  internal/general_copy_if.cpp:30-33), before any kernel runs, so its inputs are untouched.
* A user Functor that does not compile: NVRTC's error becomes SystemError and the log is
  available through trtc_last_error(); the library keeps working.
(A server request larger than the server's budget is refused in tests/test_server_gpu.py.)
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trtc(cuda):
    import thrustrtc_b200 as t
    from thrustrtc_b200 import _native as N
    t.init()
    N.lib.trtc_test_scan_lookback_timeout.restype = ctypes.c_int
    N.lib.trtc_test_scan_lookback_timeout.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong,
                                                      ctypes.c_void_p]
    N.lib.trtc_set_alloc_limit.restype = None
    N.lib.trtc_set_alloc_limit.argtypes = [ctypes.c_ulonglong]
    return t


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_lookback_wait_runs_out_and_the_next_call_succeeds(trtc):
    import torch
    from thrustrtc_b200 import _native as N
    n = (1 << 20) + 3
    x = torch.randint(-1000, 1001, (n,), dtype=torch.int32, device="cuda")
    out = torch.zeros_like(x)
    for _ in range(2):
        assert N.lib.trtc_test_scan_lookback_timeout(_p(x), _p(out), n, None) == -1
        assert "look-back wait exceeded its bound" in N.last_error()
        # the same stream and workspace serve the next scans correctly
        assert N.lib.trtc_raw_scan(4, 0, 0, _p(x), _p(out), n, None, None) == 0
        assert N.lib.trtc_raw_sync(None) == 0
        assert np.array_equal(out.cpu().numpy(), O.scan(x.cpu().numpy()))
    # a sort on the same stream after the failure
    k = torch.randint(-2**31, 2**31 - 1, (n,), dtype=torch.int32, device="cuda")
    k0 = k.cpu().numpy()
    assert N.lib.trtc_raw_sort(4, _p(k), n, 0, None) == 0
    assert N.lib.trtc_raw_sync(None) == 0
    assert np.array_equal(k.cpu().numpy(), O.sort(k0))


def test_allocation_above_the_cap_fails_cleanly(trtc):
    from thrustrtc_b200 import _native as N
    n = 1 << 20
    rng = np.random.default_rng(2)
    keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.int32)
    dk = trtc.device_vector_from_numpy(keys)
    dv = trtc.device_vector_from_numpy(vals)
    N.lib.trtc_set_alloc_limit(1 << 20)  # the sort's temporaries need 4 MiB each
    try:
        with pytest.raises(SystemError):
            trtc.Sort_By_Key(dk, dv)
        assert "exceeds the limit" in N.last_error()
        assert dk.to_host().tobytes() == keys.tobytes() and dv.to_host().tobytes() == vals.tobytes()
        with pytest.raises(SystemError):  # DVVector storage above the cap: NULL handle
            trtc.device_vector("int32_t", n)
        small = trtc.device_vector_from_numpy(keys[:1000].copy())
        trtc.Sort(small)  # fits under the cap
        assert small.to_host().tobytes() == O.sort(keys[:1000]).tobytes()
    finally:
        N.lib.trtc_set_alloc_limit(0)
    trtc.Sort_By_Key(dk, dv)
    ek, ev = O.sort_by_key(keys, vals)
    assert dk.to_host().tobytes() == ek.tobytes() and dv.to_host().tobytes() == ev.tobytes()


def test_malformed_functor_raises_systemerror_with_the_nvrtc_log(trtc):
    from thrustrtc_b200 import _native as N
    x = np.arange(100, dtype=np.int32)
    d = trtc.device_vector_from_numpy(x)
    out = trtc.device_vector("int32_t", 100)
    bad = trtc.Functor({}, ["x"], "        return x +* ;\n")
    with pytest.raises(SystemError):
        trtc.Copy_If(d, out, bad)
    assert "NVRTC compilation failed" in N.last_error() and "error" in N.last_error()
    good = trtc.Functor({}, ["x"], "        return x % 3 == 0;\n")
    c = trtc.Copy_If(d, out, good)
    assert out.to_host(0, c).tolist() == x[x % 3 == 0].tolist()
