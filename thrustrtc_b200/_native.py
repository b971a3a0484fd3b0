"""Loads libPyThrustRTC.so (the C ABI of thrustrtc_b200) with ctypes.

The library is built in-tree by ``thrustrtc_b200/build.py``.  There is no fallback: if the
library is missing or cannot be loaded, importing the package raises, so no CPU path can
stand in for the CUDA kernels.
"""
import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libPyThrustRTC.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("thrustrtc_b200: %s is missing; build it with `python thrustrtc_b200/build.py`" % LIB_PATH)

lib = ctypes.CDLL(LIB_PATH)

vp = ctypes.c_void_p
u64 = ctypes.c_ulonglong
i32 = ctypes.c_int
u32 = ctypes.c_uint
f32 = ctypes.c_float
f64 = ctypes.c_double
cstr = ctypes.c_char_p
i64 = ctypes.c_longlong


def _sig(name, restype, *argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


# ---- raw-pointer ABI (include/trtc_raw.h)
_sig("trtc_last_error", cstr)
_sig("trtc_launch_count", u64)
_sig("trtc_raw_sync", i32, vp)
_sig("trtc_timing_enable", None, i32)
_sig("trtc_timing_count", i32)
_sig("trtc_timing_get", i32, i32, ctypes.c_char_p, u64, ctypes.POINTER(ctypes.c_float))
_sig("trtc_raw_sort", i32, i32, vp, u64, i32, vp)
_sig("trtc_raw_sort_by_key", i32, i32, vp, vp, u64, u64, i32, vp)
_sig("trtc_raw_min_element", u64, i32, vp, u64, vp)
_sig("trtc_raw_scan", i32, i32, i32, i32, vp, vp, u64, vp, vp)
_sig("trtc_raw_reduce", i32, i32, i32, vp, u64, vp, vp, vp)
_sig("trtc_raw_reduce_async", i32, i32, i32, vp, u64, vp, ctypes.POINTER(vp), vp)
_sig("trtc_raw_scan_by_key", i32, i32, i32, i32, vp, vp, vp, u64, vp, vp)
_sig("trtc_raw_remove_copy", u64, i32, vp, vp, u64, vp, vp)
_sig("trtc_raw_unique_copy", u64, i32, vp, vp, u64, vp)

TYPE_CODES = {
    "int8_t": 0, "uint8_t": 1, "int16_t": 2, "uint16_t": 3, "int32_t": 4, "uint32_t": 5,
    "int64_t": 6, "uint64_t": 7, "float": 8, "double": 9,
}
OP_CODES = {"Plus": 0, "Maximum": 1, "Minimum": 2}


def last_error():
    e = lib.trtc_last_error()
    return e.decode() if e else ""


def launch_count():
    """Number of thrustrtc_b200 kernels launched by this process so far."""
    return int(lib.trtc_launch_count())


def timing_enable(on=True):
    """Starts (or stops) recording the device time of every launch of this library."""
    lib.trtc_timing_enable(1 if on else 0)


def timing_records():
    """[(kernel name, ms)] of the launches recorded since timing_enable(); synchronises."""
    c = lib.trtc_timing_count()
    if c < 0:
        raise RuntimeError("timing: " + last_error())
    out = []
    buf = ctypes.create_string_buffer(256)
    ms = ctypes.c_float()
    for i in range(c):
        if lib.trtc_timing_get(i, buf, 256, ctypes.byref(ms)) == 0:
            out.append((buf.value.decode(), ms.value))
    return out
