"""Seeded hot-path cases run through a ThrustRTC-shaped Python API.

``run_all(T)`` takes a module with the reference package's API (``import ThrustRTC`` over the
reference's own library, or ``thrustrtc_b200``) and returns ``{name: ndarray}`` with every
case's inputs (``<case>/in_*``) and outputs (``<case>/out_*``).  tests/golden/make_ref_fixtures.py
runs it against the reference on a GPU and stores the result as ref_fixtures.npz; the tests
compare the oracle (CPU) and this library (GPU) with those stored outputs.

Sizes are chosen so that every case spans several tiles of the library's kernels (tiles of
4096-8192 elements) and ragged last tiles, while the fixture file stays small.
"""
import zlib

import numpy as np

F32_NAN = np.uint32(0x7FC00000)
F32_NNAN = np.uint32(0xFFC00000)
F32_NAN_PAYLOAD = np.uint32(0x7FC00123)
F64_NAN = np.uint64(0x7FF8000000000000)
F64_NNAN = np.uint64(0xFFF8000000000000)


def float_keys(n, seed, nan_at_0=None, dtype=np.float32):
    """N(0,1) keys with 1 % -0.0, 1 % +0.0, 0.2 % NaN (+, -, payload), 10 % duplicates."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n).astype(dtype)
    u = rng.random(n)
    x[u < 0.01] = -0.0
    x[(u >= 0.01) & (u < 0.02)] = 0.0
    x[(u >= 0.02) & (u < 0.12)] = x[rng.integers(0, n, int(((u >= 0.02) & (u < 0.12)).sum()))]
    bits = x.view(np.uint32 if dtype == np.float32 else np.uint64)
    nan_pos = rng.choice(n, max(3, n // 500), replace=False)
    if dtype == np.float32:
        pats = np.array([F32_NAN, F32_NNAN, F32_NAN_PAYLOAD], dtype=np.uint32)
    else:
        pats = np.array([F64_NAN, F64_NNAN, F64_NAN | np.uint64(0x123)], dtype=np.uint64)
    bits[nan_pos] = pats[np.arange(len(nan_pos)) % 3]
    if nan_at_0 == "+":
        bits[0] = pats[0]
    elif nan_at_0 == "-":
        bits[0] = pats[1]
    elif nan_at_0 == "none":
        # NaN-free first 256-block: the tree's first round cannot absorb at slot 0
        bad = np.isnan(x[:256])
        x[:256][bad] = 0.5
    return x


def runs(n, seed, mean=8):
    """int32 keys in runs of geometric length (segment ids), for scan/reduce/unique by key."""
    rng = np.random.default_rng(seed)
    lens = rng.geometric(1.0 / mean, n)
    ids = np.repeat(np.arange(len(lens), dtype=np.int64), lens)[:n]
    return (ids * 7 % 1000).astype(np.int32)  # adjacent runs always differ (7 and 1000 coprime)


def _dv(T, a):
    return T.device_vector_from_numpy(np.ascontiguousarray(a))


def _host(v, n=None):
    return v.to_host() if n is None else v.to_host(0, n)


def case_sort(T, out):
    specs = [
        ("sbk_u32_i32", np.uint32, 20001, None),
        ("sbk_u32_i32_desc", np.uint32, 20001, "Greater"),
        ("sbk_i32_i32", np.int32, 12345, None),
        ("sbk_i64_i32", np.int64, 12001, None),
        ("sbk_i64_i32_desc", np.int64, 12001, "Greater"),
        ("sbk_u8_i32", np.uint8, 9000, None),
        ("sbk_i16_i32", np.int16, 9000, None),
    ]
    for name, dt, n, comp in specs:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        if dt == np.int64:
            k = (0x0123456700000000 + rng.integers(0, 1 << 20, n)).astype(np.int64)
            k[::3] = -k[::3]
        else:
            info = np.iinfo(dt)
            k = rng.integers(int(info.min), int(info.max) + 1, n, dtype=np.int64).astype(dt)
        v = np.arange(n, dtype=np.int32)
        dk, dv = _dv(T, k), _dv(T, v)
        T.Sort_By_Key(dk, dv, T.Greater() if comp else None)
        out[name + "/in_keys"] = k
        out[name + "/out_keys"] = _host(dk)
        out[name + "/out_values"] = _host(dv)


def case_float_sort(T, out):
    for dt, tag, n in ((np.float32, "f32", 12001), (np.float64, "f64", 7001)):
        for nan0 in ("none", "+", "-", None):
            for desc in (False, True):
                name = "fsort_%s_nan0%s_%s" % (tag, {"none": "no", "+": "pos", "-": "neg", None: "rnd"}[nan0],
                                               "desc" if desc else "asc")
                k = float_keys(n, 11 + len(name), nan0, dt)
                v = np.arange(n, dtype=np.int32)
                dk, dv = _dv(T, k), _dv(T, v)
                T.Sort_By_Key(dk, dv, T.Greater() if desc else None)
                out[name + "/in_keys"] = k
                out[name + "/out_keys"] = _host(dk)
                out[name + "/out_values"] = _host(dv)
                # keys-only form
                dk2 = _dv(T, k)
                T.Sort(dk2, T.Greater() if desc else None)
                out[name + "/out_sort"] = _host(dk2)
        # Min_Element over NaN-bearing keys (the index the sort offsets by)
        k = float_keys(n, 99, "+" if tag == "f32" else None, dt)
        out["minel_%s/in" % tag] = k
        out["minel_%s/out" % tag] = np.array([T.Min_Element(_dv(T, k))], dtype=np.int64)


def case_scans(T, out):
    n = 30001
    rng = np.random.default_rng(5)
    x = rng.integers(-1000, 1001, n).astype(np.int32)
    d = _dv(T, x)
    o = T.device_vector("int32_t", n)
    T.Inclusive_Scan(d, o)
    out["scan_i32/in"] = x
    out["scan_i32/out_incl"] = _host(o)
    T.Exclusive_Scan(d, o, T.DVInt32(7))
    out["scan_i32/out_excl_init7"] = _host(o)
    T.Inclusive_Scan(d, o, T.Maximum())
    out["scan_i32/out_incl_max"] = _host(o)
    neg = T.Negate()
    T.Transform_Inclusive_Scan(d, o, neg, T.Plus())
    out["scan_i32/out_tincl_neg"] = _host(o)
    T.Transform_Exclusive_Scan(d, o, neg, T.DVInt32(3), T.Plus())
    out["scan_i32/out_texcl_neg_init3"] = _host(o)
    # in place
    d2 = _dv(T, x)
    T.Exclusive_Scan(d2, d2)
    out["scan_i32/out_excl_inplace"] = _host(d2)


def case_scan_by_key(T, out):
    n = 30001
    k = runs(n, 3, mean=24)
    rng = np.random.default_rng(6)
    vi = rng.integers(-50, 51, n).astype(np.int32)
    dk, dv = _dv(T, k), _dv(T, vi)
    o = T.device_vector("int32_t", n)
    T.Inclusive_Scan_By_Key(dk, dv, o)
    out["sbk_scan/in_keys"] = k
    out["sbk_scan/in_values"] = vi
    out["sbk_scan/out_incl"] = _host(o)
    T.Exclusive_Scan_By_Key(dk, dv, o)
    out["sbk_scan/out_excl"] = _host(o)
    T.Exclusive_Scan_By_Key(dk, dv, o, T.DVInt32(5))
    out["sbk_scan/out_excl_init5"] = _host(o)
    T.Inclusive_Scan_By_Key(dk, dv, o, T.EqualTo(), T.Maximum())
    out["sbk_scan/out_incl_max"] = _host(o)
    # float values (tolerance case: the reference's association order is its own)
    vf = rng.random(n).astype(np.float32)
    of = T.device_vector("float", n)
    T.Inclusive_Scan_By_Key(dk, _dv(T, vf), of)
    out["sbk_scan/in_values_f32"] = vf
    out["sbk_scan/out_incl_f32"] = _host(of)


def _is_even(T):
    return T.Functor({}, ["x"], "\n         return x % 2 == 0;\n")


def case_compaction(T, out):
    even = _is_even(T)
    for sel_name, seed, mod in (("half", 7, None), ("all", 8, "even"), ("none", 9, "odd")):
        n = 20001
        rng = np.random.default_rng(seed)
        x = rng.integers(-10**6, 10**6, n).astype(np.int32)
        if mod == "even":
            x &= ~np.int32(1)
        elif mod == "odd":
            x |= np.int32(1)
        st = rng.integers(0, 4, n).astype(np.int32)
        p = "cmp_%s/" % sel_name
        out[p + "in"] = x
        out[p + "stencil"] = st
        o = T.device_vector("int32_t", n)
        c = T.Copy_If(_dv(T, x), o, even)
        out[p + "copy_if"] = _host(o, c) if c else np.zeros(0, np.int32)
        c = T.Copy_If_Stencil(_dv(T, x), _dv(T, st), o, even)
        out[p + "copy_if_stencil"] = _host(o, c) if c else np.zeros(0, np.int32)
        d = _dv(T, x)
        T.Partition(d, even)
        out[p + "partition"] = _host(d)
        d = _dv(T, x)
        T.Partition_Stencil(d, _dv(T, st), even)
        out[p + "partition_stencil"] = _host(d)
        ot, of = T.device_vector("int32_t", n), T.device_vector("int32_t", n)
        c = T.Partition_Copy(_dv(T, x), ot, of, even)
        out[p + "partition_copy_t"] = _host(ot, c) if c else np.zeros(0, np.int32)
        out[p + "partition_copy_f"] = _host(of, n - c) if n - c else np.zeros(0, np.int32)
        c = T.Partition_Copy_Stencil(_dv(T, x), _dv(T, st), ot, of, even)
        out[p + "partition_copy_stencil_t"] = _host(ot, c) if c else np.zeros(0, np.int32)
        out[p + "partition_copy_stencil_f"] = _host(of, n - c) if n - c else np.zeros(0, np.int32)
        d = _dv(T, x)
        c = T.Remove_If(d, even)
        out[p + "remove_if"] = _host(d, c) if c else np.zeros(0, np.int32)
        c = T.Remove_Copy_If(_dv(T, x), o, even)
        out[p + "remove_copy_if"] = _host(o, c) if c else np.zeros(0, np.int32)
        d = _dv(T, x)
        c = T.Remove_If_Stencil(d, _dv(T, st), even)
        out[p + "remove_if_stencil"] = _host(d, c) if c else np.zeros(0, np.int32)
        c = T.Remove_Copy_If_Stencil(_dv(T, x), _dv(T, st), o, even)
        out[p + "remove_copy_if_stencil"] = _host(o, c) if c else np.zeros(0, np.int32)
    # Remove / Remove_Copy of a value; Unique forms over runs
    n = 20001
    rng = np.random.default_rng(10)
    x = rng.integers(0, 5, n).astype(np.int32)
    out["rm/in"] = x
    d = _dv(T, x)
    c = T.Remove(d, T.DVInt32(3))
    out["rm/remove3"] = _host(d, c)
    o = T.device_vector("int32_t", n)
    c = T.Remove_Copy(_dv(T, x), o, T.DVInt32(0))
    out["rm/remove_copy0"] = _host(o, c)
    k = runs(n, 12, mean=6)
    v = np.arange(n, dtype=np.int32)
    out["uq/in_keys"] = k
    d = _dv(T, k)
    c = T.Unique(d)
    out["uq/unique"] = _host(d, c)
    c = T.Unique_Copy(_dv(T, k), o)
    out["uq/unique_copy"] = _host(o, c)
    dk, dv = _dv(T, k), _dv(T, v)
    c = T.Unique_By_Key(dk, dv)
    out["uq/ubk_keys"] = _host(dk, c)
    out["uq/ubk_values"] = _host(dv, c)
    ok, ov = T.device_vector("int32_t", n), T.device_vector("int32_t", n)
    c = T.Unique_By_Key_Copy(_dv(T, k), _dv(T, v), ok, ov)
    out["uq/ubkc_keys"] = _host(ok, c)
    out["uq/ubkc_values"] = _host(ov, c)


def case_reduce(T, out):
    n = 20001
    k = runs(n, 13, mean=10)
    rng = np.random.default_rng(14)
    v = rng.integers(-100, 101, n).astype(np.int32)
    ok, ov = T.device_vector("int32_t", n), T.device_vector("int32_t", n)
    c = T.Reduce_By_Key(_dv(T, k), _dv(T, v), ok, ov)
    out["rbk/in_keys"] = k
    out["rbk/in_values"] = v
    out["rbk/out_keys"] = _host(ok, c)
    out["rbk/out_values"] = _host(ov, c)
    c = T.Reduce_By_Key(_dv(T, k), _dv(T, v), ok, ov, T.EqualTo(), T.Maximum())
    out["rbk/out_keys_max"] = _host(ok, c)
    out["rbk/out_values_max"] = _host(ov, c)
    x = rng.integers(-1000, 1001, 30001).astype(np.int32)
    out["red/in_i32"] = x
    out["red/sum_i32"] = np.array([T.Reduce(_dv(T, x))], dtype=np.int64)
    out["red/max_i32"] = np.array([T.Reduce(_dv(T, x), T.DVInt32(-5000), T.Maximum())], dtype=np.int64)
    f = rng.random(30001).astype(np.float32)
    out["red/in_f32"] = f
    out["red/sum_f32"] = np.array([T.Reduce(_dv(T, f))], dtype=np.float64)


# Crafted keys around the NaN / zero / denormal / infinity boundaries of both float widths:
# every sign of NaN (quiet, signalling, payloads, all-ones), the zeros, the smallest
# denormals, the normal boundary and the infinities, each sorted with its index as payload.
# -inf sits at index 0 and nothing is below it, so the Min_Element tree selects it and the
# order is the key map's own.
F64_EDGE = [0xFFF0000000000000, 0x0000000000000000, 0x8000000000000000, 0xFFF8000000000000, 0x0000000000000001,
            0x8000000000000001, 0x0008000000000000, 0x8008000000000000, 0x0007FFFFFFFFFFFF, 0x0010000000000000,
            0xFFF8000000000123, 0x7FF8000000000000, 0x3FF0000000000000, 0xBFF0000000000000, 0xFFF0000000000001,
            0x7FF0000000000001, 0xFFFFFFFFFFFFFFFF, 0x7FFFFFFFFFFFFFFF, 0x7FF0000000000000, 0x4000000000000000,
            0xC000000000000000, 0xFFF4000000000000, 0x000FFFFFFFFFFFFF, 0x800FFFFFFFFFFFFF]
F32_EDGE = [0xFF800000, 0x00000000, 0x80000000, 0xFFC00000, 0x00000001, 0x80000001, 0x00400000, 0x80400000,
            0x007FFFFF, 0x00800000, 0xFFC00123, 0x7FC00000, 0x3F800000, 0xBF800000, 0xFF800001, 0x7F800001,
            0xFFFFFFFF, 0x7FFFFFFF, 0x7F800000, 0x40000000, 0xC0000000, 0xFFA00000, 0x007FFFFE, 0x807FFFFF]


def case_float_edges(T, out):
    for tag, dt, bits_dt, pats in (("f64", np.float64, np.uint64, F64_EDGE), ("f32", np.float32, np.uint32, F32_EDGE)):
        k = np.array(pats, dtype=bits_dt).view(dt)
        k = np.concatenate([k[:1], np.tile(k[1:], 3)])  # each edge value three times: stability
        v = np.arange(len(k), dtype=np.int32)
        for desc in (False, True):
            name = "fedge_%s_%s" % (tag, "desc" if desc else "asc")
            dk, dv = _dv(T, k), _dv(T, v)
            T.Sort_By_Key(dk, dv, T.Greater() if desc else None)
            out[name + "/in_keys"] = k
            out[name + "/out_keys"] = _host(dk)
            out[name + "/out_values"] = _host(dv)


CASES = [case_sort, case_float_sort, case_scans, case_scan_by_key, case_compaction, case_reduce, case_float_edges]

# Reference behaviour that this library does not reproduce on purpose (each one documented):
# n_unique_by_key_copy passes values_in as the keys output (python/api_Reordering.cpp:120), so
# through the reference's C ABI Unique_By_Key_Copy leaves keys_out untouched and overwrites
# values_in; this library writes keys_out, as the reference's C++ TRTC_Unique_By_Key_Copy does.
ABI_DEVIATIONS = ("uq/ubkc_",)


def run_all(T):
    out = {}
    for c in CASES:
        c(T, out)
    return out


# ---------------------------------------------------------------- fixture storage
# Inputs are regenerated from their seeds and stored as (crc32, length) only; outputs are
# stored in full, except sorted keys, which equal in_keys[out_values] (values = index) and
# are stored as (crc32, length) too.  Float outputs of scans and reductions are compared
# within a relative tolerance (the reference's association order is its own).

TOLERANCE_KEYS = ("sbk_scan/out_incl_f32", "red/sum_f32")
REL_TOL = 1e-5


def _crc(a):
    return zlib.crc32(np.ascontiguousarray(a).tobytes())


def _crc_only(name, res):
    last = name.split("/")[-1]
    if last.startswith("in") or last == "stencil":
        return True
    if name.startswith(("sbk_", "fsort_")) and last in ("out_keys", "out_sort"):
        case = name.rsplit("/", 1)[0]
        perm = res.get(case + "/out_values")
        keys = res.get(case + "/in_keys")
        if perm is None or keys is None:
            return False
        derived = np.ascontiguousarray(keys)[perm.astype(np.int64)]
        return derived.tobytes() == np.ascontiguousarray(res[name]).tobytes()
    return False


def pack(res):
    out = {}
    for k, v in res.items():
        if _crc_only(k, res):
            out["crc32:" + k] = np.array([_crc(v), len(v)], dtype=np.int64)
        else:
            out[k] = np.asarray(v)
    return out


def compare(fix, res, skip=ABI_DEVIATIONS):
    """Mismatches of `res` (run_all output) against a packed fixture, as strings."""
    bad = []
    for k in fix.files if hasattr(fix, "files") else fix.keys():
        name = k[6:] if k.startswith("crc32:") else k
        if any(name.startswith(s) for s in skip):
            continue
        if name not in res:
            bad.append("missing " + name)
            continue
        got = np.asarray(res[name])
        want = fix[k]
        if k.startswith("crc32:"):
            if len(got) != int(want[1]) or _crc(got) != int(want[0]):
                bad.append("crc " + name)
        elif name in TOLERANCE_KEYS:
            w = want.astype(np.float64)
            g = got.astype(np.float64)
            if g.shape != w.shape or not np.all(np.abs(g - w) <= REL_TOL * np.maximum(np.abs(w), 1e-30) + 1e-6):
                bad.append("tolerance " + name)
        elif got.dtype != want.dtype and got.dtype.kind == want.dtype.kind == "i":
            if not np.array_equal(got.astype(np.int64), want.astype(np.int64)):
                bad.append("value " + name)
        elif got.shape != want.shape or got.tobytes() != want.tobytes():
            bad.append("bytes " + name)
    return bad
