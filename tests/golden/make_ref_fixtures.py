"""Runs the reference ThrustRTC (built by oracle/build_ref.py) on a GPU and records its outputs.

Test infrastructure: the outputs become committed fixtures that pin the oracle and the
library's kernels to what the reference itself computes.

    python tests/golden/make_ref_fixtures.py --out DIR [--fixtures] [--printouts] [--timing]

writes, under DIR:
* ``ref_fixtures.npz``: every case of tests/golden/ref_cases.py (inputs and the reference's
  outputs), run through the reference's own, unmodified Python package;
* ``ref_keymap_probe.json``: the reference's key maps (d_u64 / d_u32) evaluated on the GPU on
  the edge bit patterns of ref_cases, and those patterns after the reference's TRTC_Copy;
* ``ref_printouts.json``: the stdout of the reference's hot-path Python test programs
  (python/test/*.py, copied to oracle/_ref/python_test by the build recipe), run against
  the reference's library, and ``ours_printouts.json`` against this repository's library
  under the same unmodified package;
* ``ref_timing.json``: the reference timed on the benchmark workloads (seconds per call,
  wall clock around the call with ``Wait()`` before and after, after one warm-up call that
  absorbs the NVRTC compilations).

Each part runs in a child process whose LD_LIBRARY_PATH holds a ``libcuda.so`` link (the
reference dlopens that exact name) and whose sys.path holds the package.
"""
import argparse
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def _env(ours=False):
    from oracle import build_ref
    pkg = build_ref.package_dir(ours)
    if pkg is None:
        raise SystemExit("oracle/_ref is not built (python oracle/build_ref.py)")
    env = dict(os.environ)
    cl = build_ref.cuda_lib_dir()
    if cl:
        env["LD_LIBRARY_PATH"] = cl + (":" + env["LD_LIBRARY_PATH"] if env.get("LD_LIBRARY_PATH") else "")
    env["PYTHONPATH"] = pkg + (":" + env["PYTHONPATH"] if env.get("PYTHONPATH") else "")
    return env


def _child(mode, out):
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--worker", mode, "--out", out],
                       env=_env(), timeout=3000)
    if r.returncode:
        raise SystemExit("%s worker failed (%d)" % (mode, r.returncode))


def worker_fixtures(out):
    import numpy as np
    import ThrustRTC as T
    sys.path.insert(0, HERE)
    import ref_cases
    res = ref_cases.run_all(T)
    np.savez_compressed(os.path.join(out, "ref_fixtures.npz"), **ref_cases.pack(res))
    print("fixtures: %d arrays" % len(res))


def worker_probe(out):
    """The reference's key maps evaluated on the GPU (d_u64 / d_u32 of built_in.h, called from a
    TRTC_For kernel) on the edge bit patterns of ref_cases, and the same patterns after the
    reference's TRTC_Copy: the key the reference's radix sort actually orders by."""
    import numpy as np
    import ThrustRTC as T
    sys.path.insert(0, HERE)
    import ref_cases
    res = {}
    for tag, dt, bdt, pats, fn, cls in (("f64", np.float64, np.uint64, ref_cases.F64_EDGE, "d_u64", "uint64_t"),
                                        ("f32", np.float32, np.uint32, ref_cases.F32_EDGE, "d_u32", "uint32_t")):
        bits = np.array(pats, dtype=bdt)
        dk = T.device_vector_from_numpy(bits.view(dt))
        dmap = T.device_vector(cls, len(bits))
        T.For(["vin", "vout"], "idx", "        vout[idx] = %s(vin[idx]);\n" % fn).launch_n(len(bits), [dk, dmap])
        dcp = T.device_vector("double" if tag == "f64" else "float", len(bits))
        T.Copy(dk, dcp)
        copied = dcp.to_host().view(bdt)
        res[tag] = [{"bits": hex(int(b)), "key": hex(int(m)), "after_copy": hex(int(c))}
                    for b, m, c in zip(bits, dmap.to_host(), copied)]
    with open(os.path.join(out, "ref_keymap_probe.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("probe:", len(res["f64"]), "f64 and", len(res["f32"]), "f32 patterns")


def printouts(out):
    from oracle import build_ref
    tdir = os.path.join(build_ref.OUT, "python_test")
    for ours, fname in ((False, "ref_printouts.json"), (True, "ours_printouts.json")):
        env = _env(ours)
        res = {}
        for prog in sorted(os.listdir(tdir)):
            r = subprocess.run([sys.executable, os.path.join(tdir, prog)], env=env, capture_output=True,
                               text=True, timeout=600, cwd=tdir)
            res[prog] = {"rc": r.returncode, "stdout": r.stdout, "stderr_tail": r.stderr[-2000:]}
        with open(os.path.join(out, fname), "w") as f:
            json.dump(res, f, indent=1)
        print(fname, {k: v["rc"] for k, v in res.items()})


def worker_timing(out):
    import numpy as np
    import ThrustRTC as T
    rng = np.random.default_rng(0)
    res = {}

    def timed(name, make, call, reps=3):
        args = make()
        call(*make_small(args))  # warm-up: NVRTC compiles every kernel of the call
        T.Wait()
        ts = []
        for _ in range(reps):
            a = make() if reps > 1 else args
            T.Wait()
            t0 = time.perf_counter()
            call(*a)
            T.Wait()
            ts.append(time.perf_counter() - t0)
        res[name] = {"seconds": ts, "median_s": float(np.median(ts))}
        print(name, res[name], flush=True)

    def make_small(args):
        return [T.device_vector_from_numpy(a.to_host(0, 4096)) if hasattr(a, "to_host") else a for a in args]

    n20, n27, n28 = 1 << 20, 1 << 27, 1 << 28
    k20 = rng.integers(0, 2**32, n20, dtype=np.uint32)
    timed("c1_sort_by_key_u32_i32_2e20",
          lambda: [T.device_vector_from_numpy(k20), T.device_vector_from_numpy(np.arange(n20, dtype=np.int32))],
          lambda k, v: T.Sort_By_Key(k, v), reps=5)
    k28 = rng.integers(0, 2**32, n28, dtype=np.uint32)
    v28 = np.arange(n28, dtype=np.uint32)
    timed("c2a_sort_by_key_u32_u32_2e28",
          lambda: [T.device_vector_from_numpy(k28), T.device_vector_from_numpy(v28)],
          lambda k, v: T.Sort_By_Key(k, v), reps=2)
    del k28, v28
    x = rng.integers(-1000, 1001, n28).astype(np.int32)
    dx = T.device_vector_from_numpy(x)
    do = T.device_vector("int32_t", n28)
    timed("c2b_inclusive_scan_i32_2e28", lambda: [dx, do], lambda a, b: T.Inclusive_Scan(a, b))
    even = T.Functor({}, ["x"], "        return (x & 1) != 0;\n")
    timed("c3c_copy_if_i32_2e28", lambda: [dx, do], lambda a, b: T.Copy_If(a, b, even))
    del dx, do, x
    f = rng.random(n28, dtype=np.float32)
    df = T.device_vector_from_numpy(f)
    timed("c2c_reduce_f32_2e28", lambda: [df], lambda a: T.Reduce(a))
    del df, f
    lens = rng.geometric(1.0 / 32, n28 // 16)
    keys = np.repeat(np.arange(len(lens), dtype=np.int64), lens)[:n28].astype(np.int32)
    vals = rng.random(n28, dtype=np.float32)
    dk, dv, dout = T.device_vector_from_numpy(keys), T.device_vector_from_numpy(vals), T.device_vector("float", n28)
    timed("c3d_scan_by_key_f32_2e28", lambda: [dk, dv, dout], lambda a, b, c: T.Inclusive_Scan_By_Key(a, b, c))
    del dk, dv, dout, keys, vals
    fk = rng.standard_normal(n27).astype(np.float32)
    timed("c3a_sort_f32_2e27", lambda: [T.device_vector_from_numpy(fk)], lambda a: T.Sort(a), reps=2)
    del fk
    zk = (0x0123456700000000 + rng.zipf(1.1, n27) % (1 << 20)).astype(np.int64)
    timed("c3b_sort_by_key_i64_zipf_i32_2e27",
          lambda: [T.device_vector_from_numpy(zk), T.device_vector_from_numpy(np.arange(n27, dtype=np.int32))],
          lambda k, v: T.Sort_By_Key(k, v), reps=2)
    with open(os.path.join(out, "ref_timing.json"), "w") as fo:
        json.dump(res, fo, indent=1)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--worker", default=None)
    ap.add_argument("--fixtures", action="store_true")
    ap.add_argument("--printouts", action="store_true")
    ap.add_argument("--timing", action="store_true")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.worker == "fixtures":
        worker_fixtures(a.out)
    elif a.worker == "probe":
        worker_probe(a.out)
    elif a.worker == "timing":
        worker_timing(a.out)
    else:
        if not (a.fixtures or a.printouts or a.timing):
            a.fixtures = a.printouts = True
        if a.fixtures:
            _child("probe", a.out)
            _child("fixtures", a.out)
        if a.printouts:
            printouts(a.out)
        if a.timing:
            _child("timing", a.out)
