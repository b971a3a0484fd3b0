"""The persistent cubin cache of the NVRTC path (csrc/host/trtc_jit.cpp).

Each step runs in a fresh child process (the in-process cache starts empty there), all
sharing one cache directory (TRTC_CACHE_DIR):
  1. a Copy_If with a user Functor compiles its kernels and stores them (<id>.cubin / .name
     / .key files appear);
  2. the same program in a new process compiles nothing: every kernel comes from the disk;
  3. with every stored key altered (what an entry written by another library build, or a
     hash collision, looks like) the program compiles again instead of loading those cubins,
     and its results are still right;
  4. TRTC_JIT_DISK_CACHE=0 bypasses the directory: it compiles and writes nothing there.
The result of every step is checked against numpy.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, %(root)r)
import thrustrtc_b200 as T
from thrustrtc_b200 import _native as N
T.init()
x = np.arange(10000, dtype=np.int32) * 7 + 3  # non-negative: C++ and numpy %% agree
d = T.device_vector_from_numpy(x)
o = T.device_vector("int32_t", len(x))
f = T.Functor({}, ["x"], "        return (x %% 11) == %(token)d;\n")
c = T.Copy_If(d, o, f)
exp = x[(x %% 11) == %(token)d]
ok = c == len(exp) and o.to_host()[:c].tolist() == exp.tolist()
st = (ctypes.c_ulonglong * 3)()
N.lib.trtc_jit_cache_stats.argtypes = [ctypes.c_void_p]
N.lib.trtc_jit_cache_stats(st)
print(json.dumps({"ok": bool(ok), "compiles": st[0], "disk_hits": st[1], "mem_hits": st[2]}))
"""


def _run(cache_dir, token, extra_env=None):
    env = dict(os.environ)
    env["TRTC_CACHE_DIR"] = cache_dir
    env.pop("TRTC_JIT_DISK_CACHE", None)
    if extra_env:
        env.update(extra_env)
    r = subprocess.run([sys.executable, "-c", CHILD % {"root": ROOT, "token": token}], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def _entries(cache_dir):
    return sorted(f for f in os.listdir(cache_dir) if not f.count(".tmp")) if os.path.isdir(cache_dir) else []


def test_persistent_cubin_cache(cuda, tmp_path):
    cache = str(tmp_path / "cubins")
    token = 7  # a predicate of its own: nothing else in the run shares these kernels' source

    first = _run(cache, token)
    assert first["ok"] and first["compiles"] >= 1, first
    files = _entries(cache)
    keys = [f for f in files if f.endswith(".key")]
    assert keys and len(keys) == sum(f.endswith(".cubin") for f in files) == sum(f.endswith(".name") for f in files)

    second = _run(cache, token)
    assert second["ok"], second
    assert second["compiles"] == 0 and second["disk_hits"] >= first["compiles"], (first, second)
    assert _entries(cache) == files

    for k in keys:  # entries of another key: never loaded
        p = os.path.join(cache, k)
        with open(p, "rb") as fh:
            data = fh.read()
        with open(p, "wb") as fh:
            fh.write(data.replace(b"thrustrtc_b200 cubin cache", b"thrustrtc_b200 cubin cachE"))
    third = _run(cache, token)
    assert third["ok"], third
    assert third["compiles"] == first["compiles"] and third["disk_hits"] == 0, (first, third)

    fourth = _run(cache, token, {"TRTC_JIT_DISK_CACHE": "0"})
    assert fourth["ok"] and fourth["compiles"] >= 1 and fourth["disk_hits"] == 0, fourth
    assert _entries(cache) == files  # the third run rewrote the same entries; the fourth wrote none

    fifth = _run(cache, token)  # the rewritten entries serve again
    assert fifth["ok"] and fifth["compiles"] == 0, fifth
