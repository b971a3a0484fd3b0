"""Builds thrustrtc_b200/libPyThrustRTC.so from csrc/ with nvcc for sm_100a.

Every .cu / .cpp under csrc/host is compiled with ``nvcc -gencode
arch=compute_100a,code=sm_100a -lineinfo -O3`` into thrustrtc_b200/_build/ (objects are
rebuilt when a source or any header under csrc/ is newer), then linked into one shared
library with the CUDA runtime linked statically (the driver is loaded at run time, so the
library also loads on machines without a GPU).  The device headers are also embedded into
the library as strings for the NVRTC path.

Usage: python thrustrtc_b200/build.py [-j N] [--force]
(run as a script: importing the package needs the library this builds)
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
OUT = os.path.join(PKG, "libPyThrustRTC.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-Xcudafe", "--diag_suppress=177"]


def _headers():
    return glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) + \
        glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)


def _embed_headers():
    """Writes _build/embedded_headers.cpp: the device headers as strings for NVRTC."""
    os.makedirs(BUILD, exist_ok=True)
    names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(CSRC, "device", "*.cuh")) +
                   glob.glob(os.path.join(CSRC, "device", "*.h")))
    lines = ["// generated by thrustrtc_b200/build.py -- device headers for the NVRTC path",
             "#include <cstddef>", "namespace trtc_host {"]
    for i, name in enumerate(names):
        data = open(os.path.join(CSRC, "device", name), "rb").read()
        chunks = [data[j:j + 4000] for j in range(0, len(data), 4000)]
        lits = " ".join('R"TRTC_EMBED(%s)TRTC_EMBED"' % c.decode() for c in chunks)
        lines.append("static const char h%d[] = %s;" % (i, lits))
    lines.append("extern const int g_num_device_headers = %d;" % len(names))
    lines.append("extern const char* const g_device_header_names[] = {%s};" %
                 ", ".join('"%s"' % n for n in names))
    lines.append("extern const char* const g_device_header_sources[] = {%s};" %
                 ", ".join("h%d" % i for i in range(len(names))))
    lines.append("}  // namespace trtc_host")
    path = os.path.join(BUILD, "embedded_headers.cpp")
    text = "\n".join(lines) + "\n"
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)
    return path


INCLUDE = os.path.join(os.path.dirname(PKG), "include")


def _compile(src, obj):
    cmd = [NVCC] + ARCH + FLAGS + ["-I", CSRC, "-I", INCLUDE, "-I", os.path.join(CSRC, "host"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    # a host call into a __device__-only function compiles (as a warning) into exit(1):
    # treat every compiler warning as a build failure
    if "warning" in (r.stdout + r.stderr):
        raise RuntimeError("compile warnings in %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build(force=False, jobs=None, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "host", "*.cu")) + glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    srcs.append(_embed_headers())
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    todo, objs = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_mtime):
            todo.append((s, o))
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
    if todo:
        if verbose:
            print("thrustrtc_b200: compiling %d source(s) with %d job(s)" % (len(todo), jobs), flush=True)
        with cf.ThreadPoolExecutor(jobs) as ex:
            futs = [ex.submit(_compile, s, o) for s, o in todo]
            for f in futs:
                f.result()
    if todo or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        tmp = OUT + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static", "-ldl", "-lrt", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        os.replace(tmp, OUT)
        if verbose:
            print("thrustrtc_b200: linked", OUT, flush=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(force=a.force, jobs=a.j)
    sys.exit(0)
