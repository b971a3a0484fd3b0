"""Recipe: build the reference ThrustRTC library from its sources, as a checker for the oracle.

Test infrastructure only: nothing on the product path loads what this builds.  The result
lets the GPU box run the reference itself on seeded inputs (tests/golden/make_ref_fixtures.py),
whose outputs pin the oracle, and time the reference on the same GPU.

What it does (all outputs under oracle/_ref/, which git ignores; the reference tree is only
read):

* writes ``gen/cuda_inline_headers.hpp``: the reference's build step
  ``internal/pack_headers.cpp`` would generate this file inside the source tree; it only embeds
  ``built_in.h`` as a string table (``s_num_headers`` / ``s_name_headers`` /
  ``s_content_headers``, read at ``internal/impl_context.inl:147-150``), so this recipe writes
  the same table itself into a directory of its own;
* writes ``gen/unqlite.h``: the ``thirdparty/unqlite`` submodule is empty (``.gitmodules``).
  The reference uses four unqlite calls for an on-disk PTX cache only
  (``internal/impl_context.inl:404-648``); this stub makes every one of them fail, so every
  kernel is compiled by NVRTC in-process (warm up once per process before timing);
* compiles every library and Python-binding source that ``python/CMakeLists.txt`` lists,
  where it lies, with ``g++ -std=c++17 -fPIC -include cstdio`` (some sources call printf
  without including <cstdio>), into ``_ref/ThrustRTC/libPyThrustRTC.so`` -- except
  ``internal/launch_calc.cpp``, whose vendored occupancy calculator knows compute
  capabilities up to 8.x only: on a B200 it leaves every block size at -1 and every launch of
  the reference fails without a message.  ``oracle/ref_launch_calc.cpp`` (written here)
  answers the same two queries through the driver's occupancy API instead;
* places the reference's unmodified Python package (``python/ThrustRTC/*.py``) beside that
  library, where its ``Native.py:9-12`` looks for it, and copies the reference's hot-path
  Python test programs to ``_ref/python_test/`` (run on the GPU box, they produce golden
  printouts);
* builds ``_ref/pkg_ours/ThrustRTC/``: the same unmodified package, with this repository's
  ``thrustrtc_b200/libPyThrustRTC.so`` linked in as its library (the drop-in check).

The library loads ``libcuda.so`` by that exact name (``internal/cuda_wrapper.cpp:87``); on a
box that only has ``libcuda.so.1`` the runner puts a symlink in ``_ref/cudalib/`` on
LD_LIBRARY_PATH (``cuda_lib_dir()``).

Usage: python oracle/build_ref.py [--ref REFERENCE_TREE]   (or set TRTC_REFERENCE_ROOT)
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
DEFAULT_REF = "/root/reference"

LIB_SOURCES = """
thirdparty/crc64/crc64.cpp internal/cuda_wrapper.cpp internal/nvtrc_wrapper.cpp
internal/general_reduce.cpp internal/general_scan.cpp internal/general_scan_by_key.cpp internal/general_copy_if.cpp
internal/general_find.cpp internal/merge_sort.cpp internal/radix_sort.cpp TRTCContext.cpp DVVector.cpp DVTuple.cpp
fake_vectors/DVRange.cpp fake_vectors/DVConstant.cpp fake_vectors/DVCounter.cpp fake_vectors/DVDiscard.cpp
fake_vectors/DVPermutation.cpp fake_vectors/DVReverse.cpp fake_vectors/DVTransform.cpp fake_vectors/DVZipped.cpp
fake_vectors/DVCustomVector.cpp functor.cpp fill.cpp replace.cpp for_each.cpp adjacent_difference.cpp sequence.cpp
tabulate.cpp transform.cpp gather.cpp scatter.cpp copy.cpp swap.cpp count.cpp reduce.cpp equal.cpp extrema.cpp
inner_product.cpp transform_reduce.cpp logical.cpp scan.cpp transform_scan.cpp scan_by_key.cpp remove.cpp unique.cpp
partition.cpp find.cpp mismatch.cpp binary_search.cpp merge.cpp sort.cpp
python/api_utils.cpp python/api_Context.cpp python/api_DeviceViewable.cpp python/api_DVVector.cpp
python/api_DVTuple.cpp python/api_FakeVectors.cpp python/api_Functor.cpp python/api_Transformations.cpp
python/api_Copying.cpp python/api_Reductions.cpp python/api_PrefixSums.cpp python/api_Reordering.cpp
python/api_Searching.cpp python/api_Merging.cpp python/api_Sorting.cpp
""".split() + [os.path.join(HERE, "ref_launch_calc.cpp")]  # in place of internal/launch_calc.cpp

# the reference's hot-path Python test programs (printouts become golden files)
PY_TESTS = ["test_sort.py", "test_scan.py", "test_transform_scan.py", "test_scan_by_key.py", "test_copy.py",
            "test_partition.py", "test_remove.py", "test_unique.py", "test_reduce.py", "test_transform_reduce.py",
            "test_extrema.py", "test_binary_search.py"]

UNQLITE_STUB = """// unqlite stub written by oracle/build_ref.py: the reference's on-disk PTX cache is
// disabled (every call fails), so kernels are always compiled in-process by NVRTC.
#pragma once
typedef struct unqlite unqlite;
typedef long long unqlite_int64;
#define UNQLITE_OK 0
#define UNQLITE_IOERR (-2)
#define UNQLITE_OPEN_CREATE 0x00000004
static inline int unqlite_open(unqlite** db, const char*, unsigned int) { *db = 0; return UNQLITE_IOERR; }
static inline int unqlite_close(unqlite*) { return UNQLITE_IOERR; }
static inline int unqlite_kv_fetch(unqlite*, const void*, int, void*, unqlite_int64*) { return UNQLITE_IOERR; }
static inline int unqlite_kv_store(unqlite*, const void*, int, const void*, unqlite_int64) { return UNQLITE_IOERR; }
"""


def ref_root(arg=None):
    return arg or os.environ.get("TRTC_REFERENCE_ROOT") or DEFAULT_REF


def _packed_header(ref):
    """The string table of built_in.h that internal/impl_context.inl:147-150 registers."""
    data = open(os.path.join(ref, "built_in.h"), "rb").read()
    body = ", ".join(str(b) for b in data) + ", 0"
    return ("// written by oracle/build_ref.py: built_in.h as the header table TRTCContext registers\n"
            "static char s_filename_0[] = \"built_in.h\";\n"
            "static const unsigned char s_file_content_0[] = {%s};\n"
            "static int s_num_headers = 1;\n"
            "static const char* s_name_headers[] = {s_filename_0};\n"
            "static const char* s_content_headers[] = {(const char*)s_file_content_0};\n" % body)


def _write_if_changed(path, text):
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


def _compile(ref, gen, src, obj):
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-w", "-include", "cstdio", "-I", gen, "-I", ref,
           "-I", os.path.join(ref, "internal"), "-I", os.path.join(ref, "thirdparty", "crc64"),
           "-I", os.path.join(ref, "python"), "-c", os.path.join(ref, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference compile failed: %s\n%s" % (" ".join(cmd), r.stderr[-4000:]))
    return obj


def _install_package(ref, dst_dir, lib):
    os.makedirs(dst_dir, exist_ok=True)
    for py in glob.glob(os.path.join(ref, "python", "ThrustRTC", "*.py")):
        shutil.copyfile(py, os.path.join(dst_dir, os.path.basename(py)))
    link = os.path.join(dst_dir, "libPyThrustRTC.so")
    if os.path.lexists(link):
        os.remove(link)
    os.symlink(os.path.relpath(lib, dst_dir), link)


def build(ref=None, jobs=None, verbose=True):
    """Builds oracle/_ref; returns the reference library's path, or None without a reference tree."""
    ref = ref_root(ref)
    if not os.path.exists(os.path.join(ref, "TRTCContext.cpp")):
        return None
    gen = os.path.join(OUT, "gen")
    objdir = os.path.join(OUT, "obj")
    pkg = os.path.join(OUT, "ThrustRTC")
    for d in (gen, objdir, pkg):
        os.makedirs(d, exist_ok=True)
    _write_if_changed(os.path.join(gen, "cuda_inline_headers.hpp"), _packed_header(ref))
    _write_if_changed(os.path.join(gen, "unqlite.h"), UNQLITE_STUB)
    lib = os.path.join(pkg, "libPyThrustRTC.so.real")
    todo, objs = [], []
    for s in LIB_SOURCES:
        o = os.path.join(objdir, s.replace("/", "__") + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < os.path.getmtime(os.path.join(ref, s)):
            todo.append((s, o))
    if todo:
        if verbose:
            print("oracle/_ref: compiling %d reference source(s)" % len(todo), flush=True)
        with cf.ThreadPoolExecutor(jobs or os.cpu_count() or 4) as ex:
            for f in [ex.submit(_compile, ref, gen, s, o) for s, o in todo]:
                f.result()
    if todo or not os.path.exists(lib):
        subprocess.check_call(["g++", "-shared", "-o", lib] + objs + ["-ldl", "-lpthread"])
    # the reference's package next to its own library
    for py in glob.glob(os.path.join(ref, "python", "ThrustRTC", "*.py")):
        shutil.copyfile(py, os.path.join(pkg, os.path.basename(py)))
    link = os.path.join(pkg, "libPyThrustRTC.so")
    if os.path.lexists(link):
        os.remove(link)
    os.symlink("libPyThrustRTC.so.real", link)
    # the same unmodified package over this repository's library
    _install_package(ref, os.path.join(OUT, "pkg_ours", "ThrustRTC"),
                     os.path.join(REPO, "thrustrtc_b200", "libPyThrustRTC.so"))
    tdir = os.path.join(OUT, "python_test")
    os.makedirs(tdir, exist_ok=True)
    for t in PY_TESTS:
        p = os.path.join(ref, "python", "test", t)
        if os.path.exists(p):
            shutil.copyfile(p, os.path.join(tdir, t))
    if verbose:
        print("oracle/_ref: reference library", lib, flush=True)
    return lib


def cuda_lib_dir():
    """A directory holding a ``libcuda.so`` symlink to the driver's libcuda.so.1 (made under
    oracle/_ref/cudalib), for LD_LIBRARY_PATH of a process that loads the reference."""
    d = os.path.join(OUT, "cudalib")
    os.makedirs(d, exist_ok=True)
    link = os.path.join(d, "libcuda.so")
    if not os.path.exists(link):
        import ctypes.util
        cands = ["/usr/lib/x86_64-linux-gnu/libcuda.so.1", "/usr/lib64/libcuda.so.1", "/usr/lib/libcuda.so.1"]
        found = [c for c in cands if os.path.exists(c)]
        if not found:
            name = ctypes.util.find_library("cuda")
            found = [name] if name else []
        if not found:
            return None
        if os.path.lexists(link):
            os.remove(link)
        os.symlink(found[0], link)
    return d


def package_dir(ours=False):
    """Directory to put on sys.path to import the reference's ThrustRTC package (over the
    reference's own library, or over this repository's with ``ours``), or None."""
    d = os.path.join(OUT, "pkg_ours") if ours else OUT
    return d if os.path.exists(os.path.join(d, "ThrustRTC", "libPyThrustRTC.so")) else None


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    a = ap.parse_args()
    r = build(a.ref)
    if r is None:
        print("reference tree not present; nothing built")
    sys.exit(0)
