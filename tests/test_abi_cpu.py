"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "thrustrtc_b200", "libPyThrustRTC.so")


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:n|trtc)_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def exported():
    assert os.path.exists(LIB), "build the library first (python thrustrtc_b200/build.py)"
    out = subprocess.check_output(["nm", "-D", "--defined-only", LIB]).decode()
    return set(line.split()[-1] for line in out.splitlines() if line.strip())


@pytest.mark.parametrize("header", ["thrustrtc_b200.h", "trtc_raw.h", "trtc_server.h"])
def test_every_declared_symbol_is_exported(header, exported):
    names = _declared(header)
    assert names, header
    missing = [n for n in names if n not in exported]
    assert not missing, missing


def test_library_loads_without_gpu():
    lib = ctypes.CDLL(LIB)
    lib.trtc_launch_count.restype = ctypes.c_ulonglong
    assert lib.trtc_launch_count() == 0


def test_python_package_imports():
    import thrustrtc_b200 as trtc
    assert hasattr(trtc, "Sort_By_Key") and hasattr(trtc, "Inclusive_Scan") and hasattr(trtc, "Copy_If")


def test_no_exit_import_in_library():
    # a host-side call of a device-only helper compiles into exit(1) (the build also fails on
    # that compiler warning); the library's dynamic symbol table names no exit/abort import
    out = subprocess.check_output(["nm", "-D", "--undefined-only", LIB]).decode()
    imported = set(line.split()[-1].split("@")[0] for line in out.splitlines() if line.strip())
    assert not imported & {"exit", "_exit", "abort"}, imported & {"exit", "_exit", "abort"}


def test_python_names_of_the_reference_package():
    # every public name of python/ThrustRTC/*.py is importable from the package
    import thrustrtc_b200 as t
    names = ["DVCupyVector", "DVNumbaVector", "Dim3", "ObjArray", "StrArray", "ValueFromDVPtr", "DVTorchVector",
             "Sort_By_Key", "Merge_By_Key", "Inner_Product", "Partition_Point", "Is_Sorted_Until", "DVZipped",
             "DVCustomVector", "DVTuple", "Tabulate", "Adjacent_Difference"]
    assert [n for n in names if not hasattr(t, n)] == []


def test_cuda_array_interface_adaptor_checks_dtype_and_contiguity():
    import pytest
    import thrustrtc_b200 as t

    class Fake:
        def __init__(self, typestr, shape, strides=None):
            self.__cuda_array_interface__ = {"data": (0, False), "typestr": typestr, "shape": shape,
                                             "strides": strides, "version": 3}

    with pytest.raises(ValueError):
        t.DVCupyVector(Fake("<f2", (4,)))          # float16: no element type of the library
    with pytest.raises(ValueError):
        t.DVNumbaVector(Fake("<i4", (4,), (8,)))   # strided


def test_cpp_api_links_against_the_library(tmp_path):
    # every TRTC_* declaration of include/thrustrtc_cpp.h (the C++ API the reference's JNI and
    # C++/CLI shims call) resolves, with its declared signature, in libPyThrustRTC.so
    import re
    import shutil
    import subprocess
    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    inc = os.path.join(ROOT, "include")
    src = open(os.path.join(inc, "thrustrtc_cpp.h")).read()
    decls = re.findall(r"THRUST_RTC_API\s+([\w:<>\*&\s]+?)\s+(TRTC_\w+)\s*\(([^;{]*?)\)\s*;", src, re.S)
    assert len(decls) > 100
    lines = []
    for ret, name, params in decls:
        params = " ".join(params.split())
        types = []
        if params and params != "void":
            for p in params.split(","):
                p = re.sub(r"\s*=.*$", "", p.strip())
                types.append(re.sub(r"\s*\b\w+$", "", p))
        lines.append("    f.push_back(reinterpret_cast<void (*)()>(static_cast<%s (*)(%s)>(&%s)));"
                     % (" ".join(ret.split()), ", ".join(types), name))
    cpp = tmp_path / "api_link.cpp"
    cpp.write_text('#include "thrustrtc_cpp.h"\n#include <cstdio>\n#include <vector>\nint main() {\n'
                   "    std::vector<void (*)()> f;\n" + "\n".join(lines) +
                   '\n    std::printf("%zu\\n", f.size());\n    return 0;\n}\n')
    exe = tmp_path / "api_link"
    lib_dir = os.path.join(ROOT, "thrustrtc_b200")
    r = subprocess.run(["g++", "-std=c++17", "-I", inc, str(cpp), "-o", str(exe), "-L", lib_dir, "-lPyThrustRTC",
                        "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and int(r.stdout.strip()) == len(decls), r.stderr


def test_every_reference_export_is_present():
    # the reference's python/api.h exports (tests/golden/api_h_exports.json, written by
    # tests/golden/make_golden.py from the reference tree) all resolve in this library
    import json
    names = json.load(open(os.path.join(ROOT, "tests", "golden", "api_h_exports.json")))["names"]
    assert len(names) > 140
    lib = ctypes.CDLL(LIB)
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_segmented_tuning_table_round_trip():
    # the batched kernel's size-class table: versioned JSON in, the same entries out; another
    # format, version or an unsupported shape is refused (host-only, no GPU needed)
    lib = ctypes.CDLL(LIB)
    lib.trtc_raw_segmented_tuning_json.restype = ctypes.c_ulonglong
    lib.trtc_raw_segmented_tuning_json.argtypes = [ctypes.c_char_p, ctypes.c_ulonglong]
    lib.trtc_raw_segmented_tuning_load.restype = ctypes.c_int
    lib.trtc_raw_segmented_tuning_load.argtypes = [ctypes.c_char_p]
    import json
    t = {"format": "thrustrtc_b200.segmented_tuning", "version": 1,
         "entries": [{"key_type": 5, "items": 8, "warp_small": 32}, {"key_type": 6, "items": 16, "warp_small": 0}]}
    assert lib.trtc_raw_segmented_tuning_load(json.dumps(t).encode()) == 0
    buf = ctypes.create_string_buffer(4096)
    size = lib.trtc_raw_segmented_tuning_json(buf, 4096)
    out = json.loads(buf.value.decode())
    assert size == len(buf.value) and out["version"] == 1 and out["digit_bits"] == 8
    got = {e["key_type"]: (e["items"], e["warp_small"]) for e in out["entries"]}
    assert got[5] == (8, 32) and got[6] == (16, 0)
    bad = dict(t, version=2)
    assert lib.trtc_raw_segmented_tuning_load(json.dumps(bad).encode()) == -1
    bad = dict(t, entries=[{"key_type": 5, "items": 12, "warp_small": 32}])
    assert lib.trtc_raw_segmented_tuning_load(json.dumps(bad).encode()) == -1
    assert lib.trtc_raw_segmented_tuning_load(b'{"format": "other", "version": 1}') == -1
