"""Generates the golden fixtures under tests/golden/ (run in a container that has the
reference tree; the fixtures themselves are committed and read by the tests).

* docs_vectors.json -- the known answers printed in the reference's quick-start guide
  (docs/QuickStartGuide.md:996-1015 scans, :1038-1095 sorts) and the examples of its python
  tests whose outputs are fixed by the docs.
* test_sort_cpp.npz -- the two "big case" inputs of cpp/test/test_sort.cpp:82-168: 10,000
  values 1..10000 shuffled with glibc rand() (unseeded, i.e. seed 1, the second case
  continuing the same stream), which the reference self-checks to sort back to 1..10000
  (and values 10000-i for the by-key case).
* builtin_h_probe.json -- d_u32/d_u64 and Maximum/Minimum evaluated by the reference's own
  built_in.h compiled on the CPU (oracle/build_ref_probe.py).
* api_h_exports.json -- the names of the reference's exported C functions
  (python/api.h), which the drop-in library must export too.
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

DOCS = {
    "source": "docs/QuickStartGuide.md",
    "inclusive_scan": {"in": [1, 0, 2, 2, 1, 3], "out": [1, 1, 3, 5, 6, 9], "dtype": "int32_t",
                       "cite": "docs/QuickStartGuide.md:996-1005"},
    "exclusive_scan": {"in": [1, 0, 2, 2, 1, 3], "out": [0, 1, 1, 3, 5, 6], "dtype": "int32_t",
                       "cite": "docs/QuickStartGuide.md:1013-1016"},
    "sort": {"in": [1, 4, 2, 8, 5, 7], "out": [1, 2, 4, 5, 7, 8], "dtype": "int32_t",
             "cite": "docs/QuickStartGuide.md:1038-1053"},
    "sort_greater": {"in": [1, 4, 2, 8, 5, 7], "out": [8, 7, 5, 4, 2, 1], "dtype": "int32_t",
                     "cite": "docs/QuickStartGuide.md:1083-1095"},
    "sort_by_key_char": {"keys": [1, 4, 2, 8, 5, 7], "values": [97, 98, 99, 100, 101, 102],
                         "keys_out": [1, 2, 4, 5, 7, 8], "values_out": [97, 99, 98, 101, 102, 100],
                         "key_dtype": "int32_t", "value_dtype": "int8_t",
                         "cite": "docs/QuickStartGuide.md:1058-1071"},
    "sort_by_key_int": {"keys": [1, 4, 2, 8, 5, 7], "values": [1, 2, 3, 4, 5, 6],
                        "keys_out": [1, 2, 4, 5, 7, 8], "values_out": [1, 3, 2, 5, 6, 4],
                        "key_dtype": "int32_t", "value_dtype": "int32_t",
                        "cite": "docs/QuickStartGuide.md:1073-1080"},
}


def glibc_shuffles():
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    a = np.arange(1, 10001, dtype=np.int32)
    for i in range(9999):
        j = i + libc.rand() % (10000 - i)
        a[i], a[j] = a[j], a[i]
    keys = np.arange(1, 10001, dtype=np.int32)
    vals = (10000 - np.arange(10000)).astype(np.int32)
    for i in range(9999):
        j = i + libc.rand() % (10000 - i)
        keys[i], keys[j] = keys[j], keys[i]
        vals[i], vals[j] = vals[j], vals[i]
    return a, keys, vals


sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.build_ref import ref_root  # noqa: E402  (the reference tree this script reads)

REF_ROOT = ref_root()


def api_h_exports():
    import re
    text = open(os.path.join(REF_ROOT, "python", "api.h")).read()
    names = sorted(set(re.findall(r"PY_THRUSTRTC_API\s+[\w\s\*]+?\b(n_\w+)\s*\(", text)))
    return {"source": "python/api.h", "names": names}


def main():
    if os.path.isdir(REF_ROOT):
        with open(os.path.join(HERE, "api_h_exports.json"), "w") as f:
            json.dump(api_h_exports(), f, indent=1)
    with open(os.path.join(HERE, "docs_vectors.json"), "w") as f:
        json.dump(DOCS, f, indent=1)
    a, k, v = glibc_shuffles()
    np.savez_compressed(os.path.join(HERE, "test_sort_cpp.npz"), sort_in=a, sbk_keys=k, sbk_values=v)
    from oracle import build_ref_probe
    res = build_ref_probe.build_and_run()
    if res is not None:
        res["source"] = "built_in.h compiled by oracle/build_ref_probe.py"
        with open(os.path.join(HERE, "builtin_h_probe.json"), "w") as f:
            json.dump(res, f, indent=1)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
