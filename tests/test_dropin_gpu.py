"""Drop-in check: the reference's own, unmodified Python package (python/ThrustRTC, whose
Native.py:9-12 loads libPyThrustRTC.so from the package directory) runs the reference's
hot-path test programs (python/test/test_*.py) over this repository's libPyThrustRTC.so,
and every program prints exactly what it prints over the reference's library on a GPU
(tests/golden/ref_printouts.json, recorded by tests/golden/make_ref_fixtures.py).

The package and programs are copied next to the library by oracle/build_ref.py into
oracle/_ref/ (not part of the repository); the test is skipped where that was not built.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden", "ref_printouts.json")
PKG = os.path.join(ROOT, "oracle", "_ref", "pkg_ours")
PROGS = os.path.join(ROOT, "oracle", "_ref", "python_test")


def _programs():
    if not os.path.exists(GOLD):
        return []
    return sorted(json.load(open(GOLD)))


# Lines where this library prints the documented result and the reference does not: the
# reference's C ABI passes values_in as the keys output of Unique_By_Key_Copy
# (python/api_Reordering.cpp:120), so over its own library test_unique.py prints the untouched
# keys_out ([0 0 0 0]) and a values_out read while values_in was being overwritten.  This
# library writes keys_out, as the reference's C++ TRTC_Unique_By_Key_Copy does (unique.cpp:56-72).
EXPECTED_DEVIATIONS = {"test_unique.py": {8: "[1 3 2 1]", 9: "[9 8 5 3]", 10: "[1 3 2 1]", 11: "[9 8 5 3]"}}


@pytest.mark.parametrize("prog", _programs())
def test_reference_program_prints_the_same(cuda, prog):
    gold = json.load(open(GOLD))[prog]
    if not os.path.exists(os.path.join(PKG, "ThrustRTC", "libPyThrustRTC.so")) or \
            not os.path.exists(os.path.join(PROGS, prog)):
        pytest.skip("oracle/_ref not built here (python oracle/build_ref.py)")
    assert gold["rc"] == 0, "the reference itself failed on " + prog
    env = dict(os.environ)
    env["PYTHONPATH"] = PKG + (":" + env["PYTHONPATH"] if env.get("PYTHONPATH") else "")
    r = subprocess.run([sys.executable, os.path.join(PROGS, prog)], env=env, cwd=PROGS, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got, want = r.stdout.splitlines(), gold["stdout"].splitlines()
    assert len(got) == len(want)
    dev = EXPECTED_DEVIATIONS.get(prog, {})
    for i, (g, w) in enumerate(zip(got, want)):
        assert g == (dev[i] if i in dev else w), (i, g, w)
