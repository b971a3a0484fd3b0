"""The oracle against the reference's own outputs (tests/golden/ref_fixtures.npz).

The fixtures were produced by running the reference ThrustRTC itself (built from its sources
by oracle/build_ref.py) on a GPU through its unmodified Python package, on the seeded cases
of tests/golden/ref_cases.py: sorts of every key width including float keys with -0.0, +NaN,
-NaN, payload NaNs and NaN at index 0 (the Min_Element rotation), scans with init and
operators, transform scans, scan_by_key with init, every Partition / Remove / Unique /
Copy_If form at three selectivities, Reduce_By_Key and Min_Element.  Generator:
tests/golden/make_ref_fixtures.py.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_fixtures.npz")
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)


@pytest.fixture(scope="module")
def fixtures():
    if not os.path.exists(FIX):
        pytest.skip("reference fixtures not generated")
    return np.load(FIX)


def test_oracle_matches_reference_outputs(fixtures):
    import oracle_api
    import ref_cases
    res = ref_cases.run_all(oracle_api)
    bad = ref_cases.compare(fixtures, res)
    assert not bad, bad


def test_fixture_inputs_regenerate(fixtures):
    # the stored input checksums match the inputs the cases generate here
    import oracle_api
    import ref_cases
    res = ref_cases.run_all(oracle_api)
    names = [k[6:] for k in fixtures.files if k.startswith("crc32:") and k.split("/")[-1].startswith("in")]
    assert names
    for name in names:
        want = fixtures["crc32:" + name]
        assert ref_cases._crc(res[name]) == int(want[0]) and len(res[name]) == int(want[1]), name
