"""The CPU oracle against golden vectors produced by the reference's own GPU
build (tests/golden/make_golden.py runs bucketMultiselectWrapper, built from
the reference's unmodified sources)."""
import glob
import os

import numpy as np
import pytest

import ggms_oracle as orc

FIXTURES = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def test_fixtures_present():
    assert len(FIXTURES) >= 10, "golden fixtures missing (tests/golden/make_golden.py)"


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_reference(path):
    z = np.load(path)
    v, ks, ref = z["values"], z["ks"], z["ref_out"]
    got = orc.select(v, ks)
    if "signed_zeros" in path:
        # thrust's radix sort orders -0.0 and +0.0 as equal (stable), the oracle
        # orders -0.0 < +0.0: the values agree, the sign bit of a zero may not.
        np.testing.assert_array_equal(got, ref)
        zero = (ref == 0)
        assert np.array_equal(orc.bits(got)[~zero], orc.bits(ref)[~zero])
    else:
        np.testing.assert_array_equal(orc.bits(got), orc.bits(ref))
