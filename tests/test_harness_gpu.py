"""The comparison harness on the GPU: every generator of every value type and every
k distribution through this library's bucketMultiselect and iterativeSMOS entry
points, checked against sort-and-choose (DS/compareIterativeSMOS.cu:50-245); the rows it
appends have the reference's layout."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "ggms-distributed_b200"))

from ggms_b200 import harness as H  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32])
def test_compare_every_generator(dtype, tmp_path):
    csv = str(tmp_path / "compare.csv")
    n = 1 << 16
    rows = 0
    for gi, (gname, _) in enumerate(H.generators_for(dtype)):
        ki = gi % len(H.K_GENERATORS)
        ks = H.K_GENERATORS[ki][1](101, n, 100 + gi)
        res = H.compare_multiselect(dtype, n, ks, 2, gi, ki, csv, seed=gi, verbose=False)
        assert res["flags"] == [0, 0], gname
        assert np.all(np.isfinite(res["times_ms"])), gname
        rows += 2
    lines = open(csv).read().splitlines()
    assert len(lines) == rows
    for line in lines:
        f = line.split(",")
        assert f[0] == str(n) and f[1] == "101" and f[-1] == "0"
        assert [f[4], f[6], f[8]] == list(H.ALGORITHM_NAMES)
        assert all(float(f[i]) > 0 for i in (5, 7, 9))


def test_run_tests_sizes_and_k_counts(tmp_path):
    csv = str(tmp_path / "runs.csv")
    runs = H.run_tests(np.float32, 1, csv, 12, 14, 1, 3, 10, 30, 10)
    assert len(runs) == 3 * 3 and all(r["flags"] == [0] for r in runs)
    sizes_ks = [tuple(map(int, line.split(",")[:2])) for line in open(csv).read().splitlines()]
    assert sizes_ks == [(1 << p, k) for p in (12, 13, 14) for k in (10, 20, 30)]
