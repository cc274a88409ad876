"""The comparison harness: the reference's generator and k-distribution tables
(DS/generateProblems.cu:75-79, 438-446, 509-513, 725-730) and its CSV row layout
(DS/compareIterativeSMOS.cu:136-139, 180-210)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "ggms-distributed_b200"))

from ggms_b200 import harness as H  # noqa: E402


def test_table_names_and_order():
    assert [n for n, _ in H.FLOAT_GENERATORS] == [
        "UNIFORM FLOATS", "NORMAL FLOATS", "KILLER FLOATS", "HALF NORMAL FLOATS",
        "NORMAL FLOATS 100", "HUGE UNIFORM FLOATS", "NOISY FLOATS", "ALL ONES FLOATS",
        "ONES TWOS FLOAT", "CAUCHY FLOAT"]
    assert [n for n, _ in H.DOUBLE_GENERATORS] == ["UNIFORM DOUBLES", "NORMAL DOUBLES", "KILLER DOUBLES"]
    assert [n for n, _ in H.UINT_GENERATORS] == ["UNIFORM UNSIGNED INTEGERS", "SORTED UINTS", "UNIFORM 0-4"]
    assert [n for n, _ in H.K_GENERATORS] == [
        "Uniform Random Ks", "Uniform Ks", "Normal Random Ks", "Cluster Ks", "Sectioned Ks"]
    assert H.ALGORITHM_NAMES == ("Sort and Choose Multiselect", "Bucket Multiselect", "IterativeSMOS")
    with pytest.raises(ValueError):
        H.generators_for(np.int16)


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32])
@pytest.mark.parametrize("n", [1, 7, 300, 5000])
def test_generators_shape_type_seed(dtype, n):
    for name, gen in H.generators_for(dtype):
        a, b, c = gen(n, 3), gen(n, 3), gen(n, 4)
        assert a.dtype == np.dtype(dtype) and a.shape == (n,), name
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name   # same seed, same bits
        fixed_head = 2045 if name == "KILLER DOUBLES" else 253   # the powers of two
        if n > fixed_head and name not in ("ALL ONES FLOATS", "UNIFORM 0-4"):
            assert not np.array_equal(a, c), name


def test_generator_shapes():
    n = 10000
    k = H.bucket_killer_floats(n, 1)
    assert np.array_equal(k[:253], np.ldexp(np.float32(1), np.arange(-126, 127)).astype(np.float32))
    assert np.all((k[253:].view(np.uint32) & ~np.uint32(0x80EFFFFF)) == 0)
    kd = H.bucket_killer_doubles(3000, 1)
    assert np.array_equal(kd[:2045], np.ldexp(1.0, np.arange(-1022, 1023)))
    ot = H.ones_twos_floats(n, 1)
    assert (ot == 2).sum() == n // 2 and (ot == 1).sum() == n - n // 2
    nz = H.noisy_floats(n, 1)
    assert abs((nz > 0.5).sum() - n // 5) < 10
    assert np.array_equal(H.uniform_0_4_uints(250, 0), np.arange(250, dtype=np.uint32) % 100)
    s = H.sorted_uints(n, 2)
    assert np.all(s[1:] >= s[:-1])
    assert np.all(H.half_normal_floats(n, 1) >= 0)
    assert np.all(np.isfinite(H.cauchy_floats(n, 1)))


@pytest.mark.parametrize("name_gen", H.K_GENERATORS, ids=[n for n, _ in H.K_GENERATORS])
@pytest.mark.parametrize("count,n", [(1, 1), (5, 10), (101, 1 << 20), (1000, 1 << 20), (37, 40)])
def test_k_distributions_in_range(name_gen, count, n):
    _, gen = name_gen
    ks = gen(count, n, 5)
    assert ks.dtype == np.uint32 and ks.shape == (count,)
    assert ks.min() >= 1 and ks.max() <= n


def test_k_distribution_rules():
    n = 1 << 20
    u = H.ks_uniform(101, n, 0)
    exp = [1] + [int(np.float32(i) / np.float32(100) * np.float32(n)) for i in range(1, 100)] + [n]
    assert u.tolist() == exp
    sec = H.ks_sectioned(64, n, 9)
    assert np.all(np.diff(sec.astype(np.int64)) == 1)
    cl = H.ks_cluster(27, n, 4).astype(np.int64)
    for c in (4, 13, 22):                          # runs of nine consecutive ranks
        assert np.array_equal(cl[c - 4:c + 5], np.arange(cl[c] - 4, cl[c] + 5))
    cl = H.ks_cluster(30, n, 4).astype(np.int64)   # three entries after the last run
    assert np.all(np.diff(cl[27:]) == 1) and cl[-1] <= n - 1
    nr = H.ks_normal_random(1000, n, 2)
    assert nr.min() >= n // 2                      # (|z| + 7) n / 14 >= n / 2


def test_csv_row_layout():
    row = H.csv_row(1048576, 101, "UNIFORM FLOATS", "Uniform Ks",
                    [("Sort and Choose Multiselect", 3.25), ("Bucket Multiselect", 0.123456789),
                     ("IterativeSMOS", 1234567.0)], 0)
    assert row == ("1048576,101,UNIFORM FLOATS,Uniform Ks,Sort and Choose Multiselect,3.25,"
                   "Bucket Multiselect,0.123457,IterativeSMOS,1.23457e+06,0\n")
    err = H.error_lines(2, 5, 1024, 77, 3, 10, 1, 0.5, 0.25)
    assert err == ("\nERROR ON TEST 2 of 5 tests!!!!!\nvector size = 1024\nvector seed = 77\n"
                   "numKs = 3\nwrong k = 10 kIndex = 1 wrong result = 0.5 correct result = 0.25\n")


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32, np.int32])
def test_sort_and_choose_checker_order(dtype):
    """The harness's checker (algorithm 0) on CPU tensors: the k-th largest under the
    total order -NaN < -Inf < ... < -0 < +0 < ... < +Inf < +NaN, as bit patterns."""
    import torch
    g = np.random.default_rng(1)
    n = 4099
    if np.dtype(dtype).kind == "f":
        v = g.standard_normal(n).astype(dtype)
        v[:6] = [np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0]
        v[6:40] = v[40]                                     # duplicates
    else:
        v = g.integers(np.iinfo(dtype).min, np.iinfo(dtype).max, size=n, dtype=dtype)
    ks = np.concatenate([[1, n], g.integers(1, n + 1, size=200)]).astype(np.uint32)
    raw = H._raw_tensor(torch, v, "cpu")
    got = H._sort_and_choose(torch, raw, ks, dtype)
    ib = np.uint64 if v.dtype.itemsize == 8 else np.uint32
    bits = v.view(ib)
    if np.dtype(dtype).kind == "f":
        top = ib(1) << ib(8 * v.dtype.itemsize - 1)
        key = np.where(bits & top, ~bits, bits | top)
    elif np.dtype(dtype) == np.int32:
        key = bits ^ ib(0x80000000)
    else:
        key = bits
    srt = bits[np.argsort(key, kind="stable")]
    assert np.array_equal(got.view(ib), srt[n - ks.astype(np.int64)])


def test_command_line_answers_and_file_name():
    a = H.parse_answers("0 0 1 20 26 101 1 101 5".split())
    assert a == dict(type=0, generator=0, k_distribution=1, start_power=20, stop_power=26,
                     start_k=101, k_jump=1, stop_k=101, tests=5)
    assert H.file_name(a, "box", "Thu Dec  3 10:00:00 2026") == (
        "float UNIFORM FLOATS k-dist:Uniform Ks 2^20 to 2^26 (101:1:101) 5-tests on box at "
        "Thu Dec  3 10:00:00 2026")
    d = H.parse_answers(["1", "2", "3", "10", "12", "9", "9", "27", "1"])
    assert H.file_name(d, "h", "t").startswith("double KILLER DOUBLES k-dist:Cluster Ks 2^10 to 2^12 (9:9:27)")
    for bad in ("3 0 0 20 26 1 1 1 1", "0 10 0 20 26 1 1 1 1", "0 0 5 20 26 1 1 1 1",
                "0 0 0 26 20 1 1 1 1", "0 0 0 20 26 5 0 9 1", "0 0 0 20 26 1 1 1"):
        with pytest.raises(ValueError):
            H.parse_answers(bad.split())
