"""The CPU oracle (sort-and-choose) and the CPU baselines, no GPU needed."""
import numpy as np
import pytest

import ggms_oracle as orc


def brute(values, ks):
    """Pure numpy restatement: sort keys ascending, take sorted[n - k]."""
    k = orc.keys(values)
    order = np.argsort(k, kind="stable")
    s = values[order]
    return s[len(values) - ks.astype(np.int64)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32, np.int32])
@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 1000, 4099])
def test_oracle_matches_numpy(dtype, n):
    g = np.random.default_rng(n)
    if np.dtype(dtype).kind == "f":
        v = g.standard_normal(n).astype(dtype)
    else:
        v = g.integers(np.iinfo(dtype).min, np.iinfo(dtype).max, size=n, dtype=dtype, endpoint=True)
    ks = g.integers(1, n + 1, size=57).astype(np.uint32)
    np.testing.assert_array_equal(orc.bits(orc.select(v, ks)), orc.bits(brute(v, ks)))


def test_key_order_specials():
    v = np.array([np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-45, -1e-45, 3.0, -3.0],
                 dtype=np.float32)
    v[0] = np.frombuffer(np.uint32(0x7FC00000).tobytes(), np.float32)[0]
    v[1] = np.frombuffer(np.uint32(0xFFC00000).tobytes(), np.float32)[0]
    n = len(v)
    asc = orc.select(v, np.arange(n, 0, -1, dtype=np.uint32))  # k = n .. 1 -> ascending
    expect = [0xFFC00000, 0xFF800000, 0xC0400000, 0x80000001, 0x80000000,
              0x00000000, 0x00000001, 0x40400000, 0x7F800000, 0x7FC00000]
    assert [int(x) for x in orc.bits(asc)] == expect


def test_key_map_roundtrip_and_order():
    g = np.random.default_rng(1)
    u = g.integers(0, 2**32, size=10000, dtype=np.uint32)
    f = u.view(np.float32)
    k = orc.keys(f)
    assert len(np.unique(k)) == len(np.unique(u))
    fin = f[np.isfinite(f)]
    kf = orc.keys(fin)
    o1 = np.argsort(kf, kind="stable")
    assert np.all(np.diff(fin[o1].astype(np.float64)) >= 0)
    for x in (0.0, -0.0, 1.5, -2.25, np.inf):
        assert orc.lib().ggms_oracle_key_f32(x) == int(orc.keys(np.array([x], np.float32))[0])


def test_k_convention_largest():
    v = np.array([5, 1, 4, 2, 3], dtype=np.uint32)
    assert list(orc.select(v, np.array([1, 2, 5], dtype=np.uint32))) == [5, 4, 1]


def test_duplicates_and_duplicate_ks():
    v = np.array([7] * 50 + [3] * 50, dtype=np.int32)
    ks = np.array([1, 50, 51, 100, 50, 51], dtype=np.uint32)
    assert list(orc.select(v, ks)) == [7, 7, 3, 3, 7, 3]


@pytest.mark.parametrize("bad", [[0], [6], [1, 2, 7]])
def test_oracle_rejects_bad_k(bad):
    with pytest.raises(ValueError):
        orc.select(np.arange(5, dtype=np.uint32), np.array(bad, dtype=np.uint32))


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32])
def test_cpu_baseline_matches_oracle(method, dtype):
    g = np.random.default_rng(7)
    n = 200_003
    if np.dtype(dtype).kind == "f":
        v = g.standard_normal(n).astype(dtype)
        v[::997] = v[5]  # duplicates
    else:
        v = g.integers(0, 2**32, size=n, dtype=np.uint32)
    ks = g.integers(1, n + 1, size=301).astype(np.uint32)
    np.testing.assert_array_equal(orc.bits(orc.cpu_multiselect(v, ks, threads=4, method=method)),
                                  orc.bits(orc.select(v, ks)))


def test_segmented_oracle():
    g = np.random.default_rng(3)
    lens = [1, 5, 100, 1000]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    v = g.standard_normal(off[-1]).astype(np.float32)
    nks = [1, 3, 0, 10]
    koff = np.concatenate([[0], np.cumsum(nks)]).astype(np.int64)
    ks = np.concatenate([g.integers(1, l + 1, size=c) for l, c in zip(lens, nks)]).astype(np.uint32)
    out = orc.select_segmented(v, off, ks, koff)
    for s in range(len(lens)):
        a, b = koff[s], koff[s + 1]
        if b > a:
            np.testing.assert_array_equal(out[a:b], orc.select(v[off[s]:off[s + 1]], ks[a:b]))


@pytest.mark.parametrize("dtype", [np.float32, np.uint32])
def test_cpu_segmented_matches_oracle(dtype):
    """The OpenMP per-segment checker used at the batched benchmark's full shape
    gives the oracle's answers on the same kind of batch."""
    from ggms_b200 import datagen as D
    vals, seg_off, ks, k_off = D.segmented_batch(96, 7, 4, 16, kmax=64, dtype=dtype)
    vals[::101] = vals[3]  # duplicates across segments
    got = orc.cpu_multiselect_segmented(vals, seg_off, ks, k_off, threads=4)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select_segmented(vals, seg_off, ks, k_off)))
