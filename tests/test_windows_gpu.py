"""PASS 1 windows: bit-exact answers whether the predicted k positions hold or not.

With clustered ks (the top 1% of ranks plus k = 1 and k = n) PASS 1 buckets only
the runs of buckets the sample predicts for the ks and counts every other key per
gap.  The answers must not depend on the prediction: the tests compare with the
CPU oracle with the default margin, with a margin far too small (many ks then land
in a gap, whose whole key range becomes their segment) and with windows off.
"""
import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu

N = (1 << 22) + 5

CASES = [
    ("half_normal_f32", np.float32),
    ("cauchy_f32", np.float32),
    ("distinct256_f32", np.float32),
    ("normal_f64", np.float64),
    ("uniform_u32", np.uint32),
    ("sorted_desc_u32", np.uint32),
]


@pytest.mark.parametrize("gen,dtype", CASES)
@pytest.mark.parametrize("assigner", [G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO])
@pytest.mark.parametrize("window_z", [0.0, 0.001, -1.0])
def test_windows_exact(ctx, gen, dtype, assigner, window_z):
    v = D.VALUE_GENERATORS[gen](N, 5)
    assert v.dtype == dtype
    ks = D.ks_top1pct(N, 1024, 6)
    exp = orc.select(v, ks)
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), N, ks, dtype, assigner=assigner, stats=True,
                       window_z=window_z)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(exp))
    if window_z < 0:
        assert st["window_runs"] == 0
    elif window_z == 0.0 and gen != "distinct256_f32":
        # clustered ks: the default margin keeps windows on (top run + the minimum's run)
        assert 1 <= st["window_runs"] <= 4, st


@pytest.mark.parametrize("window_z", [0.0, 0.001])
def test_windows_extremes_and_middle(ctx, window_z):
    """Runs at both ends and in the middle, with a duplicate k."""
    n = N
    v = D.VALUE_GENERATORS["normal_f32"](n, 9)
    mid = n // 2
    ks = np.array([1, 2, 3, mid, mid + 1, mid + 1, n - 2, n - 1, n], dtype=np.uint32)
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), n, ks, np.float32, stats=True, window_z=window_z)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    if window_z == 0.0:
        assert st["window_runs"] == 3, st


def test_windows_off_when_ks_spread(ctx):
    """ks spread over all ranks cover every bucket: windows stay off."""
    v = D.VALUE_GENERATORS["uniform_f32"](N, 11)
    ks = D.ks_uniform(N, 1000, 12)
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), N, ks, np.float32, stats=True)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    assert st["window_runs"] == 0


def test_windows_topk(ctx):
    n = N
    v = D.VALUE_GENERATORS["half_normal_f32"](n, 13)
    d = to_device(v)
    K = 4096
    out = G.topk(ctx, d.data_ptr(), n, K, np.float32)
    exp = np.sort(v)[::-1][:K]
    np.testing.assert_array_equal(orc.bits(out), orc.bits(exp))


def test_focused_buckets_cut_candidates(ctx):
    """With clustered ks the learned model spends most buckets on the ks' windows:
    the buckets that hold a k are smaller, so PASS 2 copies fewer candidates."""
    n = 1 << 24
    v = D.VALUE_GENERATORS["half_normal_f32"](n, 21)
    ks = D.ks_top1pct(n, 1024, 21)
    d = to_device(v)
    exp = orc.select(v, ks)
    res = {}
    for z in (0.0, -1.0):
        out, st = G.select(ctx, d.data_ptr(), n, ks, np.float32, assigner=G.ASSIGNER_LEARNED_PL,
                           stats=True, window_z=z)
        np.testing.assert_array_equal(orc.bits(out), orc.bits(exp))
        assert st["assigner_used"] == "learned_pl", st
        res[z] = st
    assert res[0.0]["window_runs"] >= 1
    assert res[0.0]["candidates"] * 3 < res[-1.0]["candidates"], res


def _f32_bits(u):
    return np.array(u, dtype=np.uint32).view(np.float32)


@pytest.mark.parametrize("case", ["specials", "all_negative", "signed_zeros"])
@pytest.mark.parametrize("window_z", [0.0, 0.001])
def test_windows_raw_bit_runs(ctx, case, window_z):
    """fp32 window runs are tested on the raw bits of the input, not on keys:
    runs within one sign, runs over both signs from the smallest key or up to
    the largest (one cyclic range of raw bits), and runs over +-0 in the middle
    (which keep the key test).  NaNs of both signs, +-Inf, +-0 and subnormals are
    among the values, and ks sit at both ends, in the top 1 % and at the sign
    boundary."""
    g = np.random.default_rng({"specials": 31, "all_negative": 32, "signed_zeros": 33}[case])
    n = N
    if case == "all_negative":
        v = -np.abs(g.standard_normal(n)).astype(np.float32)
        v[g.integers(0, n, 50)] = -0.0
    elif case == "signed_zeros":
        v = (1e-3 * g.standard_normal(n)).astype(np.float32)
        z = g.random(n)
        v[z < 0.05] = 0.0
        v[(z >= 0.05) & (z < 0.10)] = -0.0
    else:
        v = g.standard_normal(n).astype(np.float32)
        specials = _f32_bits([0x7FC00000, 0xFFC00000, 0x7F800000, 0xFF800000, 0x00000000, 0x80000000,
                              0x00000001, 0x80000001, 0x007FFFFF, 0x807FFFFF, 0x7FFFFFFF, 0xFFFFFFFF])
        for s in specials:
            v[g.integers(0, n, 40)] = s
    neg = int(np.count_nonzero(v.view(np.uint32) >> 31))  # keys below +0.0
    ks = np.concatenate([D.ks_top1pct(n, 1024, 7),
                         np.clip(n - neg + np.arange(-3, 4), 1, n),
                         [2, 3, n - 1, n - 2]]).astype(np.uint32)
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), n, ks, np.float32, stats=True, window_z=window_z)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    out_s = G.select(ctx, d.data_ptr(), n, ks, np.float32, assigner=G.ASSIGNER_SAMPLED, window_z=window_z)
    np.testing.assert_array_equal(orc.bits(out_s), orc.bits(orc.select(v, ks)))


@pytest.mark.parametrize("assigner", [G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED])
def test_windows_extreme_keys_f64(ctx, assigner):
    """fp64 with the NaN payloads whose keys are 0 and the largest 64-bit key,
    +-Inf and +-0, windows on: every bucket range of the windows and of the
    level-0 children keeps the largest key, whichever bucket the model gives it."""
    g = np.random.default_rng(34)
    n = N
    v = g.standard_normal(n)
    for s in [0x7FFFFFFFFFFFFFFF, 0xFFFFFFFFFFFFFFFF, 0x7FF8000000000000, 0xFFF8000000000000,
              0x7FF0000000000000, 0xFFF0000000000000, 0x0000000000000000, 0x8000000000000000]:
        v[g.integers(0, n, 40)] = np.array([s], dtype=np.uint64).view(np.float64)[0]
    ks = np.concatenate([D.ks_top1pct(n, 1024, 8), [2, 3, n - 1, n - 2]]).astype(np.uint32)
    d = to_device(v)
    out = G.select(ctx, d.data_ptr(), n, ks, np.float64, assigner=assigner)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))


@pytest.mark.parametrize("shape,buckets,offset", [((256, 4), 0, 0), ((256, 8), 0, 0), ((512, 2), 0, 0),
                                                  ((512, 8), 0, 0), ((1024, 2), 0, 0), ((1024, -1), 0, 0),
                                                  ((1024, -2), 0, 0), ((1024, 4), 32768, 0),
                                                  ((1024, 4), 4096, 0), ((1024, 4), 0, 1), ((1024, -1), 0, 3)])
def test_windows_raw_bit_pass_shapes(ctx, shape, buckets, offset):
    """The windowed passes in every streaming shape (register loads of 2-8
    vectors, the TMA ring, per-thread async copies), other bucket counts, and a
    vector starting 4 or 12 bytes past a 16-byte boundary (its head and tail go
    through the key test, the body through the raw-bit test): mixed-sign fp32
    with NaNs, +-Inf and +-0, ks at both ends, in the top 1 % and at the sign
    boundary; AUTO and sampled, bit-exact."""
    import torch

    g = np.random.default_rng(35)
    n = N
    v = g.standard_normal(n + offset).astype(np.float32)
    for s in [0x7FC00000, 0xFFC00000, 0x7F800000, 0xFF800000, 0x00000000, 0x80000000, 0x7FFFFFFF, 0xFFFFFFFF]:
        v[g.integers(0, n + offset, 40)] = np.array([s], dtype=np.uint32).view(np.float32)[0]
    w = v[offset:]
    neg = int(np.count_nonzero(w.view(np.uint32) >> 31))
    ks = np.concatenate([D.ks_top1pct(n, 1024, 9), np.clip(n - neg + np.arange(-2, 3), 1, n),
                         [2, n - 1]]).astype(np.uint32)
    exp = orc.select(w, ks)
    base = to_device(v)
    ptr = base.data_ptr() + 4 * offset
    kw = dict(pass_threads=shape[0], pass_unroll=shape[1])
    if buckets:
        kw["num_buckets"] = buckets
    for a in (G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED):
        out = G.select(ctx, ptr, n, ks, np.float32, assigner=a, **kw)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(orc.bits(out), orc.bits(exp))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_windows_topk_extreme_keys(ctx, dtype):
    """Top-k with the largest keys in the data (+NaN with the largest payload,
    other +NaNs, +Inf): the ks 1..K form one window run at the top of the key
    space, which must keep the largest key whatever bucket the model gives it."""
    g = np.random.default_rng(36)
    n = N
    v = g.standard_normal(n).astype(dtype)
    if dtype == np.float32:
        sp = np.array([0x7FFFFFFF, 0x7FC00000, 0x7F800000], np.uint32).view(np.float32)
    else:
        sp = np.array([0x7FFFFFFFFFFFFFFF, 0x7FF8000000000000, 0x7FF0000000000000], np.uint64).view(np.float64)
    for s in sp:
        v[g.integers(0, n, 30)] = s
    d = to_device(v)
    K = 4096
    for a in (G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED):
        out = G.topk(ctx, d.data_ptr(), n, K, dtype, assigner=a)
        np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, np.arange(1, K + 1, dtype=np.uint32))))
