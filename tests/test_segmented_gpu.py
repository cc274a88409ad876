"""Batched segmented selection and top-k through the C ABI, bit-exact against
the oracle (per segment)."""
import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu


def run_segmented(ctx, vals, seg_off, ks, k_off):
    import torch
    dv = to_device(vals)
    dso = torch.from_numpy(seg_off).cuda()
    dk = to_device(ks)
    dko = torch.from_numpy(k_off).cuda()
    tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.uint32): torch.int32}[vals.dtype]
    dout = torch.empty(len(ks), dtype=tdt, device="cuda")
    rc = G.segmented(ctx, dv.data_ptr(), dso.data_ptr(), len(seg_off) - 1, dk.data_ptr(),
                     dko.data_ptr(), dout.data_ptr(), vals.dtype)
    assert rc == 0, G.status_string(rc)
    torch.cuda.synchronize()
    out = dout.cpu().numpy()
    return out.view(np.uint32) if vals.dtype == np.uint32 else out


@pytest.mark.parametrize("dtype", [np.float32, np.uint32])
@pytest.mark.parametrize("nseg,lo,hi", [(1, 10, 10), (7, 0, 6), (64, 4, 14), (300, 10, 16)])
def test_segmented_small(ctx, dtype, nseg, lo, hi):
    vals, seg_off, ks, k_off = D.segmented_batch(nseg, nseg + lo, lo, hi, kmax=40, dtype=dtype)
    got = run_segmented(ctx, vals, seg_off, ks, k_off)
    exp = orc.select_segmented(vals, seg_off, ks, k_off)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(exp))


def test_segmented_with_empty_k_segments_and_duplicates(ctx):
    g = np.random.default_rng(5)
    lens = np.array([5, 0, 1000, 3, 70000, 1], dtype=np.int64)
    seg_off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    vals = g.integers(0, 50, size=seg_off[-1]).astype(np.float32)  # heavy duplicates
    nks = np.array([2, 0, 0, 3, 100, 1])
    k_off = np.concatenate([[0], np.cumsum(nks)]).astype(np.int64)
    ks = np.concatenate([g.integers(1, max(l, 1) + 1, size=c) for l, c in zip(lens, nks)]).astype(np.uint32)
    got = run_segmented(ctx, vals, seg_off, ks, k_off)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select_segmented(vals, seg_off, ks, k_off)))


@pytest.mark.parametrize("dtype", [np.float32, np.uint32])
def test_segmented_config5_shape(ctx, dtype):
    # the benchmark's batched shape, scaled to 2^26 elements in total for test time
    vals, seg_off, ks, k_off = D.segmented_batch(1024, 41, 10, 22, kmax=512, dtype=dtype,
                                                 total_cap=1 << 26)
    got = run_segmented(ctx, vals, seg_off, ks, k_off)
    exp = orc.select_segmented(vals, seg_off, ks, k_off)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(exp))


@pytest.mark.parametrize("dtype", [np.float32, np.uint32])
def test_segmented_config5_full(ctx, dtype):
    """The batched benchmark at its stated shape: 4096 segments, lengths
    log-uniform in [2^10, 2^24] scaled to 2^30 keys in all (the stated length
    law alone would give ~7*2^30), 1-512 random ks each; float32 segments
    alternate uniform and normal values, the second batch is uint32.  Checked
    per segment against the OpenMP per-segment multi-select, which the CPU
    tests check against the oracle."""
    vals, seg_off, ks, k_off = D.segmented_batch(4096, 41, 10, 24, kmax=512, dtype=dtype,
                                                 total_cap=1 << 30)
    assert len(seg_off) == 4097 and (1 << 30) - 4096 <= seg_off[-1] <= (1 << 30)
    got = run_segmented(ctx, vals, seg_off, ks, k_off)
    exp = orc.cpu_multiselect_segmented(vals, seg_off, ks, k_off)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(exp))


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32, np.int32])
@pytest.mark.parametrize("n,K", [(1, 1), (1000, 1000), (100_000, 17), (1 << 20, 4096), (1 << 22, 100)])
def test_topk(ctx, dtype, n, K):
    g = np.random.default_rng(n + K)
    if np.dtype(dtype).kind == "f":
        v = g.standard_normal(n).astype(dtype)
    else:
        v = g.integers(np.iinfo(dtype).min, np.iinfo(dtype).max, size=n, dtype=dtype, endpoint=True)
    d = to_device(v)
    got = G.topk(ctx, d.data_ptr(), n, K, dtype)
    exp = orc.select(v, np.arange(1, K + 1, dtype=np.uint32))
    np.testing.assert_array_equal(orc.bits(got), orc.bits(exp))


@pytest.mark.parametrize("dtype", [np.float32, np.uint32])
def test_segmented_size_classes(ctx, dtype):
    """Segments at the borders of the finishing classes (warp <= 2048 keys,
    CTA below 4096, sample-quantile bins from 4096 on), sorted, constant and
    heavily duplicated ones, each with its extreme ks and a run of ks."""
    g = np.random.default_rng(17)
    lens = [2047, 2048, 2049, 4095, 4096, 4097, 65536, 300001, 1 << 20]
    parts, ks_l = [], []
    for i, ln in enumerate(lens):
        if i % 3 == 0:
            v = np.sort(g.integers(0, 1 << 31, size=ln)).astype(np.uint32)[::-1]  # sorted descending
        elif i % 3 == 1:
            v = g.integers(0, 7, size=ln).astype(np.uint32)  # 7 distinct values
        else:
            v = g.integers(0, 1 << 32, size=ln, dtype=np.uint64).astype(np.uint32)
        if dtype == np.float32:
            v = (v.astype(np.float64) / 1000.0 - 5e5).astype(np.float32)
        parts.append(v)
        k = np.concatenate([[1, ln, (ln + 1) // 2], g.integers(1, ln + 1, size=40), np.arange(1, 20)])
        ks_l.append(k.astype(np.uint32))
    parts.append(np.full(5000, 3, dtype=np.uint32).astype(dtype))  # constant segment
    ks_l.append(np.array([1, 2500, 5000], np.uint32))
    vals = np.concatenate(parts).astype(dtype)
    seg_off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
    k_off = np.concatenate([[0], np.cumsum([len(k) for k in ks_l])]).astype(np.int64)
    ks = np.concatenate(ks_l).astype(np.uint32)
    got = run_segmented(ctx, vals, seg_off, ks, k_off)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select_segmented(vals, seg_off, ks, k_off)))


@pytest.mark.parametrize("dtype", [np.float32, np.uint32])
def test_segmented_extreme_keys(ctx, dtype):
    """Segments of every finishing class holding the smallest and largest keys
    (fp32: the NaN payloads 0xFFFFFFFF and 0x7FFFFFFF, +-Inf, +-0; uint32: 0 and
    2^32 - 1), each with its extreme ks and a run of ks."""
    g = np.random.default_rng(18)
    lens = [100, 3000, 5000, 70000, 1 << 20]
    parts, ks_l = [], []
    for ln in lens:
        if dtype == np.float32:
            v = g.standard_normal(ln).astype(np.float32)
            sp = np.array([0x7FFFFFFF, 0xFFFFFFFF, 0x7F800000, 0xFF800000, 0x80000000, 0x00000000], np.uint32)
            v[g.integers(0, ln, 12)] = sp[g.integers(0, len(sp), 12)].view(np.float32)
        else:
            v = g.integers(0, 1 << 32, size=ln, dtype=np.uint64).astype(np.uint32)
            v[g.integers(0, ln, 12)] = np.array([0, 0xFFFFFFFF], np.uint32)[g.integers(0, 2, 12)]
        parts.append(v)
        k = np.concatenate([[1, 2, ln - 1, ln, (ln + 1) // 2], g.integers(1, ln + 1, size=20)])
        ks_l.append(k.astype(np.uint32))
    vals = np.concatenate(parts).astype(dtype)
    seg_off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    k_off = np.concatenate([[0], np.cumsum([len(k) for k in ks_l])]).astype(np.int64)
    ks = np.concatenate(ks_l).astype(np.uint32)
    got = run_segmented(ctx, vals, seg_off, ks, k_off)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select_segmented(vals, seg_off, ks, k_off)))
