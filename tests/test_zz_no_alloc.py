"""ggms_multiselect_noalloc_f32: the entry point that allocates nothing.

Argument checks run on the host before any CUDA call, so the rejection tests
need no GPU.  The GPU test makes calls back to back on one stream (no sync
between them, so the second reuses the scratch region right after the first)
and compares every answer with the context-based entry point
ggms_multiselect_f32_ex on the same inputs.  Tolerance: none -- both return an
element of the input, so the answers must be bit-identical.
"""
import numpy as np
import pytest

import ggms_b200 as G
from ggms_b200 import datagen as D

from conftest import to_device

FAKE_DEV_PTR = 1 << 20  # aligned and non-null; never dereferenced by the host checks


def test_noalloc_rejects_more_ks_than_its_scratch_holds():
    ks = np.arange(1, G.NOALLOC_MAX_KS + 2, dtype=np.uint32)
    rc = G.multiselect_noalloc_f32(FAKE_DEV_PTR, 10_000, ks, FAKE_DEV_PTR)
    assert rc == G.GGMS_E_UNSUPPORTED
    assert G.status_string(rc) == "unsupported"


@pytest.mark.parametrize("n,ks,d_in,d_out", [
    (0, [1], FAKE_DEV_PTR, FAKE_DEV_PTR),             # empty vector
    (1 << 32, [1], FAKE_DEV_PTR, FAKE_DEV_PTR),       # counts are 32-bit
    (100, [0], FAKE_DEV_PTR, FAKE_DEV_PTR),           # k is 1-based
    (100, [101], FAKE_DEV_PTR, FAKE_DEV_PTR),         # k > n
    (100, [5], 0, FAKE_DEV_PTR),                      # null input
    (100, [5], FAKE_DEV_PTR, 0),                      # null output
    (100, [5], FAKE_DEV_PTR + 2, FAKE_DEV_PTR),       # misaligned input
    (100, [5], FAKE_DEV_PTR, FAKE_DEV_PTR + 1),       # misaligned output
])
def test_noalloc_rejects_invalid_arguments(n, ks, d_in, d_out):
    assert G.multiselect_noalloc_f32(d_in, n, np.array(ks, np.uint32), d_out) == G.GGMS_E_INVALID_ARG


def test_noalloc_no_ks_is_a_no_op():
    assert G.multiselect_noalloc_f32(FAKE_DEV_PTR, 100, np.zeros(0, np.uint32), FAKE_DEV_PTR) == G.GGMS_OK


def _special_mixture(n, seed):
    v = D.mixture8_f32(n, seed)
    rng = np.random.default_rng(seed)
    v[rng.integers(0, n, n // 8)] = np.float32(1.5)            # a heavy atom
    idx = rng.integers(0, n, 64)
    v[idx[:16]] = np.inf
    v[idx[16:32]] = -np.inf
    v[idx[32:40]] = np.float32(-0.0)
    v[idx[40:48]] = np.float32(0.0)
    v[idx[48:64]] = np.nan
    return v


@pytest.mark.gpu
def test_noalloc_matches_multiselect_ex_on_calls_in_a_row(ctx):
    import torch

    rng = np.random.default_rng(7)
    na = (1 << 22) + 3
    va = D.half_normal_f32(na, 41)
    ka = np.concatenate([[1, na, na // 2, 2, 2], rng.integers(1, na + 1, G.NOALLOC_MAX_KS - 5)])
    ka = ka.astype(np.uint32)                                  # the maximum number of ks, duplicates included
    nb = 1_000_003
    vb = _special_mixture(nb, 43)
    kb = rng.integers(1, nb + 1, 300).astype(np.uint32)
    cases = [(va, ka), (vb, kb), (va, ka[::-1].copy()), (np.array([2.5], np.float32), np.array([1], np.uint32))]

    dev = [to_device(v) for v, _ in cases]
    outs = [torch.empty(len(k), dtype=torch.float32, device="cuda") for _, k in cases]
    expected = []
    for d, (v, k) in zip(dev, cases):
        expected.append(G.select(ctx, d.data_ptr(), len(v), k, np.float32))  # the context-based entry point
    torch.cuda.synchronize()

    # first call: does the one-time set-up
    assert G.multiselect_noalloc_f32(dev[0].data_ptr(), len(cases[0][0]), cases[0][1], outs[0].data_ptr()) == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    # the calls in a row: one stream, no sync between them
    for d, o, (v, k) in zip(dev, outs, cases):
        assert G.multiselect_noalloc_f32(d.data_ptr(), len(v), k, o.data_ptr()) == G.GGMS_OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, "device memory changed across no-allocation calls"

    for o, ref, (v, k) in zip(outs, expected, cases):
        got = o.cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
        # and the plain definition: the k-th largest of the sorted keys
        keys = v.view(np.uint32) ^ np.where(v.view(np.uint32) >> 31 == 1, np.uint32(0xFFFFFFFF), np.uint32(0x80000000))
        srt = np.sort(keys)
        want_keys = srt[len(v) - k.astype(np.int64)]
        got_keys = got.view(np.uint32) ^ np.where(got.view(np.uint32) >> 31 == 1, np.uint32(0xFFFFFFFF),
                                                   np.uint32(0x80000000))
        np.testing.assert_array_equal(got_keys, want_keys)
