"""Coarse level 0: when most buckets hold a k (many ks spread over all ranks),
level 0 copies NGRP = 256 groups of buckets, staged through shared memory in
group order.  The answers must be bit-exact against the CPU oracle whatever the
data, the pass shape (chunk sizes, unroll below 4) and the input's alignment
(the unaligned head and the tail go through the one-key-at-a-time path).

Detection: with the coarse mode on, level 0 has at most 256 active children
(the stats' active_buckets), against about one per bucket otherwise.
"""
import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu

N = (1 << 22) + 7


@pytest.mark.parametrize("gen", ["mixture8_f32", "distinct256_f32", "normal_f64", "uniform_u32",
                                 "sorted_desc_u32"])
@pytest.mark.parametrize("assigner", [G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO])
def test_coarse_exact(ctx, gen, assigner):
    v = D.VALUE_GENERATORS[gen](N, 3)
    ks = D.ks_uniform(N, 8192, 4)  # 4 ks per bucket on average: every bucket holds one
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), N, ks, v.dtype, assigner=assigner, stats=True)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    if gen != "distinct256_f32":
        assert st["active_buckets"] <= 256, st


@pytest.mark.parametrize("shape", [(256, 8), (512, 2), (1024, 2), (1024, 4), (1024, -1), (1024, -2)])
def test_coarse_pass_shapes(ctx, shape):
    v = D.VALUE_GENERATORS["lognormal_f32"](N, 5)
    ks = D.ks_uniform(N, 6000, 6)
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), N, ks, np.float32, stats=True, pass_threads=shape[0],
                       pass_unroll=shape[1])
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    assert st["active_buckets"] <= 256, st


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_coarse_unaligned_input(ctx, offset):
    """The vector starts 4, 8 or 12 bytes past a 16-byte boundary."""
    import torch

    v = D.VALUE_GENERATORS["normal_f32"](N + offset, 7)
    ks = D.ks_uniform(N, 8192, 8)
    base = to_device(v)
    ptr = base.data_ptr() + 4 * offset
    out, st = G.select(ctx, ptr, N, ks, np.float32, stats=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v[offset:], ks)))
    assert st["active_buckets"] <= 256, st


def test_few_ks_stay_fine(ctx):
    """Few ks: most buckets hold none, level 0 keeps one child per bucket."""
    v = D.VALUE_GENERATORS["uniform_f32"](N, 9)
    ks = D.ks_uniform(N, 300, 10)
    d = to_device(v)
    out, st = G.select(ctx, d.data_ptr(), N, ks, np.float32, stats=True, window_z=-1.0)
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    assert st["active_buckets"] > 256, st
