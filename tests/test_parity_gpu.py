"""Bit-exact parity of the CUDA path (through the C ABI) with the CPU oracle.

Edge cases follow what the reference's differential test exercises
(DistributedSMOS/compareIterativeSMOS.cu:64-247: random problems of every
generator, every k distribution, compared with != against sort-and-choose)
plus the cases its code does not handle (NaN, signed zeros, k = 1 / k = n,
duplicate ks, tiny and ragged n).
"""
import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu

DTYPES = [np.float32, np.float64, np.uint32, np.int32]


def expected(v, ks):
    if len(v) <= (1 << 22):
        return orc.select(v, ks)
    return orc.cpu_multiselect(v, ks)  # OpenMP nth_element: the same answers, faster


def assert_bits(got, exp):
    np.testing.assert_array_equal(orc.bits(got), orc.bits(exp))


def run(ctx, v, ks, entry=None, **kw):
    d = to_device(v)
    if entry:
        return G.dropin(entry, d.data_ptr(), len(v), ks, v.dtype)
    return G.select(ctx, d.data_ptr(), len(v), ks, v.dtype, **kw)


def rand_values(dtype, n, seed):
    g = np.random.default_rng(seed)
    if np.dtype(dtype).kind == "f":
        return g.standard_normal(n).astype(dtype)
    info = np.iinfo(dtype)
    return g.integers(info.min, info.max, size=n, dtype=dtype, endpoint=True)


def rand_ks(n, count, seed):
    g = np.random.default_rng(seed + 1)
    ks = g.integers(1, n + 1, size=count).astype(np.uint32)
    ks[:2] = [1, n]                     # k = 1 (max) and k = n (min)
    if count > 4:
        ks[2] = ks[3]                   # a duplicate k
    return ks


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 1023, 1024, 1025, 65543, (1 << 20) + 3])
@pytest.mark.parametrize("assigner", [G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO])
def test_sizes(ctx, dtype, n, assigner):
    v = rand_values(dtype, n, n)
    ks = rand_ks(n, 37, n)
    assert_bits(run(ctx, v, ks, assigner=assigner), expected(v, ks))


@pytest.mark.parametrize("entry", ["bucket_multiselect", "iterative_smos"])
@pytest.mark.parametrize("dtype", DTYPES)
def test_dropin_entry_points(entry, dtype):
    v = rand_values(dtype, 100_003, 5)
    ks = rand_ks(len(v), 101, 5)
    assert_bits(run(None, v, ks, entry=entry), expected(v, ks))


def specials_f32():
    b = np.array([0x7FC00000, 0xFFC00000, 0x7F800000, 0xFF800000, 0x00000000, 0x80000000,
                  0x00000001, 0x80000001, 0x007FFFFF, 0x807FFFFF, 0x3F800000, 0xBF800000,
                  0x7FC00001, 0xFFFFFFFF], dtype=np.uint32)
    return b.view(np.float32)


@pytest.mark.parametrize("reps", [1, 1000, 50_000])
def test_nan_inf_signed_zero_subnormal_f32(ctx, reps):
    g = np.random.default_rng(reps)
    v = np.tile(specials_f32(), reps)
    v = np.concatenate([v, g.standard_normal(3 * reps).astype(np.float32)])
    g.shuffle(v)
    n = len(v)
    ks = np.arange(1, n + 1, dtype=np.uint32) if n <= 64 else rand_ks(n, 211, reps)
    for a in (G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO):
        assert_bits(run(ctx, v, ks, assigner=a), expected(v, ks))


def test_nan_inf_f64(ctx):
    g = np.random.default_rng(2)
    v = g.standard_normal(200_000)
    v[::101] = np.nan
    v[::103] = -np.inf
    v[::107] = np.inf
    v[::109] = -0.0
    v[::113] = 0.0
    v[::127] = -np.nan
    ks = rand_ks(len(v), 333, 2)
    assert_bits(run(ctx, v, ks), expected(v, ks))


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [1, 7, 5000, 1 << 20])
def test_all_equal(ctx, dtype, n):
    v = np.full(n, 3, dtype=dtype)
    ks = rand_ks(n, 9, n)
    assert_bits(run(ctx, v, ks), expected(v, ks))


@pytest.mark.parametrize("dtype", DTYPES)
def test_two_values_and_256_distinct(ctx, dtype):
    g = np.random.default_rng(9)
    n = 1 << 20
    two = np.where(g.random(n) < 0.3, 1, 2).astype(dtype)
    ks = rand_ks(n, 65, 9)
    assert_bits(run(ctx, two, ks), expected(two, ks))
    table = rand_values(dtype, 256, 10)
    d256 = table[g.integers(0, 256, size=n)]
    assert_bits(run(ctx, d256, ks), expected(d256, ks))


@pytest.mark.parametrize("dtype", DTYPES)
def test_sorted_and_reverse(ctx, dtype):
    v = np.sort(rand_values(dtype, 300_001, 11))
    ks = rand_ks(len(v), 77, 11)
    assert_bits(run(ctx, v, ks), expected(v, ks))
    r = v[::-1].copy()
    assert_bits(run(ctx, r, ks), expected(r, ks))


def test_unaligned_pointer(ctx):
    v = rand_values(np.float32, 100_000, 12)
    d = to_device(v)
    for off in (1, 2, 3):
        sub = v[off:off + 77_777]
        ks = rand_ks(len(sub), 31, off)
        got = G.select(ctx, d.data_ptr() + 4 * off, len(sub), ks, np.float32)
        assert_bits(got, expected(sub, ks))


def test_every_rank_small(ctx):
    v = rand_values(np.int32, 3000, 13)
    v[::3] = v[1]  # heavy duplicates
    ks = np.arange(1, len(v) + 1, dtype=np.uint32)
    assert_bits(run(ctx, v, ks), expected(v, ks))


def test_many_ks_random(ctx):
    v = rand_values(np.float32, 1 << 22, 14)
    ks = D.ks_uniform(len(v), 1 << 14, 14)
    assert_bits(run(ctx, v, ks), expected(v, ks))


def test_input_not_modified():
    import torch
    v = rand_values(np.float32, 1 << 20, 15)
    d = to_device(v)
    ks = rand_ks(len(v), 101, 15)
    for entry in ("bucket_multiselect", "iterative_smos"):
        G.dropin(entry, d.data_ptr(), len(v), ks, np.float32)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), v.view(np.uint32))


def test_workspace_reuse_across_shapes(ctx):
    for n, dt in [(1 << 18, np.float64), (1000, np.float32), (1 << 21, np.uint32), (17, np.int32)]:
        v = rand_values(dt, n, n)
        ks = rand_ks(n, 50, n)
        assert_bits(run(ctx, v, ks), expected(v, ks))


@pytest.mark.parametrize("bad", ["k0", "kbig", "n0", "null"])
def test_invalid_arguments(bad):
    lib = G.load()
    v = to_device(rand_values(np.float32, 100, 1))
    ks = np.array([1, 5], dtype=np.uint32)
    out = np.zeros(2, np.float32)
    import ctypes
    kp = ks.ctypes.data_as(ctypes.c_void_p)
    op = out.ctypes.data_as(ctypes.c_void_p)
    if bad == "k0":
        ks[0] = 0
        rc = lib.ggms_bucket_multiselect_f32(v.data_ptr(), 100, kp, 2, op, 148, 1024)
    elif bad == "kbig":
        ks[1] = 101
        rc = lib.ggms_bucket_multiselect_f32(v.data_ptr(), 100, kp, 2, op, 148, 1024)
    elif bad == "n0":
        rc = lib.ggms_bucket_multiselect_f32(v.data_ptr(), 0, kp, 2, op, 148, 1024)
    else:
        rc = lib.ggms_bucket_multiselect_f32(None, 100, kp, 2, op, 148, 1024)
    assert rc == G.GGMS_E_INVALID_ARG


def test_device_ks_device_out(ctx):
    import torch
    v = rand_values(np.float64, 500_000, 16)
    ks = rand_ks(len(v), 99, 16)
    d = to_device(v)
    dk = to_device(ks)
    dout = torch.empty(len(ks), dtype=torch.float64, device="cuda")
    o = G.default_opts(ks_on_device=1, out_on_device=1)
    rc = G.multiselect_ex(ctx, d.data_ptr(), len(v), dk.data_ptr(), len(ks), dout.data_ptr(),
                          np.float64, o)
    assert rc == 0
    torch.cuda.synchronize()
    assert_bits(dout.cpu().numpy(), expected(v, ks))


# ---------------------------------------------------------------- the benchmark configs
def test_config1_bucket_multiselect():
    n = 1 << 20
    v = D.uniform_f32(n, 0)
    ks = D.ks_percentiles(n, 101)
    assert_bits(run(None, v, ks, entry="bucket_multiselect"), orc.select(v, ks))


@pytest.mark.parametrize("gen,seed", [("normal_f32", 1), ("normal_f64", 2), ("uniform_u32", 3)])
def test_config2_iterative_smos(gen, seed):
    n = 1 << 26
    v = D.VALUE_GENERATORS[gen](n, seed)
    ks = D.ks_uniform_distinct(n, 1001, 11)
    assert_bits(run(None, v, ks, entry="iterative_smos"), expected(v, ks))


@pytest.mark.parametrize("gen", ["half_normal_f32", "cauchy_f32", "distinct256_f32", "sorted_desc_u32"])
def test_config3_adversarial(ctx, gen):
    n = 1 << 28
    v = D.VALUE_GENERATORS[gen](n, 21)
    ks = D.ks_top1pct(n, 1024, 21)
    exp = expected(v, ks)
    for a in (G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO):
        assert_bits(run(ctx, v, ks, assigner=a), exp)


@pytest.mark.parametrize("gen,seed", [("mixture8_f32", 31), ("lognormal_f32", 32)])
def test_config4_learned(ctx, gen, seed):
    """The learned-assigner benchmark as configured: 2^28 keys, 2^14 random ks;
    the sampled pivots, the 256-knot PL-CDF model, the default (512-knot) PL
    model, the 1-32-32-1 MLP and AUTO, every answer exact."""
    n = 1 << 28
    v = D.VALUE_GENERATORS[gen](n, seed)
    ks = D.ks_uniform(n, 1 << 14, 33)
    exp = expected(v, ks)
    for a, kw in ((G.ASSIGNER_SAMPLED, {}), (G.ASSIGNER_LEARNED_PL, {"pl_knots": 256}),
                  (G.ASSIGNER_LEARNED_PL, {}), (G.ASSIGNER_LEARNED_MLP, {}), (G.ASSIGNER_AUTO, {})):
        assert_bits(run(ctx, v, ks, assigner=a, **kw), exp)


def test_many_ks_unfused_between_steps(ctx):
    """More than 65536 ks: the steps between the passes run as separate
    launches (scan, locate, mode, children, relabel) instead of one CTA."""
    n = 1 << 22
    v = D.normal_f32(n, 71)
    ks = D.ks_uniform(n, 70_000, 72)
    ks[:3] = [1, n, n // 2]
    for a in (G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO):
        assert_bits(run(ctx, v, ks, assigner=a), orc.select(v, ks))
