"""Device-side generators (include/ggms_generate.h): the reference's generator
tables (DistributedSMOS/generateProblems.cu:75-79, 438-446, 509-513) filled on the
GPU.  Checked: determinism per seed, each distribution's defining properties
(exact counts for the two-valued kinds, strata for sorted uints, moments for the
continuous ones), and exact multiselect answers on the generated vectors."""
import math

import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc

pytestmark = pytest.mark.gpu

N = 1 << 20
FLOAT_KINDS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9]


def _gen(dtype, kind, seed, n=N):
    import torch
    tdt = {np.float32: torch.float32, np.float64: torch.float64, np.uint32: torch.int32}[dtype]
    t = torch.empty(n, dtype=tdt, device="cuda")
    assert G.generate(t.data_ptr(), n, dtype, kind, seed) == 0
    torch.cuda.synchronize()
    return t, t.cpu().numpy().view(dtype)


@pytest.mark.parametrize("dtype,kind", [(np.float32, k) for k in FLOAT_KINDS]
                         + [(np.float64, 0), (np.float64, 1), (np.float64, 2), (np.uint32, 0), (np.uint32, 1),
                            (np.uint32, 2)])
def test_deterministic_per_seed(dtype, kind):
    _, a = _gen(dtype, kind, 7)
    _, b = _gen(dtype, kind, 7)
    _, c = _gen(dtype, kind, 8)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    if not (dtype == np.float32 and kind == 7) and not (dtype == np.uint32 and kind == 2):
        assert not np.array_equal(a, c)


def test_float_distributions():
    n = N
    _, u = _gen(np.float32, 0, 1)
    assert u.min() >= 0 and u.max() < 1 and abs(u.mean() - 0.5) < 0.005
    _, z = _gen(np.float32, 1, 2)
    assert np.all(np.isfinite(z)) and abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
    assert abs((np.abs(z) < 1).mean() - 0.6827) < 0.005
    _, h = _gen(np.float32, 3, 3)
    assert h.min() >= 0 and abs(h.mean() - math.sqrt(2 / math.pi)) < 0.01
    _, z100 = _gen(np.float32, 4, 4)
    assert abs(z100.std() - 100) < 1
    _, hu = _gen(np.float32, 5, 5)
    assert hu.min() >= 0 and hu.max() < 1e6 and abs(hu.mean() - 5e5) < 5e3
    _, nz = _gen(np.float32, 6, 6)
    assert (nz > 0.5).sum() == n // 5 and abs(nz[nz < 0.5].std() - 0.01) < 0.001
    _, ones = _gen(np.float32, 7, 7)
    assert np.all(ones == 1)
    _, ot = _gen(np.float32, 8, 8)
    assert (ot == 2).sum() == n // 2 and (ot == 1).sum() == n - n // 2
    assert 0.4 < (ot[: n // 2] == 2).mean() < 0.6            # twos spread, not a block
    _, ca = _gen(np.float32, 9, 9)
    assert np.all(np.isfinite(ca)) and abs(np.median(ca)) < 0.01
    assert abs((np.abs(ca) < 1).mean() - 0.5) < 0.005


def test_double_and_uint_distributions():
    n = N
    _, u = _gen(np.float64, 0, 1)
    assert u.min() >= 0 and u.max() < 1 and abs(u.mean() - 0.5) < 0.005
    _, z = _gen(np.float64, 1, 2)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
    _, w = _gen(np.uint32, 0, 3)
    assert abs(w.astype(np.float64).mean() / 2**32 - 0.5) < 0.005
    for m in (N, 1000, 3, 1):
        _, s = _gen(np.uint32, 1, 4, m)
        i = np.arange(m, dtype=np.uint64)
        lo = (i << np.uint64(32)) // np.uint64(m)
        hi = ((i + np.uint64(1)) << np.uint64(32)) // np.uint64(m)
        assert np.all(s[1:] >= s[:-1]) and np.all(s >= lo) and np.all(s <= hi)
    _, r = _gen(np.uint32, 2, 5)
    assert np.array_equal(r, (np.arange(n) % 100).astype(np.uint32))


@pytest.mark.parametrize("dtype,npow,mant,bias,mask", [
    (np.float32, 253, 23, 127, 0x80EFFFFF), (np.float64, 2045, 52, 1023, 0x800FFFFFFFFFFFFF)])
@pytest.mark.parametrize("n", [N, 300_001, 2045, 100, 1])
def test_killer_kinds(dtype, npow, mant, bias, mask, n):
    """KILLER FLOATS / DOUBLES (DistributedSMOS/generateProblems.cu:422-436,
    493-507): kind 0's draw for the same seed with the exponent masked away, sorted
    as bit patterns, then 2^(1-bias), 2^(2-bias), ... in the first slots."""
    ib = np.uint32 if dtype == np.float32 else np.uint64
    _, k = _gen(dtype, 2, 31, n)
    _, u = _gen(dtype, 0, 31, n)
    kb, ub = k.view(ib), u.view(ib)
    head = min(n, npow)
    powers = ((np.arange(head) + 1).astype(ib) << ib(mant))   # exponent fields 1 .. npow
    assert np.array_equal(kb[:head], powers)
    assert np.array_equal(k[:head], np.ldexp(np.ones(head, dtype), np.arange(head) + 1 - bias))
    want = np.sort(ub & ib(mask))[head:]
    assert np.array_equal(kb[head:], want)
    if n == N:
        assert (kb[head:] >> ib(mant) <= 1).all() and (kb[head:] >> ib(mant) == 0).any()


@pytest.mark.parametrize("n", [1, 2, 5, 1000, 65537])
def test_two_valued_counts_small_n(n):
    _, ot = _gen(np.float32, 8, 11, n)
    assert (ot == 2).sum() == n // 2 and (ot == 1).sum() == n - n // 2
    _, nz = _gen(np.float32, 6, 12, n)
    assert (nz > 0.5).sum() == n // 5


@pytest.mark.parametrize("dtype,kind", [(np.float32, k) for k in FLOAT_KINDS]
                         + [(np.float64, 0), (np.float64, 1), (np.float64, 2), (np.uint32, 0), (np.uint32, 1),
                            (np.uint32, 2)])
def test_multiselect_on_generated(dtype, kind):
    t, v = _gen(dtype, kind, 100 + kind)
    g = np.random.default_rng(kind)
    ks = np.concatenate([[1, N], g.integers(1, N + 1, size=200)]).astype(np.uint32)
    got = G.dropin("bucket_multiselect", t.data_ptr(), N, ks, dtype)
    exp = orc.select(v, ks)
    ib = np.uint64 if np.dtype(dtype).itemsize == 8 else np.uint32
    assert np.array_equal(got.view(ib), exp.view(ib))
