"""Context API through the C ABI: the device-side status of asynchronous calls,
the options layout without pl_knots, per-phase profiling, the counted passes
and the learned model's knot count."""
import ctypes

import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu


def _dev_call(ctx, d, n, dk, nk, dout, **kw):
    o = G.default_opts(ks_on_device=1, out_on_device=1, **kw)
    return G.multiselect_ex(ctx, d.data_ptr(), n, dk.data_ptr(), nk, dout.data_ptr(), np.float32, o)


def test_status_reports_device_k_out_of_range():
    """ks and answers in device memory: the call returns at once, and a k outside
    [1, n] is reported by ggms_context_status, not by the return value."""
    import torch
    ctx = G.Context(0)
    n = 100_000
    v = np.random.default_rng(1).standard_normal(n).astype(np.float32)
    d = to_device(v)
    dout = torch.empty(4, dtype=torch.float32, device="cuda")
    good = np.array([1, 7, n, 500], dtype=np.uint32)
    bad = np.array([1, 7, n + 1, 500], dtype=np.uint32)
    assert ctx.status() == G.GGMS_OK  # nothing enqueued yet
    assert _dev_call(ctx, d, n, to_device(bad), 4, dout) == G.GGMS_OK
    assert ctx.status() == G.GGMS_E_INVALID_ARG
    assert _dev_call(ctx, d, n, to_device(good), 4, dout) == G.GGMS_OK
    assert ctx.status(torch.cuda.current_stream().cuda_stream) == G.GGMS_OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(orc.bits(dout.cpu().numpy()), orc.bits(orc.select(v, good)))
    # the same call again replays its captured graph: the status is still read
    dk_bad = to_device(bad)
    for _ in range(3):
        assert _dev_call(ctx, d, n, dk_bad, 4, dout) == G.GGMS_OK
        assert ctx.status() == G.GGMS_E_INVALID_ARG
    ctx.close()


def test_status_of_segmented_call():
    import torch
    ctx = G.Context(0)
    vals, seg_off, ks, k_off = D.segmented_batch(8, 3, 6, 14, kmax=5)
    ks = ks.copy()
    ks[int(k_off[3])] = np.uint32(seg_off[4] - seg_off[3] + 1)  # one past segment 3's length
    dout = torch.empty(len(ks), dtype=torch.float32, device="cuda")
    dv, dso, dk, dko = (to_device(vals), torch.from_numpy(seg_off).cuda(), to_device(ks),
                        torch.from_numpy(k_off).cuda())
    rc = G.segmented(ctx, dv.data_ptr(), dso.data_ptr(), 8, dk.data_ptr(), dko.data_ptr(),
                     dout.data_ptr(), np.float32)
    assert rc == G.GGMS_OK
    assert ctx.status() == G.GGMS_E_INVALID_ARG
    ctx.close()


def test_options_without_pl_knots_accepted():
    """A caller built against the options layout that ends at `stats` (struct_size
    = offset of pl_knots) is accepted; any other size is rejected."""
    import torch
    n = 1 << 16
    v = np.random.default_rng(2).random(n, dtype=np.float32)
    d = to_device(v)
    ks = np.array([1, 2, 3, n], dtype=np.uint32)
    out = np.empty(4, np.float32)
    st = G.Stats()
    st.model_segments = -7  # an old caller's stats struct has no such field: left untouched
    o = G.default_opts(stats=ctypes.pointer(st))
    o.struct_size = G.Opts.pl_knots.offset
    assert G.multiselect_ex(None, d.data_ptr(), n, ks, 4, out, np.float32, o) == G.GGMS_OK
    np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)))
    assert st.full_passes == 2 and st.model_segments == -7
    o.struct_size = G.Opts.pl_knots.offset + 4
    assert G.multiselect_ex(None, d.data_ptr(), n, ks, 4, out, np.float32, o) == G.GGMS_E_INVALID_ARG


def test_phase_times_cover_the_call():
    import torch
    ctx = G.Context(0)
    n = 1 << 24
    v = D.half_normal_f32(n, 5)
    ks = D.ks_top1pct(n, 256, 5)
    d, dk = to_device(v), to_device(ks)
    dout = torch.empty(len(ks), dtype=torch.float32, device="cuda")
    G.load().ggms_context_profile(ctx.ptr, 1)
    for _ in range(3):
        assert _dev_call(ctx, d, n, dk, len(ks), dout) == G.GGMS_OK
    p1 = (ctypes.c_float * 1)()
    calls = ctx.phase_times(8)
    assert len(calls) == 3
    for c in calls:
        assert set(c) == set(G.PHASES)
        assert all(t >= 0.0 for t in c.values())
        assert c["pass1"] > 0.0 and c["pass2"] > 0.0
    assert G.load().ggms_context_pass_times(ctx.ptr, p1, None, None, 1) == 0  # ring drained
    torch.cuda.synchronize()
    np.testing.assert_array_equal(orc.bits(dout.cpu().numpy()), orc.bits(orc.select(v, ks)))
    ctx.close()


@pytest.mark.parametrize("assigner", [G.ASSIGNER_SAMPLED, G.ASSIGNER_AUTO])
def test_full_passes_are_counted(ctx, assigner):
    n = 1 << 22
    v = D.normal_f32(n, 9)
    ks = D.ks_uniform(n, 300, 9)
    got, st = G.select(ctx, to_device(v).data_ptr(), n, ks, np.float32, assigner=assigner, stats=True)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select(v, ks)))
    assert st["full_passes"] == 2


def test_segmented_passes_are_counted():
    """Only caller segments of 4096 keys or more go through the level-0 count and
    copy; a batch of small segments is finished straight from the input."""
    import torch
    ctx = G.Context(0)
    for lo, hi, want in ((6, 11, 0), (13, 16, 2)):
        vals, seg_off, ks, k_off = D.segmented_batch(40, 11, lo, hi, kmax=8)
        if hi <= 11:
            assert (np.diff(seg_off) < 4096).all()
        st = G.Stats()
        o = G.default_opts(stats=ctypes.pointer(st))
        dout = torch.empty(len(ks), dtype=torch.float32, device="cuda")
        dv, dso, dk, dko = (to_device(vals), torch.from_numpy(seg_off).cuda(), to_device(ks),
                            torch.from_numpy(k_off).cuda())
        rc = G.segmented(ctx, dv.data_ptr(), dso.data_ptr(), len(seg_off) - 1, dk.data_ptr(),
                         dko.data_ptr(), dout.data_ptr(), np.float32, o)
        assert rc == G.GGMS_OK
        assert st.full_passes == want
        np.testing.assert_array_equal(orc.bits(dout.cpu().numpy()),
                                      orc.bits(orc.select_segmented(vals, seg_off, ks, k_off)))
    ctx.close()


@pytest.mark.parametrize("knots", [16, 256, 1024])
@pytest.mark.parametrize("assigner", [G.ASSIGNER_LEARNED_PL, G.ASSIGNER_LEARNED_MLP])
def test_pl_knots_option(ctx, assigner, knots):
    n = 1 << 22
    v = D.mixture8_f32(n, 4)
    ks = D.ks_uniform(n, 777, 4)
    got, st = G.select(ctx, to_device(v).data_ptr(), n, ks, np.float32, assigner=assigner, stats=True,
                       pl_knots=knots, imbalance_bound=1e9, num_buckets=8192)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select(v, ks)))
    assert st["assigner_used"] == G.ASSIGNER_NAMES[assigner]
    # quantile knots, deduplicated; an atom may add one knot
    assert knots // 2 <= st["model_segments"] <= knots + 8


def test_pl_knots_out_of_range_rejected(ctx):
    n = 4096
    v = np.arange(n, dtype=np.float32)
    for bad in (1, 15, 1025):
        with pytest.raises(G.GGMSError):
            G.select(ctx, to_device(v).data_ptr(), n, np.array([1], np.uint32), np.float32,
                     assigner=G.ASSIGNER_LEARNED_PL, pl_knots=bad)
