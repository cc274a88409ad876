"""Repeated calls with the same arguments: the second is captured into a CUDA
graph and later ones replay it.  The graph holds pointers, not values, so every
call must see the current contents of the vector, the ks and the segment tables.
Answers are compared bit for bit with the oracle on every call."""
import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc
from ggms_b200 import datagen as D
from conftest import to_device

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("assigner", [G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED])
def test_repeated_calls_see_new_data_and_ks(ctx, assigner):
    import torch
    lib = G.load()
    g0 = lib.ggms_context_graph_launches(ctx.ptr)
    n = (1 << 21) + 7
    d = to_device(D.half_normal_f32(n, 1))
    for call in range(5):
        v = D.VALUE_GENERATORS["normal_f32" if call % 2 else "half_normal_f32"](n, 100 + call)
        d.copy_(torch.from_numpy(v))           # same device buffer, new contents
        ks = D.ks_top1pct(n, 300, 200 + call)  # same count, new values (host ks)
        out = G.select(ctx, d.data_ptr(), n, ks, np.float32, assigner=assigner)
        np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)), err_msg=f"call {call}")
    assert lib.ggms_context_graph_launches(ctx.ptr) - g0 >= 4  # calls 2..5 replay the graph


def test_repeated_async_calls_with_device_ks(ctx):
    import torch
    n = 1 << 20
    vals = [D.uniform_f32(n, 300 + i) for i in range(4)]
    ks = D.ks_uniform(n, 257, 9)
    d = to_device(vals[0])
    dk = torch.from_numpy(ks.view(np.int32)).cuda()
    outs = [torch.empty(len(ks), dtype=torch.float32, device="cuda") for _ in vals]
    o = G.default_opts(ks_on_device=1, out_on_device=1)
    for v, out in zip(vals, outs):
        d.copy_(torch.from_numpy(v))           # stream-ordered after the previous call
        assert G.multiselect_ex(ctx, d.data_ptr(), n, dk.data_ptr(), len(ks), out.data_ptr(),
                                np.float32, o) == 0
    torch.cuda.synchronize()
    for v, out in zip(vals, outs):
        np.testing.assert_array_equal(orc.bits(out.cpu().numpy()), orc.bits(orc.select(v, ks)))


def test_repeated_segmented_calls(ctx):
    import torch
    vals, seg_off, ks, k_off = D.segmented_batch(64, 5, 8, 16, kmax=40, dtype=np.float32)
    dv = torch.from_numpy(vals).cuda()
    dso = torch.from_numpy(seg_off).cuda()
    dko = torch.from_numpy(k_off).cuda()
    dks = torch.from_numpy(ks.view(np.int32)).cuda()
    out = torch.empty(len(ks), dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(3)
    lib = G.load()
    g0 = lib.ggms_context_graph_launches(ctx.ptr)
    for call in range(4):
        v = rng.standard_normal(len(vals)).astype(np.float32)
        dv.copy_(torch.from_numpy(v))
        kk = np.concatenate([rng.integers(1, seg_off[s + 1] - seg_off[s] + 1, k_off[s + 1] - k_off[s])
                             for s in range(len(seg_off) - 1)]).astype(np.uint32)
        dks.copy_(torch.from_numpy(kk.view(np.int32)))
        rc = G.segmented(ctx, dv.data_ptr(), dso.data_ptr(), len(seg_off) - 1, dks.data_ptr(),
                         dko.data_ptr(), out.data_ptr(), np.float32)
        assert rc == 0
        torch.cuda.synchronize()
        exp = orc.select_segmented(v, seg_off, kk, k_off)
        np.testing.assert_array_equal(orc.bits(out.cpu().numpy()), orc.bits(exp), err_msg=f"call {call}")
    assert lib.ggms_context_graph_launches(ctx.ptr) - g0 >= 3


def test_autotune_single_picks_a_candidate_and_stays_exact(ctx):
    n = (1 << 22) + 1
    v = D.VALUE_GENERATORS["half_normal_f32"](n, 41)
    d = to_device(v)
    ks = D.ks_top1pct(n, 512, 42)
    exp = orc.select(v, ks)
    for _ in range(2):  # first call tunes, second uses the kept choice
        out, st = G.select(ctx, d.data_ptr(), n, ks, np.float32, stats=True, autotune=1)
        np.testing.assert_array_equal(orc.bits(out), orc.bits(exp))
        assert st["num_buckets"] in (4096, 8192, 16384), st


def test_autotune_segmented_stays_exact(ctx):
    import torch
    vals, seg_off, ks, k_off = D.segmented_batch(32, 8, 10, 16, kmax=30, dtype=np.float32)
    dv = torch.from_numpy(vals).cuda()
    dso = torch.from_numpy(seg_off).cuda()
    dko = torch.from_numpy(k_off).cuda()
    dks = torch.from_numpy(ks.view(np.int32)).cuda()
    out = torch.empty(len(ks), dtype=torch.float32, device="cuda")
    exp = orc.select_segmented(vals, seg_off, ks, k_off)
    o = G.default_opts(autotune=1)
    for _ in range(2):
        rc = G.segmented(ctx, dv.data_ptr(), dso.data_ptr(), len(seg_off) - 1, dks.data_ptr(),
                         dko.data_ptr(), out.data_ptr(), np.float32, o)
        assert rc == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(orc.bits(out.cpu().numpy()), orc.bits(exp))


@pytest.mark.parametrize("gen,assigner", [("normal_f32", G.ASSIGNER_SAMPLED), ("distinct256_f32", G.ASSIGNER_AUTO)])
def test_replayed_graph_runs_refinement_levels_when_needed(ctx, gen, assigner):
    """Spread ks and duplicates make segments too big for the shared-memory select, so
    refinement levels must run inside the replayed graph (their IF nodes open)."""
    import torch
    n = 1 << 23
    d = to_device(D.VALUE_GENERATORS[gen](n, 1))
    for call in range(4):
        v = D.VALUE_GENERATORS[gen](n, 50 + call)
        d.copy_(torch.from_numpy(v))
        ks = D.ks_uniform(n, 4096, 60 + call)
        out, st = None, None
        out = G.select(ctx, d.data_ptr(), n, ks, np.float32, assigner=assigner)
        np.testing.assert_array_equal(orc.bits(out), orc.bits(orc.select(v, ks)), err_msg=f"call {call}")
    _, st = G.select(ctx, d.data_ptr(), n, ks, np.float32, assigner=assigner, stats=True)
    assert st["levels"] >= 1, st
