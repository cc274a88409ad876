#!/usr/bin/env python3
"""Benchmark: exact multiple order statistics on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload headline|spread|c4_mixture|c4_lognormal|c5_f32|c5_u32]

Workloads (each a step = one call over one batch of synthetic input, seeded):
  headline      2^28 fp32 half-normal, 1026 ks: 1024 distinct ks among the top
                1% of ranks plus k = 1 and k = n (the adversarial single-vector
                configuration at the headline's n and K).  The default.
  spread        the same vector, 1024 ks uniform over all ranks by the
                reference's "Uniform Random Ks" rule
                (DistributedSMOS/generateProblems.cu:584-600).
  c4_mixture    2^28 fp32 from a mixture of 8 Gaussians, 2^14 random ks
  c4_lognormal  2^28 fp32 lognormal(0, 2), 2^14 random ks
  c5_f32        4096 segments, lengths log-uniform in [2^10, 2^24] scaled to
                2^30 keys in all, 1-512 random ks each, fp32 uniform / normal
                alternating per segment
  c5_u32        the same shape, uint32 uniform

ours:
  value  elements/s with the vector, the ks and the answers resident in HBM
         (one _ex / segmented call per step, no host sync inside the timed
         region); the default assigner (AUTO: learned PL-CDF, sampled-pivot
         fallback).  Repeated calls replay the library's captured CUDA graph.
  e2e    the same metric through the reference-facing C ABI with host buffers:
         single-vector workloads call ggms_bucket_multiselect_f32 (host ks in,
         host answers out, the vector a device pointer -- the reference's own
         API and timing protocol, DistributedSMOS/iterativeSMOSTimingFunctions.cu:
         134-156); the batched workloads copy their ks and offsets host->device
         and the answers device->host inside every step.
  sampled / pl256 / mlp   the same timed loop with the other assigners.
  spread (headline only)  the spread workload's device-timed value, beside it.
  phases mean per-phase device times of profiled calls (ggms_context_phase_times).
reference:
  the reference's own bucketMultiselectWrapper, compiled unmodified from its
  sources for sm_100a (oracle/_ref), timed with its own protocol on the same
  GPU.  For the batched workloads (the reference has no batched API) a loop of
  per-segment calls over a seeded subset of the segments, scaled to all 4096.
N > 1: independent replicas (the path does not shard: one problem per GPU),
timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(REPO, "ggms-distributed_b200"), os.path.join(REPO, "oracle")]

METRIC = "elements/s & HBM GB/s, n=2^28 fp32, 1024 ks: learned vs sampled buckets, exact"
N_HEAD = 1 << 28

WORKLOADS = {
    "headline": dict(kind="single", gen="half_normal_f32", n=N_HEAD, ks="top1pct", nk=1024, seed_v=21,
                     seed_k=21, desc="half_normal_f32 n=2^28, 1024 top-1% ks + k=1 + k=n (exact k-th largest)"),
    "spread": dict(kind="single", gen="half_normal_f32", n=N_HEAD, ks="uniform_random", nk=1024, seed_v=21,
                   seed_k=21, desc="half_normal_f32 n=2^28, 1024 uniform-random ks (exact k-th largest)"),
    "c4_mixture": dict(kind="single", gen="mixture8_f32", n=N_HEAD, ks="uniform", nk=1 << 14, seed_v=31,
                       seed_k=33, desc="mixture of 8 Gaussians f32 n=2^28, 2^14 random ks (exact)"),
    "c4_lognormal": dict(kind="single", gen="lognormal_f32", n=N_HEAD, ks="uniform", nk=1 << 14, seed_v=32,
                         seed_k=33, desc="lognormal(0,2) f32 n=2^28, 2^14 random ks (exact)"),
    "c5_f32": dict(kind="segmented", dtype=np.float32, nseg=4096, seed=41, total=1 << 30,
                   desc="4096 f32 segments (uniform/normal), log-uniform lengths scaled to 2^30 keys, "
                        "1-512 ks each (exact)"),
    "c5_u32": dict(kind="segmented", dtype=np.uint32, nseg=4096, seed=41, total=1 << 30,
                   desc="4096 uint32 segments, log-uniform lengths scaled to 2^30 keys, 1-512 ks each (exact)"),
}

# DRAM bytes (read + write) per input element of the two passes, from one ncu
# capture of the same kernels on the same half-normal workload at n = 2^26
# (profiles/l0_passes_half_normal_f32_n26.md); both passes read the input once,
# so the traffic of a launch grows in proportion to n.
PASS_TRAFFIC_PER_ELEM = {"l0_count": (268579072 + 3161088) / 2**26,
                         "l0_compact": (272013824 + 3980544) / 2**26}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(os.environ.get("GGMS_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"ggms_clocks_gpu{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                c = [x.strip() for x in line.split(",")]
                if len(c) < 9:
                    continue
                try:
                    sm.append(float(c[1]))
                    mx = float(c[2])
                except ValueError:
                    continue
                for nm, val in zip(names, c[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ inputs
def single_inputs(w):
    from ggms_b200 import datagen as D
    from ggms_b200 import harness as H
    v = D.VALUE_GENERATORS[w["gen"]](w["n"], w["seed_v"])
    if w["ks"] == "top1pct":
        ks = D.ks_top1pct(w["n"], w["nk"], w["seed_k"])
    elif w["ks"] == "uniform_random":
        ks = H.ks_uniform_random(w["nk"], w["n"], w["seed_k"])
    else:
        ks = D.ks_uniform(w["n"], w["nk"], w["seed_k"])
    return v, ks


def segmented_inputs(w):
    from ggms_b200 import datagen as D
    return D.segmented_batch(w["nseg"], w["seed"], 10, 24, kmax=512, dtype=w["dtype"], total_cap=w["total"])


def config_of(w, world):
    """The config dict, identical in both arms."""
    if w["kind"] == "single":
        return {"workload": w["desc"], "n": w["n"], "num_ks": int(w["nk"] + (2 if w["ks"] == "top1pct" else 0)),
                "l2": "inputs larger than L2 (1 GiB per pass)", "parallelism": f"replicas x{world}"}
    return {"workload": w["desc"], "n": w["total"], "segments": w["nseg"],
            "l2": "inputs larger than L2 (4 GiB per pass)", "parallelism": f"replicas x{world}"}


# ------------------------------------------------------------------ helpers
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.backend == "auto" else args.backend
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a per-rank device time over all ranks (every rank gets it).
    device None: a CPU tensor (gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(elems_per_rank: int, world: int, ms_total_max: float, steps: int) -> float:
    """elements/s of the whole job: every rank processed elems_per_rank per step;
    the slowest rank's time bounds the job (weak scaling, replicas)."""
    return world * elems_per_rank / (ms_total_max / steps / 1e3)


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def time_loop(fn, steps, warmup, stream, world, dev):
    """Device time of `steps` calls (events on the launching stream), max over ranks."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier(world, dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world, dev)
    ms = e0.elapsed_time(e1)
    return max_over_ranks(ms, world, dev)


def cpu_baseline_single(v, w):
    """Both multithreaded CPU methods of the oracle library on a bounded sample
    (the first 2^26 elements, the workload's k rule at that length); the faster
    one is the reported baseline."""
    import ggms_oracle as orc
    from ggms_b200 import datagen as D
    from ggms_b200 import harness as H
    threads = orc.cpu_threads()
    sample_n = min(len(v), 1 << 26)
    sv = v[:sample_n]
    if w["ks"] == "top1pct":
        sks = D.ks_top1pct(sample_n, w["nk"], w["seed_k"])
    elif w["ks"] == "uniform_random":
        sks = H.ks_uniform_random(w["nk"], sample_n, w["seed_k"])
    else:
        sks = D.ks_uniform(sample_n, w["nk"], w["seed_k"])
    rates = {}
    for method, name in ((0, "parallel sort-and-choose (__gnu_parallel::sort)"),
                         (1, "recursive std::nth_element multi-select (OpenMP tasks)")):
        t0 = time.perf_counter()
        orc.cpu_multiselect(sv, sks, threads=threads, method=method)
        dt = time.perf_counter() - t0
        reps = max(1, min(5, int(6.0 / max(dt, 1e-3))))
        t0 = time.perf_counter()
        for _ in range(reps):
            orc.cpu_multiselect(sv, sks, threads=threads, method=method)
        rates[name] = (sample_n / ((time.perf_counter() - t0) / reps), reps)
    best = max(rates, key=lambda k: rates[k][0])
    return {"value": rates[best][0], "unit": "elements/s", "cores": threads, "kind": "port",
            "method": best, "methods": {k: r for k, (r, _) in rates.items()},
            "sample": f"first 2^26 elements of the same input, {len(sks)} ks by the workload's k rule at that "
                      f"length; the faster of the two OpenMP methods ({rates[best][1]} reps)"}


def cpu_baseline_segmented(vals, seg_off, ks, k_off):
    """The OpenMP per-segment multi-select on a bounded sample: the first 512 segments."""
    import ggms_oracle as orc
    threads = orc.cpu_threads()
    m = min(512, len(seg_off) - 1)
    so = seg_off[:m + 1]
    ko = k_off[:m + 1]
    sv, sk = vals[:so[-1]], ks[:ko[-1]]
    t0 = time.perf_counter()
    orc.cpu_multiselect_segmented(sv, so, sk, ko, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": float(so[-1]) / dt, "unit": "elements/s", "cores": threads, "kind": "port",
            "sample": f"the first {m} segments ({int(so[-1])} keys, {int(ko[-1])} ks); OpenMP per-segment "
                      f"std::nth_element multi-select, segments spread over the threads"}


# ------------------------------------------------------------------ ours: one vector
def run_ours_single(args, w, world, rank, local):
    import torch
    import ggms_b200 as G
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    lib = G.load()
    n = w["n"]
    v, ks = single_inputs(w)
    nk = len(ks)
    d_v = torch.from_numpy(v).to(dev)
    d_k = torch.from_numpy(ks.view(np.int32)).to(dev)
    d_out = torch.empty(nk, dtype=torch.float32, device=dev)
    ctx = G.Context(local)

    def call(assigner, d_keys=d_k, count=nk, **kw):
        o = G.default_opts(assigner=assigner, ks_on_device=1, out_on_device=1, **kw)

        def f():
            rc = G.multiselect_ex(ctx, d_v.data_ptr(), n, d_keys.data_ptr(), count, d_out.data_ptr(),
                                  np.float32, o, stream.cuda_stream)
            if rc:
                raise G.GGMSError(rc, "ggms_multiselect_f32_ex")
        return f

    variants = [("auto", G.ASSIGNER_AUTO, {}), ("sampled", G.ASSIGNER_SAMPLED, {})]
    if w["ks"] == "uniform" and w["nk"] >= (1 << 14):  # the learned-assigner configuration
        variants += [("pl256", G.ASSIGNER_LEARNED_PL, {"pl_knots": 256}), ("mlp", G.ASSIGNER_LEARNED_MLP, {})]

    # correctness of this very run (answers are exact or the bench fails)
    exp = None
    if rank == 0:
        import ggms_oracle as orc
        exp = orc.cpu_multiselect(v, ks)
        for name, a, kw in variants:
            call(a, **kw)()
            torch.cuda.synchronize()
            if ctx.status() != 0:
                raise SystemExit(f"device status {ctx.status()} ({name})")
            got = d_out.cpu().numpy()
            if not np.array_equal(got.view(np.uint32), exp.view(np.uint32)):
                raise SystemExit(f"answers differ from the oracle (assigner {name})")

    # value: device-resident, AUTO
    launches0 = lib.ggms_context_launches(ctx.ptr)
    graphs0 = lib.ggms_context_graph_launches(ctx.ptr)
    with Clocks(local) as clk:
        ms = time_loop(call(G.ASSIGNER_AUTO), args.steps, args.warmup, stream, world, dev)
    launches = (lib.ggms_context_launches(ctx.ptr) - launches0) * args.steps // (args.steps + args.warmup)
    graph_calls = lib.ggms_context_graph_launches(ctx.ptr) - graphs0
    if ctx.status() != 0:
        raise SystemExit(f"device status {ctx.status()} in the timed loop")
    # phase times: the same calls with the profiling hooks on (events at the
    # phase boundaries on the call's stream; such calls run without the graph)
    lib.ggms_context_profile(ctx.ptr, 1)
    time_loop(call(G.ASSIGNER_AUTO), args.steps, args.warmup, stream, world, dev)
    lib.ggms_context_profile(ctx.ptr, 0)
    ph = ctx.phase_times(args.steps + args.warmup)[args.warmup:]
    phases = {k: statistics.mean(c[k] for c in ph) for k in G.PHASES} if ph else {}
    ms_step = ms / args.steps
    value = whole_job_rate(n, world, ms, args.steps)

    # the other assigners, same loop, with their statistics
    others = {}
    for name, a, kw in variants:
        _, st = G.select(ctx, d_v.data_ptr(), n, ks, np.float32, assigner=a, stats=True, **kw)
        if name == "auto":
            others[name] = {"stats": st}
            continue
        ms_a = time_loop(call(a, **kw), args.steps, args.warmup, stream, world, dev)
        others[name] = {"value": world * n / (ms_a / args.steps / 1e3), "ms_per_step": ms_a / args.steps,
                        "stats": st}

    # e2e through the reference-facing drop-in (host ks, host answers)
    ks_host = np.ascontiguousarray(ks)
    out_host = np.empty(nk, dtype=np.float32)
    kp = ks_host.ctypes.data_as(ctypes.c_void_p)
    op = out_host.ctypes.data_as(ctypes.c_void_p)

    def dropin():
        rc = lib.ggms_bucket_multiselect_f32(d_v.data_ptr(), n, kp, nk, op, 148, 1024)
        if rc:
            raise G.GGMSError(rc, "ggms_bucket_multiselect_f32")
    ms_e2e = time_loop(dropin, args.steps, args.warmup, torch.cuda.default_stream(), world, dev)
    if exp is not None and not np.array_equal(out_host.view(np.uint32), exp.view(np.uint32)):
        raise SystemExit("drop-in answers differ from the oracle")
    # ... and with the vector upload from pinned host memory in every step
    pinned = torch.from_numpy(v).pin_memory()
    d_v2 = torch.empty_like(d_v)

    def dropin_h2d():
        d_v2.copy_(pinned, non_blocking=True)
        rc = lib.ggms_bucket_multiselect_f32(d_v2.data_ptr(), n, kp, nk, op, 148, 1024)
        if rc:
            raise G.GGMSError(rc, "ggms_bucket_multiselect_f32")
    e2e_steps = max(3, min(args.steps, 5))
    ms_e2e_h2d = time_loop(dropin_h2d, e2e_steps, 1, torch.cuda.default_stream(), world, dev)
    del pinned, d_v2

    # the spread-k workload beside the headline (same vector, device-timed)
    spread = None
    if args.workload == "headline":
        ws = WORKLOADS["spread"]
        _, ks_s = single_inputs(ws)
        d_ks = torch.from_numpy(ks_s.view(np.int32)).to(dev)
        f = call(G.ASSIGNER_AUTO, d_keys=d_ks, count=len(ks_s))
        f()
        torch.cuda.synchronize()
        exact = None
        if rank == 0:
            import ggms_oracle as orc
            exact = bool(np.array_equal(d_out[:len(ks_s)].cpu().numpy().view(np.uint32),
                                        orc.cpu_multiselect(v, ks_s).view(np.uint32)))
        ms_sp = time_loop(f, args.steps, args.warmup, stream, world, dev)
        _, st_sp = G.select(ctx, d_v.data_ptr(), n, ks_s, np.float32, stats=True)
        peak, _ = peaks()
        spread = {"workload": ws["desc"], "value": world * n / (ms_sp / args.steps / 1e3), "unit": "elements/s",
                  "ms_per_step": ms_sp / args.steps, "exact_vs_oracle": exact,
                  "two_pass_frac": 2 * n * 4 / (ms_sp / args.steps / 1e3) / 1e9 / peak, "stats": st_sp}

    peak, peak_kind = peaks()
    bytes_pass = n * 4
    t1, t2 = phases.get("pass1", float("nan")), phases.get("pass2", float("nan"))
    dom_name, dom_ms = ("l0_count", t1) if t1 >= t2 else ("l0_compact", t2)
    achieved = bytes_pass / (dom_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic: seeded {w['gen']} fp32 (numpy PCG64, seed {w['seed_v']}), generated on the host",
        "config": config_of(w, world),
        "assigner": "auto (learned PL-CDF, sampled-pivot fallback)",
        "hbm_gbs_alg": world * 2 * bytes_pass / (ms_step / 1e3) / 1e9,
        "passes": others["auto"]["stats"]["full_passes"],
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": PASS_TRAFFIC_PER_ELEM[dom_name] * n,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at n=2^26, "
                                       "scaled by n (profiles/l0_passes_half_normal_f32_n26.md)",
                     "bytes_per_launch": bytes_pass,
                     "pass1_ms": t1, "pass2_ms": t2,
                     "two_pass_frac": 2 * bytes_pass / (ms_step / 1e3) / 1e9 / peak},
        "phases_ms": phases,
        "e2e": {"value": world * n / (ms_e2e / args.steps / 1e3), "unit": "elements/s",
                "h2d_bytes_per_step": 4 * nk, "d2h_bytes_per_step": 4 * nk,
                "api": "ggms_bucket_multiselect_f32 (vector device-resident, as the reference's API)"},
        "e2e_incl_vector_h2d": {"value": world * n / (ms_e2e_h2d / e2e_steps / 1e3),
                                "unit": "elements/s", "h2d_bytes_per_step": 4 * n + 4 * nk,
                                "d2h_bytes_per_step": 4 * nk},
        "stats": others["auto"]["stats"],
        "gpu_launches": int(launches),
        "graph_replays": int(graph_calls),
        "clocks": clk.summary(),
    }
    for name in others:
        if name != "auto":
            line[name] = others[name]
    if spread is not None:
        line["spread"] = spread
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_single(v, w)
    ctx.close()
    return line


# ------------------------------------------------------------------ ours: batched
def run_ours_segmented(args, w, world, rank, local):
    import torch
    import ggms_b200 as G
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    lib = G.load()
    vals, seg_off, ks, k_off = segmented_inputs(w)
    n = int(seg_off[-1])
    nseg = len(seg_off) - 1
    tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.uint32): torch.int32}[vals.dtype]
    view = {np.dtype(np.uint32): np.int32}.get(vals.dtype)
    d_v = torch.from_numpy(vals.view(view) if view else vals).to(dev)
    d_so = torch.from_numpy(seg_off).to(dev)
    d_k = torch.from_numpy(ks.view(np.int32)).to(dev)
    d_ko = torch.from_numpy(k_off).to(dev)
    d_out = torch.empty(len(ks), dtype=tdt, device=dev)
    ctx = G.Context(local)

    def f():
        rc = G.segmented(ctx, d_v.data_ptr(), d_so.data_ptr(), nseg, d_k.data_ptr(), d_ko.data_ptr(),
                         d_out.data_ptr(), vals.dtype, None, stream.cuda_stream)
        if rc:
            raise G.GGMSError(rc, "ggms_multiselect_segmented")

    exp = None
    if rank == 0:
        import ggms_oracle as orc
        exp = orc.cpu_multiselect_segmented(vals, seg_off, ks, k_off)
        f()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(vals.dtype)
        if ctx.status() != 0 or not np.array_equal(orc.bits(got), orc.bits(exp)):
            raise SystemExit("batched answers differ from the per-segment CPU multi-select")
    launches0 = lib.ggms_context_launches(ctx.ptr)
    graphs0 = lib.ggms_context_graph_launches(ctx.ptr)
    with Clocks(local) as clk:
        ms = time_loop(f, args.steps, args.warmup, stream, world, dev)
    launches = (lib.ggms_context_launches(ctx.ptr) - launches0) * args.steps // (args.steps + args.warmup)
    graph_calls = lib.ggms_context_graph_launches(ctx.ptr) - graphs0
    st = G.Stats()
    o = G.default_opts(stats=ctypes.pointer(st))
    rc = G.segmented(ctx, d_v.data_ptr(), d_so.data_ptr(), nseg, d_k.data_ptr(), d_ko.data_ptr(),
                     d_out.data_ptr(), vals.dtype, o, stream.cuda_stream)
    if rc:
        raise G.GGMSError(rc, "ggms_multiselect_segmented (stats)")

    # e2e: the ks and offsets go host -> device and the answers device -> host every step
    h_k = torch.from_numpy(ks.view(np.int32)).pin_memory()
    h_so = torch.from_numpy(seg_off).pin_memory()
    h_ko = torch.from_numpy(k_off).pin_memory()
    h_out = torch.empty(len(ks), dtype=tdt).pin_memory()

    def f_e2e():
        d_k.copy_(h_k, non_blocking=True)
        d_so.copy_(h_so, non_blocking=True)
        d_ko.copy_(h_ko, non_blocking=True)
        f()
        h_out.copy_(d_out, non_blocking=True)
    ms_e2e = time_loop(f_e2e, args.steps, args.warmup, stream, world, dev)
    if exp is not None:
        import ggms_oracle as orc
        if not np.array_equal(orc.bits(h_out.numpy().view(vals.dtype)), orc.bits(exp)):
            raise SystemExit("batched e2e answers differ")

    peak, peak_kind = peaks()
    ms_step = ms / args.steps
    achieved = 2 * n * 4 / (ms_step / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": whole_job_rate(n, world, ms, args.steps), "unit": "elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if vals.dtype == np.float32 else "u32",
        "data": f"synthetic: seeded batch (numpy PCG64, seed {w['seed']}), generated on the host",
        "config": config_of(w, world),
        "roofline": {"bound": "hbm", "kernel": "whole call (level-0 count + copy over all segments)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "bytes_per_launch": 2 * n * 4},
        "e2e": {"value": world * n / (ms_e2e / args.steps / 1e3), "unit": "elements/s",
                "h2d_bytes_per_step": 4 * len(ks) + 8 * 2 * (nseg + 1), "d2h_bytes_per_step": 4 * len(ks)},
        "stats": {"full_passes": st.full_passes, "levels": st.levels, "refine_elements": st.refine_elements},
        "num_ks": int(len(ks)),
        "gpu_launches": int(launches),
        "graph_replays": int(graph_calls),
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_segmented(vals, seg_off, ks, k_off)
    ctx.close()
    return line


def run_ours(args):
    w = WORKLOADS[args.workload]
    world, rank, local = dist_setup(args)
    if w["kind"] == "single":
        line = run_ours_single(args, w, world, rank, local)
    else:
        line = run_ours_segmented(args, w, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import ggms_oracle as orc
    w = WORKLOADS[args.workload]
    if not orc.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libggms_ref.so not built (needs the reference sources at build time)"}))
        return
    if w["kind"] == "single":
        v, ks = single_inputs(w)
        n = len(v)
        times = []
        out = None
        for i in range(args.warmup + args.steps):
            out, ms = orc.ref_select("bucket_multiselect", v, ks)
            if i >= args.warmup:
                times.append(ms)
        exact = bool(np.array_equal(orc.bits(out), orc.bits(orc.cpu_multiselect(v, ks))))
        ms_step = statistics.mean(times)
        sample = ("the full workload: the reference's bucketMultiselectWrapper is GPU code, built unmodified "
                  "from its sources for sm_100a and run on the B200 with its own protocol (vector uploaded "
                  "before the timer, CUDA events around the wrapper call); one host thread drives it")
        extra = {"ms_per_step_median": statistics.median(times)}
    else:
        vals, seg_off, ks, k_off = segmented_inputs(w)
        n = int(seg_off[-1])
        nseg = len(seg_off) - 1
        lens = np.diff(seg_off)
        nks = np.diff(k_off)
        g = np.random.default_rng(w["seed"] + 1)
        # segments the reference's veneer accepts and that are at least as long as
        # the smallest vector it has run on this GPU (5000 keys, the int32 golden case)
        ok = [s for s in range(nseg) if lens[s] >= 5000 and
              np.any((ks[k_off[s]:k_off[s + 1]] != 1) & (ks[k_off[s]:k_off[s + 1]] != lens[s]))]
        pick = sorted(g.choice(ok, size=min(len(ok), 64 * max(1, args.steps // 4)), replace=False))
        per_seg, exact = [], True
        for s in pick:
            sv = vals[seg_off[s]:seg_off[s + 1]]
            sk = ks[k_off[s]:k_off[s + 1]]
            out, ms = orc.ref_select("bucket_multiselect", sv, sk)
            exact = exact and bool(np.array_equal(orc.bits(out), orc.bits(orc.select(sv, sk))))
            per_seg.append((int(lens[s]), ms))
        # scale to all segments: a measured segment stands for the segments of
        # similar length; a segment shorter than any measured one is charged the
        # smallest measured time (a lower bound on the reference's time)
        m_len = np.array([a for a, _ in per_seg], dtype=np.float64)
        m_ms = np.array([b for _, b in per_seg], dtype=np.float64)
        order = np.argsort(m_len)
        m_len, m_ms = m_len[order], m_ms[order]
        est = 0.0
        for s in range(nseg):
            if nks[s] == 0:
                continue
            j = int(np.clip(np.searchsorted(m_len, lens[s]), 0, len(m_len) - 1))
            est += float(m_ms[j])
        ms_step = est
        times = [ms_step]
        sample = (f"a loop of per-segment bucketMultiselectWrapper calls (the reference has no batched API) on "
                  f"{len(pick)} seeded segments of >= 5000 keys, each call timed by the reference's own "
                  f"protocol; the 4096-segment total is estimated by charging every segment the time of the "
                  f"measured segment of nearest length at or above it (shorter ones: the smallest measured), "
                  f"a lower bound on the full loop")
        extra = {"segments_measured": len(pick), "measured_ms_sum": float(m_ms.sum())}
    value = n / (ms_step / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: the same seeded inputs as the ours arm",
        "config": config_of(w, world),
        "exact_vs_oracle": exact,
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": 1, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ms_per_step_each": times,
    }
    line.update(extra)
    print(json.dumps(line), flush=True)


def run_kernels_only(args):
    """Short fixed run for profilers: a few device-resident calls per assigner."""
    import torch
    import ggms_b200 as G
    torch.cuda.set_device(0)
    w = dict(WORKLOADS[args.workload])
    if w["kind"] != "single":  # the batched workloads (4096 segments; 2^30 keys unless --total-log2)
        w["total"] = 1 << args.total_log2
        vals, seg_off, ks, k_off = segmented_inputs(w)
        view = {np.dtype(np.uint32): np.int32}.get(vals.dtype)
        d_v = torch.from_numpy(vals.view(view) if view else vals).cuda()
        d_so, d_ko = torch.from_numpy(seg_off).cuda(), torch.from_numpy(k_off).cuda()
        d_k = torch.from_numpy(ks.view(np.int32)).cuda()
        d_out = torch.empty(len(ks), dtype=torch.int32, device="cuda")
        ctx = G.Context(0)
        for _ in range(args.steps):
            rc = G.segmented(ctx, d_v.data_ptr(), d_so.data_ptr(), len(seg_off) - 1, d_k.data_ptr(),
                             d_ko.data_ptr(), d_out.data_ptr(), vals.dtype)
            if rc:
                raise G.GGMSError(rc, "segmented")
        torch.cuda.synchronize()
        ctx.close()
        print("kernels-only run done", int(seg_off[-1]), args.steps)
        return
    w["n"] = 1 << args.n_log2
    v, ks = single_inputs(w)
    d_v = torch.from_numpy(v).cuda()
    d_k = torch.from_numpy(ks.view(np.int32)).cuda()
    d_out = torch.empty(len(ks), dtype=torch.float32, device="cuda")
    ctx = G.Context(0)
    for a in (G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED):
        o = G.default_opts(assigner=a, ks_on_device=1, out_on_device=1)
        for _ in range(args.steps):
            rc = G.multiselect_ex(ctx, d_v.data_ptr(), w["n"], d_k.data_ptr(), len(ks),
                                  d_out.data_ptr(), np.float32, o)
            if rc:
                raise G.GGMSError(rc, "multiselect")
    torch.cuda.synchronize()
    ctx.close()
    print("kernels-only run done", w["n"], args.steps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="headline")
    ap.add_argument("--backend", default="auto")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--n-log2", type=int, default=28, help="vector length (--kernels-only runs only)")
    ap.add_argument("--total-log2", type=int, default=30,
                    help="keys of a batched workload in all (--kernels-only runs only)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="a few device-resident calls and exit (for profilers); no JSON line")
    args = ap.parse_args()
    if args.kernels_only:
        run_kernels_only(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
