#!/usr/bin/env python3
"""Benchmark: exact multiple order statistics, n = 2^28 fp32, 1024 ks, one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the headline of the reference's single-GPU path): 2^28 fp32 values,
seeded half-normal, and 1026 ks -- 1024 distinct ks among the top 1% of ranks
plus k = 1 and k = n -- each answer the exact k-th largest.

ours:
  value  elements/s with the vector, the ks and the answers resident in HBM
         (one _ex call per step, no host sync inside the timed region);
         the default assigner (learned PL-CDF, sampled-pivot fallback).
  e2e    the same metric through the reference-facing C ABI
         (ggms_bucket_multiselect_f32: host ks in, host answers out, the vector
         a device pointer -- exactly the reference's own timing protocol,
         DistributedSMOS/iterativeSMOSTimingFunctions.cu:134-156);
         e2e_incl_vector_h2d adds the 1 GiB host->device copy of the vector
         from pinned memory to every step.
  sampled the same timed loop with the sampled-pivot assigner (the reference's
         bucket method) for the learned-vs-sampled comparison.
reference:
  the reference's own bucketMultiselectWrapper, compiled unmodified from its
  sources (oracle/_ref), timed with its own protocol on the same GPU.
N > 1: independent replicas (the path does not shard: one vector per GPU),
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
N_ELEMS = 1 << 28
NK_TOP = 1024
SEED_VALUES = 21
SEED_KS = 21
WORKLOAD = "half_normal_f32 n=2^28, 1024 top-1% ks + k=1 + k=n (exact k-th largest)"


# DRAM bytes (read + write) per input element of the two passes, from one ncu
# capture of the same kernels on the same half-normal workload at n = 2^26
# (profiles/l0_passes_half_normal_f32_n26.md); both passes read the input once,
# so the traffic of a launch grows in proportion to n.
PASS_TRAFFIC_PER_ELEM = {"l0_count": (268580096 + 3641344) / 2**26,
                         "l0_compact": (271806720 + 3763712) / 2**26}


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


def workload():
    from ggms_b200 import datagen as D
    v = D.half_normal_f32(N_ELEMS, SEED_VALUES)
    ks = D.ks_top1pct(N_ELEMS, NK_TOP, SEED_KS)
    return v, ks


def run_kernels_only(args):
    """Short fixed run for profilers: a few device-resident calls per assigner.
    --spread-ks swaps the clustered ks for 1024 ks uniform over all ranks."""
    import torch
    import ggms_b200 as G
    from ggms_b200 import datagen as D
    torch.cuda.set_device(0)
    v, ks = workload()
    if args.spread_ks:
        ks = D.ks_uniform(N_ELEMS, NK_TOP, SEED_KS)
    d_v = torch.from_numpy(v).cuda()
    d_k = torch.from_numpy(ks.view(np.int32)).cuda()
    d_out = torch.empty(len(ks), dtype=torch.float32, device="cuda")
    ctx = G.Context(0)
    for a in (G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED):
        o = G.default_opts(assigner=a, ks_on_device=1, out_on_device=1)
        for _ in range(args.steps):
            rc = G.multiselect_ex(ctx, d_v.data_ptr(), N_ELEMS, d_k.data_ptr(), len(ks),
                                  d_out.data_ptr(), np.float32, o)
            if rc:
                raise G.GGMSError(rc, "multiselect")
    torch.cuda.synchronize()
    ctx.close()
    print("kernels-only run done", N_ELEMS, args.steps)


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


def cpu_baseline_leg(v, ks):
    """The oracle's multithreaded nth_element multiselect on a bounded sample."""
    import ggms_oracle as orc
    from ggms_b200 import datagen as D
    threads = orc.cpu_threads()
    sample_n = 1 << 26
    sv = v[:sample_n]
    sks = D.ks_top1pct(sample_n, NK_TOP, SEED_KS)
    t0 = time.perf_counter()
    orc.cpu_multiselect(sv, sks, threads=threads, method=1)
    dt = time.perf_counter() - t0
    reps = max(1, min(8, int(10.0 / max(dt, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(reps):
        orc.cpu_multiselect(sv, sks, threads=threads, method=1)
    dt = (time.perf_counter() - t0) / reps
    return {"value": sample_n / dt, "unit": "elements/s", "cores": threads, "kind": "port",
            "sample": f"first 2^26 elements of the same half-normal input, 1024 top-1% ks + k=1 "
                      f"+ k=n of that sample; OpenMP recursive std::nth_element, {reps} reps"}


def run_ours(args):
    import torch
    import ggms_b200 as G
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    lib = G.load()
    v, ks = workload()
    nk = len(ks)
    d_v = torch.from_numpy(v).to(dev)
    d_k = torch.from_numpy(ks.view(np.int32)).to(dev)
    d_out = torch.empty(nk, dtype=torch.float32, device=dev)
    ctx = G.Context(local)

    def call(assigner):
        o = G.default_opts(assigner=assigner, ks_on_device=1, out_on_device=1)

        def f():
            rc = G.multiselect_ex(ctx, d_v.data_ptr(), N_ELEMS, d_k.data_ptr(), nk, d_out.data_ptr(),
                                  np.float32, o, stream.cuda_stream)
            if rc:
                raise G.GGMSError(rc, "ggms_multiselect_f32_ex")
        return f

    # correctness of this very run (answers are exact or the bench fails)
    if rank == 0:
        import ggms_oracle as orc
        exp = orc.cpu_multiselect(v, ks)
        for a in (G.ASSIGNER_AUTO, G.ASSIGNER_SAMPLED):
            call(a)()
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            if not np.array_equal(got.view(np.uint32), exp.view(np.uint32)):
                raise SystemExit(f"answers differ from the oracle (assigner {a})")

    # value: device-resident, learned (auto) assigner.  Repeated calls replay a
    # captured CUDA graph (the second call captures it), as in a real loop.
    launches0 = lib.ggms_context_launches(ctx.ptr)
    graphs0 = lib.ggms_context_graph_launches(ctx.ptr)
    with Clocks(local) as clk:
        ms = time_loop(call(G.ASSIGNER_AUTO), args.steps, args.warmup, stream, world, dev)
    launches = (lib.ggms_context_launches(ctx.ptr) - launches0) * args.steps // (args.steps + args.warmup)
    graph_calls = lib.ggms_context_graph_launches(ctx.ptr) - graphs0
    # pass times: the same calls with the profiling hooks on (events around the
    # passes on the call's stream; such calls run without the graph)
    lib.ggms_context_profile(ctx.ptr, 1)
    time_loop(call(G.ASSIGNER_AUTO), args.steps, args.warmup, stream, world, dev)
    cnt = args.steps + args.warmup
    p1 = (ctypes.c_float * cnt)()
    p2 = (ctypes.c_float * cnt)()
    pc = (ctypes.c_float * cnt)()
    got = lib.ggms_context_pass_times(ctx.ptr, p1, p2, pc, cnt)
    lib.ggms_context_profile(ctx.ptr, 0)
    p1 = list(p1)[args.warmup:got]
    p2 = list(p2)[args.warmup:got]
    ms_step = ms / args.steps
    value = whole_job_rate(N_ELEMS, world, ms, args.steps)

    # stats of one call (passes, candidates, occupancy)
    _, st_auto = G.select(ctx, d_v.data_ptr(), N_ELEMS, ks, np.float32, assigner=G.ASSIGNER_AUTO,
                          stats=True)
    _, st_samp = G.select(ctx, d_v.data_ptr(), N_ELEMS, ks, np.float32, assigner=G.ASSIGNER_SAMPLED,
                          stats=True)

    # the sampled-pivot path, same loop
    ms_s = time_loop(call(G.ASSIGNER_SAMPLED), args.steps, args.warmup, stream, world, dev)

    # e2e through the reference-facing drop-in (host ks, host answers)
    ks_host = np.ascontiguousarray(ks)
    out_host = np.empty(nk, dtype=np.float32)
    kp = ks_host.ctypes.data_as(ctypes.c_void_p)
    op = out_host.ctypes.data_as(ctypes.c_void_p)

    def dropin():
        rc = lib.ggms_bucket_multiselect_f32(d_v.data_ptr(), N_ELEMS, kp, nk, op, 148, 1024)
        if rc:
            raise G.GGMSError(rc, "ggms_bucket_multiselect_f32")
    ms_e2e = time_loop(dropin, args.steps, args.warmup, torch.cuda.default_stream(), world, dev)
    # ... and with the vector upload from pinned host memory in every step
    pinned = torch.from_numpy(v).pin_memory()
    d_v2 = torch.empty_like(d_v)

    def dropin_h2d():
        d_v2.copy_(pinned, non_blocking=True)
        rc = lib.ggms_bucket_multiselect_f32(d_v2.data_ptr(), N_ELEMS, kp, nk, op, 148, 1024)
        if rc:
            raise G.GGMSError(rc, "ggms_bucket_multiselect_f32")
    e2e_steps = max(3, min(args.steps, 5))
    ms_e2e_h2d = time_loop(dropin_h2d, e2e_steps, 1, torch.cuda.default_stream(), world, dev)

    peak, peak_kind = peaks()
    bytes_pass = N_ELEMS * 4
    t1 = statistics.mean(p1) if p1 else float("nan")
    t2 = statistics.mean(p2) if p2 else float("nan")
    dom_name, dom_ms = ("l0_count", t1) if t1 >= t2 else ("l0_compact", t2)
    achieved = bytes_pass / (dom_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded half-normal fp32 (numpy PCG64, seed 21), generated on the host",
        "config": {"workload": WORKLOAD, "n": N_ELEMS, "num_ks": nk, "assigner": "auto (learned PL-CDF)",
                   "l2": "inputs larger than L2 (1 GiB per pass)", "parallelism": f"replicas x{world}"},
        "hbm_gbs_alg": world * 2 * bytes_pass / (ms_step / 1e3) / 1e9,
        "passes": st_auto["full_passes"],
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": PASS_TRAFFIC_PER_ELEM[dom_name] * N_ELEMS,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at n=2^26, "
                                       "scaled by n (profiles/l0_passes_half_normal_f32_n26.md)",
                     "bytes_per_launch": bytes_pass,
                     "pass1_ms": t1, "pass2_ms": t2,
                     "two_pass_frac": 2 * bytes_pass / (ms_step / 1e3) / 1e9 / peak},
        "e2e": {"value": world * N_ELEMS / (ms_e2e / args.steps / 1e3), "unit": "elements/s",
                "h2d_bytes_per_step": 4 * nk, "d2h_bytes_per_step": 4 * nk,
                "api": "ggms_bucket_multiselect_f32 (vector device-resident, as the reference's API)"},
        "e2e_incl_vector_h2d": {"value": world * N_ELEMS / (ms_e2e_h2d / e2e_steps / 1e3),
                                "unit": "elements/s", "h2d_bytes_per_step": 4 * N_ELEMS + 4 * nk,
                                "d2h_bytes_per_step": 4 * nk},
        "sampled": {"value": world * N_ELEMS / (ms_s / args.steps / 1e3), "ms_per_step": ms_s / args.steps,
                    "stats": st_samp},
        "stats": st_auto,
        "gpu_launches": int(launches),
        "graph_replays": int(graph_calls),
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_leg(v, ks)
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import ggms_oracle as orc
    if not orc.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libggms_ref.so not built (needs the reference sources at build time)"}))
        return
    v, ks = workload()
    times = []
    for i in range(args.warmup + args.steps):
        out, ms = orc.ref_select("bucket_multiselect", v, ks)
        if i >= args.warmup:
            times.append(ms)
    exact = bool(np.array_equal(orc.bits(out), orc.bits(orc.cpu_multiselect(v, ks))))
    ms_step = statistics.mean(times)
    value = N_ELEMS / (ms_step / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded half-normal fp32 (numpy PCG64, seed 21)",
        "config": {"workload": WORKLOAD, "n": N_ELEMS, "num_ks": len(ks), "parallelism": "none"},
        "exact_vs_oracle": exact,
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": 1, "kind": "reference",
                         "sample": "the full workload: the reference's bucketMultiselectWrapper is GPU "
                                   "code, built unmodified from its sources for sm_100a and run on the "
                                   "B200 with its own protocol (vector uploaded before the timer, CUDA "
                                   "events around the wrapper call); one host thread drives it"},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ms_per_step_each": times,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--backend", default="auto")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--n-log2", type=int, default=28, help="vector length (profiling runs only)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="a few device-resident calls and exit (for profilers); no JSON line")
    ap.add_argument("--spread-ks", action="store_true",
                    help="with --kernels-only: 1024 ks uniform over all ranks instead of the top 1%%")
    args = ap.parse_args()
    global N_ELEMS
    N_ELEMS = 1 << args.n_log2
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
