"""Comparison harness with the reference's problem tables and CSV row format.

A user of the reference drives its selectors through
`CompareIterativeSMOS::compareMultiselectAlgorithms` (DS/compareIterativeSMOS.cu:50-245):
pick a value generator and a k distribution by index, run each algorithm in a shuffled
order on the same vector, time it, flag any answer that differs from sort-and-choose,
and append one CSV row per test.  This module keeps that interface so existing
post-processing reads our rows unchanged:

* `FLOAT_GENERATORS` / `DOUBLE_GENERATORS` / `UINT_GENERATORS`: the reference's tables
  (DS/generateProblems.cu:75-79, 438-446, 509-513), same names and index order.  The
  values are drawn from numpy's PCG64 on the host instead of cuRAND, so the numbers
  differ from a reference run with the same seed; each distribution's shape follows
  the reference's generator (cited per function).
* `K_GENERATORS`: the five k distributions (DS/generateProblems.cu:584-730), with
  the reference's arithmetic (float32 where it multiplies in float) and its clamps.
* `csv_row` / `error_lines`: one row per test, byte for byte the reference's
  layout (DS/compareIterativeSMOS.cu:136-139, 180-208): size, numKs, generator
  name, k-distribution name, then `name,time,` per algorithm run, then the
  mismatch count.
* `compare_multiselect`: the driver.  Algorithm 0 is sort-and-choose on the GPU
  (torch's sort of the order-preserving keys; it only checks the others),
  algorithms 1 and 2 are this library's `bucketMultiselect` and `iterativeSMOS`
  drop-in entry points, timed like the reference's timing functions
  (DS/iterativeSMOSTimingFunctions.cu:134-156, 207-229): the vector is already on the
  device, CUDA events bracket the call, host ks in, host answers out.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

ALGORITHM_NAMES = ("Sort and Choose Multiselect", "Bucket Multiselect", "IterativeSMOS")


def _g(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


def _shuffled_two_values(n: int, first: float, first_pct: int, second: float, seed: int) -> np.ndarray:
    # createVector + scatter (DS/generateProblems.cu:166-189): first_pct % of the
    # entries hold `first` (integer percentage, rounded down), the rest `second`,
    # in shuffled order.
    n_first = (n * first_pct) // 100
    v = np.full(n, np.float32(second), dtype=np.float32)
    v[:n_first] = np.float32(first)
    _g(seed).shuffle(v)
    return v


# ------------------------------------------------------------------ float values
def uniform_floats(n: int, seed: int) -> np.ndarray:          # :86-92
    return _g(seed).random(n, dtype=np.float32)


def normal_floats(n: int, seed: int) -> np.ndarray:           # :94-110, N(0, 1)
    return _g(seed).standard_normal(n, dtype=np.float32)


def bucket_killer_floats(n: int, seed: int) -> np.ndarray:    # :422-436
    """Uniform floats masked with 0x80EFFFFF (exponent bits 24-30 and mantissa bit
    20 cleared: every value subnormal or just above the smallest normal), sorted as
    bit patterns; the first 253 entries (fewer if n is smaller) replaced by
    2^-126 .. 2^126, so the range spans every float exponent while almost all the
    mass sits in two tiny exponents."""
    bits = _g(seed).random(n, dtype=np.float32).view(np.uint32) & np.uint32(0x80EFFFFF)
    bits.sort()
    v = bits.view(np.float32)
    m = min(n, 253)
    v[:m] = np.ldexp(np.float32(1.0), np.arange(-126, -126 + m)).astype(np.float32)
    return v


def half_normal_floats(n: int, seed: int) -> np.ndarray:      # :381-401
    return np.abs(_g(seed).standard_normal(n, dtype=np.float32))


def normal_floats_100(n: int, seed: int) -> np.ndarray:       # :349-360, N(0, 100^2)
    return _g(seed).standard_normal(n, dtype=np.float32) * np.float32(100.0)


def huge_uniform_floats(n: int, seed: int) -> np.ndarray:     # :335-343, U[0,1) * 1e6
    return _g(seed).random(n, dtype=np.float32) * np.float32(1000000.0)


def noisy_floats(n: int, seed: int) -> np.ndarray:            # :286-322
    """20 % ones and 80 % zeros, shuffled, plus N(0, 0.01^2) noise."""
    base = _shuffled_two_values(n, 1.0, 20, 0.0, seed)
    return base + _g(seed + 1).standard_normal(n, dtype=np.float32) * np.float32(0.01)


def all_ones_floats(n: int, seed: int) -> np.ndarray:         # :217-229
    return np.ones(n, dtype=np.float32)


def ones_twos_floats(n: int, seed: int) -> np.ndarray:        # :191-215
    """Half twos (rounded down), the rest ones, shuffled."""
    return _shuffled_two_values(n, 2.0, 50, 1.0, seed)


def cauchy_floats(n: int, seed: int) -> np.ndarray:           # :246-277
    """tan(pi (u - 1/2)) with u in [0, 1), u == 0 moved to 0.0001 as the reference does."""
    u = _g(seed).random(n, dtype=np.float32)
    u[u == np.float32(0.0)] = np.float32(0.0001)
    return np.tan(np.float32(np.pi) * (u - np.float32(0.5))).astype(np.float32)


# ------------------------------------------------------------------ double values
def uniform_doubles(n: int, seed: int) -> np.ndarray:         # :456-462
    return _g(seed).random(n, dtype=np.float64)


def normal_doubles(n: int, seed: int) -> np.ndarray:          # :464-478
    return _g(seed).standard_normal(n, dtype=np.float64)


def bucket_killer_doubles(n: int, seed: int) -> np.ndarray:   # :493-507
    """As the float version with mask 0x800FFFFFFFFFFFFF (exponent cleared: zero
    and subnormals), sorted as bit patterns, the first 2045 entries replaced by
    2^-1022 .. 2^1022."""
    bits = _g(seed).random(n, dtype=np.float64).view(np.uint64) & np.uint64(0x800FFFFFFFFFFFFF)
    bits.sort()
    v = bits.view(np.float64)
    m = min(n, 2045)
    v[:m] = np.ldexp(1.0, np.arange(-1022, -1022 + m))
    return v


# ------------------------------------------------------------------ uint values
def uniform_uints(n: int, seed: int) -> np.ndarray:           # :43-50
    return _g(seed).integers(0, 2**32, size=n, dtype=np.uint32)


def sorted_uints(n: int, seed: int) -> np.ndarray:            # :52-62 (ascending)
    v = uniform_uints(n, seed)
    v.sort()
    return v


def uniform_0_4_uints(n: int, seed: int) -> np.ndarray:       # :64-73
    """The reference's "UNIFORM 0-4" table entry writes i % 100, kept as it is."""
    return (np.arange(n, dtype=np.uint64) % 100).astype(np.uint32)


Generator = Tuple[str, Callable[[int, int], np.ndarray]]

FLOAT_GENERATORS: List[Generator] = [
    ("UNIFORM FLOATS", uniform_floats), ("NORMAL FLOATS", normal_floats),
    ("KILLER FLOATS", bucket_killer_floats), ("HALF NORMAL FLOATS", half_normal_floats),
    ("NORMAL FLOATS 100", normal_floats_100), ("HUGE UNIFORM FLOATS", huge_uniform_floats),
    ("NOISY FLOATS", noisy_floats), ("ALL ONES FLOATS", all_ones_floats),
    ("ONES TWOS FLOAT", ones_twos_floats), ("CAUCHY FLOAT", cauchy_floats),
]
DOUBLE_GENERATORS: List[Generator] = [
    ("UNIFORM DOUBLES", uniform_doubles), ("NORMAL DOUBLES", normal_doubles),
    ("KILLER DOUBLES", bucket_killer_doubles),
]
UINT_GENERATORS: List[Generator] = [
    ("UNIFORM UNSIGNED INTEGERS", uniform_uints), ("SORTED UINTS", sorted_uints),
    ("UNIFORM 0-4", uniform_0_4_uints),
]


def generators_for(dtype) -> List[Generator]:
    """The generator table of a value type (`returnGenFunctions`, DS/generateProblems.cu:518-535)."""
    dt = np.dtype(dtype)
    if dt == np.float32:
        return FLOAT_GENERATORS
    if dt == np.float64:
        return DOUBLE_GENERATORS
    if dt == np.uint32:
        return UINT_GENERATORS
    raise ValueError(f"no generator table for {dt}")


# ------------------------------------------------------------------ k distributions
def _clamp_ks(k: np.ndarray, n: int) -> np.ndarray:
    return np.clip(k, 1, n).astype(np.uint32)


def ks_uniform_random(count: int, n: int, seed: int) -> np.ndarray:   # :584-600
    u = _g(seed).random(count, dtype=np.float32)
    return _clamp_ks((u * np.float32(n)).astype(np.int64), n)


def ks_uniform(count: int, n: int, seed: int) -> np.ndarray:          # :608-620
    """1, then (i / (count-1)) * n in float32 for the inner entries, then n: with
    count = 101 these are the 0th..100th percentiles."""
    k = np.empty(count, dtype=np.int64)
    if count >= 1:
        i = np.arange(count, dtype=np.float32)
        k[:] = ((i / np.float32(max(count - 1, 1))) * np.float32(n)).astype(np.int64)
        k[0] = 1
        k[-1] = n
    return _clamp_ks(k, n)


def ks_normal_random(count: int, n: int, seed: int) -> np.ndarray:    # :622-652
    """(|z| + 7) * (n / 14) in double: ks in the upper half of the ranks."""
    z = _g(seed).standard_normal(count, dtype=np.float32)
    k = ((np.abs(z).astype(np.float64) + 7.0) * (n / 14.0)).astype(np.int64)
    return _clamp_ks(k, n)


def ks_cluster(count: int, n: int, seed: int) -> np.ndarray:          # :654-696
    """Runs of nine consecutive ranks around centres u * (n - 10) + 5 (float32);
    the entries after the last full run continue one rank apart from a new centre,
    capped at n - 1."""
    u = _g(seed).random(count // 9 + 2, dtype=np.float32)
    k = np.zeros(count, dtype=np.int64)
    fi = 0
    max_assigned = 0
    for i in range(4, count, 9):
        c = int(u[fi] * np.float32(n - 10) + np.float32(5))
        fi += 1
        k[i] = c
        for j in range(1, 5):
            k[i - j] = c - j
            if i + j < count:
                k[i + j] = c + j
            max_assigned = max(max_assigned, i + j)
    k = np.clip(k, 1, n)
    if max_assigned < count - 1:
        k[max_assigned + 1] = int(u[fi] * np.float32(n - 10) + np.float32(5))
        for j in range(max_assigned + 2, count):
            k[j] = min(k[j - 1] + 1, n - 1)
    return _clamp_ks(k, n)


def ks_sectioned(count: int, n: int, seed: int) -> np.ndarray:        # :698-720
    """`count` consecutive ranks from a random start u * (n - count).  The reference
    can start at rank 0, which is not a valid k; the start is raised to 1 here."""
    u = _g(seed).random(1, dtype=np.float32)[0]
    start = int(u * np.float32(max(n - count, 0)))
    return _clamp_ks(start + np.arange(count, dtype=np.int64), n)


K_GENERATORS: List[Tuple[str, Callable[[int, int, int], np.ndarray]]] = [
    ("Uniform Random Ks", ks_uniform_random), ("Uniform Ks", ks_uniform),
    ("Normal Random Ks", ks_normal_random), ("Cluster Ks", ks_cluster),
    ("Sectioned Ks", ks_sectioned),
]


# ------------------------------------------------------------------ CSV rows
def _cpp_float(x: float) -> str:
    """A float as `std::ostream <<` prints it by default (6 significant digits)."""
    return "%g" % x


def csv_row(size: int, num_ks: int, gen_name: str, k_gen_name: str,
            times: Sequence[Tuple[str, float]], flag: int) -> str:
    """One test's row (DS/compareIterativeSMOS.cu:136-139, 180-182, 210)."""
    head = f"{size},{num_ks},{gen_name},{k_gen_name},"
    body = "".join(f"{name},{_cpp_float(t)}," for name, t in times)
    return head + body + f"{flag}\n"


def error_lines(test: int, num_tests: int, size: int, seed: int, num_ks: int,
                k: int, k_index: int, wrong, correct) -> str:
    """The block the reference writes into the row for each wrong answer
    (DS/compareIterativeSMOS.cu:189-195)."""
    return (f"\nERROR ON TEST {test} of {num_tests} tests!!!!!\n"
            f"vector size = {size}\nvector seed = {seed}\n"
            f"numKs = {num_ks}\n"
            f"wrong k = {k} kIndex = {k_index} wrong result = {wrong} correct result = {correct}\n")


# ------------------------------------------------------------------ the driver
def _raw_tensor(torch, h_vec: np.ndarray, device: str):
    """The vector as a signed integer tensor of its own width (bit patterns kept),
    so no torch dtype beyond int32/int64 is needed on the device."""
    return torch.from_numpy(h_vec.view(np.int64 if h_vec.dtype.itemsize == 8 else np.int32)).to(device)


def _sort_and_choose(torch, raw, ks: np.ndarray, dtype) -> np.ndarray:
    """k-th largest by a full sort of order-preserving signed 64-bit keys
    (-NaN < -Inf < ... < -0 < +0 < ... < +Inf < +NaN) on `raw`'s device; answers
    are gathered by index, so they are the input's own bit patterns."""
    dt = np.dtype(dtype)
    n = raw.numel()
    key = raw.to(torch.int64)
    if dt == np.float32:
        key = torch.where(key < 0, key ^ 0x7FFFFFFF, key)
    elif dt == np.float64:
        key = torch.where(key < 0, key ^ 0x7FFFFFFFFFFFFFFF, key)
    elif dt == np.uint32:
        key = key & 0xFFFFFFFF
    order = torch.sort(key, stable=True).indices
    pos = torch.from_numpy(n - ks.astype(np.int64)).to(raw.device)
    return raw[order[pos]].cpu().numpy().view(dt)


def compare_multiselect(dtype, size: int, ks: np.ndarray, num_tests: int, gen_type: int,
                        k_gen_type: int, csv_path: Optional[str] = None,
                        algorithms: Sequence[int] = (1, 1, 1), seed: int = 0,
                        device: int = 0, verbose: bool = True) -> dict:
    """Run the reference's comparison loop over this library's entry points.

    Mirrors `compareMultiselectAlgorithms(size, kVals, numKs, numTests,
    algorithmsToTest, generateType, kGenerateType, fileNamecsv)`: `ks` are 1-based
    k-th largest, `algorithms[j]` switches algorithm j on, `gen_type` indexes the
    value type's generator table and `k_gen_type` names the k distribution in the
    rows (`K_GENERATORS`).  Test i draws its vector from `seed + i` (the
    reference seeds from the time of day) and its run order from the same seed.
    Appends one row per test to `csv_path` (if given) and returns the times
    (ms, per algorithm per test), the winners and the mismatch counts.
    """
    import torch

    from . import dropin

    dt = np.dtype(dtype)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    gen_name, gen = generators_for(dt)[gen_type]
    k_gen_name = K_GENERATORS[k_gen_type][0]
    entries = {1: "bucket_multiselect", 2: "iterative_smos"}
    torch.cuda.set_device(device)
    times = np.full((len(ALGORITHM_NAMES), num_tests), np.nan, dtype=np.float64)
    winners, flags = [], []
    out = open(csv_path, "a") if csv_path else None
    try:
        for t in range(num_tests):
            test_seed = seed + t
            order = list(range(len(ALGORITHM_NAMES)))
            _g(test_seed).shuffle(order)
            h_vec = gen(size, test_seed)
            d_vec = _raw_tensor(torch, h_vec, f"cuda:{device}")
            results = {}
            for j in order:
                if not algorithms[j]:
                    continue
                torch.cuda.synchronize()
                start = torch.cuda.Event(enable_timing=True)
                stop = torch.cuda.Event(enable_timing=True)
                start.record()
                if j == 0:
                    res = _sort_and_choose(torch, d_vec, ks, dt)
                else:
                    res = dropin(entries[j], d_vec.data_ptr(), size, ks, dt)
                stop.record()
                stop.synchronize()
                times[j, t] = start.elapsed_time(stop)
                results[j] = res
            row_times = [(ALGORITHM_NAMES[j], times[j, t]) for j in range(len(ALGORITHM_NAMES))
                         if algorithms[j]]
            errors, flag = "", 0
            if 0 in results:
                ref_bits = results[0].view(np.uint64 if dt.itemsize == 8 else np.uint32)
                for j in sorted(results):
                    if j == 0:
                        continue
                    bits = results[j].view(ref_bits.dtype)
                    for idx in np.nonzero(bits != ref_bits)[0]:
                        flag += 1
                        errors += error_lines(t, num_tests, size, test_seed, len(ks), int(ks[idx]),
                                              int(idx), results[j][idx], results[0][idx])
            valid = [j for j in range(len(ALGORITHM_NAMES)) if algorithms[j]]
            winners.append(min(valid, key=lambda j: times[j, t]))
            flags.append(flag)
            if out is not None:
                row = csv_row(size, len(ks), gen_name, k_gen_name, row_times, flag)
                # the reference writes the error block before the count that ends the row
                out.write(row[: row.rindex(",") + 1] + errors + f"{flag}\n")
            del d_vec
    finally:
        if out is not None:
            out.close()
    if verbose:
        for j in range(len(ALGORITHM_NAMES)):
            if algorithms[j]:
                print("%-20s averaged: %f ms" % (ALGORITHM_NAMES[j], np.nanmean(times[j])))
        for j in range(len(ALGORITHM_NAMES)):
            if algorithms[j]:
                print("%s won %u times" % (ALGORITHM_NAMES[j], winners.count(j)))
    return {"times_ms": times, "winners": winners, "flags": flags, "generator": gen_name}


def run_tests(dtype, gen_type: int, csv_path: str, start_power: int, stop_power: int,
              times_to_test_each_k: int, k_distribution: int, start_k: int, stop_k: int,
              k_jump: int, seed: int = 0) -> List[dict]:
    """`runTests` (DS/compareIterativeSMOS.cu:251-290): for each size 2^p, p in
    [start_power, stop_power], draw stop_k ks from k distribution `k_distribution`
    once, then compare on the first start_k, start_k + k_jump, ... of them."""
    k_gen = K_GENERATORS[k_distribution][1]
    runs = []
    for p in range(start_power, stop_power + 1):
        size = 1 << p
        all_ks = k_gen(stop_k, size, seed + p)
        for nk in range(start_k, stop_k + 1, max(k_jump, 1)):
            runs.append(compare_multiselect(dtype, size, all_ks[:nk], times_to_test_each_k, gen_type,
                                            k_distribution, csv_path, seed=seed + p, verbose=False))
    return runs


__all__ = [
    "ALGORITHM_NAMES", "FLOAT_GENERATORS", "DOUBLE_GENERATORS", "UINT_GENERATORS",
    "K_GENERATORS", "generators_for", "csv_row", "error_lines", "compare_multiselect",
    "run_tests",
]


# ------------------------------------------------------------------ command line
_TYPES = (("float", np.float32), ("double", np.float64), ("uint", np.uint32))
_QUESTIONS = ("type (0-float 1-double 2-uint)", "distribution type", "K distribution type",
              "start power", "stop power", "start number of K values",
              "number of K values to jump by", "stop number of K values",
              "number of tests to run per K")


def parse_answers(tokens: Sequence[str]) -> dict:
    """The nine answers of the reference's interactive `main`
    (DS/compareIterativeSMOS.cu:316-338), in its order: type, distribution, k
    distribution, start power, stop power, start K, K jump, stop K, tests per K."""
    if len(tokens) < 9:
        raise ValueError(f"expected 9 answers ({', '.join(_QUESTIONS)}), got {len(tokens)}")
    t, g, kd, p0, p1, k0, kj, k1, nt = (int(x) for x in tokens[:9])
    if not 0 <= t < len(_TYPES):
        raise ValueError("type must be 0 (float), 1 (double) or 2 (uint)")
    if not 0 <= g < len(generators_for(_TYPES[t][1])) or not 0 <= kd < len(K_GENERATORS):
        raise ValueError("generator or k distribution out of range")
    if not (0 < p0 <= p1 <= 40 and 0 < k0 <= k1 and kj > 0 and nt > 0):
        raise ValueError("powers, K counts, jump and test count must be positive and ordered")
    return dict(type=t, generator=g, k_distribution=kd, start_power=p0, stop_power=p1,
                start_k=k0, k_jump=kj, stop_k=k1, tests=nt)


def file_name(a: dict, host: str, when: str) -> str:
    """The reference's results file name (DS/compareIterativeSMOS.cu:355-359)."""
    tname, dt = _TYPES[a["type"]]
    return (f"{tname} {generators_for(dt)[a['generator']][0]} "
            f"k-dist:{K_GENERATORS[a['k_distribution']][0]} 2^{a['start_power']} to 2^{a['stop_power']} "
            f"({a['start_k']}:{a['k_jump']}:{a['stop_k']}) {a['tests']}-tests on {host} at {when}")


def main(argv: Optional[Sequence[str]] = None) -> int:
    """`python -m ggms_b200.harness [9 answers] [--csv PATH] [--seed S]`; without the
    answers on the command line they are read from standard input, one per line, in
    the order the reference's harness asks for them."""
    import argparse
    import socket
    import sys
    import time as _time

    ap = argparse.ArgumentParser(description="compare the selectors the way compareIterativeSMOS does")
    ap.add_argument("answers", nargs="*", help="; ".join(_QUESTIONS))
    ap.add_argument("--csv", default=None, help="results file (default: the reference's file name)")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    tokens = list(args.answers) or sys.stdin.read().split()
    a = parse_answers(tokens)
    path = args.csv or file_name(a, socket.gethostname()[:20], _time.asctime())
    print(f"File Name: {path} ")
    runs = run_tests(_TYPES[a["type"]][1], a["generator"], path, a["start_power"], a["stop_power"],
                     a["tests"], a["k_distribution"], a["start_k"], a["stop_k"], a["k_jump"], seed=args.seed)
    bad = sum(sum(r["flags"]) for r in runs)
    print(f"{len(runs)} comparisons, {bad} wrong answers")
    return 1 if bad else 0


if __name__ == "__main__":
    raise SystemExit(main())
