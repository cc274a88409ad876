"""Generate the golden vectors that pin the CPU oracle to the reference.

Runs the reference's OWN bucketMultiselectWrapper (DistributedSMOS/
bucketMultiselect.cu:853-886, built unmodified from its sources by
oracle/Makefile into oracle/_ref/libggms_ref.so) on a GPU, on seeded inputs of
every value generator and k distribution the benchmark uses, and stores
inputs, ks and the reference's answers as .npz fixtures.  tests/test_golden.py
then checks the CPU oracle against them without a GPU.

Usage (on a machine with a GPU and oracle/_ref built):
    python tests/golden/make_golden.py <outdir>
Only bucketMultiselect is run: it sorts its candidates, so it is exact by
construction.  The reference's iterativeSMOS is not run on the GPU.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "oracle"), os.path.join(REPO, "ggms-distributed_b200")]

import ggms_oracle as orc  # noqa: E402
from ggms_b200 import datagen as D  # noqa: E402


def cases():
    g = np.random.default_rng(2024)
    yield "uniform_f32_percentiles", D.uniform_f32(1 << 14, 0), D.ks_percentiles(1 << 14, 101)
    yield "normal_f32_random", D.normal_f32(10007, 1), D.ks_uniform(10007, 257, 11)
    yield "normal_f64_random", D.normal_f64(1 << 14, 2), D.ks_uniform_distinct(1 << 14, 301, 12)
    yield "uniform_u32_random", D.uniform_u32(1 << 14, 3), D.ks_uniform_distinct(1 << 14, 301, 13)
    ints = g.integers(-(2**31), 2**31, size=5000, dtype=np.int64).astype(np.int32)
    yield "int32_random", ints, D.ks_uniform(5000, 123, 14)
    yield "distinct256_f32_top1pct", D.distinct256_f32(1 << 16, 21), D.ks_top1pct(1 << 16, 200, 21)
    yield "half_normal_f32_top1pct", D.half_normal_f32(1 << 15, 21), D.ks_top1pct(1 << 15, 150, 22)
    yield "cauchy_f32_top1pct", D.cauchy_f32(1 << 15, 21), D.ks_top1pct(1 << 15, 150, 23)
    yield "sorted_desc_u32_top1pct", D.sorted_desc_u32(1 << 15, 21), D.ks_top1pct(1 << 15, 150, 24)
    yield "mixture8_f32_random", D.mixture8_f32(1 << 15, 31), D.ks_uniform(1 << 15, 1024, 33)
    yield "lognormal_f32_random", D.lognormal_f32(1 << 15, 32), D.ks_uniform(1 << 15, 1024, 34)
    two = np.where(g.random(1 << 14) < 0.3, 1.5, 2.5).astype(np.float32)
    yield "two_values_f32", two, D.ks_uniform(1 << 14, 64, 35)
    inf = D.normal_f32(1 << 14, 36)
    inf[::97] = np.inf
    inf[::89] = -np.inf
    yield "with_inf_f32", inf, D.ks_uniform(1 << 14, 128, 37)
    z = D.normal_f32(1 << 14, 38)
    z[::7] = 0.0
    z[::11] = -0.0
    yield "signed_zeros_f32", z, D.ks_uniform(1 << 14, 128, 39)


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, v, ks in cases():
        ref, ms = orc.ref_select("bucket_multiselect", v, ks)
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), values=v, ks=ks, ref_out=ref,
                            ref_ms=np.float32(ms), source=np.bytes_("bucketMultiselectWrapper"))
        agree = np.mean(orc.bits(ref) == orc.bits(orc.select(v, ks)))
        print(f"{name:28s} n={len(v):6d} nk={len(ks):5d} ref_ms={ms:8.3f} bit-agree={agree:.4f}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
