"""The reference-facing C++ shim (include/ggms_compat.hpp) compiled into a
caller that uses the reference's own call pattern (tests/compat/caller.cu),
linked to libggms_b200.so, run on the GPU for int, unsigned, float and double
through both wrappers, and checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import ggms_b200 as G
import ggms_oracle as orc

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "compat", "caller.cu")


def build_caller(out_dir):
    exe = os.path.join(out_dir, "caller")
    libdir = os.path.dirname(G.LIB_PATH)
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"), SRC, "-o", exe,
                    "-L", libdir, "-lggms_b200", "-Xlinker", f"-rpath,{libdir}"], check=True)
    return exe


def test_caller_compiles(tmp_path):
    """The header instantiates for the four types the reference instantiates
    (host compile and link only; runs without a GPU)."""
    assert os.access(build_caller(str(tmp_path)), os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("entry", ["bucket", "iterative"])
@pytest.mark.parametrize("suf,dtype", [("i32", np.int32), ("u32", np.uint32), ("f32", np.float32),
                                       ("f64", np.float64)])
def test_caller_through_the_shim(tmp_path, suf, dtype, entry):
    exe = build_caller(str(tmp_path))
    g = np.random.default_rng(len(suf) * 7 + (entry == "bucket"))
    n = 300_007
    if np.dtype(dtype).kind == "f":
        v = (g.standard_normal(n) * 1e3).astype(dtype)
        v[::1009] = v[11]
    else:
        v = g.integers(np.iinfo(dtype).min, np.iinfo(dtype).max, size=n, dtype=dtype, endpoint=True)
    ks = np.concatenate([[1, n, (n + 1) // 2], g.integers(1, n + 1, size=500)]).astype(np.uint32)
    vp, kp, op = (str(tmp_path / x) for x in ("v.bin", "k.bin", "o.bin"))
    v.tofile(vp)
    ks.tofile(kp)
    r = subprocess.run([exe, suf, entry, vp, kp, op], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    got = np.fromfile(op, dtype=dtype)
    np.testing.assert_array_equal(orc.bits(got), orc.bits(orc.select(v, ks)))


@pytest.mark.gpu
def test_caller_reports_errors_like_the_reference(tmp_path):
    """A k outside [1, n]: the shim prints the reference's "Error at" line, still
    returns (T)1, and ggms_last_status() is set (the caller exits with 4)."""
    exe = build_caller(str(tmp_path))
    v = np.arange(100, dtype=np.float32)
    vp, kp, op = (str(tmp_path / x) for x in ("v.bin", "k.bin", "o.bin"))
    v.tofile(vp)
    np.array([5, 101], dtype=np.uint32).tofile(kp)
    r = subprocess.run([exe, "f32", "bucket", vp, kp, op], capture_output=True, text=True)
    assert r.returncode == 4
    assert "Error at" in r.stdout and "invalid argument" in r.stdout
