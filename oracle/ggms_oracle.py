"""ctypes loader of the CPU oracle (and of the reference's own GPU build).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() and
by the cpu_baseline / reference legs of bench.py -- as the checker or as the
timed baseline, never as the product path.

  select(values, ks)            sort-and-choose (oracle/ggms_oracle.c), restating
                                DistributedSMOS/iterativeSMOSTimingFunctions.cu:67-120
  cpu_multiselect(values, ks)   OpenMP baselines (oracle/ggms_cpu_baseline.cpp)
  ref_lib()                     oracle/_ref/libggms_ref.so: the reference's
                                bucketMultiselectWrapper / iterativeSMOSWrapper
                                compiled from its own sources (oracle/Makefile)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "libggms_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libggms_ref.so")

_SUF = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64",
        np.dtype(np.uint32): "u32", np.dtype(np.int32): "i32"}

_lib = None
_ref = None


def build(ref: bool = False) -> None:
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        l = ctypes.CDLL(ORACLE_SO)
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        for suf in ("f32", "f64", "u32", "i32"):
            f = getattr(l, f"ggms_oracle_select_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [vp, i64, vp, i64, vp]
        for suf in ("f32", "u32"):
            f = getattr(l, f"ggms_oracle_select_segmented_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, i64, vp, vp, vp]
        for suf in ("f32", "f64", "u32"):
            f = getattr(l, f"ggms_cpu_multiselect_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [vp, i64, vp, i64, vp, ctypes.c_int, ctypes.c_int]
        for suf in ("f32", "u32"):
            f = getattr(l, f"ggms_cpu_multiselect_segmented_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [vp, vp, i64, vp, vp, vp, ctypes.c_int]
        l.ggms_cpu_max_threads.restype = ctypes.c_int
        l.ggms_oracle_key_f32.restype = ctypes.c_uint32
        l.ggms_oracle_key_f32.argtypes = [ctypes.c_float]
        l.ggms_oracle_key_f64.restype = ctypes.c_uint64
        l.ggms_oracle_key_f64.argtypes = [ctypes.c_double]
        _lib = l
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def select(values: np.ndarray, ks: np.ndarray) -> np.ndarray:
    """k-th largest (1-based) of `values` for each k, by sort-and-choose."""
    values = np.ascontiguousarray(values)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=values.dtype)
    rc = getattr(lib(), f"ggms_oracle_select_{_SUF[values.dtype]}")(
        _p(values), len(values), _p(ks), len(ks), _p(out))
    if rc:
        raise ValueError("oracle rejected the arguments")
    return out


def select_segmented(values, seg_off, ks, k_off) -> np.ndarray:
    values = np.ascontiguousarray(values)
    seg_off = np.ascontiguousarray(seg_off, dtype=np.int64)
    k_off = np.ascontiguousarray(k_off, dtype=np.int64)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=values.dtype)
    rc = getattr(lib(), f"ggms_oracle_select_segmented_{_SUF[values.dtype]}")(
        _p(values), _p(seg_off), len(seg_off) - 1, _p(ks), _p(k_off), _p(out))
    if rc:
        raise ValueError("oracle rejected the arguments")
    return out


def cpu_multiselect(values, ks, threads: int = 0, method: int = 1) -> np.ndarray:
    values = np.ascontiguousarray(values)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=values.dtype)
    rc = getattr(lib(), f"ggms_cpu_multiselect_{_SUF[values.dtype]}")(
        _p(values), len(values), _p(ks), len(ks), _p(out), threads, method)
    if rc:
        raise ValueError("cpu baseline rejected the arguments")
    return out


def cpu_multiselect_segmented(values, seg_off, ks, k_off, threads: int = 0) -> np.ndarray:
    """OpenMP per-segment multi-select (checked against select_segmented by the CPU tests)."""
    values = np.ascontiguousarray(values)
    seg_off = np.ascontiguousarray(seg_off, dtype=np.int64)
    k_off = np.ascontiguousarray(k_off, dtype=np.int64)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=values.dtype)
    rc = getattr(lib(), f"ggms_cpu_multiselect_segmented_{_SUF[values.dtype]}")(
        _p(values), _p(seg_off), len(seg_off) - 1, _p(ks), _p(k_off), _p(out), threads)
    if rc:
        raise ValueError("cpu baseline rejected the arguments")
    return out


def cpu_threads() -> int:
    return lib().ggms_cpu_max_threads()


# ------------------------------------------------------------------ keys (numpy)
def keys(values: np.ndarray) -> np.ndarray:
    """Order-preserving unsigned keys (same map as the library and the C oracle)."""
    v = np.ascontiguousarray(values)
    if v.dtype == np.float32:
        u = v.view(np.uint32)
        return u ^ np.where(u >> 31 == 1, np.uint32(0xFFFFFFFF), np.uint32(0x80000000))
    if v.dtype == np.float64:
        u = v.view(np.uint64)
        return u ^ np.where(u >> 63 == 1, np.uint64(0xFFFFFFFFFFFFFFFF), np.uint64(0x8000000000000000))
    if v.dtype == np.int32:
        return v.view(np.uint32) ^ np.uint32(0x80000000)
    if v.dtype == np.uint32:
        return v.copy()
    raise TypeError(v.dtype)


def bits(values: np.ndarray) -> np.ndarray:
    """Bit patterns, for bit-exact comparison (NaN payloads included)."""
    v = np.ascontiguousarray(values)
    return v.view({4: np.uint32, 8: np.uint64}[v.dtype.itemsize])


# ------------------------------------------------------------------ the reference's own build
def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError("reference build oracle/_ref/libggms_ref.so is absent")
        l = ctypes.CDLL(REF_SO)
        for suf in ("f32", "f64", "u32", "i32"):
            for nm in (f"ggms_ref_bucket_multiselect_{suf}", f"ggms_ref_iterative_smos_{suf}"):
                f = getattr(l, nm)
                f.restype = ctypes.c_float
                f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                              ctypes.c_void_p]
        _ref = l
    return _ref


def ref_select(entry: str, values: np.ndarray, ks: np.ndarray):
    """Run the reference's own wrapper (entry 'bucket_multiselect' or
    'iterative_smos') on the GPU; returns (answers, elapsed_ms by the
    reference's own event-timing protocol)."""
    values = np.ascontiguousarray(values)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=values.dtype)
    ms = getattr(ref_lib(), f"ggms_ref_{entry}_{_SUF[values.dtype]}")(
        _p(values), len(values), _p(ks), len(ks), _p(out))
    if ms < 0:
        raise RuntimeError(f"reference run failed ({ms})")
    return out, float(ms)
