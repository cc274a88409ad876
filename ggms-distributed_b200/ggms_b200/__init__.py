"""Python binding of the B200 multiselect library (ctypes over include/ggms.h).

The library is ``ggms-distributed_b200/lib/libggms_b200.so`` (built in-tree by
``make -C ggms-distributed_b200``).  Loading fails loudly when it is missing:
there is no CPU fallback anywhere in this package.

The drop-in names mirror the reference's entry points
(FrzNo1/GGMS-Distributed, DistributedSMOS/bucketMultiselect.cuh:101-107 and
DistributedSMOS/iterativeSMOS.cuh:214-220): a device vector, its length, a host
array of 1-based k-th-largest ranks and a host output array.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libggms_b200.so")
HEADER_PATHS = [os.path.join(REPO_ROOT, "include", "ggms.h"),
                os.path.join(REPO_ROOT, "include", "ggms_diag.h"),
                os.path.join(REPO_ROOT, "include", "ggms_noalloc.h"),
                os.path.join(REPO_ROOT, "include", "ggms_generate.h")]
NOALLOC_MAX_KS = 1024

GGMS_OK = 0
GGMS_E_INVALID_ARG = 1
GGMS_E_OOM = 2
GGMS_E_NOT_CONVERGED = 3
GGMS_E_CUDA = 4
GGMS_E_UNSUPPORTED = 5
GGMS_E_INTERNAL = 6

ASSIGNER_AUTO = 0
ASSIGNER_SAMPLED = 1
ASSIGNER_LEARNED_PL = 2
ASSIGNER_LEARNED_MLP = 3
ASSIGNER_NAMES = {0: "auto", 1: "sampled", 2: "learned_pl", 3: "learned_mlp"}
PL_KNOTS = 1024   # most segments of the learned piecewise-linear CDF (opts.pl_knots picks fewer)
PHASES = ("sample_sort", "assigner", "windows", "pass1", "between", "pass2", "finish", "answers")

SUFFIX = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64",
          np.dtype(np.uint32): "u32", np.dtype(np.int32): "i32"}


class GGMSError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: status {status} ({status_string(status)})")


class Stats(ctypes.Structure):
    _fields_ = [
        ("assigner_used", ctypes.c_int32),
        ("num_buckets", ctypes.c_int32),
        ("full_passes", ctypes.c_int32),
        ("levels", ctypes.c_int32),
        ("candidates", ctypes.c_int64),
        ("refine_elements", ctypes.c_int64),
        ("active_buckets", ctypes.c_int32),
        ("point_buckets", ctypes.c_int32),
        ("small_segments", ctypes.c_int32),
        ("sample_size", ctypes.c_int32),
        ("bucket_max_over_mean", ctypes.c_float),
        ("model_imbalance", ctypes.c_float),
        ("model_loss", ctypes.c_float),
        ("window_runs", ctypes.c_int32),
        ("model_segments", ctypes.c_int32),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["assigner_used"] = ASSIGNER_NAMES.get(self.assigner_used, self.assigner_used)
        return d


class Opts(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("assigner", ctypes.c_int32),
        ("num_buckets", ctypes.c_int32),
        ("sample_size", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("imbalance_bound", ctypes.c_float),
        ("train_steps", ctypes.c_int32),
        ("ks_on_device", ctypes.c_int32),
        ("out_on_device", ctypes.c_int32),
        ("pass_threads", ctypes.c_int32),
        ("pass_unroll", ctypes.c_int32),
        ("window_z", ctypes.c_float),
        ("autotune", ctypes.c_int32),
        ("stats", ctypes.POINTER(Stats)),
        ("pl_knots", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
    ]


_lib: Optional[ctypes.CDLL] = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"ggms CUDA library not found at {path}; build it with "
            f"`make -C {PKG_ROOT}` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    vp, i32, i64, u32p = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p
    lib.ggms_status_string.restype = ctypes.c_char_p
    lib.ggms_status_string.argtypes = [i32]
    lib.ggms_version.restype = i32
    lib.ggms_default_opts.argtypes = [ctypes.POINTER(Opts)]
    lib.ggms_create.argtypes = [ctypes.POINTER(vp), i32]
    lib.ggms_destroy.argtypes = [vp]
    for suf in ("f32", "f64", "u32", "i32"):
        for name in (f"ggms_bucket_multiselect_{suf}", f"ggms_iterative_smos_{suf}"):
            fn = getattr(lib, name)
            fn.restype = i32
            fn.argtypes = [vp, i32, u32p, i32, vp, i32, i32]
        fn = getattr(lib, f"ggms_multiselect_{suf}_ex")
        fn.restype = i32
        fn.argtypes = [vp, vp, i64, u32p, i64, vp, ctypes.POINTER(Opts), vp]
    for suf in ("f32", "f64", "u32", "i32"):
        fn = getattr(lib, f"ggms_topk_{suf}")
        fn.restype = i32
        fn.argtypes = [vp, vp, i64, i64, vp, ctypes.POINTER(Opts), vp]
    for suf in ("f32", "u32"):
        fn = getattr(lib, f"ggms_multiselect_segmented_{suf}")
        fn.restype = i32
        fn.argtypes = [vp, vp, vp, i64, vp, vp, vp, ctypes.POINTER(Opts), vp]
    lib.ggms_get_default_context.argtypes = [ctypes.POINTER(vp)]
    lib.ggms_context_profile.argtypes = [vp, i32]
    lib.ggms_context_pass_times.argtypes = [vp, vp, vp, vp, i32]
    lib.ggms_context_phase_times.restype = i32
    lib.ggms_context_phase_times.argtypes = [vp, vp, i32]
    lib.ggms_context_status.restype = i32
    lib.ggms_context_status.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_int)]
    lib.ggms_context_launches.restype = i64
    lib.ggms_context_launches.argtypes = [vp]
    lib.ggms_context_graph_launches.restype = i64
    lib.ggms_context_graph_launches.argtypes = [vp]
    lib.ggms_diag_pl_gradient.restype = i32
    lib.ggms_diag_pl_gradient.argtypes = [vp, i32, vp, vp, vp, vp, vp]
    lib.ggms_diag_mlp_gradient.restype = i32
    lib.ggms_diag_mlp_gradient.argtypes = [vp, vp, vp, vp, vp]
    lib.ggms_diag_fit.restype = i32
    lib.ggms_diag_fit.argtypes = [vp, i32, i32, i32, vp, vp, vp, vp]
    lib.ggms_multiselect_noalloc_f32.restype = i32
    lib.ggms_multiselect_noalloc_f32.argtypes = [vp, i64, u32p, ctypes.c_int32, vp, vp]
    for suf in ("f32", "f64", "u32"):
        fn = getattr(lib, f"ggms_generate_{suf}")
        fn.restype = i32
        fn.argtypes = [vp, i64, i32, ctypes.c_uint64, vp]
    _lib = lib
    return lib


def status_string(s: int) -> str:
    try:
        return load().ggms_status_string(s).decode()
    except Exception:  # library missing: still give a readable error
        return "?"


def default_opts(**kw) -> Opts:
    o = Opts()
    load().ggms_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Context:
    """Owns a device workspace; reuse it across calls on one host thread."""

    def __init__(self, device: int = 0):
        self.ptr = ctypes.c_void_p()
        rc = load().ggms_create(ctypes.byref(self.ptr), device)
        if rc:
            raise GGMSError(rc, "ggms_create")

    def close(self):
        if self.ptr:
            load().ggms_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def status(self, stream: int = 0) -> int:
        """Device-side status of the last call this context enqueued (waits for it)."""
        st = ctypes.c_int(0)
        rc = load().ggms_context_status(self.ptr, ctypes.c_void_p(stream), ctypes.byref(st))
        if rc:
            raise GGMSError(rc, "ggms_context_status")
        return st.value

    def phase_times(self, max_calls: int = 256):
        """Per-phase device times (ms) of the profiled calls: a list of dicts keyed by PHASES."""
        buf = (ctypes.c_float * (len(PHASES) * max_calls))()
        got = load().ggms_context_phase_times(self.ptr, buf, max_calls)
        if got < 0:
            raise GGMSError(-got, "ggms_context_phase_times")
        return [dict(zip(PHASES, buf[i * len(PHASES):(i + 1) * len(PHASES)])) for i in range(got)]


def _suffix(dtype) -> str:
    try:
        return SUFFIX[np.dtype(dtype)]
    except KeyError:
        raise TypeError(f"unsupported dtype {dtype}; use float32, float64, uint32 or int32")


def _np_dtype_of_torch(t):
    import torch
    return {torch.float32: np.float32, torch.float64: np.float64,
            torch.int32: np.int32}.get(t.dtype) or (np.uint32 if str(t.dtype) == "torch.uint32" else None)


def dropin(entry: str, d_ptr: int, length: int, ks: np.ndarray, dtype, blocks: int = 148,
           threads: int = 1024) -> np.ndarray:
    """Call ggms_<entry>_<suffix> (entry: 'bucket_multiselect' or 'iterative_smos')."""
    lib = load()
    suf = _suffix(dtype)
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=dtype)
    fn = getattr(lib, f"ggms_{entry}_{suf}")
    rc = fn(ctypes.c_void_p(d_ptr), int(length), ks.ctypes.data_as(ctypes.c_void_p), len(ks),
            out.ctypes.data_as(ctypes.c_void_p), blocks, threads)
    if rc:
        raise GGMSError(rc, f"ggms_{entry}_{suf}")
    return out


def multiselect_ex(ctx: Optional[Context], d_ptr: int, n: int, ks, nk: int, out, dtype,
                   opts: Optional[Opts] = None, stream: int = 0) -> int:
    """Raw _ex call.  ks / out are host numpy arrays or device pointers (ints),
    as flagged in opts.  Returns the status code."""
    lib = load()
    suf = _suffix(dtype)
    fn = getattr(lib, f"ggms_multiselect_{suf}_ex")
    kp = ks.ctypes.data_as(ctypes.c_void_p) if isinstance(ks, np.ndarray) else ctypes.c_void_p(ks)
    op = out.ctypes.data_as(ctypes.c_void_p) if isinstance(out, np.ndarray) else ctypes.c_void_p(out)
    return fn(ctx.ptr if ctx else None, ctypes.c_void_p(d_ptr), int(n), kp, int(nk), op,
              ctypes.byref(opts) if opts is not None else None, ctypes.c_void_p(stream))


def select(ctx: Optional[Context], d_ptr: int, n: int, ks: np.ndarray, dtype, assigner: int = 0,
           stats: bool = False, **kw):
    """Host ks -> host answers through the _ex entry point; optional stats."""
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.empty(len(ks), dtype=dtype)
    st = Stats()
    o = default_opts(assigner=assigner, **kw)
    if stats:
        o.stats = ctypes.pointer(st)
    rc = multiselect_ex(ctx, d_ptr, n, ks, len(ks), out, dtype, o)
    if rc:
        raise GGMSError(rc, "ggms_multiselect_ex")
    return (out, st.as_dict()) if stats else out


def topk(ctx: Optional[Context], d_ptr: int, n: int, K: int, dtype, **kw) -> np.ndarray:
    """The K largest values, largest first (host result)."""
    out = np.empty(K, dtype=dtype)
    o = default_opts(**kw)
    rc = getattr(load(), f"ggms_topk_{_suffix(dtype)}")(
        ctx.ptr if ctx else None, ctypes.c_void_p(d_ptr), int(n), int(K),
        out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(o), None)
    if rc:
        raise GGMSError(rc, "ggms_topk")
    return out


def segmented(ctx: Optional[Context], d_ptr: int, seg_off_ptr: int, nseg: int, ks_ptr: int,
              k_off_ptr: int, out_ptr: int, dtype, opts: Optional[Opts] = None,
              stream: int = 0) -> int:
    lib = load()
    suf = _suffix(dtype)
    fn = getattr(lib, f"ggms_multiselect_segmented_{suf}")
    return fn(ctx.ptr if ctx else None, ctypes.c_void_p(d_ptr), ctypes.c_void_p(seg_off_ptr),
              int(nseg), ctypes.c_void_p(ks_ptr), ctypes.c_void_p(k_off_ptr),
              ctypes.c_void_p(out_ptr), ctypes.byref(opts) if opts is not None else None,
              ctypes.c_void_p(stream))


def multiselect_noalloc_f32(d_ptr: int, n: int, ks: np.ndarray, out_ptr: int, stream: int = 0) -> int:
    """ggms_multiselect_noalloc_f32: float32 vector and output in device memory,
    ks (1-based k-th largest) in host memory; enqueues on `stream` and returns
    the status without a host sync."""
    lib = load()
    ks = np.ascontiguousarray(ks, dtype=np.uint32)
    return lib.ggms_multiselect_noalloc_f32(ctypes.c_void_p(d_ptr), int(n),
                                            ks.ctypes.data_as(ctypes.c_void_p), int(len(ks)),
                                            ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream))


def generate(d_ptr: int, n: int, dtype, kind: int, seed: int, stream: int = 0) -> int:
    """ggms_generate_<suffix>: fill n elements at device pointer d_ptr with the
    reference's generator number `kind` of that value type (float32, float64 or
    uint32); enqueued on `stream`, returns the status without a host sync."""
    lib = load()
    suf = _suffix(dtype)
    if suf == "i32":
        raise TypeError("no generator table for int32")
    return getattr(lib, f"ggms_generate_{suf}")(ctypes.c_void_p(d_ptr), int(n), int(kind),
                                                ctypes.c_uint64(seed & (2**64 - 1)),
                                                ctypes.c_void_p(stream))


def declared_symbols(paths=None):
    """Function names declared with GGMS_API in the public headers."""
    import re
    names = []
    for p in paths or HEADER_PATHS:
        with open(p) as f:
            txt = f.read()
        names += re.findall(r"GGMS_API\s+[\w\s\*]+?\b(ggms_\w+)\s*\(", txt)
    return sorted(set(names))


# ------------------------------------------------------------------ learned-model diagnostics
def _fp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def diag_pl_gradient(sorted_keys: np.ndarray, theta: np.ndarray):
    """GPU loss/gradient of the PL-CDF model; returns (loss, grad[:M], knots[:M+1])."""
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint32)
    th = np.zeros(PL_KNOTS, np.float32)
    th[:len(theta)] = theta
    loss = np.zeros(1, np.float32)
    grad = np.zeros(PL_KNOTS, np.float32)
    knots = np.zeros(PL_KNOTS + 1, np.uint32)
    m = ctypes.c_int(0)
    rc = load().ggms_diag_pl_gradient(_fp(k), len(k), _fp(th), _fp(loss), _fp(grad), _fp(knots),
                                      ctypes.byref(m))
    if rc:
        raise GGMSError(rc, "ggms_diag_pl_gradient")
    return float(loss[0]), grad[:m.value].copy(), knots[:m.value + 1].copy()


def diag_mlp_gradient(x: np.ndarray, t: np.ndarray, params: np.ndarray):
    x = np.ascontiguousarray(x, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    assert len(x) == 1024 and len(t) == 1024 and len(p) == 1153
    loss = np.zeros(1, np.float32)
    grad = np.zeros(1153, np.float32)
    rc = load().ggms_diag_mlp_gradient(_fp(x), _fp(t), _fp(p), _fp(loss), _fp(grad))
    if rc:
        raise GGMSError(rc, "ggms_diag_mlp_gradient")
    return float(loss[0]), grad


def diag_fit(sorted_keys: np.ndarray, kind: int, steps: int = 0):
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint32)
    out = np.zeros(4, np.float32)
    f = [ctypes.c_float() for _ in range(4)]
    rc = load().ggms_diag_fit(_fp(k), len(k), kind, steps, *[ctypes.byref(v) for v in f])
    if rc:
        raise GGMSError(rc, "ggms_diag_fit")
    return {"loss_before": f[0].value, "loss_after": f[1].value,
            "imbalance_model": f[2].value, "imbalance_sampled": f[3].value}
