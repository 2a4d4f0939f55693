"""ctypes binding of libb2p.so (the C-ABI declared in include/b2p.h).

This is the Python face of the library used by the tests, the benchmark and
the tuner scripts.  It mirrors the reference's algorithm entry points
(hipsycl::algorithms::reduce / transform_reduce / inclusive_scan /
exclusive_scan / copy_if, algorithms/numeric.hpp:170-297 and
algorithms/algorithm.hpp:178-243) with the same argument meaning: device
tensors in, device tensors out, asynchronous on a CUDA stream.

torch provides device memory and streams only; every computation runs in
libb2p's CUDA kernels.  If the shared library is missing the import of a
compute function raises: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re
import threading
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libb2p.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "b2p.h")

# enums of include/b2p.h
OK, ERR_INVALID_ARG, ERR_INVALID_PTR, ERR_TIMEOUT, ERR_CUDA, ERR_UNSUPPORTED, ERR_SCRATCH, \
    ERR_NO_DEVICE, ERR_IO = range(9)
I32, I64, U32, U64, F32, BF16, F64 = range(7)
SUM, PROD, MIN, MAX, AND, OR, XOR = range(7)
PRIM_REDUCE, PRIM_SCAN, PRIM_COPY_IF, PRIM_HISTOGRAM, PRIM_DOT, PRIM_SEG_REDUCE, PRIM_SEG_SCAN, \
    PRIM_SORT, PRIM_MERGE = range(9)
CMP_LT, CMP_LE, CMP_EQ, CMP_NE, CMP_GE, CMP_GT = range(6)
NUM_CONFIGS = 48
AUTO = -1
SEL_FEATURES = 11

OPS = {"sum": SUM, "plus": SUM, "prod": PROD, "multiplies": PROD, "min": MIN, "minimum": MIN,
       "max": MAX, "maximum": MAX, "and": AND, "or": OR, "xor": XOR}


class B2PError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().b2p_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: b2p status {status} ({msg})")


_lib = None
_lock = threading.Lock()


def lib():
    """Load libb2p.so.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"{LIB_PATH} is missing: build it with `python -m opensycl_b200.build`")
                L = ctypes.CDLL(LIB_PATH)
                _declare(L)
                _lib = L
    return _lib


def _declare(L):
    vp, sz, i, u64, i64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64, ctypes.c_int64
    f, d = ctypes.c_float, ctypes.c_double
    fp = ctypes.POINTER(ctypes.c_float)
    ip = ctypes.POINTER(ctypes.c_int)
    sig = {
        "b2p_version": ([], ctypes.c_char_p),
        "b2p_status_string": ([i], ctypes.c_char_p),
        "b2p_kernel_arch": ([ip, ip], i),
        "b2p_config_describe": ([i, ip, ip, ip], i),
        "b2p_config_valid": ([i, i, i], i),
        "b2p_scratch_bytes": ([i, i, sz, i64, i], sz),
        "b2p_scratch_init": ([vp, sz, vp], i),
        "b2p_reduce": ([i, i, vp, sz, vp, vp, vp, sz, i, vp], i),
        "b2p_dot": ([i, vp, vp, sz, vp, vp, vp, sz, i, vp], i),
        "b2p_reduce_static": ([i, i, vp, sz, vp, vp, vp], i),
        "b2p_scan": ([i, i, i, vp, vp, sz, vp, vp, sz, i, vp], i),
        "b2p_copy_if": ([i, vp, vp, sz, u64, i, u64, vp, vp, sz, i, vp], i),
        "b2p_histogram_u8": ([vp, sz, vp, i, i, vp], i),
        "b2p_merge": ([i, vp, sz, vp, sz, vp, i, vp, sz, vp], i),
        "b2p_sort": ([i, vp, sz, i, vp, sz, vp], i),
        "b2p_sharded_scratch_bytes": ([i, sz, i], sz),
        "b2p_sharded_reduce": ([i, i, vp, sz, vp, vp, vp, sz, i, vp, vp], i),
        "b2p_sharded_scan": ([i, i, i, vp, vp, sz, vp, vp, sz, i, vp, vp], i),
        "b2p_sharded_dot": ([i, vp, vp, sz, vp, vp, vp, sz, i, vp, vp], i),
        "b2p_shard_combine": ([i, i, vp, i, sz, vp, vp], i),
        "b2p_log_level": ([], i),
        "b2p_set_log_level": ([i], None),
        "b2p_segmented_reduce": ([i, i, vp, vp, i64, vp, vp, vp, sz, i, vp], i),
        "b2p_segmented_scan": ([i, i, i, vp, vp, vp, i64, vp, vp, sz, i, vp], i),
        "b2p_segmented_per_call": ([i, i, i, vp, vp, vp, i64, vp, sz, i, vp], i),
        "b2p_device_error": ([vp, vp, i], i),
        "b2p_set_wait_timeout_ns": ([u64], u64),
        "b2p_wait_timeout_ns": ([], u64),
        "b2p_debug_stall_tile": ([i64], None),
        "b2p_plan_segmented": ([ctypes.POINTER(vp), i, i, i, vp, vp, vp, i64, sz, i, vp], i),
        "b2p_plan_launch": ([vp, vp], i),
        "b2p_plan_config": ([vp], i),
        "b2p_plan_destroy": ([vp], None),
        "b2p_tune_shape": ([i, i, i, sz, i64, d, i, u64, fp], i),
        "b2p_selector_create": ([ctypes.POINTER(vp), u64], i),
        "b2p_selector_destroy": ([vp], None),
        "b2p_selector_features": ([i, i, sz, i64, d, fp], i),
        "b2p_selector_train": ([vp, fp, fp, i, i, f, f, fp], i),
        "b2p_selector_predict": ([vp, fp, i, ip], i),
        "b2p_selector_grad": ([vp, fp, fp, i, f, fp, fp], i),
        "b2p_selector_num_params": ([], i),
        "b2p_selector_get_params": ([vp, fp], i),
        "b2p_selector_set_params": ([vp, fp], i),
        "b2p_selector_save": ([vp, ctypes.c_char_p], i),
        "b2p_selector_load": ([vp, ctypes.c_char_p], i),
        "b2p_selector_install": ([vp], i),
        "b2p_heuristic_config": ([i, i, sz, i64], i),
        "b2p_auto_config": ([i, i, sz, i64, d], i),
        "b2p_synth_fill": ([i, u64, sz, d, d, vp], i),
        "b2p_synth_segments": ([u64, i64, d, u64, vp, ctypes.POINTER(u64)], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res


def header_functions() -> list:
    """Names of every function declared in include/b2p.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(b2p_[a-z0-9_]+)\s*\(", text)))


def check(status: int, what: str = "b2p"):
    if status != OK:
        raise B2PError(status, what)


# ------------------------------------------------------------------ torch glue

def _torch():
    import torch
    return torch


def dtype_code(t) -> int:
    torch = _torch()
    m = {torch.int32: I32, torch.int64: I64, torch.uint32: U32, torch.uint64: U64,
         torch.float32: F32, torch.bfloat16: BF16, torch.float64: F64}
    if t.dtype not in m:
        raise TypeError(f"unsupported dtype {t.dtype}")
    return m[t.dtype]


def acc_torch_dtype(code: int):
    torch = _torch()
    return {I32: torch.int32, I64: torch.int64, U32: torch.uint32, U64: torch.uint64,
            F32: torch.float32, BF16: torch.float32, F64: torch.float64}[code]


def zeros(n: int, dtype, device):
    """torch.zeros that also works for uint32/uint64 on CUDA (allocated as the
    signed type of the same width and viewed)."""
    torch = _torch()
    signed = {torch.uint32: torch.int32, torch.uint64: torch.int64}.get(dtype)
    if signed is not None:
        return torch.zeros(n, dtype=signed, device=device).view(dtype)
    return torch.zeros(n, dtype=dtype, device=device)


def _ctype_of(code: int):
    return {I32: ctypes.c_int32, I64: ctypes.c_int64, U32: ctypes.c_uint32, U64: ctypes.c_uint64,
            F32: ctypes.c_float, BF16: ctypes.c_float, F64: ctypes.c_double}[code]


def _init_ptr(code: int, init):
    if init is None:
        return None, None
    v = _ctype_of(code)(init)
    return v, ctypes.cast(ctypes.pointer(v), ctypes.c_void_p)


def _stream(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Scratch:
    """Device scratch cache, one buffer per (device, stream): the analogue of
    util::allocation_cache + allocation_group (algorithms/util/
    allocation_cache.hpp:42-181).  Buffers are zero-filled once when created
    and grow on demand; calls on one stream are ordered, so reuse is safe."""

    _bufs: dict = {}

    @classmethod
    def get(cls, nbytes: int, stream=None):
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream()
        key = (s.device.index, s.cuda_stream)
        buf = cls._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            size = max(nbytes, 1 << 20)
            with torch.cuda.stream(s):
                buf = torch.zeros(size + 256, dtype=torch.uint8, device=s.device)
            cls._bufs[key] = buf
        return buf

    @classmethod
    def release(cls):
        cls._bufs.clear()


def _aligned_ptr(buf) -> int:
    p = buf.data_ptr()
    return (p + 255) & ~255


def scratch_for(prim: int, code: int, n: int, nseg: int = 0, config: int = AUTO, stream=None):
    nbytes = lib().b2p_scratch_bytes(prim, code, n, nseg, config)
    buf = Scratch.get(nbytes + 256, stream)
    return ctypes.c_void_p(_aligned_ptr(buf)), buf.numel() - 256


# ------------------------------------------------------------------ primitives

def reduce(x, op="sum", init=0, out=None, config: int = AUTO, stream=None):
    """*out = op(init, x...) (init=None: combine with the existing *out)."""
    torch = _torch()
    code = dtype_code(x)
    opc = OPS[op] if isinstance(op, str) else int(op)
    if out is None:
        out = zeros(1, acc_torch_dtype(code), x.device)
    _, ip = _init_ptr(code, init)
    sp, sb = scratch_for(PRIM_REDUCE, code, x.numel(), 0, config, stream)
    check(lib().b2p_reduce(code, opc, x.data_ptr(), x.numel(), out.data_ptr(), ip, sp, sb, config,
                           _stream(stream)), "b2p_reduce")
    return out


def dot(a, b, init=0.0, out=None, config: int = AUTO, stream=None):
    torch = _torch()
    code = dtype_code(a)
    if out is None:
        out = zeros(1, acc_torch_dtype(code), a.device)
    _, ip = _init_ptr(code, init)
    sp, sb = scratch_for(PRIM_DOT, code, a.numel(), 0, config, stream)
    check(lib().b2p_dot(code, a.data_ptr(), b.data_ptr(), a.numel(), out.data_ptr(), ip, sp, sb,
                        config, _stream(stream)), "b2p_dot")
    return out


def scan(x, inclusive=True, op="sum", init=None, out=None, config: int = AUTO, stream=None):
    torch = _torch()
    code = dtype_code(x)
    opc = OPS[op] if isinstance(op, str) else int(op)
    if out is None:
        out = torch.empty(x.numel(), dtype=acc_torch_dtype(code), device=x.device)
    _, ip = _init_ptr(code, init)
    sp, sb = scratch_for(PRIM_SCAN, code, x.numel(), 0, config, stream)
    check(lib().b2p_scan(code, opc, int(bool(inclusive)), x.data_ptr(), out.data_ptr(), x.numel(),
                         ip, sp, sb, config, _stream(stream)), "b2p_scan")
    return out


def inclusive_scan(x, op="sum", init=None, **kw):
    return scan(x, True, op, init, **kw)


def exclusive_scan(x, init, op="sum", **kw):
    return scan(x, False, op, init, **kw)


def copy_if(x, mask, cmp, rhs, out=None, count=None, config: int = AUTO, stream=None):
    """Order-preserving compaction of elements with (x & mask) CMP rhs.
    Returns (out, count) with count a 1-element uint64 device tensor."""
    torch = _torch()
    code = dtype_code(x)
    if out is None:
        out = torch.empty_like(x)
    if count is None:
        count = zeros(1, torch.uint64, x.device)
    sp, sb = scratch_for(PRIM_COPY_IF, code, x.numel(), 0, config, stream)
    check(lib().b2p_copy_if(code, x.data_ptr(), out.data_ptr(), x.numel(), mask, cmp, rhs,
                            count.data_ptr(), sp, sb, config, _stream(stream)), "b2p_copy_if")
    return out, count


def histogram_u8(keys, bins=None, nbins=256, config: int = AUTO, stream=None):
    torch = _torch()
    if bins is None:
        bins = torch.zeros(nbins, dtype=torch.int32, device=keys.device)
    check(lib().b2p_histogram_u8(keys.data_ptr(), keys.numel(), bins.data_ptr(), nbins, config,
                                 _stream(stream)), "b2p_histogram_u8")
    return bins


def merge(a, b, out=None, descending=False, stream=None):
    """Stable merge of two sorted 1-D tensors of one dtype (elements of `a`
    first on equal keys), like std::merge with std::less / std::greater.
    The tile starts go to a buffer of their own (not the per-stream
    look-back scratch)."""
    torch = _torch()
    code = dtype_code(a)
    if dtype_code(b) != code:
        raise ValueError("merge: a and b must have the same dtype")
    total = a.numel() + b.numel()
    if out is None:
        out = torch.empty(total, dtype=a.dtype, device=a.device)
    nbytes = lib().b2p_scratch_bytes(PRIM_MERGE, code, total, 0, AUTO)
    s = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(s):
        tmp = torch.empty(nbytes, dtype=torch.uint8, device=a.device)
    check(lib().b2p_merge(code, a.data_ptr(), a.numel(), b.data_ptr(), b.numel(), out.data_ptr(),
                          int(bool(descending)), tmp.data_ptr(), nbytes, _stream(stream)), "b2p_merge")
    return out


def sort_(keys, descending=False, stream=None):
    """Stable in-place sort of a 1-D tensor, like std::stable_sort.  The
    merge passes ping-pong through a second array of n keys: a buffer of its
    own, not the per-stream scratch, whose look-back status words must only
    ever hold status words."""
    torch = _torch()
    code = dtype_code(keys)
    nbytes = lib().b2p_scratch_bytes(PRIM_SORT, code, keys.numel(), 0, AUTO)
    s = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(s):
        tmp = torch.empty(nbytes, dtype=torch.uint8, device=keys.device)
    check(lib().b2p_sort(code, keys.data_ptr(), keys.numel(), int(bool(descending)), tmp.data_ptr(),
                         nbytes, _stream(stream)), "b2p_sort")
    return keys


def segmented_reduce(x, offsets, op="sum", init=None, out=None, config: int = AUTO, stream=None):
    torch = _torch()
    code = dtype_code(x)
    opc = OPS[op] if isinstance(op, str) else int(op)
    nseg = offsets.numel() - 1
    if out is None:
        out = torch.empty(nseg, dtype=acc_torch_dtype(code), device=x.device)
    _, ip = _init_ptr(code, init)
    sp, sb = scratch_for(PRIM_SEG_REDUCE, code, x.numel(), nseg, config, stream)
    check(lib().b2p_segmented_reduce(code, opc, x.data_ptr(), offsets.data_ptr(), nseg,
                                     out.data_ptr(), ip, sp, sb, config, _stream(stream)),
          "b2p_segmented_reduce")
    return out


def segmented_scan(x, offsets, inclusive=True, op="sum", init=None, out=None, config: int = AUTO,
                   stream=None):
    torch = _torch()
    code = dtype_code(x)
    opc = OPS[op] if isinstance(op, str) else int(op)
    nseg = offsets.numel() - 1
    if out is None:
        out = torch.empty(x.numel(), dtype=acc_torch_dtype(code), device=x.device)
    _, ip = _init_ptr(code, init)
    sp, sb = scratch_for(PRIM_SEG_SCAN, code, x.numel(), nseg, config, stream)
    check(lib().b2p_segmented_scan(code, opc, int(bool(inclusive)), x.data_ptr(), out.data_ptr(),
                                   offsets.data_ptr(), nseg, ip, sp, sb, config, _stream(stream)),
          "b2p_segmented_scan")
    return out


def device_error(stream=None, clear=True, scratchless=False) -> int:
    """Sticky device-side error recorded in this stream's scratch, or with
    scratchless=True the library's word for calls without scratch (histogram)."""
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    if scratchless:
        return lib().b2p_device_error(None, _stream(s), int(clear))
    buf = Scratch.get(256, s)
    return lib().b2p_device_error(ctypes.c_void_p(_aligned_ptr(buf)), _stream(s), int(clear))


# ------------------------------------------------------------------ host-only helpers

def config_describe(c: int):
    b, it, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib().b2p_config_describe(c, ctypes.byref(b), ctypes.byref(it), ctypes.byref(g)))
    return b.value, it.value, g.value


def synth_fill(kind: int, seed: int, n: int, a: float = 0.0, b: float = 0.0):
    """Seeded synthetic workload in host memory (numpy array)."""
    import numpy as np
    dt = {0: np.int32, 1: np.float32, 2: np.float32, 3: np.uint32, 4: np.uint8, 5: np.int64,
          6: np.uint16, 7: np.uint16}[kind]
    arr = np.empty(n, dtype=dt)
    check(lib().b2p_synth_fill(kind, seed, n, a, b, arr.ctypes.data_as(ctypes.c_void_p)),
          "b2p_synth_fill")
    return arr


def synth_segments(seed: int, nseg: int, log2max: float, cap: int):
    import numpy as np
    offs = np.empty(nseg + 1, dtype=np.int64)
    tot = ctypes.c_uint64()
    check(lib().b2p_synth_segments(seed, nseg, log2max, cap, offs.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.byref(tot)), "b2p_synth_segments")
    return offs
