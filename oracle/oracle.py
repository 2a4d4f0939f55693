"""ORACLE — test infrastructure only (ctypes wrapper over oracle/oracle.c).

Used by tests/, by ``__graft_entry__.smoke()`` as the checker, and by the CPU
baseline leg of ``bench.py``.  The product never imports this module.

Every function takes and returns numpy arrays.  dtype/op codes are the C-ABI
codes of include/b2p.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

I32, I64, U32, U64, F32, BF16, F64 = range(7)
SUM, PROD, MIN, MAX, AND, OR, XOR = range(7)

NP_OF = {I32: np.int32, I64: np.int64, U32: np.uint32, U64: np.uint64,
         F32: np.float32, BF16: np.uint16, F64: np.float64}
# accumulation / output type (bf16 inputs accumulate and write fp32)
ACC_OF = {I32: np.int32, I64: np.int64, U32: np.uint32, U64: np.uint64,
          F32: np.float32, BF16: np.float32, F64: np.float64}

_lib = None


def build() -> str:
    """Compile oracle.c with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "oracle.c"))):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        L.orc_reduce.argtypes = [i, i, vp, sz, vp, vp]
        L.orc_dot.argtypes = [i, vp, vp, sz, vp, vp]
        L.orc_scan.argtypes = [i, i, i, vp, vp, sz, vp]
        L.orc_copy_if_u32.argtypes = [vp, sz, ctypes.c_uint32, i, ctypes.c_uint32, vp, vp]
        L.orc_histogram_u8.argtypes = [vp, sz, vp, i]
        L.orc_segmented_reduce.argtypes = [i, i, vp, vp, ctypes.c_int64, vp]
        L.orc_segmented_scan.argtypes = [i, i, i, vp, vp, ctypes.c_int64, vp, vp]
        L.orc_fp64_sum.argtypes = [i, vp, vp, sz, ctypes.c_double, vp, vp, vp]
        L.orc_fp64_scan.argtypes = [i, i, vp, sz, ctypes.c_double, vp]
        L.orc_fp64_segmented_sum.argtypes = [i, vp, vp, ctypes.c_int64, vp]
        L.orc_synth_fill.argtypes = [i, ctypes.c_uint64, sz, ctypes.c_double, ctypes.c_double, vp]
        L.orc_set_num_threads.argtypes = [i]
        L.orc_num_threads.restype = i
        for f in ("orc_reduce", "orc_dot", "orc_scan", "orc_copy_if_u32", "orc_histogram_u8",
                  "orc_segmented_reduce", "orc_segmented_scan", "orc_fp64_sum",
                  "orc_fp64_scan", "orc_fp64_segmented_sum", "orc_synth_fill"):
            getattr(L, f).restype = i
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _scalar(v, t):
    return np.array([v], dtype=t)


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


SYNTH_NP = {0: np.int32, 1: np.float32, 2: np.float32, 3: np.uint32, 4: np.uint8, 5: np.int64,
            6: np.uint16, 7: np.uint16}


def synth_fill(kind, seed, n, a=0.0, b=0.0, out=None):
    """Seeded synthetic inputs, the same bits as the library's b2p_synth_fill."""
    if out is None:
        out = np.empty(n, dtype=SYNTH_NP[kind])
    rc = lib().orc_synth_fill(int(kind), int(seed), int(n), float(a), float(b), _p(out))
    assert rc == 0
    return out


def reduce(dtype, op, x, init, out_init=None):
    """hipsycl::algorithms::reduce in OMP-backend order.  Returns the scalar
    written to *out, or ``out_init`` when x is empty (out untouched)."""
    x = np.ascontiguousarray(x, dtype=NP_OF[dtype])
    acc = ACC_OF[dtype]
    out = _scalar(out_init if out_init is not None else 0, acc)
    rc = lib().orc_reduce(dtype, op, _p(x), x.size, _p(_scalar(init, acc)), _p(out))
    assert rc == 0
    return out[0]


def dot(dtype, a, b, init=0.0):
    a = np.ascontiguousarray(a, dtype=NP_OF[dtype])
    b = np.ascontiguousarray(b, dtype=NP_OF[dtype])
    acc = ACC_OF[dtype]
    out = _scalar(0, acc)
    rc = lib().orc_dot(dtype, _p(a), _p(b), a.size, _p(_scalar(init, acc)), _p(out))
    assert rc == 0
    return out[0]


def scan(dtype, op, inclusive, x, init=None, out=None):
    x = np.ascontiguousarray(x, dtype=NP_OF[dtype])
    acc = ACC_OF[dtype]
    y = np.zeros(x.size, dtype=acc) if out is None else out
    assert y.dtype == acc and y.size == x.size and y.flags.c_contiguous
    ini = _scalar(init, acc) if init is not None else None
    rc = lib().orc_scan(dtype, op, int(bool(inclusive)), _p(x), _p(y), x.size, _p(ini))
    assert rc == 0
    return y


def copy_if_u32(x, mask, cmp, rhs):
    x = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.zeros(x.size, dtype=np.uint32)
    cnt = np.zeros(1, dtype=np.uint64)
    rc = lib().orc_copy_if_u32(_p(x), x.size, mask, cmp, rhs, _p(out), _p(cnt))
    assert rc == 0
    return out[: int(cnt[0])], int(cnt[0])


def histogram_u8(keys, nbins=256, bins=None):
    keys = np.ascontiguousarray(keys, dtype=np.uint8)
    b = np.zeros(256, dtype=np.uint32) if bins is None else np.array(bins, dtype=np.uint32).copy()
    if b.size < 256:
        b = np.concatenate([b, np.zeros(256 - b.size, dtype=np.uint32)])
    rc = lib().orc_histogram_u8(_p(keys), keys.size, _p(b), nbins)
    assert rc == 0
    return b[:nbins]


def segmented_reduce(dtype, op, x, offsets):
    x = np.ascontiguousarray(x, dtype=NP_OF[dtype])
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    nseg = offs.size - 1
    out = np.zeros(nseg, dtype=ACC_OF[dtype])
    rc = lib().orc_segmented_reduce(dtype, op, _p(x), _p(offs), nseg, _p(out))
    assert rc == 0
    return out


def segmented_scan(dtype, op, inclusive, x, offsets, init=None):
    x = np.ascontiguousarray(x, dtype=NP_OF[dtype])
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    acc = ACC_OF[dtype]
    y = np.zeros(x.size, dtype=acc)
    ini = _scalar(init, acc) if init is not None else None
    rc = lib().orc_segmented_scan(dtype, op, int(bool(inclusive)), _p(x), _p(offs),
                                  offs.size - 1, _p(y), _p(ini))
    assert rc == 0
    return y


def fp64_sum(dtype, a, b=None, init=0.0):
    """Double-double sum (or dot when b is given).  Returns (value, sum_abs)."""
    a = np.ascontiguousarray(a, dtype=NP_OF[dtype])
    if b is not None:
        b = np.ascontiguousarray(b, dtype=NP_OF[dtype])
    hi = np.zeros(1); lo = np.zeros(1); ab = np.zeros(1)
    rc = lib().orc_fp64_sum(dtype, _p(a), _p(b), a.size, float(init), _p(hi), _p(lo), _p(ab))
    assert rc == 0
    return float(hi[0]) + float(lo[0]), float(ab[0])


def fp64_scan(dtype, inclusive, x, init=0.0):
    x = np.ascontiguousarray(x, dtype=NP_OF[dtype])
    y = np.zeros(x.size, dtype=np.float64)
    rc = lib().orc_fp64_scan(dtype, int(bool(inclusive)), _p(x), x.size, float(init), _p(y))
    assert rc == 0
    return y


def fp64_segmented_sum(dtype, x, offsets):
    x = np.ascontiguousarray(x, dtype=NP_OF[dtype])
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    out = np.zeros(offs.size - 1, dtype=np.float64)
    rc = lib().orc_fp64_segmented_sum(dtype, _p(x), _p(offs), offs.size - 1, _p(out))
    assert rc == 0
    return out


def bf16_round(x):
    """Round fp32 values to bf16 (round-to-nearest-even); returns uint16 bits."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def bf16_to_f32(h):
    return (np.asarray(h, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def merge(a, b, descending=False):
    """Stable merge of two sorted arrays: on equal keys the elements of `a`
    come first (std::merge, which AdaptiveCpp's tests/pstl/merge.cpp:24-43
    compare hipsycl::algorithms::merge against; algorithm.hpp:531-560).
    A stable sort of a ++ b gives exactly that order."""
    x = np.concatenate([np.asarray(a), np.asarray(b)])
    return sort(x, descending)


def sort(x, descending=False):
    """Stable sort (std::stable_sort with std::less / std::greater); for keys
    that compare equal only when identical this is also the unique result of
    std::sort and of the reference's bitonic sort
    (algorithms/sort/bitonic_sort.hpp:69-110), which tests/pstl/sort.cpp:24-37
    compares against std::sort."""
    x = np.asarray(x)
    if not descending:
        return x[np.argsort(x, kind="stable")]
    # descending and stable: reverse, sort ascending stably, reverse back
    r = x[::-1]
    return r[np.argsort(r, kind="stable")][::-1].copy()
