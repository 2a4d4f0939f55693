"""b2p_reduce_static, the reduce for callers that cannot allocate device
memory (allocator callbacks, fixed-memory real-time paths, runtimes that own
the device heap).  Its scratch lives in the library image instead of a
caller buffer.

Checked through the C-ABI, two calls in a row each time (the second call
reuses the array the first one left behind):
  * integer results against the CPU oracle, bit for bit;
  * float results bit-equal to b2p_reduce on the same input (the float
    reduce result does not depend on the launch configuration);
  * an input that starts off its 16-byte boundary (the path with the most
    runs, so the largest scratch need);
  * a call right after a rejected call still gives the right answer.
This file runs last so that a failure here does not stop the rest of the GPU
suite."""
import ctypes

import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _static(code, op, x, init):
    L = C.lib()
    out = C.zeros(1, C.acc_torch_dtype(code), x.device)
    iv = C._ctype_of(code)(init)
    s = torch.cuda.current_stream()
    rc = L.b2p_reduce_static(code, op, x.data_ptr(), x.numel(), out.data_ptr(),
                             ctypes.cast(ctypes.pointer(iv), ctypes.c_void_p),
                             ctypes.c_void_p(s.cuda_stream))
    assert rc == C.OK, L.b2p_status_string(rc)
    return out


NP_INT = {C.I32: np.int32, C.I64: np.int64, C.U32: np.uint32}


def _input(rng, code, n):
    if code in (C.F32, C.F64):
        a = rng.standard_normal(n).astype(np.float32 if code == C.F32 else np.float64)
        return a, torch.from_numpy(a).cuda()
    if code == C.BF16:
        x = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda().to(torch.bfloat16)
        return None, x
    info = np.iinfo(NP_INT[code])
    a = rng.integers(info.min, info.max, n, dtype=NP_INT[code], endpoint=True)
    return a, torch.from_numpy(a).cuda()


def _init(code, op):
    if op in (C.SUM, C.XOR):
        return 0
    if op == C.MIN:
        return np.inf
    return np.iinfo(np.int64).min


def _check(code, op, host, x, init):
    first = _static(code, op, x, init).cpu().numpy()[0]
    second = _static(code, op, x, init).cpu().numpy()[0]
    if code in (C.F32, C.BF16, C.F64):
        ref = C.reduce(x, op, init=init).cpu().numpy()[0]
        for got in (first, second):
            assert got.tobytes() == ref.tobytes(), (x.numel(), got, ref)
    else:
        ref = O.reduce(code, op, host, init)
        for got in (first, second):
            assert int(got) == int(ref), (x.numel(), got, ref)


@pytest.mark.parametrize("code,op", [(C.I32, C.SUM), (C.I64, C.MAX), (C.U32, C.XOR),
                                     (C.F32, C.SUM), (C.BF16, C.SUM), (C.F64, C.MIN)])
def test_reduce_static_matches_oracle_and_reduce(dev, code, op):
    rng = np.random.default_rng(41 + code * 7 + op)
    init = _init(code, op)
    for n in (1, 1000, (1 << 20) + 3, 1 << 26):
        host, x = _input(rng, code, n)
        _check(code, op, host, x, init)
    # an input one element past a 16-byte boundary
    host, x = _input(rng, code, (1 << 22) + 5)
    _check(code, op, None if host is None else host[1:], x[1:], init)


def test_reduce_static_after_rejected_call(dev):
    L = C.lib()
    rng = np.random.default_rng(5)
    host, x = _input(rng, C.I32, 1 << 21)
    out = torch.zeros(1, dtype=torch.float32, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # XOR is not defined for floats: rejected before the shared array is touched
    rc = L.b2p_reduce_static(C.F32, C.XOR, x.data_ptr(), x.numel(), out.data_ptr(), None, s)
    assert rc == C.ERR_INVALID_ARG
    # a pointer off its element alignment is rejected too
    rc = L.b2p_reduce_static(C.I32, C.SUM, x.data_ptr() + 2, 16, out.data_ptr(), None, s)
    assert rc == C.ERR_INVALID_PTR
    _check(C.I32, C.SUM, host, x, 0)


def test_reduce_static_rejects_oversize(dev):
    L = C.lib()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.b2p_reduce_static(C.I32, C.SUM, x.data_ptr(), (1 << 34) + 1, out.data_ptr(), None, None)
    assert rc == C.ERR_INVALID_ARG
