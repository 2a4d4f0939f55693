"""b2p_reduce_static, the reduce for callers that cannot allocate device
memory (allocator callbacks, fixed-memory real-time paths, runtimes that own
the device heap).  Its scratch lives in the library image instead of a
caller buffer.  Checked through the C-ABI against b2p_reduce on the same
inputs, two calls in a row each time (the second call reuses the array the
first one left behind).  This file runs last so that a failure here does
not stop the rest of the GPU suite."""
import ctypes

import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C

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


@pytest.mark.parametrize("code,op", [(C.I32, C.SUM), (C.I64, C.MAX), (C.U32, C.XOR),
                                     (C.F32, C.SUM), (C.BF16, C.SUM), (C.F64, C.MIN)])
def test_reduce_static_matches_reduce(dev, code, op):
    rng = np.random.default_rng(41 + code * 7 + op)
    for n in (1, 1000, (1 << 20) + 3, 1 << 26):
        if code in (C.F32, C.F64):
            a = rng.standard_normal(n).astype(np.float32 if code == C.F32 else np.float64)
            x = torch.from_numpy(a).cuda()
        elif code == C.BF16:
            x = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda().to(torch.bfloat16)
        else:
            info = np.iinfo({C.I32: np.int32, C.I64: np.int64, C.U32: np.uint32}[code])
            a = rng.integers(info.min, info.max, n, dtype={C.I32: np.int32, C.I64: np.int64,
                                                           C.U32: np.uint32}[code], endpoint=True)
            x = torch.from_numpy(a).cuda()
        init = 0 if op in (C.SUM, C.XOR) else (np.inf if op == C.MIN else np.iinfo(np.int64).min)
        ref = C.reduce(x, op, init=init).cpu().numpy()[0]
        first = _static(code, op, x, init).cpu().numpy()[0]
        second = _static(code, op, x, init).cpu().numpy()[0]
        for got in (first, second):
            if code in (C.F32, C.BF16, C.F64):
                assert abs(float(got) - float(ref)) <= 1e-6 * abs(float(ref)) + 1e-30, (n, got, ref)
            else:
                assert got == ref, (n, got, ref)


def test_reduce_static_rejects_oversize(dev):
    L = C.lib()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.b2p_reduce_static(C.I32, C.SUM, x.data_ptr(), (1 << 34) + 1, out.data_ptr(), None, None)
    assert rc == C.ERR_INVALID_ARG
