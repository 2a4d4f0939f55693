"""Parity at the benchmark's full sizes (the five workload configurations),
on the seeded synthetic inputs the benchmark uses.  Integer results are
bit-exact against the oracle; float results are within 1e-6 relative of the
FP64 oracle."""
import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N24, N28 = 1 << 24, 1 << 28


def dev_bf16(bits):
    return torch.from_numpy(bits.view(np.int16)).cuda().view(torch.bfloat16)


def test_config1_int32_reduce_and_scan(dev):
    x = C.synth_fill(0, 0, N24, -1000, 1000)
    xd = torch.from_numpy(x).cuda()
    assert C.reduce(xd, "sum", init=0).item() == O.reduce(O.I32, O.SUM, x, 0)
    y = C.scan(xd, True, "sum", None).cpu().numpy()
    assert np.array_equal(y, O.scan(O.I32, O.SUM, True, x))


def test_config2_fp32_dot_and_scan(dev):
    a = C.synth_fill(1, 1, N28, 0.125, 1e-6)
    b = C.synth_fill(1, 2, N28, 0.125, 1e-6)
    ref, sabs = O.fp64_sum(O.F32, a, b)
    got = C.dot(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()).item()
    assert abs(got - ref) <= 1e-6 * abs(ref), (got, ref)
    del b
    x = C.synth_fill(2, 3, N28, 0.125, 1e-6)
    xd = torch.from_numpy(x).cuda()
    y = C.scan(xd, True, "sum", None).cpu().numpy().astype(np.float64)
    r = O.fp64_scan(O.F32, True, x)
    assert np.max(np.abs(y - r) / r) <= 1e-6


def test_config2_bf16_dot_and_scan(dev):
    a = C.synth_fill(6, 1, N28, 0.125, 1e-6)
    b = C.synth_fill(6, 2, N28, 0.125, 1e-6)
    ref, _ = O.fp64_sum(O.BF16, a, b)
    got = C.dot(dev_bf16(a), dev_bf16(b)).item()
    assert abs(got - ref) <= 1e-6 * abs(ref), (got, ref)
    del a, b
    x = C.synth_fill(7, 3, N28, 0.125, 1e-6)
    y = C.scan(dev_bf16(x), True, "sum", None).cpu().numpy().astype(np.float64)
    r = O.fp64_scan(O.BF16, True, x)
    assert np.max(np.abs(y - r) / r) <= 1e-6


def test_config3_exclusive_scan_copy_if_histogram(dev):
    x = C.synth_fill(3, 4, N28)
    xd = torch.from_numpy(x).cuda()
    y = C.scan(xd, False, "sum", 0).cpu().numpy()
    assert np.array_equal(y, O.scan(O.U32, O.SUM, False, x, 0))
    del y
    out, cnt = C.copy_if(xd, 7, C.CMP_LT, 3)
    ref, rc = O.copy_if_u32(x, 7, C.CMP_LT, 3)
    assert int(cnt.item()) == rc and 0.37 < rc / N28 < 0.38
    assert np.array_equal(out[:rc].cpu().numpy(), ref)
    del xd, out
    k = C.synth_fill(4, 5, N28, 1.2)
    bins = C.histogram_u8(torch.from_numpy(k).cuda())
    assert np.array_equal(bins.cpu().numpy().astype(np.int64), O.histogram_u8(k).astype(np.int64))
