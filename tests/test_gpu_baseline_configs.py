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


def _plan_run(prim, code, x, out, od, nseg, total):
    import ctypes
    L = C.lib()
    plan = ctypes.c_void_p()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    C.check(L.b2p_plan_segmented(ctypes.byref(plan), prim, code, C.SUM, x.data_ptr(), out.data_ptr(),
                                 od.data_ptr(), nseg, total, C.AUTO, s), "plan")
    try:
        for _ in range(2):  # a replayed graph gives the same result
            out.fill_(7)
            C.check(L.b2p_plan_launch(plan, s), "launch")
            torch.cuda.synchronize()
    finally:
        L.b2p_plan_destroy(plan)
    return out.cpu().numpy()


def test_config4_segmented_full_shape(dev):
    """10,000 segments with lengths log-uniform in [1, 2^20] scaled to 2^28
    elements in total (seed 6), fp32 N(0,1) (seed 7) and int64
    U[-2^20, 2^20] (seed 8): per-segment sum and inclusive scan through the
    CUDA-graph plan, as the benchmark runs them.  int64 bit-exact against the
    oracle; fp32 against float64 within 1e-6 relative, plus a condition term
    for segments and prefixes whose sum cancels (values of both signs):
    reduce 1e-12 * sum|x|, scan 2^-22 * prefix sum|x| (one fp32 rounding of
    the thread-local running value)."""
    nseg = 10000
    offs = C.synth_segments(6, nseg, 20.0, N28)
    total = int(offs[-1])
    assert total > 0.99 * N28 and np.diff(offs).min() >= 1
    od = torch.from_numpy(offs).cuda()
    # int64
    x = C.synth_fill(5, 8, total, -(1 << 20), 1 << 20)
    xd = torch.from_numpy(x).cuda()
    got = _plan_run(C.PRIM_SEG_REDUCE, C.I64, xd, torch.empty(nseg, dtype=torch.int64, device="cuda"),
                    od, nseg, total)
    assert np.array_equal(got, O.segmented_reduce(O.I64, O.SUM, x, offs))
    yd = torch.empty(total, dtype=torch.int64, device="cuda")
    got = _plan_run(C.PRIM_SEG_SCAN, C.I64, xd, yd, od, nseg, total)
    assert np.array_equal(got, O.segmented_scan(O.I64, O.SUM, True, x, offs))
    del x, xd, yd, got
    # fp32
    x = C.synth_fill(1, 7, total, 0.0, 0.0)
    xd = torch.from_numpy(x).cuda()
    got = _plan_run(C.PRIM_SEG_REDUCE, C.F32, xd, torch.empty(nseg, dtype=torch.float32, device="cuda"),
                    od, nseg, total).astype(np.float64)
    ref = O.fp64_segmented_sum(O.F32, x, offs)
    sabs = np.add.reduceat(np.abs(x).astype(np.float64), offs[:-1])
    assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-12 * sabs)
    yd = torch.empty(total, dtype=torch.float32, device="cuda")
    y = _plan_run(C.PRIM_SEG_SCAN, C.F32, xd, yd, od, nseg, total)
    del yd, xd
    worst = 0.0
    for s in range(nseg):
        a, b = int(offs[s]), int(offs[s + 1])
        seg = x[a:b].astype(np.float64)
        r = np.cumsum(seg)
        cabs = np.cumsum(np.abs(seg))
        err = np.abs(y[a:b].astype(np.float64) - r)
        tol = 1e-6 * np.abs(r) + 2.0 ** -22 * cabs
        assert np.all(err <= tol), (s, float(np.max(err / tol)))
        worst = max(worst, float(np.max(err / np.maximum(cabs, 1e-300))))
    assert worst <= 2.0 ** -22
