"""Segmented reduce / scan (one persistent launch for all segments) and the
CUDA-graph plans, against per-segment oracle calls."""
import ctypes

import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NP = {C.I32: np.int32, C.I64: np.int64, C.F32: np.float32, C.F64: np.float64}
SEG_CONFIGS = [0, 6, 22, 41, C.AUTO]


def make_offsets(rng, nseg, kind):
    if kind == "small":
        lens = rng.integers(0, 40, nseg)
    elif kind == "mixed":
        lens = np.floor(2.0 ** (rng.random(nseg) * 17)).astype(np.int64)
        lens[rng.random(nseg) < 0.1] = 0
    else:  # long: many pieces per segment
        lens = rng.integers(20000, 90000, nseg)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)


def values(rng, code, n):
    if code in (C.F32, C.F64):
        return rng.standard_normal(n).astype(NP[code])
    return rng.integers(-(1 << 20), 1 << 20, n).astype(NP[code])


def valid(code, cfgs):
    L = C.lib()
    return [c for c in cfgs if c == C.AUTO or L.b2p_config_valid(C.PRIM_SEG_REDUCE, code, c)]


@pytest.mark.parametrize("kind", ["small", "mixed", "long"])
@pytest.mark.parametrize("code", [C.I32, C.I64, C.F32])
def test_segmented_reduce(dev, kind, code):
    rng = np.random.default_rng(hash((kind, code)) % 2**32)
    nseg = {"small": 3000, "mixed": 700, "long": 40}[kind]
    offs = make_offsets(rng, nseg, kind)
    x = values(rng, code, int(offs[-1]))
    xd = torch.from_numpy(x).cuda()
    od = torch.from_numpy(offs).cuda()
    if code == C.F32:
        ref = O.fp64_segmented_sum(code, x, offs)
        sabs = np.array([np.abs(x[offs[s]:offs[s + 1]]).astype(np.float64).sum() for s in range(nseg)])
    else:
        ref = O.segmented_reduce(code, C.SUM, x, offs)
    for cfg in valid(code, SEG_CONFIGS):
        got = C.segmented_reduce(xd, od, "sum", config=cfg).cpu().numpy()
        if code == C.F32:
            err = np.abs(got.astype(np.float64) - ref)
            assert np.all(err <= 1e-6 * np.abs(ref) + 1e-12 * sabs + 1e-30), (kind, cfg)
        else:
            assert np.array_equal(got, ref), (kind, cfg)
    if code != C.F32:
        for op in (C.MIN, C.MAX):
            got = C.segmented_reduce(xd, od, op, config=C.AUTO).cpu().numpy()
            info = np.iinfo(NP[code])
            ident = info.max if op == C.MIN else info.min
            exp = np.array([(x[offs[s]:offs[s + 1]].min() if op == C.MIN else x[offs[s]:offs[s + 1]].max())
                            if offs[s + 1] > offs[s] else ident for s in range(nseg)], dtype=NP[code])
            assert np.array_equal(got, exp)


@pytest.mark.parametrize("kind", ["small", "mixed", "long"])
@pytest.mark.parametrize("code", [C.I64, C.F32])
def test_segmented_scan(dev, kind, code):
    rng = np.random.default_rng(7 + hash((kind, code)) % 2**31)
    nseg = {"small": 2000, "mixed": 500, "long": 30}[kind]
    offs = make_offsets(rng, nseg, kind)
    x = values(rng, code, int(offs[-1]))
    if code == C.F32:
        x = np.abs(x)
    xd = torch.from_numpy(x).cuda()
    od = torch.from_numpy(offs).cuda()
    for cfg in valid(code, SEG_CONFIGS):
        for inclusive, init in ((True, None), (True, 3), (False, 5)):
            got = C.segmented_scan(xd, od, inclusive, "sum", init, config=cfg).cpu().numpy()
            if code == C.F32:
                ref = np.concatenate([O.fp64_scan(O.F32, inclusive, x[offs[s]:offs[s + 1]],
                                                  float(init or 0)) for s in range(nseg)
                                      if offs[s + 1] > offs[s]])
                ok = np.abs(got.astype(np.float64) - ref) <= 1e-6 * np.abs(ref) + 1e-30
                assert ok.all(), (kind, cfg, inclusive)
            else:
                ref = O.segmented_scan(code, C.SUM, inclusive, x, offs, init)
                assert np.array_equal(got, ref), (kind, cfg, inclusive, init)


def test_segmented_plan_graph(dev):
    rng = np.random.default_rng(3)
    offs = make_offsets(rng, 1000, "mixed")
    x = values(rng, C.I64, int(offs[-1]))
    xd = torch.from_numpy(x).cuda()
    od = torch.from_numpy(offs).cuda()
    out = torch.zeros(1000, dtype=torch.int64, device="cuda")
    L = C.lib()
    plan = ctypes.c_void_p()
    s = torch.cuda.current_stream()
    C.check(L.b2p_plan_segmented(ctypes.byref(plan), C.PRIM_SEG_REDUCE, C.I64, C.SUM, xd.data_ptr(),
                                 out.data_ptr(), od.data_ptr(), 1000, int(offs[-1]), C.AUTO,
                                 ctypes.c_void_p(s.cuda_stream)), "plan")
    ref = O.segmented_reduce(C.I64, C.SUM, x, offs)
    for _ in range(3):
        out.zero_()
        C.check(L.b2p_plan_launch(plan, ctypes.c_void_p(s.cuda_stream)), "launch")
        assert np.array_equal(out.cpu().numpy(), ref)
    assert 0 <= L.b2p_plan_config(plan) < 48
    L.b2p_plan_destroy(plan)
