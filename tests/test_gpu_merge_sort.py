"""GPU parity of b2p_merge / b2p_sort (the hipsycl::algorithms::merge /
sort path) against the oracle's stable merge and sort, through the C-ABI.

Bar: bit-exact (keys are moved, never computed), including the order of
keys that compare equal but differ in their bits (-0.0 / +0.0: the stable
order).  Cases: the known answers of the reference's tests/pstl/merge.cpp
and sort.cpp (tests/golden/merge_sort_cases.npz), every key type in both
directions at sizes around the merge and radix tiles (b2p_sort runs the
radix sort from 2^15 keys on), ragged and empty inputs, extreme keys,
duplicates-heavy keys, and at 2^28 keys size-independent properties
(sorted, the same multiset as the input: the sum of the keys and the
histogram of their top byte).
"""
import os

import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "merge_sort_cases.npz")
DT = [C.I32, C.I64, C.U32, C.U64, C.F32, C.F64]
NP = {C.I32: np.int32, C.I64: np.int64, C.U32: np.uint32, C.U64: np.uint64, C.F32: np.float32,
      C.F64: np.float64}
# around the merge sort's 4096-key tiles, the radix sort's start (2^15 keys)
# and its 8192-key tiles
SIZES = [1, 2, 7, 255, 2047, 2048, 2049, 4096, 3 * 2048 + 17, 32767, 32768, 5 * 8192, 5 * 8192 + 1, 100003,
         (1 << 20) + 5]


def keys(rng, code, n, dup=False):
    if dup:  # few distinct values: long runs of equal keys
        v = rng.integers(0, 17, n)
        if code in (C.F32, C.F64):  # equal keys with different bits: -0.0 and +0.0
            v = np.where(v == 0, np.where(rng.random(n) < 0.5, -0.0, 0.0), v - 8.0)
        return v.astype(NP[code])
    if code in (C.F32, C.F64):
        return rng.standard_normal(n).astype(NP[code])
    info = np.iinfo(NP[code])
    return rng.integers(info.min, info.max, n, dtype=NP[code], endpoint=True)


def same_bits(got, ref):
    return got.dtype == ref.dtype and np.array_equal(got.view(np.uint8), ref.view(np.uint8))


def test_golden_merge_and_sort(dev):
    g = np.load(GOLDEN)
    names = sorted({k.rsplit("/", 1)[0] for k in g.files})
    for nm in names:
        if nm.startswith("merge/"):
            out = C.merge(dev_t(g[nm + "/a"]), dev_t(g[nm + "/b"]))
            assert np.array_equal(out.cpu().numpy(), g[nm + "/out"]), nm
        else:
            t = dev_t(g[nm + "/in"])
            C.sort_(t)
            assert np.array_equal(t.cpu().numpy(), g[nm + "/out"]), nm
    torch.cuda.synchronize()


def dev_t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("code", DT)
@pytest.mark.parametrize("desc", [False, True])
def test_sort_parity(dev, code, desc):
    rng = np.random.default_rng(100 + code + 10 * desc)
    for n in SIZES:
        for dup in (False, True):
            x = keys(rng, code, n, dup)
            t = dev_t(x)
            C.sort_(t, descending=desc)
            assert same_bits(t.cpu().numpy(), O.sort(x, desc)), (n, dup)


@pytest.mark.parametrize("code", DT)
@pytest.mark.parametrize("desc", [False, True])
def test_merge_parity(dev, code, desc):
    rng = np.random.default_rng(200 + code + 10 * desc)
    for na, nb in [(0, 0), (0, 5), (5, 0), (1, 1), (2047, 1), (2048, 2048), (3000, 100003), (100003, 3000),
                   ((1 << 20) + 1, (1 << 19) + 7)]:
        for dup in (False, True):
            a = O.sort(keys(rng, code, na, dup), desc)
            b = O.sort(keys(rng, code, nb, dup), desc)
            out = C.merge(dev_t(a), dev_t(b), descending=desc)
            assert same_bits(out.cpu().numpy(), O.merge(a, b, desc)), (na, nb, dup)


def test_merge_disjoint_and_interleaved(dev):
    """All of a before all of b, the reverse, and a perfect interleave: the
    merge path runs along the matrix edges and the diagonal."""
    n = 1 << 20
    lo, hi = np.arange(n, dtype=np.int64), np.arange(n, 2 * n, dtype=np.int64)
    ev, od = np.arange(0, 2 * n, 2, dtype=np.int64), np.arange(1, 2 * n, 2, dtype=np.int64)
    for a, b in [(lo, hi), (hi, lo), (ev, od), (od, ev)]:
        out = C.merge(dev_t(a), dev_t(b)).cpu().numpy()
        assert np.array_equal(out, O.merge(a, b))


def test_sort_full_size_properties(dev):
    """2^28 uint32 keys (1 GiB): sorted, and the same multiset (the sum of the
    keys is unchanged and the counts of the top byte match)."""
    n = 1 << 28
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randint(0, 1 << 31, (n,), generator=g, device="cuda", dtype=torch.int64).to(torch.int32)
    x = x.view(torch.uint32)
    xi = x.view(torch.int32).to(torch.int64)
    s0 = int(xi.sum())
    h0 = torch.bincount((x.view(torch.int32).to(torch.int64) >> 24) & 0xFF, minlength=256)
    C.sort_(x)
    xi = x.view(torch.int32).to(torch.int64)
    u = xi & 0xFFFFFFFF
    assert bool((u[1:] >= u[:-1]).all())
    assert int(xi.sum()) == s0
    assert torch.equal(torch.bincount((xi >> 24) & 0xFF, minlength=256), h0)
    del xi, u


def test_sort_descending_int64_full_size_properties(dev):
    n = 1 << 26
    g = torch.Generator(device="cuda").manual_seed(6)
    x = torch.randint(-(1 << 62), 1 << 62, (n,), generator=g, device="cuda", dtype=torch.int64)
    s0 = int(x.sum())
    C.sort_(x, descending=True)
    assert bool((x[1:] <= x[:-1]).all())
    assert int(x.sum()) == s0


def test_bf16_and_bad_args_are_rejected(dev):
    t = torch.zeros(16, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(C.B2PError):
        C.sort_(t)
    L = C.lib()
    a = dev_t(np.arange(8, dtype=np.int32))
    assert L.b2p_sort(C.I32, a.data_ptr(), 1 << 16, 0, None, 0, None) == C.ERR_SCRATCH
    o = torch.empty(16, dtype=torch.int32, device="cuda")
    assert L.b2p_merge(99, a.data_ptr(), 8, a.data_ptr(), 8, o.data_ptr(), 0, None, 0, None) == C.ERR_INVALID_ARG
    assert L.b2p_merge(C.I32, a.data_ptr(), 8, a.data_ptr(), 8, o.data_ptr(), 0, None, 0, None) == C.ERR_SCRATCH
    host = np.zeros(8, dtype=np.int32)
    assert L.b2p_sort(C.I32, host.ctypes.data, 8, 0, None, 0, None) == C.ERR_INVALID_PTR


@pytest.mark.parametrize("code", DT)
def test_sort_extreme_and_uniform_keys(dev, code):
    """Every key the same (one digit value in every radix pass), and the
    extremes of the type (minimum, maximum, infinities, both zeros) mixed
    into random keys, in both directions."""
    rng = np.random.default_rng(300 + code)
    n = 100003
    same = np.full(n, 5, dtype=NP[code])
    t = dev_t(same)
    C.sort_(t)
    assert same_bits(t.cpu().numpy(), same)
    x = keys(rng, code, n)
    if code in (C.F32, C.F64):
        ext = np.array([np.inf, -np.inf, 0.0, -0.0, np.finfo(NP[code]).max, np.finfo(NP[code]).min,
                        np.finfo(NP[code]).tiny, -np.finfo(NP[code]).tiny], dtype=NP[code])
    else:
        info = np.iinfo(NP[code])
        ext = np.array([info.min, info.max, 0, 1, info.max - 1, info.min + 1], dtype=NP[code])
    idx = rng.integers(0, n, 4000)
    x[idx] = ext[rng.integers(0, ext.size, idx.size)]
    for desc in (False, True):
        t = dev_t(x)
        C.sort_(t, descending=desc)
        assert same_bits(t.cpu().numpy(), O.sort(x, desc)), desc


def test_sort_largest_radix_input(dev):
    """2^31 - 5 int32 keys (8 GiB), just below the radix sort's 2^31 limit of
    32-bit output slots: sorted, and the same multiset (sum of the keys and
    counts of the top byte)."""
    n = (1 << 31) - 5
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device="cuda", dtype=torch.int32)
    s0 = int(torch.sum(x, dtype=torch.int64))
    h0 = torch.bincount(((x >> 24) & 0xFF).to(torch.int32), minlength=256)
    C.sort_(x)
    assert bool((x[1:] >= x[:-1]).all())
    assert int(torch.sum(x, dtype=torch.int64)) == s0
    assert torch.equal(torch.bincount(((x >> 24) & 0xFF).to(torch.int32), minlength=256), h0)
    del x
    torch.cuda.empty_cache()
