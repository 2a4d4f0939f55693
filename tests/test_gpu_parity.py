"""GPU parity: every primitive of libb2p against the CPU oracle (oracle/),
through the C-ABI, on seeded inputs.

Bars:
  * integer / index / byte results: bit-exact against the oracle;
  * fp32 / bf16 SUM (reduce, dot, scan): |got - ref| <= 1e-6 |ref| + 1e-12 S
    where ref is the FP64 oracle and S the sum of magnitudes (the second
    term only matters when the exact result cancels to ~0);
  * float MIN / MAX: bit-exact against numpy;
  * float PROD: relative 4 n 2^-24 against FP64 (plain arithmetic).
"""
import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INT_DT = [C.I32, C.I64, C.U32, C.U64]
FLOAT_DT = [C.F32, C.BF16, C.F64]
NP = {C.I32: np.int32, C.I64: np.int64, C.U32: np.uint32, C.U64: np.uint64,
      C.F32: np.float32, C.BF16: np.uint16, C.F64: np.float64}
TD = {C.I32: torch.int32, C.I64: torch.int64, C.U32: torch.uint32, C.U64: torch.uint64,
      C.F32: torch.float32, C.BF16: torch.bfloat16, C.F64: torch.float64}
SIZES = [1, 2, 5, 127, 128, 1000, 4099, 65537, (1 << 20) + 3]
REDUCE_CONFIGS = [0, 9, 22, 47, C.AUTO]
SCAN_CONFIGS = [0, 6, 19, 22, 23, 26, 41, C.AUTO]
FLOAT_TOL = 1e-6


def valid(prim, code, cfgs):
    """Configs of `cfgs` the library accepts for this primitive and dtype."""
    L = C.lib()
    return [c for c in cfgs if c == C.AUTO or L.b2p_config_valid(prim, code, c)]


def to_dev(a, code, offset=0):
    """numpy -> device tensor; `offset` elements of padding in front make the
    returned view start off a 16-byte boundary."""
    if offset:
        a = np.concatenate([np.zeros(offset, dtype=a.dtype), a])
    if code == C.BF16:
        t = torch.from_numpy(a.view(np.int16)).cuda().view(torch.bfloat16)
    else:
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t[offset:]


def to_np(t):
    if t.dtype == torch.bfloat16:
        return t.view(torch.int16).cpu().numpy().view(np.uint16)
    return t.cpu().numpy()


def rand_ints(rng, code, n, op):
    if op == C.PROD:  # keep products meaningful: mostly ones, some twos/threes
        v = rng.choice(np.array([1, 1, 1, 1, 2, 3, -1] if code in (C.I32, C.I64) else [1, 1, 1, 2, 3]), n)
        return v.astype(NP[code])
    info = np.iinfo(NP[code])
    return rng.integers(info.min, info.max, n, dtype=NP[code], endpoint=True)


def rand_floats(rng, code, n, positive=False):
    x = rng.standard_normal(n)
    x[rng.random(n) < 0.125] *= 1e-6
    if positive:
        x = np.abs(x)
    if code == C.BF16:
        return O.bf16_round(x.astype(np.float32))
    return x.astype(NP[code])


def as_f64(a, code):
    return O.bf16_to_f32(a).astype(np.float64) if code == C.BF16 else a.astype(np.float64)


def float_ok(got, ref, sabs):
    return abs(float(got) - ref) <= FLOAT_TOL * abs(ref) + 1e-12 * sabs


# ------------------------------------------------------------------ reduce

@pytest.mark.parametrize("code", INT_DT)
@pytest.mark.parametrize("op", [C.SUM, C.PROD, C.MIN, C.MAX, C.AND, C.OR, C.XOR])
def test_reduce_int_bit_exact(dev, code, op):
    rng = np.random.default_rng(100 + 7 * code + op)
    for n in SIZES:
        x = rand_ints(rng, code, n, op)
        init = rand_ints(rng, code, 1, op)[0]
        ref = O.reduce(code, op, x, init)
        for off in (0, 1):
            xd = to_dev(x, code, off)
            for cfg in REDUCE_CONFIGS:
                got = C.reduce(xd, op, init=init, config=cfg)
                assert to_np(got)[0] == ref, (n, off, cfg)


@pytest.mark.parametrize("code", FLOAT_DT)
def test_reduce_float_sum_vs_fp64(dev, code):
    rng = np.random.default_rng(200 + code)
    for n in SIZES:
        x = rand_floats(rng, code, n)
        ref, sabs = O.fp64_sum(code, x, init=0.5)
        for off in (0, 3):
            xd = to_dev(x, code, off)
            for cfg in REDUCE_CONFIGS:
                got = to_np(C.reduce(xd, "sum", init=0.5, config=cfg))[0]
                assert float_ok(got, ref, sabs), (n, off, cfg, got, ref)


@pytest.mark.parametrize("code", FLOAT_DT)
@pytest.mark.parametrize("op", [C.MIN, C.MAX, C.PROD])
def test_reduce_float_other_ops(dev, code, op):
    rng = np.random.default_rng(300 + code * 3 + op)
    for n in SIZES:
        if op == C.PROD:
            x64 = 1.0 + (rng.random(n) - 0.5) * 1e-3
            x = O.bf16_round(x64.astype(np.float32)) if code == C.BF16 else x64.astype(NP[code])
        else:
            x = rand_floats(rng, code, n)
        xd = to_dev(x, code)
        xf = as_f64(x, code)
        for cfg in (0, 22, C.AUTO):
            got = to_np(C.reduce(xd, op, init=1.0 if op == C.PROD else (np.inf if op == C.MIN else -np.inf),
                                 config=cfg))[0]
            if op == C.MIN:
                assert got == xf.min()
            elif op == C.MAX:
                assert got == xf.max()
            else:
                ref = np.prod(xf)
                eps = 2.0 ** -24 if code != C.F64 else 2.0 ** -53
                assert abs(got - ref) <= 4 * n * eps * abs(ref)


def test_reduce_float_config_independent(dev):
    """fp32 SUM is bit-identical for all 48 launch configurations."""
    rng = np.random.default_rng(7)
    for n in (1000, 65537, (1 << 22) + 5):
        x = rand_floats(rng, C.F32, n)
        xd = to_dev(x, C.F32, 1)
        vals = {to_np(C.reduce(xd, "sum", init=0.0, config=c))[0].tobytes() for c in range(48)}
        assert len(vals) == 1, n
        bd = to_dev(rand_floats(rng, C.F32, n), C.F32)
        dots = {to_np(C.dot(xd, bd, config=c))[0].tobytes() for c in range(48)}
        assert len(dots) == 1, n


def test_reduce_no_init_combines_with_out(dev):
    x = to_dev(np.arange(1000, dtype=np.int32), C.I32)
    out = torch.tensor([7], dtype=torch.int32, device="cuda")
    C.reduce(x, "sum", init=None, out=out)
    C.reduce(x, "sum", init=None, out=out)
    assert out.item() == 7 + 2 * 499500  # incremental sycl::reduction (reduction.cpp:326-350)


def test_reduce_empty_leaves_out_untouched(dev):
    x = torch.zeros(0, dtype=torch.float32, device="cuda")
    out = torch.tensor([42.0], device="cuda")
    C.reduce(x, "sum", init=1.0, out=out)
    assert out.item() == 42.0


# ------------------------------------------------------------------ dot

@pytest.mark.parametrize("code", FLOAT_DT)
def test_dot_vs_fp64(dev, code):
    rng = np.random.default_rng(400 + code)
    for n in SIZES:
        a = rand_floats(rng, code, n)
        b = rand_floats(rng, code, n)
        ref, sabs = O.fp64_sum(code, a, b, init=0.25)
        for oa, ob in ((0, 0), (1, 1), (0, 1)):  # (0, 1): differently aligned -> scalar path
            ad, bd = to_dev(a, code, oa), to_dev(b, code, ob)
            for cfg in (0, 22, C.AUTO):
                got = to_np(C.dot(ad, bd, init=0.25, config=cfg))[0]
                assert float_ok(got, ref, sabs), (n, oa, ob, cfg, got, ref)


# ------------------------------------------------------------------ scan

@pytest.mark.parametrize("code", INT_DT)
@pytest.mark.parametrize("op", [C.SUM, C.PROD, C.MIN, C.MAX, C.AND, C.OR, C.XOR])
def test_scan_int_bit_exact(dev, code, op):
    rng = np.random.default_rng(500 + 7 * code + op)
    sizes = [1, 31, 512, 513, 4096, 8191, 8192, 8193, 100003]
    for n in sizes:
        x = rand_ints(rng, code, n, op)
        init = rand_ints(rng, code, 1, op)[0]
        r_inc = O.scan(code, op, True, x)
        r_inc_i = O.scan(code, op, True, x, init)
        r_exc = O.scan(code, op, False, x, init)
        for off in (0, 1):
            xd = to_dev(x, code, off)
            for cfg in valid(C.PRIM_SCAN, code, SCAN_CONFIGS):
                assert np.array_equal(to_np(C.scan(xd, True, op, None, config=cfg)), r_inc), (n, off, cfg)
                assert np.array_equal(to_np(C.scan(xd, True, op, init, config=cfg)), r_inc_i), (n, off, cfg)
                assert np.array_equal(to_np(C.scan(xd, False, op, init, config=cfg)), r_exc), (n, off, cfg)


@pytest.mark.parametrize("code", FLOAT_DT)
def test_scan_float_sum_vs_fp64(dev, code):
    rng = np.random.default_rng(600 + code)
    for n in [1, 31, 4097, 100003, (1 << 20) + 7]:
        x = rand_floats(rng, code, n, positive=True)
        ref_i = O.fp64_scan(code, True, x, 0.0)
        ref_e = O.fp64_scan(code, False, x, 1.5)
        xd = to_dev(x, code)
        for cfg in valid(C.PRIM_SCAN, code, SCAN_CONFIGS):
            gi = to_np(C.scan(xd, True, "sum", None, config=cfg)).astype(np.float64)
            ge = to_np(C.scan(xd, False, "sum", 1.5, config=cfg)).astype(np.float64)
            pos = ref_i > 0
            assert np.max(np.abs(gi - ref_i)[pos] / ref_i[pos]) <= FLOAT_TOL, (n, cfg)
            assert np.max(np.abs(ge - ref_e) / ref_e) <= FLOAT_TOL, (n, cfg)


# Pipelined (TMA) scan configurations: 128 x 32, 256 x 16, 256 x 32 (512 x 16,
# configuration 26, has no pipelined kernel and runs the two-phase kernel).
TMA_SCAN_CONFIGS = [19, 22, 23]


@pytest.mark.parametrize("code", [C.I32, C.I64, C.U32])
def test_scan_pipelined_row_tails(dev, code):
    """Sizes around tile and 128-byte-row boundaries: the last tile may be
    partly or wholly past the complete rows that the bulk tensor copies
    cover, and the elements after them go through plain loads and stores."""
    rng = np.random.default_rng(550 + code)
    es = np.dtype(NP[code]).itemsize
    epr = 128 // es
    for cfg in TMA_SCAN_CONFIGS:
        blk, items = C.config_describe(cfg)[:2]
        tile = blk * items
        for n in [tile, tile + 1, 3 * tile - 1, 3 * tile + epr - 1, 5 * tile + 256 * epr,
                  5 * tile + 256 * epr + 3, 7 * tile + tile // 2 + 5]:
            x = rand_ints(rng, code, n, C.SUM)
            init = rand_ints(rng, code, 1, C.SUM)[0]
            xd = to_dev(x, code)
            assert np.array_equal(to_np(C.scan(xd, True, C.SUM, None, config=cfg)),
                                  O.scan(code, C.SUM, True, x)), (cfg, n)
            assert np.array_equal(to_np(C.scan(xd, False, C.SUM, init, config=cfg)),
                                  O.scan(code, C.SUM, False, x, init)), (cfg, n)


def test_scan_pipelined_bf16_in_fp32_out(dev):
    """bf16 input, fp32 output through the pipelined kernel (the output tile
    sits beside the input tile in each stage): SUM against FP64, MAX exact,
    around 64-element input rows and 32-element output rows."""
    rng = np.random.default_rng(570)
    for cfg in TMA_SCAN_CONFIGS:
        blk, items = C.config_describe(cfg)[:2]
        tile = blk * items
        for n in [tile, 2 * tile + 63, 3 * tile + 32 * 5 + 7, 5 * tile + tile // 2 + 1]:
            x = rand_floats(rng, C.BF16, n, positive=True)
            xd = to_dev(x, C.BF16)
            ref_i = O.fp64_scan(C.BF16, True, x, 0.0)
            ref_e = O.fp64_scan(C.BF16, False, x, 1.5)
            gi = to_np(C.scan(xd, True, "sum", None, config=cfg)).astype(np.float64)
            ge = to_np(C.scan(xd, False, "sum", 1.5, config=cfg)).astype(np.float64)
            pos = ref_i > 0
            assert np.max(np.abs(gi - ref_i)[pos] / ref_i[pos]) <= FLOAT_TOL, (cfg, n)
            assert np.max(np.abs(ge - ref_e) / ref_e) <= FLOAT_TOL, (cfg, n)
            xs = O.bf16_to_f32(rand_floats(rng, C.BF16, n))
            xsd = to_dev(O.bf16_round(xs), C.BF16)
            gm = to_np(C.scan(xsd, True, C.MAX, None, config=cfg))
            assert np.array_equal(gm, np.maximum.accumulate(xs).astype(np.float32)), (cfg, n)


def test_scan_pipelined_fp32_long_exclusive(dev):
    """fp32 SUM longer than 2^24 (FP64 tile carries) through the pipelined
    kernel, inclusive and exclusive with init."""
    rng = np.random.default_rng(560)
    n = (1 << 24) + 12345
    x = rand_floats(rng, C.F32, n, positive=True)
    ref_i = O.fp64_scan(C.F32, True, x, 0.0)
    ref_e = O.fp64_scan(C.F32, False, x, 1.5)
    xd = to_dev(x, C.F32)
    for cfg in (22, 23):
        gi = to_np(C.scan(xd, True, "sum", None, config=cfg)).astype(np.float64)
        ge = to_np(C.scan(xd, False, "sum", 1.5, config=cfg)).astype(np.float64)
        assert np.max(np.abs(gi - ref_i) / ref_i) <= FLOAT_TOL, cfg
        assert np.max(np.abs(ge - ref_e) / ref_e) <= FLOAT_TOL, cfg


@pytest.mark.parametrize("code", [C.F32, C.F64])
@pytest.mark.parametrize("op", [C.MIN, C.MAX])
def test_scan_float_minmax_exact(dev, code, op):
    rng = np.random.default_rng(700 + code + op)
    x = rand_floats(rng, code, 100003)
    ref = (np.minimum if op == C.MIN else np.maximum).accumulate(x)
    got = to_np(C.scan(to_dev(x, code), True, op, None, config=C.AUTO))
    assert np.array_equal(got, ref.astype(got.dtype))


def test_scan_in_place(dev):
    rng = np.random.default_rng(8)
    x = rng.integers(-1000, 1000, 50001).astype(np.int32)
    xd = to_dev(x, C.I32)
    C.scan(xd, True, "sum", None, out=xd)
    assert np.array_equal(to_np(xd), O.scan(C.I32, C.SUM, True, x))
    xd = to_dev(x, C.I32)
    C.scan(xd, False, "sum", 3, out=xd)
    assert np.array_equal(to_np(xd), O.scan(C.I32, C.SUM, False, x, 3))


def test_scan_repeated_calls_share_scratch(dev):
    """Epoch-tagged tile status: back-to-back calls on one scratch buffer
    never read a previous call's status words."""
    rng = np.random.default_rng(9)
    for n in (70001, 9000, 300000, 9000):
        x = rng.integers(-5, 5, n).astype(np.int64)
        xd = to_dev(x, C.I64)
        for _ in range(3):
            assert np.array_equal(to_np(C.scan(xd, True, "sum", None, config=0)),
                                  O.scan(C.I64, C.SUM, True, x))


# ------------------------------------------------------------------ copy_if

@pytest.mark.parametrize("code", [C.U32, C.I32, C.F32, C.I64, C.U64])
def test_copy_if_bit_exact(dev, code):
    rng = np.random.default_rng(800 + code)
    for n in [1, 2, 100, 4095, 4096, 4097, 100003, (1 << 20) + 1]:
        bits = rng.integers(0, 1 << 32, n, dtype=np.uint64)
        if np.dtype(NP[code]).itemsize == 8:
            u = bits | (rng.integers(0, 1 << 32, n, dtype=np.uint64) << np.uint64(32))
        else:
            u = bits.astype(np.uint32)
        x = u.view(NP[code])
        for mask, cmp, rhs in ((7, C.CMP_LT, 3), (1, C.CMP_EQ, 0), (0, C.CMP_EQ, 0), (0xFF, C.CMP_GT, 255)):
            keep = {C.CMP_LT: (u & mask) < rhs, C.CMP_EQ: (u & mask) == rhs,
                    C.CMP_GT: (u & mask) > rhs}[cmp]
            ref = x[keep]
            for off in (0, 1):
                xd = to_dev(x, code, off)
                for cfg in valid(C.PRIM_COPY_IF, code, (0, 6, 19, 22, 23, 26, C.AUTO)):
                    out, cnt = C.copy_if(xd, mask, cmp, rhs, config=cfg)
                    k = int(cnt.item())
                    assert k == ref.size, (n, mask, cmp, off, cfg)
                    assert np.array_equal(to_np(out[:k]).view(u.dtype), ref.view(u.dtype))


@pytest.mark.parametrize("code", [C.U32, C.U64])
def test_copy_if_pipelined_unaligned_output(dev, code):
    """Pipelined copy_if writes the 16-byte-aligned middle of each tile's
    output with one bulk copy and the ends with plain stores: outputs that
    start at every 16-byte phase, sizes around tile and row boundaries."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(810 + code)
    es = np.dtype(NP[code]).itemsize
    for cfg in TMA_SCAN_CONFIGS:
        blk, items = C.config_describe(cfg)[:2]
        tile = blk * items
        for n in [tile, 3 * tile + 5, 6 * tile + 128 // es * 7 + 1]:
            u = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(NP[code])
            keep = (u & 7) < 3
            ref = u[keep]
            xd = to_dev(u, code)
            for shift in range(16 // es):
                big = torch.empty(n + 4, dtype=TD[code], device="cuda")
                out = big[shift:shift + n]
                _, cnt = C.copy_if(xd, 7, C.CMP_LT, 3, out=out, config=cfg)
                k = int(cnt.item())
                assert k == ref.size, (cfg, n, shift)
                assert np.array_equal(to_np(out[:k]), ref), (cfg, n, shift)


@pytest.mark.parametrize("code", [C.U32, C.U64])
def test_copy_if_pipelined_regular_patterns(dev, code):
    """Regular keep patterns through the pipelined copy_if kernels: all kept
    (the output is the input), none kept, every other element, one element
    per tile; sizes with a partial last tile."""
    rng = np.random.default_rng(870 + code)
    for cfg in TMA_SCAN_CONFIGS:
        blk, items = C.config_describe(cfg)[:2]
        tile = blk * items
        n = 5 * tile + 77
        u = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(NP[code])
        u = (u & ~np.array(7, dtype=NP[code])) | (np.arange(n) % 8).astype(NP[code])  # low 3 bits = index mod 8
        xd = to_dev(u, code)
        for cmp, rhs in [(C.CMP_LT, 8), (C.CMP_GT, 7), (C.CMP_EQ, 0), (C.CMP_LT, 4)]:
            keep = (u & 7) < 8 if (cmp, rhs) == (C.CMP_LT, 8) else \
                (u & 7) > 7 if cmp == C.CMP_GT else (u & 7) == 0 if cmp == C.CMP_EQ else (u & 7) < 4
            ref = u[keep]
            out, cnt = C.copy_if(xd, 7, cmp, rhs, config=cfg)
            k = int(cnt.item())
            assert k == ref.size, (cfg, cmp, rhs)
            assert np.array_equal(to_np(out[:k]), ref), (cfg, cmp, rhs)
        # one kept element per tile
        v = np.zeros(n, dtype=NP[code])
        v[::tile] = 1
        out, cnt = C.copy_if(to_dev(v, code), 1, C.CMP_EQ, 1, config=cfg)
        assert int(cnt.item()) == v[::tile].size and np.all(to_np(out[:int(cnt.item())]) == 1)


def test_copy_if_oracle_u32(dev):
    rng = np.random.default_rng(11)
    x = rng.integers(0, 1 << 32, 1 << 20, dtype=np.uint64).astype(np.uint32)
    ref, cnt = O.copy_if_u32(x, 7, C.CMP_LT, 3)
    out, c = C.copy_if(to_dev(x, C.U32), 7, C.CMP_LT, 3)
    assert int(c.item()) == cnt and np.array_equal(to_np(out[:cnt]), ref)


# ------------------------------------------------------------------ histogram

def test_histogram_bit_exact(dev):
    rng = np.random.default_rng(12)
    for n in [1, 15, 16, 17, 1000, 100003, (1 << 22) + 9]:
        for dist in ("uniform", "zipf", "single"):
            if dist == "uniform":
                k = rng.integers(0, 256, n).astype(np.uint8)
            elif dist == "zipf":
                k = C.synth_fill(4, int(rng.integers(1 << 30)), n, 1.2)
            else:
                k = np.full(n, 7, dtype=np.uint8)
            for nbins in (256, 100):
                base = rng.integers(0, 1000, nbins).astype(np.int32)
                ref = O.histogram_u8(k, nbins, bins=base.astype(np.uint32)).astype(np.int64)
                for off in (0, 5):
                    for cfg in (0, 30, C.AUTO):
                        bins = torch.from_numpy(base.copy()).cuda()
                        kd = torch.from_numpy(np.concatenate([np.zeros(off, np.uint8), k])).cuda()[off:]
                        C.histogram_u8(kd, bins=bins, nbins=nbins, config=cfg)
                        assert np.array_equal(bins.cpu().numpy().astype(np.int64), ref), (n, dist, nbins, off, cfg)


def test_histogram_streamed_chunks(dev):
    """Grid mode 1 streams keys through a ring of shared stages with bulk
    copies: many chunks per block (the ring wraps), a partial last chunk,
    unaligned heads and ragged tails; the scratch-less error word stays clear."""
    rng = np.random.default_rng(13)
    for n in [(40 << 20) + 3, (9 << 20) + 4095]:
        k = C.synth_fill(4, int(rng.integers(1 << 30)), n, 1.2)
        ref = O.histogram_u8(k, 256).astype(np.int64)
        for off in (0, 1, 15):
            for cfg in (23, 30, 31):
                assert C.config_describe(cfg)[2] == 1
                bins = torch.zeros(256, dtype=torch.int32, device="cuda")
                kd = torch.from_numpy(np.concatenate([np.zeros(off, np.uint8), k])).cuda()[off:]
                C.histogram_u8(kd, bins=bins, config=cfg)
                assert np.array_equal(bins.cpu().numpy().astype(np.int64), ref), (n, off, cfg)
    assert C.device_error(scratchless=True) == C.OK


# ------------------------------------------------------------------ errors

def test_errors_are_status_codes(dev):
    L = C.lib()
    import ctypes
    host = np.zeros(1024, dtype=np.float32)
    out = torch.zeros(1, device="cuda")
    sp, sb = C.scratch_for(C.PRIM_REDUCE, C.F32, 1024)
    rc = L.b2p_reduce(C.F32, C.SUM, host.ctypes.data_as(ctypes.c_void_p), 1024, out.data_ptr(),
                      None, sp, sb, 0, None)
    assert rc in (C.ERR_INVALID_PTR, C.OK)  # OK only where pageable memory is device-accessible
    x = torch.zeros(1024, device="cuda")
    assert L.b2p_reduce(C.F32, C.AND, x.data_ptr(), 1024, out.data_ptr(), None, sp, sb, 0, None) == C.ERR_INVALID_ARG
    assert L.b2p_reduce(C.F32, C.SUM, x.data_ptr(), 1024, out.data_ptr(), None, sp, sb, 48, None) == C.ERR_INVALID_ARG
    assert L.b2p_reduce(C.F32, C.SUM, x.data_ptr(), 1024, out.data_ptr(), None, sp, 8, 0, None) == C.ERR_SCRATCH
    assert L.b2p_scan(C.F32, C.SUM, 0, x.data_ptr(), x.data_ptr(), 1024, None, sp, sb, 0, None) == C.ERR_INVALID_ARG
    # misaligned element pointer
    assert L.b2p_reduce(C.F32, C.SUM, x.data_ptr() + 2, 10, out.data_ptr(), None, sp, sb, 0, None) == C.ERR_INVALID_PTR
    torch.cuda.synchronize()
    assert C.device_error() == C.OK


def test_kernels_are_sm100a(dev):
    """The kernels the CUDA runtime loads from libb2p are sm_100a machine code
    (cudaFuncGetAttributes binaryVersion 100), with no PTX to JIT."""
    import ctypes
    b, p = ctypes.c_int(0), ctypes.c_int(-1)
    C.check(C.lib().b2p_kernel_arch(ctypes.byref(b), ctypes.byref(p)), "b2p_kernel_arch")
    assert b.value == 100, b.value
