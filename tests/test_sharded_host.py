"""Sharded primitives (opensycl_b200.sharded) on two gloo ranks on the CPU.

The local primitives are the oracle's (numpy arrays), so these tests check
the exchange logic -- partial combination, carries, output offsets, bin
reduction, segment partition -- against the oracle on the whole array, with
ragged and empty shards."""
import os
import socket

import numpy as np
import pytest

from opensycl_b200 import capi as C
from opensycl_b200 import sharded as S
from oracle import oracle as O


class OracleOps:
    """LocalOps over numpy arrays, computed by the oracle."""

    def __init__(self, code):
        self._code = code

    def code(self, x):
        return self._code

    def numel(self, x):
        return x.size

    def reduce(self, x, op, init):
        return O.reduce(self._code, S._op_code(op), x, init)

    def dot(self, a, b, init):
        return float(O.dot(self._code, a, b, init))

    def scan(self, x, inclusive, op, init):
        return O.scan(self._code, S._op_code(op), inclusive, x, init)

    def copy_if(self, x, mask, cmp, rhs):
        return O.copy_if_u32(x, mask, cmp, rhs)

    def histogram(self, keys, nbins):
        import torch
        return torch.from_numpy(O.histogram_u8(keys, nbins).astype(np.int32))

    def segmented_reduce(self, x, offsets, op, init):
        return O.segmented_reduce(self._code, S._op_code(op), x, offsets)

    def slice(self, x, a, b):
        return x[a:b]


def _shard(x, rank, frac):
    cut = int(round(x.size * frac))
    return x[:cut] if rank == 0 else x[cut:]


def _worker(rank, world, port, frac):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(2024)
        n = 100003
        xi = rng.integers(-1000, 1000, n).astype(np.int32)
        xs = _shard(xi, rank, frac)
        lo = 0 if rank == 0 else n - xs.size
        ops = OracleOps(C.I32)
        # reduce: bit-exact, same value on every rank
        assert S.sharded_reduce(xs, "sum", 5, ops=ops) == O.reduce(C.I32, C.SUM, xi, 5)
        assert S.sharded_reduce(xs, "max", None, ops=ops) == xi.max()
        # scans: this rank's slice of the global scan, bit-exact
        assert np.array_equal(S.sharded_scan(xs, True, "sum", None, ops=ops),
                              O.scan(C.I32, C.SUM, True, xi)[lo:lo + xs.size])
        assert np.array_equal(S.sharded_scan(xs, True, "sum", 7, ops=ops),
                              O.scan(C.I32, C.SUM, True, xi, 7)[lo:lo + xs.size])
        assert np.array_equal(S.sharded_scan(xs, False, "sum", -3, ops=ops),
                              O.scan(C.I32, C.SUM, False, xi, -3)[lo:lo + xs.size])
        assert np.array_equal(S.sharded_scan(xs, True, "min", None, ops=ops),
                              O.scan(C.I32, C.MIN, True, xi)[lo:lo + xs.size])
        # fp32 reduce and dot against the FP64 oracle
        xf = rng.random(n, dtype=np.float32)
        yf = rng.random(n, dtype=np.float32)
        fops = OracleOps(C.F32)
        ref, _ = O.fp64_sum(C.F32, xf)
        assert abs(S.sharded_reduce(_shard(xf, rank, frac), "sum", 0.0, ops=fops) - ref) <= 1e-6 * abs(ref)
        refd, _ = O.fp64_sum(C.F32, xf, yf)
        got = S.sharded_dot(_shard(xf, rank, frac), _shard(yf, rank, frac), 0.5, ops=fops)
        assert abs(got - (refd + 0.5)) <= 1e-6 * abs(refd)
        # copy_if: local part and its place in the global result
        xu = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        full, total = O.copy_if_u32(xu, 7, C.CMP_LT, 3)
        part, cnt, off, tot = S.sharded_copy_if(_shard(xu, rank, frac), 7, C.CMP_LT, 3, ops=OracleOps(C.U32))
        assert tot == total and np.array_equal(part, full[off:off + cnt])
        # histogram: every rank ends with the global bins
        keys = rng.integers(0, 256, n).astype(np.uint8)
        bins = S.sharded_histogram(_shard(keys, rank, frac), 256, ops=OracleOps(C.U32))
        assert np.array_equal(bins.numpy().astype(np.int64), O.histogram_u8(keys).astype(np.int64))
        # segmented reduce: balanced groups of segments, no exchange
        offs = np.concatenate([[0], np.cumsum(rng.integers(0, 300, 997))]).astype(np.int64)
        xseg = rng.integers(-50, 50, int(offs[-1])).astype(np.int32)
        s0, res = S.sharded_segmented_reduce(xseg, offs, "sum", None, ops=ops)
        fullr = O.segmented_reduce(C.I32, C.SUM, xseg, offs)
        assert np.array_equal(res, fullr[s0:s0 + res.size])
        sizes = [S.partition_segments(offs, world)[r + 1] - S.partition_segments(offs, world)[r] for r in range(world)]
        assert sum(sizes) == offs.size - 1
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("frac", [0.37, 0.0, 1.0])
def test_sharded_two_gloo_ranks(frac):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), frac), nprocs=2, join=True)


def test_partition_segments_balanced():
    rng = np.random.default_rng(5)
    offs = np.concatenate([[0], np.cumsum(rng.integers(0, 1000, 10000))]).astype(np.int64)
    for parts in (1, 2, 3, 8):
        b = S.partition_segments(offs, parts)
        assert b[0] == 0 and b[-1] == offs.size - 1 and all(b[i] <= b[i + 1] for i in range(parts))
        work = [int(offs[b[i + 1]] - offs[b[i]]) for i in range(parts)]
        assert max(work) - min(work) <= 2 * 1000 + 1  # within two segments of perfect balance
    # empty segments and a single huge one
    offs = np.array([0, 0, 0, 10 ** 6, 10 ** 6, 10 ** 6 + 5], dtype=np.int64)
    b = S.partition_segments(offs, 4)
    assert b[0] == 0 and b[-1] == 5 and sorted(b) == b


def test_carry_and_combine_wrap():
    big = np.iinfo(np.int32).max
    assert S.combine(C.I32, "sum", big, 1) == np.int32(-2 ** 31)
    assert S.shard_carry(C.I32, "sum", [1, 2, 3], 2, 10) == 13
    assert S.shard_carry(C.U32, "max", [5, 9, 2], 3, None) == 9
    assert S._from_bits(C.F32, S._to_bits(C.F32, 0.1)) == 0.1
    assert S._from_bits(C.U64, S._to_bits(C.U64, np.uint64(2 ** 63 + 5))) == np.uint64(2 ** 63 + 5)


# ----------------------------------------------- C-ABI host combination
# b2p_shard_combine is the rank-order combination that b2p_sharded_reduce
# and b2p_sharded_scan apply to the gathered partials (a C/C++ host with its
# own transport calls it directly); it must agree with the Python layer's
# combine / shard_carry, integer wrap-around included.

import ctypes  # noqa: E402

_NP = {C.I32: np.int32, C.I64: np.int64, C.U32: np.uint32, C.U64: np.uint64, C.F32: np.float32, C.F64: np.float64}


def _combine_c(code, op, values, init):
    L = C.lib()
    vals = np.ascontiguousarray(values, dtype=_NP[code])
    res = np.zeros(1, dtype=_NP[code])
    ip = None
    if init is not None:
        ib = np.array([init], dtype=_NP[code])
        ip = ib.ctypes.data_as(ctypes.c_void_p)
    rc = L.b2p_shard_combine(code, op, vals.ctypes.data_as(ctypes.c_void_p) if vals.size else None, vals.size,
                             vals.itemsize, ip, res.ctypes.data_as(ctypes.c_void_p))
    return rc, res[0]


@pytest.mark.parametrize("code", [C.I32, C.I64, C.U32, C.U64, C.F32, C.F64])
@pytest.mark.parametrize("op", [C.SUM, C.PROD, C.MIN, C.MAX, C.AND, C.OR, C.XOR])
def test_shard_combine_matches_python_layer(code, op):
    if code in (C.F32, C.F64) and op > C.MAX:
        assert _combine_c(code, op, [1, 2], 0)[0] == C.ERR_INVALID_ARG
        return
    rng = np.random.default_rng(code * 10 + op)
    if code in (C.F32, C.F64):
        vals = rng.standard_normal(7).astype(_NP[code])
        init = 0.5
    else:
        info = np.iinfo(_NP[code])
        vals = rng.integers(info.min, info.max, 7, dtype=_NP[code], endpoint=True)  # sums and products wrap
        init = 3
    for rank in range(len(vals) + 1):
        rc, got = _combine_c(code, op, vals[:rank], init)
        assert rc == C.OK
        want = S.shard_carry(code, op, list(vals), rank, _NP[code](init))
        if code == C.F32:
            assert got == np.float32(want)
        else:
            assert got == _NP[code](want), (rank, got, want)
    # no init: the first value starts the fold; nothing to fold is an error
    rc, got = _combine_c(code, op, vals[:3], None)
    assert rc == C.OK and got == _NP[code](S.shard_carry(code, op, list(vals[1:]), 2, vals[0]))
    assert _combine_c(code, op, vals[:0], None)[0] == C.ERR_INVALID_ARG
