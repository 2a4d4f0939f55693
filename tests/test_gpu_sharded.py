"""Sharded primitives through libb2p's kernels: two ranks (processes) on one
GPU, exchanging over gloo.  The ranks' kernels never wait on each other (the
only exchange is the host-side collective), so sharing one GPU is safe."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from opensycl_b200 import capi as C
from opensycl_b200 import sharded as S
from oracle import oracle as O


def _shard(x, rank, cut):
    return x[:cut] if rank == 0 else x[cut:]


def _worker(rank, world, port):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        rng = np.random.default_rng(77)
        n = (1 << 22) + 12345
        cut = (1 << 21) + 999
        lo = 0 if rank == 0 else cut
        xi = rng.integers(-1000, 1000, n).astype(np.int32)
        xd = torch.from_numpy(_shard(xi, rank, cut).copy()).cuda()
        assert S.sharded_reduce(xd, "sum", 5) == O.reduce(C.I32, C.SUM, xi, 5)
        for inc, init in ((True, None), (True, 7), (False, -3)):
            got = S.sharded_scan(xd, inc, "sum", init).cpu().numpy()
            assert np.array_equal(got, O.scan(C.I32, C.SUM, inc, xi, init)[lo:lo + got.size]), (inc, init)
        xf = rng.random(n, dtype=np.float32)
        ref = O.fp64_scan(C.F32, True, xf, 0.0)
        gf = S.sharded_scan(torch.from_numpy(_shard(xf, rank, cut).copy()).cuda(), True, "sum").cpu().numpy()
        assert np.max(np.abs(gf - ref[lo:lo + gf.size]) / ref[lo:lo + gf.size]) <= 1e-6
        xu = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        full, total = O.copy_if_u32(xu, 7, C.CMP_LT, 3)
        part, cnt, off, tot = S.sharded_copy_if(torch.from_numpy(_shard(xu, rank, cut).copy()).cuda(), 7, C.CMP_LT, 3)
        assert tot == total and np.array_equal(part[:cnt].cpu().numpy(), full[off:off + cnt])
        keys = C.synth_fill(4, 9, n, 1.2)
        bins = S.sharded_histogram(torch.from_numpy(_shard(keys, rank, cut).copy()).cuda())
        assert np.array_equal(bins.cpu().numpy().astype(np.int64), O.histogram_u8(keys).astype(np.int64))
        offs = np.concatenate([[0], np.cumsum(rng.integers(0, 3000, 2000))]).astype(np.int64)
        xs = rng.integers(-50, 50, int(offs[-1])).astype(np.int32)
        s0, res = S.sharded_segmented_reduce(torch.from_numpy(xs).cuda(), offs, "sum")
        res = res.cpu().numpy()
        assert np.array_equal(res, O.segmented_reduce(C.I32, C.SUM, xs, offs)[s0:s0 + res.size])
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


def test_sharded_two_ranks_one_gpu():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(2, port), nprocs=2, join=True)


def _nccl_single_rank_comm():
    """A one-rank NCCL communicator on the current device, from the
    libnccl.so.2 of this process (the one libb2p resolves NCCL in)."""
    import ctypes

    class UniqueId(ctypes.Structure):
        _fields_ = [("internal", ctypes.c_char * 128)]

    lib = ctypes.CDLL("libnccl.so.2")
    uid = UniqueId()
    assert lib.ncclGetUniqueId(ctypes.byref(uid)) == 0
    comm = ctypes.c_void_p()
    lib.ncclCommInitRank.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, UniqueId, ctypes.c_int]
    assert lib.ncclCommInitRank(ctypes.byref(comm), 1, uid, 0) == 0
    return lib, comm


@pytest.mark.gpu
def test_sharded_c_abi_single_rank(dev):
    """b2p_sharded_reduce / b2p_sharded_scan through an NCCL communicator of
    one rank (this run has one GPU): the exchange path (local partial,
    all-gather, host combination) against b2p_reduce / b2p_scan; the carry
    logic for more ranks is b2p_shard_combine, tested on the host."""
    import ctypes
    import torch
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")
    lib, comm = _nccl_single_rank_comm()
    try:
        L = C.lib()
        sh = C._stream(None)
        rng = np.random.default_rng(3)
        for code, x in ((C.I64, torch.from_numpy(rng.integers(-1000, 1000, (1 << 20) + 7)).cuda()),
                        (C.F32, torch.from_numpy(rng.standard_normal((1 << 20) + 7).astype(np.float32)).cuda())):
            n = x.numel()
            sb = L.b2p_sharded_scratch_bytes(code, n, 1)
            scratch = torch.zeros(sb, dtype=torch.uint8, device="cuda")
            out = torch.zeros(1, dtype=x.dtype, device="cuda")
            init = np.array([5], dtype=np.int64 if code == C.I64 else np.float32)
            ip = init.ctypes.data_as(ctypes.c_void_p)
            assert L.b2p_sharded_reduce(code, C.SUM, x.data_ptr(), n, out.data_ptr(), ip, scratch.data_ptr(), sb,
                                        C.AUTO, comm, sh) == C.OK
            ref = C.reduce(x, "sum", init=init[0].item())
            torch.cuda.synchronize()
            if code == C.I64:
                assert out.item() == ref.item()
            else:
                assert abs(out.item() - ref.item()) <= 1e-6 * abs(ref.item()) + 1e-3
            if code == C.F32:
                x2 = torch.flip(x, [0]).contiguous()
                od = torch.zeros(1, dtype=torch.float32, device="cuda")
                assert L.b2p_sharded_dot(code, x.data_ptr(), x2.data_ptr(), n, od.data_ptr(), None,
                                         scratch.data_ptr(), sb, C.AUTO, comm, sh) == C.OK
                rd = C.dot(x, x2)
                torch.cuda.synchronize()
                assert abs(od.item() - rd.item()) <= 1e-6 * abs(rd.item()) + 1e-3
            y = torch.empty_like(x)
            assert L.b2p_sharded_scan(code, C.SUM, 1, x.data_ptr(), y.data_ptr(), n, None, scratch.data_ptr(), sb,
                                      C.AUTO, comm, sh) == C.OK
            yr = C.scan(x, True, "sum")
            torch.cuda.synchronize()
            assert torch.equal(y, yr)
    finally:
        lib.ncclCommDestroy(comm)
