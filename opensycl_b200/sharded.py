"""Sharded primitives over several GPUs: one process per GPU, torch.distributed.

The reference runs every algorithm on one queue, i.e. one device
(algorithms/numeric.hpp, algorithms/algorithm.hpp take a single sycl::queue);
this module spreads one logical array over P ranks.  Rank r holds the r-th
contiguous shard (rank order is element order).  Local work runs in libb2p's
kernels; the ranks exchange one small set of values per call:

  reduce / dot   local partial, all-gather of the P partials, combined in
                 rank order (the same bits on every rank)
  scan           local total (a reduce), all-gather of the P totals, then one
                 local scan whose init is the carry of the ranks before:
                 12 bytes per 4-byte element instead of the 16 of
                 scan-then-add-carry
  copy_if        local compaction, all-gather of the P counts: each rank's
                 output offset in the global result (the output stays
                 distributed)
  histogram      local bins, all-reduce (sum) of the counters
  segmented      segments split into P contiguous groups of balanced element
                 counts; no exchange

Exchanged values travel as 64-bit patterns (exact for integers and floats)
through the process group's backend: CUDA tensors for NCCL, host tensors
otherwise.  The local primitives come from a `LocalOps` object, the CUDA one
by default (libb2p through opensycl_b200.capi).
"""
from __future__ import annotations

import numpy as np

from . import capi as C

_INT_NP = {C.I32: np.int32, C.I64: np.int64, C.U32: np.uint32, C.U64: np.uint64}


def _op_code(op) -> int:
    return C.OPS[op] if isinstance(op, str) else int(op)


def combine(code: int, op, a, b):
    """a op b for scalars of dtype `code` (integers wrap as in the kernels;
    floats are combined in float64)."""
    opc = _op_code(op)
    if code in _INT_NP:
        t = _INT_NP[code]
        x, y = np.array([a], dtype=t), np.array([b], dtype=t)
        with np.errstate(over="ignore"):
            r = {C.SUM: x + y, C.PROD: x * y, C.MIN: np.minimum(x, y), C.MAX: np.maximum(x, y),
                 C.AND: x & y, C.OR: x | y, C.XOR: x ^ y}[opc]
        return r[0]
    x, y = float(a), float(b)
    return {C.SUM: x + y, C.PROD: x * y, C.MIN: x if x < y else y, C.MAX: y if x < y else x}[opc]


def identity(code: int, op):
    opc = _op_code(op)
    if code in _INT_NP:
        info = np.iinfo(_INT_NP[code])
        return {C.SUM: 0, C.OR: 0, C.XOR: 0, C.PROD: 1, C.AND: -1 if info.min < 0 else info.max,
                C.MIN: info.max, C.MAX: info.min}[opc]
    return {C.SUM: 0.0, C.PROD: 1.0, C.MIN: float("inf"), C.MAX: float("-inf")}[opc]


def _to_bits(code: int, v) -> int:
    if code in _INT_NP:
        return int(np.array([v], dtype=_INT_NP[code]).astype(np.int64)[0])
    return int(np.array([float(v)], dtype=np.float64).view(np.int64)[0])


def _from_bits(code: int, b: int):
    if code in _INT_NP:
        return np.array([b], dtype=np.int64).astype(_INT_NP[code])[0]
    return float(np.array([b], dtype=np.int64).view(np.float64)[0])


class Group:
    """The process group and the device its exchange tensors live on."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.backend = dist.get_backend(group)

    def _device(self):
        import torch
        return torch.device("cuda", torch.cuda.current_device()) if self.backend == "nccl" else torch.device("cpu")

    def all_gather_i64(self, vals) -> np.ndarray:
        """All-gather a fixed-length vector of int64 from every rank: (P, k)."""
        import torch
        t = torch.tensor(np.asarray(vals, dtype=np.int64), device=self._device())
        parts = [torch.empty_like(t) for _ in range(self.size)]
        self.dist.all_gather(parts, t, group=self.group)
        return np.stack([p.cpu().numpy() for p in parts])

    def all_reduce_sum_(self, t):
        """In-place sum over ranks of an integer tensor (moved through the host for
        non-NCCL backends)."""
        if self.backend == "nccl":
            self.dist.all_reduce(t, group=self.group)
            return t
        h = t.cpu()
        self.dist.all_reduce(h, group=self.group)
        t.copy_(h)
        return t


class LocalOps:
    """Local primitives on this rank's GPU (libb2p).  Inputs and outputs are
    torch tensors on the current CUDA device."""

    def code(self, x):
        return C.dtype_code(x)

    def numel(self, x):
        return x.numel()

    def reduce(self, x, op, init):
        init = int(init) if C.dtype_code(x) in _INT_NP else float(init)
        return self.scalar(C.reduce(x, op, init=init))

    def dot(self, a, b, init):
        return self.scalar(C.dot(a, b, init=init))

    def scan(self, x, inclusive, op, init):
        if init is not None:
            init = int(init) if C.dtype_code(x) in _INT_NP else float(init)
        return C.scan(x, inclusive, op, init)

    def copy_if(self, x, mask, cmp, rhs):
        out, cnt = C.copy_if(x, mask, cmp, rhs)
        return out, int(cnt.item())

    def histogram(self, keys, nbins):
        return C.histogram_u8(keys, nbins=nbins)

    def segmented_reduce(self, x, offsets, op, init):
        import torch
        return C.segmented_reduce(x, torch.as_tensor(offsets, dtype=torch.int64, device=x.device), op, init)

    def slice(self, x, a, b):
        return x[a:b]

    def scalar(self, t):
        return t.item()


def sharded_reduce(x, op="sum", init=0, group=None, ops: LocalOps | None = None):
    """init op x_0 op ... over the concatenation of every rank's shard; every
    rank returns the same value."""
    ops = ops or LocalOps()
    g = Group(group)
    code = ops.code(x)
    part = ops.reduce(x, op, identity(code, op)) if ops.numel(x) else identity(code, op)
    allp = g.all_gather_i64([_to_bits(code, part)])[:, 0]
    r = identity(code, op) if init is None else init
    for b in allp:
        r = combine(code, op, r, _from_bits(code, int(b)))
    return r


def sharded_dot(a, b, init=0.0, group=None, ops: LocalOps | None = None):
    """init + sum of a_i * b_i over all shards (float64 combination of the P
    compensated partials, in rank order)."""
    ops = ops or LocalOps()
    g = Group(group)
    part = ops.dot(a, b, 0.0) if ops.numel(a) else 0.0
    allp = g.all_gather_i64([_to_bits(C.F64, part)])[:, 0]
    return float(init) + sum(_from_bits(C.F64, int(v)) for v in allp)


def shard_carry(code: int, op, totals, rank: int, init):
    """init op totals[0] op ... op totals[rank - 1] (init None: identity)."""
    c = identity(code, op) if init is None else init
    for t in totals[:rank]:
        c = combine(code, op, c, t)
    return c


def sharded_scan(x, inclusive=True, op="sum", init=None, group=None, ops: LocalOps | None = None):
    """This rank's part of the scan of the concatenated shards: a reduce, one
    exchange of shard totals, then one scan of the shard with the carry as
    init.  Exclusive scans need init (the identity when None)."""
    ops = ops or LocalOps()
    g = Group(group)
    code = ops.code(x)
    if g.size == 1:  # nothing to exchange: no shard total is needed
        return ops.scan(x, inclusive, op, init if (init is not None or inclusive) else identity(code, op))
    tot = ops.reduce(x, op, identity(code, op)) if ops.numel(x) else identity(code, op)
    totals = [_from_bits(code, int(v)) for v in g.all_gather_i64([_to_bits(code, tot)])[:, 0]]
    if inclusive and init is None:
        if g.rank == 0:
            return ops.scan(x, True, op, None)
        return ops.scan(x, True, op, shard_carry(code, op, totals, g.rank, None))
    base = identity(code, op) if init is None else init
    return ops.scan(x, inclusive, op, shard_carry(code, op, totals, g.rank, base))


def sharded_copy_if(x, mask, cmp, rhs, group=None, ops: LocalOps | None = None):
    """Local compaction plus one exchange of counts.  Returns (local_out,
    local_count, offset, total): this rank's kept elements belong at
    [offset, offset + local_count) of the global result."""
    ops = ops or LocalOps()
    g = Group(group)
    out, cnt = ops.copy_if(x, mask, cmp, rhs)
    counts = g.all_gather_i64([cnt])[:, 0]
    return out, cnt, int(counts[:g.rank].sum()), int(counts.sum())


def sharded_histogram(keys, nbins=256, group=None, ops: LocalOps | None = None):
    """Byte histogram of all shards: local bins, then one all-reduce."""
    ops = ops or LocalOps()
    g = Group(group)
    bins = ops.histogram(keys, nbins)
    return g.all_reduce_sum_(bins)


def partition_segments(offsets, parts: int):
    """Split the segments of CSR `offsets` (nseg + 1 non-decreasing values)
    into `parts` contiguous groups with balanced element counts.  Returns the
    parts + 1 segment boundaries (group p = segments [b[p], b[p+1]))."""
    off = np.asarray(offsets, dtype=np.int64)
    nseg = off.size - 1
    total = int(off[-1] - off[0])
    b = [0]
    for p in range(1, parts):
        target = off[0] + (total * p) // parts
        # the first segment boundary at or after the target, never before the previous cut
        s = int(np.searchsorted(off, target, side="left"))
        b.append(min(max(s, b[-1]), nseg))
    b.append(nseg)
    return b


def sharded_segmented_reduce(x, offsets, op="sum", init=None, group=None, ops: LocalOps | None = None):
    """Segmented reduce of a batch whose input `x` and CSR `offsets` every rank
    holds: rank r reduces its balanced group of segments, no exchange.
    Returns (first_segment, results) for this rank's group."""
    ops = ops or LocalOps()
    g = Group(group)
    off = np.asarray(offsets, dtype=np.int64)
    b = partition_segments(off, g.size)
    s0, s1 = b[g.rank], b[g.rank + 1]
    local = off[s0:s1 + 1] - off[s0]
    xs = ops.slice(x, int(off[s0]), int(off[s1]))
    return s0, ops.segmented_reduce(xs, local, op, init)
