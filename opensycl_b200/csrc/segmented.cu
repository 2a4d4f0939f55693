// Segmented reduce / scan over CSR offsets in one persistent launch, and
// the batched plans that capture it in a CUDA graph.
//
// The reference has no segmented entry point; its analogue is one
// algorithms::reduce / inclusive_scan call per segment (numeric.hpp:226-279),
// i.e. one or more launches plus host planning per segment.
//
// Work decomposition ("pieces", built on the host from the offsets):
//  * consecutive short segments are packed whole into one piece of at most
//    BLOCK x ITEMS elements (and at most kMaxSegsPerPiece segments);
//  * a segment longer than a piece is split into single-segment pieces;
//    only those pieces need a carry, which comes from a bounded
//    decoupled look-back that stops at the segment's first piece (that
//    piece publishes its inclusive prefix immediately).
// Every piece is one work item fetched dynamically by persistent blocks.
// Inside a piece, elements are scanned with the segmented operator
// (flag, value): (f1, v1) + (f2, v2) = (f1 | f2, f2 ? v2 : v1 + v2).
#include "b2p_device/scan_tile.cuh"
#include "internal.h"
#include "tuning.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace b2p {

constexpr int kMaxSegsPerPiece = 64;

struct __align__(16) Piece {
  long long elem_begin;  // first element
  int elem_count;        // elements in the piece
  int seg_begin;         // first segment
  int seg_count;         // segments (whole ones, or 1 for a long segment)
  int flags;             // kPieceFirst | kPieceLast | kPieceMulti
  long long pad;
};
constexpr int kPieceFirst = 1;  // first piece of its (long) segment
constexpr int kPieceLast = 2;   // last piece of its (long) segment
constexpr int kPieceMulti = 4;  // whole segments packed together

struct SegParams {
  const void *in;
  void *out;
  const long long *offsets;
  long long nseg;
  const Piece *pieces;
  long long npieces;
  int reduce;     // 1: per-segment reduce, 0: scan
  int inclusive;  // scan only
  unsigned long long init_bits;  // Acc-typed init (identity when absent)
  ScratchHeader *hdr;
  StatusWord *status;  // one word per piece
  unsigned long long timeout_ns;
};

template <class P, int ITEMS>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    segmented_kernel(SegParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Pair = SegPair<P>;

  extern __shared__ __align__(16) char smem[];
  __shared__ Pair s_pair[32];
  __shared__ long long s_off[kMaxSegsPerPiece + 1];
  __shared__ unsigned long long s_item, s_carry, s_epoch;

  const int tile_elems = blockDim.x * ITEMS;
  In *xs = reinterpret_cast<In *>(smem);
  const In *in = reinterpret_cast<const In *>(p.in);
  Out *out = reinterpret_cast<Out *>(p.out);

  if (threadIdx.x == 0) s_epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
  __syncthreads();
  const unsigned long long epoch_tag = s_epoch << 8;
  const Acc init = P::unpack(p.init_bits);

  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    const long long item = (long long)s_item;
    if (item >= p.npieces) break;
    const Piece pc = p.pieces[item];
    const int count = min(pc.elem_count, tile_elems);
    const bool multi = (pc.flags & kPieceMulti) != 0;
    const int nsegs = min(pc.seg_count, kMaxSegsPerPiece);
    // elements (coalesced scalar loads: pieces start anywhere) and, for a
    // multi-segment piece, its segment boundaries relative to the piece
    for (int i = threadIdx.x; i < count; i += blockDim.x) xs[i] = in[pc.elem_begin + i];
    if (multi)
      for (int s = threadIdx.x; s <= nsegs; s += blockDim.x)
        s_off[s] = p.offsets[pc.seg_begin + s] - pc.elem_begin;
    __syncthreads();

    // This thread's elements are [e0, e0 + ITEMS).  Segment heads exist
    // only inside multi-segment pieces (a long segment's head is handled by
    // the carry of its first piece).  seg = segment containing e0.
    const int e0 = threadIdx.x * ITEMS;
    int seg = 0;
    if (multi) {
      int lo = 0, hi = nsegs;  // invariant: s_off[lo] <= e0 < s_off[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_off[mid] <= e0) lo = mid;
        else hi = mid;
      }
      seg = lo;
    }
    // thread aggregate without init: f = a head lies in [e0, e0 + ITEMS),
    // v = sum after the last head (or of all elements when f == 0)
    Pair agg = SegOps<P>::identity();
    {
      int s = seg;
      for (int j = 0; j < ITEMS; ++j) {
        const int e = e0 + j;
        if (e >= count) break;
        bool head = false;
        if (multi) {
          if (j == 0) head = s_off[s] == e;
          while (s + 1 <= nsegs && s_off[s + 1] <= e) {
            ++s;
            head = true;
          }
        }
        if (head) {
          agg.f = 1;
          agg.v = P::identity();
        }
        P::add(agg.v, xs[e]);
      }
      if constexpr (P::kCompensated) agg.v = df_norm(agg.v);
    }
    Pair tot;
    const Pair texcl = block_exclusive_scan<SegOps<P>>(agg, s_pair, &tot);

    // carry into the piece: init for a piece that starts its segment(s),
    // init (+) the look-back over the segment's earlier pieces otherwise.
    // Published payloads never include init; the first piece of a long
    // segment publishes its total as an inclusive prefix so that look-backs
    // stop there.
    if (threadIdx.x < 32) {
      Acc carry = init;
      if (!multi && !(pc.flags & kPieceFirst)) {
        if (threadIdx.x == 0) st_status(p.status + item, P::pack(tot.v), epoch_tag | kFlagAgg);
        bool err;
        carry = P::combine(init, lookback<AccOps<P>>(p.status, item, epoch_tag, p.timeout_ns, err));
        if (threadIdx.x == 0 && err) record_error(p.hdr, B2P_ERR_TIMEOUT);
      } else if (!multi && threadIdx.x == 0) {
        st_status(p.status + item, P::pack(tot.v), epoch_tag | kFlagPrefix);
      }
      if (threadIdx.x == 0) s_carry = P::pack(carry);
    }
    __syncthreads();
    const Acc carry = P::unpack(s_carry);

    // emit: value entering this thread, then one element at a time
    {
      Acc run = texcl.f ? P::combine(init, texcl.v) : P::combine(carry, texcl.v);
      int s = seg;
      for (int j = 0; j < ITEMS; ++j) {
        const int e = e0 + j;
        if (e >= count) break;
        bool head = false;
        if (multi) {
          if (j == 0) head = s_off[s] == e;
          while (s + 1 <= nsegs && s_off[s + 1] <= e) {
            ++s;
            head = true;
          }
        }
        if (head) run = init;
        if (p.reduce) {
          P::add(run, xs[e]);
          const bool seg_end = multi ? (s_off[s + 1] == e + 1)
                                     : ((pc.flags & kPieceLast) && e + 1 == count);
          if (seg_end) out[pc.seg_begin + (multi ? s : 0)] = P::finalize(run);
        } else if (p.inclusive) {
          P::add(run, xs[e]);
          out[pc.elem_begin + e] = P::finalize(run);
        } else {
          out[pc.elem_begin + e] = P::finalize(run);
          P::add(run, xs[e]);
        }
      }
    }
    // empty segments of a multi-segment piece get init
    if (p.reduce && multi)
      for (int s = threadIdx.x; s < nsegs; s += blockDim.x)
        if (s_off[s + 1] == s_off[s]) out[pc.seg_begin + s] = P::finalize(init);
    __syncthreads();
  }
  finish_launch(p.hdr, s_epoch, nullptr, 0);
}

// ---------------------------------------------------------------- host

namespace {

bool seg_tile_ok(int dtype, int config) {
  if (config < 0 || config >= B2P_NUM_CONFIGS) return false;
  LaunchConfig lc = describe_config(config);
  const long long tile = (long long)lc.block * lc.items;
  if (tile > 8192) return false;
  return (size_t)tile * dtype_size(dtype) <= 96 * 1024;
}

}  // namespace

// Pieces for one offsets array and piece capacity (host side).
std::vector<Piece> build_pieces(const int64_t *offs, int64_t nseg, int cap) {
  std::vector<Piece> v;
  v.reserve((size_t)nseg + 16);
  int64_t s = 0;
  while (s < nseg) {
    const int64_t len = offs[s + 1] - offs[s];
    if (len > cap) {
      const int64_t np = (len + cap - 1) / cap;
      for (int64_t k = 0; k < np; ++k) {
        Piece pc{};
        pc.elem_begin = offs[s] + k * cap;
        pc.elem_count = (int)std::min<int64_t>(cap, len - k * cap);
        pc.seg_begin = (int)s;
        pc.seg_count = 1;
        pc.flags = (k == 0 ? kPieceFirst : 0) | (k == np - 1 ? kPieceLast : 0);
        v.push_back(pc);
      }
      ++s;
      continue;
    }
    Piece pc{};
    pc.elem_begin = offs[s];
    pc.seg_begin = (int)s;
    pc.flags = kPieceMulti | kPieceFirst | kPieceLast;
    int64_t e = s, total = 0;
    while (e < nseg && e - s < kMaxSegsPerPiece) {
      const int64_t l = offs[e + 1] - offs[e];
      if (l > cap || total + l > cap) break;
      total += l;
      ++e;
    }
    pc.elem_count = (int)total;
    pc.seg_count = (int)(e - s);
    v.push_back(pc);
    s = e;
  }
  return v;
}

size_t pieces_upper_bound(size_t n, int64_t nseg, int cap) {
  return (size_t)nseg + n / (size_t)cap + 2;
}

size_t segmented_scratch_bytes(int dtype, size_t n, int64_t nseg, int config) {
  int cap = 512;  // smallest piece of the table
  size_t flat = segmented_tma_scratch(n, 128, 16);  // smallest tile of the pipelined kernel
  if (config >= 0) {
    LaunchConfig lc = describe_config(config);
    cap = lc.block * lc.items;
    flat = lc.grid_mode == 1 ? segmented_tma_scratch(n, lc.block, lc.items) : 0;
  }
  (void)dtype;
  const size_t np = pieces_upper_bound(n, nseg, cap);
  return std::max(kScratchPrefix + np * (sizeof(StatusWord) + sizeof(Piece)), flat) + 256;
}

bool segmented_config_valid(int dtype, int config) { return seg_tile_ok(dtype, config); }

namespace {

template <class P, int ITEMS>
int launch_seg_items(SegParams &p, const LaunchConfig &lc, cudaStream_t st) {
  using In = typename P::In;
  const size_t smem = (size_t)lc.block * ITEMS * sizeof(In);
  const void *kfn = (const void *)segmented_kernel<P, ITEMS>;
  int rc = ensure_dynamic_smem(kfn, smem);
  if (rc) return rc;
  int grid = grid_for(lc.grid_mode, std::max<long long>(p.npieces, 1), 1, kfn, lc.block, smem);
  segmented_kernel<P, ITEMS><<<grid, lc.block, smem, st>>>(p);
  return cuda_status(cudaGetLastError());
}

template <class P>
int launch_seg_t(SegParams &p, const void *init, int config, cudaStream_t st) {
  using Out = typename P::Out;
  LaunchConfig lc = describe_config(config);
  if (init) {
    Out v;
    memcpy(&v, init, sizeof(Out));
    // device-side conversion of init to the accumulator happens in the kernel
    // through from_out; pack here as Acc bits computed on the host
    p.init_bits = 0;
    if constexpr (P::kCompensated) {
      float hl[2] = {(float)v, 0.f};
      memcpy(&p.init_bits, hl, 8);
    } else {
      memcpy(&p.init_bits, &v, sizeof(Out));
    }
  }
  switch (lc.items) {
  case 4: return launch_seg_items<P, 4>(p, lc, st);
  case 8: return launch_seg_items<P, 8>(p, lc, st);
  case 16: return launch_seg_items<P, 16>(p, lc, st);
  default: return launch_seg_items<P, 32>(p, lc, st);
  }
}

// Identity bits of the accumulator, computed on the host.
template <class T>
unsigned long long host_bits(T v) {
  unsigned long long b = 0;
  memcpy(&b, &v, sizeof(T));
  return b;
}

unsigned long long identity_bits(int dtype, int op) {
  const bool fl = dtype_is_float(dtype);
  switch (op) {
  case B2P_SUM: return 0;
  case B2P_PROD:
    if (dtype == B2P_F64) return host_bits(1.0);
    if (fl) return host_bits(1.0f);  // DF{1, 0} for SUM never happens; plain float
    return dtype_size(dtype) == 8 ? host_bits<int64_t>(1) : host_bits<int32_t>(1);
  case B2P_MIN:
    switch (dtype) {
    case B2P_I32: return host_bits<int32_t>(INT32_MAX);
    case B2P_I64: return host_bits<int64_t>(INT64_MAX);
    case B2P_U32: return host_bits<uint32_t>(UINT32_MAX);
    case B2P_U64: return host_bits<uint64_t>(UINT64_MAX);
    case B2P_F64: return host_bits(INFINITY * 1.0);
    default: return host_bits((float)INFINITY);
    }
  case B2P_MAX:
    switch (dtype) {
    case B2P_I32: return host_bits<int32_t>(INT32_MIN);
    case B2P_I64: return host_bits<int64_t>(INT64_MIN);
    case B2P_U32: case B2P_U64: return 0;
    case B2P_F64: return host_bits(-INFINITY * 1.0);
    default: return host_bits((float)-INFINITY);
    }
  case B2P_AND: return dtype_size(dtype) == 8 ? ~0ull : 0xffffffffull;
  default: return 0;
  }
}

template <int DT>
int seg_dispatch(int op, SegParams &p, const void *init, int config, cudaStream_t st) {
  switch (op) {
  case B2P_SUM: return launch_seg_t<typename PolicyOf<DT, B2P_SUM>::type>(p, init, config, st);
  case B2P_PROD: return launch_seg_t<typename PolicyOf<DT, B2P_PROD>::type>(p, init, config, st);
  case B2P_MIN: return launch_seg_t<typename PolicyOf<DT, B2P_MIN>::type>(p, init, config, st);
  case B2P_MAX: return launch_seg_t<typename PolicyOf<DT, B2P_MAX>::type>(p, init, config, st);
  default: break;
  }
  if constexpr (DT == B2P_F32 || DT == B2P_BF16 || DT == B2P_F64) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    switch (op) {
    case B2P_AND: return launch_seg_t<typename PolicyOf<DT, B2P_AND>::type>(p, init, config, st);
    case B2P_OR: return launch_seg_t<typename PolicyOf<DT, B2P_OR>::type>(p, init, config, st);
    case B2P_XOR: return launch_seg_t<typename PolicyOf<DT, B2P_XOR>::type>(p, init, config, st);
    default: return B2P_ERR_INVALID_ARG;
    }
  }
}

int seg_launch_with_pieces(int prim, int dtype, int op, int inclusive, const void *in, void *out,
                           const int64_t *offsets, int64_t nseg, const void *init,
                           const Piece *dpieces, long long npieces, void *scratch, int config,
                           cudaStream_t st) {
  SegParams p{};
  p.in = in;
  p.out = out;
  p.offsets = reinterpret_cast<const long long *>(offsets);
  p.nseg = nseg;
  p.pieces = dpieces;
  p.npieces = npieces;
  p.reduce = prim == B2P_PRIM_SEG_REDUCE;
  p.inclusive = inclusive;
  p.init_bits = identity_bits(dtype, op);
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix);
  p.timeout_ns = wait_timeout_ns();
  switch (dtype) {
  case B2P_I32: return seg_dispatch<B2P_I32>(op, p, init, config, st);
  case B2P_I64: return seg_dispatch<B2P_I64>(op, p, init, config, st);
  case B2P_U32: return seg_dispatch<B2P_U32>(op, p, init, config, st);
  case B2P_U64: return seg_dispatch<B2P_U64>(op, p, init, config, st);
  case B2P_F32: return seg_dispatch<B2P_F32>(op, p, init, config, st);
  case B2P_BF16: return seg_dispatch<B2P_BF16>(op, p, init, config, st);
  case B2P_F64: return seg_dispatch<B2P_F64>(op, p, init, config, st);
  default: return B2P_ERR_INVALID_ARG;
  }
}

}  // namespace

// Whether a call runs the pipelined flat kernel (seg_tma.cu): grid mode 1
// with a shape it has, SUM, offsets starting at 0, 16-byte aligned input
// (and output for a scan), at least one tile of elements.
bool seg_tma_fits(int prim, int dtype, int op, int config, const void *in, const void *out, const int64_t *h,
                  int64_t nseg, size_t total) {
  const LaunchConfig lc = describe_config(config);
  if (lc.grid_mode != 1 || !segmented_tma_shape(dtype, op, lc.block, lc.items)) return false;
  if (h[0] != 0 || nseg >= (1ll << 31) - 2 || total < (size_t)lc.block * lc.items) return false;
  if (reinterpret_cast<uintptr_t>(in) & 15) return false;
  if (prim == B2P_PRIM_SEG_SCAN && (reinterpret_cast<uintptr_t>(out) & 15)) return false;
  return true;
}

// The per-tile records of the pipelined kernel, copied into scratch after
// its status words (synchronous: the records are a host temporary).
int seg_tma_prepare(const int64_t *h, int64_t nseg, size_t total, int config, void *scratch, size_t scratch_bytes,
                    cudaStream_t st) {
  const LaunchConfig lc = describe_config(config);
  if (scratch_bytes < segmented_tma_scratch(total, lc.block, lc.items)) return B2P_ERR_SCRATCH;
  const size_t tile = (size_t)lc.block * lc.items, ntiles = (total + tile - 1) / tile;
  std::vector<int> tk(ntiles * 64);
  segmented_tile_records(h, nseg, total, lc.block, lc.items, tk.data());
  char *dst = reinterpret_cast<char *>(scratch) + kScratchPrefix + ntiles * sizeof(StatusWord);
  cudaError_t e = cudaMemcpyAsync(dst, tk.data(), tk.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cuda_status(e);
}

int launch_segmented(int prim, int dtype, int op, int inclusive, const void *in, void *out,
                     const int64_t *offsets, int64_t nseg, size_t total, const void *init,
                     void *scratch, size_t scratch_bytes, int config, cudaStream_t st) {
  if (!seg_tile_ok(dtype, config)) return B2P_ERR_INVALID_ARG;
  if (reinterpret_cast<uintptr_t>(scratch) & 255) return B2P_ERR_SCRATCH;
  LaunchConfig lc = describe_config(config);
  const int cap = lc.block * lc.items;
  // the piece map is built on the host from the offsets (one copy back)
  std::vector<int64_t> h((size_t)nseg + 1);
  cudaError_t e = cudaMemcpyAsync(h.data(), offsets, h.size() * sizeof(int64_t), cudaMemcpyDefault, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e);
  for (int64_t s = 0; s < nseg; ++s)
    if (h[(size_t)s + 1] < h[(size_t)s] || h[0] < 0) return B2P_ERR_INVALID_ARG;
  if ((size_t)h[(size_t)nseg] != total) return B2P_ERR_INVALID_ARG;
  if (seg_tma_fits(prim, dtype, op, config, in, out, h.data(), nseg, total)) {
    int rc = seg_tma_prepare(h.data(), nseg, total, config, scratch, scratch_bytes, st);
    if (rc) return rc;
    rc = launch_segmented_tma(prim, dtype, op, inclusive, in, out, offsets, nseg, total, init, scratch, lc.block,
                              lc.items, st);
    if (rc != B2P_ERR_UNSUPPORTED) return rc;
  }
  std::vector<Piece> pieces = build_pieces(h.data(), nseg, cap);
  const size_t np = pieces.size();
  const size_t need = kScratchPrefix + np * (sizeof(StatusWord) + sizeof(Piece));
  if (scratch_bytes < need) return B2P_ERR_SCRATCH;
  Piece *dp = reinterpret_cast<Piece *>(reinterpret_cast<char *>(scratch) + kScratchPrefix +
                                        np * sizeof(StatusWord));
  e = cudaMemcpyAsync(dp, pieces.data(), np * sizeof(Piece), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // `pieces` is a host temporary
  if (e != cudaSuccess) return cuda_status(e);
  return seg_launch_with_pieces(prim, dtype, op, inclusive, in, out, offsets, nseg, init, dp,
                                (long long)np, scratch, config, st);
}

}  // namespace b2p

// ------------------------------------------------------------ plans (C-ABI)

struct b2p_plan_s {
  int prim, dtype, op, config;
  size_t n = 0;       // elements (call records)
  int64_t nseg = 0;
  double bytes = 0;   // algorithmic bytes of one launch
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

using namespace b2p;

extern "C" {

int b2p_plan_segmented(b2p_plan *plan, int prim, int dtype, int op, const void *in, void *out,
                       const int64_t *offsets, int64_t nseg, size_t total_elems, int config,
                       b2p_stream stream) {
  if (!plan) return B2P_ERR_INVALID_ARG;
  *plan = nullptr;
  if (prim != B2P_PRIM_SEG_REDUCE && prim != B2P_PRIM_SEG_SCAN) return B2P_ERR_INVALID_ARG;
  if (nseg <= 0 || dtype_size(dtype) == 0) return B2P_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<int64_t> h((size_t)nseg + 1);
  cudaError_t e = cudaMemcpyAsync(h.data(), offsets, h.size() * sizeof(int64_t), cudaMemcpyDefault, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e);
  if ((size_t)h[(size_t)nseg] != total_elems) return B2P_ERR_INVALID_ARG;
  if (config == B2P_CONFIG_AUTO) {
    // coefficient of variation of the segment lengths, a selector feature
    double m = (double)total_elems / (double)nseg, var = 0.0;
    for (int64_t s = 0; s < nseg; ++s) {
      const double d = (double)(h[(size_t)s + 1] - h[(size_t)s]) - m;
      var += d * d;
    }
    const double cv = m > 0 ? std::sqrt(var / (double)nseg) / m : 0.0;
    config = b2p_auto_config(prim, dtype, total_elems, nseg, cv);
  }
  if (!seg_tile_ok(dtype, config)) return B2P_ERR_INVALID_ARG;
  LaunchConfig lc = describe_config(config);
  const bool flat = seg_tma_fits(prim, dtype, op, config, in, out, h.data(), nseg, total_elems);
  std::vector<Piece> pieces = build_pieces(h.data(), nseg, lc.block * lc.items);
  const size_t np = pieces.size();
  b2p_plan_s *pl = new b2p_plan_s();
  pl->prim = prim;
  pl->dtype = dtype;
  pl->n = total_elems;
  pl->nseg = nseg;
  pl->bytes = (double)total_elems * dtype_size(dtype) * (prim == B2P_PRIM_SEG_SCAN ? 2 : 1) + 8.0 * nseg;
  pl->op = op;
  pl->config = config;
  pl->scratch_bytes = kScratchPrefix + np * (sizeof(StatusWord) + sizeof(Piece));
  if (flat) pl->scratch_bytes = std::max(pl->scratch_bytes, segmented_tma_scratch(total_elems, lc.block, lc.items));
  e = cudaMalloc(&pl->scratch, pl->scratch_bytes);
  if (e != cudaSuccess) {
    b2p_plan_destroy(pl);
    return cuda_status(e);
  }
  Piece *dp = reinterpret_cast<Piece *>(reinterpret_cast<char *>(pl->scratch) + kScratchPrefix +
                                        np * sizeof(StatusWord));
  // The flat kernel first; the piece kernel when the flat one turns out not
  // to have the shape (its scratch contents differ, so each attempt fills the
  // scratch before its capture).
  int rc = B2P_ERR_UNSUPPORTED;
  for (int attempt = flat ? 0 : 1; attempt < 2 && rc == B2P_ERR_UNSUPPORTED; ++attempt) {
    const bool use_flat = attempt == 0;
    e = cudaMemsetAsync(pl->scratch, 0, pl->scratch_bytes, st);
    if (e == cudaSuccess && !use_flat)
      e = cudaMemcpyAsync(dp, pieces.data(), np * sizeof(Piece), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      rc = cuda_status(e);
      break;
    }
    if (use_flat) {
      rc = seg_tma_prepare(h.data(), nseg, total_elems, config, pl->scratch, pl->scratch_bytes, st);
      if (rc) break;
    }
    // capture the single launch into a graph
    cudaStream_t cs;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      rc = cuda_status(e);
      break;
    }
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      if (use_flat)
        rc = launch_segmented_tma(prim, dtype, op, 1, in, out, offsets, nseg, total_elems, nullptr, pl->scratch,
                                  lc.block, lc.items, cs);
      else
        rc = seg_launch_with_pieces(prim, dtype, op, 1, in, out, offsets, nseg, nullptr, dp, (long long)np,
                                    pl->scratch, config, cs);
      cudaGraph_t g = nullptr;
      cudaError_t e2 = cudaStreamEndCapture(cs, &g);
      if (rc == B2P_OK && e2 == cudaSuccess) {
        pl->graph = g;
        e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
      } else {
        if (g) cudaGraphDestroy(g);
        if (rc == B2P_OK) e = e2;
      }
    } else {
      rc = B2P_OK;
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) rc = cuda_status(e);
  }
  if (rc != B2P_OK) {
    b2p_plan_destroy(pl);
    return rc;
  }
  *plan = pl;
  return B2P_OK;
}

int b2p_segmented_per_call(int prim, int dtype, int op, const void *in, void *out,
                           const int64_t *offs, int64_t nseg, void *scratch, size_t scratch_bytes,
                           int config, b2p_stream stream) {
  if (!offs || nseg < 0) return B2P_ERR_INVALID_ARG;
  if (prim != B2P_PRIM_SEG_REDUCE && prim != B2P_PRIM_SEG_SCAN) return B2P_ERR_INVALID_ARG;
  const size_t es = dtype_size(dtype), os = acc_size(dtype);
  if (!es) return B2P_ERR_INVALID_ARG;
  const unsigned long long ident = identity_bits(dtype, op);
  for (int64_t s = 0; s < nseg; ++s) {
    const int64_t b = offs[s], len = offs[s + 1] - offs[s];
    int rc = B2P_OK;
    if (prim == B2P_PRIM_SEG_REDUCE) {
      char *o = reinterpret_cast<char *>(out) + (size_t)s * os;
      if (len == 0) {
        // identity of the accumulator, as the output type (fp32 SUM: 0)
        rc = cuda_status(cudaMemcpyAsync(o, &ident, os, cudaMemcpyHostToDevice, (cudaStream_t)stream));
      } else {
        rc = b2p_reduce(dtype, op, reinterpret_cast<const char *>(in) + (size_t)b * es, (size_t)len, o,
                        nullptr, scratch, scratch_bytes, config, stream);
      }
    } else if (len > 0) {
      rc = b2p_scan(dtype, op, 1, reinterpret_cast<const char *>(in) + (size_t)b * es,
                    reinterpret_cast<char *>(out) + (size_t)b * os, (size_t)len, nullptr, scratch,
                    scratch_bytes, config, stream);
    }
    if (rc) return rc;
  }
  return B2P_OK;
}

int b2p_plan_launch(b2p_plan plan, b2p_stream stream) {
  CallScope cs("b2p_plan_launch", plan ? plan->dtype : -1, plan ? plan->n : 0, plan ? plan->nseg : 0,
               plan ? plan->bytes : 0.0, stream);
  if (!plan || !plan->exec) return cs.done(B2P_ERR_INVALID_ARG);
  note_config(plan->config);
  return cs.done(cuda_status(cudaGraphLaunch(plan->exec, (cudaStream_t)stream)));
}

int b2p_plan_config(b2p_plan plan) { return plan ? plan->config : -1; }

void b2p_plan_destroy(b2p_plan plan) {
  if (!plan) return;
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->graph) cudaGraphDestroy(plan->graph);
  if (plan->scratch) cudaFree(plan->scratch);
  delete plan;
}

}  // extern "C"
