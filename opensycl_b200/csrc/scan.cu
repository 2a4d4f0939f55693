// Scan and order-preserving copy_if.
//
// Replaces algorithms/scan/decoupled_lookback_scan.hpp:555-655 (init kernel
// + main kernel of 128 work-items x 16 items, Kogge-Stone in local memory,
// serial one-predecessor look-back on separate status/value words, unbounded
// spin at :244-246) and the copy_if built on it (algorithms/algorithm.hpp:
// 178-243, a 64-bit exclusive flag scan that reads the input twice).
//
// Two kernel families, chosen by the launch configuration's grid mode:
//
// * grid mode 0 -- decoupled look-back (the reference's algorithm, made
//   bounded): per tile of BLOCK x ITEMS elements, a dynamic tile id,
//   16-byte loads into a swizzled shared tile, a blocked per-thread scan, a
//   block scan, then warp 0 publishes the tile aggregate and runs a
//   warp-parallel look-back over 128 predecessors per step on epoch-tagged
//   128-bit status words.  One launch, 2 x n element traffic; its speed is
//   bounded by how fast prefixes propagate between tiles.
//
// * grid modes 1, 2 -- L2-blocked two-phase scan (persistent blocks): the
//   input is cut into chunks of ~16 MB that stay resident in the 126 MB L2.
//   Phase 1 of chunk k reduces each tile (DRAM read, L2 evict_last) and
//   publishes its total; the last block to finish chunk k scans the chunk's
//   tile totals into per-tile prefixes and marks the chunk ready.  Phase 2
//   re-reads each tile from L2 (evict_first), scans it from its prefix and
//   streams the output to DRAM.  One work queue orders phase 1 of chunk
//   k + 2 before phase 2 of chunk k, so blocks never wait on a chain of
//   predecessors and DRAM still moves only the algorithmic 2 x n elements.
//
// fp32/bf16 SUM accumulates with compensated (TwoSum) arithmetic; scans
// longer than 2^24 carry cross-tile prefixes in FP64.  All waits are bounded
// and report B2P_ERR_TIMEOUT through the scratch error word.
#include "b2p_device/scan_tile.cuh"
#include "internal.h"

#include <algorithm>
#include <cstdlib>

namespace b2p {

struct ScanParams {
  const void *in;
  void *out;
  unsigned long long n;
  long long ntiles;
  int inclusive;
  int has_init;
  unsigned long long init_bits;  // Out-typed init value
  int vec_in;                    // input 16-byte aligned
  int vec_out;                   // output 16-byte aligned
  ScratchHeader *hdr;
  StatusWord *status;            // one word per tile
  StatusWord *chunk_status;      // two-phase: chunk totals / inclusive prefixes (look-back)
  StatusWord *chunk_carry;       // two-phase: exclusive carry of each chunk
  unsigned *counters;            // two-phase: phase-1 arrivals per chunk
  long long chunk_tiles, nchunks;
  int lookahead;
  unsigned long long timeout_ns;
  long long stall_tile;
  // copy_if
  unsigned long long mask, rhs;
  int cmp;
  unsigned long long *num_copied;
};

template <class P, bool WIDE>
__device__ __forceinline__ unsigned long long init_value(const ScanParams &p) {
  using Out = typename P::Out;
  if (!p.has_init) {
    if constexpr (WIDE) return F64Ops::pack(0.0);
    else return P::pack(P::identity());
  }
  const Out v = from_bits64<Out>(p.init_bits);
  if constexpr (WIDE) return F64Ops::pack((double)v);
  else return P::pack(P::from_out(v));
}

// Work queue of the two-phase kernels.  Segments, in order:
//   P1(0) .. P1(D-1), then P1(k), P2(k-D) for k = D .. K-1, then
//   P2(K-D) .. P2(K-1)
// where P1(k) / P2(k) hold the tiles of chunk k (CT each, the last chunk
// may be shorter) and D = min(lookahead, K).
struct WorkItem {
  int phase;
  long long chunk, tile;
};

__device__ __forceinline__ WorkItem decode_work(long long w, long long ntiles, long long CT,
                                                long long K, int lookahead) {
  const long long D = lookahead < K ? lookahead : K;
  const long long slast = ntiles - (K - 1) * CT;
  const long long p1 = (K - 1 < D) ? K - 1 : D + 2 * (K - 1 - D);  // segment of P1(K-1)
  const long long p2 = 2 * K - 1;                                    // segment of P2(K-1)
  auto start = [&](long long s) {
    return s * CT - (long long)((p1 < s) + (p2 < s)) * (CT - slast);
  };
  auto size = [&](long long s) { return (s == p1 || s == p2) ? slast : CT; };
  long long s = w / CT;
  if (s > 2 * K - 1) s = 2 * K - 1;
  for (int guard = 0; guard < 8; ++guard) {
    const long long st = start(s);
    if (w < st) --s;
    else if (w >= st + size(s)) ++s;
    else break;
  }
  const long long j = w - start(s);
  WorkItem it;
  if (s < D) {
    it.phase = 1;
    it.chunk = s;
  } else if (s - D < 2 * (K - D)) {
    const long long u = s - D;
    if ((u & 1) == 0) {
      it.phase = 1;
      it.chunk = D + u / 2;
    } else {
      it.phase = 2;
      it.chunk = u / 2;
    }
  } else {
    it.phase = 2;
    it.chunk = K - D + (s - D - 2 * (K - D));
  }
  it.tile = it.chunk * CT + j;
  return it;
}

// Last block of a chunk's phase 1.  (1) Turn the chunk's tile totals into
// chunk-relative exclusive prefixes (no waiting).  (2) Publish the chunk
// total and obtain the chunk's exclusive carry with a warp-parallel
// look-back over the chunk totals (so chunks do not wait for each other's
// finalisation in sequence), then publish the carry.  Phase 2 combines the
// carry with a tile's relative prefix.
template <class Ops>
__device__ void finalize_chunk(const ScanParams &p, long long k, unsigned long long epoch_tag,
                               unsigned long long init_bits, typename Ops::Pub *s_pub,
                               unsigned long long *s_bits, int *s_err) {
  using Pub = typename Ops::Pub;
  const long long c0 = k * p.chunk_tiles;
  const long long S = min(p.chunk_tiles, p.ntiles - c0);
  Pub rel = Ops::identity();
  for (long long b = 0; b < S; b += blockDim.x) {
    const long long i = b + threadIdx.x;
    Pub v = i < S ? Ops::unpack(ld_status(p.status + c0 + i).payload) : Ops::identity();
    Pub tot;
    Pub ex = block_exclusive_scan<Ops>(v, s_pub, &tot);
    if (i < S) st_status(p.status + c0 + i, Ops::pack(Ops::combine(rel, ex)), epoch_tag | kFlagPrefix);
    rel = Ops::combine(rel, tot);
    __syncthreads();
  }
  __threadfence();  // every writer: relative prefixes visible before the carry below
  if (threadIdx.x < 32) {
    Pub carry = Ops::unpack(init_bits);
    bool err = false;
    if (k == 0) {
      if (threadIdx.x == 0)
        st_status(p.chunk_status, Ops::pack(Ops::combine(carry, rel)), epoch_tag | kFlagPrefix);
    } else {
      if (threadIdx.x == 0) st_status(p.chunk_status + k, Ops::pack(rel), epoch_tag | kFlagAgg);
      // chunk 0's prefix includes init and later chunks' totals do not, so
      // the look-back result already counts init exactly once
      carry = lookback<Ops>(p.chunk_status, k, epoch_tag, p.timeout_ns, err);
    }
    if (threadIdx.x == 0) {
      *s_bits = Ops::pack(carry);
      *s_err = err;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const bool err = *s_err != 0;
    if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
    if (k > 0) {
      st_status(p.chunk_status + k, Ops::pack(Ops::combine(Ops::unpack(*s_bits), rel)),
                epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
    }
    __threadfence();  // relative prefixes before the carry that enables phase 2
    st_status(p.chunk_carry + k, *s_bits, epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
  }
}

// ---------------------------------------------------------- scan kernels

template <class P, int ITEMS, bool WIDE>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    scan_lookback_kernel(ScanParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Ops = typename std::conditional<WIDE, F64Ops, AccOps<P>>::type;
  using Pub = typename Ops::Pub;
  constexpr bool kSame = sizeof(In) == sizeof(Out);

  extern __shared__ __align__(16) char smem[];
  __shared__ Acc s_warp[32];
  __shared__ unsigned long long s_tile, s_carry, s_epoch;

  const int warp = threadIdx.x >> 5;
  const int tile_elems = blockDim.x * ITEMS;
  char *buf = smem;
  char *obuf = kSame ? smem : smem + tile_elems * (int)sizeof(In);
  const In *in = reinterpret_cast<const In *>(p.in);
  Out *out = reinterpret_cast<Out *>(p.out);
  const unsigned long long pol = l2_policy_stream();

  if (threadIdx.x == 0) s_epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
  __syncthreads();
  const unsigned long long epoch = s_epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const unsigned long long init_bits = init_value<P, WIDE>(p);

  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    const long long tile = (long long)s_tile;
    if (tile >= p.ntiles) break;
    const unsigned long long base = (unsigned long long)tile * tile_elems;
    const int count = (int)min((unsigned long long)tile_elems, p.n - base);
    load_tile_smem<In>(buf, in + base, count, tile_elems, p.vec_in, pol);
    __syncthreads();

    const Acc agg = thread_total<P, ITEMS>(buf, count);
    Acc tile_agg;
    const Acc texcl = block_exclusive_scan<AccOps<P>>(agg, s_warp, &tile_agg);

    if (warp == 0) {
      const unsigned long long agg_bits = publish_value<P, WIDE>(tile_agg);
      const bool publish = tile != p.stall_tile;
      Pub carry;
      if (tile == 0) {
        carry = Ops::unpack(init_bits);
        if ((threadIdx.x & 31) == 0 && publish)
          st_status(p.status, Ops::pack(Ops::combine(carry, Ops::unpack(agg_bits))), epoch_tag | kFlagPrefix);
      } else {
        if ((threadIdx.x & 31) == 0 && publish) st_status(p.status + tile, agg_bits, epoch_tag | kFlagAgg);
        bool err;
        carry = lookback<Ops>(p.status, tile, epoch_tag, p.timeout_ns, err);
        if ((threadIdx.x & 31) == 0) {
          if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
          if (publish)
            st_status(p.status + tile, Ops::pack(Ops::combine(carry, Ops::unpack(agg_bits))),
                      epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
        }
      }
      if ((threadIdx.x & 31) == 0) s_carry = Ops::pack(carry);
    }
    __syncthreads();
    emit_scan<P, ITEMS>(buf, obuf, start_value<P, WIDE>(s_carry, texcl), p.inclusive);
    __syncthreads();
    store_tile<Out>(obuf, out + base, count, tile_elems, p.vec_out);
    __syncthreads();
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

template <class P, int ITEMS, bool WIDE>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    scan_twophase_kernel(ScanParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Ops = typename std::conditional<WIDE, F64Ops, AccOps<P>>::type;
  using Pub = typename Ops::Pub;
  constexpr bool kSame = sizeof(In) == sizeof(Out);

  extern __shared__ __align__(16) char smem[];
  __shared__ Acc s_warp[32];
  __shared__ Pub s_pub[32];
  __shared__ unsigned long long s_w[2], s_carry, s_epoch, s_bits;
  __shared__ int s_fin, s_err;

  const int tile_elems = blockDim.x * ITEMS;
  const int in_bytes = tile_elems * (int)sizeof(In);
  char *bufs[2] = {smem, smem + in_bytes};
  char *obuf_sep = smem + 2 * in_bytes;
  const In *in = reinterpret_cast<const In *>(p.in);
  Out *out = reinterpret_cast<Out *>(p.out);
  const unsigned long long keep = l2_policy_keep(), stream = l2_policy_stream();
  const long long nitems = 2 * p.ntiles;

  if (threadIdx.x == 0) {
    s_epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
    s_w[0] = atomicAdd(&p.hdr->tile_ctr, 1ull);
  }
  __syncthreads();
  const unsigned long long epoch = s_epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const unsigned long long init_bits = init_value<P, WIDE>(p);
  long long known_chunk = -1;  // thread 0: chunk whose carry is in known_bits
  unsigned long long known_bits = 0;

  // Bring the input tile of work id w into buf (phase-1 reads are kept in
  // L2 for phase 2; phase-2 reads release their lines).
  auto prefetch = [&](long long w, char *buf) {
    if (w < nitems) {
      const WorkItem it = decode_work(w, p.ntiles, p.chunk_tiles, p.nchunks, p.lookahead);
      if (it.tile >= 0 && it.tile < p.ntiles) {
        const unsigned long long b = (unsigned long long)it.tile * tile_elems;
        prefetch_tile<In>(buf, in + b, (int)min((unsigned long long)tile_elems, p.n - b), tile_elems,
                          p.vec_in, it.phase == 1 ? keep : stream);
        return;
      }
    }
    cp_async_commit();
  };
  prefetch((long long)s_w[0], bufs[0]);

  for (int i = 0;; ++i) {
    const long long w = (long long)s_w[i & 1];
    if (w >= nitems) break;
    char *buf = bufs[i & 1];
    if (threadIdx.x == 0) s_w[(i + 1) & 1] = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    prefetch((long long)s_w[(i + 1) & 1], bufs[(i + 1) & 1]);
    const WorkItem item = decode_work(w, p.ntiles, p.chunk_tiles, p.nchunks, p.lookahead);
    const long long tile = item.tile;
    if (tile < 0 || tile >= p.ntiles) {  // never taken: decode_work covers [0, 2 ntiles)
      if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_INVALID_ARG);
      cp_async_wait_1();
      __syncthreads();
      continue;
    }
    const unsigned long long base = (unsigned long long)tile * tile_elems;
    const int count = (int)min((unsigned long long)tile_elems, p.n - base);
    if (item.phase == 2 && threadIdx.x == 0) {
      // tile carry = chunk carry (+) chunk-relative prefix of the tile
      if (item.chunk != known_chunk) {
        bool err = false;
        known_bits = wait_flag(p.chunk_carry + item.chunk, epoch_tag, kFlagPrefix, p.timeout_ns, &err);
        if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
        known_chunk = item.chunk;
      }
      s_carry = Ops::pack(Ops::combine(Ops::unpack(known_bits),
                                       Ops::unpack(ld_status(p.status + tile).payload)));
    }
    cp_async_wait_1();  // this item's tile has landed
    __syncthreads();

    const Acc agg = thread_total<P, ITEMS>(buf, count);
    Acc tile_agg;
    const Acc texcl = block_exclusive_scan<AccOps<P>>(agg, s_warp, &tile_agg);
    if (item.phase == 1) {
      if (threadIdx.x == 0) {
        int fin = 0;
        if (tile != p.stall_tile) {
          st_status(p.status + tile, publish_value<P, WIDE>(tile_agg), epoch_tag | kFlagAgg);
          __threadfence();
          const long long S = min(p.chunk_tiles, p.ntiles - item.chunk * p.chunk_tiles);
          fin = atomicAdd(p.counters + item.chunk, 1u) == (unsigned)(S - 1);
        }
        s_fin = fin;
      }
      __syncthreads();
      if (s_fin) {
        __threadfence();
        finalize_chunk<Ops>(p, item.chunk, epoch_tag, init_bits, s_pub, &s_bits, &s_err);
      }
    } else {
      char *obuf = kSame ? buf : obuf_sep;
      emit_scan<P, ITEMS>(buf, obuf, start_value<P, WIDE>(s_carry, texcl), p.inclusive);
      __syncthreads();
      store_tile<Out>(obuf, out + base, count, tile_elems, p.vec_out);
    }
    __syncthreads();
  }
  finish_launch(p.hdr, epoch, p.counters, p.nchunks);
}

// ------------------------------------------------------- copy_if kernels

// Predicate flags of this thread's ITEMS consecutive elements.
template <class T, int ITEMS>
__device__ __forceinline__ unsigned thread_flags(const char *buf, int count, const ScanParams &p,
                                                 int *kept) {
  constexpr int EPV = 16 / (int)sizeof(T);
  constexpr int VPT = ITEMS / EPV;
  const int first = threadIdx.x * ITEMS;
  unsigned keep = 0;
  int n = 0;
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    const T *e = reinterpret_cast<const T *>(&w);
#pragma unroll
    for (int q = 0; q < EPV; ++q) {
      const int j = k * EPV + q;
      const bool kb = (first + j < count) && pred_bits(e[q], p.mask, p.cmp, p.rhs);
      keep |= (unsigned)kb << j;
      n += kb;
    }
  }
  *kept = n;
  return keep;
}

// Compact the kept elements of this thread into the staging tile at `o`.
template <class T, int ITEMS>
__device__ __forceinline__ void emit_kept(const char *buf, char *obuf, unsigned keep, int o) {
  constexpr int EPV = 16 / (int)sizeof(T);
  constexpr int VPT = ITEMS / EPV;
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    if ((keep >> (k * EPV)) & ((1u << EPV) - 1u)) {
      const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
      const T *e = reinterpret_cast<const T *>(&w);
#pragma unroll
      for (int q = 0; q < EPV; ++q)
        if (keep & (1u << (k * EPV + q))) *smem_elem_ptr<T>(obuf, o++) = e[q];
    }
  }
}

template <class T, int ITEMS>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    copy_if_lookback_kernel(ScanParams p) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long s_warp[32];
  __shared__ unsigned long long s_tile, s_carry, s_epoch;

  const int warp = threadIdx.x >> 5;
  const int tile_elems = blockDim.x * ITEMS;
  char *buf = smem;
  char *obuf = smem + tile_elems * (int)sizeof(T);
  const T *in = reinterpret_cast<const T *>(p.in);
  T *out = reinterpret_cast<T *>(p.out);
  const unsigned long long pol = l2_policy_stream();

  if (threadIdx.x == 0) s_epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
  __syncthreads();
  const unsigned long long epoch = s_epoch;
  const unsigned long long epoch_tag = epoch << 8;

  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    const long long tile = (long long)s_tile;
    if (tile >= p.ntiles) break;
    const unsigned long long base = (unsigned long long)tile * tile_elems;
    const int count = (int)min((unsigned long long)tile_elems, p.n - base);
    load_tile_smem<T>(buf, in + base, count, tile_elems, p.vec_in, pol);
    __syncthreads();
    int kept;
    const unsigned keep = thread_flags<T, ITEMS>(buf, count, p, &kept);
    unsigned long long tile_kept;
    const unsigned long long texcl =
        block_exclusive_scan<CountOps>((unsigned long long)kept, s_warp, &tile_kept);

    if (warp == 0) {
      const bool publish = tile != p.stall_tile;
      unsigned long long carry = 0;
      if (tile == 0) {
        if ((threadIdx.x & 31) == 0 && publish) st_status(p.status, tile_kept, epoch_tag | kFlagPrefix);
      } else {
        if ((threadIdx.x & 31) == 0 && publish) st_status(p.status + tile, tile_kept, epoch_tag | kFlagAgg);
        bool err;
        carry = lookback<CountOps>(p.status, tile, epoch_tag, p.timeout_ns, err);
        if ((threadIdx.x & 31) == 0) {
          if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
          if (publish)
            st_status(p.status + tile, carry + tile_kept,
                      epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
        }
      }
      if ((threadIdx.x & 31) == 0) {
        s_carry = carry;
        if (tile == p.ntiles - 1 && p.num_copied) *p.num_copied = carry + tile_kept;
      }
    }
    emit_kept<T, ITEMS>(buf, obuf, keep, (int)texcl);
    __syncthreads();
    const unsigned long long obase = s_carry;
    if (obase <= p.n && tile_kept <= p.n - obase) {
      for (int i = threadIdx.x; i < (int)tile_kept; i += blockDim.x)
        out[obase + i] = *smem_elem_ptr<T>(obuf, i);
    } else if (threadIdx.x == 0) {
      record_error(p.hdr, B2P_ERR_INVALID_ARG);
    }
    __syncthreads();
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

template <class T, int ITEMS>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    copy_if_twophase_kernel(ScanParams p) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned long long s_warp[32];
  __shared__ unsigned long long s_w[2], s_carry, s_epoch, s_bits;
  __shared__ int s_fin, s_err;

  const int tile_elems = blockDim.x * ITEMS;
  const int buf_bytes = tile_elems * (int)sizeof(T);
  char *bufs[2] = {smem, smem + buf_bytes};
  char *obuf = smem + 2 * buf_bytes;  // compacted output staging
  const T *in = reinterpret_cast<const T *>(p.in);
  T *out = reinterpret_cast<T *>(p.out);
  const unsigned long long keepp = l2_policy_keep(), stream = l2_policy_stream();
  const long long nitems = 2 * p.ntiles;

  if (threadIdx.x == 0) {
    s_epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
    s_w[0] = atomicAdd(&p.hdr->tile_ctr, 1ull);
  }
  __syncthreads();
  const unsigned long long epoch = s_epoch;
  const unsigned long long epoch_tag = epoch << 8;
  long long known_chunk = -1;  // thread 0: chunk whose carry is in known_bits
  unsigned long long known_bits = 0;

  auto prefetch = [&](long long w, char *buf) {
    if (w < nitems) {
      const WorkItem it = decode_work(w, p.ntiles, p.chunk_tiles, p.nchunks, p.lookahead);
      if (it.tile >= 0 && it.tile < p.ntiles) {
        const unsigned long long b = (unsigned long long)it.tile * tile_elems;
        prefetch_tile<T>(buf, in + b, (int)min((unsigned long long)tile_elems, p.n - b), tile_elems,
                         p.vec_in, it.phase == 1 ? keepp : stream);
        return;
      }
    }
    cp_async_commit();
  };
  prefetch((long long)s_w[0], bufs[0]);

  for (int i = 0;; ++i) {
    const long long w = (long long)s_w[i & 1];
    if (w >= nitems) break;
    char *buf = bufs[i & 1];
    if (threadIdx.x == 0) s_w[(i + 1) & 1] = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    prefetch((long long)s_w[(i + 1) & 1], bufs[(i + 1) & 1]);
    const WorkItem item = decode_work(w, p.ntiles, p.chunk_tiles, p.nchunks, p.lookahead);
    const long long tile = item.tile;
    if (tile < 0 || tile >= p.ntiles) {  // never taken: decode_work covers [0, 2 ntiles)
      if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_INVALID_ARG);
      cp_async_wait_1();
      __syncthreads();
      continue;
    }
    const unsigned long long base = (unsigned long long)tile * tile_elems;
    const int count = (int)min((unsigned long long)tile_elems, p.n - base);
    if (item.phase == 2 && threadIdx.x == 0) {
      if (item.chunk != known_chunk) {
        bool err = false;
        known_bits = wait_flag(p.chunk_carry + item.chunk, epoch_tag, kFlagPrefix, p.timeout_ns, &err);
        if (err) {
          record_error(p.hdr, B2P_ERR_TIMEOUT);
          known_bits = ~0ull;
        }
        known_chunk = item.chunk;
      }
      // the offset is an output address: accept it only from this launch's
      // words (after a time-out they may be stale)
      const StatusWord w = ld_status(p.status + tile);
      const bool ok = known_bits != ~0ull && (w.meta & ~0xffull) == epoch_tag && (w.meta & kFlagPrefix);
      s_carry = ok ? known_bits + w.payload : ~0ull;
    }
    cp_async_wait_1();
    __syncthreads();

    int kept;
    const unsigned keep = thread_flags<T, ITEMS>(buf, count, p, &kept);
    unsigned long long tile_kept;
    const unsigned long long texcl =
        block_exclusive_scan<CountOps>((unsigned long long)kept, s_warp, &tile_kept);
    if (item.phase == 1) {
      if (threadIdx.x == 0) {
        int fin = 0;
        if (tile != p.stall_tile) {
          st_status(p.status + tile, tile_kept, epoch_tag | kFlagAgg);
          __threadfence();
          const long long S = min(p.chunk_tiles, p.ntiles - item.chunk * p.chunk_tiles);
          fin = atomicAdd(p.counters + item.chunk, 1u) == (unsigned)(S - 1);
        }
        s_fin = fin;
      }
      __syncthreads();
      if (s_fin) {
        __threadfence();
        finalize_chunk<CountOps>(p, item.chunk, epoch_tag, 0ull, s_warp, &s_bits, &s_err);
        if (threadIdx.x == 0 && item.chunk == p.nchunks - 1 && p.num_copied)
          *p.num_copied = ld_status(p.chunk_status + item.chunk).payload;  // inclusive count
      }
    } else {
      emit_kept<T, ITEMS>(buf, obuf, keep, (int)texcl);
      __syncthreads();
      const unsigned long long obase = s_carry;
      if (obase <= p.n && tile_kept <= p.n - obase) {
        for (int i2 = threadIdx.x; i2 < (int)tile_kept; i2 += blockDim.x)
          out[obase + i2] = *smem_elem_ptr<T>(obuf, i2);
      } else if (threadIdx.x == 0 && obase != ~0ull) {
        record_error(p.hdr, B2P_ERR_INVALID_ARG);
      }
    }
    __syncthreads();
  }
  finish_launch(p.hdr, epoch, p.counters, p.nchunks);
}

// ---------------------------------------------------------------- host

namespace {

constexpr int kMaxTileElems = 8192;

// Chunk size of the two-phase kernels (bytes of input per chunk) and how
// many chunks phase 1 runs ahead of phase 2.  B2P_SCAN_CHUNK_MB and
// B2P_SCAN_LOOKAHEAD override them (read once).
size_t chunk_bytes() {
  static const size_t v = [] {
    const char *e = getenv("B2P_SCAN_CHUNK_MB");
    long mb = e ? atol(e) : 16;
    return (size_t)(mb > 0 ? mb : 16) << 20;
  }();
  return v;
}
int lookahead_chunks() {
  static const int v = [] {
    const char *e = getenv("B2P_SCAN_LOOKAHEAD");
    int d = e ? atoi(e) : 2;
    return d > 0 ? d : 2;
  }();
  return v;
}

// Shared memory of one block: the input tile, plus a second tile for
// outputs whose element size differs (scan) or for the compacted elements
// (copy_if).  A thread's row must be whole 16-byte vectors.
size_t tile_smem(size_t esize_in, size_t esize_out, int block, int items, bool compaction) {
  const size_t t = (size_t)block * items;
  return t * (esize_in + ((compaction || esize_in != esize_out) ? esize_out : 0));
}

bool tile_ok(size_t esize_in, size_t esize_out, int block, int items, bool compaction = false) {
  if (block * items > kMaxTileElems) return false;
  if ((items * esize_in) % 16 || (items * esize_out) % 16) return false;
  // the two-phase kernels add a second input tile
  return tile_smem(esize_in, esize_out, block, items, compaction) + (size_t)block * items * esize_in <=
         200 * 1024;
}

struct Layout {
  long long ntiles, chunk_tiles, nchunks;
  size_t bytes;
};

Layout layout_for(size_t n, size_t esize_in, long long tile) {
  Layout l;
  l.ntiles = (long long)((n + tile - 1) / tile);
  l.chunk_tiles = std::max<long long>(1, (long long)(chunk_bytes() / ((size_t)tile * esize_in)));
  // at most kCounterSlots chunks (larger chunks for very long inputs)
  l.chunk_tiles = std::max<long long>(l.chunk_tiles, (l.ntiles + (long long)kCounterSlots - 1) /
                                                         (long long)kCounterSlots);
  l.nchunks = (l.ntiles + l.chunk_tiles - 1) / l.chunk_tiles;
  l.bytes = kScratchPrefix + (size_t)(l.ntiles + 2 * l.nchunks) * sizeof(StatusWord);
  return l;
}

void fill_layout(ScanParams &p, const Layout &l, void *scratch) {
  char *s = reinterpret_cast<char *>(scratch);
  p.hdr = reinterpret_cast<ScratchHeader *>(s);
  p.ntiles = l.ntiles;
  p.chunk_tiles = l.chunk_tiles;
  p.nchunks = l.nchunks;
  p.lookahead = lookahead_chunks();
  p.counters = reinterpret_cast<unsigned *>(s + kHeaderBytes);
  p.status = reinterpret_cast<StatusWord *>(s + kScratchPrefix);
  p.chunk_status = p.status + l.ntiles;
  p.chunk_carry = p.chunk_status + l.nchunks;
}

template <class K>
int launch_kernel(K kernel, ScanParams &p, const LaunchConfig &lc, size_t smem, long long units,
                  cudaStream_t st) {
  const void *kfn = (const void *)kernel;
  int rc = ensure_dynamic_smem(kfn, smem);
  if (rc) return rc;
  int grid = grid_for(lc.grid_mode, units, 1, kfn, lc.block, smem);
  kernel<<<grid, lc.block, smem, st>>>(p);
  return cuda_status(cudaGetLastError());
}

template <class P, int ITEMS, bool WIDE>
int launch_scan_kernel(ScanParams &p, const LaunchConfig &lc, size_t smem, cudaStream_t st) {
  if (lc.grid_mode == 0)
    return launch_kernel(scan_lookback_kernel<P, ITEMS, WIDE>, p, lc, smem, p.ntiles, st);
  // the two-phase kernel double-buffers its input tile
  const size_t smem2 = smem + (size_t)lc.block * ITEMS * sizeof(typename P::In);
  return launch_kernel(scan_twophase_kernel<P, ITEMS, WIDE>, p, lc, smem2, 2 * p.ntiles, st);
}

template <class P, int ITEMS>
int launch_scan_items(ScanParams &p, const LaunchConfig &lc, bool wide, cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  if constexpr ((ITEMS * sizeof(In)) % 16 != 0 || (ITEMS * sizeof(Out)) % 16 != 0) {
    return B2P_ERR_INVALID_ARG;  // masked by tile_ok; never instantiated
  } else {
    const size_t smem = tile_smem(sizeof(In), sizeof(Out), lc.block, ITEMS, false);
    if constexpr (P::kCompensated) {
      if (wide) return launch_scan_kernel<P, ITEMS, true>(p, lc, smem, st);
    }
    return launch_scan_kernel<P, ITEMS, false>(p, lc, smem, st);
  }
}

template <class P>
int launch_scan_t(int inclusive, const void *in, void *out, size_t n, const void *init,
                  void *scratch, size_t sb, int config, cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  LaunchConfig lc = describe_config(config);
  if (!tile_ok(sizeof(In), sizeof(Out), lc.block, lc.items)) return B2P_ERR_INVALID_ARG;
  const Layout l = layout_for(n, sizeof(In), (long long)lc.block * lc.items);
  if (sb < l.bytes || (reinterpret_cast<uintptr_t>(scratch) & 255)) return B2P_ERR_SCRATCH;
  ScanParams p{};
  p.in = in;
  p.out = out;
  p.n = n;
  fill_layout(p, l, scratch);
  p.inclusive = inclusive;
  p.has_init = init != nullptr;
  if (init) memcpy(&p.init_bits, init, sizeof(Out));
  p.vec_in = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
  p.vec_out = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  p.timeout_ns = wait_timeout_ns();
  p.stall_tile = debug_stall_tile();
  const bool wide = n > (1ull << 24);
  switch (lc.items) {
  case 4: return launch_scan_items<P, 4>(p, lc, wide, st);
  case 8: return launch_scan_items<P, 8>(p, lc, wide, st);
  case 16: return launch_scan_items<P, 16>(p, lc, wide, st);
  default: return launch_scan_items<P, 32>(p, lc, wide, st);
  }
}

template <int DT>
int scan_dispatch(int op, int inclusive, const void *in, void *out, size_t n, const void *init,
                  void *scratch, size_t sb, int config, cudaStream_t st) {
#define B2P_SCAN_CASE(OP)                                                                       \
  case OP:                                                                                      \
    return launch_scan_t<typename PolicyOf<DT, OP>::type>(inclusive, in, out, n, init, scratch, \
                                                          sb, config, st);
  switch (op) {
    B2P_SCAN_CASE(B2P_SUM)
    B2P_SCAN_CASE(B2P_PROD)
    B2P_SCAN_CASE(B2P_MIN)
    B2P_SCAN_CASE(B2P_MAX)
  default: break;
  }
  if constexpr (DT == B2P_F32 || DT == B2P_BF16 || DT == B2P_F64) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    switch (op) {
      B2P_SCAN_CASE(B2P_AND)
      B2P_SCAN_CASE(B2P_OR)
      B2P_SCAN_CASE(B2P_XOR)
    default: return B2P_ERR_INVALID_ARG;
    }
  }
#undef B2P_SCAN_CASE
}

template <class T, int ITEMS>
int launch_copy_if_items(ScanParams &p, const LaunchConfig &lc, cudaStream_t st) {
  const size_t smem = tile_smem(sizeof(T), sizeof(T), lc.block, ITEMS, true);
  if (lc.grid_mode == 0)
    return launch_kernel(copy_if_lookback_kernel<T, ITEMS>, p, lc, smem, p.ntiles, st);
  const size_t smem2 = smem + (size_t)lc.block * ITEMS * sizeof(T);
  return launch_kernel(copy_if_twophase_kernel<T, ITEMS>, p, lc, smem2, 2 * p.ntiles, st);
}

template <class T>
int launch_copy_if_t(const void *in, void *out, size_t n, uint64_t mask, int cmp, uint64_t rhs,
                     uint64_t *num_copied, void *scratch, size_t sb, int config, cudaStream_t st) {
  LaunchConfig lc = describe_config(config);
  if (!tile_ok(sizeof(T), sizeof(T), lc.block, lc.items, true)) return B2P_ERR_INVALID_ARG;
  const Layout l = layout_for(n, sizeof(T), (long long)lc.block * lc.items);
  if (sb < l.bytes || (reinterpret_cast<uintptr_t>(scratch) & 255)) return B2P_ERR_SCRATCH;
  ScanParams p{};
  p.in = in;
  p.out = out;
  p.n = n;
  fill_layout(p, l, scratch);
  p.vec_in = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
  p.timeout_ns = wait_timeout_ns();
  p.stall_tile = debug_stall_tile();
  p.mask = mask;
  p.rhs = rhs;
  p.cmp = cmp;
  p.num_copied = reinterpret_cast<unsigned long long *>(num_copied);
  switch (lc.items) {
  case 4: return launch_copy_if_items<T, 4>(p, lc, st);
  case 8: return launch_copy_if_items<T, 8>(p, lc, st);
  case 16: return launch_copy_if_items<T, 16>(p, lc, st);
  default: return launch_copy_if_items<T, 32>(p, lc, st);
  }
}

}  // namespace

bool scan_config_valid(int dtype, int config) {
  if (config < 0 || config >= B2P_NUM_CONFIGS) return false;
  LaunchConfig lc = describe_config(config);
  return tile_ok(dtype_size(dtype), acc_size(dtype), lc.block, lc.items);
}

bool copy_if_config_valid(int dtype, int config) {
  if (config < 0 || config >= B2P_NUM_CONFIGS) return false;
  const size_t es = dtype_size(dtype);
  if (es != 4 && es != 8) return false;
  LaunchConfig lc = describe_config(config);
  return tile_ok(es, es, lc.block, lc.items, true);
}

size_t scan_scratch_bytes(int dtype, size_t n, int config) {
  const size_t es = dtype_size(dtype);
  if (config >= 0) {
    LaunchConfig lc = describe_config(config);
    return layout_for(n, es, (long long)lc.block * lc.items).bytes;
  }
  size_t m = 0;
  for (int c = 0; c < B2P_NUM_CONFIGS; ++c) {
    LaunchConfig lc = describe_config(c);
    m = std::max(m, layout_for(n, es, (long long)lc.block * lc.items).bytes);
  }
  return m;
}

size_t copy_if_scratch_bytes(int dtype, size_t n, int config) {
  return scan_scratch_bytes(dtype, n, config);
}

int launch_scan(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
                const void *init, void *scratch, size_t sb, int config, cudaStream_t st) {
  if (config >= 0 && config < B2P_NUM_CONFIGS) {
    const LaunchConfig lc = describe_config(config);
    if (lc.grid_mode == 1 && scan_tma_shape(dtype, lc.block, lc.items) &&
        sb >= scan_scratch_bytes(dtype, n, config)) {
      const int rc = launch_scan_tma(dtype, op, inclusive, in, out, n, init, scratch, lc.block, lc.items, st);
      if (rc != B2P_ERR_UNSUPPORTED) return rc;
    }
  }
  switch (dtype) {
  case B2P_I32: return scan_dispatch<B2P_I32>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  case B2P_I64: return scan_dispatch<B2P_I64>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  case B2P_U32: return scan_dispatch<B2P_U32>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  case B2P_U64: return scan_dispatch<B2P_U64>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  case B2P_F32: return scan_dispatch<B2P_F32>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  case B2P_BF16: return scan_dispatch<B2P_BF16>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  case B2P_F64: return scan_dispatch<B2P_F64>(op, inclusive, in, out, n, init, scratch, sb, config, st);
  default: return B2P_ERR_INVALID_ARG;
  }
}

int launch_copy_if(int dtype, const void *in, void *out, size_t n, uint64_t mask, int cmp,
                   uint64_t rhs, uint64_t *num_copied, void *scratch, size_t sb, int config,
                   cudaStream_t st) {
  if (config >= 0 && config < B2P_NUM_CONFIGS) {
    const LaunchConfig lc = describe_config(config);
    if (lc.grid_mode == 1 && copy_if_tma_shape(dtype, lc.block, lc.items) &&
        sb >= copy_if_scratch_bytes(dtype, n, config)) {
      const int rc = launch_copy_if_tma(dtype, in, out, n, mask, cmp, rhs, num_copied, scratch, lc.block,
                                        lc.items, st);
      if (rc != B2P_ERR_UNSUPPORTED) return rc;
    }
  }
  switch (dtype_size(dtype)) {
  case 4: return launch_copy_if_t<uint32_t>(in, out, n, mask, cmp, rhs, num_copied, scratch, sb, config, st);
  case 8: return launch_copy_if_t<unsigned long long>(in, out, n, mask, cmp, rhs, num_copied, scratch, sb, config, st);
  default: return B2P_ERR_UNSUPPORTED;
  }
}

}  // namespace b2p
