// Pipelined single-pass scan: grid mode 1 of scans whose element and
// output sizes match (every dtype but bf16).
//
// Same algorithm as the reference's decoupled look-back scan
// (algorithms/scan/decoupled_lookback_scan.hpp:555-655: per-tile aggregate,
// look-back over predecessors' aggregates/prefixes, then the tile's scan
// from its carry), arranged for B200 as one persistent block per SM with
// three kinds of warps:
//
//  * a producer warp takes dynamic tile ids in order and streams each tile
//    into a ring of shared-memory stages with TMA bulk tensor loads
//    (128-byte swizzle, completion on an mbarrier);
//  * consumer warps reduce every tile as soon as it lands and publish its
//    aggregate at once, then emit an older tile (LAG tiles behind) in place
//    and write it back with a TMA bulk tensor store;
//  * two look-back warps resolve the carries of the reduced tiles in
//    parallel (warp-parallel bounded look-back over epoch-tagged 128-bit
//    status words), so the DRAM latency skew between tiles that the
//    look-back waits on overlaps with the reduction of later tiles.
//
// Elements past the last complete 128-byte row are read and written with
// plain accesses.  Every wait is bounded; a wait that runs out records
// B2P_ERR_TIMEOUT in the scratch header and the block leaves its loops.
#include "scan_tile.cuh"
#include "tma.cuh"
#include "internal.h"

#include <algorithm>
#include <mutex>

namespace b2p {

namespace {

constexpr int kMaxStages = 12;
constexpr int kMaxLag = 6;
constexpr int kLookWarps = 2;
constexpr size_t kStageBudget = 196 * 1024;

struct TmaParams {
  unsigned long long n;
  long long ntiles;
  long long rows_full;            // complete 128-byte rows (the tensor maps' extent)
  unsigned long long tail_begin;  // first element past the complete rows
  int inclusive;
  int has_init;
  unsigned long long init_raw;    // Out-typed init value
  int stages, lag;
  const void *in;
  void *out;
  ScratchHeader *hdr;
  StatusWord *status;
  unsigned long long timeout_ns;
  long long stall_tile;
  // copy_if
  unsigned long long mask, rhs;
  int cmp;
  unsigned long long *num_copied;
};

// Block-shared state of the pipeline: per stage, the TMA fill barrier
// (full), the stage-free barrier (empty), the aggregate-published barrier
// (aggr: consumers -> look-back warps) and the carry-ready barrier (cready:
// look-back warps -> consumers), with the stage's tile id, aggregate and
// carry.
struct PipeState {
  uint64_t full[kMaxStages], empty[kMaxStages], aggr[kMaxStages], cready[kMaxStages];
  long long tile[kMaxStages];
  unsigned long long agg[kMaxStages], carry[kMaxStages];
  unsigned long long epoch;
  long long end_item;
};

// Thread total over ITEMS consecutive elements of a full tile.
template <class P, int ITEMS>
__device__ __forceinline__ typename P::Acc thread_total_full(const char *buf) {
  using In = typename P::In;
  constexpr int IPV = 16 / (int)sizeof(In);
  constexpr int VPT = ITEMS * (int)sizeof(In) / 16;
  typename P::Acc agg = P::identity();
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    const In *e = reinterpret_cast<const In *>(&w);
#pragma unroll
    for (int q = 0; q < IPV; ++q) P::add(agg, e[q]);
  }
  if constexpr (P::kCompensated) agg = df_norm(agg);
  return agg;
}

// fp32 SUM, pass 1: compensated (TwoSum) running sums of the thread's
// elements from zero, written back in place rounded to fp32 (inclusive: after
// adding the element, exclusive: before).  Returns the thread total.
template <int ITEMS, bool INCLUSIVE>
__device__ __forceinline__ DF thread_runs_f32(char *buf) {
  constexpr int VPT = ITEMS / 4;
  DF run{0.f, 0.f};
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    float4 *slot = reinterpret_cast<float4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    float4 w = *slot;
    float *e = reinterpret_cast<float *>(&w);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if constexpr (INCLUSIVE) {
        df_accumulate(run, e[q]);
        e[q] = __fadd_rn(run.hi, run.lo);
      } else {
        const float before = __fadd_rn(run.hi, run.lo);
        df_accumulate(run, e[q]);
        e[q] = before;
      }
    }
    *slot = w;
  }
  return df_norm(run);
}

// fp32 SUM, pass 2: output = start + run.  The run carries at most one
// rounding of its exact value, so each output is within ~2 ulp of the exact
// prefix for same-signed data.
template <int ITEMS>
__device__ __forceinline__ void emit_f32_runs(char *buf, DF start) {
  constexpr int VPT = ITEMS / 4;
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    float4 *slot = reinterpret_cast<float4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    float4 w = *slot;
    w.x = __fadd_rn(start.hi, __fadd_rn(start.lo, w.x));
    w.y = __fadd_rn(start.hi, __fadd_rn(start.lo, w.y));
    w.z = __fadd_rn(start.hi, __fadd_rn(start.lo, w.z));
    w.w = __fadd_rn(start.hi, __fadd_rn(start.lo, w.w));
    *slot = w;
  }
}

// Block exclusive scan over the NC consumer threads (named barrier 1; the
// producer and look-back warps do not take part).
template <class Ops, int NC>
__device__ __forceinline__ typename Ops::Pub consumer_exclusive_scan(typename Ops::Pub v,
                                                                     typename Ops::Pub *s_warp,
                                                                     typename Ops::Pub *total) {
  using Pub = typename Ops::Pub;
  constexpr int kWarps = NC / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Pub incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Pub o = shfl_up(incl, d);
    if (lane >= d) incl = Ops::combine(o, incl);
  }
  if (lane == 31) s_warp[warp] = incl;
  bar_named(1, NC);
  if (warp == 0) {
    Pub w = lane < kWarps ? s_warp[lane] : Ops::identity();
#pragma unroll
    for (int d = 1; d < kWarps; d <<= 1) {
      Pub o = shfl_up(w, d);
      if (lane >= d) w = Ops::combine(o, w);
    }
    if (lane < kWarps) s_warp[lane] = w;
  }
  bar_named(1, NC);
  Pub ex = shfl_up(incl, 1);
  if (lane == 0) ex = Ops::identity();
  if (warp > 0) ex = Ops::combine(s_warp[warp - 1], ex);
  *total = s_warp[kWarps - 1];
  return ex;
}

// Position in the ring of S stages: stage index and mbarrier phase parity
// of an item, advanced without divisions.
struct RingPos {
  int s = 0;
  unsigned ph = 0;
  __device__ __forceinline__ void advance(int k, int S) {
    s += k;
    while (s >= S) {
      s -= S;
      ph ^= 1u;
    }
  }
};

// Carry of tile 0 (init, or the identity), in the published representation.
template <class P, bool WIDE>
__device__ __forceinline__ unsigned long long tile0_carry(const TmaParams &p) {
  using Out = typename P::Out;
  if (!p.has_init) {
    if constexpr (WIDE) return F64Ops::pack(0.0);
    else return P::pack(P::identity());
  }
  const Out v = from_bits64<Out>(p.init_raw);
  if constexpr (WIDE) return F64Ops::pack((double)v);
  else return P::pack(P::from_out(v));
}

// Thread 0 of the block: barriers and the launch epoch.
__device__ __forceinline__ void pipe_init(PipeState &ps, const TmaParams &p) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < p.stages; ++i) {
      mbar_init(&ps.full[i], 1);
      mbar_init(&ps.empty[i], 1);
      mbar_init(&ps.aggr[i], 1);
      mbar_init(&ps.cready[i], 1);
    }
    mbar_init_fence();
    ps.epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
    ps.end_item = 0x7fffffffffffffffll;
  }
}

// Producer (one thread): dynamic tile ids in order; each tile's complete
// rows streamed into the next free stage (stages `stride` bytes apart) in
// boxes of `box` rows.  A tile past the last complete row completes its
// stage without a copy.  Tile id -1 ends the consumers.
__device__ __forceinline__ void producer_loop(const CUtensorMap *tin, const TmaParams &p, PipeState &ps,
                                              char *smem, unsigned stride, int rows, int box) {
  prefetch_tensormap(tin);
  const unsigned long long pol = l2_policy_stream();
  const int S = p.stages;
  for (RingPos r;; r.advance(1, S)) {
    const int s = r.s;
    if (!mbar_wait(&ps.empty[s], r.ph ^ 1u, p.timeout_ns)) {
      record_error(p.hdr, B2P_ERR_TIMEOUT);
      ps.tile[s] = -1;
      mbar_arrive(&ps.full[s]);
      return;
    }
    const long long tile = (long long)atomicAdd(&p.hdr->tile_ctr, 1ull);
    if (tile >= p.ntiles) {
      ps.tile[s] = -1;
      mbar_arrive(&ps.full[s]);
      return;
    }
    ps.tile[s] = tile;
    const long long r0 = tile * rows;
    const long long rows_in = min((long long)rows, p.rows_full - r0);
    const int nbox = rows_in > 0 ? (int)((rows_in + box - 1) / box) : 0;
    if (nbox == 0) {
      mbar_arrive(&ps.full[s]);
    } else {
      mbar_arrive_expect_tx(&ps.full[s], (unsigned)nbox * (unsigned)box * 128u);
      for (int b = 0; b < nbox; ++b)
        tma_load_2d(smem + (size_t)s * stride + (size_t)b * box * 128, tin, 0, (int)(r0 + (long long)b * box),
                    &ps.full[s], pol);
    }
  }
}

// Look-back warp wi of kLookWarps: items wi, wi + kLookWarps, ... in stage
// order.  Resolves each reduced tile's carry, publishes its inclusive prefix
// and hands the carry to the consumers.
template <class Ops>
__device__ __forceinline__ void lookback_loop(const TmaParams &p, PipeState &ps, int wi,
                                              unsigned long long init_bits, unsigned long long epoch_tag) {
  using Pub = typename Ops::Pub;
  const int lane = threadIdx.x & 31;
  const int S = p.stages;
  RingPos r;
  r.advance(wi, S);
  for (long long it = wi;; it += kLookWarps, r.advance(kLookWarps, S)) {
    const int s = r.s;
    const bool ok = __shfl_sync(0xffffffffu, (int)mbar_wait(&ps.aggr[s], r.ph, p.timeout_ns), 0) != 0;
    if (!ok) {
      if (lane == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
      return;
    }
    if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) return;
    const long long tile = ps.tile[s];
    const unsigned long long agg_bits = ps.agg[s];
    Pub carry = Ops::unpack(init_bits);
    if (tile > 0) {
      bool err;
      // tile 0's prefix includes init, so the look-back result already does
      carry = lookback<Ops, false>(p.status, tile, epoch_tag, p.timeout_ns, err);
      if (lane == 0) {
        if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
        if (tile != p.stall_tile)
          st_status(p.status + tile, Ops::pack(Ops::combine(carry, Ops::unpack(agg_bits))),
                    epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
      }
    }
    if (lane == 0) {
      ps.carry[s] = Ops::pack(carry);
      mbar_arrive(&ps.cready[s]);
    }
    __syncwarp();
  }
}

// Consumer thread 0 after the last item: end the look-back warps (they wait
// on items it .. it + kLookWarps - 1) and the outstanding bulk stores.
__device__ __forceinline__ void consumers_finish(const TmaParams &p, PipeState &ps, long long it, RingPos rr) {
  if (threadIdx.x == 0) {
    bulk_wait_all();
    ps.end_item = it;
    for (int j = 0; j < kLookWarps; ++j, rr.advance(1, p.stages)) mbar_arrive(&ps.aggr[rr.s]);
  }
}

// Elements past the complete rows (only in the last tile) into the stage.
template <class T, int NC>
__device__ __forceinline__ void load_row_tail(const TmaParams &p, char *buf, long long tile, int tile_elems) {
  const int ntail = (int)(p.n - p.tail_begin);
  const long long j0 = (long long)p.tail_begin - tile * tile_elems;
  if ((int)threadIdx.x < ntail)
    *smem_elem_ptr<T>(buf, (int)j0 + (int)threadIdx.x) =
        reinterpret_cast<const T *>(p.in)[p.tail_begin + threadIdx.x];
  bar_named(1, NC);
}

template <class P, int NC, int ITEMS, bool WIDE>
__global__ void __launch_bounds__(NC + 32 * kLookWarps + 32, 1)
    scan_tma_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
                    TmaParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Ops = typename std::conditional<WIDE, F64Ops, AccOps<P>>::type;
  static_assert(sizeof(In) == sizeof(Out), "in-place emission needs equal element sizes");
  constexpr int kTile = NC * ITEMS;
  constexpr int kEpr = 128 / (int)sizeof(In);  // elements per 128-byte row
  static_assert(kTile % (8 * kEpr) == 0, "a stage is a whole number of 1024-byte swizzle atoms");
  constexpr int kRows = kTile / kEpr;
  constexpr int kBox = kRows < 256 ? kRows : 256;
  static_assert(kRows % kBox == 0, "box rows");
  constexpr unsigned kStageBytes = (unsigned)kRows * 128u;
  constexpr bool kFast = std::is_same<P, FloatSumPolicy<float>>::value;

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) PipeState ps;
  __shared__ Acc s_warp[32];

  pipe_init(ps, p);
  __syncthreads();
  const unsigned long long epoch = ps.epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const unsigned long long init_bits = tile0_carry<P, WIDE>(p);
  const int warp = threadIdx.x >> 5;

  if (warp == NC / 32 + kLookWarps) {
    if ((threadIdx.x & 31) == 0) {
      prefetch_tensormap(&tout);
      producer_loop(&tin, p, ps, smem, kStageBytes, kRows, kBox);
    }
  } else if (warp >= NC / 32) {
    lookback_loop<Ops>(p, ps, warp - NC / 32, init_bits, epoch_tag);
  } else {
    const unsigned long long spol = l2_policy_stream();
    const int S = p.stages, LAG = p.lag;
    const long long last = p.ntiles - 1;
    const int ntail = (int)(p.n - p.tail_begin);
    Out *out = reinterpret_cast<Out *>(p.out);
    Acc q[kMaxLag + 1];  // thread prefixes of reduced, not yet emitted tiles (oldest first)
#pragma unroll
    for (int i = 0; i <= kMaxLag; ++i) q[i] = P::identity();
    int npend = 0;
    long long it = 0;
    bool ok = true;
    RingPos er, rr;   // ring positions of the next item to emit / to reduce
    int prev_s = -1;  // stage of the previous emission (its store may still read it)

    auto emit_one = [&]() -> bool {
      const int s = er.s;
      if (!mbar_wait(&ps.cready[s], er.ph, p.timeout_ns)) {
        if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        return false;
      }
      const long long tile = ps.tile[s];
      char *buf = smem + (size_t)s * kStageBytes;
      const Acc texcl = q[0];
#pragma unroll
      for (int i = 0; i < kMaxLag; ++i) q[i] = q[i + 1];
      const Acc start = start_value<P, WIDE>(ps.carry[s], texcl);
      if constexpr (kFast) emit_f32_runs<ITEMS>(buf, start);
      else emit_scan<P, ITEMS>(buf, buf, start, p.inclusive != 0);
      fence_async_smem();
      bar_named(1, NC);
      if (tile == last && ntail > 0) {
        const long long j0 = (long long)p.tail_begin - tile * kTile;
        if ((int)threadIdx.x < ntail)
          out[p.tail_begin + threadIdx.x] = *smem_elem_ptr<Out>(buf, (int)j0 + (int)threadIdx.x);
        bar_named(1, NC);
      }
      if (threadIdx.x == 0) {
        const long long r0 = tile * kRows;
        const long long rows_out = min((long long)kRows, p.rows_full - r0);
        for (long long r = 0; r < rows_out; r += kBox)
          tma_store_2d(&tout, 0, (int)(r0 + r), buf + r * 128, spol);
        bulk_commit();
        bulk_wait_read<1>();  // the previous emission's store has read its stage
        if (prev_s >= 0) mbar_arrive(&ps.empty[prev_s]);
      }
      prev_s = s;
      er.advance(1, S);
      return true;
    };

    for (;; ++it, rr.advance(1, S)) {
      const int s = rr.s;
      if (!mbar_wait(&ps.full[s], rr.ph, p.timeout_ns)) {
        if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        ok = false;
        break;
      }
      const long long tile = ps.tile[s];
      if (tile < 0) break;
      char *buf = smem + (size_t)s * kStageBytes;
      if (tile == last && ntail > 0) load_row_tail<In, NC>(p, buf, tile, kTile);
      Acc agg;
      if constexpr (kFast) agg = p.inclusive ? thread_runs_f32<ITEMS, true>(buf) : thread_runs_f32<ITEMS, false>(buf);
      else agg = thread_total_full<P, ITEMS>(buf);
      Acc tile_agg;
      const Acc texcl = consumer_exclusive_scan<AccOps<P>, NC>(agg, s_warp, &tile_agg);
#pragma unroll
      for (int i = 0; i <= kMaxLag; ++i)
        if (i == npend) q[i] = texcl;
      if (threadIdx.x == 0) {
        const unsigned long long bits = publish_value<P, WIDE>(tile_agg);
        if (tile != p.stall_tile) {
          if (tile == 0)
            st_status(p.status, Ops::pack(Ops::combine(Ops::unpack(init_bits), Ops::unpack(bits))),
                      epoch_tag | kFlagPrefix);
          else
            st_status(p.status + tile, bits, epoch_tag | kFlagAgg);
        }
        ps.agg[s] = bits;
        mbar_arrive(&ps.aggr[s]);
      }
      ++npend;
      if (npend > LAG) {
        if (!emit_one()) {
          ok = false;
          break;
        }
        --npend;
      }
    }
    if (ok) {
      while (npend > 0) {
        if (!emit_one()) break;
        --npend;
      }
    }
    consumers_finish(p, ps, it, rr);
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

// Order-preserving compaction (copy_if) on the same pipeline.  A tile's
// aggregate is its kept count; its carry is the output position of its
// first kept element.  At emission the kept elements are packed, in order,
// into the stage with the output's 16-byte phase, the 16-byte-aligned middle
// is written with one bulk copy and the unaligned ends with plain stores.
// Stages are kStageBytes + 1024 apart: packing may shift the tile by up to
// 15 bytes.
template <class T, int NC, int ITEMS>
__global__ void __launch_bounds__(NC + 32 * kLookWarps + 32, 1)
    copy_if_tma_kernel(const __grid_constant__ CUtensorMap tin, TmaParams p) {
  constexpr int kTile = NC * ITEMS;
  constexpr int kEpr = 128 / (int)sizeof(T);
  static_assert(kTile % (8 * kEpr) == 0, "a stage is a whole number of 1024-byte swizzle atoms");
  constexpr int kRows = kTile / kEpr;
  constexpr int kBox = kRows < 256 ? kRows : 256;
  static_assert(kRows % kBox == 0, "box rows");
  constexpr unsigned kStride = (unsigned)kRows * 128u + 1024u;
  constexpr int EPV = 16 / (int)sizeof(T);
  constexpr int VPT = ITEMS / EPV;
  static_assert(ITEMS <= 32, "keep mask is 32 bits");

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) PipeState ps;
  __shared__ unsigned long long s_warp[32];

  pipe_init(ps, p);
  __syncthreads();
  const unsigned long long epoch = ps.epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const int warp = threadIdx.x >> 5;

  if (warp == NC / 32 + kLookWarps) {
    if ((threadIdx.x & 31) == 0) producer_loop(&tin, p, ps, smem, kStride, kRows, kBox);
  } else if (warp >= NC / 32) {
    lookback_loop<CountOps>(p, ps, warp - NC / 32, 0ull, epoch_tag);
  } else {
    const int S = p.stages, LAG = p.lag;
    const long long last = p.ntiles - 1;
    const int ntail = (int)(p.n - p.tail_begin);
    T *out = reinterpret_cast<T *>(p.out);
    unsigned long long q[kMaxLag + 1];
#pragma unroll
    for (int i = 0; i <= kMaxLag; ++i) q[i] = 0;
    int npend = 0;
    long long it = 0;
    bool ok = true;
    RingPos er, rr;
    int prev_s = -1;

    // predicate flags of this thread's elements of a tile (count valid ones)
    auto flags = [&](const uint4 (&v)[VPT], int count, int *kept) -> unsigned {
      const int first = threadIdx.x * ITEMS;
      unsigned keep = 0;
      int c = 0;
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const T *e = reinterpret_cast<const T *>(&v[k]);
#pragma unroll
        for (int qq = 0; qq < EPV; ++qq) {
          const int j = k * EPV + qq;
          const bool kb = (first + j < count) && pred_bits(e[qq], p.mask, p.cmp, p.rhs);
          keep |= (unsigned)kb << j;
          c += kb;
        }
      }
      *kept = c;
      return keep;
    };
    auto load_v = [&](const char *buf, uint4 (&v)[VPT]) {
#pragma unroll
      for (int k = 0; k < VPT; ++k) v[k] = *reinterpret_cast<const uint4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    };

    auto emit_one = [&]() -> bool {
      const int s = er.s;
      if (!mbar_wait(&ps.cready[s], er.ph, p.timeout_ns)) {
        if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        return false;
      }
      const long long tile = ps.tile[s];
      char *buf = smem + (size_t)s * kStride;
      const unsigned long long texcl = q[0];
#pragma unroll
      for (int i = 0; i < kMaxLag; ++i) q[i] = q[i + 1];
      const unsigned long long carry = ps.carry[s];
      unsigned long long kept_total = ps.agg[s];
      if (carry > p.n || kept_total > p.n - carry) {  // only after a broken chain: write nothing
        if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        kept_total = 0;
      }
      const int count = (int)min((unsigned long long)kTile, p.n - (unsigned long long)tile * kTile);
      uint4 v[VPT];
      load_v(buf, v);
      int kept;
      const unsigned keep = flags(v, count, &kept);
      bar_named(1, NC);  // every thread holds its elements: the stage may be overwritten
      // pack with the output's 16-byte phase: element k at byte phase + k * sizeof(T)
      const uintptr_t g0 = reinterpret_cast<uintptr_t>(out + carry);
      const unsigned phase = (unsigned)(g0 & 15u);
      unsigned long long o = texcl;
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const T *e = reinterpret_cast<const T *>(&v[k]);
#pragma unroll
        for (int qq = 0; qq < EPV; ++qq)
          if (keep & (1u << (k * EPV + qq))) {
            if (o < kept_total) *reinterpret_cast<T *>(buf + phase + o * sizeof(T)) = e[qq];
            ++o;
          }
      }
      fence_async_smem();
      bar_named(1, NC);
      const uintptr_t g1 = g0 + kept_total * sizeof(T);
      const uintptr_t a0 = (g0 + 15) & ~uintptr_t(15), a1 = g1 & ~uintptr_t(15);
      const bool mid = a1 > a0;
      const long long nhead = mid ? (long long)((a0 - g0) / sizeof(T)) : (long long)kept_total;
      const long long tail0 = mid ? (long long)((a1 - g0) / sizeof(T)) : (long long)kept_total;
      const long long ntl = (long long)kept_total - tail0;
      if ((long long)threadIdx.x < nhead)
        out[carry + threadIdx.x] = *reinterpret_cast<const T *>(buf + phase + threadIdx.x * sizeof(T));
      if (threadIdx.x >= 32 && (long long)threadIdx.x - 32 < ntl) {
        const long long k = tail0 + (threadIdx.x - 32);
        out[carry + k] = *reinterpret_cast<const T *>(buf + phase + k * sizeof(T));
      }
      if (threadIdx.x == 0) {
        if (mid) {
          const unsigned bytes = (unsigned)(a1 - a0);
          asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(a0),
                       "r"(smem_u32(buf + phase + (a0 - g0))), "r"(bytes)
                       : "memory");
        }
        bulk_commit();
        if (tile == last && p.num_copied) *p.num_copied = carry + kept_total;
      }
      bar_named(1, NC);  // plain stores of the ends done before the stage can be released
      if (threadIdx.x == 0) {
        bulk_wait_read<1>();
        if (prev_s >= 0) mbar_arrive(&ps.empty[prev_s]);
      }
      prev_s = s;
      er.advance(1, S);
      return true;
    };

    for (;; ++it, rr.advance(1, S)) {
      const int s = rr.s;
      if (!mbar_wait(&ps.full[s], rr.ph, p.timeout_ns)) {
        if (threadIdx.x == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        ok = false;
        break;
      }
      const long long tile = ps.tile[s];
      if (tile < 0) break;
      char *buf = smem + (size_t)s * kStride;
      if (tile == last && ntail > 0) load_row_tail<T, NC>(p, buf, tile, kTile);
      const int count = (int)min((unsigned long long)kTile, p.n - (unsigned long long)tile * kTile);
      uint4 v[VPT];
      load_v(buf, v);
      int kept;
      (void)flags(v, count, &kept);
      unsigned long long tile_kept;
      const unsigned long long texcl =
          consumer_exclusive_scan<CountOps, NC>((unsigned long long)kept, s_warp, &tile_kept);
#pragma unroll
      for (int i = 0; i <= kMaxLag; ++i)
        if (i == npend) q[i] = texcl;
      if (threadIdx.x == 0) {
        if (tile != p.stall_tile)
          st_status(p.status + tile, tile_kept, epoch_tag | (tile == 0 ? kFlagPrefix : kFlagAgg));
        ps.agg[s] = tile_kept;
        mbar_arrive(&ps.aggr[s]);
      }
      ++npend;
      if (npend > LAG) {
        if (!emit_one()) {
          ok = false;
          break;
        }
        --npend;
      }
    }
    if (ok) {
      while (npend > 0) {
        if (!emit_one()) break;
        --npend;
      }
    }
    consumers_finish(p, ps, it, rr);
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

// ------------------------------------------------------------------ host

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}

template <class P, int NC, int ITEMS, bool WIDE>
int launch_shape(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, cudaStream_t st) {
  auto kfn = scan_tma_kernel<P, NC, ITEMS, WIDE>;
  const size_t smem = (size_t)p.stages * NC * ITEMS * sizeof(typename P::In) + 1024;
  int rc = ensure_dynamic_smem((const void *)kfn, smem);
  if (rc) return rc;
  const int threads = NC + 32 * kLookWarps + 32;
  if (occupancy((const void *)kfn, threads, smem) < 1) return B2P_ERR_UNSUPPORTED;
  const int grid = (int)std::min<long long>(p.ntiles, (long long)device_info().sm_count);
  kfn<<<grid, threads, smem, st>>>(tin, tout, p);
  return cuda_status(cudaGetLastError());
}

template <class P, bool WIDE>
int launch_policy(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, int block, int items,
                  cudaStream_t st) {
  if (block == 128 && items == 32) return launch_shape<P, 128, 32, WIDE>(p, tin, tout, st);
  if (block == 256 && items == 16) return launch_shape<P, 256, 16, WIDE>(p, tin, tout, st);
  if (block == 256 && items == 32) return launch_shape<P, 256, 32, WIDE>(p, tin, tout, st);
  if (block == 512 && items == 16) return launch_shape<P, 512, 16, WIDE>(p, tin, tout, st);
  return B2P_ERR_UNSUPPORTED;
}

template <class P>
int launch_t(int inclusive, const void *in, void *out, size_t n, const void *init, void *scratch,
             int block, int items, cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  const size_t es = sizeof(In);
  const long long tile = (long long)block * items;
  const size_t stage = (size_t)tile * es;
  const int stages = (int)std::min<size_t>(kMaxStages, kStageBudget / stage);
  if (stages < 3) return B2P_ERR_UNSUPPORTED;
  TmaParams p{};
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  const long long epr = 128 / (long long)es;
  p.rows_full = (long long)(n / (size_t)epr);
  p.tail_begin = (unsigned long long)p.rows_full * epr;
  if (p.rows_full + tile / epr >= (1ll << 31)) return B2P_ERR_UNSUPPORTED;
  p.inclusive = inclusive;
  p.stages = stages;
  p.lag = std::max(1, std::min(kMaxLag, stages - 3));
  p.in = in;
  p.out = out;
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix);
  p.timeout_ns = wait_timeout_ns();
  p.stall_tile = debug_stall_tile();
  const bool wide = P::kCompensated && n > (1ull << 24);
  p.has_init = init != nullptr;
  if (init) memcpy(&p.init_raw, init, sizeof(Out));
  CUtensorMap tin, tout;
  const int box = (int)std::min<long long>(256, tile / epr);
  if (!encode_row_tensor(&tin, in, (unsigned long long)p.rows_full, box) ||
      !encode_row_tensor(&tout, out, (unsigned long long)p.rows_full, box))
    return B2P_ERR_UNSUPPORTED;
  if constexpr (P::kCompensated) {
    if (wide) return launch_policy<P, true>(p, tin, tout, block, items, st);
  }
  return launch_policy<P, false>(p, tin, tout, block, items, st);
}

template <int DT>
int dispatch(int op, int inclusive, const void *in, void *out, size_t n, const void *init, void *scratch,
             int block, int items, cudaStream_t st) {
#define B2P_TMA_CASE(OP) \
  case OP:               \
    return launch_t<typename PolicyOf<DT, OP>::type>(inclusive, in, out, n, init, scratch, block, items, st);
  switch (op) {
    B2P_TMA_CASE(B2P_SUM)
    B2P_TMA_CASE(B2P_PROD)
    B2P_TMA_CASE(B2P_MIN)
    B2P_TMA_CASE(B2P_MAX)
  default: break;
  }
  if constexpr (DT == B2P_F32 || DT == B2P_F64) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    switch (op) {
      B2P_TMA_CASE(B2P_AND)
      B2P_TMA_CASE(B2P_OR)
      B2P_TMA_CASE(B2P_XOR)
    default: return B2P_ERR_UNSUPPORTED;
    }
  }
#undef B2P_TMA_CASE
}

template <class T, int NC, int ITEMS>
int launch_copy_shape(TmaParams &p, const CUtensorMap &tin, cudaStream_t st) {
  auto kfn = copy_if_tma_kernel<T, NC, ITEMS>;
  const size_t smem = (size_t)p.stages * ((size_t)NC * ITEMS * sizeof(T) + 1024) + 1024;
  int rc = ensure_dynamic_smem((const void *)kfn, smem);
  if (rc) return rc;
  const int threads = NC + 32 * kLookWarps + 32;
  if (occupancy((const void *)kfn, threads, smem) < 1) return B2P_ERR_UNSUPPORTED;
  const int grid = (int)std::min<long long>(p.ntiles, (long long)device_info().sm_count);
  kfn<<<grid, threads, smem, st>>>(tin, p);
  return cuda_status(cudaGetLastError());
}

template <class T>
int launch_copy_t(const void *in, void *out, size_t n, uint64_t mask, int cmp, uint64_t rhs, uint64_t *num_copied,
                  void *scratch, int block, int items, cudaStream_t st) {
  const size_t es = sizeof(T);
  const long long tile = (long long)block * items;
  const size_t stride = (size_t)tile * es + 1024;
  const int stages = (int)std::min<size_t>(kMaxStages, kStageBudget / stride);
  if (stages < 3) return B2P_ERR_UNSUPPORTED;
  TmaParams p{};
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  const long long epr = 128 / (long long)es;
  p.rows_full = (long long)(n / (size_t)epr);
  p.tail_begin = (unsigned long long)p.rows_full * epr;
  if (p.rows_full + tile / epr >= (1ll << 31)) return B2P_ERR_UNSUPPORTED;
  p.stages = stages;
  p.lag = std::max(1, std::min(kMaxLag, stages - 3));
  p.in = in;
  p.out = out;
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix);
  p.timeout_ns = wait_timeout_ns();
  p.stall_tile = debug_stall_tile();
  p.mask = mask;
  p.rhs = rhs;
  p.cmp = cmp;
  p.num_copied = reinterpret_cast<unsigned long long *>(num_copied);
  CUtensorMap tin;
  if (!encode_row_tensor(&tin, in, (unsigned long long)p.rows_full, (int)std::min<long long>(256, tile / epr)))
    return B2P_ERR_UNSUPPORTED;
  if (block == 128 && items == 32) return launch_copy_shape<T, 128, 32>(p, tin, st);
  if (block == 256 && items == 16) return launch_copy_shape<T, 256, 16>(p, tin, st);
  if (block == 256 && items == 32) return launch_copy_shape<T, 256, 32>(p, tin, st);
  if (block == 512 && items == 16) return launch_copy_shape<T, 512, 16>(p, tin, st);
  return B2P_ERR_UNSUPPORTED;
}

}  // namespace

bool encode_row_tensor(CUtensorMap *map, const void *base, unsigned long long rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || !base || (reinterpret_cast<uintptr_t>(base) & 15) || rows < 1 || rows >= (1ull << 31) ||
      box_rows < 1 || box_rows > 256)
    return false;
  const cuuint64_t dims[2] = {128, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {128};
  const cuuint32_t box[2] = {128, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool scan_tma_shape(int dtype, int block, int items) {
  if (dtype == B2P_BF16 || dtype_size(dtype) == 0) return false;
  const bool shape = (block == 128 && items == 32) || (block == 256 && items == 16) ||
                     (block == 256 && items == 32) || (block == 512 && items == 16);
  return shape && (size_t)block * items * dtype_size(dtype) * 3 <= kStageBudget;
}

int launch_scan_tma(int dtype, int op, int inclusive, const void *in, void *out, size_t n, const void *init,
                    void *scratch, int block, int items, cudaStream_t st) {
  if (!scan_tma_shape(dtype, block, items)) return B2P_ERR_UNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(in) & 15) || (reinterpret_cast<uintptr_t>(out) & 15) ||
      (reinterpret_cast<uintptr_t>(scratch) & 255))
    return B2P_ERR_UNSUPPORTED;
  if (n < (size_t)block * items) return B2P_ERR_UNSUPPORTED;  // at least one full tile
  switch (dtype) {
  case B2P_I32: return dispatch<B2P_I32>(op, inclusive, in, out, n, init, scratch, block, items, st);
  case B2P_I64: return dispatch<B2P_I64>(op, inclusive, in, out, n, init, scratch, block, items, st);
  case B2P_U32: return dispatch<B2P_U32>(op, inclusive, in, out, n, init, scratch, block, items, st);
  case B2P_U64: return dispatch<B2P_U64>(op, inclusive, in, out, n, init, scratch, block, items, st);
  case B2P_F32: return dispatch<B2P_F32>(op, inclusive, in, out, n, init, scratch, block, items, st);
  case B2P_F64: return dispatch<B2P_F64>(op, inclusive, in, out, n, init, scratch, block, items, st);
  default: return B2P_ERR_UNSUPPORTED;
  }
}

bool copy_if_tma_shape(int dtype, int block, int items) {
  const size_t es = dtype_size(dtype);
  if (es != 4 && es != 8) return false;
  const bool shape = (block == 128 && items == 32) || (block == 256 && items == 16) ||
                     (block == 256 && items == 32) || (block == 512 && items == 16);
  return shape && ((size_t)block * items * es + 1024) * 3 <= kStageBudget;
}

int launch_copy_if_tma(int dtype, const void *in, void *out, size_t n, uint64_t mask, int cmp, uint64_t rhs,
                       uint64_t *num_copied, void *scratch, int block, int items, cudaStream_t st) {
  if (!copy_if_tma_shape(dtype, block, items)) return B2P_ERR_UNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(in) & 15) || (reinterpret_cast<uintptr_t>(scratch) & 255))
    return B2P_ERR_UNSUPPORTED;
  if (n < (size_t)block * items) return B2P_ERR_UNSUPPORTED;
  if (dtype_size(dtype) == 4)
    return launch_copy_t<uint32_t>(in, out, n, mask, cmp, rhs, num_copied, scratch, block, items, st);
  return launch_copy_t<unsigned long long>(in, out, n, mask, cmp, rhs, num_copied, scratch, block, items, st);
}

}  // namespace b2p
