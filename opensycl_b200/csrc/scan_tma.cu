// Pipelined single-pass scan and copy_if: grid mode 1 for scans whose
// element and output sizes match (every dtype but bf16) and for copy_if.
//
// Same algorithm as the reference's decoupled look-back scan
// (algorithms/scan/decoupled_lookback_scan.hpp:555-655: per-tile aggregate,
// look-back over predecessors' aggregates/prefixes, then the tile's scan
// from its carry), arranged for B200 as one persistent block per SM in which
// every step has its own warps, joined by mbarriers on a ring of shared
// stages:
//
//   producer warp    dynamic tile ids in order; TMA 2-D bulk tensor loads of
//                    each tile into the next free stage (128-byte swizzle)
//   reducer warps    as soon as a tile lands: per-thread totals, block scan,
//                    the thread prefixes kept beside the stage, the tile
//                    aggregate published at once -- never waiting for carries
//   look-back warps  two warps resolve the carries of reduced tiles in
//                    parallel (bounded warp-parallel look-back over
//                    epoch-tagged 128-bit status words)
//   emitter warps    as soon as a carry is known: the tile's outputs written
//                    in place into its stage
//   store warp       TMA bulk store of each emitted stage, then frees it
//
// A tile occupies a stage from its load to the end of its store; the
// reducers run ahead of the emitters by as many tiles as the look-back
// latency needs, bounded only by the number of stages.  Elements after the
// last complete 128-byte row use plain loads and stores.  Every wait is
// bounded; a wait that runs out records B2P_ERR_TIMEOUT in the scratch
// header and the block leaves its loops.
#include "b2p_device/copy_if.cuh"
#include "internal.h"

#include <algorithm>
#include <mutex>

namespace b2p {

namespace {

// ------------------------------------------------------------------- scan

template <class P, int NC, int ITEMS, bool WIDE>
__global__ void __launch_bounds__(pipe_threads(NC), 1)
    scan_tma_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
                    TmaParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Ops = typename std::conditional<WIDE, F64Ops, AccOps<P>>::type;
  static_assert(sizeof(Out) == sizeof(In) || sizeof(Out) == 2 * sizeof(In), "output tile layout");
  constexpr int kTile = NC * ITEMS;
  constexpr int kEpr = 128 / (int)sizeof(In);      // input elements per 128-byte row
  constexpr int kEprOut = 128 / (int)sizeof(Out);  // output elements per 128-byte row
  static_assert(kTile % (8 * kEpr) == 0 && kTile % (8 * kEprOut) == 0,
                "input and output tiles are whole numbers of 1024-byte swizzle atoms");
  constexpr int kRows = kTile / kEpr, kRowsOut = kTile / kEprOut;
  constexpr int kBox = kRows < 256 ? kRows : 256, kBoxOut = kRowsOut < 256 ? kRowsOut : 256;
  static_assert(kRows % kBox == 0 && kRowsOut % kBoxOut == 0, "box rows");
  // fp32 and bf16-input SUM keep compensated runs in the output tile
  constexpr bool kFast = std::is_same<P, FloatSumPolicy<float>>::value || std::is_same<P, FloatSumPolicy<uint16_t>>::value;

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // thread prefixes of every stage, after the stages
  Acc *texcl_all = reinterpret_cast<Acc *>(smem + (size_t)p.stages * p.stage_stride);
  __shared__ __align__(8) PipeState ps;
  __shared__ Acc s_warp[32];

  pipe_init(ps, p);
  __syncthreads();
  const unsigned long long epoch = ps.epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const unsigned long long init_bits = tile0_carry<P, WIDE>(p);
  const int warp = threadIdx.x >> 5;
  const int S = p.stages;
  const long long last = p.ntiles - 1;
  const int ntail = (int)(p.n - p.tail_begin);
  const int ntail_out = (int)(p.n - p.tail_out_begin);

  if (warp < NC / 32) {
    // ------------------------------------------------------------ reducers
    const int t = threadIdx.x;
    long long it = 0;
    RingPos r;
    for (;; ++it, r.advance(1, S)) {
      const int s = r.s;
      if (!mbar_wait(&ps.full[s], r.ph, p.timeout_ns)) {
        if (t == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        break;
      }
      const long long tile = ps.tile[s];
      if (tile < 0) break;
      char *buf = smem + (size_t)s * p.stage_stride;
      if (tile == last && ntail > 0) load_row_tail<In, NC>(p, buf, tile, kTile);
      Acc agg;
      if constexpr (kFast)
        agg = p.inclusive ? thread_runs<In, ITEMS, true>(buf, buf + p.out_offset, t)
                          : thread_runs<In, ITEMS, false>(buf, buf + p.out_offset, t);
      else agg = thread_total_t<P, ITEMS>(buf, t);
      Acc tile_agg;
      texcl_all[(size_t)s * NC + t] = group_exclusive_scan<AccOps<P>, NC>(agg, s_warp, &tile_agg, t, 1);
      bar_named(1, NC);  // every thread prefix (and fp32 run) is in place
      if (t == 0) {
        const unsigned long long bits = publish_value<P, WIDE>(tile_agg);
        if (tile != p.stall_tile) {
          if (tile == 0)
            st_status(p.status, Ops::pack(Ops::combine(Ops::unpack(init_bits), Ops::unpack(bits))),
                      epoch_tag | kFlagPrefix);
          else
            st_status(p.status + tile, bits, epoch_tag | kFlagAgg);
        }
        ps.agg[s] = bits;
        mbar_arrive(&ps.aggr[s]);  // releases the thread prefixes and the in-place runs too
      }
    }
    if (t == 0) *reinterpret_cast<volatile long long *>(&ps.end_item) = it;
  } else if (warp < 2 * NC / 32) {
    // ------------------------------------------------------------ emitters
    const int t = threadIdx.x - NC;
    Out *out = reinterpret_cast<Out *>(p.out);
    RingPos r;
    for (long long it = 0;; ++it, r.advance(1, S)) {
      const int w = emitter_wait(p, ps, r, it);
      if (w <= 0) {
        if (w < 0 && t == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        if (w == 0 && t == 0) emitters_finish(p, ps, r);
        break;
      }
      const int s = r.s;
      const long long tile = ps.tile[s];
      char *buf = smem + (size_t)s * p.stage_stride;
      char *obuf = buf + p.out_offset;
      const Acc start = start_value<P, WIDE>(ps.carry[s], texcl_all[(size_t)s * NC + t]);
      if constexpr (kFast) emit_f32_runs<ITEMS>(obuf, start, t);
      else emit_generic<P, ITEMS>(buf, obuf, start, p.inclusive != 0, t);
      fence_async_smem();
      bar_named(2, NC);
      if (tile == last && ntail_out > 0) {
        const long long j0 = (long long)p.tail_out_begin - tile * kTile;
        if (t < ntail_out) out[p.tail_out_begin + t] = *smem_elem_ptr<Out>(obuf, (int)j0 + t);
        bar_named(2, NC);
      }
      if (t == 0) mbar_arrive(&ps.emitted[s]);
    }
  } else if (warp < 2 * NC / 32 + kLookWarps) {
    lookback_loop<Ops>(p, ps, warp - 2 * NC / 32, init_bits, epoch_tag, S);
  } else if (warp == 2 * NC / 32 + kLookWarps) {
    if ((threadIdx.x & 31) == 0) producer_loop(&tin, p, ps, smem, kRows, kBox, ps.tile);
  } else {
    // ---------------------------------------------------------- store warp
    if ((threadIdx.x & 31) == 0) {
      prefetch_tensormap(&tout);
      const unsigned long long spol = l2_policy_stream();
      RingPos r;
      StoreRelease<> rel;
      for (long long it = 0;; ++it, r.advance(1, S)) {
        const int s = r.s;
        if (!mbar_wait(&ps.emitted[s], r.ph, p.timeout_ns)) {
          record_error(p.hdr, B2P_ERR_TIMEOUT);
          break;
        }
        if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
        const long long tile = ps.tile[s];
        const long long r0 = tile * kRowsOut;
        const long long rows_out = min((long long)kRowsOut, p.rows_full_out - r0);
        for (long long rr = 0; rr < rows_out; rr += kBoxOut)
          tma_store_2d(&tout, 0, (int)(r0 + rr), smem + (size_t)s * p.stage_stride + p.out_offset + rr * 128, spol);
        bulk_commit();
        rel.committed(ps.empty, S);
      }
      rel.drain(ps.empty, S);
      bulk_wait_all();
    }
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

// ------------------------------------------------------ scan, TMEM-staged
//
// The same roles as scan_tma_kernel, with a third place for a tile to wait:
// reducers read a landed tile into registers, hand the input stage straight
// back to the producer, and park the tile's running values in a TMEM slot
// (32-bit cells: thread t of the reducer group owns lane 32 (w % 4) + t % 32
// of its warp w and kCols consecutive columns of the slot).  Emitters take a
// slot once its carry is known, add the carry and write the outputs into a
// separate output stage for the store warp.  Shared memory then only holds
// tiles on their way in and out, while up to 512 / kSlotCols tiles wait for
// their carries in TMEM.

// Reducer pass: the thread's ITEMS elements from the landed stage, their
// running values from the identity (inclusive: after adding the element,
// exclusive: before) as 32-bit words for TMEM, and the thread total.
// Compensated sums (fp32 / bf16) run in FP64: the thread's values are exact
// in FP64 and their sum far inside its precision, each parked word is one
// rounding of the running value, and the total leaves as the double-float
// (hi, lo) split of the FP64 sum.
template <class P, int ITEMS, bool INCL>
__device__ __forceinline__ typename P::Acc tmem_runs(const char *inbuf, uint32_t *w, int t) {
  using In = typename P::In;
  using Out = typename P::Out;
  constexpr int IPV = 16 / (int)sizeof(In), VPT = ITEMS / IPV, WPO = (int)sizeof(Out) / 4;
  if constexpr (P::kCompensated) {
    double rd = 0.0;
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      const uint4 u = *reinterpret_cast<const uint4 *>(inbuf + swz(t * VPT + k) * 16);
      const In *e = reinterpret_cast<const In *>(&u);
#pragma unroll
      for (int q = 0; q < IPV; ++q) {
        const double x = (double)P::lift_f(e[q]);
        const Out o = (Out)(INCL ? rd + x : rd);
        rd += x;
        memcpy(w + (k * IPV + q) * WPO, &o, sizeof(Out));
      }
    }
    const float h = (float)rd;
    return typename P::Acc{h, (float)(rd - (double)h)};
  } else {
    typename P::Acc run = P::identity();
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      const uint4 u = *reinterpret_cast<const uint4 *>(inbuf + swz(t * VPT + k) * 16);
      const In *e = reinterpret_cast<const In *>(&u);
#pragma unroll
      for (int q = 0; q < IPV; ++q) {
        Out o;
        if constexpr (INCL) {
          P::add(run, e[q]);
          o = P::finalize(run);
        } else {
          o = P::finalize(run);
          P::add(run, e[q]);
        }
        memcpy(w + (k * IPV + q) * WPO, &o, sizeof(Out));
      }
    }
    return run;
  }
}

// Emitter pass: outputs = start combined with the parked running values,
// written to the output stage in the swizzled layout.
template <class P, int ITEMS>
__device__ __forceinline__ void tmem_emit(const uint32_t *w, typename P::Acc start, char *obuf, int t) {
  using Out = typename P::Out;
  constexpr int OPV = 16 / (int)sizeof(Out), VPT = ITEMS / OPV, WPO = (int)sizeof(Out) / 4;
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    uint4 u;
    Out *oe = reinterpret_cast<Out *>(&u);
#pragma unroll
    for (int q = 0; q < OPV; ++q) {
      Out r;
      memcpy(&r, w + (k * OPV + q) * WPO, sizeof(Out));
      if constexpr (P::kCompensated) oe[q] = __fadd_rn(start.hi, __fadd_rn(start.lo, r));
      else oe[q] = P::finalize(P::combine(start, P::from_out(r)));
    }
    *reinterpret_cast<uint4 *>(obuf + swz(t * VPT + k) * 16) = u;
  }
}

// Combination of the reducers' per-thread totals inside a tile, done off
// the reducers' path: the aggregator warp forms the tile total, the emitters
// the threads' exclusive prefixes.  Compensated sums combine in FP64 (a
// normalised double-float total converts to double exactly, and a tile's
// 256 double additions stay far below the sums' error bound); other
// policies combine their own accumulator.
template <class P>
struct TileOps {
  static constexpr bool kF64 = P::kCompensated;
  using Acc = typename P::Acc;
  using Pub = typename std::conditional<kF64, double, Acc>::type;
  __device__ static Pub identity() {
    if constexpr (kF64) return 0.0;
    else return P::identity();
  }
  __device__ static Pub combine(Pub a, Pub b) {
    if constexpr (kF64) return a + b;
    else return P::combine(a, b);
  }
  __device__ static Pub from(Acc a) {
    if constexpr (kF64) return (double)a.hi + (double)a.lo;
    else return a;
  }
  __device__ static Acc to_acc(Pub v) {
    if constexpr (kF64) {
      const float h = (float)v;
      return DF{h, (float)(v - (double)h)};
    } else {
      return v;
    }
  }
};

// Aggregator warp of the TMEM-staged scan, item by item: wait until every
// reducer warp has parked the tile (slot_ready: one arrival per reducer
// warp), sum the tile's NC thread totals, publish the aggregate (tile 0: its
// inclusive prefix) and hand it to the look-back warps (aggr).  Aggregates go
// out in tile order as soon as tiles are parked, whatever the look-backs are
// waiting for.  Ends when the reducers have published the item count and it
// has handled that many items.
template <class P, class Ops, int NC, bool WIDE>
__device__ __forceinline__ void scan_aggregator_loop(const TmaParams &p, PipeState &ps,
                                                     const typename P::Acc *aggs_all,
                                                     unsigned long long init_bits, unsigned long long epoch_tag,
                                                     int S) {
  using TO = TileOps<P>;
  using V = typename TO::Pub;
  const int lane = threadIdx.x & 31;
  RingPos r;
  for (long long it = 0;; ++it, r.advance(1, S)) {
    const int s = r.s;
    int go = 0;
    if (lane == 0) {
      uint64_t t0 = 0;
      for (unsigned k = 0;; ++k) {
        if (mbar_try_hint(&ps.slot_ready[s], r.ph, 2000)) {
          go = 1;
          break;
        }
        if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
        if ((k & 7) == 7) {
          const uint64_t now = globaltimer_ns();
          if (t0 == 0) {
            t0 = now;
          } else if (now - t0 > p.timeout_ns) {
            record_error(p.hdr, B2P_ERR_TIMEOUT);
            go = -1;
            break;
          }
        }
      }
    }
    go = __shfl_sync(0xffffffffu, go, 0);
    if (go <= 0) return;
    (void)mbar_try(&ps.slot_ready[s], r.ph);  // completed: this lane's acquire of the parked totals
    const long long tile = ps.tile[s];
    // the tile total: NC / 32 totals per lane, then a shuffle tree
    V v = TO::identity();
#pragma unroll
    for (int k = 0; k < NC / 32; ++k) v = TO::combine(v, TO::from(aggs_all[(size_t)s * NC + k * 32 + lane]));
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v = TO::combine(v, shfl_xor(v, m));
    if (lane == 0) {
      unsigned long long bits;
      if constexpr (WIDE) bits = F64Ops::pack(v);
      else bits = publish_value<P, WIDE>(TO::to_acc(v));
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
    __syncwarp();
  }
}

// Threads of the TMEM-staged scan: the pipeline's roles plus the aggregator.
constexpr int scan_tmem_threads(int nc) { return pipe_threads(nc) + 32; }

template <class P, int NC, int ITEMS, bool WIDE>
__global__ void __launch_bounds__(scan_tmem_threads(NC), 1)
    scan_tmem_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
                     TmaParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Ops = typename std::conditional<WIDE, F64Ops, AccOps<P>>::type;
  constexpr int kTile = NC * ITEMS;
  constexpr int kEpr = 128 / (int)sizeof(In), kEprOut = 128 / (int)sizeof(Out);
  static_assert(kTile % (8 * kEpr) == 0 && kTile % (8 * kEprOut) == 0,
                "input and output tiles are whole numbers of 1024-byte swizzle atoms");
  constexpr int kRows = kTile / kEpr, kRowsOut = kTile / kEprOut;
  constexpr int kBox = kRows < 256 ? kRows : 256, kBoxOut = kRowsOut < 256 ? kRowsOut : 256;
  static_assert(kRows % kBox == 0 && kRowsOut % kBoxOut == 0, "box rows");
  constexpr int kCols = tmem_cols<P, ITEMS>();
  static_assert(kCols == 16 || kCols == 32, "TMEM columns per thread");
  static_assert(NC % 128 == 0, "reducer and emitter groups cover the four TMEM lane quarters evenly");
  constexpr int kSlotCols = kCols * (NC / 128);

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  char *obase = smem + p.out_base;
  Acc *aggs_all = reinterpret_cast<Acc *>(smem + p.texcl_base);  // per slot: each reducer thread's total
  __shared__ __align__(8) PipeState ps;
  __shared__ typename TileOps<P>::Pub s_warp[32];
  __shared__ int s_go[2];

  const int warp = threadIdx.x >> 5;
  tmem_pipe_init(ps, p, NC / 32);
  if (warp == 0) {
    __syncwarp();
    tmem_alloc(&ps.tmem_base, 512);
  }
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tbase = ps.tmem_base;
  const unsigned long long epoch = ps.epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const unsigned long long init_bits = tile0_carry<P, WIDE>(p);
  const int SI = p.stages, SL = p.slots, SO = p.out_stages;
  const long long last = p.ntiles - 1;
  const int ntail = (int)(p.n - p.tail_begin);
  const int ntail_out = (int)(p.n - p.tail_out_begin);

  if (warp < NC / 32) {
    // ------------------------------------------------------------ reducers
    // The group leader waits (bounded) and shares the outcome, so that the
    // group always takes the same branch.
    const int t = threadIdx.x;
    const uint32_t tcol = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * kCols);
    long long it = 0;
    RingPos ri, rs;
    for (;; ++it, ri.advance(1, SI), rs.advance(1, SL)) {
      if (t == 0) {
        int go = mbar_wait(&ps.full[ri.s], ri.ph, p.timeout_ns) ? 1 : -1;
        if (go > 0 && ps.tile_in[ri.s] < 0) go = 0;
        if (go > 0 && !mbar_wait(&ps.slot_free[rs.s], rs.ph ^ 1u, p.timeout_ns)) go = -1;
        if (go < 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        s_go[0] = go;
      }
      bar_named(1, NC);
      if (s_go[0] <= 0) break;
      (void)mbar_try(&ps.full[ri.s], ri.ph);  // completed: this thread's acquire of the TMA bytes
      tmem_fence_after();
      const long long tile = ps.tile_in[ri.s];
      char *buf = smem + (size_t)ri.s * p.stage_stride;
      if (tile == last && ntail > 0) load_row_tail<In, NC>(p, buf, tile, kTile);
      uint32_t w[kCols];
      const Acc agg = p.inclusive ? tmem_runs<P, ITEMS, true>(buf, w, t) : tmem_runs<P, ITEMS, false>(buf, w, t);
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.empty[ri.s]);  // this warp is done with the input stage
      const uint32_t ta = tcol + (uint32_t)(rs.s * kSlotCols);
      tmem_st16(ta, w);
      if constexpr (kCols == 32) tmem_st16(ta + 16, w + 16);
      // the tile total and the threads' prefixes are formed by the aggregator
      // warp and the emitters: the reducers only park the thread totals
      aggs_all[(size_t)rs.s * NC + t] = agg;
      if (t == 0) ps.tile[rs.s] = tile;
      tmem_wait_st();
      tmem_fence_before();
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.slot_ready[rs.s]);  // this warp's slot columns and totals
    }
    if (t == 0) *reinterpret_cast<volatile long long *>(&ps.end_item) = it;
  } else if (warp < 2 * NC / 32) {
    // ------------------------------------------------------------ emitters
    const int t = threadIdx.x - NC;
    const uint32_t tcol = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(((t >> 5) >> 2) * kCols);
    Out *out = reinterpret_cast<Out *>(p.out);
    RingPos rs, ro;
    for (long long it = 0;; ++it, rs.advance(1, SL), ro.advance(1, SO)) {
      if (t == 0) {
        // the carry is ready only after every reducer warp parked the tile
        int go = emitter_wait(p, ps, rs, it);
        if (go > 0 && !mbar_wait(&ps.out_empty[ro.s], ro.ph ^ 1u, p.timeout_ns)) go = -1;
        if (go < 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        if (go == 0) {
          // every earlier item passed the look-back warps and the store warp:
          // end them (look-back warps wait on items it .. it + kLookWarps - 1)
          mbar_arrive(&ps.emitted[ro.s]);
          RingPos r = rs;
          for (int j = 0; j < kLookWarps; ++j, r.advance(1, SL)) mbar_arrive(&ps.aggr[r.s]);
        }
        s_go[1] = go;
      }
      bar_named(2, NC);
      if (s_go[1] <= 0) break;
      tmem_fence_after();
      const long long tile = ps.tile[rs.s];
      uint32_t w[kCols];
      const uint32_t ta = tcol + (uint32_t)(rs.s * kSlotCols);
      if constexpr (kCols == 32) tmem_load32(ta, w);
      else tmem_load16(ta, w);
      using TO = TileOps<P>;
      typename TO::Pub tile_total;
      const typename TO::Pub ex =
          group_exclusive_scan_1bar<TO, NC>(TO::from(aggs_all[(size_t)rs.s * NC + t]), s_warp, &tile_total, t, 2);
      Acc start;
      if constexpr (WIDE && TO::kF64) start = TO::to_acc(F64Ops::unpack(ps.carry[rs.s]) + ex);
      else start = start_value<P, WIDE>(ps.carry[rs.s], TO::to_acc(ex));
      tmem_fence_before();
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.slot_free[rs.s]);  // slot, carry and prefixes read
      char *obuf = obase + (size_t)ro.s * p.out_stage_stride;
      tmem_emit<P, ITEMS>(w, start, obuf, t);
      fence_async_smem();
      bar_named(2, NC);
      if (tile == last && ntail_out > 0) {
        const long long j0 = (long long)p.tail_out_begin - tile * kTile;
        if (t < ntail_out) out[p.tail_out_begin + t] = *smem_elem_ptr<Out>(obuf, (int)j0 + t);
        bar_named(2, NC);
      }
      if (t == 0) {
        ps.tile_out[ro.s] = tile;
        mbar_arrive(&ps.emitted[ro.s]);
      }
    }
  } else if (warp < 2 * NC / 32 + kLookWarps) {
    lookback_loop<Ops>(p, ps, warp - 2 * NC / 32, init_bits, epoch_tag, SL);
  } else if (warp == 2 * NC / 32 + kLookWarps) {
    if ((threadIdx.x & 31) == 0) producer_loop(&tin, p, ps, smem, kRows, kBox, ps.tile_in);
  } else if (warp == 2 * NC / 32 + kLookWarps + 2) {
    scan_aggregator_loop<P, Ops, NC, WIDE>(p, ps, aggs_all, init_bits, epoch_tag, SL);
  } else {
    // ---------------------------------------------------------- store warp
    if ((threadIdx.x & 31) == 0) {
      prefetch_tensormap(&tout);
      const unsigned long long spol = l2_policy_stream();
      RingPos ro;
      StoreRelease<kTmemStoresInFlight> rel;
      for (long long it = 0;; ++it, ro.advance(1, SO)) {
        if (!mbar_wait(&ps.emitted[ro.s], ro.ph, p.timeout_ns)) {
          record_error(p.hdr, B2P_ERR_TIMEOUT);
          break;
        }
        if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
        const long long tile = ps.tile_out[ro.s];
        const long long r0 = tile * kRowsOut;
        const long long rows_out = min((long long)kRowsOut, p.rows_full_out - r0);
        const char *src = obase + (size_t)ro.s * p.out_stage_stride;
        for (long long rr = 0; rr < rows_out; rr += kBoxOut) tma_store_2d(&tout, 0, (int)(r0 + rr), src + rr * 128, spol);
        bulk_commit();
        rel.committed(ps.out_empty, SO);
      }
      rel.drain(ps.out_empty, SO);
      bulk_wait_all();
    }
  }
  tmem_fence_before();
  __syncthreads();
  if (warp == 0) {
    tmem_fence_after();
    tmem_dealloc(tbase, 512);
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

// ---------------------------------------------------------------- copy_if

// Order-preserving compaction on the same pipeline.  A tile's aggregate is
// its kept count; its carry is the output position of its first kept
// element.  The emitters pack the kept elements, in order, into the stage
// with the output's 16-byte phase and write the unaligned ends with plain
// stores; the store warp writes the 16-byte-aligned middle with one bulk
// copy.  Stages are 1024 bytes longer than a tile: packing may shift it by
// up to 15 bytes.
template <class T, int NC, int ITEMS, int CMP>
__global__ void __launch_bounds__(pipe_threads(NC), 1)
    copy_if_tma_kernel(const __grid_constant__ CUtensorMap tin, TmaParams p) {
  constexpr int kTile = NC * ITEMS;
  constexpr int kEpr = 128 / (int)sizeof(T);
  static_assert(kTile % (8 * kEpr) == 0, "a stage is a whole number of 1024-byte swizzle atoms");
  constexpr int kRows = kTile / kEpr;
  constexpr int kBox = kRows < 256 ? kRows : 256;
  static_assert(kRows % kBox == 0, "box rows");
  constexpr int EPV = 16 / (int)sizeof(T);
  constexpr int VPT = ITEMS / EPV;
  static_assert(ITEMS <= 32, "keep mask is 32 bits");

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned long long *texcl_all = reinterpret_cast<unsigned long long *>(smem + (size_t)p.stages * p.stage_stride);
  unsigned *keep_all = reinterpret_cast<unsigned *>(texcl_all + (size_t)p.stages * NC);
  __shared__ __align__(8) PipeState ps;
  __shared__ unsigned long long s_warp[32];

  pipe_init(ps, p);
  __syncthreads();
  const unsigned long long epoch = ps.epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const int warp = threadIdx.x >> 5;
  const int S = p.stages;
  const long long last = p.ntiles - 1;
  const int ntail = (int)(p.n - p.tail_begin);
  T *out = reinterpret_cast<T *>(p.out);

  using U = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
  const U mask = (U)p.mask, rhs = (U)p.rhs;
  // predicate bits of thread t's elements of a tile (the first `count`
  // elements of the tile are real); the comparison is a template argument
  auto flags = [&](const char *buf, int t, int count, int *kept) -> unsigned {
    const int first = t * ITEMS;
    unsigned keep = 0;
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
      const U *e = reinterpret_cast<const U *>(&w);
#pragma unroll
      for (int qq = 0; qq < EPV; ++qq) {
        const U a = e[qq] & mask;
        bool kb;
        if constexpr (CMP == B2P_CMP_LT) kb = a < rhs;
        else if constexpr (CMP == B2P_CMP_LE) kb = a <= rhs;
        else if constexpr (CMP == B2P_CMP_EQ) kb = a == rhs;
        else if constexpr (CMP == B2P_CMP_NE) kb = a != rhs;
        else if constexpr (CMP == B2P_CMP_GE) kb = a >= rhs;
        else kb = a > rhs;
        keep |= (unsigned)kb << (k * EPV + qq);
      }
    }
    if (count < first + ITEMS) keep &= count <= first ? 0u : ((1u << (count - first)) - 1u);  // count - first < 32 here
    *kept = __popc(keep);
    return keep;
  };

  if (warp < NC / 32) {
    // ------------------------------------------------------------ reducers
    const int t = threadIdx.x;
    long long it = 0;
    RingPos r;
    for (;; ++it, r.advance(1, S)) {
      const int s = r.s;
      if (!mbar_wait(&ps.full[s], r.ph, p.timeout_ns)) {
        if (t == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        break;
      }
      const long long tile = ps.tile[s];
      if (tile < 0) break;
      char *buf = smem + (size_t)s * p.stage_stride;
      if (tile == last && ntail > 0) load_row_tail<T, NC>(p, buf, tile, kTile);
      const int count = (int)min((unsigned long long)kTile, p.n - (unsigned long long)tile * kTile);
      int kept;
      keep_all[(size_t)s * NC + t] = flags(buf, t, count, &kept);
      unsigned long long tile_kept;
      texcl_all[(size_t)s * NC + t] =
          group_exclusive_scan<CountOps, NC>((unsigned long long)kept, s_warp, &tile_kept, t, 1);
      bar_named(1, NC);  // every thread prefix is in place
      if (t == 0) {
        if (tile != p.stall_tile)
          st_status(p.status + tile, tile_kept, epoch_tag | (tile == 0 ? kFlagPrefix : kFlagAgg));
        ps.agg[s] = tile_kept;
        mbar_arrive(&ps.aggr[s]);
      }
    }
    if (t == 0) *reinterpret_cast<volatile long long *>(&ps.end_item) = it;
  } else if (warp < 2 * NC / 32) {
    // ------------------------------------------------------------ emitters
    const int t = threadIdx.x - NC;
    RingPos r;
    for (long long it = 0;; ++it, r.advance(1, S)) {
      const int w = emitter_wait(p, ps, r, it);
      if (w <= 0) {
        if (w < 0 && t == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        if (w == 0 && t == 0) emitters_finish(p, ps, r);
        break;
      }
      const int s = r.s;
      const long long tile = ps.tile[s];
      char *buf = smem + (size_t)s * p.stage_stride;
      const unsigned long long carry = ps.carry[s];
      unsigned long long kept_total = ps.agg[s];
      if (carry > p.n || kept_total > p.n - carry) {  // only after a broken chain: write nothing
        if (t == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        kept_total = 0;
      }
      const unsigned keep = keep_all[(size_t)s * NC + t];
      uint4 v[VPT];
#pragma unroll
      for (int k = 0; k < VPT; ++k) v[k] = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
      bar_named(2, NC);  // every emitter holds its elements: the stage may be overwritten
      const uintptr_t g0 = reinterpret_cast<uintptr_t>(out + carry);
      const unsigned phase = (unsigned)(g0 & 15u);
      const unsigned o = (unsigned)texcl_all[(size_t)s * NC + t];
      const unsigned lim = (unsigned)kept_total;
#pragma unroll
      for (int k = 0; k < VPT; ++k) {
        const T *e = reinterpret_cast<const T *>(&v[k]);
#pragma unroll
        for (int qq = 0; qq < EPV; ++qq) {
          const int j = k * EPV + qq;
          const unsigned pos = o + __popc(keep & ((1u << j) - 1u));
          if (((keep >> j) & 1u) && pos < lim) *reinterpret_cast<T *>(buf + phase + pos * sizeof(T)) = e[qq];
        }
      }
      fence_async_smem();
      bar_named(2, NC);
      const uintptr_t g1 = g0 + kept_total * sizeof(T);
      const uintptr_t a0 = (g0 + 15) & ~uintptr_t(15), a1 = g1 & ~uintptr_t(15);
      const bool mid = a1 > a0;
      const long long nhead = mid ? (long long)((a0 - g0) / sizeof(T)) : (long long)kept_total;
      const long long tail0 = mid ? (long long)((a1 - g0) / sizeof(T)) : (long long)kept_total;
      const long long ntl = (long long)kept_total - tail0;
      if (t < nhead) out[carry + t] = *reinterpret_cast<const T *>(buf + phase + t * sizeof(T));
      if (t >= 32 && t - 32 < ntl) {
        const long long k = tail0 + (t - 32);
        out[carry + k] = *reinterpret_cast<const T *>(buf + phase + k * sizeof(T));
      }
      if (t == 0 && tile == last && p.num_copied) *p.num_copied = carry + kept_total;
      bar_named(2, NC);  // the plain stores are done with the stage
      if (t == 0) mbar_arrive(&ps.emitted[s]);
    }
  } else if (warp < 2 * NC / 32 + kLookWarps) {
    lookback_loop<CountOps>(p, ps, warp - 2 * NC / 32, 0ull, epoch_tag, S);
  } else if (warp == 2 * NC / 32 + kLookWarps) {
    if ((threadIdx.x & 31) == 0) producer_loop(&tin, p, ps, smem, kRows, kBox, ps.tile);
  } else {
    // ---------------------------------------------------------- store warp
    if ((threadIdx.x & 31) == 0) {
      RingPos r;
      StoreRelease<> rel;
      for (long long it = 0;; ++it, r.advance(1, S)) {
        const int s = r.s;
        if (!mbar_wait(&ps.emitted[s], r.ph, p.timeout_ns)) {
          record_error(p.hdr, B2P_ERR_TIMEOUT);
          break;
        }
        if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
        const unsigned long long carry = ps.carry[s];
        unsigned long long kept_total = ps.agg[s];
        if (carry > p.n || kept_total > p.n - carry) kept_total = 0;
        const uintptr_t g0 = reinterpret_cast<uintptr_t>(out + carry);
        const uintptr_t g1 = g0 + kept_total * sizeof(T);
        const uintptr_t a0 = (g0 + 15) & ~uintptr_t(15), a1 = g1 & ~uintptr_t(15);
        if (a1 > a0) {
          const char *src = smem + (size_t)s * p.stage_stride + (g0 & 15u) + (a0 - g0);
          asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(a0),
                       "r"(smem_u32(src)), "r"((unsigned)(a1 - a0))
                       : "memory");
        }
        bulk_commit();
        rel.committed(ps.empty, S);
      }
      rel.drain(ps.empty, S);
      bulk_wait_all();
    }
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

// ------------------------------------------------------------------ host
template <class P, int NC, int ITEMS, bool WIDE>
int launch_shape(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, cudaStream_t st) {
  auto kfn = scan_tma_kernel<P, NC, ITEMS, WIDE>;
  const size_t smem = (size_t)p.stages * (p.stage_stride + NC * sizeof(typename P::Acc)) + 1024;
  int rc = ensure_dynamic_smem((const void *)kfn, smem);
  if (rc) return rc;
  const int threads = pipe_threads(NC);
  if (occupancy((const void *)kfn, threads, smem) < 1) return B2P_ERR_UNSUPPORTED;
  const int grid = (int)std::min<long long>(p.ntiles, (long long)device_info().sm_count);
  kfn<<<grid, threads, smem, st>>>(tin, tout, p);
  return cuda_status(cudaGetLastError());
}

template <class P, int NC, int ITEMS, bool WIDE>
int launch_tmem_shape(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, cudaStream_t st) {
  constexpr int cols = tmem_cols<P, ITEMS>();
  if constexpr (!TmemExact<P>::value || (cols != 16 && cols != 32)) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    auto kfn = scan_tmem_kernel<P, NC, ITEMS, WIDE>;
    const size_t smem = p.texcl_base + (size_t)p.slots * NC * sizeof(typename P::Acc) + 1024;
    int rc = ensure_dynamic_smem((const void *)kfn, smem);
    if (rc) return rc;
    const int threads = scan_tmem_threads(NC);
    if (occupancy((const void *)kfn, threads, smem) < 1) return B2P_ERR_UNSUPPORTED;
    const int grid = (int)std::min<long long>(p.ntiles, (long long)device_info().sm_count);
    kfn<<<grid, threads, smem, st>>>(tin, tout, p);
    return cuda_status(cudaGetLastError());
  }
}

template <class P, bool WIDE>
int launch_tmem_policy(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, int block, int items,
                       cudaStream_t st) {
  if (block == 128 && items == 32) return launch_tmem_shape<P, 128, 32, WIDE>(p, tin, tout, st);
  if (block == 256 && items == 16) return launch_tmem_shape<P, 256, 16, WIDE>(p, tin, tout, st);
  if (block == 256 && items == 32) return launch_tmem_shape<P, 256, 32, WIDE>(p, tin, tout, st);
  return B2P_ERR_UNSUPPORTED;
}

// Shared-memory layout of the TMEM-staged kernel for (block, items): input
// stages, two output stages, thread prefixes of every slot; as many slots as
// 512 TMEM columns hold.  False when the policy or shape has no TMEM kernel.
template <class P>
bool tmem_layout(TmaParams &p, int block, int items) {
  constexpr size_t es = sizeof(typename P::In), eo = sizeof(typename P::Out);
  if (!kUseTmem || !TmemExact<P>::value || (block != 128 && block != 256)) return false;
  const int cols = items * (int)eo / 4;
  if (cols != 16 && cols != 32) return false;
  const int slots = std::min(kMaxStages, 512 / (cols * block / 128));
  const size_t in_b = (size_t)block * items * es, out_b = (size_t)block * items * eo;
  const size_t texcl = ((size_t)slots * block * sizeof(typename P::Acc) + 1023) & ~size_t(1023);
  const int so = kScanOutStages;
  if (so * out_b + texcl + 2 * in_b > kSmemBudget) return false;
  const int si = (int)std::min<size_t>(kScanMaxInStages, (kSmemBudget - so * out_b - texcl) / in_b);
  p.stages = si;
  p.stage_stride = (unsigned)in_b;
  p.slots = slots;
  p.out_stages = so;
  p.out_stage_stride = (unsigned)out_b;
  p.out_base = (unsigned)(si * in_b);
  p.texcl_base = (unsigned)(si * in_b + so * out_b);
  return true;
}

template <class P, bool WIDE>
int launch_policy(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, int block, int items,
                  cudaStream_t st) {
  if (block == 128 && items == 32) return launch_shape<P, 128, 32, WIDE>(p, tin, tout, st);
  if (block == 256 && items == 16) return launch_shape<P, 256, 16, WIDE>(p, tin, tout, st);
  if (block == 256 && items == 32) return launch_shape<P, 256, 32, WIDE>(p, tin, tout, st);
  return B2P_ERR_UNSUPPORTED;
}

template <class P>
int launch_t(int inclusive, const void *in, void *out, size_t n, const void *init, void *scratch,
             int block, int items, cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  const size_t es = sizeof(In), eo = sizeof(Out);
  const long long tile = (long long)block * items;
  // a stage holds the input tile, and after it the output tile when the
  // output element is wider (bf16 in, fp32 out)
  const size_t in_bytes = (size_t)tile * es;
  const size_t stage = in_bytes + (eo != es ? (size_t)tile * eo : 0);
  const int stages = (int)std::min<size_t>(kMaxStages, kSmemBudget / (stage + block * sizeof(typename P::Acc)));
  TmaParams p{};
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  const long long epr = 128 / (long long)es, epr_out = 128 / (long long)eo;
  p.rows_full = (long long)(n / (size_t)epr);
  p.tail_begin = (unsigned long long)p.rows_full * epr;
  p.rows_full_out = (long long)(n / (size_t)epr_out);
  p.tail_out_begin = (unsigned long long)p.rows_full_out * epr_out;
  if (p.rows_full_out + tile / epr_out >= (1ll << 31)) return B2P_ERR_UNSUPPORTED;
  p.out_offset = eo != es ? (unsigned)in_bytes : 0u;
  p.inclusive = inclusive;
  p.stages = stages;
  p.stage_stride = (unsigned)stage;
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
  if (!encode_row_tensor(&tin, in, (unsigned long long)p.rows_full, (int)std::min<long long>(256, tile / epr)) ||
      !encode_row_tensor(&tout, out, (unsigned long long)p.rows_full_out,
                         (int)std::min<long long>(256, tile / epr_out)))
    return B2P_ERR_UNSUPPORTED;
  if (tmem_layout<P>(p, block, items)) {
    if constexpr (P::kCompensated) {
      if (wide) return launch_tmem_policy<P, true>(p, tin, tout, block, items, st);
    }
    return launch_tmem_policy<P, false>(p, tin, tout, block, items, st);
  }
  if (stages < kMinStages) return B2P_ERR_UNSUPPORTED;
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
  if constexpr (DT == B2P_F32 || DT == B2P_F64 || DT == B2P_BF16) {
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

template <class T, int NC, int ITEMS, int CMP>
int launch_copy_shape(TmaParams &p, const CUtensorMap &tin, cudaStream_t st) {
  auto kfn = copy_if_tma_kernel<T, NC, ITEMS, CMP>;
  const size_t smem = (size_t)p.stages * (p.stage_stride + NC * (sizeof(unsigned long long) + 4)) + 1024;
  int rc = ensure_dynamic_smem((const void *)kfn, smem);
  if (rc) return rc;
  const int threads = pipe_threads(NC);
  if (occupancy((const void *)kfn, threads, smem) < 1) return B2P_ERR_UNSUPPORTED;
  const int grid = (int)std::min<long long>(p.ntiles, (long long)device_info().sm_count);
  kfn<<<grid, threads, smem, st>>>(tin, p);
  return cuda_status(cudaGetLastError());
}

template <class T, int NC, int ITEMS>
int launch_copy_items(TmaParams &p, const CUtensorMap &tin, cudaStream_t st) {
  if (p.slots > 0) {
    const int sms = device_info().sm_count;
    switch (p.cmp) {
    case B2P_CMP_LT: return launch_copy_tmem_shape<T, NC, ITEMS>(p, tin, MaskCmp<T, B2P_CMP_LT>{p.mask, p.rhs}, sms, st);
    case B2P_CMP_LE: return launch_copy_tmem_shape<T, NC, ITEMS>(p, tin, MaskCmp<T, B2P_CMP_LE>{p.mask, p.rhs}, sms, st);
    case B2P_CMP_EQ: return launch_copy_tmem_shape<T, NC, ITEMS>(p, tin, MaskCmp<T, B2P_CMP_EQ>{p.mask, p.rhs}, sms, st);
    case B2P_CMP_NE: return launch_copy_tmem_shape<T, NC, ITEMS>(p, tin, MaskCmp<T, B2P_CMP_NE>{p.mask, p.rhs}, sms, st);
    case B2P_CMP_GE: return launch_copy_tmem_shape<T, NC, ITEMS>(p, tin, MaskCmp<T, B2P_CMP_GE>{p.mask, p.rhs}, sms, st);
    default: return launch_copy_tmem_shape<T, NC, ITEMS>(p, tin, MaskCmp<T, B2P_CMP_GT>{p.mask, p.rhs}, sms, st);
    }
  }
  switch (p.cmp) {
  case B2P_CMP_LT: return launch_copy_shape<T, NC, ITEMS, B2P_CMP_LT>(p, tin, st);
  case B2P_CMP_LE: return launch_copy_shape<T, NC, ITEMS, B2P_CMP_LE>(p, tin, st);
  case B2P_CMP_EQ: return launch_copy_shape<T, NC, ITEMS, B2P_CMP_EQ>(p, tin, st);
  case B2P_CMP_NE: return launch_copy_shape<T, NC, ITEMS, B2P_CMP_NE>(p, tin, st);
  case B2P_CMP_GE: return launch_copy_shape<T, NC, ITEMS, B2P_CMP_GE>(p, tin, st);
  default: return launch_copy_shape<T, NC, ITEMS, B2P_CMP_GT>(p, tin, st);
  }
}

template <class T>
int launch_copy_cmp(TmaParams &p, const CUtensorMap &tin, int block, int items, cudaStream_t st) {
  if (block == 128 && items == 32) return launch_copy_items<T, 128, 32>(p, tin, st);
  if (block == 256 && items == 16) return launch_copy_items<T, 256, 16>(p, tin, st);
  if (block == 256 && items == 32) return launch_copy_items<T, 256, 32>(p, tin, st);
  return B2P_ERR_UNSUPPORTED;
}

template <class T>
int launch_copy_t(const void *in, void *out, size_t n, uint64_t mask, int cmp, uint64_t rhs, uint64_t *num_copied,
                  void *scratch, int block, int items, cudaStream_t st) {
  const size_t es = sizeof(T);
  const long long tile = (long long)block * items;
  const size_t stride = (size_t)tile * es + 1024;
  const int stages = (int)std::min<size_t>(kMaxStages, kSmemBudget / (stride + block * (sizeof(unsigned long long) + 4)));
  TmaParams p{};
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  const long long epr = 128 / (long long)es;
  p.rows_full = (long long)(n / (size_t)epr);
  p.tail_begin = (unsigned long long)p.rows_full * epr;
  if (p.rows_full + tile / epr >= (1ll << 31)) return B2P_ERR_UNSUPPORTED;
  p.stages = stages;
  p.stage_stride = (unsigned)stride;
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
  if (!copy_tmem_layout(p, es, block, items) && stages < kMinStages) return B2P_ERR_UNSUPPORTED;
  CUtensorMap tin;
  if (!encode_row_tensor(&tin, in, (unsigned long long)p.rows_full, (int)std::min<long long>(256, tile / epr)))
    return B2P_ERR_UNSUPPORTED;
  return launch_copy_cmp<T>(p, tin, block, items, st);
}

}  // namespace


bool scan_tma_shape(int dtype, int block, int items) {
  if (dtype_size(dtype) == 0) return false;
  const bool shape = (block == 128 && items == 32) || (block == 256 && items == 16) || (block == 256 && items == 32);
  const size_t es = dtype_size(dtype), eo = acc_size(dtype);
  const size_t stage = (size_t)block * items * (es + (eo != es ? eo : 0));
  const size_t acc = dtype_is_float(dtype) && dtype != B2P_F64 ? 8 : acc_size(dtype);
  return shape && (stage + (size_t)block * acc) * kMinStages <= kSmemBudget;
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
  case B2P_BF16: return dispatch<B2P_BF16>(op, inclusive, in, out, n, init, scratch, block, items, st);
  default: return B2P_ERR_UNSUPPORTED;
  }
}

bool copy_if_tma_shape(int dtype, int block, int items) {
  const size_t es = dtype_size(dtype);
  if (es != 4 && es != 8) return false;
  const bool shape = (block == 128 && items == 32) || (block == 256 && items == 16) || (block == 256 && items == 32);
  return shape && ((size_t)block * items * es + 1024 + (size_t)block * 12) * kMinStages <= kSmemBudget;
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
