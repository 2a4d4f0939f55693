// The warp-specialised pipeline shared by the single-pass TMA kernels
// (scan, copy_if, segmented reduce / scan): launch parameters, the block's
// barrier ring state, the per-thread tile passes, the group scans of the
// reducer and emitter warps, and the producer, look-back and store roles.
//
// One persistent block per SM; every step has its own warps, joined by
// mbarriers on a ring of shared stages:
//
//   producer warp    dynamic tile ids in order; TMA 2-D bulk tensor loads of
//                    each tile into the next free stage (128-byte swizzle)
//   reducer warps    as soon as a tile lands: per-thread totals, group scan,
//                    the tile aggregate published at once
//   look-back warps  resolve the carries of reduced tiles (bounded
//                    warp-parallel look-back over epoch-tagged status words)
//   emitter warps    as soon as a carry is known: the tile's outputs
//   store warp       TMA bulk store of each emitted stage, then frees it
//
// Every wait is bounded; a wait that runs out records B2P_ERR_TIMEOUT in the
// scratch header and the block leaves its loops.
#pragma once

#include "scan_tile.cuh"
#include "tma.cuh"
#include "tmem.cuh"

#include <mutex>

namespace b2p {


constexpr int kMaxStages = 16;
constexpr int kLookWarps = 2;
// Bulk stores a store warp keeps in flight before it waits for the oldest
// one to finish reading its stage (2 and 3 measured slower: a stage held by
// a store is a stage the producer cannot fill).
constexpr int kStoresInFlight = 1;
// Fewest stages a pipelined launch runs with.
constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int kMinStages = cmax(3, cmax(kLookWarps, kStoresInFlight));
constexpr size_t kSmemBudget = 210 * 1024;  // stages + thread prefixes
// Scans stage tiles that wait for their carries in TMEM where the policy
// and shape allow it.
constexpr bool kUseTmem = true;
// Output stages of the TMEM-staged copy_if.
constexpr int kCopyOutStages = 2;
// Output stages of the TMEM-staged scan, and the bulk tensor stores its
// store warp keeps in flight (at most kScanOutStages - 1).
constexpr int kScanOutStages = 2;
constexpr int kTmemStoresInFlight = 1;
constexpr int kScanMaxInStages = kMaxStages;

// Threads of a pipelined block with NC reducer and NC emitter threads.
constexpr int pipe_threads(int nc) { return 2 * nc + 32 * kLookWarps + 64; }

struct TmaParams {
  unsigned long long n;
  long long ntiles;
  long long rows_full;            // complete 128-byte input rows (the input tensor map's extent)
  unsigned long long tail_begin;  // first element past the complete input rows
  long long rows_full_out;        // complete 128-byte output rows (scans)
  unsigned long long tail_out_begin;  // first element past the complete output rows
  unsigned out_offset;            // byte offset of a stage's output tile (0: in place)
  int inclusive;
  int has_init;
  unsigned long long init_raw;    // Out-typed init value
  int stages;
  unsigned stage_stride;          // bytes between stages
  // TMEM-staged scan: carry slots in TMEM, output stages after the input
  // stages, thread prefixes per slot after the output stages
  int slots;
  int out_stages;
  unsigned out_stage_stride;
  unsigned out_base;
  unsigned texcl_base;
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
  // segmented: CSR offsets (nseg + 1), and one record per tile (kSegRecInts
  // ints: the index kb of the first offset at or after the tile's first
  // element, the count m of offsets from kb up to and including the first
  // one at or after the tile's end, and those m offsets relative to the
  // tile's first element when they fit)
  const long long *offsets;
  long long nseg;
  const int *seg_rec;
  unsigned info_base;  // shared-memory offset of the per-slot thread words
  unsigned rend_base;  // ... of the per-slot entering-segment ends (reduce)
  unsigned rec_base;   // ... of the per-stage tile records
};

// Per-tile record of the segmented kernel: 64 ints = 256 bytes.
constexpr int kSegRecInts = 64;
constexpr int kSegRecCap = kSegRecInts - 2;

// Block-shared state of the pipeline.  Per stage: the TMA fill barrier
// (full: producer -> reducers), aggregate published (aggr: reducers ->
// look-back warps), carry known (cready: look-back warps -> emitters),
// outputs in place (emitted: emitters -> store warp), stage free (empty:
// store warp -> producer); the stage's tile id, aggregate and carry.
struct PipeState {
  uint64_t full[kMaxStages], empty[kMaxStages], aggr[kMaxStages], cready[kMaxStages], emitted[kMaxStages];
  long long tile[kMaxStages];
  // TMEM-staged scan: slot handed back by the emitters, output stage handed
  // back by the store warp, tile ids of input and output stages, TMEM base
  uint64_t slot_free[kMaxStages], out_empty[kMaxStages], slot_ready[kMaxStages];
  long long tile_in[kMaxStages], tile_out[kMaxStages];
  unsigned long long out_carry[kMaxStages], out_count[kMaxStages];  // copy_if: output stage's position, count
  uint32_t tmem_base;
  unsigned long long agg[kMaxStages], carry[kMaxStages];
  int sflags[kMaxStages];  // segmented: head / carry flags of the slot's tile
  // segmented reduce: the tile-local value and index of the segment that
  // needs the tile's carry (the tile's first segment, ending in the tile)
  unsigned long long local[kMaxStages];
  long long lseg[kMaxStages];
  unsigned long long epoch;
  long long end_item;  // number of tiles this block handles, once the reducers know it
};


// --------------------------------------------------- per-thread tile passes
// `t` is the thread's index inside its warp group (reducers or emitters).

template <class P, int ITEMS>
__device__ __forceinline__ typename P::Acc thread_total_t(const char *buf, int t) {
  using In = typename P::In;
  constexpr int IPV = 16 / (int)sizeof(In);
  constexpr int VPT = ITEMS * (int)sizeof(In) / 16;
  typename P::Acc agg = P::identity();
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
    const In *e = reinterpret_cast<const In *>(&w);
#pragma unroll
    for (int q = 0; q < IPV; ++q) P::add(agg, e[q]);
  }
  if constexpr (P::kCompensated) agg = df_norm(agg);
  return agg;
}

// fp32 / bf16-input SUM, reducer pass: compensated (TwoSum) running sums of
// the thread's elements from zero, rounded to fp32 and written to the
// stage's output tile (in place for fp32 input; inclusive: after adding the
// element, exclusive: before).  Returns the thread total.
template <class In, int ITEMS, bool INCLUSIVE>
__device__ __forceinline__ DF thread_runs(const char *inbuf, char *outbuf, int t) {
  constexpr int IPV = 16 / (int)sizeof(In);
  constexpr int VPT_IN = ITEMS / IPV, VPT_OUT = ITEMS / 4, OPI = IPV / 4;
  DF run{0.f, 0.f};
#pragma unroll
  for (int k = 0; k < VPT_IN; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(inbuf + swz(t * VPT_IN + k) * 16);
    const In *e = reinterpret_cast<const In *>(&w);
#pragma unroll
    for (int m = 0; m < OPI; ++m) {
      float4 o;
      float *oe = reinterpret_cast<float *>(&o);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float x;
        if constexpr (sizeof(In) == 2) x = bf16_bits_to_f32(e[m * 4 + q]);
        else x = e[m * 4 + q];
        if constexpr (INCLUSIVE) {
          df_accumulate(run, x);
          oe[q] = __fadd_rn(run.hi, run.lo);
        } else {
          oe[q] = __fadd_rn(run.hi, run.lo);
          df_accumulate(run, x);
        }
      }
      *reinterpret_cast<float4 *>(outbuf + swz(t * VPT_OUT + k * OPI + m) * 16) = o;
    }
  }
  (void)VPT_OUT;
  return df_norm(run);
}

// fp32 SUM, emitter pass: output = start + run.  The run carries at most one
// rounding of its exact value, so each output is within ~2 ulp of the exact
// prefix for same-signed data.
template <int ITEMS>
__device__ __forceinline__ void emit_f32_runs(char *buf, DF start, int t) {
  constexpr int VPT = ITEMS / 4;
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    float4 *slot = reinterpret_cast<float4 *>(buf + swz(t * VPT + k) * 16);
    float4 w = *slot;
    w.x = __fadd_rn(start.hi, __fadd_rn(start.lo, w.x));
    w.y = __fadd_rn(start.hi, __fadd_rn(start.lo, w.y));
    w.z = __fadd_rn(start.hi, __fadd_rn(start.lo, w.z));
    w.w = __fadd_rn(start.hi, __fadd_rn(start.lo, w.w));
    *slot = w;
  }
}

// Generic emitter pass: the thread's outputs from its running value, into
// the stage's output tile (in place when input and output sizes match; each
// output vector overwrites only input this thread has already read).
template <class P, int ITEMS>
__device__ __forceinline__ void emit_generic(const char *inbuf, char *outbuf, typename P::Acc run, bool inclusive,
                                             int t) {
  using In = typename P::In;
  using Out = typename P::Out;
  constexpr int IPV = 16 / (int)sizeof(In);
  constexpr int OPV = 16 / (int)sizeof(Out);
  constexpr int VPT_IN = ITEMS / IPV, VPT_OUT = ITEMS / OPV, OPI = IPV / OPV;
#pragma unroll
  for (int k = 0; k < VPT_IN; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(inbuf + swz(t * VPT_IN + k) * 16);
    const In *e = reinterpret_cast<const In *>(&w);
#pragma unroll
    for (int m = 0; m < OPI; ++m) {
      uint4 o;
      Out *oe = reinterpret_cast<Out *>(&o);
#pragma unroll
      for (int q = 0; q < OPV; ++q) {
        if (inclusive) {
          P::add(run, e[m * OPV + q]);
          oe[q] = P::finalize(run);
        } else {
          oe[q] = P::finalize(run);
          P::add(run, e[m * OPV + q]);
        }
      }
      *reinterpret_cast<uint4 *>(outbuf + swz(t * VPT_OUT + k * OPI + m) * 16) = o;
    }
  }
}

// Exclusive scan over one warp group of NC threads (named barrier `bar`);
// t = index in the group.
template <class Ops, int NC>
__device__ __forceinline__ typename Ops::Pub group_exclusive_scan(typename Ops::Pub v, typename Ops::Pub *s_warp,
                                                                  typename Ops::Pub *total, int t, int bar) {
  using Pub = typename Ops::Pub;
  constexpr int kWarps = NC / 32;
  const int lane = t & 31, warp = t >> 5;
  Pub incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Pub o = shfl_up(incl, d);
    if (lane >= d) incl = Ops::combine(o, incl);
  }
  if (lane == 31) s_warp[warp] = incl;
  bar_named(bar, NC);
  if (warp == 0) {
    Pub w = lane < kWarps ? s_warp[lane] : Ops::identity();
#pragma unroll
    for (int d = 1; d < kWarps; d <<= 1) {
      Pub o = shfl_up(w, d);
      if (lane >= d) w = Ops::combine(o, w);
    }
    if (lane < kWarps) s_warp[lane] = w;
  }
  bar_named(bar, NC);
  Pub ex = shfl_up(incl, 1);
  if (lane == 0) ex = Ops::identity();
  if (warp > 0) ex = Ops::combine(s_warp[warp - 1], ex);
  *total = s_warp[kWarps - 1];
  return ex;  // callers end with a bar_named(bar, NC) before s_warp is used again
}

// Exclusive scan over one warp group of NC threads with a single named
// barrier: after the warp totals are in s_warp, every warp scans them itself
// (the same combine tree warp 0 runs in group_exclusive_scan, so the same
// bits).  s_warp may be written again only after a later barrier of the
// group.
template <class Ops, int NC>
__device__ __forceinline__ typename Ops::Pub group_exclusive_scan_1bar(typename Ops::Pub v,
                                                                       typename Ops::Pub *s_warp,
                                                                       typename Ops::Pub *total, int t, int bar) {
  using Pub = typename Ops::Pub;
  constexpr int kWarps = NC / 32;
  const int lane = t & 31, warp = t >> 5;
  Pub incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Pub o = shfl_up(incl, d);
    if (lane >= d) incl = Ops::combine(o, incl);
  }
  if (lane == 31) s_warp[warp] = incl;
  bar_named(bar, NC);
  Pub w = lane < kWarps ? s_warp[lane] : Ops::identity();
#pragma unroll
  for (int d = 1; d < kWarps; d <<= 1) {
    Pub o = shfl_up(w, d);
    if (lane >= d) w = Ops::combine(o, w);
  }
  const Pub before = shfl_idx(w, warp > 0 ? warp - 1 : 0);
  *total = shfl_idx(w, kWarps - 1);
  Pub ex = shfl_up(incl, 1);
  if (lane == 0) ex = Ops::identity();
  if (warp > 0) ex = Ops::combine(before, ex);
  return ex;
}

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

// ------------------------------------------------------------ warp roles

// Thread 0 of the block: barriers and the launch epoch.
__device__ __forceinline__ void pipe_init(PipeState &ps, const TmaParams &p) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < p.stages; ++i) {
      mbar_init(&ps.full[i], 1);
      mbar_init(&ps.empty[i], 1);
      mbar_init(&ps.aggr[i], 1);
      mbar_init(&ps.cready[i], 1);
      mbar_init(&ps.emitted[i], 1);
    }
    mbar_init_fence();
    ps.epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
    ps.end_item = 0x7fffffffffffffffll;
  }
}

// Producer (one thread): each tile's complete rows into the next free stage
// in boxes of `box` rows, and, when `rec_g` is given, the tile's
// `rec_bytes`-byte record (rec_g + tile * rec_bytes) into rec_s + stage *
// rec_bytes on the same barrier.  A tile wholly past the complete rows
// completes its stage without a row copy.  Tile id -1 ends the reducers.
// The next tile id is fetched while the current one is issued, so the
// counter's round trip overlaps the stage wait; ids stay in order per
// block, and every id a block holds is loaded as soon as it has a stage (a
// block only ever waits for tiles of lower ids, so every wait ends).
// `end_markers` consumer groups take items in turn; each gets an end marker.
__device__ __forceinline__ void producer_loop(const CUtensorMap *tin, const TmaParams &p, PipeState &ps,
                                              char *smem, int rows, int box, long long *tiles,
                                              const char *rec_g = nullptr, char *rec_s = nullptr,
                                              unsigned rec_bytes = 0, int end_markers = 1) {
  prefetch_tensormap(tin);
  const unsigned long long pol = l2_policy_stream();
  const int S = p.stages;
  long long next = (long long)atomicAdd(&p.hdr->tile_ctr, 1ull);
  for (RingPos r;; r.advance(1, S)) {
    const int s = r.s;
    if (!mbar_wait(&ps.empty[s], r.ph ^ 1u, p.timeout_ns)) {
      record_error(p.hdr, B2P_ERR_TIMEOUT);
      tiles[s] = -1;
      mbar_arrive(&ps.full[s]);
      return;
    }
    const long long tile = next;
    if (tile >= p.ntiles) {
      tiles[s] = -1;
      mbar_arrive(&ps.full[s]);
      if (--end_markers > 0) continue;
      return;
    }
    next = (long long)atomicAdd(&p.hdr->tile_ctr, 1ull);
    tiles[s] = tile;
    const long long r0 = tile * rows;
    const long long rows_in = min((long long)rows, p.rows_full - r0);
    const int nbox = rows_in > 0 ? (int)((rows_in + box - 1) / box) : 0;
    const unsigned extra = rec_g ? rec_bytes : 0u;
    if (nbox == 0 && extra == 0) {
      mbar_arrive(&ps.full[s]);
    } else {
      mbar_arrive_expect_tx(&ps.full[s], (unsigned)nbox * (unsigned)box * 128u + extra);
      for (int b = 0; b < nbox; ++b)
        tma_load_2d(smem + (size_t)s * p.stage_stride + (size_t)b * box * 128, tin, 0,
                    (int)(r0 + (long long)b * box), &ps.full[s], pol);
      if (extra) bulk_load(rec_s + (size_t)s * rec_bytes, rec_g + (size_t)tile * rec_bytes, rec_bytes, &ps.full[s], pol);
    }
  }
}

// Look-back warp wi of kLookWarps: items wi, wi + kLookWarps, ... in stage
// order.  Resolves each reduced tile's carry, publishes its inclusive prefix
// and hands the carry to the emitters.
template <class Ops>
__device__ __forceinline__ void lookback_loop(const TmaParams &p, PipeState &ps, int wi,
                                              unsigned long long init_bits, unsigned long long epoch_tag, int S) {
  using Pub = typename Ops::Pub;
  const int lane = threadIdx.x & 31;
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

// Emitter group: wait for item `it`'s carry, or learn that the block's items
// are exhausted (the reducers publish the count when they meet the end).
// Returns 1 = carry ready, 0 = no more items, -1 = timeout.
__device__ __forceinline__ int emitter_wait(const TmaParams &p, PipeState &ps, const RingPos &r, long long it) {
  uint64_t t0 = 0;
  for (unsigned k = 0;; ++k) {
    // parked up to 2 us per try: the end of the items is seen within that
    if (mbar_try_hint(&ps.cready[r.s], r.ph, 2000)) return 1;
    if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) return 0;
    if ((k & 7) == 7) {
      const uint64_t now = globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > p.timeout_ns) return -1;
    }
  }
}

// Emitter leader after the last item (`it` = item count): every earlier item
// passed the look-back warps and was handed to the store warp, so their
// barriers are in step; end the look-back warps (waiting on items it and
// it + 1) and the store warp (waiting on item it).
__device__ __forceinline__ void emitters_finish(const TmaParams &p, PipeState &ps, RingPos r) {
  mbar_arrive(&ps.emitted[r.s]);
  for (int j = 0; j < kLookWarps; ++j, r.advance(1, p.stages)) mbar_arrive(&ps.aggr[r.s]);
}

// Store warp: stages whose bulk stores were committed but may still read
// shared memory.  A stage is handed back to the producer (empty barrier)
// once its store has read it; up to kStoresInFlight stores overlap.
template <int D = kStoresInFlight>
struct StoreRelease {
  RingPos oldest;
  int pending = 0;
  // after committing a store group for the ring of S barriers `freed`
  __device__ __forceinline__ void committed(uint64_t *freed, int S) {
    if (++pending < D) return;
    bulk_wait_read<D - 1>();
    mbar_arrive(&freed[oldest.s]);
    oldest.advance(1, S);
    --pending;
  }
  __device__ __forceinline__ void drain(uint64_t *freed, int S) {
    bulk_wait_read<0>();
    for (; pending > 0; --pending, oldest.advance(1, S)) mbar_arrive(&freed[oldest.s]);
  }
};

// Elements past the complete rows (only in the last tile) into the stage,
// by the reducer group (threads 0 .. ntail-1 of the block).
template <class T, int NC>
__device__ __forceinline__ void load_row_tail(const TmaParams &p, char *buf, long long tile, int tile_elems) {
  const int ntail = (int)(p.n - p.tail_begin);
  const long long j0 = (long long)p.tail_begin - tile * tile_elems;
  if ((int)threadIdx.x < ntail)
    *smem_elem_ptr<T>(buf, (int)j0 + (int)threadIdx.x) =
        reinterpret_cast<const T *>(p.in)[p.tail_begin + threadIdx.x];
  bar_named(1, NC);
}

// Policies whose outputs the TMEM kernel forms as combine(start, run) with
// the bits of the in-place kernel's sequential pass: integer operators (exact
// in wrap-around arithmetic) and fp32 / bf16-input SUM (the same
// start.hi + (start.lo + run) formula).  Floating-point PROD, MIN, MAX and
// fp64 SUM stay on the in-place kernel.
template <class P>
struct TmemExact : std::integral_constant<bool, P::kCompensated || std::is_integral<typename P::Acc>::value> {};

// TMEM columns a reducer thread fills per tile.
template <class P, int ITEMS>
constexpr int tmem_cols() {
  return ITEMS * (int)sizeof(typename P::Out) / 4;
}

// Thread 0: barriers of the three rings (input stages, TMEM slots, output
// stages) and the launch epoch.  Reducer and emitter warps arrive one by one
// on the barriers that hand back input stages and slots.
__device__ __forceinline__ void tmem_pipe_init(PipeState &ps, const TmaParams &p, unsigned group_warps,
                                               unsigned aggr_count = 1) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < p.stages; ++i) {
      mbar_init(&ps.full[i], 1);
      mbar_init(&ps.empty[i], group_warps);
    }
    for (int i = 0; i < p.slots; ++i) {
      mbar_init(&ps.aggr[i], aggr_count);
      mbar_init(&ps.cready[i], 1);
      mbar_init(&ps.slot_free[i], group_warps);
      mbar_init(&ps.slot_ready[i], group_warps);
    }
    for (int i = 0; i < p.out_stages; ++i) {
      mbar_init(&ps.emitted[i], 1);
      mbar_init(&ps.out_empty[i], 1);
    }
    mbar_init_fence();
    ps.epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
    ps.end_item = 0x7fffffffffffffffll;
  }
}

}  // namespace b2p
