// Segmented reduce / scan on the TMA pipeline: the flat segmented scan of
// the concatenated segments (segment heads reset the running value), for
// SUM over integer, fp32 and bf16 inputs with 16-byte aligned buffers; the
// persistent piece kernel of segmented.cu covers everything else.
#include "b2p_device/pipe.cuh"
#include "internal.h"

#include <algorithm>

namespace b2p {

namespace {

// ------------------------------------------------- segmented, TMEM-staged
//
// Segmented reduce / scan over CSR offsets as ONE scan of the concatenated
// segments on the TMEM-staged pipeline, with the segmented operator
// (f1, v1) + (f2, v2) = (f1 | f2, f2 ? v2 : v1 + v2): a segment head resets
// the running value (to init), so every tile is a fixed-size, 16-byte
// aligned piece of the flat array whatever the segment lengths, loaded by
// TMA like any scan tile.  Per tile:
//   producer   with each tile's data, a 256-byte record built on the host:
//              the tile's segment boundaries (and the first one after it)
//              relative to the tile, so no boundary is looked up on the way;
//   reducers   find each thread's heads and segment ends by a binary search
//              in the record (bit masks), and run the thread's values from
//              the identity, restarting at init on each head; the tile aggregate is (has a head,
//              value after the last head).  A tile with a head publishes
//              that value as its inclusive prefix at once (nothing before
//              its last head matters to later tiles), so look-backs stop at
//              the first tile with a head.
//   look-back  only tiles whose first element is not a head need a carry.
//   emitters   scan: outputs before the thread's first head are
//              start (+) run, later ones are the run itself; reduce: the
//              reducers already wrote every segment that ends after a head
//              in the same thread, the emitters write the one segment per
//              thread that entered it (if it ends there).
// Empty segments (reduce) get init, written by the thread whose element
// range holds their position.  A reduce needs no TMEM and no output
// stages: only the per-thread words pass from reducers to emitters.

// Double-float form of an FP64 value: hi its rounding to float, lo the
// rounded rest.
__device__ __forceinline__ DF df_of_f64(double d) {
  const float h = (float)d;
  return DF{h, (float)(d - (double)h)};
}

// FP64 stand-in for a compensated policy in a tile's group scans (the
// segmented operator over (flag, FP64 value) pairs)
struct F64Sum {
  using Acc = double;
  __device__ static double identity() { return 0.0; }
  __device__ static double combine(double a, double b) { return a + b; }
};

constexpr int kSegHasHead = 1;
constexpr int kSegNeedCarry = 2;  // some output of the tile needs the carry
// per-thread word from reducers to emitters
constexpr unsigned long long kSegTexclF = 1ull << 63;  // the thread's exclusive prefix has a head

// Boundary i of the tile, relative to the tile's first element (the staged
// record, or global memory when the tile has more than a record holds).
struct SegBounds {
  const int *s;
  const long long *g;
  long long t0;
  int m;
  __device__ __forceinline__ long long at(int i) const { return s ? (long long)s[i] : g[i] - t0; }
  // first i with at(i) >= v
  __device__ __forceinline__ int lower(long long v) const {
    int lo = 0, hi = m;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (at(mid) < v) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  }
};

// Reducer groups of a reduce (the reduce needs no emitters): as many as fit
// in 1024 threads beside the look-back, producer and store warps.
constexpr int seg_groups(int nc, bool reduce) { return reduce ? (nc <= 128 ? 4 : 3) : 1; }
constexpr int seg_threads(int nc, bool reduce) {
  return reduce ? seg_groups(nc, true) * nc + 32 * kLookWarps + 64 : pipe_threads(nc);
}

template <class P, int NC, int ITEMS, bool WIDE, bool REDUCE>
__global__ void __launch_bounds__(seg_threads(NC, REDUCE), 1)
    seg_tmem_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
                    TmaParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Pair = SegPair<P>;
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
  static_assert(ITEMS <= 32, "head mask is 32 bits");
  // look-back warps of a reduce (its emitter places hold the second group)
  constexpr int kSegLookWarps = kLookWarps;
  constexpr int kSlotCols = kCols * (NC / 128);

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  char *obase = smem + p.out_base;
  Acc *texcl_all = reinterpret_cast<Acc *>(smem + p.texcl_base);
  unsigned long long *info_all = reinterpret_cast<unsigned long long *>(smem + p.info_base);
  __shared__ __align__(8) PipeState ps;
  // A reduce has several reducer groups taking items in turn (it has no
  // emitters); a scan has one.  Per group: the leader's verdict,
  // the group scan's warp values, and whether a thread ends the tile's first
  // segment (reduce).
  constexpr int kGroups = seg_groups(NC, REDUCE);
  // warps before the look-back warps: the reducer groups (a reduce) or the
  // reducer and emitter groups (a scan)
  constexpr int kWorkWarps = REDUCE ? kGroups * NC / 32 : 2 * NC / 32;
  __shared__ Pair s_warp_g[kGroups][32];
  __shared__ Acc s_acc_g[kGroups][32];  // clean tiles: warp totals (reduce) or the scan's warp values
  __shared__ double s_dbl_g[kGroups][32];  // clean tiles of a compensated sum: FP64 warp totals / values
  __shared__ SegPair<F64Sum> s_pd_g[kGroups][32];  // compensated tiles with boundaries: FP64 warp values
  __shared__ int s_go[kGroups > 2 ? kGroups : 2];  // [g]: reducer group g; [1] of a scan: the emitters
  __shared__ int s_entering_end_g[kGroups];
  __shared__ long long s_stop[kGroups];  // reduce: the item at which each group met the end

  const int warp = threadIdx.x >> 5;
  if (threadIdx.x < kGroups) s_entering_end_g[threadIdx.x] = 0;
  // a reduce hands slots back from one look-back lane, a scan from every
  // emitter warp
  tmem_pipe_init(ps, p, NC / 32);
  if (REDUCE && threadIdx.x == 0) {
    for (int i = 0; i < p.slots; ++i) mbar_init(&ps.slot_free[i], 1);
    mbar_init_fence();
  }
  if constexpr (!REDUCE) {
    if (warp == 0) {
      __syncwarp();
      tmem_alloc(&ps.tmem_base, 512);
    }
    tmem_fence_before();
  }
  __syncthreads();
  if constexpr (!REDUCE) tmem_fence_after();
  const uint32_t tbase = REDUCE ? 0u : ps.tmem_base;
  const unsigned long long epoch = ps.epoch;
  const unsigned long long epoch_tag = epoch << 8;
  const int SI = p.stages, SL = p.slots, SO = p.out_stages;
  if (REDUCE && SL < kSegLookWarps) return;  // the host gives a reduce kMaxStages slots
  const long long last = p.ntiles - 1;
  const int ntail = (int)(p.n - p.tail_begin);
  const int ntail_out = (int)(p.n - p.tail_out_begin);
  Out *out = reinterpret_cast<Out *>(p.out);
  // segment start value: init, or the identity
  const Acc init_acc = p.has_init ? P::from_out(from_bits64<Out>(p.init_raw)) : P::identity();

  if (warp < kGroups * NC / 32) {
    // ------------------------------------------------------------ reducers
    // group g takes items g, g + kGroups, ...
    const int g = warp / (NC / 32);
    const int t = threadIdx.x - g * NC;
    const int gbar = 1 + g;
    Pair *s_warp = s_warp_g[g];
    Acc *s_acc = s_acc_g[g];
    int &s_entering_end = s_entering_end_g[g];
    const uint32_t tcol = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * kCols);
    long long it = g;
    RingPos ri, rs;
    ri.advance(g, SI);
    rs.advance(g, SL);
    for (;; it += kGroups, ri.advance(kGroups, SI), rs.advance(kGroups, SL)) {
      if (t == 0) {
        int go = mbar_wait(&ps.full[ri.s], ri.ph, p.timeout_ns) ? 1 : -1;
        if (go > 0 && ps.tile_in[ri.s] < 0) go = 0;
        if (go > 0 && !mbar_wait(&ps.slot_free[rs.s], rs.ph ^ 1u, p.timeout_ns)) go = -1;
        if (go < 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        s_go[g] = go;
      }
      bar_named(gbar, NC);
      if (s_go[g] <= 0) break;
      (void)mbar_try(&ps.full[ri.s], ri.ph);  // completed: this thread's acquire of the TMA bytes
      if constexpr (!REDUCE) tmem_fence_after();
      const long long tile = ps.tile_in[ri.s];
      char *buf = smem + (size_t)ri.s * p.stage_stride;
      if (tile == last && ntail > 0) {
        // elements past the complete rows (only in the last tile)
        const long long j0 = (long long)p.tail_begin - tile * kTile;
        if (t < ntail) *smem_elem_ptr<In>(buf, (int)j0 + t) = reinterpret_cast<const In *>(p.in)[p.tail_begin + t];
        bar_named(gbar, NC);
      }
      const long long T0 = tile * kTile;
      const int count = (int)min((unsigned long long)kTile, p.n - (unsigned long long)T0);
      // the tile's boundaries plus the first one after it, from the tile's
      // record (landed with the tile); a tile with more boundaries than a
      // record holds reads them from the offsets in global memory
      const int *rec = reinterpret_cast<const int *>(smem + p.rec_base) + (size_t)ri.s * kSegRecInts;
      const int kb = rec[0];
      const int m = rec[1];
      SegBounds B{nullptr, p.offsets + kb, T0, m};
      if (m <= kSegRecCap) B.s = rec + 2;
      // this thread's elements [e0, e0 + lim) of the tile (lim <= 0: none)
      const int e0 = t * ITEMS;
      const int lim = min(ITEMS, count - e0);
      // A clean tile has no segment boundary inside it (a reduce: none at
      // positions 0 .. count, a scan: no head before count); every tile
      // inside a long segment is clean.  It needs no segmented operator:
      // its aggregate is the plain combination of the thread totals, and no
      // thread has a head or an end to find.
      const bool clean = m >= 1 && (REDUCE ? B.at(0) > count : B.at(0) >= count);
      const int i0 = clean ? 0 : B.lower(e0);
      // heads: bit j = a segment starts at e0 + j; ends: bit j = one ends at
      // e0 + j.  Boundaries that share a position with the next one start
      // empty segments (a reduce gives them init), and so does every
      // boundary below nseg at the end of the data.
      unsigned heads = 0, ends = 0;
      if (lim > 0 && !clean) {
        for (int i = i0; i < m; ++i) {
          const long long at = B.at(i);
          const int r = (int)(at - e0);
          if (r > lim) break;
          const bool data_end = tile == last && at == count;
          if (r < lim) {
            if (i + 1 < m && B.at(i + 1) == at) {
              if (REDUCE && kb + i < p.nseg) out[kb + i] = P::finalize(init_acc);
            } else {
              heads |= 1u << r;
            }
          } else if (REDUCE && data_end && kb + i < p.nseg) {
            out[kb + i] = P::finalize(init_acc);
          }
          if (r >= 1) ends |= 1u << (r - 1);
        }
      }
      Acc run = P::identity();
      int f = 0;
      int j_end = -1;
      Acc r_end = P::identity();
      uint32_t w[kCols];
      constexpr int IPV = 16 / (int)sizeof(In), VPT = ITEMS / IPV, WPO = (int)sizeof(Out) / 4;
      if constexpr (P::kCompensated) {
        // fp32 / bf16 SUM: a thread's run is an FP64 sum of its values (32 at
        // most, each exact in FP64), two instructions per element against
        // the seven of a double-float TwoSum step; every output is one
        // rounding of it, and the run goes on as (hi, lo), the FP64 value
        // split into two floats
        const double init_d = (double)init_acc.hi + (double)init_acc.lo;
        double rd = 0.0;
        if (REDUCE && heads == 0 && ends == 0) {
          // a reduce, no segment starts or ends here: only the thread total
          // matters, summed in four independent chains (element j to chain
          // j % 4) so that the dependent additions overlap
          double ch[4] = {0.0, 0.0, 0.0, 0.0};
          if (lim == ITEMS) {
#pragma unroll
            for (int k = 0; k < VPT; ++k) {
              const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
              const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
              for (int q = 0; q < IPV; ++q) ch[(k * IPV + q) & 3] += (double)P::lift_f(ev[q]);
            }
          } else {
#pragma unroll
            for (int k = 0; k < VPT; ++k) {
              const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
              const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
              for (int q = 0; q < IPV; ++q)
                if (k * IPV + q < lim) ch[(k * IPV + q) & 3] += (double)P::lift_f(ev[q]);
            }
          }
          rd = (ch[0] + ch[1]) + (ch[2] + ch[3]);
        } else if (!REDUCE && heads == 0) {
          // a scan, no segment starts here (the common case inside long segments)
#pragma unroll
          for (int k = 0; k < VPT; ++k) {
            const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
            const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
            for (int q = 0; q < IPV; ++q) {
              const int j = k * IPV + q;
              const double x = j < lim ? (double)P::lift_f(ev[q]) : 0.0;
              const Out o = (Out)(p.inclusive ? rd + x : rd);
              rd += x;
              memcpy(w + j * WPO, &o, sizeof(Out));
            }
          }
        } else {
          int ip = i0;                            // next boundary not yet passed (reduce)
          long long seg = (long long)kb + i0 - 1;  // segment of the current run (reduce)
#pragma unroll
          for (int k = 0; k < VPT; ++k) {
            const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
            const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
            for (int q = 0; q < IPV; ++q) {
              const int j = k * IPV + q;
              if ((heads >> j) & 1u) {
                f = 1;
                rd = init_d;
                if constexpr (REDUCE) {
                  // the segment starting here is the last boundary at e0 + j
                  while (ip < m && B.at(ip) <= e0 + j) ++ip;
                  seg = (long long)kb + ip - 1;
                }
              }
              const double x = j < lim ? (double)P::lift_f(ev[q]) : 0.0;
              if constexpr (REDUCE) {
                rd += x;
                if ((ends >> j) & 1u) {
                  if (f) {
                    out[seg] = (Out)rd;
                  } else {
                    j_end = j;
                    r_end = df_of_f64(rd);
                  }
                }
              } else {
                const Out o = (Out)(p.inclusive ? rd + x : rd);
                rd += x;
                memcpy(w + j * WPO, &o, sizeof(Out));
              }
            }
          }
        }
        run = df_of_f64(rd);
      } else if (REDUCE && heads == 0 && ends == 0) {
        // a reduce, no segment starts or ends here: only the thread total matters
        const bool full = lim == ITEMS;
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
          const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
          const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
          for (int q = 0; q < IPV; ++q)
            if (full || k * IPV + q < lim) P::add(run, ev[q]);
        }
      } else if (!REDUCE && heads == 0) {
        // a scan, no segment starts here (the common case inside long segments)
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
          const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
          const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
          for (int q = 0; q < IPV; ++q) {
            const int j = k * IPV + q;
            Out o;
            if (p.inclusive) {
              if (j < lim) P::add(run, ev[q]);
              o = P::finalize(run);
            } else {
              o = P::finalize(run);
              if (j < lim) P::add(run, ev[q]);
            }
            memcpy(w + j * WPO, &o, sizeof(Out));
          }
        }
      } else {
        int ip = i0;                            // next boundary not yet passed (reduce)
        long long seg = (long long)kb + i0 - 1;  // segment of the current run (reduce)
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
          const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * VPT + k) * 16);
          const In *ev = reinterpret_cast<const In *>(&u);
#pragma unroll
          for (int q = 0; q < IPV; ++q) {
            const int j = k * IPV + q;
            const bool valid = j < lim;
            if ((heads >> j) & 1u) {
              f = 1;
              run = init_acc;
              if constexpr (REDUCE) {
                // the segment starting here is the last boundary at e0 + j
                while (ip < m && B.at(ip) <= e0 + j) ++ip;
                seg = (long long)kb + ip - 1;
              }
            }
            Out o;
            if (p.inclusive) {
              if (valid) P::add(run, ev[q]);
              o = P::finalize(run);
            } else {
              o = P::finalize(run);
              if (valid) P::add(run, ev[q]);
            }
            if constexpr (REDUCE) {
              if ((ends >> j) & 1u) {
                if (f) {
                  out[seg] = o;
                } else {
                  j_end = j;
                  r_end = run;
                }
              }
            } else {
              memcpy(w + j * WPO, &o, sizeof(Out));
            }
          }
        }
      }
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.empty[ri.s]);  // this warp is done with the input stage
      if constexpr (!REDUCE) {
        const uint32_t ta = tcol + (uint32_t)(rs.s * kSlotCols);
        tmem_st16(ta, w);
        if constexpr (kCols == 32) tmem_st16(ta + 16, w + 16);
      }
      if (clean) {
        Acc tile_tot;
        if constexpr (REDUCE && P::kCompensated) {
          // the double-float thread totals combine in FP64: exact conversions,
          // one add per shuffle step instead of a double-float add
          double d = (double)run.hi + (double)run.lo;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
          if ((t & 31) == 0) s_dbl_g[g][t >> 5] = d;
          bar_named(gbar, NC);
          double sum = s_dbl_g[g][0];
#pragma unroll
          for (int w = 1; w < NC / 32; ++w) sum += s_dbl_g[g][w];
          const float h = (float)sum;
          tile_tot = Acc{h, (float)(sum - (double)h)};
        } else if constexpr (REDUCE) {
          const Acc wt = warp_allreduce<P>(run);
          if ((t & 31) == 0) s_acc[t >> 5] = wt;
          bar_named(gbar, NC);
          tile_tot = s_acc[0];
#pragma unroll
          for (int w = 1; w < NC / 32; ++w) tile_tot = P::combine(tile_tot, s_acc[w]);
        } else {
          Acc tex;
          if constexpr (P::kCompensated) {
            double tot_d;
            const double ex_d =
                group_exclusive_scan_1bar<F64Ops, NC>((double)run.hi + (double)run.lo, s_dbl_g[g], &tot_d, t, gbar);
            tile_tot = df_of_f64(tot_d);
            tex = df_of_f64(ex_d);
          } else {
            tex = group_exclusive_scan_1bar<AccOps<P>, NC>(run, s_acc, &tile_tot, t, gbar);
          }
          texcl_all[(size_t)rs.s * NC + t] = tex;
          info_all[(size_t)rs.s * NC + t] = 0ull;
        }
        if (t == 0) {
          const unsigned long long bits = publish_value<P, WIDE>(tile_tot);
          if (tile != p.stall_tile) st_status(p.status + tile, bits, epoch_tag | kFlagAgg);
          ps.tile[rs.s] = tile;
          ps.agg[rs.s] = bits;
          ps.sflags[rs.s] = REDUCE ? 0 : kSegNeedCarry;
          mbar_arrive(&ps.aggr[rs.s]);
        }
        if constexpr (!REDUCE) {
          tmem_wait_st();
          tmem_fence_before();
        }
        __syncwarp();
        if ((t & 31) == 0) mbar_arrive(&ps.slot_ready[rs.s]);
        continue;
      }
      Pair tile_agg, tex;
      if constexpr (P::kCompensated) {
        using PD = SegPair<F64Sum>;
        PD agg_d;
        const PD ex_d = group_exclusive_scan_1bar<SegOps<F64Sum>, NC>(PD{(double)run.hi + (double)run.lo, f},
                                                                     s_pd_g[g], &agg_d, t, gbar);
        tile_agg = Pair{df_of_f64(agg_d.v), agg_d.f};
        tex = Pair{df_of_f64(ex_d.v), ex_d.f};
      } else {
        tex = group_exclusive_scan_1bar<SegOps<P>, NC>(Pair{run, f}, s_warp, &tile_agg, t, gbar);
      }
      if constexpr (REDUCE) {
        // the segment entering this thread ends at j_end: after a head of an
        // earlier thread of the tile its value is complete; otherwise it is
        // the tile's first segment and needs the tile's carry, which the
        // look-back warp adds
        if (j_end >= 0) {
          const Acc v = P::combine(tex.v, r_end);
          const long long sg = (long long)kb + i0 - 1;
          if (tex.f) {
            out[sg] = P::finalize(v);
          } else {
            ps.local[rs.s] = P::pack(v);
            ps.lseg[rs.s] = sg;
            s_entering_end = 1;
          }
        }
        bar_named(gbar, NC);  // the tile's value needing the carry is in place
      } else {
        texcl_all[(size_t)rs.s * NC + t] = tex.v;
        info_all[(size_t)rs.s * NC + t] = (tex.f ? kSegTexclF : 0ull) | heads;
      }
      if (t == 0) {
        // a scan needs the carry unless the tile starts with a head; a reduce
        // only when the tile's first segment ends in it (the others end in
        // later tiles, whose look-backs pass over this tile's aggregate)
        bool need = !(heads & 1u);
        if constexpr (REDUCE) {
          need = need && s_entering_end != 0;
          s_entering_end = 0;
        }
        const int sf = (tile_agg.f ? kSegHasHead : 0) | (need ? kSegNeedCarry : 0);
        const unsigned long long bits = publish_value<P, WIDE>(tile_agg.v);
        if (tile != p.stall_tile && tile_agg.f) st_status(p.status + tile, bits, epoch_tag | kFlagPrefix);
        else if (tile != p.stall_tile) st_status(p.status + tile, bits, epoch_tag | kFlagAgg);
        ps.tile[rs.s] = tile;
        ps.agg[rs.s] = bits;
        ps.sflags[rs.s] = sf;
        mbar_arrive(&ps.aggr[rs.s]);
      }
      if constexpr (!REDUCE) {
        tmem_wait_st();
        tmem_fence_before();
      }
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.slot_ready[rs.s]);  // this warp's slot columns and words
    }
    if constexpr (REDUCE) {
      // both groups stopped: the item count is the lower of their end items;
      // wake every look-back warp on the items after the last (end ..
      // end + kSegLookWarps - 1, one per warp), each slot once its previous
      // item is done
      if (t == 0) s_stop[g] = it;
      bar_named(kGroups + 1, kGroups * NC);
      if (threadIdx.x == 0) {
        long long end = s_stop[0];
        for (int q = 1; q < kGroups; ++q) end = min(end, s_stop[q]);
        *reinterpret_cast<volatile long long *>(&ps.end_item) = end;
        RingPos r;
        r.advance((int)(end % SL), SL);
        // the phase parity of slot (end % SL) for item `end`
        if ((end / SL) & 1) r.ph ^= 1u;
        for (int j = 0; j < kSegLookWarps; ++j, r.advance(1, SL)) {
          if (!mbar_wait(&ps.slot_free[r.s], r.ph ^ 1u, p.timeout_ns)) record_error(p.hdr, B2P_ERR_TIMEOUT);
          mbar_arrive(&ps.aggr[r.s]);
        }
      }
    } else if (t == 0) {
      *reinterpret_cast<volatile long long *>(&ps.end_item) = it;
    }
  } else if (REDUCE && warp < kWorkWarps + kLookWarps) {
    // ----------------------------------------- look-back warps of a reduce
    // item wi, wi + kSegLookWarps, ...
    const int wi = warp - kWorkWarps;
    const int lane = threadIdx.x & 31;
    RingPos r;
    r.advance(wi, SL);
    for (long long it = wi;; it += kSegLookWarps, r.advance(kSegLookWarps, SL)) {
      const int s = r.s;
      const bool ok = __shfl_sync(0xffffffffu, (int)mbar_wait(&ps.aggr[s], r.ph, p.timeout_ns), 0) != 0;
      if (!ok) {
        if (lane == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        break;
      }
      if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
      const long long tile = ps.tile[s];
      if (tile > 0 && (ps.sflags[s] & kSegNeedCarry)) {
        bool err;
        const typename Ops::Pub carry = lookback<Ops, false>(p.status, tile, epoch_tag, p.timeout_ns, err);
        if (lane == 0) {
          if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
          out[ps.lseg[s]] = P::finalize(start_value<P, WIDE>(Ops::pack(carry), P::unpack(ps.local[s])));
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&ps.slot_free[s]);
    }
  } else if (!REDUCE && warp < 2 * NC / 32) {
    // ------------------------------------------------------------ emitters
    const int t = threadIdx.x - NC;
    const uint32_t tcol = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(((t >> 5) >> 2) * kCols);
    RingPos rs, ro;
    for (long long it = 0;; ++it, rs.advance(1, SL), ro.advance(1, SO)) {
      if (t == 0) {
        int go = emitter_wait(p, ps, rs, it);
        if (go > 0 && !mbar_wait(&ps.slot_ready[rs.s], rs.ph, p.timeout_ns)) go = -1;
        if (!REDUCE && go > 0 && !mbar_wait(&ps.out_empty[ro.s], ro.ph ^ 1u, p.timeout_ns)) go = -1;
        if (go < 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        if (go == 0) {
          if (!REDUCE) mbar_arrive(&ps.emitted[ro.s]);
          RingPos r = rs;
          for (int j = 0; j < kLookWarps; ++j, r.advance(1, SL)) mbar_arrive(&ps.aggr[r.s]);
        }
        s_go[1] = go;
      }
      bar_named(2, NC);
      if (s_go[1] <= 0) break;
      const long long tile = ps.tile[rs.s];
      const unsigned long long info = info_all[(size_t)rs.s * NC + t];
      const Acc tex = texcl_all[(size_t)rs.s * NC + t];
      const Acc start = (info & kSegTexclF) ? tex : start_value<P, WIDE>(ps.carry[rs.s], tex);
      if constexpr (!REDUCE) {
        tmem_fence_after();
        uint32_t w[kCols];
        const uint32_t ta = tcol + (uint32_t)(rs.s * kSlotCols);
        if constexpr (kCols == 32) tmem_load32(ta, w);
        else tmem_load16(ta, w);
        tmem_fence_before();
        __syncwarp();
        if ((t & 31) == 0) mbar_arrive(&ps.slot_free[rs.s]);  // slot, carry and words read
        char *obuf = obase + (size_t)ro.s * p.out_stage_stride;
        constexpr int OPV = 16 / (int)sizeof(Out), VPTO = ITEMS / OPV, WPO = (int)sizeof(Out) / 4;
        const unsigned heads = (unsigned)(info & 0xffffffffull);
#pragma unroll
        for (int k = 0; k < VPTO; ++k) {
          uint4 u;
          Out *oe = reinterpret_cast<Out *>(&u);
#pragma unroll
          for (int q = 0; q < OPV; ++q) {
            const int j = k * OPV + q;
            Out r;
            memcpy(&r, w + j * WPO, sizeof(Out));
            const bool seen = (heads & (2u << j) - 1u) != 0;  // a head at or before j
            if (seen) oe[q] = r;
            else if constexpr (P::kCompensated) oe[q] = __fadd_rn(start.hi, __fadd_rn(start.lo, r));
            else oe[q] = P::finalize(P::combine(start, P::from_out(r)));
          }
          *reinterpret_cast<uint4 *>(obuf + swz(t * VPTO + k) * 16) = u;
        }
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
    }
  } else if (!REDUCE && warp < 2 * NC / 32 + kLookWarps) {
    // ------------------------------------------------------ look-back warps
    const int wi = warp - 2 * NC / 32;
    const int lane = threadIdx.x & 31;
    RingPos r;
    r.advance(wi, SL);
    for (long long it = wi;; it += kLookWarps, r.advance(kLookWarps, SL)) {
      const int s = r.s;
      const bool ok = __shfl_sync(0xffffffffu, (int)mbar_wait(&ps.aggr[s], r.ph, p.timeout_ns), 0) != 0;
      if (!ok) {
        if (lane == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        break;
      }
      if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
      const long long tile = ps.tile[s];
      const int sf = ps.sflags[s];
      typename Ops::Pub carry = Ops::identity();
      if (tile > 0 && (sf & kSegNeedCarry)) {
        bool err;
        carry = lookback<Ops, false>(p.status, tile, epoch_tag, p.timeout_ns, err);
        if (lane == 0) {
          if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
          if (!REDUCE && !(sf & kSegHasHead) && tile != p.stall_tile)
            st_status(p.status + tile, Ops::pack(Ops::combine(carry, Ops::unpack(ps.agg[s]))),
                      epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
        }
      }
      if (lane == 0) {
        ps.carry[s] = Ops::pack(carry);
        mbar_arrive(&ps.cready[s]);
      }
      __syncwarp();
    }
  } else if (warp == kWorkWarps + kLookWarps) {
    if ((threadIdx.x & 31) == 0)
      producer_loop(&tin, p, ps, smem, kRows, kBox, ps.tile_in, reinterpret_cast<const char *>(p.seg_rec),
                    smem + p.rec_base, (unsigned)(kSegRecInts * sizeof(int)), kGroups);
  } else if constexpr (!REDUCE) {
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
  if constexpr (!REDUCE) {
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
      tmem_fence_after();
      tmem_dealloc(tbase, 512);
    }
  }
  finish_launch(p.hdr, epoch, nullptr, 0);
}

// ------------------------------------------------------------------ host

// Shared-memory layout for (block, items): input stages, output stages
// (scan), per-slot thread prefixes and words (and entering-segment ends for
// a reduce), the per-stage tile records.  False when the shape does not fit.
template <class P, bool REDUCE>
bool seg_layout(TmaParams &p, int block, int items) {
  constexpr size_t es = sizeof(typename P::In), eo = sizeof(typename P::Out), ea = sizeof(typename P::Acc);
  const int cols = items * (int)eo / 4;
  if (cols != 16 && cols != 32) return false;
  const size_t in_b = (size_t)block * items * es, out_b = REDUCE ? 0 : (size_t)block * items * eo;
  int slots = REDUCE ? kMaxStages : std::min(kMaxStages, 512 / (cols * block / 128));
  const int so = REDUCE ? 1 : kScanOutStages;
  for (;; --slots) {
    if (slots < 2) return false;
    const size_t per_slot = REDUCE ? 0 : (size_t)block * (ea + 8);
    const size_t fixed = so * out_b + ((slots * per_slot + 1023) & ~size_t(1023));
    const size_t rec_b = kSegRecInts * sizeof(int);
    if (fixed + 4 * (in_b + rec_b) > kSmemBudget) continue;  // keep at least 4 input stages
    const int si = (int)std::min<size_t>(kScanMaxInStages, (kSmemBudget - fixed) / (in_b + rec_b));
    p.stages = si;
    p.stage_stride = (unsigned)in_b;
    p.slots = slots;
    p.out_stages = so;
    p.out_stage_stride = (unsigned)out_b;
    p.out_base = (unsigned)(si * in_b);
    p.texcl_base = (unsigned)(si * in_b + so * out_b);
    p.info_base = (unsigned)(p.texcl_base + (REDUCE ? 0 : (size_t)slots * block * ea));
    p.rend_base = (unsigned)(p.info_base + (REDUCE ? 0 : (size_t)slots * block * 8));
    p.rec_base = (unsigned)((p.rend_base + 15) & ~size_t(15));
    return true;
  }
}

template <class P, int NC, int ITEMS, bool WIDE, bool REDUCE>
int launch_seg_shape(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, cudaStream_t st) {
  constexpr int cols = tmem_cols<P, ITEMS>();
  constexpr int kEpr = 128 / (int)sizeof(typename P::In), kEprOut = 128 / (int)sizeof(typename P::Out);
  constexpr bool ok_shape = (cols == 16 || cols == 32) && (NC * ITEMS) % (8 * kEpr) == 0 &&
                            (NC * ITEMS) % (8 * kEprOut) == 0;
  if constexpr (!TmemExact<P>::value || !ok_shape) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    auto kfn = seg_tmem_kernel<P, NC, ITEMS, WIDE, REDUCE>;
    const size_t smem = (size_t)p.rec_base + (size_t)p.stages * kSegRecInts * sizeof(int) + 1024;
    int rc = ensure_dynamic_smem((const void *)kfn, smem);
    if (rc) return rc;
    const int threads = seg_threads(NC, REDUCE);
    if (occupancy((const void *)kfn, threads, smem) < 1) return B2P_ERR_UNSUPPORTED;
    const int grid = (int)std::min<long long>(p.ntiles, (long long)device_info().sm_count);
    kfn<<<grid, threads, smem, st>>>(tin, tout, p);
    return cuda_status(cudaGetLastError());
  }
}

template <class P, bool WIDE, bool REDUCE>
int launch_seg_items(TmaParams &p, const CUtensorMap &tin, const CUtensorMap &tout, int block, int items,
                     cudaStream_t st) {
  if (block == 128 && items == 16) return launch_seg_shape<P, 128, 16, WIDE, REDUCE>(p, tin, tout, st);
  if (block == 128 && items == 32) return launch_seg_shape<P, 128, 32, WIDE, REDUCE>(p, tin, tout, st);
  if (block == 256 && items == 8) return launch_seg_shape<P, 256, 8, WIDE, REDUCE>(p, tin, tout, st);
  if (block == 256 && items == 16) return launch_seg_shape<P, 256, 16, WIDE, REDUCE>(p, tin, tout, st);
  if (block == 256 && items == 32) return launch_seg_shape<P, 256, 32, WIDE, REDUCE>(p, tin, tout, st);
  return B2P_ERR_UNSUPPORTED;
}

template <class P>
int launch_seg_t(bool reduce, int inclusive, const void *in, void *out, const int64_t *offsets, int64_t nseg,
                 size_t n, const void *init, void *scratch, const int *seg_rec, int block, int items,
                 cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  const size_t es = sizeof(In), eo = sizeof(Out);
  const long long tile = (long long)block * items;
  TmaParams p{};
  const bool ok = reduce ? seg_layout<P, true>(p, block, items) : seg_layout<P, false>(p, block, items);
  if (!ok) return B2P_ERR_UNSUPPORTED;
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  const long long epr = 128 / (long long)es, epr_out = 128 / (long long)eo;
  p.rows_full = (long long)(n / (size_t)epr);
  p.tail_begin = (unsigned long long)p.rows_full * epr;
  p.rows_full_out = (long long)(n / (size_t)epr_out);
  p.tail_out_begin = (unsigned long long)p.rows_full_out * epr_out;
  if (p.rows_full < 1 || p.rows_full + tile / epr >= (1ll << 31) || p.rows_full_out + tile / epr_out >= (1ll << 31))
    return B2P_ERR_UNSUPPORTED;
  p.inclusive = reduce ? 1 : inclusive;
  p.in = in;
  p.out = out;
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix);
  p.timeout_ns = wait_timeout_ns();
  p.stall_tile = debug_stall_tile();
  p.has_init = init != nullptr;
  if (init) memcpy(&p.init_raw, init, sizeof(Out));
  p.offsets = reinterpret_cast<const long long *>(offsets);
  p.nseg = nseg;
  p.seg_rec = seg_rec;
  // a long compensated sum carries its look-back prefixes in FP64
  const bool wide = P::kCompensated && n > (1ull << 24);
  CUtensorMap tin, tout;
  if (!encode_row_tensor(&tin, in, (unsigned long long)p.rows_full, (int)std::min<long long>(256, tile / epr)))
    return B2P_ERR_UNSUPPORTED;
  if (reduce) {
    tout = tin;  // unused: a reduce writes one value per segment with plain stores
  } else if (!encode_row_tensor(&tout, out, (unsigned long long)std::max<long long>(p.rows_full_out, 1),
                                (int)std::min<long long>(256, tile / epr_out))) {
    return B2P_ERR_UNSUPPORTED;
  }
  if constexpr (P::kCompensated) {
    if (wide) {
      return reduce ? launch_seg_items<P, true, true>(p, tin, tout, block, items, st)
                    : launch_seg_items<P, true, false>(p, tin, tout, block, items, st);
    }
  }
  return reduce ? launch_seg_items<P, false, true>(p, tin, tout, block, items, st)
                : launch_seg_items<P, false, false>(p, tin, tout, block, items, st);
}

}  // namespace

bool segmented_tma_shape(int dtype, int op, int block, int items) {
  if (op != B2P_SUM) return false;
  if (dtype != B2P_I32 && dtype != B2P_I64 && dtype != B2P_U32 && dtype != B2P_U64 && dtype != B2P_F32 &&
      dtype != B2P_BF16)
    return false;
  const int cols = items * (int)acc_size(dtype) / 4;
  if (cols != 16 && cols != 32) return false;
  return (block == 128 && (items == 16 || items == 32)) || (block == 256 && (items == 8 || items == 16 || items == 32));
}

size_t segmented_tma_scratch(size_t n, int block, int items) {
  const size_t tile = (size_t)block * items;
  const size_t ntiles = (n + tile - 1) / tile;
  return kScratchPrefix + ntiles * (sizeof(StatusWord) + kSegRecInts * sizeof(int));
}

void segmented_tile_records(const int64_t *offs, int64_t nseg, size_t n, int block, int items, int *rec) {
  const size_t tile = (size_t)block * items;
  const size_t ntiles = (n + tile - 1) / tile;
  int64_t k = 0;
  for (size_t t = 0; t < ntiles; ++t) {
    const int64_t t0 = (int64_t)(t * tile), t1 = std::min<int64_t>(t0 + (int64_t)tile, (int64_t)n);
    while (k <= nseg && offs[k] < t0) ++k;
    int64_t ke = k;
    while (ke <= nseg && offs[ke] < t1) ++ke;
    // the last tile lists every boundary up to nseg (empty segments at n)
    const int64_t m = (t + 1 == ntiles ? nseg + 1 : std::min<int64_t>(ke + 1, nseg + 1)) - k;
    int *r = rec + t * kSegRecInts;
    r[0] = (int)k;
    r[1] = (int)m;
    for (int i = 0; i < kSegRecCap; ++i)
      r[2 + i] = i < m ? (int)std::min<int64_t>(offs[k + i] - t0, (int64_t)tile + 1) : 0;
  }
}

int launch_segmented_tma(int prim, int dtype, int op, int inclusive, const void *in, void *out,
                         const int64_t *offsets, int64_t nseg, size_t n, const void *init, void *scratch,
                         int block, int items, cudaStream_t st) {
  if (!segmented_tma_shape(dtype, op, block, items) || nseg <= 0 || nseg >= (1ll << 31) - 2) return B2P_ERR_UNSUPPORTED;
  const size_t tile = (size_t)block * items;
  const size_t ntiles = (n + tile - 1) / tile;
  const int *recs = reinterpret_cast<const int *>(reinterpret_cast<const char *>(scratch) + kScratchPrefix +
                                                  ntiles * sizeof(StatusWord));
  const bool reduce = prim == B2P_PRIM_SEG_REDUCE;
  switch (dtype) {
  case B2P_I32:
    return launch_seg_t<PolicyOf<B2P_I32, B2P_SUM>::type>(reduce, inclusive, in, out, offsets, nseg, n, init, scratch,
                                                          recs, block, items, st);
  case B2P_I64:
    return launch_seg_t<PolicyOf<B2P_I64, B2P_SUM>::type>(reduce, inclusive, in, out, offsets, nseg, n, init, scratch,
                                                          recs, block, items, st);
  case B2P_U32:
    return launch_seg_t<PolicyOf<B2P_U32, B2P_SUM>::type>(reduce, inclusive, in, out, offsets, nseg, n, init, scratch,
                                                          recs, block, items, st);
  case B2P_U64:
    return launch_seg_t<PolicyOf<B2P_U64, B2P_SUM>::type>(reduce, inclusive, in, out, offsets, nseg, n, init, scratch,
                                                          recs, block, items, st);
  case B2P_F32:
    return launch_seg_t<PolicyOf<B2P_F32, B2P_SUM>::type>(reduce, inclusive, in, out, offsets, nseg, n, init, scratch,
                                                          recs, block, items, st);
  case B2P_BF16:
    return launch_seg_t<PolicyOf<B2P_BF16, B2P_SUM>::type>(reduce, inclusive, in, out, offsets, nseg, n, init,
                                                           scratch, recs, block, items, st);
  default:
    return B2P_ERR_UNSUPPORTED;
  }
}

}  // namespace b2p
