// The TMEM-staged pipelined copy_if, shared by libb2p (b2p_copy_if, whose
// predicate is (bits & mask) CMP rhs) and the header-only C++ layer
// (hipsycl::algorithms::copy_if and std::copy_if with any predicate
// functor or lambda).  Replaces the reference's compaction through a 64-bit
// exclusive flag scan (algorithms/algorithm.hpp:178-243) with one pass:
// a tile's aggregate is its kept count, its carry is the output position of
// its first kept element.
#pragma once

#include "pipe.cuh"

#include <atomic>

namespace b2p {

// (bits of v & mask) CMP rhs, compared as unsigned: the predicate family of
// the C-ABI.
template <class T, int CMP>
struct MaskCmp {
  unsigned long long mask, rhs;
  __device__ __forceinline__ bool operator()(const T &v) const {
    using U = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
    U u;
    memcpy(&u, &v, sizeof(T));
    const U a = u & (U)mask, r = (U)rhs;
    if constexpr (CMP == B2P_CMP_LT) return a < r;
    else if constexpr (CMP == B2P_CMP_LE) return a <= r;
    else if constexpr (CMP == B2P_CMP_EQ) return a == r;
    else if constexpr (CMP == B2P_CMP_NE) return a != r;
    else if constexpr (CMP == B2P_CMP_GE) return a >= r;
    else return a > r;
  }
};

// -------------------------------------------------- copy_if, TMEM-staged
//
// copy_if_tma_kernel's compaction with the TMEM staging of scan_tmem_kernel:
// reducers park each thread's raw elements in a TMEM slot (keep masks and
// thread offsets beside it in shared memory) and hand the input stage back
// at once; emitters pack the kept elements into an output stage.
//
// Thread t owns elements t * ITEMS .. t * ITEMS + ITEMS - 1 (16-byte reads
// of the swizzled stage) and packs them in order.  Both groups work through
// one tile at a time, so the per-element work is kept to a few instructions;
// the price is bank conflicts in the packing stores for regular keep patterns
// (every lane keeping 32 elements puts all 32 lanes of a store on one bank),
// where the pipeline falls to about 1.8 TB/s.  A warp-striped layout with
// ballot packing, and lane-rotated element order, were both measured: free
// of conflicts, but slower at typical selectivities.

// Keep bits of a thread's ITEMS elements (w: the elements as 32-bit words,
// element j at tile index first + j); only the first `count` elements of the
// tile are real.
template <class T, int ITEMS, class Pred>
__device__ __forceinline__ unsigned keep_bits(const uint32_t *w, const Pred &pred, int first, int count) {
  unsigned keep = 0;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    T e;
    memcpy(&e, w + j * (int)(sizeof(T) / 4), sizeof(T));
    keep |= (unsigned)static_cast<bool>(pred(e)) << j;
  }
  if (count < first + ITEMS) keep &= count <= first ? 0u : ((1u << (count - first)) - 1u);  // count - first < 32 here
  return keep;
}

// Exclusive scan of one 32-bit count per thread over the NC threads of a
// warp group with one named barrier: warp totals through s_cnt (NC / 32
// words, written again only after a later barrier of the group), then every
// thread adds the totals of the warps before its own.
template <int NC>
__device__ __forceinline__ unsigned count_scan_1bar(unsigned v, unsigned *s_cnt, unsigned *total, int t, int bar) {
  const int lane = t & 31, warp = t >> 5;
  unsigned incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned o = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += o;
  }
  if (lane == 31) s_cnt[warp] = incl;
  bar_named(bar, NC);
  unsigned before = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < NC / 32; ++w) {
    const unsigned c = s_cnt[w];
    before += w < warp ? c : 0u;
    tot += c;
  }
  *total = tot;
  return before + incl - v;
}

template <class T, int NC, int ITEMS, class Pred>
__global__ void __launch_bounds__(pipe_threads(NC), 1)
    copy_if_tmem_kernel(const __grid_constant__ CUtensorMap tin, TmaParams p, Pred pred) {
  constexpr int kTile = NC * ITEMS;
  constexpr int kEpr = 128 / (int)sizeof(T);
  static_assert(kTile % (8 * kEpr) == 0, "a stage is a whole number of 1024-byte swizzle atoms");
  constexpr int kRows = kTile / kEpr;
  constexpr int kBox = kRows < 256 ? kRows : 256;
  static_assert(kRows % kBox == 0, "box rows");
  static_assert(ITEMS <= 32, "keep mask is 32 bits");
  static_assert(kTile <= 65536, "thread offsets are 16 bits");
  constexpr int kCols = ITEMS * (int)sizeof(T) / 4;
  static_assert(kCols == 16 || kCols == 32, "TMEM columns per thread");
  static_assert(NC % 128 == 0, "reducer and emitter groups cover the four TMEM lane quarters evenly");
  constexpr int kSlotCols = kCols * (NC / 128);

  extern __shared__ char smem_raw[];
  char *smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  char *obase = smem + p.out_base;
  unsigned *keep_all = reinterpret_cast<unsigned *>(smem + p.texcl_base);
  uint16_t *texcl_all = reinterpret_cast<uint16_t *>(keep_all + (size_t)p.slots * NC);  // offsets < 2^16
  __shared__ __align__(8) PipeState ps;
  __shared__ unsigned s_cnt[NC / 32];
  __shared__ int s_go[2];

  const int warp = threadIdx.x >> 5;
  // aggr completes when every reducer warp has parked its part of the tile
  tmem_pipe_init(ps, p, NC / 32, NC / 32);
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
  const int SI = p.stages, SL = p.slots, SO = p.out_stages;
  const long long last = p.ntiles - 1;
  const int ntail = (int)(p.n - p.tail_begin);
  T *out = reinterpret_cast<T *>(p.out);

  if (warp < NC / 32) {
    // ------------------------------------------------------------ reducers
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
      if (tile == last && ntail > 0) load_row_tail<T, NC>(p, buf, tile, kTile);
      uint32_t w[kCols];
#pragma unroll
      for (int k = 0; k < kCols / 4; ++k) {
        const uint4 u = *reinterpret_cast<const uint4 *>(buf + swz(t * (kCols / 4) + k) * 16);
        w[4 * k] = u.x;
        w[4 * k + 1] = u.y;
        w[4 * k + 2] = u.z;
        w[4 * k + 3] = u.w;
      }
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.empty[ri.s]);  // this warp is done with the input stage
      // the predicate first: it waits for the shared loads, and the TMEM
      // stores after it then issue without waiting
      const int count = (int)min((unsigned long long)kTile, p.n - (unsigned long long)tile * kTile);
      const unsigned keep = keep_bits<T, ITEMS>(w, pred, t * ITEMS, count);
      const uint32_t ta = tcol + (uint32_t)(rs.s * kSlotCols);
      tmem_st16(ta, w);
      if constexpr (kCols == 32) tmem_st16(ta + 16, w + 16);
      unsigned kept32;
      const unsigned ex = count_scan_1bar<NC>((unsigned)__popc(keep), s_cnt, &kept32, t, 1);
      const unsigned long long tile_kept = kept32;
      if (t == 0) {  // the kept count goes out as soon as the count scan knows it
        if (tile != p.stall_tile)
          st_status(p.status + tile, tile_kept, epoch_tag | (tile == 0 ? kFlagPrefix : kFlagAgg));
        ps.tile[rs.s] = tile;
        ps.agg[rs.s] = tile_kept;
      }
      texcl_all[(size_t)rs.s * NC + t] = (uint16_t)ex;
      keep_all[(size_t)rs.s * NC + t] = keep;
      tmem_wait_st();
      tmem_fence_before();
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.aggr[rs.s]);  // this warp's slot columns, masks and offsets
    }
    if (t == 0) *reinterpret_cast<volatile long long *>(&ps.end_item) = it;
  } else if (warp < 2 * NC / 32) {
    // ------------------------------------------------------------ emitters
    const int t = threadIdx.x - NC;
    const uint32_t tcol = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(((t >> 5) >> 2) * kCols);
    RingPos rs, ro;
    for (long long it = 0;; ++it, rs.advance(1, SL), ro.advance(1, SO)) {
      if (t == 0) {
        int go = emitter_wait(p, ps, rs, it);
        if (go > 0 && !mbar_wait(&ps.out_empty[ro.s], ro.ph ^ 1u, p.timeout_ns)) go = -1;
        if (go < 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        if (go == 0) {
          // end the store warp and the look-back warps (waiting on items it ..
          // it + kLookWarps - 1, each barrier completing after NC / 32 arrivals)
          mbar_arrive(&ps.emitted[ro.s]);
          RingPos r = rs;
          for (int j = 0; j < kLookWarps; ++j, r.advance(1, SL))
            for (int k = 0; k < NC / 32; ++k) mbar_arrive(&ps.aggr[r.s]);
        }
        s_go[1] = go;
      }
      bar_named(2, NC);
      if (s_go[1] <= 0) break;
      tmem_fence_after();
      const long long tile = ps.tile[rs.s];
      const unsigned long long carry = ps.carry[rs.s];
      unsigned long long kept_total = ps.agg[rs.s];
      const bool broken = carry > p.n || kept_total > p.n - carry;
      if (broken) {  // only after a broken chain: write nothing
        if (t == 0) record_error(p.hdr, B2P_ERR_TIMEOUT);
        kept_total = 0;
      }
      const unsigned keep = keep_all[(size_t)rs.s * NC + t];
      const unsigned o = texcl_all[(size_t)rs.s * NC + t];
      uint32_t w[kCols];
      const uint32_t ta = tcol + (uint32_t)(rs.s * kSlotCols);
      if constexpr (kCols == 32) tmem_load32(ta, w);
      else tmem_load16(ta, w);
      tmem_fence_before();
      __syncwarp();
      if ((t & 31) == 0) mbar_arrive(&ps.slot_free[rs.s]);  // slot, masks and offsets read
      char *obuf = obase + (size_t)ro.s * p.out_stage_stride;
      const uintptr_t g0 = reinterpret_cast<uintptr_t>(out + carry);
      const unsigned phase = (unsigned)(g0 & 15u);
      if (!broken) {
        T *ob = reinterpret_cast<T *>(obuf + phase) + o;  // phase is a multiple of sizeof(T)
        unsigned pos = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
          const unsigned b = (keep >> j) & 1u;
          if (b) {
            T v;
            memcpy(&v, w + j * (int)(sizeof(T) / 4), sizeof(T));
            ob[pos] = v;
          }
          pos += b;
        }
      }
      fence_async_smem();
      bar_named(2, NC);  // the output stage is packed
      if (t == 0 && tile == last && p.num_copied) *p.num_copied = carry + kept_total;
      if (t == 0) {
        ps.out_carry[ro.s] = carry;
        ps.out_count[ro.s] = kept_total;
        mbar_arrive(&ps.emitted[ro.s]);
      }
    }
  } else if (warp < 2 * NC / 32 + kLookWarps) {
    lookback_loop<CountOps>(p, ps, warp - 2 * NC / 32, 0ull, epoch_tag, SL);
  } else if (warp == 2 * NC / 32 + kLookWarps) {
    if ((threadIdx.x & 31) == 0) producer_loop(&tin, p, ps, smem, kRows, kBox, ps.tile_in);
  } else {
    // ---------------------------------------------------------- store warp
    if ((threadIdx.x & 31) == 0) {
      RingPos ro;
      for (long long it = 0;; ++it, ro.advance(1, SO)) {
        if (!mbar_wait(&ps.emitted[ro.s], ro.ph, p.timeout_ns)) {
          record_error(p.hdr, B2P_ERR_TIMEOUT);
          break;
        }
        if (it >= *reinterpret_cast<volatile long long *>(&ps.end_item)) break;
        const unsigned long long carry = ps.out_carry[ro.s];
        const unsigned long long kept_total = ps.out_count[ro.s];
        const uintptr_t g0 = reinterpret_cast<uintptr_t>(out + carry);
        const uintptr_t g1 = g0 + kept_total * sizeof(T);
        const uintptr_t a0 = (g0 + 15) & ~uintptr_t(15), a1 = g1 & ~uintptr_t(15);
        const char *obuf = obase + (size_t)ro.s * p.out_stage_stride + (g0 & 15u);  // output element 0
        // the elements before the first and after the last 16-byte boundary
        // (fewer than 16 bytes each; all of them when no boundary pair
        // encloses a block): plain stores
        const long long nhead = a1 > a0 ? (long long)((a0 - g0) / sizeof(T)) : (long long)kept_total;
        const long long tail0 = a1 > a0 ? (long long)((a1 - g0) / sizeof(T)) : (long long)kept_total;
        for (long long k = 0; k < nhead; ++k) out[carry + k] = reinterpret_cast<const T *>(obuf)[k];
        for (long long k = tail0; k < (long long)kept_total; ++k) out[carry + k] = reinterpret_cast<const T *>(obuf)[k];
        if (a1 > a0) {
          const char *src = obuf + (a0 - g0);
          asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(a0),
                       "r"(smem_u32(src)), "r"((unsigned)(a1 - a0))
                       : "memory");
        }
        bulk_commit();
        bulk_wait_read<0>();
        mbar_arrive(&ps.out_empty[ro.s]);
      }
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



// ------------------------------------------------------------------ host

// Shared-memory layout of the TMEM-staged copy_if for (block, items):
// input stages, two output stages (a tile plus 1024 bytes for the output's
// 16-byte phase), thread offsets and keep masks of every slot.  Leaves
// p.slots = 0 (in-place kernel) when the shape has no TMEM kernel.
inline bool copy_tmem_layout(TmaParams &p, size_t es, int block, int items) {
  p.slots = 0;
  if (!kUseTmem || (block != 128 && block != 256)) return false;
  const int cols = items * (int)es / 4;
  if (cols != 16 && cols != 32) return false;
  const int slots = std::min(kMaxStages, 512 / (cols * block / 128));
  const size_t in_b = (size_t)block * items * es, out_b = in_b + 1024;
  const size_t side = ((size_t)slots * block * 6 + 1023) & ~size_t(1023);
  const int so = kCopyOutStages;
  if (so * out_b + side + 2 * in_b > kSmemBudget) return false;
  const int si = (int)std::min<size_t>(kMaxStages, (kSmemBudget - so * out_b - side) / in_b);
  p.stages = si;
  p.stage_stride = (unsigned)in_b;
  p.slots = slots;
  p.out_stages = so;
  p.out_stage_stride = (unsigned)out_b;
  p.out_base = (unsigned)(si * in_b);
  p.texcl_base = (unsigned)(si * in_b + so * out_b);
  return true;
}

// Launch state of one kernel on one device: the dynamic shared-memory
// attribute raised and the occupancy checked once.
template <auto K>
struct KernelOnce {
  static inline std::atomic<int> state[64];  // 0 unknown, 1 runnable, 2 not runnable
};

// Launch copy_if_tmem_kernel for a layout made by copy_tmem_layout.
// Returns B2P_ERR_UNSUPPORTED, having launched nothing, when the shape has
// no TMEM kernel or does not fit on the device.
template <class T, int NC, int ITEMS, class Pred>
int launch_copy_tmem_shape(TmaParams &p, const CUtensorMap &tin, const Pred &pred, int sm_count, cudaStream_t st) {
  constexpr int cols = ITEMS * (int)sizeof(T) / 4;
  if constexpr (cols != 16 && cols != 32) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    auto kfn = copy_if_tmem_kernel<T, NC, ITEMS, Pred>;
    const size_t smem = p.texcl_base + (size_t)p.slots * NC * 6 + 1024;
    int dev = 0;
    cudaGetDevice(&dev);
    std::atomic<int> &st_once = KernelOnce<copy_if_tmem_kernel<T, NC, ITEMS, Pred>>::state[dev & 63];
    if (st_once.load() == 0) {
      int nb = 0;
      bool ok = cudaFuncSetAttribute((const void *)kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                cudaSuccess;
      ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)kfn, pipe_threads(NC), smem) ==
                     cudaSuccess && nb >= 1;
      if (!ok) cudaGetLastError();
      st_once.store(ok ? 1 : 2);
    }
    if (st_once.load() != 1) return B2P_ERR_UNSUPPORTED;
    const int grid = (int)std::min<long long>(p.ntiles, (long long)sm_count);
    kfn<<<grid, pipe_threads(NC), smem, st>>>(tin, p, pred);
    return cudaGetLastError() == cudaSuccess ? B2P_OK : B2P_ERR_CUDA;
  }
}

// Pipelined copy_if of `n` elements of T (4 or 8 bytes) with any predicate
// functor: the TMEM-staged kernel for tile shapes (128 x 32), (256 x 16),
// (256 x 32).  `in` 16-byte aligned, n at least one tile, scratch a
// zero-initialised libb2p scratch buffer (header + one status word per
// tile).  Returns B2P_ERR_UNSUPPORTED, having launched nothing, when the
// call does not fit.
template <class T, class Pred>
int launch_copy_if_pred(const T *in, T *out, size_t n, const Pred &pred, unsigned long long *num_copied,
                        void *scratch, int block, int items, int sm_count, unsigned long long timeout_ns,
                        long long stall_tile, cudaStream_t st) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "pipelined copy_if: 4- or 8-byte elements");
  const size_t es = sizeof(T);
  const long long tile = (long long)block * items;
  if ((reinterpret_cast<uintptr_t>(in) & 15) || (reinterpret_cast<uintptr_t>(scratch) & 255) ||
      n < (size_t)tile)
    return B2P_ERR_UNSUPPORTED;
  TmaParams p{};
  if (!copy_tmem_layout(p, es, block, items)) return B2P_ERR_UNSUPPORTED;
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  const long long epr = 128 / (long long)es;
  p.rows_full = (long long)(n / (size_t)epr);
  p.tail_begin = (unsigned long long)p.rows_full * epr;
  if (p.rows_full + tile / epr >= (1ll << 31)) return B2P_ERR_UNSUPPORTED;
  p.in = in;
  p.out = out;
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix);
  p.timeout_ns = timeout_ns;
  p.stall_tile = stall_tile;
  p.num_copied = num_copied;
  CUtensorMap tin;
  if (!encode_row_tensor(&tin, in, (unsigned long long)p.rows_full, (int)std::min<long long>(256, tile / epr)))
    return B2P_ERR_UNSUPPORTED;
  if (block == 128 && items == 32) return launch_copy_tmem_shape<T, 128, 32>(p, tin, pred, sm_count, st);
  if (block == 256 && items == 16) return launch_copy_tmem_shape<T, 256, 16>(p, tin, pred, sm_count, st);
  if (block == 256 && items == 32) return launch_copy_tmem_shape<T, 256, 32>(p, tin, pred, sm_count, st);
  return B2P_ERR_UNSUPPORTED;
}

}  // namespace b2p
