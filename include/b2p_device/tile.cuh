// Tile-level building blocks shared by the scan, copy_if and segmented
// kernels: the swizzled shared-memory tile, cache-hinted global accesses,
// block scans, the bounded warp-parallel look-back and the launch epilogue.
#pragma once

#include "common.cuh"

namespace b2p {

// ------------------------------------------------------------ shared tile

// 16-byte-granular XOR swizzle of a shared tile: vector v lives in slot
// v ^ ((v >> 3) & 7).  Conflict-free for striped 16-byte accesses and for
// blocked 16-byte accesses of 1, 2, 4 or 8 vectors per thread.
__device__ __forceinline__ int swz(int v) { return v ^ ((v >> 3) & 7); }

template <class T>
__device__ __forceinline__ T *smem_elem_ptr(char *tile, int i) {
  const int byte = i * (int)sizeof(T);
  return reinterpret_cast<T *>(tile + swz(byte >> 4) * 16 + (byte & 15));
}

// L2 residency policies (createpolicy): inputs read twice are kept
// (evict_last) on the first read and released (evict_first) on the last.
__device__ __forceinline__ unsigned long long l2_policy_keep() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_policy_stream() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint4 ld_hint_v4(const void *p, unsigned long long pol) {
  uint4 r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ void cp_async16_hint(void *smem_dst, const void *gsrc,
                                                unsigned long long pol) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc),
               "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Start bringing a tile into the swizzled shared buffer: cp.async for a full
// 16-byte aligned tile (completes in the background, no registers), a
// synchronous element copy otherwise.  Commits exactly one cp.async group.
template <class T>
__device__ __forceinline__ void prefetch_tile(char *buf, const T *src, int count, int tile_elems,
                                              bool vec, unsigned long long pol) {
  if (vec && count == tile_elems) {
    const int nv = tile_elems * (int)sizeof(T) / 16;
    const char *g = reinterpret_cast<const char *>(src);
    for (int v = threadIdx.x; v < nv; v += blockDim.x)
      cp_async16_hint(buf + swz(v) * 16, g + (size_t)v * 16, pol);
  } else {
    for (int i = threadIdx.x; i < count; i += blockDim.x) *smem_elem_ptr<T>(buf, i) = src[i];
  }
  cp_async_commit();
}

// Copy `count` elements of a tile from global memory into the swizzled
// shared buffer (16-byte striped loads for a full aligned tile).
template <class T>
__device__ __forceinline__ void load_tile_smem(char *buf, const T *src, int count, int tile_elems,
                                               bool vec, unsigned long long pol) {
  if (vec && count == tile_elems) {
    const int nv = tile_elems * (int)sizeof(T) / 16;
    const char *g = reinterpret_cast<const char *>(src);
    for (int v = threadIdx.x; v < nv; v += blockDim.x)
      *reinterpret_cast<uint4 *>(buf + swz(v) * 16) = ld_hint_v4(g + (size_t)v * 16, pol);
  } else {
    for (int i = threadIdx.x; i < count; i += blockDim.x) *smem_elem_ptr<T>(buf, i) = src[i];
  }
}

// Store `count` elements from the swizzled shared buffer (streaming stores).
template <class T>
__device__ __forceinline__ void store_tile(const char *tile, T *dst, int count, int tile_elems,
                                           bool vec) {
  if (vec && count == tile_elems) {
    const int nv = tile_elems * (int)sizeof(T) / 16;
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    for (int v = threadIdx.x; v < nv; v += blockDim.x)
      st_stream_v4(d + v, *reinterpret_cast<const uint4 *>(tile + swz(v) * 16));
  } else {
    for (int i = threadIdx.x; i < count; i += blockDim.x)
      dst[i] = *smem_elem_ptr<T>(const_cast<char *>(tile), i);
  }
}

// ------------------------------------------------------- published values
//
// "Ops" describe the value carried between tiles: the accumulator of the
// element policy, an FP64 carry (fp32/bf16 SUM scans longer than 2^24), or
// an element count (copy_if).

template <class P>
struct AccOps {
  using Pub = typename P::Acc;
  __device__ static Pub identity() { return P::identity(); }
  __device__ static Pub combine(Pub a, Pub b) { return P::combine(a, b); }
  __device__ static Pub unpack(unsigned long long v) { return P::unpack(v); }
  __device__ static unsigned long long pack(Pub v) { return P::pack(v); }
};

struct F64Ops {
  using Pub = double;
  __device__ static double identity() { return 0.0; }
  __device__ static double combine(double a, double b) { return a + b; }
  __device__ static double unpack(unsigned long long v) { return __longlong_as_double((long long)v); }
  __device__ static unsigned long long pack(double v) { return (unsigned long long)__double_as_longlong(v); }
};

struct CountOps {
  using Pub = unsigned long long;
  __device__ static unsigned long long identity() { return 0; }
  __device__ static unsigned long long combine(unsigned long long a, unsigned long long b) {
    return a + b;
  }
  __device__ static unsigned long long unpack(unsigned long long v) { return v; }
  __device__ static unsigned long long pack(unsigned long long v) { return v; }
};

// Block-wide inclusive scan of one value per thread with a generic combine
// (shuffles inside warps, shared memory across warps).  Returns the
// thread's exclusive prefix; *total receives the block total.  s_warp needs
// 32 slots.  Contains __syncthreads.
template <class Ops>
__device__ __forceinline__ typename Ops::Pub block_exclusive_scan(typename Ops::Pub v,
                                                                  typename Ops::Pub *s_warp,
                                                                  typename Ops::Pub *total) {
  using Pub = typename Ops::Pub;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  Pub incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Pub o = shfl_up(incl, d);
    if (lane >= d) incl = Ops::combine(o, incl);
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    Pub w = lane < nwarps ? s_warp[lane] : Ops::identity();
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      Pub o = shfl_up(w, d);
      if (lane >= d) w = Ops::combine(o, w);
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  Pub ex = shfl_up(incl, 1);
  if (lane == 0) ex = Ops::identity();
  if (warp > 0) ex = Ops::combine(s_warp[warp - 1], ex);
  *total = s_warp[nwarps - 1];
  return ex;
}

// ------------------------------------------------------------ look-back

__device__ __forceinline__ void record_error(ScratchHeader *hdr, unsigned code) {
  atomicCAS(&hdr->error, 0u, code);
}

// Warp-parallel look-back (called by all 32 lanes of one warp).  One step
// inspects kLookW x 32 predecessors: lane l watches tiles win - l - 32 j for
// j < kLookW, so the prefix frontier advances up to 128 tiles per L2 round
// trip.  The warp polls jointly and waits only for the predecessors nearer
// than the closest one whose inclusive prefix is published, then combines
// their payloads.  Every wait is bounded by timeout_ns (%globaltimer,
// checked every 64 polls); predecessors still missing at the deadline count
// as broken links.  Returns the exclusive prefix; sets err when the chain is
// broken.  kBackoff: sleep between polls (blocks that wait inline); a
// dedicated look-back warp polls without sleeping.
constexpr int kLookW = 4;

// W words per lane and step (W x 32 predecessors per L2 round trip).
template <class Ops, int W, bool kBackoff>
__device__ typename Ops::Pub lookback_w(const StatusWord *status, long long tile,
                                        unsigned long long epoch_tag, unsigned long long timeout_ns,
                                        bool &err);

template <class Ops, bool kBackoff = true>
__device__ __forceinline__ typename Ops::Pub lookback(const StatusWord *status, long long tile,
                                                      unsigned long long epoch_tag,
                                                      unsigned long long timeout_ns, bool &err) {
  return lookback_w<Ops, kLookW, kBackoff>(status, tile, epoch_tag, timeout_ns, err);
}

template <class Ops, int W, bool kBackoff>
__device__ typename Ops::Pub lookback_w(const StatusWord *status, long long tile,
                                        unsigned long long epoch_tag, unsigned long long timeout_ns,
                                        bool &err) {
  constexpr int kLookW = W;
  using Pub = typename Ops::Pub;
  const int lane = threadIdx.x & 31;
  Pub acc = Ops::identity();
  long long win = tile - 1;
  err = false;
  uint64_t t0 = 0;
  while (true) {
    bool have[kLookW];
    unsigned long long payload[kLookW];
    unsigned flags[kLookW];
#pragma unroll
    for (int j = 0; j < kLookW; ++j) {
      have[j] = (win - lane - 32 * j) < 0;  // never needed: tile 0 always publishes a prefix
      payload[j] = 0;
      flags[j] = have[j] ? (unsigned)kFlagPrefix : 0u;
    }
    int jstop = kLookW, lstop = 31;
    for (unsigned it = 0;; ++it) {
#pragma unroll
      for (int j = 0; j < kLookW; ++j) {
        if (!have[j]) {
          StatusWord w = ld_status(status + (win - lane - 32 * j));
          if ((w.meta & ~0xffull) == epoch_tag && (w.meta & (kFlagAgg | kFlagPrefix))) {
            have[j] = true;
            payload[j] = w.payload;
            flags[j] = (unsigned)(w.meta & 0xff);
          }
        }
      }
      bool ok = true;
      jstop = kLookW;
#pragma unroll
      for (int j = 0; j < kLookW; ++j) {
        const unsigned hm = __ballot_sync(0xffffffffu, have[j]);
        const unsigned sm = __ballot_sync(0xffffffffu, have[j] && (flags[j] & (kFlagPrefix | kFlagError)));
        if (jstop == kLookW && ok) {
          if (sm) {
            jstop = j;
            lstop = __ffs(sm) - 1;
            const unsigned need = (2u << lstop) - 1u;
            ok = (hm & need) == need;
          } else {
            ok = hm == 0xffffffffu;
          }
        }
      }
      if (ok) break;
      if (kBackoff && it >= 8) __nanosleep(it < 64 ? 32 : 256);
      if ((it & 63) == 63) {
        uint64_t now = __shfl_sync(0xffffffffu, globaltimer_ns(), 0);
        if (t0 == 0) {
          t0 = now;
        } else if (now - t0 > timeout_ns) {
#pragma unroll
          for (int j = 0; j < kLookW; ++j)
            if (!have[j]) {
              have[j] = true;
              flags[j] = (unsigned)kFlagError;
            }
        }
      }
    }
    Pub v = Ops::identity();
#pragma unroll
    for (int j = 0; j < kLookW; ++j) {
      const bool take = (j < jstop || (j == jstop && lane <= lstop)) &&
                        (win - lane - 32 * j) >= 0 && !(flags[j] & kFlagError);
      if (take) v = Ops::combine(v, Ops::unpack(payload[j]));
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v = Ops::combine(v, shfl_xor(v, m));
    acc = Ops::combine(v, acc);
    if (jstop < kLookW) {
      unsigned sf = 0;
#pragma unroll
      for (int j = 0; j < kLookW; ++j) {
        const unsigned f = __shfl_sync(0xffffffffu, flags[j], lstop);
        if (j == jstop) sf = f;
      }
      err = (sf & kFlagError) != 0;
      return acc;
    }
    win -= 32 * kLookW;
  }
}

// Bounded wait (one thread) for a status word of this launch carrying
// `flag`.  Returns its payload; *err is set on time-out or when the word
// carries kFlagError.
__device__ __forceinline__ unsigned long long wait_flag(const StatusWord *w,
                                                        unsigned long long epoch_tag,
                                                        unsigned long long flag,
                                                        unsigned long long timeout_ns, bool *err) {
  uint64_t t0 = 0;
  for (unsigned it = 0;; ++it) {
    StatusWord s = ld_status(w);
    if ((s.meta & ~0xffull) == epoch_tag && (s.meta & flag)) {
      __threadfence();  // acquire: data published before the flag is visible
      if (s.meta & kFlagError) *err = true;
      return s.payload;
    }
    if (it >= 8) __nanosleep(it < 64 ? 64 : 512);
    if ((it & 63) == 63) {
      uint64_t now = globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > timeout_ns) {
        *err = true;
        return 0;
      }
    }
  }
}

// Launch epilogue: the last block to arrive resets the tile counter and the
// per-launch counters and advances the epoch.  Every block has fetched its
// terminating work id and read the epoch before it arrives.
__device__ __forceinline__ void finish_launch(ScratchHeader *hdr, unsigned long long epoch,
                                              unsigned *counters, long long ncounters) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicInc(&hdr->done_ctr, gridDim.x - 1);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  for (long long i = threadIdx.x; i < ncounters; i += blockDim.x) counters[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicExch(&hdr->tile_ctr, 0ull);
    atomicExch(&hdr->epoch, epoch + 1ull);
  }
}

}  // namespace b2p
