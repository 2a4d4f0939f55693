// Single-pass scan and order-preserving copy_if (decoupled look-back).
//
// Replaces algorithms/scan/decoupled_lookback_scan.hpp:555-655 (init kernel
// + main kernel of 128 work-items x 16 items, Kogge-Stone in local memory,
// serial one-predecessor look-back on separate status/value words, unbounded
// spin at :244-246) and the copy_if built on it (algorithms/algorithm.hpp:
// 178-243, a 64-bit exclusive flag scan that reads the input twice).
//
// Here, per tile of BLOCK x ITEMS elements:
//   1. dynamic tile id (atomicAdd), so a tile's predecessors have all
//      started before it waits on them;
//   2. 16-byte coalesced loads into a swizzled shared-memory tile, then each
//      thread scans ITEMS consecutive elements in registers (fp32/bf16 SUM
//      with compensated TwoSum arithmetic);
//   3. block scan of the thread totals with warp shuffles;
//   4. warp 0 publishes the tile aggregate and runs a warp-parallel
//      look-back over 32 predecessors per step.  Status and payload share one
//      128-bit word tagged with the launch's epoch, so stale words from an
//      earlier launch are never mistaken for current ones and the status
//      array never needs clearing.  Every wait is bounded (%globaltimer);
//      on time-out the chain is marked broken and the error is recorded;
//   5. outputs go back through the shared tile for coalesced stores.
// fp32/bf16 SUM scans longer than 2^24 carry the cross-tile prefix in FP64.
#include "common.cuh"
#include "internal.h"

#include <algorithm>

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
  StatusWord *status;
  unsigned long long timeout_ns;
  long long stall_tile;
  // copy_if
  unsigned long long mask, rhs;
  int cmp;
  unsigned long long *num_copied;
};

// 16-byte-granular XOR swizzle of the shared tile: vector v lives in slot
// v ^ ((v >> 3) & 7).  Conflict-free for striped 16-byte writes and for
// blocked 16-byte reads of 1, 2, 4 or 8 vectors per thread.
__device__ __forceinline__ int swz(int v) { return v ^ ((v >> 3) & 7); }

template <class T>
__device__ __forceinline__ T *smem_elem_ptr(char *tile, int i) {
  const int byte = i * (int)sizeof(T);
  return reinterpret_cast<T *>(tile + swz(byte >> 4) * 16 + (byte & 15));
}

// Load `count` elements of a tile into the swizzled shared buffer.
template <class T>
__device__ __forceinline__ void load_tile(char *tile, const T *src, int count, int tile_elems,
                                          bool vec) {
  if (vec && count == tile_elems) {
    const int nv = tile_elems * (int)sizeof(T) / 16;
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    for (int v = threadIdx.x; v < nv; v += blockDim.x)
      *reinterpret_cast<uint4 *>(tile + swz(v) * 16) = ld_stream_v4(s + v);
  } else {
    for (int i = threadIdx.x; i < count; i += blockDim.x) *smem_elem_ptr<T>(tile, i) = src[i];
  }
}

// Store `count` elements from the swizzled shared buffer.
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

// Read this thread's ITEMS consecutive elements (blocked arrangement).
template <class T, int ITEMS>
__device__ __forceinline__ void read_blocked(const char *tile, T (&x)[ITEMS]) {
  constexpr int BYTES = ITEMS * (int)sizeof(T);
  const int t = threadIdx.x;
  if constexpr (BYTES % 16 == 0) {
    constexpr int VPT = BYTES / 16;
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      uint4 w = *reinterpret_cast<const uint4 *>(tile + swz(t * VPT + k) * 16);
      const T *e = reinterpret_cast<const T *>(&w);
#pragma unroll
      for (int j = 0; j < 16 / (int)sizeof(T); ++j) x[k * (16 / sizeof(T)) + j] = e[j];
    }
  } else {
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) x[j] = *smem_elem_ptr<T>(const_cast<char *>(tile), t * ITEMS + j);
  }
}

template <class T, int ITEMS>
__device__ __forceinline__ void write_blocked(char *tile, const T (&y)[ITEMS]) {
  constexpr int BYTES = ITEMS * (int)sizeof(T);
  const int t = threadIdx.x;
  if constexpr (BYTES % 16 == 0) {
    constexpr int VPT = BYTES / 16;
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
      uint4 w;
      T *e = reinterpret_cast<T *>(&w);
#pragma unroll
      for (int j = 0; j < 16 / (int)sizeof(T); ++j) e[j] = y[k * (16 / sizeof(T)) + j];
      *reinterpret_cast<uint4 *>(tile + swz(t * VPT + k) * 16) = w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) *smem_elem_ptr<T>(tile, t * ITEMS + j) = y[j];
  }
}

// ------------------------------------------------------------ look-back

// Warp-parallel look-back (called by all 32 lanes of one warp).  Lane l
// watches predecessor win - l.  The warp polls jointly and waits only for
// the lanes nearer than the closest predecessor whose inclusive prefix is
// published, then combines those payloads.  Every wait is bounded by
// timeout_ns (%globaltimer, checked every 64 polls); lanes still missing at
// the deadline count as broken links.  Returns the exclusive prefix; sets
// err when the chain is broken.
template <class Pub, class Ops>
__device__ Pub lookback(const StatusWord *status, long long tile, unsigned long long epoch_tag,
                        unsigned long long timeout_ns, bool &err) {
  const int lane = threadIdx.x & 31;
  Pub acc = Ops::identity();
  long long win = tile - 1;
  err = false;
  uint64_t t0 = 0;
  while (true) {
    const long long pred = win - lane;
    bool have = pred < 0;  // never needed: tile 0 always publishes a prefix
    unsigned long long payload = 0, flags = have ? kFlagPrefix : 0;
    unsigned stop_mask = 0;
    for (unsigned it = 0;; ++it) {
      if (!have) {
        StatusWord w = ld_status(status + pred);
        if ((w.meta & ~0xffull) == epoch_tag && (w.meta & (kFlagAgg | kFlagPrefix))) {
          have = true;
          payload = w.payload;
          flags = w.meta & 0xff;
        }
      }
      const unsigned have_mask = __ballot_sync(0xffffffffu, have);
      stop_mask = __ballot_sync(0xffffffffu, have && (flags & (kFlagPrefix | kFlagError)));
      const unsigned need = stop_mask ? ((2u << (__ffs(stop_mask) - 1)) - 1u) : 0xffffffffu;
      if ((have_mask & need) == need) break;
      if (it >= 8) __nanosleep(it < 64 ? 32 : 256);
      if ((it & 63) == 63) {
        uint64_t now = __shfl_sync(0xffffffffu, globaltimer_ns(), 0);
        if (t0 == 0) {
          t0 = now;
        } else if (now - t0 > timeout_ns) {
          if (!have) {
            have = true;
            flags = kFlagError;
          }
        }
      }
    }
    const int stop = stop_mask ? __ffs(stop_mask) - 1 : 31;
    Pub v = (pred >= 0 && lane <= stop && !(flags & kFlagError)) ? Ops::unpack(payload)
                                                                   : Ops::identity();
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v = Ops::combine(v, shfl_xor(v, m));
    acc = Ops::combine(v, acc);
    if (stop_mask) {
      const unsigned long long sf = __shfl_sync(0xffffffffu, flags, stop);
      err = (sf & kFlagError) != 0;
      return acc;
    }
    win -= 32;
  }
}

template <class P>
struct AccOps {
  using Pub = typename P::Acc;
  __device__ static Pub identity() { return P::identity(); }
  __device__ static Pub combine(Pub a, Pub b) { return P::combine(a, b); }
  __device__ static Pub unpack(unsigned long long v) { return P::unpack(v); }
  __device__ static unsigned long long pack(Pub v) { return P::pack(v); }
};

struct F64Ops {
  __device__ static double identity() { return 0.0; }
  __device__ static double combine(double a, double b) { return a + b; }
  __device__ static double unpack(unsigned long long v) { return __longlong_as_double((long long)v); }
  __device__ static unsigned long long pack(double v) { return (unsigned long long)__double_as_longlong(v); }
};

struct CountOps {
  __device__ static unsigned long long identity() { return 0; }
  __device__ static unsigned long long combine(unsigned long long a, unsigned long long b) {
    return a + b;
  }
  __device__ static unsigned long long unpack(unsigned long long v) { return v; }
  __device__ static unsigned long long pack(unsigned long long v) { return v; }
};

__device__ __forceinline__ void record_error(ScratchHeader *hdr, unsigned code) {
  atomicCAS(&hdr->error, 0u, code);
}

// Persistent-loop prologue/epilogue shared by scan and copy_if.
struct TileLoop {
  unsigned long long epoch_tag;
  unsigned epoch;
};

__device__ __forceinline__ void finish_launch(ScratchHeader *hdr, unsigned epoch) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicInc(&hdr->done_ctr, gridDim.x - 1);
    if (t == gridDim.x - 1) {
      // Every block has fetched its terminating tile id and read the epoch.
      atomicExch(&hdr->tile_ctr, 0ull);
      atomicExch(&hdr->epoch, epoch + 1);
    }
  }
}

// --------------------------------------------------------------- scan

template <class P, int ITEMS, bool WIDE>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    scan_kernel(ScanParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  using Ops = typename std::conditional<WIDE, F64Ops, AccOps<P>>::type;
  using Pub = decltype(Ops::identity());

  extern __shared__ __align__(16) char smem[];
  __shared__ Acc s_warp[32];
  __shared__ unsigned long long s_tile, s_carry;
  __shared__ unsigned s_epoch;
  __shared__ int s_has_carry;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int tile_elems = blockDim.x * ITEMS;
  if (threadIdx.x == 0) s_epoch = *reinterpret_cast<volatile unsigned *>(&p.hdr->epoch);
  __syncthreads();
  const unsigned epoch = s_epoch;
  const unsigned long long epoch_tag = (unsigned long long)epoch << 8;
  const In *in = reinterpret_cast<const In *>(p.in);
  Out *out = reinterpret_cast<Out *>(p.out);

  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    const long long tile = (long long)s_tile;
    if (tile >= p.ntiles) break;
    const unsigned long long base = (unsigned long long)tile * tile_elems;
    const int count = (int)min((unsigned long long)tile_elems, p.n - base);

    load_tile<In>(smem, in + base, count, tile_elems, p.vec_in);
    __syncthreads();

    In x[ITEMS];
    read_blocked<In, ITEMS>(smem, x);
    Acc r[ITEMS];
    const int first = threadIdx.x * ITEMS;
    Acc run = P::identity();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      if (first + j < count) P::add(run, x[j]);
      r[j] = run;
    }
    Acc agg = run;
    if constexpr (P::kCompensated) agg = df_norm(agg);

    // block scan of thread totals
    Acc incl = warp_inclusive_scan<P>(agg, lane);
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      Acc w = lane < nwarps ? s_warp[lane] : P::identity();
      w = warp_inclusive_scan<P>(w, lane);
      s_warp[lane] = w;
    }
    __syncthreads();
    Acc texcl = shfl_up(incl, 1);
    if (lane == 0) texcl = P::identity();
    if (warp > 0) texcl = P::combine(s_warp[warp - 1], texcl);
    const Acc tile_agg = s_warp[nwarps - 1];

    // cross-tile prefix (warp 0)
    if (warp == 0) {
      Pub agg_pub;
      if constexpr (WIDE) agg_pub = (double)tile_agg.hi + (double)tile_agg.lo;
      else agg_pub = tile_agg;
      const bool publish = tile != p.stall_tile;
      Pub carry = Ops::identity();
      unsigned long long has_carry = 0;
      if (tile == 0) {
        if (p.has_init) {
          if constexpr (WIDE) carry = (double)from_bits64<Out>(p.init_bits);
          else carry = P::from_out(from_bits64<Out>(p.init_bits));
          has_carry = 1;
        }
        if (lane == 0 && publish)
          st_status(p.status, Ops::pack(has_carry ? Ops::combine(carry, agg_pub) : agg_pub),
                    epoch_tag | kFlagPrefix);
      } else {
        if (lane == 0 && publish)
          st_status(p.status + tile, Ops::pack(agg_pub), epoch_tag | kFlagAgg);
        bool err;
        carry = lookback<Pub, Ops>(p.status, tile, epoch_tag, p.timeout_ns, err);
        has_carry = 1;
        if (lane == 0) {
          if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
          if (publish)
            st_status(p.status + tile, Ops::pack(Ops::combine(carry, agg_pub)),
                      epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
        }
      }
      if (lane == 0) {
        s_carry = Ops::pack(carry);
        s_has_carry = (int)has_carry;
      }
    }
    __syncthreads();
    const bool has_carry = s_has_carry != 0;
    // base = carry (+) thread exclusive prefix
    Acc basev = texcl;
    if (has_carry) {
      if constexpr (WIDE) {
        double c = F64Ops::unpack(s_carry) + ((double)texcl.hi + (double)texcl.lo);
        float h = (float)c;
        basev = DF{h, (float)(c - (double)h)};
      } else {
        basev = P::combine(Ops::unpack(s_carry), texcl);
      }
    }
    Out y[ITEMS];
    if (p.inclusive) {
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) y[j] = P::finalize(P::combine(basev, r[j]));
    } else {
      y[0] = P::finalize(basev);
#pragma unroll
      for (int j = 1; j < ITEMS; ++j) y[j] = P::finalize(P::combine(basev, r[j - 1]));
    }
    write_blocked<Out, ITEMS>(smem, y);
    __syncthreads();
    store_tile<Out>(smem, out + base, count, tile_elems, p.vec_out);
    __syncthreads();
  }
  finish_launch(p.hdr, epoch);
}

// ------------------------------------------------------------ copy_if

template <class T>
__device__ __forceinline__ bool pred_bits(T v, unsigned long long mask, int cmp,
                                          unsigned long long rhs) {
  using U = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
  U u;
  memcpy(&u, &v, sizeof(T));
  const U a = u & (U)mask, r = (U)rhs;
  switch (cmp) {
  case B2P_CMP_LT: return a < r;
  case B2P_CMP_LE: return a <= r;
  case B2P_CMP_EQ: return a == r;
  case B2P_CMP_NE: return a != r;
  case B2P_CMP_GE: return a >= r;
  default: return a > r;
  }
}

template <class T, int ITEMS>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 8192 / ITEMS)
    copy_if_kernel(ScanParams p) {
  extern __shared__ __align__(16) char smem[];
  __shared__ unsigned s_warp[32];
  __shared__ unsigned long long s_tile, s_carry;
  __shared__ unsigned s_epoch;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int tile_elems = blockDim.x * ITEMS;
  if (threadIdx.x == 0) s_epoch = *reinterpret_cast<volatile unsigned *>(&p.hdr->epoch);
  __syncthreads();
  const unsigned epoch = s_epoch;
  const unsigned long long epoch_tag = (unsigned long long)epoch << 8;
  const T *in = reinterpret_cast<const T *>(p.in);
  T *out = reinterpret_cast<T *>(p.out);

  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&p.hdr->tile_ctr, 1ull);
    __syncthreads();
    const long long tile = (long long)s_tile;
    if (tile >= p.ntiles) break;
    const unsigned long long base = (unsigned long long)tile * tile_elems;
    const int count = (int)min((unsigned long long)tile_elems, p.n - base);

    load_tile<T>(smem, in + base, count, tile_elems, p.vec_in);
    __syncthreads();
    T x[ITEMS];
    read_blocked<T, ITEMS>(smem, x);
    const int first = threadIdx.x * ITEMS;
    unsigned keep = 0;
    int kept = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      bool k = (first + j < count) && pred_bits(x[j], p.mask, p.cmp, p.rhs);
      keep |= (unsigned)k << j;
      kept += k;
    }
    // block exclusive scan of per-thread counts
    unsigned incl = (unsigned)kept;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      unsigned o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      unsigned w = lane < nwarps ? s_warp[lane] : 0;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        unsigned o = __shfl_up_sync(0xffffffffu, w, d);
        if (lane >= d) w += o;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    unsigned texcl = incl - (unsigned)kept + (warp > 0 ? s_warp[warp - 1] : 0u);
    const unsigned tile_kept = s_warp[nwarps - 1];

    if (warp == 0) {
      const bool publish = tile != p.stall_tile;
      unsigned long long carry = 0;
      if (tile == 0) {
        if (lane == 0 && publish) st_status(p.status, tile_kept, epoch_tag | kFlagPrefix);
      } else {
        if (lane == 0 && publish) st_status(p.status + tile, tile_kept, epoch_tag | kFlagAgg);
        bool err;
        carry = lookback<unsigned long long, CountOps>(p.status, tile, epoch_tag, p.timeout_ns, err);
        if (lane == 0) {
          if (err) record_error(p.hdr, B2P_ERR_TIMEOUT);
          if (publish)
            st_status(p.status + tile, carry + tile_kept,
                      epoch_tag | kFlagPrefix | (err ? kFlagError : 0));
        }
      }
      if (lane == 0) {
        s_carry = carry;
        if (tile == p.ntiles - 1 && p.num_copied) *p.num_copied = carry + tile_kept;
      }
    }
    __syncthreads();  // everyone has read the input tile; reuse it for output
    {
      int o = (int)texcl;
#pragma unroll
      for (int j = 0; j < ITEMS; ++j)
        if (keep & (1u << j)) *smem_elem_ptr<T>(smem, o++) = x[j];
    }
    __syncthreads();
    const unsigned long long obase = s_carry;
    for (int i = threadIdx.x; i < (int)tile_kept; i += blockDim.x)
      out[obase + i] = *smem_elem_ptr<T>(smem, i);
    __syncthreads();
  }
  finish_launch(p.hdr, epoch);
}

// ---------------------------------------------------------------- host

namespace {

constexpr int kMaxTileElems = 8192;

bool tile_ok(size_t esize_in, size_t esize_out, int block, int items) {
  if (block * items > kMaxTileElems) return false;
  size_t bytes = (size_t)block * items * std::max(esize_in, esize_out);
  return bytes <= 200 * 1024;
}

template <class K>
int launch_tiles(K kernel, ScanParams &p, const LaunchConfig &lc, size_t smem, cudaStream_t st) {
  const void *kfn = (const void *)kernel;
  int rc = ensure_dynamic_smem(kfn, smem);
  if (rc) return rc;
  int grid = grid_for(lc.grid_mode, p.ntiles, 1, kfn, lc.block, smem);
  kernel<<<grid, lc.block, smem, st>>>(p);
  return cuda_status(cudaGetLastError());
}

template <class P, int ITEMS>
int launch_scan_items(ScanParams &p, const LaunchConfig &lc, bool wide, cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  size_t smem = (size_t)lc.block * ITEMS * std::max(sizeof(In), sizeof(Out));
  if constexpr (P::kCompensated) {
    if (wide) return launch_tiles(scan_kernel<P, ITEMS, true>, p, lc, smem, st);
  }
  return launch_tiles(scan_kernel<P, ITEMS, false>, p, lc, smem, st);
}

template <class P>
int launch_scan_t(int inclusive, const void *in, void *out, size_t n, const void *init,
                  void *scratch, size_t sb, int config, cudaStream_t st) {
  using In = typename P::In;
  using Out = typename P::Out;
  LaunchConfig lc = describe_config(config);
  if (!tile_ok(sizeof(In), sizeof(Out), lc.block, lc.items)) return B2P_ERR_INVALID_ARG;
  const long long tile = (long long)lc.block * lc.items;
  ScanParams p{};
  p.in = in;
  p.out = out;
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  size_t need = kHeaderBytes + (size_t)p.ntiles * sizeof(StatusWord);
  if (sb < need || (reinterpret_cast<uintptr_t>(scratch) & 255)) return B2P_ERR_SCRATCH;
  p.inclusive = inclusive;
  p.has_init = init != nullptr;
  if (init) memcpy(&p.init_bits, init, sizeof(Out));
  p.vec_in = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
  p.vec_out = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kHeaderBytes);
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
#define B2P_SCAN_CASE(OP)                                                                   \
  case OP:                                                                                  \
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

template <class T>
int launch_copy_if_t(const void *in, void *out, size_t n, uint64_t mask, int cmp, uint64_t rhs,
                     uint64_t *num_copied, void *scratch, size_t sb, int config, cudaStream_t st) {
  LaunchConfig lc = describe_config(config);
  if (!tile_ok(sizeof(T), sizeof(T), lc.block, lc.items)) return B2P_ERR_INVALID_ARG;
  const long long tile = (long long)lc.block * lc.items;
  ScanParams p{};
  p.in = in;
  p.out = out;
  p.n = n;
  p.ntiles = (long long)((n + tile - 1) / tile);
  size_t need = kHeaderBytes + (size_t)p.ntiles * sizeof(StatusWord);
  if (sb < need || (reinterpret_cast<uintptr_t>(scratch) & 255)) return B2P_ERR_SCRATCH;
  p.vec_in = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.status = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kHeaderBytes);
  p.timeout_ns = wait_timeout_ns();
  p.stall_tile = debug_stall_tile();
  p.mask = mask;
  p.rhs = rhs;
  p.cmp = cmp;
  p.num_copied = reinterpret_cast<unsigned long long *>(num_copied);
  size_t smem = (size_t)lc.block * lc.items * sizeof(T);
  switch (lc.items) {
  case 4: return launch_tiles(copy_if_kernel<T, 4>, p, lc, smem, st);
  case 8: return launch_tiles(copy_if_kernel<T, 8>, p, lc, smem, st);
  case 16: return launch_tiles(copy_if_kernel<T, 16>, p, lc, smem, st);
  default: return launch_tiles(copy_if_kernel<T, 32>, p, lc, smem, st);
  }
}

}  // namespace

bool scan_config_valid(int dtype, int config) {
  if (config < 0 || config >= B2P_NUM_CONFIGS) return false;
  LaunchConfig lc = describe_config(config);
  return tile_ok(dtype_size(dtype), acc_size(dtype), lc.block, lc.items);
}

size_t scan_scratch_bytes(int dtype, size_t n, int config) {
  long long tile = 512;  // smallest tile of the table
  if (config >= 0) {
    LaunchConfig lc = describe_config(config);
    tile = (long long)lc.block * lc.items;
  }
  (void)dtype;
  return kHeaderBytes + (size_t)((n + tile - 1) / tile) * sizeof(StatusWord);
}

size_t copy_if_scratch_bytes(int dtype, size_t n, int config) {
  return scan_scratch_bytes(dtype, n, config);
}

int launch_scan(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
                const void *init, void *scratch, size_t sb, int config, cudaStream_t st) {
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
  switch (dtype_size(dtype)) {
  case 4: return launch_copy_if_t<uint32_t>(in, out, n, mask, cmp, rhs, num_copied, scratch, sb, config, st);
  case 8: return launch_copy_if_t<unsigned long long>(in, out, n, mask, cmp, rhs, num_copied, scratch, sb, config, st);
  default: return B2P_ERR_UNSUPPORTED;
  }
}

}  // namespace b2p
