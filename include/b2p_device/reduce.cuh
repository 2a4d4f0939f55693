// The single-pass reduce kernels, shared by libb2p (b2p_reduce, b2p_dot)
// and the header-only C++ layer (sycl::reduction in parallel_for,
// transform_reduce with a user transform or operator).
//
// Replaces AdaptiveCpp's multi-launch work-group reduction
// (algorithms/numeric.hpp:67-161, reduction/reduction_engine.hpp:116-390,
// util/memory_streaming.hpp:85-91): there, a grid-stride main kernel of
// 4*CUs groups x 128 work-items writes group partials and ceil(G/128)-wide
// stage kernels re-reduce them (3 launches for large n).  Here one launch
// streams the input and finishes in the last block to arrive (no spin
// waits).
//
// Canonical decomposition.  The input is cut into "runs" of 32 lanes x K
// units (16-byte vectors of a contiguous array, or single indices of a
// generated sequence); lane l of the warp that owns a run folds units
// l, l+32, l+64, ... in order, then the warp butterfly combines the 32 lane
// values.  K depends only on n and the element size, never on the launch
// configuration, and the run partials are combined by a fixed 512-wide tree
// in the last block.  A float result is therefore bit-identical for every
// configuration, and run-to-run.
#pragma once

#include "common.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <type_traits>

namespace b2p {

struct ReduceParams {
  const void *a;
  const void *b;
  unsigned long long n;
  unsigned long long head;  // elements before the first 16-byte boundary
  unsigned long long nvec;  // full vectors in the aligned body
  unsigned long long tail;  // elements after the last full vector
  long long runs;
  int K;  // vectors per lane per run
  int B;  // vectors in flight per lane (from the launch configuration)
  void *out;
  unsigned long long init_bits;
  int has_init;
  ScratchHeader *hdr;
  StatusWord *partials;  // one epoch-tagged word per run
};

constexpr int kFinalWidth = 512;

// Every block calls this once after its last partial: true in the block
// that arrives last (which then sees every other block's partials).
__device__ __forceinline__ bool last_block_arrives(ScratchHeader *hdr) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicInc(&hdr->done_ctr, gridDim.x - 1);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  const bool last = s_last != 0;
  if (last) __threadfence();
  return last;
}

// Last block: the run partials combined by the fixed tree (slot v of
// kFinalWidth folds partials v, v + kFinalWidth, ... in order, then a
// halving tree); the result is left in s_v[0] (packed).
template <class P>
__device__ __forceinline__ void combine_run_partials(const StatusWord *partials, long long runs,
                                                     unsigned long long *s_v) {
  using Acc = typename P::Acc;
  for (int v = threadIdx.x; v < kFinalWidth; v += blockDim.x) {
    Acc acc = P::identity();
    long long r = v;
    for (; r + 3 * kFinalWidth < runs; r += 4 * kFinalWidth) {
      unsigned long long x0 = ld_status(partials + r).payload;
      unsigned long long x1 = ld_status(partials + r + kFinalWidth).payload;
      unsigned long long x2 = ld_status(partials + r + 2 * kFinalWidth).payload;
      unsigned long long x3 = ld_status(partials + r + 3 * kFinalWidth).payload;
      acc = P::combine(acc, P::unpack(x0));
      acc = P::combine(acc, P::unpack(x1));
      acc = P::combine(acc, P::unpack(x2));
      acc = P::combine(acc, P::unpack(x3));
    }
    for (; r < runs; r += kFinalWidth) acc = P::combine(acc, P::unpack(ld_status(partials + r).payload));
    s_v[v] = P::pack(acc);
  }
  __syncthreads();
  for (int w = kFinalWidth / 2; w >= 1; w >>= 1) {
    for (int v = threadIdx.x; v < w; v += blockDim.x)
      s_v[v] = P::pack(P::combine(P::unpack(s_v[v]), P::unpack(s_v[v + w])));
    __syncthreads();
  }
}


template <class In, bool VEC>
struct VecOf {
  using type = typename std::conditional<VEC, uint4, In>::type;
  static constexpr int kElems = VEC ? int(16 / sizeof(In)) : 1;
};

template <class In, bool VEC>
__device__ __forceinline__ typename VecOf<In, VEC>::type load_vec(const In *base, long long vi) {
  if constexpr (VEC) {
    return ld_stream_v4(reinterpret_cast<const uint4 *>(base) + vi);
  } else {
    return __ldg(base + vi);
  }
}

template <class In, class VT>
__device__ __forceinline__ In vec_elem(const VT &v, int i) {
  if constexpr (std::is_same<VT, uint4>::value) {
    const In *e = reinterpret_cast<const In *>(&v);
    return e[i];
  } else {
    return v;
  }
}

// acc op= a (reduce) or acc += a*b (dot).
template <class P, bool DOT>
__device__ __forceinline__ void fold(typename P::Acc &acc, typename P::In a, typename P::In b) {
  using In = typename P::In;
  if constexpr (!DOT) {
    P::add(acc, a);
  } else if constexpr (P::kCompensated && sizeof(In) == 4) {
    // Dot2 (Ogita-Rump-Oishi): TwoProduct via fma, TwoSum on the product.
    float p = __fmul_rn(a, b);
    float ep = __fmaf_rn(a, b, -p);
    float s, e;
    two_sum(acc.hi, p, s, e);
    acc.hi = s;
    acc.lo = __fadd_rn(acc.lo, __fadd_rn(e, ep));
  } else if constexpr (P::kCompensated) {
    // bf16 x bf16 is exact in fp32.
    df_accumulate(acc, __fmul_rn(bf16_bits_to_f32(a), bf16_bits_to_f32(b)));
  } else {
    acc = fma(a, b, acc);
  }
}

template <class P, bool DOT, bool VEC>
__global__ void __launch_bounds__(1024) reduce_kernel(ReduceParams p) {
  using In = typename P::In;
  using Acc = typename P::Acc;
  using VT = typename VecOf<In, VEC>::type;
  constexpr int V = VecOf<In, VEC>::kElems;
  constexpr int kMaxB = (DOT || sizeof(In) == 8) ? 4 : 8;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const long long gw = (long long)blockIdx.x * wpb + warp;
  const long long tw = (long long)gridDim.x * wpb;
  const In *a = reinterpret_cast<const In *>(p.a) + p.head;
  const In *b = DOT ? reinterpret_cast<const In *>(p.b) + p.head : nullptr;
  const long long nvec = (long long)p.nvec;
  const int B = min(p.B, kMaxB);
  const unsigned long long epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);

  // Compensated folds keep kChains accumulators (element e of each vector
  // goes to chain e % kChains: two for fp32, four for bf16), shortening the
  // dependent TwoSum chain; the order depends only on element positions, so
  // every launch configuration gives the same bits.
  constexpr int kChains = !P::kCompensated || V == 1 ? 1 : (V >= 8 ? 4 : 2);
  for (long long run = gw; run < p.runs; run += tw) {
    Acc acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = P::identity();
    const long long base = run * 32LL * p.K + lane;
    for (int j0 = 0; j0 < p.K; j0 += B) {
      const long long v0 = base + (long long)j0 * 32;
      if (v0 + (long long)(B - 1) * 32 < nvec) {
        // whole batch in range: B independent 16-byte loads in flight
        VT va[kMaxB], vb[kMaxB];
#pragma unroll
        for (int k = 0; k < kMaxB; ++k)
          if (k < B) {
            va[k] = load_vec<In, VEC>(a, v0 + k * 32);
            if constexpr (DOT) vb[k] = load_vec<In, VEC>(b, v0 + k * 32);
          }
#pragma unroll
        for (int k = 0; k < kMaxB; ++k)
          if (k < B) {
#pragma unroll
            for (int e = 0; e < V; ++e) {
              In xa = vec_elem<In>(va[k], e);
              In xb = DOT ? vec_elem<In>(vb[k], e) : xa;
              fold<P, DOT>(acc[e % kChains], xa, xb);
            }
          }
      } else {
        // ragged end of the last run
        for (int k = 0; k < B; ++k) {
          const long long vi = v0 + k * 32;
          if (vi < nvec) {
            VT xa = load_vec<In, VEC>(a, vi);
            VT xb = xa;
            if constexpr (DOT) xb = load_vec<In, VEC>(b, vi);
#pragma unroll
            for (int e = 0; e < V; ++e)
              fold<P, DOT>(acc[e % kChains], vec_elem<In>(xa, e), DOT ? vec_elem<In>(xb, e) : vec_elem<In>(xa, e));
          }
        }
      }
    }
    if constexpr (kChains == 4) {
      acc[0] = P::combine(acc[0], acc[1]);
      acc[2] = P::combine(acc[2], acc[3]);
    }
    if constexpr (kChains >= 2) acc[0] = P::combine(acc[0], acc[kChains / 2]);
    Acc r = acc[0];
    if constexpr (P::kCompensated) r = df_norm(r);
    r = warp_allreduce<P>(r);
    if (lane == 0) st_status(p.partials + run, P::pack(r), (epoch << 8) | kFlagAgg);
  }

  // ---- last block to arrive combines everything (no waiting).
  __shared__ unsigned long long s_v[kFinalWidth];
  if (!last_block_arrives(p.hdr)) return;
  combine_run_partials<P>(p.partials, p.runs, s_v);
  if (threadIdx.x == 0) {
    const In *a0 = reinterpret_cast<const In *>(p.a);
    const In *b0 = reinterpret_cast<const In *>(p.b);
    Acc h = P::identity();
    for (unsigned long long i = 0; i < p.head; ++i) fold<P, DOT>(h, a0[i], DOT ? b0[i] : a0[i]);
    Acc t = P::identity();
    const unsigned long long ts = p.head + p.nvec * V;
    for (unsigned long long i = ts; i < ts + p.tail; ++i) fold<P, DOT>(t, a0[i], DOT ? b0[i] : a0[i]);
    if constexpr (P::kCompensated) {
      h = df_norm(h);
      t = df_norm(t);
    }
    Acc total = P::combine(P::combine(h, P::unpack(s_v[0])), t);
    using Out = typename P::Out;
    Out *out = reinterpret_cast<Out *>(p.out);
    Out basev = p.has_init ? from_bits64<Out>(p.init_bits) : *out;
    *out = P::finalize(P::combine(P::from_out(basev), total));
    // every block read the epoch before arriving; the next launch sees this
    atomicAdd(&p.hdr->epoch, 1ull);
  }
}


// ------------------------------------------------- generated sequences
//
// The same runs over a generated sequence of n units: unit i is folded by
// `src.accumulate(acc, i)` (a transform of one or two inputs, or a user
// kernel that combines into a reducer).  Lane l of a run handles units
// base + l + 32 j, so a unit that reads element i of an array reads it
// coalesced across the warp; UNROLL consecutive units are evaluated before
// they are folded, which keeps UNROLL independent loads in flight per lane.
// A compensated policy folds even and odd j into two chains.
//
// The policy's result rule: `P::write(out, total, has_init, init_bits)` when
// the policy has one (operators without a known identity), otherwise
// *out = op(init, total), or op(*out, total) without init.

template <class Src>
struct ReduceGenParams {
  Src src;
  unsigned long long n;
  long long runs;
  int K;  // units per lane per run
  void *out;
  unsigned long long init_bits;
  int has_init;
  ScratchHeader *hdr;
  StatusWord *partials;
};

// A source whose unit i is one value, value(i) of the derived class: the
// fold adds it to the lane's accumulator; a batch evaluates all its values
// before folding them, so their loads are in flight together.
template <class Derived, class T>
struct ValueSource {
  template <class P>
  __device__ __forceinline__ void accumulate(typename P::Acc &acc, long long i) const {
    P::add(acc, static_cast<typename P::In>(static_cast<const Derived *>(this)->value(i)));
  }
  template <class P, int U, int C>
  __device__ __forceinline__ void accumulate_batch(typename P::Acc *acc, long long i0) const {
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = static_cast<const Derived *>(this)->value(i0 + 32LL * u);
#pragma unroll
    for (int u = 0; u < U; ++u) P::add(acc[u % C], static_cast<typename P::In>(v[u]));
  }
};

template <class P, class = void>
struct has_custom_write : std::false_type {};
template <class P>
struct has_custom_write<P, std::void_t<decltype(P::kCustomWrite)>> : std::true_type {};

template <class P, class Src, int UNROLL>
__global__ void __launch_bounds__(512) reduce_gen_kernel(ReduceGenParams<Src> p) {
  using Acc = typename P::Acc;
  using Out = typename P::Out;
  constexpr int kChains = P::kCompensated ? 2 : 1;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const long long gw = (long long)blockIdx.x * wpb + warp;
  const long long tw = (long long)gridDim.x * wpb;
  const unsigned long long epoch = *reinterpret_cast<volatile unsigned long long *>(&p.hdr->epoch);
  const long long n = (long long)p.n;
  for (long long run = gw; run < p.runs; run += tw) {
    Acc acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = P::identity();
    const long long base = run * 32LL * p.K + lane;
    for (int j0 = 0; j0 < p.K; j0 += UNROLL) {
      const long long i0 = base + (long long)j0 * 32;
      if (i0 + (long long)(UNROLL - 1) * 32 < n) {
        p.src.template accumulate_batch<P, UNROLL, kChains>(acc, i0);
      } else {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
          if (i0 + (long long)u * 32 < n) p.src.template accumulate<P>(acc[(j0 + u) % kChains], i0 + (long long)u * 32);
      }
    }
    if constexpr (kChains == 2) acc[0] = P::combine(acc[0], acc[1]);
    Acc r = acc[0];
    if constexpr (P::kCompensated) r = df_norm(r);
    r = warp_allreduce<P>(r);
    if (lane == 0) st_status(p.partials + run, P::pack(r), (epoch << 8) | kFlagAgg);
  }
  __shared__ unsigned long long s_v[kFinalWidth];
  if (!last_block_arrives(p.hdr)) return;
  combine_run_partials<P>(p.partials, p.runs, s_v);
  if (threadIdx.x == 0) {
    const Acc total = P::unpack(s_v[0]);
    Out *out = reinterpret_cast<Out *>(p.out);
    if constexpr (has_custom_write<P>::value) {
      P::write(out, total, p.has_init != 0, p.init_bits);
    } else {
      const Out basev = p.has_init ? from_bits64<Out>(p.init_bits) : *out;
      *out = P::finalize(P::combine(P::from_out(basev), total));
    }
    atomicAdd(&p.hdr->epoch, 1ull);
  }
}

// SM count of a device, and blocks per SM of one kernel instantiation at
// one block size, each looked up once per device.
inline int device_sm_count(int dev) {
  static std::atomic<int> sms[64];
  int v = sms[dev & 63].load();
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    sms[dev & 63].store(v);
  }
  return v;
}
template <auto K>
struct KernelOccupancy {
  static inline std::atomic<int> occ[64];
  static int get(int dev, int threads) {
    int v = occ[dev & 63].load();
    if (v <= 0) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, (const void *)K, threads, 0) != cudaSuccess || v < 1) {
        cudaGetLastError();
        v = 1;
      }
      occ[dev & 63].store(v);
    }
    return v;
  }
};

// Run shape of a generated sequence: K a power of two from n alone, at least
// 4736 runs (148 SMs x 32 warps) for large n: the user kernel's scalar loads
// need more warps in flight than the library's 16-byte loads (measured: 2.5 %
// faster at 2^28 fp32 than 2368 runs; 32 loads per lane instead of 16 was
// slower).
struct GenShape {
  int K;
  long long runs;
};
inline GenShape reduce_gen_shape(unsigned long long n) {
  GenShape s{};
  const unsigned long long per = n / (32ull * 4736ull);
  int K = 64;
  while ((unsigned long long)K * 2 <= per) K *= 2;
  s.K = K;
  s.runs = (long long)((n + 32ull * K - 1) / (32ull * K));
  return s;
}

// Scratch of a generated-sequence reduce of n units: the prefix and one
// status word per run.
inline size_t reduce_gen_scratch_bytes(unsigned long long n) {
  return kScratchPrefix + (size_t)std::max<long long>(reduce_gen_shape(n).runs, 1) * sizeof(StatusWord);
}

// Launch the generated-sequence reduce: *out = op(init, total), or
// op(*out, total) when init is null (the policy's own rule when it has one).
// scratch: libb2p scratch (zero-filled once, 256-byte aligned) of at least
// reduce_gen_scratch_bytes(n).  Asynchronous on st.
template <class P, class Src, int UNROLL = (sizeof(typename P::In) <= 4 ? 16 : 8)>
int launch_reduce_gen(const Src &src, unsigned long long n, void *out, const void *init, void *scratch,
                      size_t scratch_bytes, cudaStream_t st) {
  // a run's K units (a power of two, at least 64) split into whole batches
  static_assert(64 % UNROLL == 0, "UNROLL divides every K");
  if (n == 0) return B2P_OK;
  const GenShape sh = reduce_gen_shape(n);
  if (!scratch || scratch_bytes < reduce_gen_scratch_bytes(n) || (reinterpret_cast<uintptr_t>(scratch) & 255))
    return B2P_ERR_SCRATCH;
  ReduceGenParams<Src> p{src, n, sh.runs, sh.K, out, 0ull, init != nullptr,
                         reinterpret_cast<ScratchHeader *>(scratch),
                         reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix)};
  if (init) memcpy(&p.init_bits, init, sizeof(typename P::Out));
  auto kfn = reduce_gen_kernel<P, Src, UNROLL>;
  constexpr int kThreads = 512;
  int dev = 0;
  cudaGetDevice(&dev);
  const int occ = KernelOccupancy<reduce_gen_kernel<P, Src, UNROLL>>::get(dev, kThreads);
  const long long want = (sh.runs + kThreads / 32 - 1) / (kThreads / 32);
  const int grid = (int)std::max<long long>(1, std::min<long long>(want, (long long)device_sm_count(dev) * occ));
  kfn<<<grid, kThreads, 0, st>>>(p);
  return cudaGetLastError() == cudaSuccess ? B2P_OK : B2P_ERR_CUDA;
}

// ------------------------------------------------------ host-side shapes

struct Shape {
  size_t esize;
  bool vec;
  unsigned long long head, nvec, tail;
  int K;
  long long runs;
};

inline Shape reduce_shape(size_t esize, size_t n, const void *a, const void *b) {
  Shape s{};
  s.esize = esize;
  const uintptr_t ma = reinterpret_cast<uintptr_t>(a) & 15;
  const uintptr_t mb = b ? (reinterpret_cast<uintptr_t>(b) & 15) : ma;
  s.vec = (ma == mb);
  size_t V = s.vec ? 16 / esize : 1;
  size_t head = 0;
  if (s.vec && ma) head = std::min<size_t>((16 - ma) / esize, n);
  s.head = head;
  s.nvec = (n - head) / V;
  s.tail = n - head - s.nvec * V;
  // Runs: >= 2368 (= 148 SMs x 16 warps) for large inputs, >= 16 vectors
  // per lane; K is a power of two fixed by n and the element size only.
  unsigned long long per = s.nvec / (32ull * 2368ull);
  int K = 16;
  while ((unsigned long long)K * 2 <= per) K *= 2;
  s.K = K;
  s.runs = (long long)((s.nvec + 32ull * K - 1) / (32ull * K));
  return s;
}

}  // namespace b2p
