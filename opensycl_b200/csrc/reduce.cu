// Single-pass reduce and dot product.
//
// Replaces AdaptiveCpp's multi-launch work-group reduction
// (algorithms/numeric.hpp:67-161, reduction/reduction_engine.hpp:116-390,
// util/memory_streaming.hpp:85-91): there, a grid-stride main kernel of
// 4*CUs groups x 128 work-items writes group partials and ceil(G/128)-wide
// stage kernels re-reduce them (3 launches for large n).  Here one launch
// streams the input with 16-byte loads and finishes in the last block to
// arrive (no spin waits).
//
// Canonical decomposition.  The aligned body of the input is cut into
// "runs" of 32 lanes x K 16-byte vectors; lane l of the warp that owns a
// run folds vectors l, l+32, l+64, ... in order, then the warp butterfly
// combines the 32 lane values.  K depends only on n and the dtype, never on
// the launch configuration, and the run partials are combined by a fixed
// 512-wide tree in the last block, followed by the unaligned head and the
// tail.  A float result is therefore bit-identical for every configuration,
// and run-to-run.
#include "common.cuh"
#include "internal.h"

#include <algorithm>

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
  __shared__ int s_last;
  __shared__ unsigned long long s_v[kFinalWidth];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicInc(&p.hdr->done_ctr, gridDim.x - 1);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();

  for (int v = threadIdx.x; v < kFinalWidth; v += blockDim.x) {
    Acc acc = P::identity();
    long long r = v;
    for (; r + 3 * kFinalWidth < p.runs; r += 4 * kFinalWidth) {
      unsigned long long x0 = ld_status(p.partials + r).payload;
      unsigned long long x1 = ld_status(p.partials + r + kFinalWidth).payload;
      unsigned long long x2 = ld_status(p.partials + r + 2 * kFinalWidth).payload;
      unsigned long long x3 = ld_status(p.partials + r + 3 * kFinalWidth).payload;
      acc = P::combine(acc, P::unpack(x0));
      acc = P::combine(acc, P::unpack(x1));
      acc = P::combine(acc, P::unpack(x2));
      acc = P::combine(acc, P::unpack(x3));
    }
    for (; r < p.runs; r += kFinalWidth) acc = P::combine(acc, P::unpack(ld_status(p.partials + r).payload));
    s_v[v] = P::pack(acc);
  }
  __syncthreads();
  for (int w = kFinalWidth / 2; w >= 1; w >>= 1) {
    for (int v = threadIdx.x; v < w; v += blockDim.x)
      s_v[v] = P::pack(P::combine(P::unpack(s_v[v]), P::unpack(s_v[v + w])));
    __syncthreads();
  }
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

// ---------------------------------------------------------------- host

namespace {

struct Shape {
  size_t esize;
  bool vec;
  unsigned long long head, nvec, tail;
  int K;
  long long runs;
};

Shape reduce_shape(size_t esize, size_t n, const void *a, const void *b) {
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

template <class P, bool DOT>
int launch_t(const void *a, const void *b, size_t n, void *out, const void *init, void *scratch,
             size_t scratch_bytes, int config, cudaStream_t st) {
  using In = typename P::In;
  Shape sh = reduce_shape(sizeof(In), n, a, DOT ? b : nullptr);
  size_t need = kScratchPrefix + (size_t)std::max<long long>(sh.runs, 1) * sizeof(StatusWord);
  if (scratch_bytes < need || (reinterpret_cast<uintptr_t>(scratch) & 255)) return B2P_ERR_SCRATCH;
  LaunchConfig lc = describe_config(config);
  ReduceParams p{};
  p.a = a;
  p.b = b;
  p.n = n;
  p.head = sh.head;
  p.nvec = sh.nvec;
  p.tail = sh.tail;
  p.runs = sh.runs;
  p.K = sh.K;
  size_t vbytes = sh.vec ? 16 : sizeof(In);
  p.B = (int)std::max<size_t>(1, std::min<size_t>(8, lc.items * sizeof(In) / vbytes));
  while (sh.K % p.B) p.B >>= 1;
  p.out = out;
  p.has_init = init != nullptr;
  p.init_bits = 0;
  if (init) memcpy(&p.init_bits, init, sizeof(typename P::Out));
  p.hdr = reinterpret_cast<ScratchHeader *>(scratch);
  p.partials = reinterpret_cast<StatusWord *>(reinterpret_cast<char *>(scratch) + kScratchPrefix);
  int wpb = lc.block / 32;
  if constexpr (DOT) {
    if (!sh.vec) {
      const void *kfn = (const void *)reduce_kernel<P, DOT, false>;
      int grid = grid_for(lc.grid_mode, std::max<long long>(sh.runs, 1), wpb, kfn, lc.block, 0);
      reduce_kernel<P, DOT, false><<<grid, lc.block, 0, st>>>(p);
      return cuda_status(cudaGetLastError());
    }
  }
  const void *kfn = (const void *)reduce_kernel<P, DOT, true>;
  int grid = grid_for(lc.grid_mode, std::max<long long>(sh.runs, 1), wpb, kfn, lc.block, 0);
  reduce_kernel<P, DOT, true><<<grid, lc.block, 0, st>>>(p);
  return cuda_status(cudaGetLastError());
}

template <int DT>
int dispatch_op(int op, const void *a, const void *b, size_t n, void *out, const void *init,
                void *scratch, size_t sb, int config, cudaStream_t st) {
  if (b) {
    if constexpr (DT == B2P_F32 || DT == B2P_BF16 || DT == B2P_F64)
      return launch_t<typename PolicyOf<DT, B2P_SUM>::type, true>(a, b, n, out, init, scratch, sb,
                                                                 config, st);
    return B2P_ERR_UNSUPPORTED;
  }
  switch (op) {
  case B2P_SUM: return launch_t<typename PolicyOf<DT, B2P_SUM>::type, false>(a, b, n, out, init, scratch, sb, config, st);
  case B2P_PROD: return launch_t<typename PolicyOf<DT, B2P_PROD>::type, false>(a, b, n, out, init, scratch, sb, config, st);
  case B2P_MIN: return launch_t<typename PolicyOf<DT, B2P_MIN>::type, false>(a, b, n, out, init, scratch, sb, config, st);
  case B2P_MAX: return launch_t<typename PolicyOf<DT, B2P_MAX>::type, false>(a, b, n, out, init, scratch, sb, config, st);
  default: break;
  }
  if constexpr (DT == B2P_F32 || DT == B2P_BF16 || DT == B2P_F64) {
    return B2P_ERR_UNSUPPORTED;
  } else {
    switch (op) {
    case B2P_AND: return launch_t<typename PolicyOf<DT, B2P_AND>::type, false>(a, b, n, out, init, scratch, sb, config, st);
    case B2P_OR: return launch_t<typename PolicyOf<DT, B2P_OR>::type, false>(a, b, n, out, init, scratch, sb, config, st);
    case B2P_XOR: return launch_t<typename PolicyOf<DT, B2P_XOR>::type, false>(a, b, n, out, init, scratch, sb, config, st);
    default: return B2P_ERR_INVALID_ARG;
    }
  }
}

template <int DT, int OP>
int preload_one() {
  cudaFuncAttributes fa;
  cudaError_t e =
      cudaFuncGetAttributes(&fa, (const void *)reduce_kernel<typename PolicyOf<DT, OP>::type, false, true>);
  return cuda_status(e);
}

template <int DT>
int preload_dtype() {
  int rc = preload_one<DT, B2P_SUM>();
  if (!rc) rc = preload_one<DT, B2P_PROD>();
  if (!rc) rc = preload_one<DT, B2P_MIN>();
  if (!rc) rc = preload_one<DT, B2P_MAX>();
  if constexpr (DT != B2P_F32 && DT != B2P_BF16 && DT != B2P_F64) {
    if (!rc) rc = preload_one<DT, B2P_AND>();
    if (!rc) rc = preload_one<DT, B2P_OR>();
    if (!rc) rc = preload_one<DT, B2P_XOR>();
  }
  return rc;
}

}  // namespace

int preload_reduce_kernels() {
  int rc = preload_dtype<B2P_I32>();
  if (!rc) rc = preload_dtype<B2P_I64>();
  if (!rc) rc = preload_dtype<B2P_U32>();
  if (!rc) rc = preload_dtype<B2P_U64>();
  if (!rc) rc = preload_dtype<B2P_F32>();
  if (!rc) rc = preload_dtype<B2P_BF16>();
  if (!rc) rc = preload_dtype<B2P_F64>();
  return rc;
}

size_t reduce_scratch_bytes(int dtype, size_t n, const void *a, const void *b) {
  size_t es = dtype_size(dtype);
  if (!es) return 0;
  // Without pointers, assume the worst alignment (scalar path has the most runs).
  Shape sh = reduce_shape(es, n, a ? a : (const void *)(uintptr_t)16,
                          b ? b : (a ? a : (const void *)(uintptr_t)16));
  if (!a) {
    Shape s2 = reduce_shape(es, n, (const void *)(uintptr_t)16, (const void *)(uintptr_t)8);
    sh.runs = std::max(sh.runs, s2.runs);
  }
  return kScratchPrefix + (size_t)std::max<long long>(sh.runs, 1) * sizeof(StatusWord);
}

int launch_reduce(int dtype, int op, const void *a, const void *b, size_t n, void *out,
                  const void *init, void *scratch, size_t sb, int config, cudaStream_t st) {
  switch (dtype) {
  case B2P_I32: return dispatch_op<B2P_I32>(op, a, b, n, out, init, scratch, sb, config, st);
  case B2P_I64: return dispatch_op<B2P_I64>(op, a, b, n, out, init, scratch, sb, config, st);
  case B2P_U32: return dispatch_op<B2P_U32>(op, a, b, n, out, init, scratch, sb, config, st);
  case B2P_U64: return dispatch_op<B2P_U64>(op, a, b, n, out, init, scratch, sb, config, st);
  case B2P_F32: return dispatch_op<B2P_F32>(op, a, b, n, out, init, scratch, sb, config, st);
  case B2P_BF16: return dispatch_op<B2P_BF16>(op, a, b, n, out, init, scratch, sb, config, st);
  case B2P_F64: return dispatch_op<B2P_F64>(op, a, b, n, out, init, scratch, sb, config, st);
  default: return B2P_ERR_INVALID_ARG;
  }
}

}  // namespace b2p

extern "C" int b2p_kernel_arch(int *binary_version, int *ptx_version) {
  using P = b2p::PolicyOf<B2P_I32, B2P_SUM>::type;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)b2p::reduce_kernel<P, false, true>);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return B2P_ERR_CUDA;
  }
  if (binary_version) *binary_version = fa.binaryVersion;
  if (ptx_version) *ptx_version = fa.ptxVersion;
  return B2P_OK;
}
