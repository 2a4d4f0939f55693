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
#include "b2p_device/reduce.cuh"
#include "internal.h"

#include <algorithm>

namespace b2p {

// ---------------------------------------------------------------- host

namespace {

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
