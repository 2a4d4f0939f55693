// Tensor-memory-accelerator (TMA) plumbing of the pipelined kernels: the
// mbarrier protocol between the producer warp, the look-back warps and the
// consumer warps of one block, 2-D bulk tensor copies between global memory
// and 128-byte-swizzled shared tiles, bulk-store groups, and the host-side
// encoding of a byte array as a 2-D "rows of 128 bytes" tensor.
//
// The 128-byte swizzle of a TMA tile places 16-byte chunk c of row r at
// chunk c ^ (r & 7) of a 1024-byte-aligned buffer: exactly the layout swz()
// in tile.cuh produces, so the blocked per-thread reads of the tile kernels
// work on TMA-filled buffers unchanged and stay bank-conflict free.
//
// Every wait here is bounded (%globaltimer); a caller that sees a wait run
// out records B2P_ERR_TIMEOUT and leaves its loop.
#pragma once

#include <cuda.h>

#include "common.cuh"

#include <mutex>

namespace b2p {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async proxy (TMA) before use.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// Arrive and announce `bytes` of TMA transactions for the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint: the thread is parked (issues nothing)
// until the phase completes or about `hint_ns` pass.  Waiting warps of the
// pipelined kernels share their SM sub-partitions with the warps doing the
// work; a wait that spins on try_wait without the hint takes issue slots
// from them.
__device__ __forceinline__ bool mbar_try_hint(uint64_t *b, unsigned parity, unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity to complete; false after
// timeout_ns without completion.  Each try_wait parks the thread for up to
// 100 us (it resumes as soon as the phase completes); the clock is read
// between tries.
constexpr unsigned kWaitHintNs = 100000;
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity, unsigned long long timeout_ns) {
  uint64_t t0 = 0;
  for (;;) {
    if (mbar_try_hint(b, parity, kWaitHintNs)) return true;
    const uint64_t now = globaltimer_ns();
    if (t0 == 0) t0 = now;
    else if (now - t0 > timeout_ns) return false;
  }
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// Global -> shared tile copy of box (x, y); completes `bytes` on *bar.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar, unsigned long long l2_policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      ".L2::cache_hint [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(l2_policy)
      : "memory");
}

// Shared -> global tile copy of box (x, y); rows outside the tensor are
// not written.  Tracked by the issuing thread's bulk groups.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int x, int y, const void *src,
                                             unsigned long long l2_policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group.L2::cache_hint"
      " [%0, {%1, %2}], [%3], %4;" ::"l"(map),
      "r"(x), "r"(y), "r"(smem_u32(src)), "l"(l2_policy)
      : "memory");
}

// Global -> shared untiled bulk copy of `bytes` (16-byte aligned addresses,
// a multiple of 16 bytes); completes `bytes` on *bar.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                          unsigned long long pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Wait until at most N of this thread's bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Wait until all of this thread's bulk groups completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Order this thread's generic shared-memory writes before later async-proxy
// (TMA) reads of them.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Barrier over the first `count` threads of the block (named barrier `id`).
__device__ __forceinline__ void bar_named(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Position in the ring of stages: stage index and mbarrier phase parity of
// an item, advanced without divisions.
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

// Host: describe [base, base + rows * 128) as a tensor of `rows` rows of 128
// bytes, read and written in boxes of box_rows rows with the 128-byte
// swizzle.  base must be 16-byte aligned, 1 <= rows < 2^31, 1 <= box_rows
// <= 256.  Returns false when the driver entry point is missing or rejects
// the description.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_fn() {
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

inline bool encode_row_tensor(CUtensorMap *map, const void *base, unsigned long long rows, int box_rows) {
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


}  // namespace b2p
