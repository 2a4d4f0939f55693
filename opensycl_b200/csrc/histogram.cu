// 256-bin byte histogram with atomic_ref::fetch_add semantics.
//
// The reference pattern is a parallel_for whose work-items each call
// sycl::atomic_ref<uint32_t, relaxed, device>::fetch_add(1) on bins[key]
// (sycl/libkernel/atomic_ref.hpp:143-149,253-260; on CUDA one global
// atomicAdd per element, generic/hiplike/atomic_builtins.hpp:439-447), so hot
// bins of a skewed key distribution serialise in L2.
//
// Here each block keeps 32 replicas of the 256 counters in shared memory,
// replica = lane: counter (key, lane) lives at word key*32 + lane, which is
// always bank `lane`, so a warp's 32 increments never conflict on a bank and
// never hit the same word, however skewed the keys are.  Replicas are summed
// at the end and added to the global bins with one atomicAdd per non-zero
// bin per block.  Keys are read 16 per thread per 16-byte load.
//
// Two ways of bringing the keys in:
//   histogram_u8_kernel      every thread loads its own 16-byte vectors
//                            (small inputs, grid modes 0 and 2)
//   histogram_u8_tma_kernel  one block per SM; a producer warp streams
//                            ~31 KiB chunks of keys into a ring of shared
//                            stages with bulk copies (cp.async.bulk) while
//                            31 counting warps work on landed chunks, so
//                            loads stay in flight while the atomics run
//                            (grid mode 1)
#include "b2p_device/common.cuh"
#include "internal.h"
#include "b2p_device/tile.cuh"
#include "b2p_device/tma.cuh"

#include <algorithm>

namespace b2p {

// Error word of the calls that take no scratch buffer (the histogram):
// B2P_ERR_TIMEOUT when a bounded wait ran out.  Read by b2p_device_error
// with a null scratch pointer.
__device__ unsigned g_scratchless_error;

namespace {

// Shared-memory byte offset of counter (key, lane): word key * 32 + lane, so
// (key << 7) | (lane << 2); the key is byte b of w.
__device__ __forceinline__ unsigned counter_offset(unsigned w, int b, unsigned lane4) {
  const unsigned k7 = b == 0 ? (w << 7) : (w >> (8 * b - 7));
  return (k7 & 0x7f80u) | lane4;
}

__device__ __forceinline__ void count_word(char *hist, unsigned w, unsigned lane4) {
#pragma unroll
  for (int b = 0; b < 4; ++b) atomicAdd(reinterpret_cast<unsigned *>(hist + counter_offset(w, b, lane4)), 1u);
}

// Sum the 32 replicas of each bin into the global bins.
__device__ __forceinline__ void flush_bins(const unsigned *hist, uint32_t *bins, int nbins) {
  for (int bin = threadIdx.x; bin < nbins; bin += blockDim.x) {
    const unsigned *row = hist + bin * 32;
    unsigned s = 0;
#pragma unroll
    for (int r = 0; r < 32; ++r) s += row[(r + bin) & 31];  // rotate to spread banks
    if (s) atomicAdd(bins + bin, s);
  }
}

}  // namespace

__global__ void __launch_bounds__(1024) histogram_u8_kernel(const uint8_t *__restrict__ keys,
                                                            unsigned long long n,
                                                            unsigned long long head,
                                                            uint32_t *__restrict__ bins, int nbins,
                                                            int vec_per_iter) {
  extern __shared__ __align__(16) unsigned hist[];  // 256 * 32 words
  const int lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < 256 * 32; i += blockDim.x) hist[i] = 0;
  __syncthreads();

  unsigned *mine = hist + lane;
  const unsigned lane4 = (unsigned)lane * 4u;
  auto count4 = [&](unsigned w) { count_word(reinterpret_cast<char *>(hist), w, lane4); };

  // unaligned head (< 16 keys), block 0 only
  if (blockIdx.x == 0)
    for (unsigned long long i = threadIdx.x; i < head; i += blockDim.x)
      atomicAdd(mine + ((unsigned)keys[i] << 5), 1u);

  const uint4 *kv = reinterpret_cast<const uint4 *>(keys + head);
  const unsigned long long nvec = (n - head) / 16;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long v = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  // vec_per_iter 16-byte loads in flight per thread
  for (; v + (unsigned long long)(vec_per_iter - 1) * stride < nvec;
       v += (unsigned long long)vec_per_iter * stride) {
    uint4 buf[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k < vec_per_iter) buf[k] = ld_stream_v4(kv + v + (unsigned long long)k * stride);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k < vec_per_iter) {
        count4(buf[k].x);
        count4(buf[k].y);
        count4(buf[k].z);
        count4(buf[k].w);
      }
  }
  for (; v < nvec; v += stride) {
    uint4 w = ld_stream_v4(kv + v);
    count4(w.x);
    count4(w.y);
    count4(w.z);
    count4(w.w);
  }
  // tail (< 16 keys), last block only
  if (blockIdx.x == gridDim.x - 1) {
    const unsigned long long ts = head + nvec * 16;
    for (unsigned long long i = ts + threadIdx.x; i < n; i += blockDim.x)
      atomicAdd(mine + ((unsigned)keys[i] << 5), 1u);
  }
  __syncthreads();
  flush_bins(hist, bins, nbins);
}

constexpr int kHistCountWarps = 31;  // + 1 producer warp = 1024 threads
constexpr int kHistVecPerThread = 2;
constexpr unsigned kHistChunk = kHistCountWarps * 32 * 16 * kHistVecPerThread;  // 31,744 bytes
constexpr int kHistStages = 4;

// Body = the 16-byte-aligned keys [head, head + body); chunk c = bytes
// [c * kHistChunk, ...) of the body, block b takes chunks b, b + grid, ...
// Keys before the body (head, < 16) and after it (tail, < 16) use plain
// loads.
__global__ void __launch_bounds__(1024, 1)
    histogram_u8_tma_kernel(const uint8_t *__restrict__ keys, unsigned long long n, unsigned long long head,
                            unsigned long long body, uint32_t *__restrict__ bins, int nbins,
                            unsigned long long timeout_ns) {
  extern __shared__ __align__(16) unsigned hist[];  // 256 * 32 counters, then the stages
  char *stages = reinterpret_cast<char *>(hist + 256 * 32);
  __shared__ __align__(8) uint64_t full[kHistStages], empty[kHistStages];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lane4 = (unsigned)lane * 4u;
  for (int i = threadIdx.x; i < 256 * 32; i += blockDim.x) hist[i] = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kHistStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kHistCountWarps);
    }
    mbar_init_fence();
  }
  __syncthreads();
  const unsigned long long nchunks = (body + kHistChunk - 1) / kHistChunk;
  const uint8_t *base = keys + head;

  if (warp == kHistCountWarps) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      const unsigned long long pol = l2_policy_stream();
      RingPos r;
      unsigned long long it = 0;
      for (unsigned long long c = blockIdx.x; c < nchunks; c += gridDim.x, ++it, r.advance(1, kHistStages)) {
        if (!mbar_wait(&empty[r.s], r.ph ^ 1u, timeout_ns)) {
          atomicCAS(&g_scratchless_error, 0u, (unsigned)B2P_ERR_TIMEOUT);
          break;
        }
        const unsigned bytes = (unsigned)min((unsigned long long)kHistChunk, body - c * kHistChunk);
        mbar_arrive_expect_tx(&full[r.s], bytes);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
            " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(stages + (size_t)r.s * kHistChunk)),
            "l"(base + c * kHistChunk), "r"(bytes), "r"(smem_u32(&full[r.s])), "l"(pol)
            : "memory");
      }
      // the copies still in flight land before the block leaves
      RingPos q;
      for (unsigned long long j = 0; j < it; ++j, q.advance(1, kHistStages))
        if (j + kHistStages >= it) (void)mbar_wait(&full[q.s], q.ph, timeout_ns);
    }
  } else {
    // ------------------------------------------------------ counting warps
    const int ct = threadIdx.x;  // 0 .. 32 * kHistCountWarps - 1
    RingPos r;
    for (unsigned long long c = blockIdx.x; c < nchunks; c += gridDim.x, r.advance(1, kHistStages)) {
      if (!mbar_wait(&full[r.s], r.ph, timeout_ns)) {
        if (lane == 0) atomicCAS(&g_scratchless_error, 0u, (unsigned)B2P_ERR_TIMEOUT);
        break;
      }
      const unsigned nv = (unsigned)(min((unsigned long long)kHistChunk, body - c * kHistChunk) / 16);
      const uint4 *src = reinterpret_cast<const uint4 *>(stages + (size_t)r.s * kHistChunk);
      uint4 v[kHistVecPerThread];
#pragma unroll
      for (int k = 0; k < kHistVecPerThread; ++k) {
        const unsigned i = (unsigned)ct + (unsigned)k * (32u * kHistCountWarps);
        v[k] = i < nv ? src[i] : make_uint4(0, 0, 0, 0);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[r.s]);  // the stage is read
#pragma unroll
      for (int k = 0; k < kHistVecPerThread; ++k) {
        if ((unsigned)ct + (unsigned)k * (32u * kHistCountWarps) < nv) {
          count_word(reinterpret_cast<char *>(hist), v[k].x, lane4);
          count_word(reinterpret_cast<char *>(hist), v[k].y, lane4);
          count_word(reinterpret_cast<char *>(hist), v[k].z, lane4);
          count_word(reinterpret_cast<char *>(hist), v[k].w, lane4);
        }
      }
    }
    // head (< 16 keys) in block 0, tail (< 16 keys) in the last block
    char *h = reinterpret_cast<char *>(hist);
    if (blockIdx.x == 0 && (unsigned long long)ct < head)
      atomicAdd(reinterpret_cast<unsigned *>(h + ((unsigned)keys[ct] << 7) + lane4), 1u);
    const unsigned long long ts = head + body;
    if (blockIdx.x == gridDim.x - 1 && ts + (unsigned long long)ct < n)
      atomicAdd(reinterpret_cast<unsigned *>(h + ((unsigned)keys[ts + ct] << 7) + lane4), 1u);
  }
  __syncthreads();
  flush_bins(hist, bins, nbins);
}

int launch_histogram_u8(const uint8_t *keys, size_t n, uint32_t *bins, int nbins, int config,
                        cudaStream_t st) {
  LaunchConfig lc = describe_config(config);
  if (lc.grid_mode == 1 && n >= ((size_t)1 << 22)) {
    const size_t smem = 256 * 32 * sizeof(unsigned) + (size_t)kHistStages * kHistChunk;
    const void *kfn = (const void *)histogram_u8_tma_kernel;
    int rc = ensure_dynamic_smem(kfn, smem);
    if (rc) return rc;
    if (occupancy(kfn, 1024, smem) >= 1) {
      const unsigned long long head =
          std::min<unsigned long long>((16 - (reinterpret_cast<uintptr_t>(keys) & 15)) & 15, n);
      const unsigned long long body = (n - head) / 16 * 16;
      const unsigned long long nchunks = (body + kHistChunk - 1) / kHistChunk;
      const int grid = (int)std::min<unsigned long long>(nchunks, (unsigned long long)device_info().sm_count);
      histogram_u8_tma_kernel<<<grid, 1024, smem, st>>>(keys, n, head, body, bins, nbins, wait_timeout_ns());
      return cuda_status(cudaGetLastError());
    }
  }
  const size_t smem = 256 * 32 * sizeof(unsigned);
  const void *kfn = (const void *)histogram_u8_kernel;
  int rc = ensure_dynamic_smem(kfn, smem);
  if (rc) return rc;
  unsigned long long head = (16 - (reinterpret_cast<uintptr_t>(keys) & 15)) & 15;
  if (head > n) head = n;
  const unsigned long long nvec = (n - head) / 16;
  int vpi = lc.items / 4;  // items {4,8,16,32} -> {1,2,4,8} vectors in flight
  if (vpi < 1) vpi = 1;
  if (vpi > 8) vpi = 8;
  long long units = (long long)((nvec + (unsigned long long)lc.block * vpi - 1) /
                                ((unsigned long long)lc.block * vpi));
  int grid = grid_for(lc.grid_mode, units > 0 ? units : 1, 1, kfn, lc.block, smem);
  histogram_u8_kernel<<<grid, lc.block, smem, st>>>(keys, n, head, bins, nbins, vpi);
  return cuda_status(cudaGetLastError());
}

int scratchless_error(int clear) {
  unsigned v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_scratchless_error, sizeof(v));
  if (e != cudaSuccess) return cuda_status(e);
  if (clear && v) {
    const unsigned z = 0;
    e = cudaMemcpyToSymbol(g_scratchless_error, &z, sizeof(z));
    if (e != cudaSuccess) return cuda_status(e);
  }
  return (int)v;
}

}  // namespace b2p
