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
#include "common.cuh"
#include "internal.h"

namespace b2p {

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
  auto count4 = [&](unsigned w) {
#pragma unroll
    for (int b = 0; b < 4; ++b) atomicAdd(mine + (((w >> (8 * b)) & 0xffu) << 5), 1u);
  };

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
  for (int bin = threadIdx.x; bin < nbins; bin += blockDim.x) {
    const unsigned *row = hist + bin * 32;
    unsigned s = 0;
#pragma unroll
    for (int r = 0; r < 32; ++r) s += row[(r + bin) & 31];  // rotate to spread banks
    if (s) atomicAdd(bins + bin, s);
  }
}

int launch_histogram_u8(const uint8_t *keys, size_t n, uint32_t *bins, int nbins, int config,
                        cudaStream_t st) {
  LaunchConfig lc = describe_config(config);
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

}  // namespace b2p
