// LSD radix sort of 4- and 8-byte keys: b2p_sort's path for the standard key
// types (int32/int64/uint32/uint64/float/double with < or >), where the
// reference runs its bitonic network (algorithms/sort/bitonic_sort.hpp:
// 69-110, log2(n)^2 / 2 global passes).
//
// Keys are mapped to unsigned "order keys" whose unsigned order is the key
// order (signed: sign bit flipped; floats: all bits flipped when negative,
// else the sign bit set; -0.0 takes the order key of +0.0, so the two zeros
// are equal as under <; descending: the complement).  The sort moves the
// original bits and is stable, so its result is the stable sort by the key
// order: the same as a stable merge sort with < or >.
//
// Each digit pass (4 for 32-bit keys, 8 for 64-bit) is a reduce-then-scan
// over persistent blocks, ping-ponging between the keys and a second array:
//   * upsweep: block b counts the digits of its contiguous chunk of tiles
//     (per-warp shared-memory counts), counts[d][b];
//   * spine: per digit, an exclusive scan of its counts over the chunks and
//     its total; a digit's first slot in chunk b is then the keys of smaller
//     digits plus the keys of that digit in chunks before b;
//   * downsweep: block b walks its chunk's tiles in order.  Its warps rank
//     each tile's keys in key order (warp w owns 32 consecutive keys per
//     round; lanes holding the same digit find each other with one ballot
//     per digit bit, and a per-warp count per digit gives each key its
//     rank), the keys are
//     reordered by digit in shared memory, written to their slots (running
//     slot of the digit + position in the tile's run of that digit), and the
//     running slots advance by the tile's counts.
// Nothing waits on another block, and the sort is stable: chunks, tiles and
// keys inside a tile are taken in index order.
#pragma once

#include "common.cuh"

#include <algorithm>

namespace b2p {

constexpr int kRadixBits = 8, kRadixBins = 1 << kRadixBits;
constexpr int kRadixThreads = 256, kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;  // 4096 keys
constexpr int kRadixWarps = kRadixThreads / 32;
constexpr int kRadixBlocksPerSm = 4;
constexpr int kRadixSpineThreads = 1024;
// 32-bit slots: inputs below 2^31 keys
constexpr size_t kRadixMaxKeys = (size_t)1 << 31;

template <class T>
struct RadixKey {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte keys");
  using U = typename std::conditional<sizeof(T) == 4, unsigned, unsigned long long>::type;
  static constexpr int kPasses = (int)sizeof(T) * 8 / kRadixBits;
  static constexpr U kSign = (U)1 << (sizeof(T) * 8 - 1);
  __device__ __forceinline__ static U order(const T &x, bool desc) {
    U u;
    memcpy(&u, &x, sizeof(T));
    U k;
    if constexpr (std::is_floating_point<T>::value) {
      if (u == kSign) u = 0;  // -0.0 == +0.0
      k = (u & kSign) ? (U)~u : (U)(u | kSign);
    } else if constexpr (std::is_signed<T>::value) {
      k = u ^ kSign;
    } else {
      k = u;
    }
    return desc ? (U)~k : k;
  }
  __device__ __forceinline__ static unsigned digit(const T &x, bool desc, int pass) {
    return (unsigned)(order(x, desc) >> (pass * kRadixBits)) & (kRadixBins - 1);
  }
};

// Scratch of a radix sort of n keys of T with `blocks` persistent blocks:
// the per-chunk digit counts (then their prefixes), the digit totals and the
// second key array.
struct RadixLayout {
  size_t counts, totals, keys, total;
  long long ntiles;
  int blocks;
  long long chunk;  // tiles per block
};

template <class T>
inline RadixLayout radix_layout(size_t n, int sm_count) {
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  RadixLayout l;
  l.ntiles = (long long)((n + kRadixTile - 1) / kRadixTile);
  const long long want = (long long)std::max(sm_count, 1) * kRadixBlocksPerSm;
  l.chunk = (l.ntiles + want - 1) / want;
  l.blocks = (int)((l.ntiles + l.chunk - 1) / l.chunk);
  l.counts = kHeaderBytes;
  l.totals = l.counts + up((size_t)kRadixBins * l.blocks * 4);
  l.keys = l.totals + up((size_t)kRadixBins * 4);
  l.total = l.keys + up(n * sizeof(T));
  return l;
}

// Scratch bytes for any device of up to 256 SMs (the block count follows the
// SM count).
template <class T>
inline size_t radix_scratch_bytes(size_t n) {
  return radix_layout<T>(n, 256).total + 256;
}

// Lanes of the warp whose label (a digit, or 256 for a key past the end)
// equals this lane's: one ballot per label bit (BITS = 8 when every key of
// the round is real, 9 otherwise).
template <int BITS>
__device__ __forceinline__ unsigned radix_peers(unsigned label) {
  unsigned peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    const bool bit = (label >> b) & 1u;
    const unsigned m = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

// Upsweep: digit counts of block b's chunk of tiles, counts[d * blocks + b].
template <class T>
__global__ void __launch_bounds__(kRadixThreads) radix_upsweep_kernel(const T *keys, size_t n, bool desc, int pass,
                                                                    long long chunk, unsigned *counts) {
  __shared__ unsigned sh[kRadixWarps][kRadixBins];  // one histogram per warp
  for (int i = threadIdx.x; i < kRadixWarps * kRadixBins; i += kRadixThreads) (&sh[0][0])[i] = 0;
  __syncthreads();
  unsigned *wsh = sh[threadIdx.x >> 5];
  const size_t b0 = (size_t)blockIdx.x * chunk * kRadixTile;
  const size_t b1 = min(n, b0 + (size_t)chunk * kRadixTile);
  // a tile at a time, every thread's kRadixItems loads in flight together
  for (size_t base = b0; base < b1; base += kRadixTile) {
    T key[kRadixItems];
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const size_t i = base + (size_t)r * kRadixThreads + threadIdx.x;
      if (i < b1) key[r] = keys[i];
    }
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const size_t i = base + (size_t)r * kRadixThreads + threadIdx.x;
      if (i < b1) atomicAdd(&wsh[RadixKey<T>::digit(key[r], desc, pass)], 1u);
    }
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadixBins; d += kRadixThreads) {
    unsigned c = 0;
#pragma unroll
    for (int w = 0; w < kRadixWarps; ++w) c += sh[w][d];
    counts[(size_t)d * gridDim.x + blockIdx.x] = c;
  }
}

// Spine, one block per digit d: exclusive scan of the digit's chunk counts
// counts[d][0 .. blocks) in place (blocks <= kRadixSpineThreads), and the
// digit's total into totals[d].
__global__ void __launch_bounds__(kRadixSpineThreads) radix_spine_kernel(unsigned *counts, int blocks,
                                                                       unsigned *totals) {
  __shared__ unsigned s_warp[kRadixSpineThreads / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  unsigned *row = counts + (size_t)blockIdx.x * blocks;
  const unsigned c = t < blocks ? row[t] : 0u;
  unsigned incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  unsigned before = 0;
  for (int w = 0; w < warp; ++w) before += s_warp[w];
  if (t < blocks) row[t] = before + incl - c;
  if (t == kRadixSpineThreads - 1) totals[blockIdx.x] = before + incl;
}

// Dynamic shared memory of radix_downsweep_kernel<T>: the tile's keys,
// per-warp digit counts (257 buckets: 256 = past the end), the tile's
// counts, the running output slots and the tile-local digit starts.
template <class T>
constexpr size_t radix_pass_smem() {
  return sizeof(T) * kRadixTile + sizeof(unsigned) * (kRadixWarps * (kRadixBins + 1) + 3 * kRadixBins);
}

// Downsweep: block b moves its chunk's keys from `in` to their slots in
// `out` by digit `pass`, tile by tile; prefix[d * blocks + b] counts digit d
// in the chunks before b, totals[d] in the whole input (the spine's results).
template <class T>
__global__ void __launch_bounds__(kRadixThreads, kRadixBlocksPerSm)
    radix_downsweep_kernel(const T *in, T *out, size_t n, bool desc, int pass, long long chunk,
                           const unsigned *prefix, const unsigned *totals) {
  extern __shared__ __align__(16) unsigned char radix_smem[];
  T *s_keys = reinterpret_cast<T *>(radix_smem);
  unsigned *s_wh = reinterpret_cast<unsigned *>(radix_smem + sizeof(T) * kRadixTile);
  unsigned *s_tot = s_wh + kRadixWarps * (kRadixBins + 1);
  unsigned *s_run = s_tot + kRadixBins;
  unsigned *s_lstart = s_run + kRadixBins;
  __shared__ unsigned s_scan[kRadixBins / 32];

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  {
    // first slot of digit t for this chunk: keys of smaller digits (an
    // exclusive scan of the digit totals) + keys of digit t in earlier chunks
    const unsigned c = totals[t];
    unsigned incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_scan[warp] = incl;
    __syncthreads();
    unsigned before = 0;
    for (int w = 0; w < warp; ++w) before += s_scan[w];
    s_run[t] = before + incl - c + prefix[(size_t)t * gridDim.x + blockIdx.x];
    __syncthreads();
  }
  const long long tile_begin = (long long)blockIdx.x * chunk;
  const long long ntiles = (long long)((n + kRadixTile - 1) / kRadixTile);
  const long long tile_end = min(ntiles, tile_begin + chunk);
  const unsigned lt = (1u << lane) - 1u;
  const int wbase = warp * (32 * kRadixItems);
  unsigned *wh = s_wh + warp * (kRadixBins + 1);

  for (long long tile = tile_begin; tile < tile_end; ++tile) {
    for (int i = t; i < kRadixWarps * (kRadixBins + 1); i += kRadixThreads) s_wh[i] = 0;
    __syncthreads();  // also: the previous tile's keys and slots are used up
    const size_t tile0 = (size_t)tile * kRadixTile;
    const int count = (int)min((size_t)kRadixTile, n - tile0);
    // keys of this thread: warp-owned run, 32 consecutive keys per round; a
    // key's digit (9 bits: 256 = past the end) and its rank among the warp's
    // keys of that digit (13 bits) share one register
    T key[kRadixItems];
    unsigned rd[kRadixItems];
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const int j = wbase + r * 32 + lane;
      if (j < count) key[r] = in[tile0 + j];
    }
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const int j = wbase + r * 32 + lane;
      const unsigned d = j < count ? RadixKey<T>::digit(key[r], desc, pass) : (unsigned)kRadixBins;
      // a full tile has no key past the end: the 9th label bit is always 0
      const unsigned peers = count == kRadixTile ? radix_peers<kRadixBits>(d) : radix_peers<kRadixBits + 1>(d);
      const unsigned base = wh[d];
      rd[r] = ((base + (unsigned)__popc(peers & lt)) << 9) | d;
      __syncwarp();
      if (lane == __ffs(peers) - 1) wh[d] = base + (unsigned)__popc(peers);
      __syncwarp();
    }
    __syncthreads();
    for (int d = t; d < kRadixBins; d += kRadixThreads) {
      // this digit's per-warp counts -> exclusive bases, and the tile count
      unsigned sum = 0;
#pragma unroll
      for (int w = 0; w < kRadixWarps; ++w) {
        const unsigned c = s_wh[w * (kRadixBins + 1) + d];
        s_wh[w * (kRadixBins + 1) + d] = sum;
        sum += c;
      }
      s_tot[d] = sum;
    }
    __syncthreads();
    // first slot of each digit inside the tile: exclusive scan of the counts
    // (one digit per thread: kRadixThreads == kRadixBins)
    {
      const unsigned c = s_tot[t];
      unsigned incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane == 31) s_scan[warp] = incl;
      __syncthreads();
      unsigned before = 0;
      for (int w = 0; w < warp; ++w) before += s_scan[w];
      s_lstart[t] = before + incl - c;
    }
    __syncthreads();
    // reorder the tile by digit in shared memory (stable)
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const unsigned d = rd[r] & 511u;
      if (d < kRadixBins) {
        const unsigned pos = s_lstart[d] + s_wh[warp * (kRadixBins + 1) + d] + (rd[r] >> 9);
        s_keys[pos] = key[r];
      }
    }
    __syncthreads();
    // each key to its slot
    for (int i = t; i < count; i += kRadixThreads) {
      const T x = s_keys[i];
      const unsigned d = RadixKey<T>::digit(x, desc, pass);
      const size_t g = (size_t)s_run[d] + (unsigned)(i - (int)s_lstart[d]);
      if (g < n) out[g] = x;
    }
    __syncthreads();
    s_run[t] += s_tot[t];
  }
}

// Radix sort of keys[0..n) in place (stable, by the key order; descending:
// the reversed order, still stable).  1 < n < kRadixMaxKeys; scratch:
// radix_scratch_bytes<T>(n) bytes of device memory, 256-byte aligned.
template <class T>
int launch_radix_sort(T *keys, size_t n, bool desc, void *scratch, size_t scratch_bytes, int sm_count,
                      cudaStream_t st) {
  static_assert(kRadixThreads == kRadixBins, "one digit per thread in the tile scans");
  constexpr int P = RadixKey<T>::kPasses;
  if (n <= 1) return B2P_OK;
  if (n >= kRadixMaxKeys || sm_count > 256) return B2P_ERR_UNSUPPORTED;
  const RadixLayout l = radix_layout<T>(n, sm_count);
  if (!scratch || scratch_bytes < l.total || (reinterpret_cast<uintptr_t>(scratch) & 255)) return B2P_ERR_SCRATCH;
  char *s = reinterpret_cast<char *>(scratch);
  unsigned *counts = reinterpret_cast<unsigned *>(s + l.counts);
  unsigned *totals = reinterpret_cast<unsigned *>(s + l.totals);
  T *buf = reinterpret_cast<T *>(s + l.keys);
  if (l.blocks > kRadixSpineThreads) return B2P_ERR_UNSUPPORTED;
  constexpr size_t smem = radix_pass_smem<T>();
  if (cudaFuncSetAttribute((const void *)radix_downsweep_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return B2P_ERR_CUDA;
  const T *src = keys;
  T *dst = buf;
  for (int p = 0; p < P; ++p) {
    radix_upsweep_kernel<T><<<l.blocks, kRadixThreads, 0, st>>>(src, n, desc, p, l.chunk, counts);
    radix_spine_kernel<<<kRadixBins, kRadixSpineThreads, 0, st>>>(counts, l.blocks, totals);
    radix_downsweep_kernel<T><<<l.blocks, kRadixThreads, smem, st>>>(src, dst, n, desc, p, l.chunk, counts,
                                                                      totals);
    src = dst;
    dst = (dst == buf) ? keys : buf;
  }
  // an even number of passes ends in `keys`
  return cudaGetLastError() == cudaSuccess ? B2P_OK : B2P_ERR_CUDA;
}

}  // namespace b2p
