// Merge and sort, shared by libb2p (b2p_merge, b2p_sort) and the
// header-only C++ layer (hipsycl::algorithms::merge / sort and the stdpar
// std::merge / std::sort overloads with any comparator).
//
// Replaces the reference's merge (algorithms/merge/merge.hpp:222-313:
// merge-path partitioning, hierarchical hybrid merge) and sort
// (algorithms/sort/bitonic_sort.hpp:69-110: an in-place bitonic network of
// log2(n)^2 / 2 global passes) with:
//   merge  one pass over the output in tiles: a partition kernel finds
//          where every tile starts on the merge path (one warp per tile,
//          a 32-way search along the tile's first diagonal), then each
//          block stages its tile's two input ranges in shared memory and
//          every thread merges its ITEMS outputs after its own merge-path
//          search in shared memory; outputs leave in coalesced rows.
//          Reads each input once, writes each output once.
//   sort   a merge sort: blocks sort tiles in shared memory (a stable
//          odd-even sort of each thread's ITEMS keys in registers, then
//          log2(threads) rounds of merge-path merges of runs in shared
//          memory), then log2(n / tile) global passes of the merge above on
//          pairs of runs, ping-ponging between the keys and a scratch array.
// Both are stable: on equal keys the element of the first range (the
// earlier run) comes first, as std::merge requires.  comp(x, y) is a strict
// weak order ("x before y").
#pragma once

#include "common.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>

namespace b2p {

constexpr int kMergeThreads = 256;
// Keys per thread: 64 bytes of keys (the block sort's two shared tiles stay
// within 32 KiB), at most 16.
template <class T>
__host__ __device__ constexpr int merge_items() {
  return sizeof(T) <= 4 ? 16 : (sizeof(T) <= 8 ? 8 : (sizeof(T) <= 16 ? 4 : (sizeof(T) <= 32 ? 2 : 1)));
}
template <class T>
__host__ __device__ constexpr int merge_tile() {
  return kMergeThreads * merge_items<T>();
}

// Number of elements of `a` among the first `diag` outputs of the stable
// merge of a[0..na) and b[0..nb) (a(i), b(i) read element i): the first i
// in [max(0, diag - nb), min(diag, na)] whose b[diag - 1 - i] is strictly
// before a[i].
template <class T, class Comp, class IdxA, class IdxB>
__device__ __forceinline__ long long merge_path(IdxA a, long long na, IdxB b, long long nb, long long diag,
                                                const Comp &comp) {
  long long lo = diag > nb ? diag - nb : 0;
  long long hi = diag < na ? diag : na;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    // a[mid] goes before b[diag - 1 - mid] unless b's key is strictly smaller
    if (!comp(b(diag - 1 - mid), a(mid))) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// merge_path() by one warp: each round the 32 lanes test 32 evenly spaced
// points of the remaining range at once and keep the gap where the answer
// lies (a range of `span` shrinks to about span / 33 per round: 6 rounds of
// global-memory latency for 2^28 keys instead of 28).  Every lane returns
// the same value.
template <class T, class Comp, class IdxA, class IdxB>
__device__ __forceinline__ long long merge_path_warp(IdxA a, long long na, IdxB b, long long nb, long long diag,
                                                     const Comp &comp) {
  const int lane = threadIdx.x & 31;
  long long lo = diag > nb ? diag - nb : 0;
  long long hi = diag < na ? diag : na;
  while (lo < hi) {
    const long long span = hi - lo;
    if (span <= 32) {
      const bool p = lane < span && comp(b(diag - 1 - (lo + lane)), a(lo + lane));
      const unsigned m = __ballot_sync(0xffffffffu, p);
      return m ? lo + (__ffs(m) - 1) : hi;
    }
    // probes lo + span * (k + 1) / 33, k = 0..31: strictly increasing, < hi
    const long long pk = lo + span * (lane + 1) / 33;
    const bool p = comp(b(diag - 1 - pk), a(pk));
    const unsigned m = __ballot_sync(0xffffffffu, p);
    const int j = m ? __ffs(m) - 1 : 32;
    const long long new_lo = j == 0 ? lo : lo + span * j / 33 + 1;
    const long long new_hi = j == 32 ? hi : lo + span * (j + 1) / 33;
    lo = new_lo;
    hi = new_hi;
  }
  return lo;
}

// Shared-memory slot of tile element i: one pad slot after every 32, so
// the threads of a warp, whose runs start ITEMS (a power of two) apart,
// read and write 32 different banks.
__device__ __forceinline__ int spad(int i) { return i + (i >> 5); }
__host__ __device__ constexpr int spad_size(int n) { return n + n / 32; }
// Shared slots of a padded tile of n keys plus the spare slot one past it
// (read, never used, by merge_serial when a side ends at the tile's end).
__host__ __device__ constexpr int spad_alloc(int n) { return spad_size(n) + 1; }

// Serial stable merge of ITEMS outputs starting at a[ia], b[ib] of the two
// ranges s[pad(a0 + i)] and s[pad(b0 + i)] of one padded shared array
// into out[]; the current key of each range stays in a register, and each
// output costs one shared load, without branches (the warp's threads take
// different sides).  Outputs past the end of both ranges are left
// unspecified.  The second range follows the first (b0 >= a0 + na), and
// reads stay in slots a0 .. b0 + nb: one past the end of a side is the
// first slot of the next range or, past the tile, the array's spare last
// slot (kept by spad_alloc); once both sides are exhausted the a-side index,
// which keeps counting, is held at b0 + nb.  Keys read past a side's end
// are never compared or used.
template <class T, int ITEMS, class Comp>
__device__ __forceinline__ void merge_serial(const T *s, int a0, int ia, int na, int b0, int ib, int nb,
                                             T (&out)[ITEMS], const Comp &comp) {
  const int end = b0 + nb;
  T va = s[spad(a0 + ia)];
  T vb = s[spad(b0 + ib)];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const bool take_b = ib < nb && (ia >= na || comp(vb, va));
    out[k] = take_b ? vb : va;
    ia += take_b ? 0 : 1;
    ib += take_b ? 1 : 0;  // ib <= nb: b is taken only while ib < nb
    // the next key of the side just taken (one past its end when exhausted)
    const T v = s[spad(take_b ? b0 + ib : min(a0 + ia, end))];
    vb = take_b ? v : vb;
    va = take_b ? va : v;
  }
}

// Store the ITEMS keys of v to dst[0..count): 16-byte vector stores when the
// whole run is there and dst is 16-byte aligned.
template <class T, int ITEMS>
__device__ __forceinline__ void store_run(T *dst, const T (&v)[ITEMS], int count) {
  constexpr int kBytes = (int)sizeof(T) * ITEMS;
  if constexpr (kBytes % 16 == 0) {
    if (count == ITEMS && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
      uint4 w[kBytes / 16];
      memcpy(w, v, kBytes);
#pragma unroll
      for (int j = 0; j < kBytes / 16; ++j) reinterpret_cast<uint4 *>(dst)[j] = w[j];
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < ITEMS; ++k)
    if (k < count) dst[k] = v[k];
}

// Where each tile starts on its merge path, for the pairwise merge of runs
// of length `run` (PAIRS; a == b == src, na = n, nb = 0) or the one merge
// of a[0..na) and b[0..nb): one warp per tile, splits[t] = the number of
// keys of the tile's first range (A) before the tile's first output.  All
// searches run at once, so the merge kernel starts loading at once.
template <class T>
struct PairView {
  const T *A, *B;
  long long nA, nB, base;
};

template <class T, bool PAIRS>
__device__ __forceinline__ PairView<T> pair_of(const T *a, long long na, const T *b, long long nb, long long run,
                                               long long d0) {
  PairView<T> v{a, b, na, nb, 0};
  if constexpr (PAIRS) {
    v.base = d0 / (2 * run) * (2 * run);
    v.A = a + v.base;
    v.nA = min(run, na - v.base);
    v.B = a + v.base + v.nA;
    v.nB = min(run, na - v.base - v.nA);
  }
  return v;
}

template <class T, class Comp, bool PAIRS>
__global__ void __launch_bounds__(256) merge_partition_kernel(const T *a, long long na, const T *b, long long nb,
                                                              long long run, long long ntiles, long long *splits,
                                                              Comp comp) {
  constexpr int kMergeTile = merge_tile<T>();
  const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= ntiles) return;  // whole warps leave together
  const PairView<T> v = pair_of<T, PAIRS>(a, na, b, nb, run, t * kMergeTile);
  const T *A = v.A, *B = v.B;
  auto ga = [&](long long i) { return A[i]; };
  auto gb = [&](long long i) { return B[i]; };
  const long long sp = merge_path_warp<T>(ga, v.nA, gb, v.nB, t * kMergeTile - v.base, comp);
  if ((threadIdx.x & 31) == 0) splits[t] = sp;
}

// Merge tile `blockIdx.x` of the pairwise merge of runs of length `run`
// (PAIRS) or of the one merge of a and b, from the tile starts in `splits`
// (merge_partition_kernel).  The tile ends where the next tile starts, or,
// for the last tile of its pair, at the end of both ranges.
template <class T, class Comp, bool PAIRS>
__global__ void __launch_bounds__(kMergeThreads) merge_kernel(const T *a, long long na, const T *b, long long nb,
                                                              T *out, long long run, const long long *splits,
                                                              Comp comp) {
  constexpr int kMergeItems = merge_items<T>(), kMergeTile = merge_tile<T>();
  __shared__ T s_in[spad_alloc(kMergeTile)];
  const long long total = PAIRS ? na : na + nb;
  const long long d0 = (long long)blockIdx.x * kMergeTile;
  if (d0 >= total) return;
  const PairView<T> v = pair_of<T, PAIRS>(a, na, b, nb, run, d0);
  const T *A = v.A, *B = v.B;
  const long long tile_end = min(d0 + kMergeTile, total);
  const long long l1 = tile_end - v.base;
  const long long i0 = splits[blockIdx.x];
  const long long i1 = l1 == v.nA + v.nB ? v.nA : splits[blockIdx.x + 1];
  const long long j0 = (d0 - v.base) - i0, j1 = l1 - i1;
  const int na_t = (int)(i1 - i0), nb_t = (int)(j1 - j0);
  const int cnt = na_t + nb_t;
  if (cnt == kMergeTile) {
    // a full tile: every thread's ITEMS loads in flight at once
    const T *pa = A + i0, *pb = B + (j0 - na_t);
    T r[kMergeItems];
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) {
      const int k = threadIdx.x + q * kMergeThreads;
      r[q] = (k < na_t ? pa : pb)[k];
    }
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) s_in[spad(threadIdx.x + q * kMergeThreads)] = r[q];
  } else {
    for (int k = threadIdx.x; k < cnt; k += kMergeThreads)
      s_in[spad(k)] = k < na_t ? A[i0 + k] : B[j0 + (k - na_t)];
  }
  __syncthreads();
  const int dt = min((int)threadIdx.x * kMergeItems, cnt);
  auto sa = [&](long long i) { return s_in[spad((int)i)]; };
  auto sb = [&](long long i) { return s_in[spad(na_t + (int)i)]; };
  const int it = (int)merge_path<T>(sa, na_t, sb, nb_t, dt, comp);
  T v_[kMergeItems];
  merge_serial(s_in, 0, it, na_t, na_t, dt - it, nb_t, v_, comp);
  // each thread's outputs are contiguous: straight from registers
  store_run(out + d0 + dt, v_, min(kMergeItems, cnt - dt));
}

// Sort tile `blockIdx.x` of keys[0..n) in place (stable).
template <class T, class Comp>
__global__ void __launch_bounds__(kMergeThreads) block_sort_kernel(T *keys, long long n, Comp comp) {
  constexpr int kMergeItems = merge_items<T>(), kMergeTile = merge_tile<T>();
  __shared__ T s_a[spad_alloc(kMergeTile)];
  __shared__ T s_b[spad_alloc(kMergeTile)];
  const long long t0 = (long long)blockIdx.x * kMergeTile;
  const int cnt = (int)min((long long)kMergeTile, n - t0);
  if (cnt == kMergeTile) {
    T r[kMergeItems];
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) r[q] = keys[t0 + threadIdx.x + q * kMergeThreads];
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) s_a[spad(threadIdx.x + q * kMergeThreads)] = r[q];
  } else {
    for (int k = threadIdx.x; k < cnt; k += kMergeThreads) s_a[spad(k)] = keys[t0 + k];
  }
  __syncthreads();
  // each thread: its ITEMS keys, sorted by odd-even transposition (stable:
  // neighbours swap only when the right one is strictly before the left)
  const int b0 = threadIdx.x * kMergeItems;
  const int mine = max(0, min(kMergeItems, cnt - b0));
  T v[kMergeItems];
#pragma unroll
  for (int k = 0; k < kMergeItems; ++k)
    if (k < mine) v[k] = s_a[spad(b0 + k)];
#pragma unroll
  for (int r = 0; r < kMergeItems; ++r) {
#pragma unroll
    for (int k = r & 1; k + 1 < kMergeItems; k += 2) {
      if (k + 1 < mine && comp(v[k + 1], v[k])) {
        const T x = v[k];
        v[k] = v[k + 1];
        v[k + 1] = x;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kMergeItems; ++k)
    if (k < mine) s_a[spad(b0 + k)] = v[k];
  __syncthreads();
  // rounds: runs of ITEMS, 2 ITEMS, ... merged pairwise in shared memory
  T *src = s_a, *dst = s_b;
  for (int run = kMergeItems; run < cnt; run *= 2) {
    const int d = b0;  // this thread's outputs [d, d + ITEMS)
    const bool last = 2 * run >= cnt;  // the same for the whole block
    if (d < cnt) {
      const int pb = d / (2 * run) * (2 * run);
      const int la = min(run, cnt - pb), lb = max(0, min(run, cnt - pb - la));
      auto sa = [&](long long i) { return src[spad(pb + (int)i)]; };
      auto sb = [&](long long i) { return src[spad(pb + la + (int)i)]; };
      const int dl = d - pb;
      const int ia = (int)merge_path<T>(sa, la, sb, lb, dl, comp);
      T w[kMergeItems];
      merge_serial(src, pb, ia, la, pb + la, dl - ia, lb, w, comp);
      if (last) {  // the sorted tile leaves from registers
        store_run(keys + t0 + d, w, min(kMergeItems, cnt - d));
      } else {
#pragma unroll
        for (int k = 0; k < kMergeItems; ++k)
          if (d + k < cnt) dst[spad(d + k)] = w[k];
      }
    }
    if (last) return;
    __syncthreads();
    T *x = src;
    src = dst;
    dst = x;
  }
  // no merge round (cnt <= ITEMS): the first thread's sorted keys
  for (int k = threadIdx.x; k < cnt; k += kMergeThreads) keys[t0 + k] = src[spad(k)];
}

// ------------------------------------------------------------------ host

// Scratch of a merge of `total` keys: the tile starts.
template <class T>
inline size_t merge_scratch_bytes(size_t total) {
  return ((total + merge_tile<T>() - 1) / merge_tile<T>() + 1) * sizeof(long long) + 256;
}

// Stable merge of a[0..na) and b[0..nb) into out (asynchronous on st);
// scratch: merge_scratch_bytes<T>(na + nb) bytes of device memory.
template <class T, class Comp>
int launch_merge(const T *a, size_t na, const T *b, size_t nb, T *out, const Comp &comp, void *scratch,
                 size_t scratch_bytes, cudaStream_t st) {
  const long long total = (long long)(na + nb);
  if (total == 0) return B2P_OK;
  const long long tiles = (total + merge_tile<T>() - 1) / merge_tile<T>();
  if (tiles > 0x7fffffffLL / 32) return B2P_ERR_INVALID_ARG;
  if (!scratch || scratch_bytes < merge_scratch_bytes<T>((size_t)total) - 256) return B2P_ERR_SCRATCH;
  long long *splits = reinterpret_cast<long long *>(scratch);
  merge_partition_kernel<T, Comp, false><<<(unsigned)((tiles * 32 + 255) / 256), 256, 0, st>>>(
      a, (long long)na, b, (long long)nb, total, tiles, splits, comp);
  merge_kernel<T, Comp, false><<<(unsigned)tiles, kMergeThreads, 0, st>>>(a, (long long)na, b, (long long)nb, out,
                                                                          total, splits, comp);
  return cudaGetLastError() == cudaSuccess ? B2P_OK : B2P_ERR_CUDA;
}

// Scratch a sort of n keys of T needs: a second array of n keys, then the
// tile starts of the merge passes.
template <class T>
inline size_t sort_keys_bytes(size_t n) {
  return (n * sizeof(T) + 255) / 256 * 256;
}
template <class T>
inline size_t sort_scratch_bytes(size_t n) {
  return sort_keys_bytes<T>(n) + merge_scratch_bytes<T>(n);
}

// Stable merge sort of keys[0..n) in place; scratch: sort_scratch_bytes<T>(n)
// bytes of device memory (none when n fits one tile).
template <class T, class Comp>
int launch_sort(T *keys, size_t n, const Comp &comp, void *scratch, size_t scratch_bytes, cudaStream_t st) {
  if (n <= 1) return B2P_OK;
  constexpr long long kMergeTile = merge_tile<T>();
  const long long tiles = ((long long)n + kMergeTile - 1) / kMergeTile;
  if (tiles > 0x7fffffffLL / 32) return B2P_ERR_INVALID_ARG;
  if (tiles > 1 && (!scratch || scratch_bytes < sort_scratch_bytes<T>(n) - 256)) return B2P_ERR_SCRATCH;
  block_sort_kernel<T, Comp><<<(unsigned)tiles, kMergeThreads, 0, st>>>(keys, (long long)n, comp);
  if (tiles == 1) return cudaGetLastError() == cudaSuccess ? B2P_OK : B2P_ERR_CUDA;
  T *src = keys, *dst = reinterpret_cast<T *>(scratch);
  long long *splits = reinterpret_cast<long long *>(reinterpret_cast<char *>(scratch) + sort_keys_bytes<T>(n));
  for (long long run = kMergeTile; run < (long long)n; run *= 2) {
    merge_partition_kernel<T, Comp, true><<<(unsigned)((tiles * 32 + 255) / 256), 256, 0, st>>>(
        src, (long long)n, src, 0, run, tiles, splits, comp);
    merge_kernel<T, Comp, true><<<(unsigned)tiles, kMergeThreads, 0, st>>>(src, (long long)n, src, 0, dst, run,
                                                                          splits, comp);
    T *x = src;
    src = dst;
    dst = x;
  }
  if (src != keys && cudaMemcpyAsync(keys, src, n * sizeof(T), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return B2P_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? B2P_OK : B2P_ERR_CUDA;
}

}  // namespace b2p
