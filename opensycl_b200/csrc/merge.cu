// b2p_merge / b2p_sort for the standard key types, ascending (std::less) or
// descending (std::greater): the merge-path merge of b2p_device/merge.cuh,
// and a sort that is the LSD radix sort of b2p_device/radix.cuh from
// kRadixMinKeys keys on (below 2^31 keys), the merge sort otherwise.
#include "b2p_device/merge.cuh"
#include "b2p_device/radix.cuh"
#include "internal.h"

namespace b2p {

namespace {

template <class T>
struct Less {
  __device__ __forceinline__ bool operator()(const T &x, const T &y) const { return x < y; }
};
template <class T>
struct Greater {
  __device__ __forceinline__ bool operator()(const T &x, const T &y) const { return y < x; }
};

template <class T>
int merge_t(const void *a, size_t na, const void *b, size_t nb, void *out, bool desc, void *scratch, size_t sb,
            cudaStream_t st) {
  const T *pa = reinterpret_cast<const T *>(a), *pb = reinterpret_cast<const T *>(b);
  T *po = reinterpret_cast<T *>(out);
  return desc ? launch_merge(pa, na, pb, nb, po, Greater<T>{}, scratch, sb, st)
              : launch_merge(pa, na, pb, nb, po, Less<T>{}, scratch, sb, st);
}

// Below this many keys one or a few merge-sort launches beat the radix
// sort's histogram and digit passes.
constexpr size_t kRadixMinKeys = (size_t)1 << 15;

template <class T>
bool use_radix(size_t n) {
  return n >= kRadixMinKeys && n < kRadixMaxKeys;
}

template <class T>
size_t scratch_t(int prim, size_t n) {
  if (prim != B2P_PRIM_SORT) return merge_scratch_bytes<T>(n);
  // the radix sort's need, or the merge sort's, whichever is larger (a
  // radix sort the device cannot run falls back to the merge sort)
  return use_radix<T>(n) ? std::max(radix_scratch_bytes<T>(n), sort_scratch_bytes<T>(n)) : sort_scratch_bytes<T>(n);
}

template <class T>
int sort_t(void *keys, size_t n, bool desc, void *scratch, size_t sb, cudaStream_t st) {
  T *k = reinterpret_cast<T *>(keys);
  if (use_radix<T>(n)) {
    const int rc = launch_radix_sort(k, n, desc, scratch, sb, device_info().sm_count, st);
    if (rc != B2P_ERR_UNSUPPORTED) return rc;  // (a device of more than 256 SMs: the merge sort)
  }
  return desc ? launch_sort(k, n, Greater<T>{}, scratch, sb, st) : launch_sort(k, n, Less<T>{}, scratch, sb, st);
}

bool sortable(int dtype) { return dtype >= B2P_I32 && dtype <= B2P_F64 && dtype != B2P_BF16; }

}  // namespace

size_t merge_sort_scratch_bytes(int prim, int dtype, size_t n) {
  switch (dtype) {
  case B2P_I32: return scratch_t<int32_t>(prim, n);
  case B2P_I64: return scratch_t<long long>(prim, n);
  case B2P_U32: return scratch_t<uint32_t>(prim, n);
  case B2P_U64: return scratch_t<unsigned long long>(prim, n);
  case B2P_F32: return scratch_t<float>(prim, n);
  case B2P_F64: return scratch_t<double>(prim, n);
  default: return 0;
  }
}

}  // namespace b2p

using namespace b2p;

static int merge_entry(int dtype, const void *a, size_t na, const void *b, size_t nb, void *out, int descending,
                       void *scratch, size_t scratch_bytes, b2p_stream stream) {
  if (!sortable(dtype)) return dtype == B2P_BF16 ? B2P_ERR_UNSUPPORTED : B2P_ERR_INVALID_ARG;
  if (na + nb == 0) return B2P_OK;
  const size_t es = dtype_size(dtype);
  int rc;
  if ((na && (rc = check_pointer(a, es))) || (nb && (rc = check_pointer(b, es))) || (rc = check_pointer(out, es)))
    return rc;
  if ((rc = check_extent(a, na * es)) || (rc = check_extent(b, nb * es)) || (rc = check_extent(out, (na + nb) * es)))
    return rc;
  if (!scratch || scratch_bytes + 256 < merge_sort_scratch_bytes(B2P_PRIM_MERGE, dtype, na + nb) ||
      check_pointer(scratch, 8))
    return B2P_ERR_SCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  const bool d = descending != 0;
  void *s = scratch;
  const size_t sb = scratch_bytes;
  switch (dtype) {
  case B2P_I32: return merge_t<int32_t>(a, na, b, nb, out, d, s, sb, st);
  case B2P_I64: return merge_t<long long>(a, na, b, nb, out, d, s, sb, st);
  case B2P_U32: return merge_t<uint32_t>(a, na, b, nb, out, d, s, sb, st);
  case B2P_U64: return merge_t<unsigned long long>(a, na, b, nb, out, d, s, sb, st);
  case B2P_F32: return merge_t<float>(a, na, b, nb, out, d, s, sb, st);
  default: return merge_t<double>(a, na, b, nb, out, d, s, sb, st);
  }
}

static int sort_entry(int dtype, void *keys, size_t n, int descending, void *scratch, size_t scratch_bytes,
                      b2p_stream stream) {
  if (!sortable(dtype)) return dtype == B2P_BF16 ? B2P_ERR_UNSUPPORTED : B2P_ERR_INVALID_ARG;
  if (n <= 1) return B2P_OK;
  const size_t es = dtype_size(dtype);
  int rc = check_pointer(keys, es);
  if (rc) return rc;
  if ((rc = check_extent(keys, n * es))) return rc;
  if (n > (size_t)merge_tile<long long>()) {
    if (!scratch || scratch_bytes + 256 < merge_sort_scratch_bytes(B2P_PRIM_SORT, dtype, n)) return B2P_ERR_SCRATCH;
    if ((rc = check_pointer(scratch, 256))) return B2P_ERR_SCRATCH;
  }
  cudaStream_t st = (cudaStream_t)stream;
  switch (dtype) {
  case B2P_I32: return sort_t<int32_t>(keys, n, descending, scratch, scratch_bytes, st);
  case B2P_I64: return sort_t<long long>(keys, n, descending, scratch, scratch_bytes, st);
  case B2P_U32: return sort_t<uint32_t>(keys, n, descending, scratch, scratch_bytes, st);
  case B2P_U64: return sort_t<unsigned long long>(keys, n, descending, scratch, scratch_bytes, st);
  case B2P_F32: return sort_t<float>(keys, n, descending, scratch, scratch_bytes, st);
  default: return sort_t<double>(keys, n, descending, scratch, scratch_bytes, st);
  }
}

extern "C" int b2p_merge(int dtype, const void *a, size_t na, const void *b, size_t nb, void *out, int descending,
                         void *scratch, size_t scratch_bytes, b2p_stream stream) {
  CallScope cs("b2p_merge", dtype, na + nb, 0, 2.0 * (double)(na + nb) * dtype_size(dtype), stream);
  return cs.done(merge_entry(dtype, a, na, b, nb, out, descending, scratch, scratch_bytes, stream));
}

extern "C" int b2p_sort(int dtype, void *keys, size_t n, int descending, void *scratch, size_t scratch_bytes,
                        b2p_stream stream) {
  CallScope cs("b2p_sort", dtype, n, 0, 2.0 * (double)n * dtype_size(dtype), stream);
  return cs.done(sort_entry(dtype, keys, n, descending, scratch, scratch_bytes, stream));
}
