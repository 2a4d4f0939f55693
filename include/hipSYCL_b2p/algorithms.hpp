// Drop-in for AdaptiveCpp's algorithms library on the data-parallel
// primitive path: hipsycl::algorithms::{reduce, transform_reduce,
// inclusive_scan, exclusive_scan, transform_inclusive_scan,
// transform_exclusive_scan, copy_if, any_of, all_of, none_of, sort, merge} and
// util::{allocation_cache,
// allocation_group}, with the reference's signatures
// (algorithms/numeric.hpp:170-327, algorithms/algorithm.hpp:178-243,
// algorithms/util/allocation_cache.hpp:42-181) and semantics:
//
//  * every call is asynchronous on the queue and returns a sycl::event;
//    `deps` are honoured (the queue's stream waits for them);
//  * first == last returns a completed default event at once, even when
//    deps are pending, and leaves *out untouched (numeric.hpp:163-169);
//  * scratch memory comes from the caller's allocation_group and returns to
//    its cache when the group is released.
//
// Dispatch.  Contiguous device-accessible ranges of int32/int64/uint32/
// uint64/float/double with a standard operator (plus, multiplies, minimum,
// maximum, bit_and/or/xor from std:: or sycl::), no transform, go to the
// libb2p kernels through the C-ABI (b2p_reduce, b2p_dot, b2p_scan,
// b2p_copy_if with a mask_compare predicate).  Everything else (user
// operators and transforms, other types, non-pointer iterators) runs
// header-only generic kernels compiled into the caller: tile reduce, scan of
// the tile totals, tile scan / compaction -- correct for any associative
// operator, without the libb2p tuning.
#pragma once

#include "sycl.hpp"
#include "../b2p_device/copy_if.cuh"
#include "../b2p_device/merge.cuh"

#include <algorithm>
#include <functional>
#include <iterator>
#include <mutex>
#include <optional>

namespace hipsycl {
namespace algorithms {
namespace util {

enum class allocation_type { device, shared, host };

class allocation_group;

// Best-fit reuse of scratch allocations, thread-safe
// (allocation_cache.hpp:42-121).
class allocation_cache {
 public:
  explicit allocation_cache(allocation_type t) : type_(t) {}
  allocation_cache(const allocation_cache &) = delete;
  allocation_cache &operator=(const allocation_cache &) = delete;
  ~allocation_cache() { purge(); }

  void purge() {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto &a : list_) {
      b2p_sycl::detail::device_guard g(a.dev);
      if (type_ == allocation_type::host) cudaFreeHost(a.ptr);
      else cudaFree(a.ptr);
    }
    cudaGetLastError();
    list_.clear();
  }
  allocation_type get_type() const { return type_; }

 private:
  friend class allocation_group;
  struct allocation {
    void *ptr = nullptr;
    size_t size = 0;
    int dev = 0;
    bool scratch_ready = false;  // zero-filled and used only as libb2p scratch since
  };

  allocation find_or_alloc(size_t size, size_t align, int dev) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      long best = -1;
      for (size_t i = 0; i < list_.size(); ++i) {
        const auto &a = list_[i];
        if (a.dev == dev && a.size >= size && reinterpret_cast<uintptr_t>(a.ptr) % align == 0 &&
            (best < 0 || a.size < list_[best].size))
          best = (long)i;
      }
      if (best >= 0) {
        allocation a = list_[best];
        list_.erase(list_.begin() + best);
        return a;
      }
    }
    allocation a;
    a.dev = dev;
    a.size = std::max<size_t>(size, 256);
    b2p_sycl::detail::device_guard g(dev);
    cudaError_t e;
    if (type_ == allocation_type::device) e = cudaMalloc(&a.ptr, a.size);
    else if (type_ == allocation_type::shared) e = cudaMallocManaged(&a.ptr, a.size);
    else e = cudaMallocHost(&a.ptr, a.size);
    b2p_sycl::detail::check_cuda(e, "allocation_cache: allocation");
    return a;
  }
  void give_back(const allocation &a) {
    std::lock_guard<std::mutex> lk(mu_);
    list_.push_back(a);
  }

  allocation_type type_;
  std::vector<allocation> list_;
  std::mutex mu_;
};

// Allocations that belong to one operation; returned to the cache on
// release/destruction.  Not thread-safe (allocation_cache.hpp:123-181).
class allocation_group {
 public:
  allocation_group() = default;
  allocation_group(allocation_cache *parent, const b2p_sycl::device &dev)
      : parent_(parent), dev_(dev.cuda_ordinal()) {}
  allocation_group(allocation_cache *parent, int cuda_ordinal) : parent_(parent), dev_(cuda_ordinal) {}
  allocation_group(const allocation_group &) = delete;
  allocation_group &operator=(const allocation_group &) = delete;
  ~allocation_group() { release(); }

  void release() {
    for (const auto &a : managed_) parent_->give_back(a);
    managed_.clear();
  }

  template <class T>
  T *obtain(size_t count) {
    auto a = parent_->find_or_alloc(count * sizeof(T), alignof(T) < 256 ? 256 : alignof(T), dev_);
    a.scratch_ready = false;  // the caller may write anything here
    managed_.push_back(a);
    return static_cast<T *>(a.ptr);
  }

  // libb2p scratch: zero-filled on first use (and after any other use of the
  // memory); later uses keep the epoch-tagged contents.
  void *obtain_scratch(size_t bytes, cudaStream_t s) {
    auto a = parent_->find_or_alloc(bytes, 256, dev_);
    if (!a.scratch_ready) {
      b2p_sycl::detail::check_b2p(b2p_scratch_init(a.ptr, a.size, (b2p_stream)s), "b2p_scratch_init");
      a.scratch_ready = true;
    }
    managed_.push_back(a);
    return a.ptr;
  }

  int get_device() const { return dev_; }

 private:
  allocation_cache *parent_ = nullptr;
  int dev_ = 0;
  std::vector<allocation_cache::allocation> managed_;
};

}  // namespace util

// Predicate with a libb2p fast path in copy_if: (bits(x) & mask) CMP rhs.
template <class T>
struct mask_compare {
  unsigned long long mask, rhs;
  int cmp;  // b2p_cmp
  B2P_HD bool operator()(const T &x) const {
    unsigned long long u = 0;
    memcpy(&u, &x, sizeof(T));
    const unsigned long long a = u & mask;
    switch (cmp) {
      case B2P_CMP_LT: return a < rhs;
      case B2P_CMP_LE: return a <= rhs;
      case B2P_CMP_EQ: return a == rhs;
      case B2P_CMP_NE: return a != rhs;
      case B2P_CMP_GE: return a >= rhs;
      default: return a > rhs;
    }
  }
};

namespace detail {

namespace bs = ::b2p_sycl;

template <class T>
constexpr int dtype_code() {
  if constexpr (std::is_same_v<T, float>) return B2P_F32;
  else if constexpr (std::is_same_v<T, double>) return B2P_F64;
  else if constexpr (std::is_integral_v<T> && !std::is_same_v<T, bool> && sizeof(T) == 4)
    return std::is_signed_v<T> ? B2P_I32 : B2P_U32;
  else if constexpr (std::is_integral_v<T> && sizeof(T) == 8) return std::is_signed_v<T> ? B2P_I64 : B2P_U64;
  else return -1;
}

template <class Op, template <class> class F>
struct is_fn : std::false_type {};
template <class U, template <class> class F>
struct is_fn<F<U>, F> : std::true_type {};

template <class Op, class T>
constexpr int op_code() {
  constexpr bool is_int = std::is_integral_v<T>;
  if constexpr (is_fn<Op, std::plus>::value || is_fn<Op, bs::plus>::value) return B2P_SUM;
  else if constexpr (is_fn<Op, std::multiplies>::value || is_fn<Op, bs::multiplies>::value) return B2P_PROD;
  else if constexpr (is_fn<Op, bs::minimum>::value) return B2P_MIN;
  else if constexpr (is_fn<Op, bs::maximum>::value) return B2P_MAX;
  else if constexpr (is_int && (is_fn<Op, std::bit_and>::value || is_fn<Op, bs::bit_and>::value)) return B2P_AND;
  else if constexpr (is_int && (is_fn<Op, std::bit_or>::value || is_fn<Op, bs::bit_or>::value)) return B2P_OR;
  else if constexpr (is_int && (is_fn<Op, std::bit_xor>::value || is_fn<Op, bs::bit_xor>::value)) return B2P_XOR;
  else return -1;
}

// The reference's reductions start every work-item from the operator's
// identity, and its identity table gives sycl::maximum<T> the value
// numeric_limits<T>::min() and sycl::minimum<T> numeric_limits<T>::max()
// (algorithms/numeric.hpp:35-53).  For floating T that is the smallest
// positive normal / the largest finite value, so a maximum over negative
// floats returns numeric_limits<T>::min().  Folding that value into init
// reproduces the reference's results exactly.
template <class Op, class T>
T reference_init(T init) {
  if constexpr (std::is_floating_point_v<T> && std::is_same_v<Op, bs::maximum<T>>)
    return init < std::numeric_limits<T>::min() ? std::numeric_limits<T>::min() : init;
  else if constexpr (std::is_floating_point_v<T> && std::is_same_v<Op, bs::minimum<T>>)
    return std::numeric_limits<T>::max() < init ? std::numeric_limits<T>::max() : init;
  else
    return init;
}

struct identity_fn {
  template <class X>
  B2P_HD X operator()(const X &x) const {
    return x;
  }
};

template <class It>
constexpr bool is_ptr = std::is_pointer_v<It>;

template <class It>
using value_t = typename std::iterator_traits<It>::value_type;

// ---------------------------------------------------------- generic kernels

constexpr int kGB = 256;   // threads per block
constexpr int kGI = 8;     // items per thread
constexpr int kGT = kGB * kGI;

// (value, present) pairs: an operator without identity skips absent values.
template <class T>
struct opt {
  T v;
  bool h;
};
template <class T, class Op>
B2P_HD opt<T> combine(const opt<T> &a, const opt<T> &b, const Op &op) {
  if (!a.h) return b;
  if (!b.h) return a;
  return {op(a.v, b.v), true};
}

// Block inclusive scan of opt<T> (Hillis-Steele in shared memory).
template <class T, class Op>
__device__ opt<T> block_scan_opt(opt<T> x, const Op &op, opt<T> *total) {
  __shared__ T sv[kGB];
  __shared__ bool sh[kGB];
  sv[threadIdx.x] = x.v;
  sh[threadIdx.x] = x.h;
  __syncthreads();
  for (int d = 1; d < kGB; d <<= 1) {
    opt<T> cur{sv[threadIdx.x], sh[threadIdx.x]};
    if ((int)threadIdx.x >= d) cur = combine(opt<T>{sv[threadIdx.x - d], sh[threadIdx.x - d]}, cur, op);
    __syncthreads();
    sv[threadIdx.x] = cur.v;
    sh[threadIdx.x] = cur.h;
    __syncthreads();
  }
  opt<T> r{sv[threadIdx.x], sh[threadIdx.x]};
  *total = opt<T>{sv[kGB - 1], sh[kGB - 1]};
  __syncthreads();
  return r;
}

// Element generator: gen(i) = transform(first[i]) or transform(a[i], b[i]).
template <class T, class It, class Tr>
struct unary_gen {
  It first;
  Tr tr;
  __device__ T operator()(size_t i) const { return static_cast<T>(tr(*(first + i))); }
};
template <class T, class It1, class It2, class Tr>
struct binary_gen {
  It1 a;
  It2 b;
  Tr tr;
  __device__ T operator()(size_t i) const { return static_cast<T>(tr(*(a + i), *(b + i))); }
};

// Units of the library reduce kernel for user transforms: value(i) =
// transform(first[i]) or transform(a[i], b[i]), converted to T.
template <class T, class It, class Tr>
struct unary_source : ::b2p::ValueSource<unary_source<T, It, Tr>, T> {
  It first;
  Tr tr;
  unary_source(It f, Tr t) : first(f), tr(t) {}
  __device__ __forceinline__ T value(long long i) const { return static_cast<T>(tr(*(first + i))); }
};
template <class T, class It1, class It2, class Tr>
struct binary_source : ::b2p::ValueSource<binary_source<T, It1, It2, Tr>, T> {
  It1 a;
  It2 b;
  Tr tr;
  binary_source(It1 a_, It2 b_, Tr t) : a(a_), b(b_), tr(t) {}
  __device__ __forceinline__ T value(long long i) const { return static_cast<T>(tr(*(a + i), *(b + i))); }
};

// Tile totals (one tile of kGT elements per block).
template <class T, class Gen, class Op>
__global__ void __launch_bounds__(kGB) tile_reduce_kernel(size_t n, Gen gen, Op op, T *tot_v, bool *tot_h) {
  const size_t base = (size_t)blockIdx.x * kGT + (size_t)threadIdx.x * kGI;
  opt<T> acc{T{}, false};
  for (int k = 0; k < kGI; ++k)
    if (base + k < n) acc = combine(acc, opt<T>{gen(base + k), true}, op);
  opt<T> total;
  (void)block_scan_opt(acc, op, &total);
  if (threadIdx.x == 0) {
    tot_v[blockIdx.x] = total.v;
    tot_h[blockIdx.x] = total.h;
  }
}

// One block: exclusive prefixes of the tile totals, starting from `init`
// (when present), and the grand total.
template <class T, class Op>
__global__ void __launch_bounds__(kGB) totals_scan_kernel(size_t ntiles, Op op, T *v, bool *h, T init, bool has_init,
                                                           T *grand, bool *grand_h) {
  opt<T> carry{init, has_init};
  for (size_t b0 = 0; b0 < ntiles; b0 += kGB) {
    const size_t i = b0 + threadIdx.x;
    opt<T> x = i < ntiles ? opt<T>{v[i], h[i]} : opt<T>{T{}, false};
    opt<T> total;
    const opt<T> incl = block_scan_opt(x, op, &total);
    // exclusive = carry (+) inclusive of the previous thread
    __shared__ T pv[kGB];
    __shared__ bool ph[kGB];
    pv[threadIdx.x] = incl.v;
    ph[threadIdx.x] = incl.h;
    __syncthreads();
    opt<T> ex = carry;
    if (threadIdx.x > 0) ex = combine(carry, opt<T>{pv[threadIdx.x - 1], ph[threadIdx.x - 1]}, op);
    __syncthreads();
    if (i < ntiles) {
      v[i] = ex.v;
      h[i] = ex.h;
    }
    carry = combine(carry, total, op);
  }
  if (threadIdx.x == 0 && grand) {
    *grand = carry.v;
    *grand_h = carry.h;
  }
}

// Tile scan from its prefix; writes out[i] = prefix (+) x[0..i] (inclusive)
// or prefix (+) x[0..i) (exclusive; the first element gets the prefix).
template <class T, class Gen, class Op, class OutIt, bool INCL>
__global__ void __launch_bounds__(kGB) tile_scan_kernel(size_t n, Gen gen, Op op, const T *pre_v, const bool *pre_h,
                                                         OutIt out) {
  const size_t base = (size_t)blockIdx.x * kGT + (size_t)threadIdx.x * kGI;
  T x[kGI];
  opt<T> acc{T{}, false};
  for (int k = 0; k < kGI; ++k) {
    if (base + k < n) {
      x[k] = gen(base + k);
      acc = combine(acc, opt<T>{x[k], true}, op);
    }
  }
  opt<T> total;
  const opt<T> incl = block_scan_opt(acc, op, &total);
  __shared__ T pv[kGB];
  __shared__ bool ph[kGB];
  pv[threadIdx.x] = incl.v;
  ph[threadIdx.x] = incl.h;
  __syncthreads();
  opt<T> run{pre_v[blockIdx.x], pre_h[blockIdx.x]};
  if (threadIdx.x > 0) run = combine(run, opt<T>{pv[threadIdx.x - 1], ph[threadIdx.x - 1]}, op);
  for (int k = 0; k < kGI; ++k) {
    if (base + k < n) {
      if constexpr (INCL) {
        run = combine(run, opt<T>{x[k], true}, op);
        *(out + (base + k)) = run.v;
      } else {
        *(out + (base + k)) = run.v;
        run = combine(run, opt<T>{x[k], true}, op);
      }
    }
  }
}

template <class T, class Op>
__global__ void __launch_bounds__(1) write_result_kernel(const T *v, const bool *h, T *out, T init, Op op) {
  *out = h[0] ? op(init, v[0]) : init;
}

// copy_if: kept count per tile, then order-preserving writes.
template <class It, class Pred>
__global__ void __launch_bounds__(kGB) tile_count_kernel(size_t n, It first, Pred pred, unsigned long long *cnt) {
  const size_t base = (size_t)blockIdx.x * kGT + (size_t)threadIdx.x * kGI;
  unsigned c = 0;
  for (int k = 0; k < kGI; ++k)
    if (base + k < n && pred(*(first + (base + k)))) ++c;
  __shared__ unsigned s[kGB];
  s[threadIdx.x] = c;
  __syncthreads();
  for (int d = kGB / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d) s[threadIdx.x] += s[threadIdx.x + d];
    __syncthreads();
  }
  if (threadIdx.x == 0) cnt[blockIdx.x] = s[0];
}

// Exclusive scan of the tile counts in place by one block (chunks of kGB
// counts, a shuffle scan per warp), and the total into *num.
template <int = 0>
__global__ void __launch_bounds__(kGB) counts_scan_kernel(size_t ntiles, unsigned long long *cnt, size_t *num) {
  __shared__ unsigned long long s_warp[kGB / 32];
  __shared__ unsigned long long s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (size_t b0 = 0; b0 < ntiles; b0 += kGB) {
    const size_t i = b0 + threadIdx.x;
    const unsigned long long c = i < ntiles ? cnt[i] : 0ull;
    unsigned long long incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    unsigned long long before = s_carry;
    for (int w = 0; w < warp; ++w) before += s_warp[w];
    if (i < ntiles) cnt[i] = before + incl - c;
    __syncthreads();
    if (threadIdx.x == kGB - 1) s_carry = before + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0 && num) *num = (size_t)s_carry;
}

template <class It, class OutIt, class Pred>
__global__ void __launch_bounds__(kGB) tile_compact_kernel(size_t n, It first, Pred pred, const unsigned long long *off,
                                                            OutIt out) {
  const size_t base = (size_t)blockIdx.x * kGT + (size_t)threadIdx.x * kGI;
  bool keep[kGI];
  unsigned c = 0;
  for (int k = 0; k < kGI; ++k) {
    keep[k] = base + k < n && pred(*(first + (base + k)));
    c += keep[k];
  }
  __shared__ unsigned s[kGB];
  s[threadIdx.x] = c;
  __syncthreads();
  for (int d = 1; d < kGB; d <<= 1) {
    const unsigned v = (int)threadIdx.x >= d ? s[threadIdx.x - d] : 0u;
    __syncthreads();
    s[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned long long o = off[blockIdx.x] + s[threadIdx.x] - c;
  for (int k = 0; k < kGI; ++k)
    if (keep[k]) *(out + (o++)) = *(first + (base + k));
}

// Generic reduce of gen(0..n) into *out = op(init, r).
template <class T, class Gen, class Op>
bs::event generic_reduce(bs::queue &q, util::allocation_group &scratch, size_t n, Gen gen, T *out, T init, Op op) {
  const size_t ntiles = (n + kGT - 1) / kGT;
  T *v = scratch.obtain<T>(ntiles + 1);
  bool *h = scratch.obtain<bool>(ntiles + 1);
  bs::detail::device_guard g(q.get_device().cuda_ordinal());
  tile_reduce_kernel<T, Gen, Op><<<(unsigned)ntiles, kGB, 0, q.cuda_stream()>>>(n, gen, op, v, h);
  totals_scan_kernel<T, Op><<<1, kGB, 0, q.cuda_stream()>>>(ntiles, op, v, h, T{}, false, v + ntiles, h + ntiles);
  write_result_kernel<T, Op><<<1, 1, 0, q.cuda_stream()>>>(v + ntiles, h + ntiles, out, init, op);
  bs::detail::check_cuda(cudaGetLastError(), "generic reduce");
  return q.record();
}

template <bool INCL, class T, class Gen, class Op, class OutIt>
bs::event generic_scan(bs::queue &q, util::allocation_group &scratch, size_t n, Gen gen, OutIt out, Op op,
                       std::optional<T> init) {
  const size_t ntiles = (n + kGT - 1) / kGT;
  T *v = scratch.obtain<T>(ntiles);
  bool *h = scratch.obtain<bool>(ntiles);
  bs::detail::device_guard g(q.get_device().cuda_ordinal());
  tile_reduce_kernel<T, Gen, Op><<<(unsigned)ntiles, kGB, 0, q.cuda_stream()>>>(n, gen, op, v, h);
  totals_scan_kernel<T, Op><<<1, kGB, 0, q.cuda_stream()>>>(ntiles, op, v, h, init ? *init : T{}, init.has_value(),
                                                             nullptr, nullptr);
  tile_scan_kernel<T, Gen, Op, OutIt, INCL><<<(unsigned)ntiles, kGB, 0, q.cuda_stream()>>>(n, gen, op, v, h, out);
  bs::detail::check_cuda(cudaGetLastError(), "generic scan");
  return q.record();
}

// The library reduce kernel over a generated sequence (a user transform of
// contiguous device inputs, a standard operator on int32/uint32/int64/uint64/
// float/double): *out = op(init, r).
template <class T, class Op, class Src>
bs::event library_reduce(bs::queue &q, util::allocation_group &scratch, size_t n, const Src &src, T *out,
                         T init) {
  using P = bs::detail::library_policy<T, Op>;
  const size_t bytes = ::b2p::reduce_gen_scratch_bytes(n);
  void *s = scratch.obtain_scratch(bytes, q.cuda_stream());
  bs::detail::device_guard g(q.get_device().cuda_ordinal());
  bs::detail::check_b2p(::b2p::launch_reduce_gen<P>(src, n, out, &init, s, bytes, q.cuda_stream()), "transform_reduce");
  return q.record();
}

// Scratch + config of a libb2p call.
inline void *b2p_scratch(util::allocation_group &scratch, bs::queue &q, int prim, int dtype, size_t n) {
  const size_t bytes = b2p_scratch_bytes(prim, dtype, n, 0, B2P_CONFIG_AUTO);
  return scratch.obtain_scratch(bytes, q.cuda_stream());
}

template <class Ptr>
bool device_accessible(Ptr p);

// Pointer iterators handed to a generic kernel must be device-accessible:
// a pageable host pointer is rejected (no host fallback).
template <class It>
void require_device(It it, const char *what) {
  if constexpr (std::is_pointer_v<It>) {
    if (!device_accessible(it))
      throw b2p_sycl::exception(B2P_ERR_INVALID_PTR, std::string(what) + ": pointer is not device-accessible");
  }
}

template <class Ptr>
bool device_accessible(Ptr p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, (const void *)p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged ||
         (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr);
}

}  // namespace detail

// ------------------------------------------------------------ reductions

template <class ForwardIt1, class ForwardIt2, class T, class BinaryReductionOp, class BinaryTransformOp>
b2p_sycl::event transform_reduce(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt1 first1,
                                 ForwardIt1 last1, ForwardIt2 first2, T *out, T init, BinaryReductionOp reduce,
                                 BinaryTransformOp transform, const std::vector<b2p_sycl::event> &deps = {}) {
  if (first1 == last1) return b2p_sycl::event{};
  q.depends_on(deps);
  const size_t n = (size_t)std::distance(first1, last1);
  init = detail::reference_init<BinaryReductionOp>(init);
  constexpr int dt = detail::dtype_code<T>();
  if constexpr (detail::is_ptr<ForwardIt1> && detail::is_ptr<ForwardIt2> && (dt == B2P_F32 || dt == B2P_F64) &&
                std::is_same_v<detail::value_t<ForwardIt1>, T> && std::is_same_v<detail::value_t<ForwardIt2>, T> &&
                detail::op_code<BinaryReductionOp, T>() == B2P_SUM &&
                (detail::is_fn<BinaryTransformOp, std::multiplies>::value ||
                 detail::is_fn<BinaryTransformOp, b2p_sycl::multiplies>::value)) {
    if (detail::device_accessible(first1) && detail::device_accessible(first2)) {
      void *s = detail::b2p_scratch(scratch, q, B2P_PRIM_DOT, dt, n);
      b2p_sycl::detail::check_b2p(
          b2p_dot(dt, &*first1, &*first2, n, out, &init, s, b2p_scratch_bytes(B2P_PRIM_DOT, dt, n, 0, B2P_CONFIG_AUTO),
                  B2P_CONFIG_AUTO, (b2p_stream)q.cuda_stream()),
          "b2p_dot");
      return q.record();
    }
  }
  detail::require_device(first1, "transform_reduce");
  detail::require_device(first2, "transform_reduce");
  detail::require_device(out, "transform_reduce");
  if constexpr (b2p_sycl::detail::library_reduction<T, BinaryReductionOp>()) {
    detail::binary_source<T, ForwardIt1, ForwardIt2, BinaryTransformOp> src(first1, first2, transform);
    return detail::library_reduce<T, BinaryReductionOp>(q, scratch, n, src, out, init);
  }
  detail::binary_gen<T, ForwardIt1, ForwardIt2, BinaryTransformOp> gen{first1, first2, transform};
  return detail::generic_reduce(q, scratch, n, gen, out, init, reduce);
}

template <class ForwardIt, class T, class BinaryReductionOp, class UnaryTransformOp>
b2p_sycl::event transform_reduce(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt first,
                                 ForwardIt last, T *out, T init, BinaryReductionOp reduce,
                                 UnaryTransformOp transform, const std::vector<b2p_sycl::event> &deps = {}) {
  if (first == last) return b2p_sycl::event{};
  q.depends_on(deps);
  const size_t n = (size_t)std::distance(first, last);
  init = detail::reference_init<BinaryReductionOp>(init);
  constexpr int dt = detail::dtype_code<T>();
  constexpr int op = detail::op_code<BinaryReductionOp, T>();
  if constexpr (detail::is_ptr<ForwardIt> && dt >= 0 && op >= 0 &&
                std::is_same_v<std::remove_cv_t<detail::value_t<ForwardIt>>, T> &&
                std::is_same_v<UnaryTransformOp, detail::identity_fn>) {
    if (detail::device_accessible(first)) {
      void *s = detail::b2p_scratch(scratch, q, B2P_PRIM_REDUCE, dt, n);
      b2p_sycl::detail::check_b2p(
          b2p_reduce(dt, op, &*first, n, out, &init, s, b2p_scratch_bytes(B2P_PRIM_REDUCE, dt, n, 0, B2P_CONFIG_AUTO),
                     B2P_CONFIG_AUTO, (b2p_stream)q.cuda_stream()),
          "b2p_reduce");
      return q.record();
    }
  }
  detail::require_device(first, "transform_reduce");
  detail::require_device(out, "transform_reduce");
  if constexpr (b2p_sycl::detail::library_reduction<T, BinaryReductionOp>()) {
    detail::unary_source<T, ForwardIt, UnaryTransformOp> src(first, transform);
    return detail::library_reduce<T, BinaryReductionOp>(q, scratch, n, src, out, init);
  }
  detail::unary_gen<T, ForwardIt, UnaryTransformOp> gen{first, transform};
  return detail::generic_reduce(q, scratch, n, gen, out, init, reduce);
}

template <class ForwardIt1, class ForwardIt2, class T>
b2p_sycl::event transform_reduce(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt1 first1,
                                 ForwardIt1 last1, ForwardIt2 first2, T *out, T init,
                                 const std::vector<b2p_sycl::event> &deps = {}) {
  return transform_reduce(q, scratch, first1, last1, first2, out, init, std::plus<T>{}, std::multiplies<T>{}, deps);
}

template <class ForwardIt, class T, class BinaryOp>
b2p_sycl::event reduce(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt first, ForwardIt last, T *out,
                       T init, BinaryOp binary_op, const std::vector<b2p_sycl::event> &deps = {}) {
  return transform_reduce(q, scratch, first, last, out, init, binary_op, detail::identity_fn{}, deps);
}

template <class ForwardIt, class T>
b2p_sycl::event reduce(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt first, ForwardIt last, T *out,
                       T init, const std::vector<b2p_sycl::event> &deps = {}) {
  return reduce(q, scratch, first, last, out, init, std::plus<T>{}, deps);
}

template <class ForwardIt>
b2p_sycl::event reduce(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt first, ForwardIt last,
                       typename std::iterator_traits<ForwardIt>::value_type *out,
                       const std::vector<b2p_sycl::event> &deps = {}) {
  return reduce(q, scratch, first, last, out, typename std::iterator_traits<ForwardIt>::value_type{}, deps);
}

// ------------------------------------------------------------------ scans

namespace detail {

template <bool INCL, class InputIt, class OutputIt, class BinaryOp, class UnaryOp, class T>
b2p_sycl::event scan_impl(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first, InputIt last,
                          OutputIt d_first, UnaryOp unary_op, BinaryOp op, std::optional<T> init,
                          const std::vector<b2p_sycl::event> &deps) {
  if (first == last) return b2p_sycl::event{};
  q.depends_on(deps);
  const size_t n = (size_t)std::distance(first, last);
  constexpr int dt = dtype_code<T>();
  constexpr int opc = op_code<BinaryOp, T>();
  if constexpr (is_ptr<InputIt> && is_ptr<OutputIt> && dt >= 0 && opc >= 0 &&
                std::is_same_v<std::remove_cv_t<value_t<InputIt>>, T> && std::is_same_v<value_t<OutputIt>, T> &&
                std::is_same_v<UnaryOp, identity_fn>) {
    if (device_accessible(first) && device_accessible(d_first)) {
      void *s = b2p_scratch(scratch, q, B2P_PRIM_SCAN, dt, n);
      T iv = init ? *init : T{};
      b2p_sycl::detail::check_b2p(b2p_scan(dt, opc, INCL ? 1 : 0, &*first, &*d_first, n, init ? &iv : nullptr, s,
                                           b2p_scratch_bytes(B2P_PRIM_SCAN, dt, n, 0, B2P_CONFIG_AUTO),
                                           B2P_CONFIG_AUTO, (b2p_stream)q.cuda_stream()),
                                  "b2p_scan");
      return q.record();
    }
  }
  require_device(first, "scan");
  require_device(d_first, "scan");
  unary_gen<T, InputIt, UnaryOp> gen{first, unary_op};
  return generic_scan<INCL, T>(q, scratch, n, gen, d_first, op, init);
}

template <class InputIt, class OutputIt>
using scan_t = std::remove_cv_t<value_t<InputIt>>;

}  // namespace detail

template <class InputIt, class OutputIt, class BinaryOp>
b2p_sycl::event inclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first, InputIt last,
                               OutputIt d_first, BinaryOp op, const std::vector<b2p_sycl::event> &deps = {}) {
  using T = detail::scan_t<InputIt, OutputIt>;
  return detail::scan_impl<true>(q, scratch, first, last, d_first, detail::identity_fn{}, op, std::optional<T>{},
                                 deps);
}

template <class InputIt, class OutputIt, class BinaryOp, class T>
b2p_sycl::event inclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first, InputIt last,
                               OutputIt d_first, BinaryOp op, T init, const std::vector<b2p_sycl::event> &deps = {}) {
  return detail::scan_impl<true>(q, scratch, first, last, d_first, detail::identity_fn{}, op, std::optional<T>{init},
                                 deps);
}

template <class InputIt, class OutputIt>
b2p_sycl::event inclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first, InputIt last,
                               OutputIt d_first, const std::vector<b2p_sycl::event> &deps = {}) {
  using T = detail::scan_t<InputIt, OutputIt>;
  return inclusive_scan(q, scratch, first, last, d_first, std::plus<T>{}, deps);
}

template <class InputIt, class OutputIt, class T, class BinaryOp>
b2p_sycl::event exclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first, InputIt last,
                               OutputIt d_first, T init, BinaryOp op, const std::vector<b2p_sycl::event> &deps = {}) {
  return detail::scan_impl<false>(q, scratch, first, last, d_first, detail::identity_fn{}, op,
                                  std::optional<T>{init}, deps);
}

template <class InputIt, class OutputIt, class T>
b2p_sycl::event exclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first, InputIt last,
                               OutputIt d_first, T init, const std::vector<b2p_sycl::event> &deps = {}) {
  return exclusive_scan(q, scratch, first, last, d_first, init, std::plus<T>{}, deps);
}

template <class InputIt, class OutputIt, class BinaryOp, class UnaryOp>
b2p_sycl::event transform_inclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first,
                                         InputIt last, OutputIt d_first, BinaryOp binary_op, UnaryOp unary_op,
                                         const std::vector<b2p_sycl::event> &deps = {}) {
  using T = std::remove_cv_t<std::remove_reference_t<decltype(unary_op(*first))>>;
  return detail::scan_impl<true>(q, scratch, first, last, d_first, unary_op, binary_op, std::optional<T>{}, deps);
}

template <class InputIt, class OutputIt, class BinaryOp, class UnaryOp, class T>
b2p_sycl::event transform_inclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first,
                                         InputIt last, OutputIt d_first, BinaryOp binary_op, UnaryOp unary_op, T init,
                                         const std::vector<b2p_sycl::event> &deps = {}) {
  return detail::scan_impl<true>(q, scratch, first, last, d_first, unary_op, binary_op, std::optional<T>{init}, deps);
}

template <class InputIt, class OutputIt, class T, class BinaryOp, class UnaryOp>
b2p_sycl::event transform_exclusive_scan(b2p_sycl::queue &q, util::allocation_group &scratch, InputIt first,
                                         InputIt last, OutputIt d_first, T init, BinaryOp binary_op,
                                         UnaryOp unary_op, const std::vector<b2p_sycl::event> &deps = {}) {
  return detail::scan_impl<false>(q, scratch, first, last, d_first, unary_op, binary_op, std::optional<T>{init},
                                  deps);
}

// ---------------------------------------------------------------- copy_if

// *num_elements_copied (device-accessible) receives the number of kept
// elements; for first == last it is set to 0 on the host
// (algorithm.hpp:184-188).
template <class ForwardIt1, class ForwardIt2, class UnaryPredicate>
b2p_sycl::event copy_if(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt1 first, ForwardIt1 last,
                        ForwardIt2 d_first, UnaryPredicate pred, std::size_t *num_elements_copied = nullptr,
                        const std::vector<b2p_sycl::event> &deps = {}) {
  if (first == last) {
    if (num_elements_copied) *num_elements_copied = 0;
    return b2p_sycl::event{};
  }
  q.depends_on(deps);
  const size_t n = (size_t)std::distance(first, last);
  using V = std::remove_cv_t<detail::value_t<ForwardIt1>>;
  constexpr int dt = detail::dtype_code<V>();
  if constexpr (detail::is_ptr<ForwardIt1> && detail::is_ptr<ForwardIt2> && dt >= 0 &&
                std::is_same_v<UnaryPredicate, mask_compare<V>>) {
    if (detail::device_accessible(first) && detail::device_accessible(d_first) &&
        (!num_elements_copied || detail::device_accessible(num_elements_copied))) {
      void *s = detail::b2p_scratch(scratch, q, B2P_PRIM_COPY_IF, dt, n);
      b2p_sycl::detail::check_b2p(
          b2p_copy_if(dt, &*first, &*d_first, n, pred.mask, pred.cmp, pred.rhs,
                      reinterpret_cast<uint64_t *>(num_elements_copied), s,
                      b2p_scratch_bytes(B2P_PRIM_COPY_IF, dt, n, 0, B2P_CONFIG_AUTO), B2P_CONFIG_AUTO,
                      (b2p_stream)q.cuda_stream()),
          "b2p_copy_if");
      return q.record();
    }
  }
  detail::require_device(first, "copy_if");
  detail::require_device(d_first, "copy_if");
  if (num_elements_copied) detail::require_device(num_elements_copied, "copy_if count");
  // Any predicate on contiguous 4- or 8-byte elements: the library's
  // TMEM-staged copy_if kernel compiled with the predicate (16-byte aligned
  // input of at least one 8192-element tile; the generic kernels otherwise).
  if constexpr (detail::is_ptr<ForwardIt1> && detail::is_ptr<ForwardIt2> &&
                (sizeof(V) == 4 || sizeof(V) == 8) && std::is_trivially_copyable_v<V> &&
                std::is_same_v<std::remove_cv_t<detail::value_t<ForwardIt2>>, V>) {
    constexpr int items = sizeof(V) == 4 ? 32 : 16;
    if (n >= (size_t)256 * items && (reinterpret_cast<uintptr_t>(&*first) & 15) == 0) {
      const int pdt = sizeof(V) == 4 ? B2P_U32 : B2P_U64;
      const size_t bytes = b2p_scratch_bytes(B2P_PRIM_COPY_IF, pdt, n, 0, B2P_CONFIG_AUTO);
      void *s = scratch.obtain_scratch(bytes, q.cuda_stream());
      b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
      const int dev = q.get_device().cuda_ordinal();
      const int rc = ::b2p::launch_copy_if_pred<V>(
          &*first, &*d_first, n, pred, reinterpret_cast<unsigned long long *>(num_elements_copied), s, 256, items,
          ::b2p::device_sm_count(dev), b2p_wait_timeout_ns(), -1, q.cuda_stream());
      if (rc == B2P_OK) return q.record();
      if (rc != B2P_ERR_UNSUPPORTED) b2p_sycl::detail::check_b2p(rc, "copy_if");
    }
  }
  const size_t ntiles = (n + detail::kGT - 1) / detail::kGT;
  unsigned long long *cnt = scratch.obtain<unsigned long long>(ntiles);
  b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
  detail::tile_count_kernel<<<(unsigned)ntiles, detail::kGB, 0, q.cuda_stream()>>>(n, first, pred, cnt);
  detail::counts_scan_kernel<<<1, detail::kGB, 0, q.cuda_stream()>>>(ntiles, cnt, num_elements_copied);
  detail::tile_compact_kernel<<<(unsigned)ntiles, detail::kGB, 0, q.cuda_stream()>>>(n, first, pred, cnt, d_first);
  b2p_sycl::detail::check_cuda(cudaGetLastError(), "copy_if");
  return q.record();
}

// ----------------------------------------------- any_of / all_of / none_of
// (algorithm.hpp:422-516).  *out receives 1 or 0; for first == last nothing
// is launched and *out is left as it is, as in the reference.  The search
// stops early: a warp that finds a hit raises a flag in *out, and every warp
// looks at the flag before each stride of 8 elements per thread.

namespace detail {
using early_exit_flag_t = int;

constexpr int kEarlyUnroll = 8;

template <class It, class Pred>
__global__ void __launch_bounds__(kGB) early_exit_kernel(size_t n, It first, Pred pred, bool negate,
                                                           early_exit_flag_t *flag) {
  const size_t span = (size_t)kGB * kEarlyUnroll;
  for (size_t base = (size_t)blockIdx.x * span; base < n; base += (size_t)gridDim.x * span) {
    int stop = 0;
    if ((threadIdx.x & 31) == 0) stop = *reinterpret_cast<volatile early_exit_flag_t *>(flag);
    if (__shfl_sync(0xffffffffu, stop, 0)) return;
    bool hit = false;
#pragma unroll
    for (int k = 0; k < kEarlyUnroll; ++k) {
      const size_t j = base + (size_t)k * kGB + threadIdx.x;
      if (j < n) {
        const bool v = static_cast<bool>(pred(first[j]));
        hit |= negate ? !v : v;
      }
    }
    if (__any_sync(0xffffffffu, hit)) {
      if ((threadIdx.x & 31) == 0) atomicExch(flag, 1);
      return;
    }
  }
}

template <int = 0>
__global__ void flip_flag_kernel(early_exit_flag_t *flag) {
  *flag = !*flag;
}

// *out = 1 if some element satisfies pred (negate: fails it), else 0.
template <class It, class Pred>
b2p_sycl::event early_exit_search(b2p_sycl::queue &q, It first, size_t n, early_exit_flag_t *out, Pred pred,
                                  bool negate, bool flip) {
  require_device(first, "early-exit search");
  require_device(out, "early-exit flag");
  b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
  b2p_sycl::detail::check_cuda(cudaMemsetAsync(out, 0, sizeof(early_exit_flag_t), q.cuda_stream()), "memset");
  int sms = 0, dev = q.get_device().cuda_ordinal();
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t span = (size_t)kGB * kEarlyUnroll;
  const size_t want = (n + span - 1) / span;
  const unsigned grid = (unsigned)std::min<size_t>(want, (size_t)std::max(sms, 1) * 8);
  early_exit_kernel<<<grid, kGB, 0, q.cuda_stream()>>>(n, first, pred, negate, out);
  if (flip) flip_flag_kernel<><<<1, 1, 0, q.cuda_stream()>>>(out);
  b2p_sycl::detail::check_cuda(cudaGetLastError(), "early-exit search");
  return q.record();
}
}  // namespace detail

template <class ForwardIt, class UnaryPredicate>
b2p_sycl::event any_of(b2p_sycl::queue &q, ForwardIt first, ForwardIt last, detail::early_exit_flag_t *out,
                       UnaryPredicate p, const std::vector<b2p_sycl::event> &deps = {}) {
  if (first == last) return b2p_sycl::event{};
  q.depends_on(deps);
  return detail::early_exit_search(q, first, (size_t)std::distance(first, last), out, p, false, false);
}

template <class ForwardIt, class UnaryPredicate>
b2p_sycl::event all_of(b2p_sycl::queue &q, ForwardIt first, ForwardIt last, detail::early_exit_flag_t *out,
                       UnaryPredicate p, const std::vector<b2p_sycl::event> &deps = {}) {
  if (first == last) return b2p_sycl::event{};
  q.depends_on(deps);
  return detail::early_exit_search(q, first, (size_t)std::distance(first, last), out, p, true, true);
}

template <class ForwardIt, class UnaryPredicate>
b2p_sycl::event none_of(b2p_sycl::queue &q, ForwardIt first, ForwardIt last, detail::early_exit_flag_t *out,
                        UnaryPredicate p, const std::vector<b2p_sycl::event> &deps = {}) {
  if (first == last) return b2p_sycl::event{};
  q.depends_on(deps);
  return detail::early_exit_search(q, first, (size_t)std::distance(first, last), out, p, false, true);
}

// ------------------------------------------------------------ sort / merge
// (algorithm.hpp:519-560).  Both are stable merge-path kernels
// (b2p_device/merge.cuh) for any comparator callable on the device: sort is
// a merge sort, merge one pass over the output.  Keys of the standard types
// with std::less / std::greater on contiguous ranges go through libb2p
// (b2p_sort, b2p_merge); other comparators and types run the same kernels
// compiled into the caller; non-pointer iterators are gathered into a
// contiguous buffer first and scattered back after.  The reference's sort is
// an in-place bitonic network without scratch; this one needs a second
// array of n keys (and the merge passes' tile starts): the queue's working
// buffer, kept across calls.

namespace detail {

template <class T, class It>
__global__ void gather_kernel(It first, size_t n, T *out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = *(first + i);
}

template <class T, class It>
__global__ void scatter_kernel(const T *in, size_t n, It out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    *(out + i) = in[i];
}

inline unsigned copy_grid(size_t n) { return (unsigned)std::min<size_t>((n + kGB - 1) / kGB, 148 * 16); }

template <class C>
struct std_order : std::integral_constant<int, 0> {};
template <class U>
struct std_order<std::less<U>> : std::integral_constant<int, 1> {};
template <class U>
struct std_order<std::greater<U>> : std::integral_constant<int, 2> {};

// dtype code of a key type libb2p sorts and merges, or -1
template <class T>
constexpr int sort_dtype() {
  constexpr int d = dtype_code<T>();
  return (d >= 0 && d != B2P_BF16) ? d : -1;
}

template <class T>
void check_sortable() {
  static_assert(std::is_trivially_copyable_v<T>, "sort/merge: keys must be trivially copyable");
  static_assert(sizeof(T) <= 64, "sort/merge: keys of more than 64 bytes are not supported");
}

}  // namespace detail

template <class RandomIt, class Compare = std::less<>>
b2p_sycl::event sort(b2p_sycl::queue &q, RandomIt first, RandomIt last, Compare comp = std::less<>{},
                     const std::vector<b2p_sycl::event> &deps = {}) {
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return b2p_sycl::event{};
  using T = std::remove_cv_t<detail::value_t<RandomIt>>;
  detail::check_sortable<T>();
  q.depends_on(deps);
  detail::require_device(first, "sort");
  b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
  cudaStream_t st = q.cuda_stream();
  T *keys = nullptr;
  constexpr bool contiguous = std::is_pointer_v<RandomIt>;
  if constexpr (contiguous) {
    keys = const_cast<T *>(&*first);
  } else {
    b2p_sycl::detail::check_cuda(cudaMallocAsync((void **)&keys, n * sizeof(T), st), "sort: keys");
    detail::gather_kernel<T><<<detail::copy_grid(n), detail::kGB, 0, st>>>(first, n, keys);
  }
  void *tmp = nullptr;
  constexpr int dt = detail::sort_dtype<T>(), ord = detail::std_order<Compare>::value;
  // libb2p's sort (radix for long inputs) sizes its own scratch
  size_t tmp_bytes = ::b2p::sort_scratch_bytes<T>(n);
  if constexpr (dt >= 0 && ord != 0) tmp_bytes = b2p_scratch_bytes(B2P_PRIM_SORT, dt, n, 0, B2P_CONFIG_AUTO);
  if (n > (size_t)::b2p::merge_tile<T>()) tmp = q.work_buffer(tmp_bytes);
  int rc;
  if constexpr (dt >= 0 && ord != 0)
    rc = b2p_sort(dt, keys, n, ord == 2, tmp, tmp ? tmp_bytes : 0, (b2p_stream)st);
  else
    rc = ::b2p::launch_sort(keys, n, comp, tmp, tmp ? tmp_bytes : 0, st);
  if constexpr (!contiguous) {
    detail::scatter_kernel<T><<<detail::copy_grid(n), detail::kGB, 0, st>>>(keys, n, first);
    cudaFreeAsync(keys, st);
  }
  b2p_sycl::detail::check_b2p(rc, "sort");
  b2p_sycl::detail::check_cuda(cudaGetLastError(), "sort");
  return q.record();
}

template <class ForwardIt1, class ForwardIt2, class ForwardIt3, class Compare = std::less<>>
b2p_sycl::event merge(b2p_sycl::queue &q, util::allocation_group &scratch, ForwardIt1 first1, ForwardIt1 last1,
                      ForwardIt2 first2, ForwardIt2 last2, ForwardIt3 d_first, Compare comp = std::less<>{},
                      const std::vector<b2p_sycl::event> &deps = {}) {
  const size_t n1 = (size_t)std::distance(first1, last1), n2 = (size_t)std::distance(first2, last2);
  if (n1 + n2 == 0) return b2p_sycl::event{};
  using T = std::remove_cv_t<detail::value_t<ForwardIt1>>;
  detail::check_sortable<T>();
  q.depends_on(deps);
  if (n1) detail::require_device(first1, "merge");
  if (n2) detail::require_device(first2, "merge");
  detail::require_device(d_first, "merge");
  b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
  cudaStream_t st = q.cuda_stream();
  // contiguous views of the inputs and the output (gathered when needed)
  auto view_in = [&](auto first, size_t n) -> const T * {
    using It = decltype(first);
    if constexpr (std::is_pointer_v<It> && std::is_same_v<std::remove_cv_t<detail::value_t<It>>, T>) {
      return n ? &*first : nullptr;
    } else {
      T *buf = scratch.obtain<T>(n ? n : 1);
      if (n) detail::gather_kernel<T><<<detail::copy_grid(n), detail::kGB, 0, st>>>(first, n, buf);
      return buf;
    }
  };
  const T *a = view_in(first1, n1);
  const T *b = view_in(first2, n2);
  constexpr bool direct_out =
      std::is_pointer_v<ForwardIt3> && std::is_same_v<std::remove_cv_t<detail::value_t<ForwardIt3>>, T> &&
      !std::is_const_v<std::remove_reference_t<decltype(*d_first)>>;
  T *out = nullptr;
  if constexpr (direct_out) out = &*d_first;
  else out = scratch.obtain<T>(n1 + n2);
  const size_t sb = ::b2p::merge_scratch_bytes<T>(n1 + n2);
  void *splits = scratch.obtain<unsigned char>(sb);
  int rc;
  constexpr int dt = detail::sort_dtype<T>(), ord = detail::std_order<Compare>::value;
  if constexpr (dt >= 0 && ord != 0)
    rc = b2p_merge(dt, a, n1, b, n2, out, ord == 2, splits, sb, (b2p_stream)st);
  else
    rc = ::b2p::launch_merge(a, n1, b, n2, out, comp, splits, sb, st);
  b2p_sycl::detail::check_b2p(rc, "merge");
  if constexpr (!direct_out)
    detail::scatter_kernel<T><<<detail::copy_grid(n1 + n2), detail::kGB, 0, st>>>(out, n1 + n2, d_first);
  b2p_sycl::detail::check_cuda(cudaGetLastError(), "merge");
  return q.record();
}

}  // namespace algorithms
}  // namespace hipsycl

namespace acpp {
namespace algorithms = ::hipsycl::algorithms;
}
