// Minimal SYCL-2020 host/device layer for the data-parallel primitive path,
// compiled with nvcc for sm_100a.  It provides what user code of the
// reference's algorithms library, sycl::reduction, group algorithms and
// atomic_ref needs, mapped directly onto CUDA:
//
//   sycl::queue         one in-order CUDA stream on one device
//                       (reference: sycl/queue.hpp; in-order queues are what
//                       the algorithms library and stdpar use,
//                       std/stdpar/detail/sycl_glue.hpp:54-58)
//   sycl::event         a CUDA event recorded after a submission
//   sycl::device        a CUDA device ordinal
//   USM                 malloc_device / malloc_shared / malloc_host / free
//   range/id/item/nd_range/nd_item/group/sub_group (1-D)
//   functors            plus, multiplies, minimum, maximum, bit_and, bit_or,
//                       bit_xor, logical_and, logical_or, known_identity
//                       (sycl/libkernel/functional.hpp:123-245)
//   sycl::reduction     reduction(var[, identity], op[, props]) with
//                       property::reduction::initialize_to_identity, reducer
//                       combine() and compound operators
//                       (sycl/libkernel/reduction.hpp:22-249), run by
//                       queue/handler::parallel_for(range, reduction, kernel)
//                       (sycl/handler.hpp:799-975)
//   group algorithms    reduce_over_group, inclusive/exclusive_scan_over_group,
//                       joint_reduce, joint_inclusive/exclusive_scan,
//                       group_barrier (sycl/libkernel/group_functions.hpp:142-239)
//   sycl::atomic_ref    on cuda::atomic_ref (sycl/libkernel/atomic_ref.hpp:45-303)
//
// Kernels passed to parallel_for are lambdas compiled for the device; nvcc
// requires those defined in host code to be extended lambdas
// (`[=] __host__ __device__ (...)`, flag --extended-lambda).  Standard
// functors need no annotation.  Errors throw sycl::exception; nothing falls
// back to the host.
#pragma once

#ifndef __CUDACC__
#error "hipSYCL_b2p/sycl.hpp contains device code: compile with nvcc"
#endif

#include <cuda_runtime.h>
#include <cuda/atomic>

#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../b2p.h"
#include "../b2p_device/reduce.cuh"

#include <mutex>

#define B2P_HD __host__ __device__

namespace b2p_sycl {

// ------------------------------------------------------------------ errors

class exception : public std::runtime_error {
 public:
  exception(int code, const std::string &what) : std::runtime_error(what), code_(code) {}
  int code() const noexcept { return code_; }

 private:
  int code_;
};

namespace detail {
inline void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw exception(B2P_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
inline void check_b2p(int st, const char *what) {
  if (st != B2P_OK) throw exception(st, std::string(what) + ": " + b2p_status_string(st));
}
// Restores the calling thread's current device on scope exit.
class device_guard {
 public:
  explicit device_guard(int dev) {
    cudaGetDevice(&old_);
    if (old_ != dev) check_cuda(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~device_guard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != old_) cudaSetDevice(old_);
  }

 private:
  int old_ = 0;
};
}  // namespace detail

// ------------------------------------------------------------------ device

class device {
 public:
  device() { detail::check_cuda(cudaGetDevice(&id_), "cudaGetDevice"); }
  explicit device(int cuda_ordinal) : id_(cuda_ordinal) {}
  int cuda_ordinal() const { return id_; }
  bool is_gpu() const { return true; }
  bool is_cpu() const { return false; }
  bool is_host() const { return false; }
  friend bool operator==(const device &a, const device &b) { return a.id_ == b.id_; }
  friend bool operator!=(const device &a, const device &b) { return a.id_ != b.id_; }

 private:
  int id_ = 0;
};

// ------------------------------------------------------------------- event

class event {
 public:
  event() = default;  // already complete
  static event record(cudaStream_t s, int dev) {
    detail::device_guard g(dev);
    auto p = std::make_shared<impl>();
    detail::check_cuda(cudaEventCreateWithFlags(&p->ev, cudaEventDisableTiming), "cudaEventCreate");
    detail::check_cuda(cudaEventRecord(p->ev, s), "cudaEventRecord");
    event e;
    e.p_ = std::move(p);
    return e;
  }
  void wait() const {
    if (p_) detail::check_cuda(cudaEventSynchronize(p_->ev), "event::wait");
  }
  void wait_and_throw() const { wait(); }
  static void wait(const std::vector<event> &evs) {
    for (const auto &e : evs) e.wait();
  }
  bool is_complete() const { return !p_ || cudaEventQuery(p_->ev) == cudaSuccess; }
  cudaEvent_t native() const { return p_ ? p_->ev : nullptr; }

 private:
  struct impl {
    cudaEvent_t ev = nullptr;
    ~impl() {
      if (ev) cudaEventDestroy(ev);
    }
  };
  std::shared_ptr<impl> p_;
};

// ------------------------------------------------------- index spaces (1-D)

template <int D = 1>
struct id;
template <>
struct id<1> {
  size_t v = 0;
  B2P_HD id() {}
  B2P_HD id(size_t i) : v(i) {}
  B2P_HD size_t operator[](int) const { return v; }
  B2P_HD size_t get(int) const { return v; }
  B2P_HD operator size_t() const { return v; }
};

template <int D = 1>
struct range;
template <>
struct range<1> {
  size_t v = 0;
  B2P_HD range() {}
  B2P_HD range(size_t n) : v(n) {}
  B2P_HD size_t operator[](int) const { return v; }
  B2P_HD size_t get(int) const { return v; }
  B2P_HD size_t size() const { return v; }
};

template <int D = 1>
struct item;
template <>
struct item<1> {
  size_t i, n;
  B2P_HD id<1> get_id() const { return id<1>(i); }
  B2P_HD size_t get_id(int) const { return i; }
  B2P_HD size_t get_linear_id() const { return i; }
  B2P_HD range<1> get_range() const { return range<1>(n); }
  B2P_HD size_t operator[](int) const { return i; }
  B2P_HD operator id<1>() const { return id<1>(i); }
};

template <int D = 1>
struct nd_range;
template <>
struct nd_range<1> {
  range<1> global, local;
  nd_range(range<1> g, range<1> l) : global(g), local(l) {}
  range<1> get_global_range() const { return global; }
  range<1> get_local_range() const { return local; }
};

// A work-group: the CUDA thread block executing the nd_range kernel.
template <int D = 1>
struct group;
template <>
struct group<1> {
  static constexpr int dimensions = 1;
  __device__ size_t get_local_linear_id() const { return threadIdx.x; }
  __device__ id<1> get_local_id() const { return id<1>(threadIdx.x); }
  __device__ size_t get_local_linear_range() const { return blockDim.x; }
  __device__ range<1> get_local_range() const { return range<1>(blockDim.x); }
  __device__ size_t get_group_linear_id() const { return blockIdx.x; }
  __device__ id<1> get_group_id() const { return id<1>(blockIdx.x); }
  __device__ range<1> get_group_range() const { return range<1>(gridDim.x); }
  __device__ bool leader() const { return threadIdx.x == 0; }
};

// A sub-group: one warp of 32 lanes (the last one of a block whose size is
// not a multiple of 32 has fewer).
struct sub_group {
  static constexpr int dimensions = 1;
  __device__ unsigned get_local_linear_id() const { return threadIdx.x & 31u; }
  __device__ id<1> get_local_id() const { return id<1>(threadIdx.x & 31u); }
  __device__ unsigned get_local_linear_range() const {
    const unsigned first = threadIdx.x & ~31u;
    const unsigned left = blockDim.x - first;
    return left < 32u ? left : 32u;
  }
  __device__ range<1> get_local_range() const { return range<1>(get_local_linear_range()); }
  __device__ range<1> get_max_local_range() const { return range<1>(32); }
  __device__ unsigned get_group_linear_id() const { return threadIdx.x >> 5; }
  __device__ id<1> get_group_id() const { return id<1>(threadIdx.x >> 5); }
  __device__ range<1> get_group_range() const { return range<1>((blockDim.x + 31) / 32); }
  __device__ bool leader() const { return (threadIdx.x & 31u) == 0; }
  __device__ unsigned member_mask() const {
    const unsigned n = get_local_linear_range();
    return n == 32u ? 0xffffffffu : ((1u << n) - 1u);
  }
};

template <int D = 1>
struct nd_item;
template <>
struct nd_item<1> {
  size_t global_size;
  __device__ size_t get_global_id(int = 0) const { return (size_t)blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ size_t get_global_linear_id() const { return get_global_id(); }
  __device__ size_t get_local_id(int = 0) const { return threadIdx.x; }
  __device__ size_t get_local_linear_id() const { return threadIdx.x; }
  __device__ size_t get_group_linear_id() const { return blockIdx.x; }
  __device__ size_t get_local_range(int = 0) const { return blockDim.x; }
  __device__ size_t get_global_range(int = 0) const { return global_size; }
  __device__ size_t get_group_range(int = 0) const { return gridDim.x; }
  __device__ group<1> get_group() const { return group<1>{}; }
  __device__ size_t get_group(int) const { return blockIdx.x; }
  __device__ sub_group get_sub_group() const { return sub_group{}; }
  __device__ void barrier() const { __syncthreads(); }
};

// -------------------------------------------------------------- functors

#define B2P_SYCL_FUNCTOR(NAME, EXPR)                                         \
  template <class T = void>                                                  \
  struct NAME {                                                              \
    B2P_HD constexpr T operator()(const T &x, const T &y) const { return EXPR; } \
  };                                                                         \
  template <>                                                                \
  struct NAME<void> {                                                        \
    template <class T, class U>                                              \
    B2P_HD constexpr auto operator()(const T &x, const U &y) const { return EXPR; } \
  };
B2P_SYCL_FUNCTOR(plus, x + y)
B2P_SYCL_FUNCTOR(multiplies, x *y)
B2P_SYCL_FUNCTOR(minimum, (x < y) ? x : y)
B2P_SYCL_FUNCTOR(maximum, (x < y) ? y : x)
B2P_SYCL_FUNCTOR(bit_and, x &y)
B2P_SYCL_FUNCTOR(bit_or, x | y)
B2P_SYCL_FUNCTOR(bit_xor, x ^ y)
B2P_SYCL_FUNCTOR(logical_and, x &&y)
B2P_SYCL_FUNCTOR(logical_or, x || y)
#undef B2P_SYCL_FUNCTOR

// known_identity / has_known_identity (sycl/libkernel/functional.hpp:123-245)
template <class Op, class T, class = void>
struct has_known_identity : std::false_type {};
template <class Op, class T>
inline constexpr bool has_known_identity_v = has_known_identity<Op, T>::value;
template <class Op, class T>
struct known_identity;

namespace detail {
template <class Op, template <class> class F>
struct is_op : std::false_type {};
template <class U, template <class> class F>
struct is_op<F<U>, F> : std::true_type {};
template <class Op, class T>
B2P_HD constexpr T identity_of() {
  if constexpr (is_op<Op, plus>::value || is_op<Op, bit_or>::value || is_op<Op, bit_xor>::value) return T{};
  else if constexpr (is_op<Op, multiplies>::value) return T{1};
  else if constexpr (is_op<Op, bit_and>::value) return ~T{};
  else if constexpr (is_op<Op, logical_and>::value) return T{true};
  else if constexpr (is_op<Op, logical_or>::value) return T{false};
  else if constexpr (is_op<Op, minimum>::value) {
    if constexpr (std::is_integral_v<T>) return std::numeric_limits<T>::max();
    else return std::numeric_limits<T>::infinity();
  } else {
    if constexpr (std::is_integral_v<T>) return std::numeric_limits<T>::lowest();
    else return -std::numeric_limits<T>::infinity();
  }
}
template <class Op, class T>
constexpr bool known_op() {
  return is_op<Op, plus>::value || is_op<Op, multiplies>::value ||
         ((is_op<Op, bit_and>::value || is_op<Op, bit_or>::value || is_op<Op, bit_xor>::value) &&
          std::is_integral_v<T>) ||
         ((is_op<Op, logical_and>::value || is_op<Op, logical_or>::value) && std::is_same_v<T, bool>) ||
         ((is_op<Op, minimum>::value || is_op<Op, maximum>::value) && std::is_arithmetic_v<T>);
}
}  // namespace detail

template <class Op, class T>
struct has_known_identity<Op, T, std::enable_if_t<detail::known_op<Op, T>()>> : std::true_type {};
template <class Op, class T>
struct known_identity {
  static constexpr T value = detail::identity_of<Op, T>();
};
template <class Op, class T>
inline constexpr T known_identity_v = known_identity<Op, T>::value;

// ------------------------------------------------------------ properties

namespace property {
namespace reduction {
struct initialize_to_identity {};
}  // namespace reduction
}  // namespace property

class property_list {
 public:
  property_list() = default;
  template <class... Props>
  property_list(Props... props) {
    (set(props), ...);
  }
  template <class P>
  bool has_property() const {
    if constexpr (std::is_same_v<P, property::reduction::initialize_to_identity>) return init_to_identity_;
    else return false;
  }

 private:
  void set(property::reduction::initialize_to_identity) { init_to_identity_ = true; }
  bool init_to_identity_ = false;
};

// -------------------------------------------------------------- reduction

// Reduction descriptor: result variable, operator and (known or given)
// identity.  Without a known identity the reducer tracks whether it holds a
// value at all, as the reference does with its initialisation flags
// (algorithms/reduction/reduction_descriptor.hpp:25-146).
template <class T, class Op>
struct reduction_descriptor {
  using value_type = T;
  using binary_operation = Op;
  T *var;
  Op op;
  T identity;
  bool has_identity;
  bool init_to_identity;
};

template <class T, class Op>
reduction_descriptor<T, Op> reduction(T *var, Op op, const property_list &props = {}) {
  T id{};
  bool known = false;
  if constexpr (has_known_identity_v<Op, T>) {
    id = known_identity_v<Op, T>;
    known = true;
  }
  return {var, op, id, known, props.has_property<property::reduction::initialize_to_identity>()};
}
template <class T, class Op>
reduction_descriptor<T, Op> reduction(T *var, const T &identity, Op op, const property_list &props = {}) {
  return {var, op, identity, true, props.has_property<property::reduction::initialize_to_identity>()};
}

// The reducer handed to the kernel: combines partial values into a
// per-work-item accumulator.
template <class T, class Op>
class reducer {
 public:
  using value_type = T;
  using binary_operation = Op;
  B2P_HD reducer(Op op, T identity, bool has_identity) : op_(op), v_(identity), has_(has_identity) {}
  B2P_HD reducer &combine(const T &x) {
    v_ = has_ ? op_(v_, x) : x;
    has_ = true;
    return *this;
  }
  B2P_HD T identity() const { return v_; }
  B2P_HD const T &value() const { return v_; }
  B2P_HD bool has_value() const { return has_; }

 private:
  Op op_;
  T v_;
  bool has_;
};

template <class T, class Op, class = std::enable_if_t<detail::is_op<Op, plus>::value>>
B2P_HD reducer<T, Op> &operator+=(reducer<T, Op> &r, const T &v) {
  return r.combine(v);
}
template <class T, class Op, class = std::enable_if_t<detail::is_op<Op, plus>::value>>
B2P_HD reducer<T, Op> &operator++(reducer<T, Op> &r) {
  return r.combine(T{1});
}
template <class T, class Op, class = std::enable_if_t<detail::is_op<Op, multiplies>::value>>
B2P_HD reducer<T, Op> &operator*=(reducer<T, Op> &r, const T &v) {
  return r.combine(v);
}
template <class T, class Op, class = std::enable_if_t<detail::is_op<Op, bit_and>::value>>
B2P_HD reducer<T, Op> &operator&=(reducer<T, Op> &r, const T &v) {
  return r.combine(v);
}
template <class T, class Op, class = std::enable_if_t<detail::is_op<Op, bit_or>::value>>
B2P_HD reducer<T, Op> &operator|=(reducer<T, Op> &r, const T &v) {
  return r.combine(v);
}
template <class T, class Op, class = std::enable_if_t<detail::is_op<Op, bit_xor>::value>>
B2P_HD reducer<T, Op> &operator^=(reducer<T, Op> &r, const T &v) {
  return r.combine(v);
}

// ------------------------------------------------ group algorithms (device)

namespace detail {

template <class T>
__device__ T shfl_idx(unsigned mask, T v, int src) {
  static_assert(sizeof(T) <= 8, "group algorithms: values of at most 8 bytes");
  if constexpr (sizeof(T) <= 4) {
    unsigned u = 0;
    memcpy(&u, &v, sizeof(T));
    u = __shfl_sync(mask, u, src);
    memcpy(&v, &u, sizeof(T));
  } else {
    unsigned long long u = 0;
    memcpy(&u, &v, sizeof(T));
    u = __shfl_sync(mask, u, src);
    memcpy(&v, &u, sizeof(T));
  }
  return v;
}

// Inclusive scan over the first `n` lanes of the warp (lanes >= n keep x).
template <class T, class Op>
__device__ T warp_inclusive(T x, Op op, unsigned mask, unsigned lane, unsigned n) {
  for (unsigned d = 1; d < n; d <<= 1) {
    const T o = shfl_idx(mask, x, (int)(lane >= d ? lane - d : lane));
    if (lane >= d && lane < n) x = op(o, x);
  }
  return x;
}

// Shared staging for block-level group algorithms: one slot per warp plus
// a broadcast slot, for values of at most 8 bytes.
__device__ inline unsigned long long *group_slots() {
  __shared__ unsigned long long slots[33];
  return slots;
}

// Inclusive scan over the work-group; *total receives the group total.
template <class T, class Op>
__device__ T block_inclusive(T x, Op op, T *total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned nw = (blockDim.x + 31) / 32;
  sub_group sg;
  const unsigned n = sg.get_local_linear_range();
  const unsigned mask = sg.member_mask();
  T incl = warp_inclusive(x, op, mask, lane, n);
  unsigned long long *slots = group_slots();
  __syncthreads();  // previous use of the slots is over
  if (lane == n - 1) memcpy(&slots[warp], &incl, sizeof(T));
  __syncthreads();
  if (warp == 0) {
    const unsigned wmask = nw >= 32 ? 0xffffffffu : ((1u << nw) - 1u);
    if (lane < nw) {
      T w;
      memcpy(&w, &slots[lane], sizeof(T));
      w = warp_inclusive(w, op, wmask, lane, nw);
      memcpy(&slots[lane], &w, sizeof(T));
    }
  }
  __syncthreads();
  if (warp > 0) {
    T prev;
    memcpy(&prev, &slots[warp - 1], sizeof(T));
    incl = op(prev, incl);
  }
  memcpy(total, &slots[nw - 1], sizeof(T));
  return incl;
}

}  // namespace detail

__device__ inline void group_barrier(group<1>) { __syncthreads(); }
__device__ inline void group_barrier(sub_group sg) { __syncwarp(sg.member_mask()); }

// reduce_over_group(g, x, op) / (g, x, init, op)
template <class T, class Op>
__device__ T reduce_over_group(group<1>, T x, Op op) {
  T total;
  (void)detail::block_inclusive(x, op, &total);
  return total;
}
template <class T, class Op>
__device__ T reduce_over_group(sub_group sg, T x, Op op) {
  const unsigned n = sg.get_local_linear_range();
  const T incl = detail::warp_inclusive(x, op, sg.member_mask(), sg.get_local_linear_id(), n);
  return detail::shfl_idx(sg.member_mask(), incl, (int)(n - 1));
}
template <class G, class V, class T, class Op>
__device__ T reduce_over_group(G g, V x, T init, Op op) {
  return op(init, reduce_over_group(g, static_cast<T>(x), op));
}

// inclusive_scan_over_group(g, x, op[, init])
template <class T, class Op>
__device__ T inclusive_scan_over_group(group<1>, T x, Op op) {
  T total;
  return detail::block_inclusive(x, op, &total);
}
template <class T, class Op>
__device__ T inclusive_scan_over_group(sub_group sg, T x, Op op) {
  return detail::warp_inclusive(x, op, sg.member_mask(), sg.get_local_linear_id(), sg.get_local_linear_range());
}
template <class G, class V, class Op, class T>
__device__ T inclusive_scan_over_group(G g, V x, Op op, T init) {
  return op(init, inclusive_scan_over_group(g, static_cast<T>(x), op));
}

// exclusive_scan_over_group(g, x, [init,] op)
template <class T, class Op>
__device__ T exclusive_scan_over_group(group<1> g, T x, T init, Op op) {
  const T incl = inclusive_scan_over_group(g, x, op);
  const unsigned lane = threadIdx.x & 31u;
  sub_group sg;
  T prev = detail::shfl_idx(sg.member_mask(), incl, lane == 0 ? 0 : (int)lane - 1);
  // lane 0 of a warp takes the previous warp's last inclusive value
  unsigned long long *slots = detail::group_slots();
  __syncthreads();
  if (lane == sg.get_local_linear_range() - 1) memcpy(&slots[threadIdx.x >> 5], &incl, sizeof(T));
  __syncthreads();
  if (lane == 0 && threadIdx.x > 0) memcpy(&prev, &slots[(threadIdx.x >> 5) - 1], sizeof(T));
  return threadIdx.x == 0 ? init : op(init, prev);
}
template <class T, class Op>
__device__ T exclusive_scan_over_group(sub_group sg, T x, T init, Op op) {
  const unsigned lane = sg.get_local_linear_id();
  const T incl = inclusive_scan_over_group(sg, x, op);
  const T prev = detail::shfl_idx(sg.member_mask(), incl, lane == 0 ? 0 : (int)lane - 1);
  return lane == 0 ? init : op(init, prev);
}
template <class G, class T, class Op>
__device__ T exclusive_scan_over_group(G g, T x, Op op) {
  static_assert(has_known_identity_v<Op, T>, "exclusive_scan_over_group without init needs a known identity");
  return exclusive_scan_over_group(g, x, known_identity_v<Op, T>, op);
}

// joint_reduce(g, first, last, [init,] op): strided partial values, then a
// group reduction (group_functions.hpp:142-239 semantics).
template <class G, class Ptr, class T, class Op>
__device__ T joint_reduce(G g, Ptr first, Ptr last, T init, Op op) {
  const size_t n = (size_t)(last - first);
  const size_t lid = g.get_local_linear_id(), lr = g.get_local_linear_range();
  bool has = false;
  T acc = init;
  for (size_t i = lid; i < n; i += lr) {
    acc = has ? op(acc, static_cast<T>(first[i])) : static_cast<T>(first[i]);
    has = true;
  }
  // members without elements contribute nothing: the combination below
  // skips them, in member order
  const T r = acc;
  if constexpr (std::is_same_v<G, sub_group>) {
    const unsigned mask = g.member_mask(), lane = g.get_local_linear_id(), cnt = g.get_local_linear_range();
    unsigned hm = __ballot_sync(mask, has);
    // reduce only over lanes with values, in lane order
    T out{};
    bool first_v = true;
    for (unsigned l = 0; l < cnt; ++l) {
      const T v = detail::shfl_idx(mask, r, (int)l);
      if ((hm >> l) & 1u) {
        out = first_v ? v : op(out, v);
        first_v = false;
      }
    }
    (void)lane;
    return first_v ? init : op(init, out);
  } else {
    unsigned long long *slots = detail::group_slots();
    __shared__ int any_slot[32];
    // warp level
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    sub_group sg;
    const unsigned mask = sg.member_mask(), cnt = sg.get_local_linear_range();
    const unsigned hm = __ballot_sync(mask, has);
    T wv{};
    bool wh = false;
    for (unsigned l = 0; l < cnt; ++l) {
      const T v = detail::shfl_idx(mask, r, (int)l);
      if ((hm >> l) & 1u) {
        wv = wh ? op(wv, v) : v;
        wh = true;
      }
    }
    __syncthreads();
    if (lane == 0) {
      memcpy(&slots[warp], &wv, sizeof(T));
      any_slot[warp] = wh;
    }
    __syncthreads();
    T out = init;
    bool got = false;
    const unsigned nw = (blockDim.x + 31) / 32;
    for (unsigned w = 0; w < nw; ++w) {
      if (any_slot[w]) {
        T v;
        memcpy(&v, &slots[w], sizeof(T));
        out = got ? op(out, v) : v;
        got = true;
      }
    }
    return got ? op(init, out) : init;
  }
}
template <class G, class Ptr, class Op>
__device__ auto joint_reduce(G g, Ptr first, Ptr last, Op op) {
  using T = std::remove_cv_t<std::remove_reference_t<decltype(*first)>>;
  static_assert(has_known_identity_v<Op, T>, "joint_reduce without init needs a known identity");
  return joint_reduce(g, first, last, known_identity_v<Op, T>, op);
}

// joint_inclusive_scan / joint_exclusive_scan: the range is scanned in
// chunks of one element per member; each chunk starts from the carry of the
// previous one (group_functions.hpp:361-432 semantics).
template <class G, class InPtr, class OutPtr, class Op, class T>
__device__ OutPtr joint_inclusive_scan(G g, InPtr first, InPtr last, OutPtr result, Op op, T init) {
  const size_t n = (size_t)(last - first);
  const size_t lid = g.get_local_linear_id(), lr = g.get_local_linear_range();
  T carry = init;
  for (size_t base = 0; base < n; base += lr) {
    const size_t i = base + lid;
    // members past the end contribute the carry-neutral position: they take
    // the last element's place but their result is not stored
    T x = i < n ? static_cast<T>(first[i]) : static_cast<T>(first[n - 1]);
    T incl = inclusive_scan_over_group(g, x, op);
    const T v = op(carry, incl);
    if (i < n) result[i] = v;
    const size_t last_i = (n - base < lr ? n - base : lr) - 1;
    if constexpr (std::is_same_v<G, sub_group>) {
      carry = detail::shfl_idx(g.member_mask(), v, (int)last_i);
    } else {
      unsigned long long *slots = detail::group_slots();
      __syncthreads();
      if (lid == last_i) memcpy(&slots[32], &v, sizeof(T));
      __syncthreads();
      memcpy(&carry, &slots[32], sizeof(T));
    }
  }
  return result + n;
}
template <class G, class InPtr, class OutPtr, class Op>
__device__ OutPtr joint_inclusive_scan(G g, InPtr first, InPtr last, OutPtr result, Op op) {
  using T = std::remove_cv_t<std::remove_reference_t<decltype(*result)>>;
  const size_t n = (size_t)(last - first);
  if (n == 0) return result;
  // the first element starts the scan: run with init = first[0] over [1, n)
  const size_t lid = g.get_local_linear_id();
  if (lid == 0) result[0] = static_cast<T>(first[0]);
  return joint_inclusive_scan(g, first + 1, last, result + 1, op, static_cast<T>(first[0]));
}
template <class G, class InPtr, class OutPtr, class T, class Op>
__device__ OutPtr joint_exclusive_scan(G g, InPtr first, InPtr last, OutPtr result, T init, Op op) {
  const size_t n = (size_t)(last - first);
  if (n == 0) return result;
  const size_t lid = g.get_local_linear_id(), lr = g.get_local_linear_range();
  T carry = init;
  for (size_t base = 0; base < n; base += lr) {
    const size_t i = base + lid;
    T x = i < n ? static_cast<T>(first[i]) : static_cast<T>(first[n - 1]);
    const T incl = inclusive_scan_over_group(g, x, op);
    const T v = op(carry, incl);
    // exclusive value of element i = carry (+) inclusive value of i-1
    T prev;
    const size_t last_i = (n - base < lr ? n - base : lr) - 1;
    if constexpr (std::is_same_v<G, sub_group>) {
      prev = detail::shfl_idx(g.member_mask(), v, lid == 0 ? 0 : (int)lid - 1);
      if (i < n) result[i] = lid == 0 ? carry : prev;
      carry = detail::shfl_idx(g.member_mask(), v, (int)last_i);
    } else {
      unsigned long long *slots = detail::group_slots();
      __shared__ unsigned long long vals[1024];
      __syncthreads();
      memcpy(&vals[lid], &v, sizeof(T));
      if (lid == last_i) memcpy(&slots[32], &v, sizeof(T));
      __syncthreads();
      if (i < n) {
        if (lid == 0) result[i] = carry;
        else memcpy(&prev, &vals[lid - 1], sizeof(T)), result[i] = prev;
      }
      memcpy(&carry, &slots[32], sizeof(T));
    }
  }
  return result + n;
}
template <class G, class InPtr, class OutPtr, class Op>
__device__ OutPtr joint_exclusive_scan(G g, InPtr first, InPtr last, OutPtr result, Op op) {
  using T = std::remove_cv_t<std::remove_reference_t<decltype(*result)>>;
  static_assert(has_known_identity_v<Op, T>, "joint_exclusive_scan without init needs a known identity");
  return joint_exclusive_scan(g, first, last, result, known_identity_v<Op, T>, op);
}

// ------------------------------------------------------------ atomic_ref

enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, generic_space };
}

namespace detail {
template <memory_scope S>
struct cuda_scope;
template <>
struct cuda_scope<memory_scope::work_item> {
  static constexpr cuda::thread_scope value = cuda::thread_scope_thread;
};
template <>
struct cuda_scope<memory_scope::sub_group> {
  static constexpr cuda::thread_scope value = cuda::thread_scope_block;
};
template <>
struct cuda_scope<memory_scope::work_group> {
  static constexpr cuda::thread_scope value = cuda::thread_scope_block;
};
template <>
struct cuda_scope<memory_scope::device> {
  static constexpr cuda::thread_scope value = cuda::thread_scope_device;
};
template <>
struct cuda_scope<memory_scope::system> {
  static constexpr cuda::thread_scope value = cuda::thread_scope_system;
};
B2P_HD constexpr cuda::std::memory_order cuda_order(memory_order o) {
  return o == memory_order::relaxed   ? cuda::std::memory_order_relaxed
         : o == memory_order::acquire ? cuda::std::memory_order_acquire
         : o == memory_order::release ? cuda::std::memory_order_release
         : o == memory_order::acq_rel ? cuda::std::memory_order_acq_rel
                                      : cuda::std::memory_order_seq_cst;
}
}  // namespace detail

// sycl::atomic_ref (sycl/libkernel/atomic_ref.hpp:45-303).  Like the
// reference, T is a 32- or 64-bit integer, float, double or a pointer.
template <class T, memory_order DefaultOrder, memory_scope DefaultScope,
          access::address_space Space = access::address_space::generic_space>
class atomic_ref {
  static_assert((sizeof(T) == 4 || sizeof(T) == 8) && std::is_arithmetic_v<T>,
                "atomic_ref: 32- or 64-bit integers, float or double");
  using impl = cuda::atomic_ref<T, detail::cuda_scope<DefaultScope>::value>;

 public:
  using value_type = T;
  static constexpr memory_order default_read_order =
      DefaultOrder == memory_order::acq_rel ? memory_order::acquire : DefaultOrder;
  static constexpr memory_order default_write_order =
      DefaultOrder == memory_order::acq_rel ? memory_order::release : DefaultOrder;

  B2P_HD explicit atomic_ref(T &ref) : a_(ref) {}
  B2P_HD T load(memory_order o = default_read_order) const { return a_.load(detail::cuda_order(o)); }
  B2P_HD void store(T v, memory_order o = default_write_order) const { a_.store(v, detail::cuda_order(o)); }
  B2P_HD operator T() const { return load(); }
  B2P_HD T operator=(T v) const {
    store(v);
    return v;
  }
  B2P_HD T exchange(T v, memory_order o = DefaultOrder) const { return a_.exchange(v, detail::cuda_order(o)); }
  B2P_HD bool compare_exchange_strong(T &expected, T desired, memory_order o = DefaultOrder) const {
    return a_.compare_exchange_strong(expected, desired, detail::cuda_order(o));
  }
  B2P_HD bool compare_exchange_weak(T &expected, T desired, memory_order o = DefaultOrder) const {
    return a_.compare_exchange_weak(expected, desired, detail::cuda_order(o));
  }
  B2P_HD T fetch_add(T v, memory_order o = DefaultOrder) const { return a_.fetch_add(v, detail::cuda_order(o)); }
  B2P_HD T fetch_sub(T v, memory_order o = DefaultOrder) const { return a_.fetch_sub(v, detail::cuda_order(o)); }
  template <class U = T, class = std::enable_if_t<std::is_integral_v<U>>>
  B2P_HD T fetch_and(T v, memory_order o = DefaultOrder) const {
    return a_.fetch_and(v, detail::cuda_order(o));
  }
  template <class U = T, class = std::enable_if_t<std::is_integral_v<U>>>
  B2P_HD T fetch_or(T v, memory_order o = DefaultOrder) const {
    return a_.fetch_or(v, detail::cuda_order(o));
  }
  template <class U = T, class = std::enable_if_t<std::is_integral_v<U>>>
  B2P_HD T fetch_xor(T v, memory_order o = DefaultOrder) const {
    return a_.fetch_xor(v, detail::cuda_order(o));
  }
  B2P_HD T fetch_min(T v, memory_order o = DefaultOrder) const {
    if constexpr (std::is_integral_v<T>) {
      return a_.fetch_min(v, detail::cuda_order(o));
    } else {
      T cur = a_.load(cuda::std::memory_order_relaxed);
      while (v < cur && !a_.compare_exchange_weak(cur, v, detail::cuda_order(o))) {
      }
      return cur;
    }
  }
  B2P_HD T fetch_max(T v, memory_order o = DefaultOrder) const {
    if constexpr (std::is_integral_v<T>) {
      return a_.fetch_max(v, detail::cuda_order(o));
    } else {
      T cur = a_.load(cuda::std::memory_order_relaxed);
      while (cur < v && !a_.compare_exchange_weak(cur, v, detail::cuda_order(o))) {
      }
      return cur;
    }
  }
  B2P_HD T operator+=(T v) const { return fetch_add(v) + v; }
  B2P_HD T operator-=(T v) const { return fetch_sub(v) - v; }
  B2P_HD T operator++(int) const { return fetch_add(T(1)); }
  B2P_HD T operator++() const { return fetch_add(T(1)) + T(1); }

 private:
  mutable impl a_;
};

// ------------------------------------------------------------------- USM

enum class usm_alloc { device, shared, host };

class queue;
namespace detail {
inline int queue_device(const queue &q);
}

// -------------------------------------------------------------- kernels

namespace detail {

constexpr int kBlock = 256;

template <class K>
__global__ void __launch_bounds__(kBlock) range_kernel(size_t n, K k) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if constexpr (std::is_invocable_v<K, item<1>>) k(item<1>{i, n});
    else k(id<1>(i));
  }
}

template <class K>
__global__ void nd_range_kernel(size_t global, K k) {
  k(nd_item<1>{global});
}

// Per-block partials of a reduction kernel: every thread folds the ids of
// its grid-stride range into its reducer; the block combines the reducers
// in thread order (members without a value are skipped).
template <class T, class Op, class K>
__global__ void __launch_bounds__(kBlock)
    reduction_partials_kernel(size_t n, K k, Op op, T identity, bool has_identity, T *partial, int *partial_has) {
  reducer<T, Op> r(op, identity, has_identity);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if constexpr (std::is_invocable_v<K, item<1>, reducer<T, Op> &>) k(item<1>{i, n}, r);
    else k(id<1>(i), r);
  }
  __shared__ T vals[kBlock];
  __shared__ int has[kBlock];
  vals[threadIdx.x] = r.value();
  has[threadIdx.x] = r.has_value();
  __syncthreads();
  for (int s = kBlock / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      const int o = threadIdx.x + s;
      if (has[o]) {
        vals[threadIdx.x] = has[threadIdx.x] ? op(vals[threadIdx.x], vals[o]) : vals[o];
        has[threadIdx.x] = 1;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = vals[0];
    partial_has[blockIdx.x] = has[0];
  }
}

// Combine the block partials in block order and apply the result rule:
// initialize_to_identity -> *var = r, otherwise *var = op(*var, r).
template <class T, class Op>
__global__ void __launch_bounds__(1) reduction_final_kernel(int nb, Op op, const T *partial, const int *partial_has,
                                                           T *var, bool init_to_identity, T identity, bool has_identity) {
  bool has = false;
  T acc{};
  for (int b = 0; b < nb; ++b) {
    if (partial_has[b]) {
      acc = has ? op(acc, partial[b]) : partial[b];
      has = true;
    }
  }
  if (init_to_identity) {
    *var = has ? acc : (has_identity ? identity : *var);
  } else if (has) {
    *var = op(*var, acc);
  }
}

// ------------------------------ reductions on the library's reduce kernel
//
// parallel_for(range, reduction(var, op), kernel) for a standard operator
// (plus, multiplies, minimum, maximum, bit_and/or/xor) on int32/uint32/
// int64/uint64/float/double runs the single-pass reduce kernel of libb2p
// (b2p_device/reduce.cuh) with the user kernel as its source: unit i calls
// kernel(id<1>(i), reducer) on a fresh reducer and folds the reducer's value
// into the lane's accumulator -- compensated (TwoSum) for float plus, and in
// a fixed combination order, so the result is the same for every launch.
// Other types and user operators take the generic kernels above.

template <class T>
constexpr int b2p_dtype() {
  if constexpr (std::is_same_v<T, float>) return B2P_F32;
  else if constexpr (std::is_same_v<T, double>) return B2P_F64;
  else if constexpr (std::is_integral_v<T> && !std::is_same_v<T, bool> && sizeof(T) == 4)
    return std::is_signed_v<T> ? B2P_I32 : B2P_U32;
  else if constexpr (std::is_integral_v<T> && !std::is_same_v<T, bool> && sizeof(T) == 8)
    return std::is_signed_v<T> ? B2P_I64 : B2P_U64;
  else return -1;
}

template <class Op, class T>
constexpr int b2p_op() {
  constexpr bool is_int = std::is_integral_v<T>;
  if constexpr (is_op<Op, plus>::value || is_op<Op, std::plus>::value) return B2P_SUM;
  else if constexpr (is_op<Op, multiplies>::value || is_op<Op, std::multiplies>::value) return B2P_PROD;
  else if constexpr (is_op<Op, minimum>::value) return B2P_MIN;
  else if constexpr (is_op<Op, maximum>::value) return B2P_MAX;
  else if constexpr (is_int && (is_op<Op, bit_and>::value || is_op<Op, std::bit_and>::value)) return B2P_AND;
  else if constexpr (is_int && (is_op<Op, bit_or>::value || is_op<Op, std::bit_or>::value)) return B2P_OR;
  else if constexpr (is_int && (is_op<Op, bit_xor>::value || is_op<Op, std::bit_xor>::value)) return B2P_XOR;
  else return -1;
}

template <class T, class Op>
constexpr bool library_reduction() {
  return b2p_dtype<T>() >= 0 && b2p_op<Op, T>() >= 0;
}

template <class T, class Op>
using library_policy = typename ::b2p::PolicyOf<b2p_dtype<T>(), b2p_op<Op, T>()>::type;

// Unit i of a reduction kernel: the value one work-item's reducer holds
// after kernel(id<1>(i), reducer) (or kernel(item<1>, reducer)).
template <class T, class Op, class K>
struct reduction_source : ::b2p::ValueSource<reduction_source<T, Op, K>, T> {
  K k;
  size_t n;
  Op op;
  T identity;
  reduction_source(K k_, size_t n_, Op op_, T id_) : k(k_), n(n_), op(op_), identity(id_) {}
  __device__ __forceinline__ T value(long long i) const {
    reducer<T, Op> r(op, identity, true);
    if constexpr (std::is_invocable_v<K, item<1>, reducer<T, Op> &>) k(item<1>{(size_t)i, n}, r);
    else k(id<1>((size_t)i), r);
    return r.value();
  }
};

// Scratch of one queue for the library's kernels: grown on demand (the
// queue waits for its own work before a larger buffer replaces the old one),
// zero-filled on allocation when `zero_fill` (the look-back scratch, whose
// status words must start at zero), freed with the queue.  Calls on one
// queue run in stream order, so they can share it.
class queue_scratch {
 public:
  explicit queue_scratch(int dev, bool zero_fill = true) : dev_(dev), zero_fill_(zero_fill) {}
  queue_scratch(const queue_scratch &) = delete;
  queue_scratch &operator=(const queue_scratch &) = delete;
  ~queue_scratch() {
    if (p_) {
      device_guard g(dev_);
      cudaFree(p_);
      cudaGetLastError();
    }
  }
  void *get(size_t bytes, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(mu_);
    if (bytes > bytes_) {
      device_guard g(dev_);
      if (p_) {
        check_cuda(cudaStreamSynchronize(s), "queue scratch");
        cudaFree(p_);
        p_ = nullptr;
      }
      const size_t b = std::max<size_t>(bytes, 64 * 1024);
      check_cuda(cudaMalloc(&p_, b), "queue scratch");
      if (zero_fill_) check_cuda(cudaMemsetAsync(p_, 0, b, s), "queue scratch");
      bytes_ = b;
    }
    return p_;
  }
  size_t size() const { return bytes_; }

 private:
  int dev_;
  bool zero_fill_;
  std::mutex mu_;
  void *p_ = nullptr;
  size_t bytes_ = 0;
};

}  // namespace detail

class handler;

// ----------------------------------------------------------------- queue

class queue {
 public:
  queue() : queue(device{}) {}
  explicit queue(const device &d) : dev_(d) {
    detail::device_guard g(dev_.cuda_ordinal());
    cudaStream_t s = nullptr;
    detail::check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = std::shared_ptr<CUstream_st>(s, [](cudaStream_t p) { cudaStreamDestroy(p); });
    scratch_ = std::make_shared<detail::queue_scratch>(dev_.cuda_ordinal());
    work_ = std::make_shared<detail::queue_scratch>(dev_.cuda_ordinal(), false);
  }
  // Working memory of the queue's library calls that overwrite it with data
  // (the second key array of hipsycl::algorithms::sort): at least `bytes`,
  // kept and reused by later calls in stream order.
  void *work_buffer(size_t bytes) { return work_->get(bytes, cuda_stream()); }
  size_t work_buffer_size() const { return work_->size(); }
  device get_device() const { return dev_; }
  cudaStream_t cuda_stream() const { return stream_.get(); }
  bool is_in_order() const { return true; }

  void wait() const {
    detail::check_cuda(cudaStreamSynchronize(cuda_stream()), "queue::wait");
  }
  void wait_and_throw() const { wait(); }

  // Make later work on this queue wait for `deps` (host-side: no blocking).
  void depends_on(const std::vector<event> &deps) const {
    for (const auto &e : deps)
      if (e.native()) detail::check_cuda(cudaStreamWaitEvent(cuda_stream(), e.native(), 0), "depends_on");
  }
  event record() const { return event::record(cuda_stream(), dev_.cuda_ordinal()); }

  event memcpy(void *dst, const void *src, size_t bytes, const std::vector<event> &deps = {}) const {
    depends_on(deps);
    detail::check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, cuda_stream()), "queue::memcpy");
    return record();
  }
  template <class T>
  event copy(const T *src, T *dst, size_t count, const std::vector<event> &deps = {}) const {
    return memcpy(dst, src, count * sizeof(T), deps);
  }
  event memset(void *p, int v, size_t bytes, const std::vector<event> &deps = {}) const {
    depends_on(deps);
    detail::check_cuda(cudaMemsetAsync(p, v, bytes, cuda_stream()), "queue::memset");
    return record();
  }
  template <class T>
  event fill(T *p, const T &v, size_t count, const std::vector<event> &deps = {}) const {
    return parallel_for(range<1>(count), [=] __device__(id<1> i) { p[i[0]] = v; }, deps);
  }

  // parallel_for(range, kernel): kernel(id<1>) or kernel(item<1>).
  template <class K>
  event parallel_for(range<1> r, K k, const std::vector<event> &deps = {}) const {
    depends_on(deps);
    if (r.size() == 0) return record();
    detail::device_guard g(dev_.cuda_ordinal());
    const int grid = grid_for(r.size());
    detail::range_kernel<K><<<grid, detail::kBlock, 0, cuda_stream()>>>(r.size(), k);
    detail::check_cuda(cudaGetLastError(), "parallel_for");
    return record();
  }

  // parallel_for(nd_range, kernel): kernel(nd_item<1>), one block per
  // work-group.
  template <class K>
  event parallel_for(nd_range<1> r, K k, const std::vector<event> &deps = {}) const {
    depends_on(deps);
    const size_t l = r.get_local_range().size(), gsz = r.get_global_range().size();
    if (l == 0 || l > 1024 || gsz % l) throw exception(B2P_ERR_INVALID_ARG, "nd_range: bad local size");
    if (gsz == 0) return record();
    detail::device_guard g(dev_.cuda_ordinal());
    detail::nd_range_kernel<K><<<(unsigned)(gsz / l), (unsigned)l, 0, cuda_stream()>>>(gsz, k);
    detail::check_cuda(cudaGetLastError(), "parallel_for(nd_range)");
    return record();
  }

  // parallel_for(range, reduction, kernel): kernel(id<1>, reducer&).
  template <class T, class Op, class K>
  event parallel_for(range<1> r, reduction_descriptor<T, Op> red, K k, const std::vector<event> &deps = {}) const {
    depends_on(deps);
    detail::device_guard g(dev_.cuda_ordinal());
    const size_t n = r.size();
    if constexpr (detail::library_reduction<T, Op>()) {
      if (red.has_identity && n > 0) {
        using P = detail::library_policy<T, Op>;
        detail::reduction_source<T, Op, K> src(k, n, red.op, red.identity);
        const size_t bytes = ::b2p::reduce_gen_scratch_bytes(n);
        void *s = scratch_->get(bytes, cuda_stream());
        // initialize_to_identity: *var = identity op r; otherwise op(*var, r)
        detail::check_b2p(::b2p::launch_reduce_gen<P>(src, n, red.var, red.init_to_identity ? &red.identity : nullptr,
                                                      s, scratch_->size(), cuda_stream()),
                          "parallel_for(reduction)");
        return record();
      }
    }
    const int grid = n ? grid_for(n) : 1;
    T *partial = nullptr;
    int *partial_has = nullptr;
    detail::check_cuda(cudaMallocAsync((void **)&partial, grid * sizeof(T), cuda_stream()), "reduction scratch");
    detail::check_cuda(cudaMallocAsync((void **)&partial_has, grid * sizeof(int), cuda_stream()),
                       "reduction scratch");
    detail::reduction_partials_kernel<T, Op, K><<<grid, detail::kBlock, 0, cuda_stream()>>>(
        n, k, red.op, red.identity, red.has_identity, partial, partial_has);
    detail::reduction_final_kernel<T, Op><<<1, 1, 0, cuda_stream()>>>(
        grid, red.op, partial, partial_has, red.var, red.init_to_identity, red.identity, red.has_identity);
    detail::check_cuda(cudaGetLastError(), "parallel_for(reduction)");
    cudaFreeAsync(partial, cuda_stream());
    cudaFreeAsync(partial_has, cuda_stream());
    return record();
  }

  template <class CGF>
  event submit(CGF cgf);

  static int grid_for(size_t n) {
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t need = (n + detail::kBlock - 1) / detail::kBlock;
    const size_t cap = (size_t)sms * 8;
    return (int)(need < cap ? (need ? need : 1) : cap);
  }

 private:
  device dev_;
  std::shared_ptr<CUstream_st> stream_;
  std::shared_ptr<detail::queue_scratch> scratch_;
  std::shared_ptr<detail::queue_scratch> work_;
};

// handler: the command-group form q.submit([&](handler& h) { ... }).
class handler {
 public:
  explicit handler(const queue &q) : q_(q) {}
  void depends_on(const event &e) { deps_.push_back(e); }
  void depends_on(const std::vector<event> &e) { deps_.insert(deps_.end(), e.begin(), e.end()); }
  template <class K>
  void parallel_for(range<1> r, K k) {
    ev_ = q_.parallel_for(r, k, deps_);
  }
  template <class K>
  void parallel_for(nd_range<1> r, K k) {
    ev_ = q_.parallel_for(r, k, deps_);
  }
  template <class T, class Op, class K>
  void parallel_for(range<1> r, reduction_descriptor<T, Op> red, K k) {
    ev_ = q_.parallel_for(r, red, k, deps_);
  }
  void memcpy(void *dst, const void *src, size_t bytes) { ev_ = q_.memcpy(dst, src, bytes, deps_); }
  event result() const { return ev_; }

 private:
  const queue &q_;
  std::vector<event> deps_;
  event ev_;
};

template <class CGF>
event queue::submit(CGF cgf) {
  handler h(*this);
  cgf(h);
  return h.result();
}

namespace detail {
inline int queue_device(const queue &q) { return q.get_device().cuda_ordinal(); }
}  // namespace detail

template <class T>
T *malloc_device(size_t count, const queue &q) {
  detail::device_guard g(q.get_device().cuda_ordinal());
  void *p = nullptr;
  detail::check_cuda(cudaMalloc(&p, count * sizeof(T)), "malloc_device");
  return static_cast<T *>(p);
}
template <class T>
T *malloc_shared(size_t count, const queue &q) {
  detail::device_guard g(q.get_device().cuda_ordinal());
  void *p = nullptr;
  detail::check_cuda(cudaMallocManaged(&p, count * sizeof(T)), "malloc_shared");
  return static_cast<T *>(p);
}
template <class T>
T *malloc_host(size_t count, const queue &q) {
  detail::device_guard g(q.get_device().cuda_ordinal());
  void *p = nullptr;
  detail::check_cuda(cudaMallocHost(&p, count * sizeof(T)), "malloc_host");
  return static_cast<T *>(p);
}
inline void free(void *p, const queue &q) {
  if (!p) return;
  detail::device_guard g(q.get_device().cuda_ordinal());
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost) cudaFreeHost(p);
  else cudaFree(p);
  cudaGetLastError();
}

}  // namespace b2p_sycl

#ifndef B2P_NO_SYCL_NAMESPACE
namespace sycl = b2p_sycl;
#endif
