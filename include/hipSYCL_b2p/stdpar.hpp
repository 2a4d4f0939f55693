// Offloaded C++ standard parallel algorithms on the primitive path:
// std::reduce (3 overloads), std::transform_reduce (3), std::inclusive_scan
// (3), std::exclusive_scan (2), std::transform_inclusive_scan (2),
// std::transform_exclusive_scan (1), std::copy_if, std::any_of / all_of
// / none_of, std::sort (2) and std::merge (2), taking the execution
// policy b2p_stdpar::par_unseq (AdaptiveCpp: the par_unseq overloads of
// std/stdpar/pstl-impl/numeric.hpp:28-576 and pstl-impl/algorithm.hpp:150-187,
// which its compiler pass substitutes for std::execution::par_unseq; here
// the caller names the policy).
//
// Each calling thread owns one in-order queue and one scratch cache
// (std/stdpar/detail/sycl_glue.hpp:60-189).  Ranges must be contiguous
// (pointers, std::vector / std::array iterators).  Device-accessible memory
// (device, managed, registered host) is used in place; pageable host memory
// is staged through device buffers from the cache (copied in, and for
// outputs copied back).  Every call here returns after its result is
// complete -- reduce/copy_if block in the reference too
// (std/stdpar/detail/offload.hpp:646-683); the scans do as well, because
// without the reference's compiler-inserted synchronisation the caller may
// read the output right away.  The offload decision is always "device"
// (there is no host fallback); the per-operation history the reference
// keeps for that decision (offload_heuristic_db.hpp:232-365) is recorded
// and can be read with b2p_stdpar::offload_history().
//
// Offload front (offload.hpp:165-238, detail/stdpar_builtins.hpp:17-37):
// managed (shared-USM) ranges are prefetched to the GPU on the call's stream
// before the kernel; the policy b2p_stdpar::par_unseq_async leaves scans
// non-blocking, as the reference's are, when no range needs staging.
// Consecutive non-blocking calls form one batch: the thread's queue stream
// records them into a CUDA graph (stream capture) instead of launching them,
// and the batch is finalised -- the graph launched once -- at
// b2p_stdpar::sync(), the barrier the reference's compiler inserts before
// host code reads the results, or at the next blocking call, which must run
// after the batch (the reference counts outstanding operations and
// finalises its batch at that barrier: stdpar_builtins.hpp:17-37,
// detail/sycl_glue.hpp:120-139, offload.hpp:597-683).  A batch of the same
// shape as the previous one updates the previous executable graph instead
// of instantiating a new one.  Ranges of calls inside a batch are not
// prefetched (the hint is not part of the graph).  reduce,
// transform_reduce, copy_if and any/all/none_of return values and always
// block; sort and merge block too (pstl-impl/algorithm.hpp:506-606).
#pragma once

#include "algorithms.hpp"

#include <chrono>
#include <map>
#include <string>
#include <vector>

namespace b2p_stdpar {

struct par_unseq_policy {
  bool nonblocking_scans = false;
};
inline constexpr par_unseq_policy par_unseq{};
// par_unseq whose scans return without waiting (see b2p_stdpar::sync)
inline constexpr par_unseq_policy par_unseq_async{true};

struct offload_record {
  std::string op;
  size_t n;
  double seconds;
};

namespace detail {

namespace alg = ::hipsycl::algorithms;

struct tls_runtime {
  b2p_sycl::queue q;
  alg::util::allocation_cache cache{alg::util::allocation_type::device};
  std::vector<offload_record> history;
  // the open batch of non-blocking calls (stream capture of q's stream)
  bool capturing = false;
  size_t batch_calls = 0;
  cudaGraphExec_t exec = nullptr;
  size_t graph_launches = 0, batched_calls = 0;

  static tls_runtime &get() {
    thread_local tls_runtime rt;
    return rt;
  }
  ~tls_runtime() {
    try {
      flush();
    } catch (...) {
    }
    if (exec) cudaGraphExecDestroy(exec);
    cudaGetLastError();
  }
  // Start recording the thread's calls into a batch (if none is open).
  void begin_batch() {
    if (capturing) return;
    b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
    b2p_sycl::detail::check_cuda(cudaStreamBeginCapture(q.cuda_stream(), cudaStreamCaptureModeRelaxed),
                                 "stdpar batch: begin capture");
    capturing = true;
    batch_calls = 0;
  }
  // Finalise the open batch: end the capture and launch its graph once on
  // the queue (asynchronously).  Nothing to do without an open batch.
  void flush() {
    if (!capturing) return;
    capturing = false;
    b2p_sycl::detail::device_guard g(q.get_device().cuda_ordinal());
    cudaGraph_t graph = nullptr;
    b2p_sycl::detail::check_cuda(cudaStreamEndCapture(q.cuda_stream(), &graph), "stdpar batch: end capture");
    if (batch_calls > 0 && graph) {
      if (exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(exec, graph, &info) != cudaSuccess) {
          cudaGetLastError();
          cudaGraphExecDestroy(exec);
          exec = nullptr;
        }
      }
      cudaError_t e = exec ? cudaSuccess : cudaGraphInstantiate(&exec, graph, 0);
      if (e == cudaSuccess) e = cudaGraphLaunch(exec, q.cuda_stream());
      cudaGraphDestroy(graph);
      b2p_sycl::detail::check_cuda(e, "stdpar batch: launch");
      ++graph_launches;
      batched_calls += batch_calls;
    } else if (graph) {
      cudaGraphDestroy(graph);
    }
    batch_calls = 0;
  }
};

template <class It>
auto raw(It it) {
  return &*it;
}

inline bool is_managed(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged;
}

// A device view of a contiguous range: the original pointer when the GPU
// can reach it, otherwise a staged device copy (copied back by copy_back()).
template <class T>
class view {
 public:
  view(alg::util::allocation_group &g, tls_runtime &rt, T *p, size_t n, bool copy_in)
      : host_(p), n_(n), rt_(rt) {
    if (alg::detail::device_accessible(p)) {
      dev_ = p;
      if (n && !rt.capturing && is_managed(p)) {  // pages move to the GPU ahead of the kernel
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaMemPrefetchAsync(p, n * sizeof(T), dev, rt.q.cuda_stream()) != cudaSuccess) cudaGetLastError();
      }
    } else {
      dev_ = g.obtain<std::remove_cv_t<T>>(n ? n : 1);
      if (copy_in && n)
        rt.q.memcpy(const_cast<std::remove_cv_t<T> *>(dev_), p, n * sizeof(T));
    }
  }
  T *get() const { return dev_; }
  bool staged() const { return dev_ != host_; }
  void copy_back(size_t count) {
    if (dev_ != host_ && count) rt_.q.memcpy(const_cast<std::remove_cv_t<T> *>(host_), dev_, count * sizeof(T));
  }

 private:
  T *host_;
  T *dev_ = nullptr;
  size_t n_;
  tls_runtime &rt_;
};

class timer {
 public:
  timer(const char *op, size_t n) : op_(op), n_(n), t0_(std::chrono::steady_clock::now()) {}
  ~timer() {
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    tls_runtime::get().history.push_back({op_, n_, s});
  }

 private:
  const char *op_;
  size_t n_;
  std::chrono::steady_clock::time_point t0_;
};

template <class T, class F>
T reduce_impl(const char *name, size_t n, F &&launch) {
  timer tm(name, n);
  auto &rt = tls_runtime::get();
  rt.flush();  // after the calls of the open batch
  alg::util::allocation_group g(&rt.cache, rt.q.get_device());
  T *d_out = g.obtain<T>(1);
  launch(g, rt, d_out);
  T r;
  rt.q.memcpy(&r, d_out, sizeof(T));
  rt.q.wait();
  return r;
}

}  // namespace detail

// Offload history of the calling thread: operation, size, seconds (for
// non-blocking scans, the time to enqueue).
inline const std::vector<offload_record> &offload_history() { return detail::tls_runtime::get().history; }

// Finalise the open batch and wait for every call this thread has
// offloaded (the barrier before host code reads the results of
// par_unseq_async scans).
inline void sync() {
  auto &rt = detail::tls_runtime::get();
  rt.flush();
  rt.q.wait();
}

// Batches of non-blocking calls finalised so far on this thread: graphs
// launched, and calls they held.
struct batch_stats_t {
  size_t graph_launches;
  size_t batched_calls;
};
inline batch_stats_t batch_stats() {
  auto &rt = detail::tls_runtime::get();
  return {rt.graph_launches, rt.batched_calls};
}

}  // namespace b2p_stdpar

namespace std {

// ----------------------------------------------------------------- reduce

template <class ForwardIt, class T, class BinaryOp>
T reduce(const b2p_stdpar::par_unseq_policy &, ForwardIt first, ForwardIt last, T init, BinaryOp op) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return init;
  return d::reduce_impl<T>("reduce", n, [&](auto &g, auto &rt, T *out) {
    using V = typename std::iterator_traits<ForwardIt>::value_type;
    d::view<const V> in(g, rt, d::raw(first), n, true);
    hipsycl::algorithms::reduce(rt.q, g, in.get(), in.get() + n, out, init, op);
  });
}

template <class ForwardIt, class T>
T reduce(const b2p_stdpar::par_unseq_policy &p, ForwardIt first, ForwardIt last, T init) {
  return std::reduce(p, first, last, init, std::plus<>{});
}

template <class ForwardIt>
typename std::iterator_traits<ForwardIt>::value_type reduce(const b2p_stdpar::par_unseq_policy &p, ForwardIt first,
                                                             ForwardIt last) {
  using V = typename std::iterator_traits<ForwardIt>::value_type;
  return std::reduce(p, first, last, V{}, std::plus<>{});
}

// ------------------------------------------------------- transform_reduce

template <class ForwardIt1, class ForwardIt2, class T, class BinaryReductionOp, class BinaryTransformOp>
T transform_reduce(const b2p_stdpar::par_unseq_policy &, ForwardIt1 first1, ForwardIt1 last1, ForwardIt2 first2,
                   T init, BinaryReductionOp reduce, BinaryTransformOp transform) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first1, last1);
  if (n == 0) return init;
  return d::reduce_impl<T>("transform_reduce", n, [&](auto &g, auto &rt, T *out) {
    using V1 = typename std::iterator_traits<ForwardIt1>::value_type;
    using V2 = typename std::iterator_traits<ForwardIt2>::value_type;
    d::view<const V1> a(g, rt, d::raw(first1), n, true);
    d::view<const V2> b(g, rt, d::raw(first2), n, true);
    hipsycl::algorithms::transform_reduce(rt.q, g, a.get(), a.get() + n, b.get(), out, init, reduce, transform);
  });
}

template <class ForwardIt1, class ForwardIt2, class T>
T transform_reduce(const b2p_stdpar::par_unseq_policy &p, ForwardIt1 first1, ForwardIt1 last1, ForwardIt2 first2,
                   T init) {
  return std::transform_reduce(p, first1, last1, first2, init, std::plus<T>{}, std::multiplies<T>{});
}

template <class ForwardIt, class T, class BinaryReductionOp, class UnaryTransformOp>
T transform_reduce(const b2p_stdpar::par_unseq_policy &, ForwardIt first, ForwardIt last, T init,
                   BinaryReductionOp reduce, UnaryTransformOp transform) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return init;
  return d::reduce_impl<T>("transform_reduce", n, [&](auto &g, auto &rt, T *out) {
    using V = typename std::iterator_traits<ForwardIt>::value_type;
    d::view<const V> in(g, rt, d::raw(first), n, true);
    hipsycl::algorithms::transform_reduce(rt.q, g, in.get(), in.get() + n, out, init, reduce, transform);
  });
}

// ------------------------------------------------------------------ scans

namespace b2p_stdpar_detail {
template <bool INCL, class InputIt, class OutputIt, class Run>
OutputIt scan_call(const b2p_stdpar::par_unseq_policy &pol, const char *name, InputIt first, InputIt last,
                   OutputIt d_first, Run run) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return d_first;
  d::timer tm(name, n);
  auto &rt = d::tls_runtime::get();
  // a non-blocking scan over ranges the GPU reaches joins the open batch;
  // any other call finalises it first
  const bool batch = pol.nonblocking_scans && hipsycl::algorithms::detail::device_accessible(d::raw(first)) &&
                     hipsycl::algorithms::detail::device_accessible(d::raw(d_first));
  if (batch) rt.begin_batch();
  else rt.flush();
  hipsycl::algorithms::util::allocation_group g(&rt.cache, rt.q.get_device());
  using V = typename std::iterator_traits<InputIt>::value_type;
  using O = std::remove_reference_t<decltype(*d_first)>;
  d::view<const V> in(g, rt, d::raw(first), n, true);
  d::view<O> out(g, rt, d::raw(d_first), n, false);
  if (batch) {
    try {
      run(rt.q, g, in.get(), in.get() + n, out.get());
    } catch (...) {
      rt.batch_calls = 0;
      try {
        rt.flush();  // ends the failed capture and drops its graph
      } catch (...) {
      }
      throw;
    }
    ++rt.batch_calls;
    return d_first + n;
  }
  run(rt.q, g, in.get(), in.get() + n, out.get());
  out.copy_back(n);
  rt.q.wait();
  return d_first + n;
}
}  // namespace b2p_stdpar_detail

template <class InputIt, class OutputIt>
OutputIt inclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last, OutputIt d_first) {
  return b2p_stdpar_detail::scan_call<true>(pol, "inclusive_scan", first, last, d_first, [](auto &q, auto &g, auto a,
                                                                                        auto b, auto o) {
    hipsycl::algorithms::inclusive_scan(q, g, a, b, o);
  });
}

template <class InputIt, class OutputIt, class BinaryOp>
OutputIt inclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last, OutputIt d_first,
                        BinaryOp op) {
  return b2p_stdpar_detail::scan_call<true>(pol, "inclusive_scan", first, last, d_first, [op](auto &q, auto &g, auto a,
                                                                                          auto b, auto o) {
    hipsycl::algorithms::inclusive_scan(q, g, a, b, o, op);
  });
}

template <class InputIt, class OutputIt, class BinaryOp, class T>
OutputIt inclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last, OutputIt d_first,
                        BinaryOp op, T init) {
  return b2p_stdpar_detail::scan_call<true>(pol, "inclusive_scan", first, last, d_first,
                                            [op, init](auto &q, auto &g, auto a, auto b, auto o) {
                                              hipsycl::algorithms::inclusive_scan(q, g, a, b, o, op, init);
                                            });
}

template <class InputIt, class OutputIt, class T, class BinaryOp>
OutputIt exclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last, OutputIt d_first, T init,
                        BinaryOp op) {
  return b2p_stdpar_detail::scan_call<false>(pol, "exclusive_scan", first, last, d_first,
                                             [op, init](auto &q, auto &g, auto a, auto b, auto o) {
                                               hipsycl::algorithms::exclusive_scan(q, g, a, b, o, init, op);
                                             });
}

template <class InputIt, class OutputIt, class T>
OutputIt exclusive_scan(const b2p_stdpar::par_unseq_policy &p, InputIt first, InputIt last, OutputIt d_first,
                        T init) {
  return std::exclusive_scan(p, first, last, d_first, init, std::plus<>{});
}

// ------------------------------------------------------- transform scans
// (pstl-impl/numeric.hpp:469-576).  User operators without a known identity
// go through the generic kernels, which carry (value, present) pairs.

template <class InputIt, class OutputIt, class BinaryOp, class UnaryOp>
OutputIt transform_inclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last,
                                  OutputIt d_first, BinaryOp binary_op, UnaryOp unary_op) {
  return b2p_stdpar_detail::scan_call<true>(pol, "transform_inclusive_scan", first, last, d_first,
                                            [binary_op, unary_op](auto &q, auto &g, auto a, auto b, auto o) {
                                              hipsycl::algorithms::transform_inclusive_scan(q, g, a, b, o, binary_op,
                                                                                            unary_op);
                                            });
}

template <class InputIt, class OutputIt, class BinaryOp, class UnaryOp, class T>
OutputIt transform_inclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last,
                                  OutputIt d_first, BinaryOp binary_op, UnaryOp unary_op, T init) {
  return b2p_stdpar_detail::scan_call<true>(pol, "transform_inclusive_scan", first, last, d_first,
                                            [binary_op, unary_op, init](auto &q, auto &g, auto a, auto b, auto o) {
                                              hipsycl::algorithms::transform_inclusive_scan(q, g, a, b, o, binary_op,
                                                                                            unary_op, init);
                                            });
}

template <class InputIt, class OutputIt, class T, class BinaryOp, class UnaryOp>
OutputIt transform_exclusive_scan(const b2p_stdpar::par_unseq_policy &pol, InputIt first, InputIt last,
                                  OutputIt d_first, T init, BinaryOp binary_op, UnaryOp unary_op) {
  return b2p_stdpar_detail::scan_call<false>(pol, "transform_exclusive_scan", first, last, d_first,
                                             [binary_op, unary_op, init](auto &q, auto &g, auto a, auto b, auto o) {
                                               hipsycl::algorithms::transform_exclusive_scan(q, g, a, b, o, init,
                                                                                             binary_op, unary_op);
                                             });
}

// ----------------------------------------------------- any / all / none
// (pstl-impl/algorithm.hpp:403-500): blocking, empty ranges give the
// standard answers without a launch.

namespace b2p_stdpar_detail {
template <class ForwardIt, class Call>
bool flag_call(const char *name, ForwardIt first, ForwardIt last, bool empty_answer, Call call) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return empty_answer;
  d::timer tm(name, n);
  auto &rt = d::tls_runtime::get();
  rt.flush();
  hipsycl::algorithms::util::allocation_group g(&rt.cache, rt.q.get_device());
  using V = typename std::iterator_traits<ForwardIt>::value_type;
  d::view<const V> in(g, rt, d::raw(first), n, true);
  int *flag = g.obtain<int>(1);
  call(rt.q, in.get(), in.get() + n, flag);
  int r = 0;
  rt.q.memcpy(&r, flag, sizeof(int));
  rt.q.wait();
  return r != 0;
}
}  // namespace b2p_stdpar_detail

template <class ForwardIt, class UnaryPredicate>
bool any_of(const b2p_stdpar::par_unseq_policy &, ForwardIt first, ForwardIt last, UnaryPredicate p) {
  return b2p_stdpar_detail::flag_call("any_of", first, last, false, [p](auto &q, auto a, auto b, int *f) {
    hipsycl::algorithms::any_of(q, a, b, f, p);
  });
}

template <class ForwardIt, class UnaryPredicate>
bool all_of(const b2p_stdpar::par_unseq_policy &, ForwardIt first, ForwardIt last, UnaryPredicate p) {
  return b2p_stdpar_detail::flag_call("all_of", first, last, true, [p](auto &q, auto a, auto b, int *f) {
    hipsycl::algorithms::all_of(q, a, b, f, p);
  });
}

template <class ForwardIt, class UnaryPredicate>
bool none_of(const b2p_stdpar::par_unseq_policy &, ForwardIt first, ForwardIt last, UnaryPredicate p) {
  return b2p_stdpar_detail::flag_call("none_of", first, last, true, [p](auto &q, auto a, auto b, int *f) {
    hipsycl::algorithms::none_of(q, a, b, f, p);
  });
}

// ---------------------------------------------------------------- copy_if

template <class ForwardIt1, class ForwardIt2, class UnaryPredicate>
ForwardIt2 copy_if(const b2p_stdpar::par_unseq_policy &, ForwardIt1 first, ForwardIt1 last, ForwardIt2 d_first,
                   UnaryPredicate pred) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return d_first;
  d::timer tm("copy_if", n);
  auto &rt = d::tls_runtime::get();
  rt.flush();
  hipsycl::algorithms::util::allocation_group g(&rt.cache, rt.q.get_device());
  using V = typename std::iterator_traits<ForwardIt1>::value_type;
  using O = std::remove_reference_t<decltype(*d_first)>;
  d::view<const V> in(g, rt, d::raw(first), n, true);
  d::view<O> out(g, rt, d::raw(d_first), n, false);
  size_t *d_count = g.obtain<size_t>(1);
  hipsycl::algorithms::copy_if(rt.q, g, in.get(), in.get() + n, out.get(), pred, d_count);
  size_t count = 0;
  rt.q.memcpy(&count, d_count, sizeof(size_t));
  rt.q.wait();
  out.copy_back(count);
  rt.q.wait();
  return d_first + count;
}

// ------------------------------------------------------------ sort / merge

template <class RandomIt, class Compare>
void sort(const b2p_stdpar::par_unseq_policy &, RandomIt first, RandomIt last, Compare comp) {
  namespace d = b2p_stdpar::detail;
  const size_t n = (size_t)std::distance(first, last);
  if (n == 0) return;
  d::timer tm("sort", n);
  auto &rt = d::tls_runtime::get();
  rt.flush();
  hipsycl::algorithms::util::allocation_group g(&rt.cache, rt.q.get_device());
  using V = typename std::iterator_traits<RandomIt>::value_type;
  d::view<V> keys(g, rt, d::raw(first), n, true);
  hipsycl::algorithms::sort(rt.q, keys.get(), keys.get() + n, comp);
  keys.copy_back(n);
  rt.q.wait();
}

template <class RandomIt>
void sort(const b2p_stdpar::par_unseq_policy &p, RandomIt first, RandomIt last) {
  std::sort(p, first, last, std::less<>{});
}

template <class ForwardIt1, class ForwardIt2, class ForwardIt3, class Compare>
ForwardIt3 merge(const b2p_stdpar::par_unseq_policy &, ForwardIt1 first1, ForwardIt1 last1, ForwardIt2 first2,
                 ForwardIt2 last2, ForwardIt3 d_first, Compare comp) {
  namespace d = b2p_stdpar::detail;
  const size_t n1 = (size_t)std::distance(first1, last1), n2 = (size_t)std::distance(first2, last2);
  if (n1 + n2 == 0) return d_first;
  d::timer tm("merge", n1 + n2);
  auto &rt = d::tls_runtime::get();
  rt.flush();
  hipsycl::algorithms::util::allocation_group g(&rt.cache, rt.q.get_device());
  using V1 = typename std::iterator_traits<ForwardIt1>::value_type;
  using V2 = typename std::iterator_traits<ForwardIt2>::value_type;
  using O = std::remove_reference_t<decltype(*d_first)>;
  // an empty range may come with no element to take the address of
  d::view<const V1> a(g, rt, n1 ? d::raw(first1) : nullptr, n1, true);
  d::view<const V2> b(g, rt, n2 ? d::raw(first2) : nullptr, n2, true);
  d::view<O> out(g, rt, d::raw(d_first), n1 + n2, false);
  hipsycl::algorithms::merge(rt.q, g, a.get(), a.get() + n1, b.get(), b.get() + n2, out.get(), comp);
  out.copy_back(n1 + n2);
  rt.q.wait();
  return d_first + (n1 + n2);
}

template <class ForwardIt1, class ForwardIt2, class ForwardIt3>
ForwardIt3 merge(const b2p_stdpar::par_unseq_policy &p, ForwardIt1 first1, ForwardIt1 last1, ForwardIt2 first2,
                 ForwardIt2 last2, ForwardIt3 d_first) {
  return std::merge(p, first1, last1, first2, last2, d_first, std::less<>{});
}

}  // namespace std
