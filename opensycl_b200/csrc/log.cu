// Call records, NVTX ranges, the checked mode and the selector choice of the
// C-ABI, all driven by the environment (read once per process):
//
//   B2P_LOG_LEVEL   0 none, 1 errors, 2 warnings (default), 3 one info line
//                   per call (operation, dtype, n, segments, configuration,
//                   status), 4 verbose: the call is also timed on its stream
//                   (the call waits for its work) and the line adds
//                   milliseconds and GB/s.  ACPP_DEBUG_LEVEL and
//                   HIPSYCL_DEBUG_LEVEL are read when B2P_LOG_LEVEL is not
//                   set, as the reference reads them
//                   (common/debug.hpp:14-21,61).  Lines go to stderr with a
//                   "[b2p error]" / "[b2p warning]" / "[b2p info]" /
//                   "[b2p verbose]" prefix.
//   B2P_CHECKED     1: every pointer argument's extent (elements x size) must
//                   lie inside one device allocation (cuMemGetAddressRange),
//                   and segment offsets are copied to the host and checked
//                   (non-decreasing, within the input); a failed check
//                   returns B2P_ERR_INVALID_PTR / B2P_ERR_INVALID_ARG before
//                   anything is launched.
//   B2P_SELECTOR    how B2P_CONFIG_AUTO picks a configuration: "learned"
//                   (default: the installed selector table, else the fixed
//                   heuristic), "heuristic" (always the fixed heuristic), or
//                   the path of a selector weights file, which is loaded and
//                   installed at the first AUTO call.
//
// Every C-ABI entry point that launches work opens an NVTX range named after
// it (b2p_reduce, b2p_scan, ...) for the duration of the host call, so
// profiler timelines show which library call issued which kernels.
#include <cuda.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace b2p {

namespace {

int env_int(const char *name, int fallback, bool *found = nullptr) {
  const char *e = getenv(name);
  if (found) *found = false;
  if (!e || !*e || strspn(e, "0123456789") != strlen(e)) return fallback;
  if (found) *found = true;
  return atoi(e);
}

std::atomic<int> g_level{-1};

const char *dtype_name(int dtype) {
  switch (dtype) {
  case B2P_I32: return "i32";
  case B2P_I64: return "i64";
  case B2P_U32: return "u32";
  case B2P_U64: return "u64";
  case B2P_F32: return "f32";
  case B2P_BF16: return "bf16";
  case B2P_F64: return "f64";
  default: return "?";
  }
}

thread_local int t_last_config = -1;

typedef CUresult (*AddressRangeFn)(CUdeviceptr *, size_t *, CUdeviceptr);

AddressRangeFn address_range_fn() {
  static AddressRangeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<AddressRangeFn>(f);
    cudaGetLastError();
  });
  return fn;
}

}  // namespace

int log_level() {
  int l = g_level.load(std::memory_order_relaxed);
  if (l >= 0) return l;
  bool found = false;
  l = env_int("B2P_LOG_LEVEL", 2, &found);
  if (!found) l = env_int("ACPP_DEBUG_LEVEL", 2, &found);
  if (!found) l = env_int("HIPSYCL_DEBUG_LEVEL", 2, &found);
  g_level.store(l, std::memory_order_relaxed);
  return l;
}

void set_log_level(int level) { g_level.store(level < 0 ? 0 : level, std::memory_order_relaxed); }

void log_line(int level, const char *fmt, ...) {
  if (level > log_level()) return;
  static const char *prefix[] = {"", "[b2p error] ", "[b2p warning] ", "[b2p info] ", "[b2p verbose] "};
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  fprintf(stderr, "%s%s\n", prefix[level < 1 ? 1 : (level > 4 ? 4 : level)], buf);
}

void note_config(int config) { t_last_config = config; }

bool checked_mode() {
  static const bool v = env_int("B2P_CHECKED", 0) != 0;
  return v;
}

int check_extent(const void *p, size_t bytes) {
  if (!checked_mode() || !p || bytes == 0) return B2P_OK;
  AddressRangeFn fn = address_range_fn();
  if (!fn) return B2P_OK;
  CUdeviceptr base = 0;
  size_t size = 0;
  if (fn(&base, &size, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) {
    // not a driver allocation (registered or managed host memory the driver
    // cannot size): nothing to check against
    cudaGetLastError();
    return B2P_OK;
  }
  const uintptr_t a = (uintptr_t)p, b0 = (uintptr_t)base;
  if (a < b0 || a - b0 > size || bytes > size - (a - b0)) {
    log_line(1, "checked mode: %zu bytes at %p run past the allocation [%p, +%zu)", bytes, p, (void *)base, size);
    return B2P_ERR_INVALID_PTR;
  }
  return B2P_OK;
}

int check_offsets(const int64_t *offsets, int64_t nseg, size_t total, cudaStream_t st) {
  if (!checked_mode()) return B2P_OK;
  std::vector<int64_t> h((size_t)nseg + 1);
  cudaError_t e = cudaMemcpyAsync(h.data(), offsets, h.size() * sizeof(int64_t), cudaMemcpyDefault, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e);
  for (int64_t i = 0; i <= nseg; ++i) {
    if (h[i] < 0 || (size_t)h[i] > total || (i > 0 && h[i] < h[i - 1])) {
      log_line(1, "checked mode: segment offset %lld = %lld is out of order or outside [0, %zu]", (long long)i,
               (long long)h[i], total);
      return B2P_ERR_INVALID_ARG;
    }
  }
  return B2P_OK;
}

int selector_mode() {
  // 0 learned (installed table, else heuristic), 1 heuristic only
  static const int mode = [] {
    const char *e = getenv("B2P_SELECTOR");
    if (!e || !*e || !strcmp(e, "learned")) return 0;
    if (!strcmp(e, "heuristic")) return 1;
    b2p_selector s = nullptr;
    int rc = b2p_selector_create(&s, 1);
    if (rc == B2P_OK) rc = b2p_selector_load(s, e);
    if (rc == B2P_OK) rc = b2p_selector_install(s);
    if (s) b2p_selector_destroy(s);
    if (rc != B2P_OK) log_line(2, "B2P_SELECTOR=%s: weights not installed (status %d); using the heuristic", e, rc);
    return 0;
  }();
  return mode;
}

CallScope::CallScope(const char *op, int dtype, size_t n, int64_t nseg, double bytes, b2p_stream stream)
    : op_(op), dtype_(dtype), n_(n), nseg_(nseg), bytes_(bytes), st_((cudaStream_t)stream) {
  nvtxRangePushA(op);
  t_last_config = -1;
  if (log_level() >= 4) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st_, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
        cudaEventCreate(&e0_) == cudaSuccess && cudaEventCreate(&e1_) == cudaSuccess &&
        cudaEventRecord(e0_, st_) == cudaSuccess) {
      timed_ = true;
    }
    cudaGetLastError();
  }
}

int CallScope::done(int status) {
  const int level = log_level();
  if (status != B2P_OK && level >= 1) {
    log_line(1, "%s dtype=%s n=%zu: status %d (%s)", op_, dtype_name(dtype_), n_, status, b2p_status_string(status));
  } else if (level >= 4 && timed_) {
    float ms = 0.f;
    if (cudaEventRecord(e1_, st_) == cudaSuccess && cudaEventSynchronize(e1_) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0_, e1_) == cudaSuccess) {
      log_line(4, "%s dtype=%s n=%zu nseg=%lld config=%d status=%d time=%.4f ms %.1f GB/s", op_, dtype_name(dtype_),
               n_, (long long)nseg_, t_last_config, status, ms, ms > 0 ? bytes_ / (ms * 1e6) : 0.0);
    }
    cudaGetLastError();
  } else if (level >= 3) {
    log_line(3, "%s dtype=%s n=%zu nseg=%lld config=%d status=%d", op_, dtype_name(dtype_), n_, (long long)nseg_,
             t_last_config, status);
  }
  return status;
}

void CallScope::set_size(size_t n, double bytes) {
  n_ = n;
  bytes_ = bytes;
}

CallScope::~CallScope() {
  if (e0_) cudaEventDestroy(e0_);
  if (e1_) cudaEventDestroy(e1_);
  nvtxRangePop();
}

}  // namespace b2p

extern "C" int b2p_log_level(void) { return b2p::log_level(); }

extern "C" void b2p_set_log_level(int level) { b2p::set_log_level(level); }
