// extern "C" entry points of libb2p (declared in include/b2p.h): argument
// and pointer validation, configuration resolution, and dispatch to the
// kernel launchers.  Also the per-device caches (SM count, occupancy,
// shared-memory attributes) the launchers use.
#include "b2p_device/common.cuh"
#include "internal.h"

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

namespace b2p {

namespace {
constexpr int kMaxDevices = 64;
DeviceInfo g_dev[kMaxDevices];
std::once_flag g_dev_once[kMaxDevices];
std::mutex g_cache_mu;
std::map<std::tuple<int, const void *, int, size_t>, int> g_occ;
std::map<std::pair<int, const void *>, size_t> g_smem_attr;
std::atomic<uint64_t> g_timeout_ns{2000000000ull};
std::atomic<long long> g_stall_tile{-1};
int g_pageable_ok[kMaxDevices] = {0};
}  // namespace

const DeviceInfo &device_info() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
  std::call_once(g_dev_once[dev], [dev] {
    DeviceInfo &d = g_dev[dev];
    d.device = dev;
    cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&d.cc_major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&d.cc_minor, cudaDevAttrComputeCapabilityMinor, dev);
    cudaDeviceGetAttribute(&g_pageable_ok[dev], cudaDevAttrPageableMemoryAccess, dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
      snprintf(d.name, sizeof(d.name), "%s", prop.name);
    if (d.sm_count <= 0) d.sm_count = 148;
  });
  return g_dev[dev];
}

int occupancy(const void *kernel, int block, size_t smem) {
  const int dev = device_info().device;
  auto key = std::make_tuple(dev, kernel, block, smem);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) return it->second;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, smem) != cudaSuccess) {
    cudaGetLastError();
    nb = 1;
  }
  if (nb < 1) nb = 1;
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_occ[key] = nb;
  return nb;
}

int ensure_dynamic_smem(const void *kernel, size_t bytes) {
  if (bytes == 0) return B2P_OK;  // static + dynamic may exceed the default even below 48 KB
  const int dev = device_info().device;
  auto key = std::make_pair(dev, kernel);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_smem_attr.find(key);
    if (it != g_smem_attr.end() && it->second >= bytes) return B2P_OK;
  }
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return cuda_status(e);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  size_t &cur = g_smem_attr[key];
  if (bytes > cur) cur = bytes;
  return B2P_OK;
}

int grid_for(int grid_mode, long long units, int units_per_block, const void *kernel, int block,
             size_t smem) {
  long long need = (units + units_per_block - 1) / units_per_block;
  if (need < 1) need = 1;
  if (grid_mode == 0) return (int)std::min<long long>(need, 0x7fffffffLL);
  const int sms = device_info().sm_count;
  int occ = occupancy(kernel, block, smem);
  if (grid_mode == 2) occ = std::max(1, occ / 2);
  return (int)std::min<long long>(need, (long long)sms * occ);
}

uint64_t wait_timeout_ns() { return g_timeout_ns.load(); }
long long debug_stall_tile() { return g_stall_tile.load(); }

int cuda_status(cudaError_t e) { return e == cudaSuccess ? B2P_OK : B2P_ERR_CUDA; }

// Device-accessibility check, mirroring the reference's stdpar pointer
// validation (std/stdpar/detail/offload.hpp:101-123) but rejecting instead
// of falling back to the host.
int check_pointer(const void *p, size_t align);
static int check_ptr(const void *p, size_t align) { return check_pointer(p, align); }
int check_pointer(const void *p, size_t align) {
  if (!p) return B2P_ERR_INVALID_PTR;
  if (reinterpret_cast<uintptr_t>(p) % align) return B2P_ERR_INVALID_PTR;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return B2P_ERR_INVALID_PTR;
  }
  const int dev = device_info().device;
  switch (a.type) {
  case cudaMemoryTypeDevice:
    return a.device == dev ? B2P_OK : B2P_ERR_INVALID_PTR;
  case cudaMemoryTypeManaged:
    return B2P_OK;
  case cudaMemoryTypeHost:
    return a.devicePointer == p ? B2P_OK : B2P_ERR_INVALID_PTR;
  default:
    return g_pageable_ok[dev] ? B2P_OK : B2P_ERR_INVALID_PTR;
  }
}

static int check_device() {
  const DeviceInfo &d = device_info();
  if (d.cc_major < 10) return B2P_ERR_NO_DEVICE;
  return B2P_OK;
}

static bool valid_dtype(int dt) { return dt >= B2P_I32 && dt <= B2P_F64; }
static bool valid_op(int dtype, int op) {
  if (op < B2P_SUM || op > B2P_XOR) return false;
  if (dtype_is_float(dtype) && op > B2P_MAX) return false;
  return true;
}

bool config_valid(int prim, int dtype, int config) {
  if (config < 0 || config >= B2P_NUM_CONFIGS) return false;
  switch (prim) {
  case B2P_PRIM_REDUCE:
  case B2P_PRIM_DOT:
  case B2P_PRIM_HISTOGRAM:
    return true;
  case B2P_PRIM_SCAN:
    return scan_config_valid(dtype, config);
  case B2P_PRIM_COPY_IF:
    return copy_if_config_valid(dtype, config);
  case B2P_PRIM_SEG_REDUCE:
  case B2P_PRIM_SEG_SCAN:
    return segmented_config_valid(dtype, config);
  default:
    return false;
  }
}

int validate_reduce(int dtype, int op, const void *in, size_t n, const void *out) {
  if (!valid_dtype(dtype) || !valid_op(dtype, op)) return B2P_ERR_INVALID_ARG;
  if (n == 0) return B2P_OK;
  int rc = check_device();
  if (rc) return rc;
  if ((rc = check_ptr(in, dtype_size(dtype))) || (rc = check_ptr(out, acc_size(dtype)))) return rc;
  return B2P_OK;
}

static int resolve(int prim, int dtype, size_t n, int64_t nseg, int config) {
  if (config == B2P_CONFIG_AUTO) config = b2p_auto_config(prim, dtype, n, nseg, 0.0);
  note_config(config);
  return config;
}

}  // namespace b2p

using namespace b2p;

extern "C" {

const char *b2p_version(void) { return "0.1.0 sm_100a"; }

const char *b2p_status_string(int s) {
  switch (s) {
  case B2P_OK: return "ok";
  case B2P_ERR_INVALID_ARG: return "invalid argument";
  case B2P_ERR_INVALID_PTR: return "pointer is not device-accessible or misaligned";
  case B2P_ERR_TIMEOUT: return "device-side wait timed out";
  case B2P_ERR_CUDA: return "CUDA runtime error";
  case B2P_ERR_UNSUPPORTED: return "dtype/op combination not supported";
  case B2P_ERR_SCRATCH: return "scratch buffer missing, too small or misaligned";
  case B2P_ERR_NO_DEVICE: return "no sm_100 CUDA device";
  case B2P_ERR_IO: return "file could not be read or does not match";
  default: return "unknown status";
  }
}

int b2p_config_describe(int config, int *block, int *items, int *grid_mode) {
  if (config < 0 || config >= B2P_NUM_CONFIGS) return B2P_ERR_INVALID_ARG;
  LaunchConfig lc = describe_config(config);
  if (block) *block = lc.block;
  if (items) *items = lc.items;
  if (grid_mode) *grid_mode = lc.grid_mode;
  return B2P_OK;
}

int b2p_config_valid(int prim, int dtype, int config) {
  return config_valid(prim, dtype, config) ? 1 : 0;
}

size_t b2p_scratch_bytes(int prim, int dtype, size_t n, int64_t nseg, int config) {
  if (!valid_dtype(dtype)) return 0;
  switch (prim) {
  case B2P_PRIM_REDUCE:
  case B2P_PRIM_DOT:
    return reduce_scratch_bytes(dtype, n, nullptr, nullptr);
  case B2P_PRIM_SCAN:
    return scan_scratch_bytes(dtype, n, config);
  case B2P_PRIM_COPY_IF:
    return copy_if_scratch_bytes(dtype, n, config);
  case B2P_PRIM_HISTOGRAM:
    return kScratchPrefix;
  case B2P_PRIM_SEG_REDUCE:
  case B2P_PRIM_SEG_SCAN:
    return segmented_scratch_bytes(dtype, n, nseg, config);
  case B2P_PRIM_SORT:
  case B2P_PRIM_MERGE:
    return merge_sort_scratch_bytes(prim, dtype, n);
  default:
    return 0;
  }
}

int b2p_scratch_init(void *scratch, size_t bytes, b2p_stream stream) {
  if (!scratch) return B2P_ERR_SCRATCH;
  return cuda_status(cudaMemsetAsync(scratch, 0, bytes, (cudaStream_t)stream));
}

static int reduce_entry(int dtype, int op, const void *in, size_t n, void *out, const void *init,
               void *scratch, size_t scratch_bytes, int config, b2p_stream stream) {
  int rc = validate_reduce(dtype, op, in, n, out);
  if (rc || n == 0) return rc;
  if ((rc = check_extent(in, n * dtype_size(dtype))) || (rc = check_extent(out, acc_size(dtype)))) return rc;
  if (!scratch) return B2P_ERR_SCRATCH;
  config = resolve(B2P_PRIM_REDUCE, dtype, n, 0, config);
  if (!config_valid(B2P_PRIM_REDUCE, dtype, config)) return B2P_ERR_INVALID_ARG;
  return launch_reduce(dtype, op, in, nullptr, n, out, init, scratch, scratch_bytes, config,
                       (cudaStream_t)stream);
}

int b2p_reduce(int dtype, int op, const void *in, size_t n, void *out, const void *init,
               void *scratch, size_t scratch_bytes, int config, b2p_stream stream) {
  CallScope cs("b2p_reduce", dtype, n, 0, (double)n * dtype_size(dtype), stream);
  return cs.done(reduce_entry(dtype, op, in, n, out, init, scratch, scratch_bytes, config, stream));
}

static int dot_entry(int dtype, const void *a, const void *b, size_t n, void *out, const void *init,
            void *scratch, size_t scratch_bytes, int config, b2p_stream stream) {
  if (dtype != B2P_F32 && dtype != B2P_BF16 && dtype != B2P_F64) return B2P_ERR_UNSUPPORTED;
  if (n == 0) return B2P_OK;
  int rc = check_device();
  if (rc) return rc;
  if ((rc = check_ptr(a, dtype_size(dtype))) || (rc = check_ptr(b, dtype_size(dtype))) ||
      (rc = check_ptr(out, acc_size(dtype))))
    return rc;
  if ((rc = check_extent(a, n * dtype_size(dtype))) || (rc = check_extent(b, n * dtype_size(dtype))) ||
      (rc = check_extent(out, acc_size(dtype))))
    return rc;
  if (!scratch) return B2P_ERR_SCRATCH;
  config = resolve(B2P_PRIM_DOT, dtype, n, 0, config);
  if (!config_valid(B2P_PRIM_DOT, dtype, config)) return B2P_ERR_INVALID_ARG;
  if (scratch_bytes < reduce_scratch_bytes(dtype, n, a, b)) return B2P_ERR_SCRATCH;
  return launch_reduce(dtype, B2P_SUM, a, b, n, out, init, scratch, scratch_bytes, config,
                       (cudaStream_t)stream);
}

int b2p_dot(int dtype, const void *a, const void *b, size_t n, void *out, const void *init,
            void *scratch, size_t scratch_bytes, int config, b2p_stream stream) {
  CallScope cs("b2p_dot", dtype, n, 0, 2.0 * n * dtype_size(dtype), stream);
  return cs.done(dot_entry(dtype, a, b, n, out, init, scratch, scratch_bytes, config, stream));
}

static int scan_entry(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
             const void *init, void *scratch, size_t scratch_bytes, int config,
             b2p_stream stream) {
  if (!valid_dtype(dtype) || !valid_op(dtype, op)) return B2P_ERR_INVALID_ARG;
  if (!inclusive && !init) return B2P_ERR_INVALID_ARG;
  if (n == 0) return B2P_OK;
  int rc = check_device();
  if (rc) return rc;
  if ((rc = check_ptr(in, dtype_size(dtype))) || (rc = check_ptr(out, acc_size(dtype)))) return rc;
  if ((rc = check_extent(in, n * dtype_size(dtype))) || (rc = check_extent(out, n * acc_size(dtype)))) return rc;
  if (!scratch) return B2P_ERR_SCRATCH;
  config = resolve(B2P_PRIM_SCAN, dtype, n, 0, config);
  if (!config_valid(B2P_PRIM_SCAN, dtype, config)) return B2P_ERR_INVALID_ARG;
  return launch_scan(dtype, op, inclusive, in, out, n, init, scratch, scratch_bytes, config,
                     (cudaStream_t)stream);
}

int b2p_scan(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
             const void *init, void *scratch, size_t scratch_bytes, int config,
             b2p_stream stream) {
  CallScope cs("b2p_scan", dtype, n, 0, (double)n * (dtype_size(dtype) + acc_size(dtype)), stream);
  return cs.done(scan_entry(dtype, op, inclusive, in, out, n, init, scratch, scratch_bytes, config, stream));
}

static int copy_if_entry(int dtype, const void *in, void *out, size_t n, uint64_t mask, int cmp,
                uint64_t rhs, uint64_t *num_copied, void *scratch, size_t scratch_bytes,
                int config, b2p_stream stream) {
  if (!valid_dtype(dtype) || dtype == B2P_BF16) return B2P_ERR_UNSUPPORTED;
  if (cmp < B2P_CMP_LT || cmp > B2P_CMP_GT) return B2P_ERR_INVALID_ARG;
  int rc = check_device();
  if (rc) return rc;
  if (num_copied && (rc = check_ptr(num_copied, 8))) return rc;
  if (n == 0) {
    if (num_copied)
      return cuda_status(cudaMemsetAsync(num_copied, 0, sizeof(uint64_t), (cudaStream_t)stream));
    return B2P_OK;
  }
  if ((rc = check_ptr(in, dtype_size(dtype))) || (rc = check_ptr(out, dtype_size(dtype)))) return rc;
  // the output must hold every element (all may be kept)
  if ((rc = check_extent(in, n * dtype_size(dtype))) || (rc = check_extent(out, n * dtype_size(dtype)))) return rc;
  if (!scratch) return B2P_ERR_SCRATCH;
  config = resolve(B2P_PRIM_COPY_IF, dtype, n, 0, config);
  if (!config_valid(B2P_PRIM_COPY_IF, dtype, config)) return B2P_ERR_INVALID_ARG;
  return launch_copy_if(dtype, in, out, n, mask, cmp, rhs, num_copied, scratch, scratch_bytes,
                        config, (cudaStream_t)stream);
}

int b2p_copy_if(int dtype, const void *in, void *out, size_t n, uint64_t mask, int cmp,
                uint64_t rhs, uint64_t *num_copied, void *scratch, size_t scratch_bytes,
                int config, b2p_stream stream) {
  CallScope cs("b2p_copy_if", dtype, n, 0, (double)n * dtype_size(dtype), stream);
  return cs.done(copy_if_entry(dtype, in, out, n, mask, cmp, rhs, num_copied, scratch, scratch_bytes, config, stream));
}

static int histogram_u8_entry(const uint8_t *keys, size_t n, uint32_t *bins, int nbins, int config,
                     b2p_stream stream) {
  if (nbins < 1 || nbins > 256) return B2P_ERR_INVALID_ARG;
  if (n == 0) return B2P_OK;
  int rc = check_device();
  if (rc) return rc;
  if ((rc = check_ptr(keys, 1)) || (rc = check_ptr(bins, 4))) return rc;
  if ((rc = check_extent(keys, n)) || (rc = check_extent(bins, 4 * (size_t)nbins))) return rc;
  config = resolve(B2P_PRIM_HISTOGRAM, B2P_U32, n, 0, config);
  if (!config_valid(B2P_PRIM_HISTOGRAM, B2P_U32, config)) return B2P_ERR_INVALID_ARG;
  return launch_histogram_u8(keys, n, bins, nbins, config, (cudaStream_t)stream);
}

int b2p_histogram_u8(const uint8_t *keys, size_t n, uint32_t *bins, int nbins, int config,
                     b2p_stream stream) {
  CallScope cs("b2p_histogram_u8", B2P_U32, n, 0, (double)n + 4.0 * nbins, stream);
  return cs.done(histogram_u8_entry(keys, n, bins, nbins, config, stream));
}

static int segmented_reduce_entry(int dtype, int op, const void *in, const int64_t *offsets, int64_t nseg,
                                  void *out, const void *init, void *scratch, size_t scratch_bytes, int config,
                                  b2p_stream stream, CallScope &cs) {
  if (!valid_dtype(dtype) || !valid_op(dtype, op) || nseg < 0) return B2P_ERR_INVALID_ARG;
  if (nseg == 0) return B2P_OK;
  int rc = check_device();
  if (rc) return rc;
  if ((rc = check_ptr(in, dtype_size(dtype))) || (rc = check_ptr(out, acc_size(dtype))) ||
      (rc = check_ptr(offsets, 8)))
    return rc;
  // total element count is needed on the host: read offsets[nseg]
  int64_t total = 0;
  cudaError_t e = cudaMemcpyAsync(&total, offsets + nseg, sizeof(int64_t), cudaMemcpyDefault,
                                  (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e);
  if (total < 0) return B2P_ERR_INVALID_ARG;
  cs.set_size((size_t)total, (double)total * dtype_size(dtype) + (double)nseg * (acc_size(dtype) + 8));
  if ((rc = check_extent(in, (size_t)total * dtype_size(dtype))) ||
      (rc = check_extent(out, (size_t)nseg * acc_size(dtype))) ||
      (rc = check_extent(offsets, 8 * ((size_t)nseg + 1))) ||
      (rc = check_offsets(offsets, nseg, (size_t)total, (cudaStream_t)stream)))
    return rc;
  if (!scratch) return B2P_ERR_SCRATCH;
  config = resolve(B2P_PRIM_SEG_REDUCE, dtype, (size_t)total, nseg, config);
  if (!config_valid(B2P_PRIM_SEG_REDUCE, dtype, config)) return B2P_ERR_INVALID_ARG;
  return launch_segmented(B2P_PRIM_SEG_REDUCE, dtype, op, 1, in, out, offsets, nseg,
                          (size_t)total, init, scratch, scratch_bytes, config,
                          (cudaStream_t)stream);
}

int b2p_segmented_reduce(int dtype, int op, const void *in, const int64_t *offsets, int64_t nseg,
                         void *out, const void *init, void *scratch, size_t scratch_bytes,
                         int config, b2p_stream stream) {
  CallScope cs("b2p_segmented_reduce", dtype, 0, nseg, 0.0, stream);
  return cs.done(segmented_reduce_entry(dtype, op, in, offsets, nseg, out, init, scratch, scratch_bytes, config, stream, cs));
}

static int segmented_scan_entry(int dtype, int op, int inclusive, const void *in, void *out,
                                const int64_t *offsets, int64_t nseg, const void *init, void *scratch,
                                size_t scratch_bytes, int config, b2p_stream stream, CallScope &cs) {
  if (!valid_dtype(dtype) || !valid_op(dtype, op) || nseg < 0) return B2P_ERR_INVALID_ARG;
  if (!inclusive && !init) return B2P_ERR_INVALID_ARG;
  if (nseg == 0) return B2P_OK;
  int rc = check_device();
  if (rc) return rc;
  if ((rc = check_ptr(in, dtype_size(dtype))) || (rc = check_ptr(out, acc_size(dtype))) ||
      (rc = check_ptr(offsets, 8)))
    return rc;
  int64_t total = 0;
  cudaError_t e = cudaMemcpyAsync(&total, offsets + nseg, sizeof(int64_t), cudaMemcpyDefault,
                                  (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e);
  if (total < 0) return B2P_ERR_INVALID_ARG;
  if (total == 0) return B2P_OK;
  cs.set_size((size_t)total, (double)total * (dtype_size(dtype) + acc_size(dtype)) + 8.0 * nseg);
  if ((rc = check_extent(in, (size_t)total * dtype_size(dtype))) ||
      (rc = check_extent(out, (size_t)total * acc_size(dtype))) ||
      (rc = check_extent(offsets, 8 * ((size_t)nseg + 1))) ||
      (rc = check_offsets(offsets, nseg, (size_t)total, (cudaStream_t)stream)))
    return rc;
  if (!scratch) return B2P_ERR_SCRATCH;
  config = resolve(B2P_PRIM_SEG_SCAN, dtype, (size_t)total, nseg, config);
  if (!config_valid(B2P_PRIM_SEG_SCAN, dtype, config)) return B2P_ERR_INVALID_ARG;
  return launch_segmented(B2P_PRIM_SEG_SCAN, dtype, op, inclusive, in, out, offsets, nseg,
                          (size_t)total, init, scratch, scratch_bytes, config,
                          (cudaStream_t)stream);
}

int b2p_segmented_scan(int dtype, int op, int inclusive, const void *in, void *out,
                       const int64_t *offsets, int64_t nseg, const void *init, void *scratch,
                       size_t scratch_bytes, int config, b2p_stream stream) {
  CallScope cs("b2p_segmented_scan", dtype, 0, nseg, 0.0, stream);
  return cs.done(segmented_scan_entry(dtype, op, inclusive, in, out, offsets, nseg, init, scratch, scratch_bytes, config, stream, cs));
}

int b2p_device_error(void *scratch, b2p_stream stream, int clear) {
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e);
  if (!scratch) return scratchless_error(clear);
  unsigned v = 0;
  ScratchHeader *h = reinterpret_cast<ScratchHeader *>(scratch);
  e = cudaMemcpy(&v, &h->error, sizeof(v), cudaMemcpyDefault);
  if (e != cudaSuccess) return cuda_status(e);
  if (clear && v) {
    unsigned z = 0;
    e = cudaMemcpy(&h->error, &z, sizeof(z), cudaMemcpyDefault);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return (int)v;
}

uint64_t b2p_set_wait_timeout_ns(uint64_t ns) { return g_timeout_ns.exchange(ns ? ns : 1); }

uint64_t b2p_wait_timeout_ns(void) { return g_timeout_ns.load(); }

void b2p_debug_stall_tile(int64_t tile) { g_stall_tile.store(tile); }

}  // extern "C"
