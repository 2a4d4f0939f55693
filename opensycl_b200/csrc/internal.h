// Host-side declarations shared by the translation units of libb2p.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/b2p.h"

namespace b2p {

struct LaunchConfig;

// Cached per-device facts (queried once per device).
struct DeviceInfo {
  int device = -1;
  int sm_count = 0;
  int max_smem_optin = 0;
  int cc_major = 0, cc_minor = 0;
  char name[256] = {0};
};
const DeviceInfo &device_info();

// Blocks per SM for (kernel, block, dynamic smem); cached.
int occupancy(const void *kernel, int block, size_t smem);

// Grid size for a launch that has `units` independent units of work
// (tiles or runs) with `units_per_block` units per block.
int grid_for(int grid_mode, long long units, int units_per_block, const void *kernel, int block,
             size_t smem);

// Raise a kernel's dynamic shared-memory limit once per (device, kernel).
int ensure_dynamic_smem(const void *kernel, size_t bytes);

// Wait bound for device-side spins (ns) and the stall test hook.
uint64_t wait_timeout_ns();
long long debug_stall_tile();

// Record a CUDA failure; returns B2P_ERR_CUDA or B2P_OK.
int cuda_status(cudaError_t e);

// Scratch bytes of b2p_sort (prim B2P_PRIM_SORT) or b2p_merge
// (B2P_PRIM_MERGE) on n keys of dtype; 0 for other dtypes.
size_t merge_sort_scratch_bytes(int prim, int dtype, size_t n);

// ------------------------------------------------ logging and checks (log.cu)
// Log level (B2P_LOG_LEVEL, else ACPP_DEBUG_LEVEL / HIPSYCL_DEBUG_LEVEL;
// default 2) and one stderr line at `level` (1 error .. 4 verbose).
int log_level();
void set_log_level(int level);
void log_line(int level, const char *fmt, ...);
// The configuration a call resolved (reported by its call record).
void note_config(int config);
// B2P_CHECKED: extents of pointer arguments and segment offsets are checked.
bool checked_mode();
int check_extent(const void *p, size_t bytes);
int check_offsets(const int64_t *offsets, int64_t nseg, size_t total, cudaStream_t st);
// B2P_SELECTOR: 0 = installed selector table, else heuristic; 1 = heuristic.
int selector_mode();

// One C-ABI call: an NVTX range over the host call, and its record at log
// level 3 (4: timed on the stream).  done(status) logs and returns status.
class CallScope {
 public:
  CallScope(const char *op, int dtype, size_t n, int64_t nseg, double bytes, b2p_stream stream);
  CallScope(const CallScope &) = delete;
  CallScope &operator=(const CallScope &) = delete;
  ~CallScope();
  void set_size(size_t n, double bytes);  // once the element count is known
  int done(int status);

 private:
  const char *op_;
  int dtype_;
  size_t n_;
  int64_t nseg_;
  double bytes_;
  cudaStream_t st_;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr;
  bool timed_ = false;
};

// Device-accessibility and alignment check of a pointer (B2P_OK or
// B2P_ERR_INVALID_PTR); no CPU fallback.
int check_pointer(const void *p, size_t align);

// Reduce / dot.  b == nullptr: reduce; otherwise dot.
// Argument, device and pointer checks of b2p_reduce (B2P_OK when n == 0).
int validate_reduce(int dtype, int op, const void *in, size_t n, const void *out);
// Loads every reduce kernel instantiation b2p_reduce can launch for a plain
// reduce (no dot) on the current device, so that later launches load no
// module (cudaFuncGetAttributes on each).
int preload_reduce_kernels();
size_t reduce_scratch_bytes(int dtype, size_t n, const void *a, const void *b);
int launch_reduce(int dtype, int op, const void *a, const void *b, size_t n, void *out,
                  const void *init, void *scratch, size_t scratch_bytes, int config,
                  cudaStream_t s);

// Scan and copy_if (decoupled look-back).
size_t scan_scratch_bytes(int dtype, size_t n, int config);
int launch_scan(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
                const void *init, void *scratch, size_t scratch_bytes, int config,
                cudaStream_t s);
size_t copy_if_scratch_bytes(int dtype, size_t n, int config);
int launch_copy_if(int dtype, const void *in, void *out, size_t n, uint64_t mask, int cmp,
                   uint64_t rhs, uint64_t *num_copied, void *scratch, size_t scratch_bytes,
                   int config, cudaStream_t s);
bool scan_config_valid(int dtype, int config);

// Pipelined (TMA) scan of grid mode 1.  Returns B2P_ERR_UNSUPPORTED, having
// launched nothing, when the call does not fit it (bf16, a pointer not
// 16-byte aligned, fewer elements than one tile, a tile shape without a
// pipelined kernel); the caller then runs the two-phase kernel.
bool scan_tma_shape(int dtype, int block, int items);
int launch_scan_tma(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
                    const void *init, void *scratch, int block, int items, cudaStream_t s);
// Pipelined copy_if of grid mode 1 (same fallback contract).
bool copy_if_tma_shape(int dtype, int block, int items);
int launch_copy_if_tma(int dtype, const void *in, void *out, size_t n, uint64_t mask, int cmp,
                       uint64_t rhs, uint64_t *num_copied, void *scratch, int block, int items,
                       cudaStream_t s);
bool copy_if_config_valid(int dtype, int config);

// Histogram.
// The device error word of scratch-less calls (histogram); clear != 0
// resets it.  Synchronous.
int scratchless_error(int clear);

int launch_histogram_u8(const uint8_t *keys, size_t n, uint32_t *bins, int nbins, int config,
                        cudaStream_t s);

// Segmented reduce / scan (one persistent launch).
size_t segmented_scratch_bytes(int dtype, size_t n, int64_t nseg, int config);
int launch_segmented(int prim, int dtype, int op, int inclusive, const void *in, void *out,
                     const int64_t *offsets, int64_t nseg, size_t total, const void *init,
                     void *scratch, size_t scratch_bytes, int config, cudaStream_t s);
bool segmented_config_valid(int dtype, int config);
// The pipelined segmented kernel (flat segmented scan on the TMA pipeline):
// whether it has the (dtype, op, block, items) shape, the scratch it needs
// (prefix, one status word per tile, then one 64-int record per tile), the
// host computation of the records, and the launch.  The records must
// already be in scratch; returns B2P_ERR_UNSUPPORTED, having launched
// nothing, when the call does not fit.
bool segmented_tma_shape(int dtype, int op, int block, int items);
size_t segmented_tma_scratch(size_t n, int block, int items);
void segmented_tile_records(const int64_t *offs, int64_t nseg, size_t n, int block, int items, int *rec);
int launch_segmented_tma(int prim, int dtype, int op, int inclusive, const void *in, void *out,
                         const int64_t *offsets, int64_t nseg, size_t n, const void *init, void *scratch,
                         int block, int items, cudaStream_t s);

// Element sizes.
inline size_t dtype_size(int dtype) {
  switch (dtype) {
  case B2P_I32: case B2P_U32: case B2P_F32: return 4;
  case B2P_I64: case B2P_U64: case B2P_F64: return 8;
  case B2P_BF16: return 2;
  default: return 0;
  }
}
// Size of the accumulation / output element (bf16 accumulates in fp32).
inline size_t acc_size(int dtype) { return dtype == B2P_BF16 ? 4 : dtype_size(dtype); }
inline bool dtype_is_float(int dtype) {
  return dtype == B2P_F32 || dtype == B2P_BF16 || dtype == B2P_F64;
}

}  // namespace b2p
