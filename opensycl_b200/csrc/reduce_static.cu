// b2p_reduce_static: the reduce entry point for callers that cannot
// allocate device memory.
//
// Some callers of this library must not call cudaMalloc or any allocating
// routine: code that runs inside a custom device-memory allocator or a
// memory-pool callback, real-time or safety-certified paths whose device
// memory is fixed at start-up, and hosts (other language runtimes, plugins)
// that own the device heap and forbid side allocations.  They cannot hand
// b2p_reduce a scratch buffer.  This variant runs the same single-pass reduce
// kernel on a scratch area that is part of the library image: a file-scope
// __device__ array, present on every GPU that loads the library until the
// process exits.
//
// Host code only ever sees a host-side stand-in for the array's name; the
// real device address comes from cudaGetSymbolAddress, with the device
// current, and is passed to the kernel as a plain pointer.
#include "b2p_device/common.cuh"
#include "internal.h"

#include <mutex>

namespace {

// Shared scratch of every b2p_reduce_static call on a device.  The reduce
// needs the scratch prefix plus one 16-byte word per run, and its run count
// stays below 4736 for every input size, so 128 KiB covers every call.
static __device__ __align__(256) unsigned char g_reduce_scratch[B2P_STATIC_SCRATCH_BYTES];

constexpr int kMaxDev = 64;
std::mutex g_mu;
// Address of g_reduce_scratch seen by the last set-up on each device.  A
// different address later means the device's context was rebuilt (for
// example after cudaDeviceReset), and the set-up runs again.
void *g_addr[kMaxDev] = {nullptr};

// Device address of g_reduce_scratch on the current device.  Looked up on
// every call (after the module is loaded this is a table read and allocates
// nothing), so an address is never reused from an earlier context.  The
// first call on a device, and the first after its context was rebuilt, also
// loads every reduce kernel this entry point can launch, so that no later
// call loads a module.
int scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return b2p::cuda_status(e);
  if (dev < 0 || dev >= kMaxDev) return B2P_ERR_NO_DEVICE;
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_reduce_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return B2P_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_addr[dev] != p) {
    int rc = b2p::preload_reduce_kernels();
    if (rc) return rc;
    g_addr[dev] = p;
  }
  *out = p;
  return B2P_OK;
}

}  // namespace

extern "C" int b2p_reduce_static(int dtype, int op, const void *in, size_t n, void *out,
                                 const void *init, b2p_stream stream) {
  if (n > B2P_STATIC_MAX_ELEMS) return B2P_ERR_INVALID_ARG;
  // Every check b2p_reduce makes comes first: a rejected call must not touch
  // the array that all calls on the device share.
  int rc = b2p::validate_reduce(dtype, op, in, n, out);
  if (rc || n == 0) return rc;
  const size_t need = b2p::reduce_scratch_bytes(dtype, n, in, nullptr);
  if (need > B2P_STATIC_SCRATCH_BYTES) return B2P_ERR_SCRATCH;
  void *scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc) return rc;
  // The block-arrival counter must start at zero; a completed call leaves
  // it zero, and clearing it here keeps that true even after a call that
  // never finished.  (cudaMemsetAsync allocates nothing.)
  cudaError_t e = cudaMemsetAsync(scratch, 0, b2p::kHeaderBytes, (cudaStream_t)stream);
  if (e != cudaSuccess) return b2p::cuda_status(e);
  // Launch shape 15 (1024 threads x 32 items, one group of runs per block)
  // needs no occupancy query; the float result is the same for every shape.
  return b2p_reduce(dtype, op, in, n, out, init, scratch, B2P_STATIC_SCRATCH_BYTES, 15, stream);
}
