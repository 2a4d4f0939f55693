// Launch-configuration choice: the fixed heuristic, the exhaustive
// autotuner (times every valid configuration for a shape) and the
// resolution of B2P_CONFIG_AUTO (learned selector table -> tuner table ->
// heuristic).
//
// The reference chooses launch shapes with fixed rules: 4*CUs groups of 128
// work-items for reductions (util/memory_streaming.hpp:30-47,
// algorithms/numeric.hpp:154-158) and 128 work-items x 16 items for scans
// (algorithms/scan/scan.hpp:26-32, decoupled_lookback_scan.hpp:481-488).
#include "b2p_device/common.cuh"
#include "internal.h"
#include "tuning.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <vector>

namespace b2p {

namespace {
std::mutex g_auto_mu;
AutoTable g_auto;  // installed selector decisions
}  // namespace

void install_auto_table(const AutoTable &t) {
  std::lock_guard<std::mutex> lk(g_auto_mu);
  g_auto = t;
}

void clear_auto_table() {
  std::lock_guard<std::mutex> lk(g_auto_mu);
  g_auto = AutoTable{};
}

int heuristic_config(int prim, int dtype, size_t n, int64_t nseg) {
  (void)nseg;
  auto cfg = [](int grid_mode, int block, int items) {
    int bi = block == 128 ? 0 : block == 256 ? 1 : block == 512 ? 2 : 3;
    int ii = items == 4 ? 0 : items == 8 ? 1 : items == 16 ? 2 : 3;
    return grid_mode * 16 + bi * 4 + ii;
  };
  // Fixed choices from configuration sweeps of 2^28-element inputs on B200.
  switch (prim) {
  case B2P_PRIM_REDUCE:
  case B2P_PRIM_DOT:
    return cfg(0, 1024, 32);
  case B2P_PRIM_SCAN:
    // pipelined (TMA) kernel from 8 MiB of input on; below that the
    // one-tile-per-block look-back kernel fills the GPU faster
    if (n * dtype_size(dtype) >= (8u << 20))
      return cfg(1, 256, dtype_size(dtype) == 8 ? 16 : 32);
    return cfg(0, 256, dtype_size(dtype) == 8 ? 16 : 32);
  case B2P_PRIM_COPY_IF:
    if (n * dtype_size(dtype) >= (8u << 20)) return cfg(1, 256, dtype_size(dtype) == 8 ? 16 : 32);
    return cfg(0, 256, dtype_size(dtype) == 8 ? 16 : 32);
  case B2P_PRIM_HISTOGRAM:
    return cfg(1, 1024, 32);
  case B2P_PRIM_SEG_REDUCE:
  case B2P_PRIM_SEG_SCAN:
    return cfg(1, 256, dtype_size(dtype) == 8 ? 16 : 32);
  default:
    return 0;
  }
}

int auto_lookup(int prim, int dtype, size_t n, int64_t nseg, double cv) {
  std::lock_guard<std::mutex> lk(g_auto_mu);
  if (!g_auto.valid) return -1;
  return g_auto.lookup(prim, dtype, n, nseg, cv);
}

// ------------------------------------------------------------- autotuner

namespace {

__global__ void fill_bits_kernel(uint32_t *p, size_t nwords, uint64_t seed, int kind) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nwords;
       i += (size_t)gridDim.x * blockDim.x) {
    uint64_t z = (i + 1) * 0x9E3779B97F4A7C15ull + seed;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    uint32_t v = (uint32_t)z;
    if (kind == 1) {  // fp32 in [-1, 1)
      v = __float_as_uint((float)((int)v) * 4.656612873077393e-10f);
    } else if (kind == 2) {  // two bf16 in [-1, 1)
      float a = (float)((int)(v & 0xffff) - 32768) * (1.0f / 32768.0f);
      float b = (float)((int)(v >> 16) - 32768) * (1.0f / 32768.0f);
      v = (__float_as_uint(a) >> 16) | (__float_as_uint(b) & 0xffff0000u);
    } else if (kind == 3) {  // small integers (no overflow concerns)
      v = (v & 0x3ff);
    }
    p[i] = v;
  }
}

}  // namespace

int tune_shape(int prim, int dtype, int op, size_t n, int64_t nseg, double cv, int reps,
               uint64_t seed, float *times_ms) {
  if (!times_ms || reps < 1 || n == 0) return B2P_ERR_INVALID_ARG;
  for (int c = 0; c < B2P_NUM_CONFIGS; ++c) times_ms[c] = INFINITY;
  const size_t es = prim == B2P_PRIM_HISTOGRAM ? 1 : dtype_size(dtype);
  const size_t os = prim == B2P_PRIM_HISTOGRAM ? 4 : acc_size(dtype);
  if (!es) return B2P_ERR_INVALID_ARG;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return B2P_ERR_CUDA;
  void *in = nullptr, *in2 = nullptr, *out = nullptr, *scratch = nullptr;
  int64_t *offs = nullptr;
  uint64_t *count = nullptr;
  int rc = B2P_OK;
  size_t sbytes = 0;
  const size_t out_elems = prim == B2P_PRIM_HISTOGRAM ? 256 : (prim == B2P_PRIM_REDUCE || prim == B2P_PRIM_DOT) ? 1 : (prim == B2P_PRIM_SEG_REDUCE ? (size_t)std::max<int64_t>(nseg, 1) : n);
  int64_t ns = nseg > 1 ? nseg : 1;
  std::vector<int64_t> hoffs;
  auto cleanup = [&]() {
    cudaFree(in);
    cudaFree(in2);
    cudaFree(out);
    cudaFree(scratch);
    cudaFree(offs);
    cudaFree(count);
    cudaStreamDestroy(st);
  };
#define B2P_TRY(x)                 \
  do {                             \
    if ((x) != cudaSuccess) {      \
      cudaGetLastError();          \
      cleanup();                   \
      return B2P_ERR_CUDA;         \
    }                              \
  } while (0)
  const size_t in_bytes = (n * es + 15) & ~(size_t)15;
  B2P_TRY(cudaMalloc(&in, in_bytes));
  if (prim == B2P_PRIM_DOT) B2P_TRY(cudaMalloc(&in2, in_bytes));
  B2P_TRY(cudaMalloc(&out, std::max<size_t>(out_elems * os, 256)));
  B2P_TRY(cudaMalloc(&count, 64));
  const int kind = (dtype == B2P_F32 || dtype == B2P_F64) ? 1 : dtype == B2P_BF16 ? 2 : 3;
  fill_bits_kernel<<<1024, 256, 0, st>>>((uint32_t *)in, in_bytes / 4, seed, prim == B2P_PRIM_HISTOGRAM ? 0 : kind);
  if (in2) fill_bits_kernel<<<1024, 256, 0, st>>>((uint32_t *)in2, in_bytes / 4, seed + 1, kind);
  if (prim == B2P_PRIM_SEG_REDUCE || prim == B2P_PRIM_SEG_SCAN) {
    hoffs.resize((size_t)ns + 1);
    uint64_t tot = 0;
    // log-uniform lengths whose spread grows with cv, scaled to n
    double log2max = std::min(30.0, std::max(1.0, 4.0 * cv + 1.0) * std::log2((double)n / ns + 1.0));
    b2p_synth_segments(seed, ns, log2max, 0, hoffs.data(), &tot);
    double f = (double)n / (double)std::max<uint64_t>(tot, 1);
    for (int64_t s = 1; s <= ns; ++s) hoffs[(size_t)s] = std::min<int64_t>((int64_t)n, (int64_t)std::llround(hoffs[(size_t)s] * f));
    hoffs[(size_t)ns] = (int64_t)n;
    for (int64_t s = 1; s <= ns; ++s) hoffs[(size_t)s] = std::max(hoffs[(size_t)s], hoffs[(size_t)s - 1]);
    B2P_TRY(cudaMalloc(&offs, (hoffs.size()) * sizeof(int64_t)));
    B2P_TRY(cudaMemcpyAsync(offs, hoffs.data(), hoffs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  }
  sbytes = b2p_scratch_bytes(prim == B2P_PRIM_HISTOGRAM ? B2P_PRIM_REDUCE : prim, prim == B2P_PRIM_HISTOGRAM ? B2P_U32 : dtype, n, ns, B2P_CONFIG_AUTO);
  B2P_TRY(cudaMalloc(&scratch, std::max<size_t>(sbytes, 256)));
  B2P_TRY(cudaMemsetAsync(scratch, 0, std::max<size_t>(sbytes, 256), st));
  cudaEvent_t e0, e1;
  B2P_TRY(cudaEventCreate(&e0));
  B2P_TRY(cudaEventCreate(&e1));
  auto run = [&](int c) -> int {
    switch (prim) {
    case B2P_PRIM_REDUCE: return b2p_reduce(dtype, op, in, n, out, nullptr, scratch, sbytes, c, (b2p_stream)st);
    case B2P_PRIM_DOT: return b2p_dot(dtype, in, in2, n, out, nullptr, scratch, sbytes, c, (b2p_stream)st);
    case B2P_PRIM_SCAN: {
      unsigned long long z = 0;
      return b2p_scan(dtype, op, 1, in, out, n, &z, scratch, sbytes, c, (b2p_stream)st);
    }
    case B2P_PRIM_COPY_IF: return b2p_copy_if(dtype == B2P_BF16 ? B2P_U32 : dtype, in, out, n, 7, B2P_CMP_LT, 3, count, scratch, sbytes, c, (b2p_stream)st);
    case B2P_PRIM_HISTOGRAM: return b2p_histogram_u8((const uint8_t *)in, n, (uint32_t *)out, 256, c, (b2p_stream)st);
    case B2P_PRIM_SEG_REDUCE: return launch_segmented(prim, dtype, op, 1, in, out, offs, ns, n, nullptr, scratch, sbytes, c, st);
    case B2P_PRIM_SEG_SCAN: return launch_segmented(prim, dtype, op, 1, in, out, offs, ns, n, nullptr, scratch, sbytes, c, st);
    default: return B2P_ERR_INVALID_ARG;
    }
  };
  std::vector<float> t((size_t)reps);
  const bool seg = prim == B2P_PRIM_SEG_REDUCE || prim == B2P_PRIM_SEG_SCAN;
  for (int c = 0; c < B2P_NUM_CONFIGS && rc == B2P_OK; ++c) {
    if (!b2p_config_valid(prim, dtype, c)) continue;
    // segmented shapes are timed as their CUDA-graph plan launches
    b2p_plan plan = nullptr;
    if (seg) {
      int r = b2p_plan_segmented(&plan, prim, dtype, op, in, out, offs, ns, n, c, (b2p_stream)st);
      if (r != B2P_OK) {
        rc = r;
        break;
      }
    }
    auto once = [&]() { return seg ? b2p_plan_launch(plan, (b2p_stream)st) : run(c); };
    int r = once();  // warm-up (also catches unsupported combinations)
    if (r != B2P_OK) {
      b2p_plan_destroy(plan);
      rc = r;
      break;
    }
    for (int k = 0; k < reps; ++k) {
      cudaEventRecord(e0, st);
      once();
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = B2P_ERR_CUDA;
        break;
      }
      cudaEventElapsedTime(&t[(size_t)k], e0, e1);
    }
    b2p_plan_destroy(plan);
    std::sort(t.begin(), t.end());
    times_ms[c] = t[(size_t)reps / 2];
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = B2P_ERR_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cleanup();
#undef B2P_TRY
  return rc;
}

}  // namespace b2p

using namespace b2p;

extern "C" {

int b2p_heuristic_config(int prim, int dtype, size_t n, int64_t nseg) {
  return heuristic_config(prim, dtype, n, nseg);
}

int b2p_auto_config(int prim, int dtype, size_t n, int64_t nseg, double cv) {
  int c = selector_mode() == 1 ? -1 : auto_lookup(prim, dtype, n, nseg, cv);
  if (c >= 0 && b2p_config_valid(prim, dtype, c)) return c;
  c = heuristic_config(prim, dtype, n, nseg);
  if (b2p_config_valid(prim, dtype, c)) return c;
  for (int k = 0; k < B2P_NUM_CONFIGS; ++k)
    if (b2p_config_valid(prim, dtype, k)) return k;
  return 0;
}

int b2p_tune_shape(int prim, int dtype, int op, size_t n, int64_t nseg, double cv, int reps,
                   uint64_t seed, float *times_ms) {
  return tune_shape(prim, dtype, op, n, nseg, cv, reps, seed, times_ms);
}

}  // extern "C"
