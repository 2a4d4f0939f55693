// Learned schedule selector: a 11 -> 64 -> 64 -> 48 MLP (ReLU, fp32) that
// maps a call's shape to one of the 48 launch configurations, trained on the
// exhaustive autotuner's own timings with the library's CUDA kernels.
//
// The reference has no launch-configuration model; its closest analogues
// are the stdpar offload heuristic database (std/stdpar/detail/
// offload_heuristic_db.hpp:232-365), which interpolates measured run times to
// decide host vs device, and the JIT's argument specialisation
// (src/runtime/adaptivity_engine.cpp:52-156).  Neither picks launch shapes.
//
// Training loss per sample, over the configurations valid for that sample:
//   L = sum_c p_c * t_c / t_min  +  ce_weight * (-log p_best)
// with p = softmax(z); the first term is the expected normalised run time of
// a configuration drawn from the model, the second anchors it on the
// fastest one.  dL/dz_c = p_c (r_c - sum_j p_j r_j) + ce_weight (p_c - [c = best]).
//
// Kernels: one forward+backward kernel (blocks of 64 threads, each block a
// contiguous slice of samples; thread j owns row j of W1, column j of W2 and
// W3 gradients, so the per-block gradient needs no atomics), a fixed-order
// reduction of the per-block gradients (deterministic), Adam, and batched
// inference with a masked argmax.
#include "b2p_device/common.cuh"
#include "internal.h"
#include "tuning.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace b2p {

constexpr int kF = B2P_SEL_FEATURES;  // 11
constexpr int kH = B2P_SEL_HIDDEN;    // 64
constexpr int kC = B2P_NUM_CONFIGS;   // 48
// parameter layout: W1[kH][kF], b1[kH], W2[kH][kH], b2[kH], W3[kC][kH], b3[kC]
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * kF;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kC * kH;
constexpr int kP = kOffB3 + kC;  // 8048
constexpr int kTrainBlocks = 64;

static_assert(kP == 8048, "selector parameter count");

// Forward pass of one sample by a block of kH threads (thread j = unit j).
// x: kF floats in shared memory.  Writes h1, h2 (post-ReLU) and z.
__device__ __forceinline__ void mlp_forward(const float *w, const float *x, float *h1, float *h2,
                                            float *z) {
  const int j = threadIdx.x;
  float a = w[kOffB1 + j];
#pragma unroll
  for (int k = 0; k < kF; ++k) a = fmaf(w[kOffW1 + j * kF + k], x[k], a);
  h1[j] = fmaxf(a, 0.f);
  __syncthreads();
  a = w[kOffB2 + j];
#pragma unroll 8
  for (int k = 0; k < kH; ++k) a = fmaf(w[kOffW2 + j * kH + k], h1[k], a);
  h2[j] = fmaxf(a, 0.f);
  __syncthreads();
  if (j < kC) {
    a = w[kOffB3 + j];
#pragma unroll 8
    for (int k = 0; k < kH; ++k) a = fmaf(w[kOffW3 + j * kH + k], h2[k], a);
    z[j] = a;
  }
  __syncthreads();
}

__device__ __forceinline__ float block64_max(float v, float *red) {
  for (int m = 16; m >= 1; m >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, m));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = fmaxf(red[0], red[1]);
  __syncthreads();
  return v;
}
__device__ __forceinline__ float block64_sum(float v, float *red) {
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = red[0] + red[1];
  __syncthreads();
  return v;
}

// One block: samples [lo, hi).  Gradients are divided by m (mean loss).
__global__ void __launch_bounds__(kH) mlp_fwd_bwd_kernel(const float *X, const float *T, int m,
                                                         const float *params, float ce_w,
                                                         float *partial, float *partial_loss) {
  extern __shared__ float sm[];
  float *w = sm;          // kP
  float *g = sm + kP;     // kP
  __shared__ float x[kF], h1[kH], h2[kH], z[kH], dz[kH], dh2[kH], dh1[kH], red[2];
  const int j = threadIdx.x;
  for (int i = j; i < kP; i += kH) {
    w[i] = params[i];
    g[i] = 0.f;
  }
  const int per = (m + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * per, hi = min(m, lo + per);
  float loss = 0.f;
  const float inv_m = 1.f / (float)m;
  __syncthreads();
  for (int s = lo; s < hi; ++s) {
    if (j < kF) x[j] = X[(size_t)s * kF + j];
    __syncthreads();
    mlp_forward(w, x, h1, h2, z);
    // masked softmax over valid configurations (finite times)
    const float t = j < kC ? T[(size_t)s * kC + j] : INFINITY;
    const bool valid = isfinite(t);
    const float tmin = -block64_max(valid ? -t : -INFINITY, red);
    const float zmax = block64_max(valid ? z[j] : -INFINITY, red);
    const float e = valid ? __expf(z[j] - zmax) : 0.f;
    const float se = block64_sum(e, red);
    const float pj = e / se;
    const float r = valid ? t / tmin : 0.f;
    const float er = block64_sum(pj * r, red);
    // index of the fastest valid configuration (lowest index on ties)
    float best_key = valid && t == tmin ? (float)j : 1e9f;
    const float best = -block64_max(-best_key, red);
    const bool is_best = (float)j == best;
    const float pbest = block64_sum(is_best ? pj : 0.f, red);
    if (j == 0) loss += er - ce_w * __logf(fmaxf(pbest, 1e-30f));
    dz[j] = valid ? (pj * (r - er) + ce_w * (pj - (is_best ? 1.f : 0.f))) * inv_m : 0.f;
    __syncthreads();
    // backward
    float a = 0.f;
    for (int c = 0; c < kC; ++c) a = fmaf(w[kOffW3 + c * kH + j], dz[c], a);
    dh2[j] = h2[j] > 0.f ? a : 0.f;
    __syncthreads();
    a = 0.f;
    for (int i = 0; i < kH; ++i) a = fmaf(w[kOffW2 + i * kH + j], dh2[i], a);
    dh1[j] = h1[j] > 0.f ? a : 0.f;
    __syncthreads();
    // gradient accumulation: thread j owns column j of W3 / W2, row j of W1
    for (int c = 0; c < kC; ++c) g[kOffW3 + c * kH + j] = fmaf(dz[c], h2[j], g[kOffW3 + c * kH + j]);
    if (j < kC) g[kOffB3 + j] += dz[j];
    for (int i = 0; i < kH; ++i) g[kOffW2 + i * kH + j] = fmaf(dh2[i], h1[j], g[kOffW2 + i * kH + j]);
    g[kOffB2 + j] += dh2[j];
#pragma unroll
    for (int k = 0; k < kF; ++k) g[kOffW1 + j * kF + k] = fmaf(dh1[j], x[k], g[kOffW1 + j * kF + k]);
    g[kOffB1 + j] += dh1[j];
    __syncthreads();
  }
  for (int i = j; i < kP; i += kH) partial[(size_t)blockIdx.x * kP + i] = g[i];
  if (j == 0) partial_loss[blockIdx.x] = loss * inv_m;
}

// grads[i] = sum over blocks of partial[b][i], in block order.
__global__ void mlp_reduce_kernel(const float *partial, const float *partial_loss, int nblocks,
                                  float *grads, float *loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kP) {
    float a = 0.f;
    for (int b = 0; b < nblocks; ++b) a += partial[(size_t)b * kP + i];
    grads[i] = a;
  }
  if (i == 0) {
    float l = 0.f;
    for (int b = 0; b < nblocks; ++b) l += partial_loss[b];
    *loss = l;
  }
}

__global__ void mlp_adam_kernel(float *params, const float *grads, float *m1, float *m2, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kP) return;
  const float gi = grads[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = v;
  params[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// Best valid configuration per row: argmax of the logits over the row's mask.
__global__ void __launch_bounds__(kH) mlp_predict_kernel(const float *X, const unsigned long long *mask,
                                                         int m, const float *params, int *out) {
  extern __shared__ float sm[];
  float *w = sm;
  __shared__ float x[kF], h1[kH], h2[kH], z[kH];
  const int j = threadIdx.x;
  for (int i = j; i < kP; i += kH) w[i] = params[i];
  __syncthreads();
  for (int s = blockIdx.x; s < m; s += gridDim.x) {
    if (j < kF) x[j] = X[(size_t)s * kF + j];
    __syncthreads();
    mlp_forward(w, x, h1, h2, z);
    if (j == 0) {
      const unsigned long long mk = mask[s];
      int best = -1;
      float bz = -INFINITY;
      for (int c = 0; c < kC; ++c)
        if (((mk >> c) & 1ull) && (best < 0 || z[c] > bz)) {
          best = c;
          bz = z[c];
        }
      out[s] = best;
    }
    __syncthreads();
  }
}

}  // namespace b2p

// -------------------------------------------------------------------- host

struct b2p_selector_s {
  float *params = nullptr;  // device
  float *grads = nullptr, *m1 = nullptr, *m2 = nullptr, *partial = nullptr, *ploss = nullptr,
        *loss = nullptr;
  int step = 0;
  int device = -1;
};

using namespace b2p;

namespace {

// row mask of valid configurations from the features' dtype/op one-hots
unsigned long long row_mask(const float *f) {
  const int dts[4] = {B2P_I32, B2P_I64, B2P_F32, B2P_BF16};
  int dtype = B2P_U32;
  for (int k = 0; k < 4; ++k)
    if (f[1 + k] > 0.5f) dtype = dts[k];
  int op = 0;
  for (int k = 0; k < 4; ++k)
    if (f[5 + k] > 0.5f) op = k;
  const bool seg = f[9] > 0.0f;
  int prim = B2P_PRIM_REDUCE;
  if (op == 0) prim = seg ? B2P_PRIM_SEG_REDUCE : B2P_PRIM_REDUCE;
  if (op == 1) prim = seg ? B2P_PRIM_SEG_SCAN : B2P_PRIM_SCAN;
  if (op == 2) prim = B2P_PRIM_COPY_IF;
  if (op == 3) prim = B2P_PRIM_HISTOGRAM;
  if (prim == B2P_PRIM_COPY_IF && dtype == B2P_BF16) dtype = B2P_U32;
  unsigned long long mk = 0;
  for (int c = 0; c < kC; ++c)
    if (b2p_config_valid(prim, dtype, c)) mk |= 1ull << c;
  return mk;
}

int alloc_sel(b2p_selector_s *s) {
  cudaError_t e = cudaSuccess;
  auto A = [&](float **p, size_t n) {
    if (e == cudaSuccess) e = cudaMalloc(p, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(*p, 0, n * sizeof(float));
  };
  A(&s->params, kP);
  A(&s->grads, kP);
  A(&s->m1, kP);
  A(&s->m2, kP);
  A(&s->partial, (size_t)kTrainBlocks * kP);
  A(&s->ploss, kTrainBlocks);
  A(&s->loss, 1);
  return cuda_status(e);
}

int run_fwd_bwd(b2p_selector_s *s, const float *dX, const float *dT, int m, float ce_w) {
  const size_t smem = 2 * (size_t)kP * sizeof(float);
  int rc = ensure_dynamic_smem((const void *)mlp_fwd_bwd_kernel, smem);
  if (rc) return rc;
  const int blocks = std::min(kTrainBlocks, std::max(1, m));
  mlp_fwd_bwd_kernel<<<blocks, kH, smem>>>(dX, dT, m, s->params, ce_w, s->partial, s->ploss);
  mlp_reduce_kernel<<<(kP + 255) / 256, 256>>>(s->partial, s->ploss, blocks, s->grads, s->loss);
  return cuda_status(cudaGetLastError());
}

struct DevBuf {
  float *p = nullptr;
  ~DevBuf() { cudaFree(p); }
};

const char kMagic[8] = {'B', '2', 'P', 'S', 'E', 'L', '0', '1'};

}  // namespace

extern "C" {

int b2p_selector_num_params(void) { return kP; }

int b2p_selector_create(b2p_selector *out, uint64_t seed) {
  if (!out) return B2P_ERR_INVALID_ARG;
  *out = nullptr;
  b2p_selector_s *s = new b2p_selector_s();
  cudaGetDevice(&s->device);
  int rc = alloc_sel(s);
  if (rc) {
    b2p_selector_destroy(s);
    return rc;
  }
  // He-style uniform init from a counter-based generator (host side)
  std::vector<float> h(kP, 0.f);
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + 1;
  auto u01 = [&]() {
    z += 0x9E3779B97F4A7C15ull;
    uint64_t t = z;
    t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
    t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
    t ^= t >> 31;
    return (double)(t >> 11) * 0x1.0p-53;
  };
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / cols);
    for (int i = 0; i < rows * cols; ++i) h[(size_t)off + i] = (float)((2.0 * u01() - 1.0) * a);
  };
  fill(kOffW1, kH, kF);
  fill(kOffW2, kH, kH);
  fill(kOffW3, kC, kH);
  rc = cuda_status(cudaMemcpy(s->params, h.data(), kP * sizeof(float), cudaMemcpyHostToDevice));
  if (rc) {
    b2p_selector_destroy(s);
    return rc;
  }
  *out = s;
  return B2P_OK;
}

void b2p_selector_destroy(b2p_selector s) {
  if (!s) return;
  cudaFree(s->params);
  cudaFree(s->grads);
  cudaFree(s->m1);
  cudaFree(s->m2);
  cudaFree(s->partial);
  cudaFree(s->ploss);
  cudaFree(s->loss);
  delete s;
}

int b2p_selector_features(int prim, int dtype, size_t n, int64_t nseg, double cv, float *f) {
  if (!f) return B2P_ERR_INVALID_ARG;
  for (int k = 0; k < kF; ++k) f[k] = 0.f;
  f[0] = (float)(std::log2((double)std::max<size_t>(n, 1)) / 32.0);
  const int dts[4] = {B2P_I32, B2P_I64, B2P_F32, B2P_BF16};
  for (int k = 0; k < 4; ++k)
    if (dtype == dts[k]) f[1 + k] = 1.f;
  if (dtype == B2P_U32) f[1] = 1.f;  // 32-bit integer family
  if (dtype == B2P_U64) f[2] = 1.f;
  if (dtype == B2P_F64) f[2] = 1.f;
  int op = 0;
  switch (prim) {
  case B2P_PRIM_REDUCE: case B2P_PRIM_DOT: case B2P_PRIM_SEG_REDUCE: op = 0; break;
  case B2P_PRIM_SCAN: case B2P_PRIM_SEG_SCAN: op = 1; break;
  case B2P_PRIM_COPY_IF: op = 2; break;
  case B2P_PRIM_HISTOGRAM: op = 3; break;
  default: return B2P_ERR_INVALID_ARG;
  }
  f[5 + op] = 1.f;
  const bool seg = prim == B2P_PRIM_SEG_REDUCE || prim == B2P_PRIM_SEG_SCAN;
  if (prim == B2P_PRIM_HISTOGRAM) {
    for (int k = 0; k < 4; ++k) f[1 + k] = 0.f;
  }
  f[9] = seg ? (float)(std::log2((double)std::max<int64_t>(nseg, 2)) / 20.0) : 0.f;
  f[10] = seg ? (float)(std::min(cv, 4.0) / 4.0) : 0.f;
  return B2P_OK;
}

int b2p_selector_grad(b2p_selector s, const float *features, const float *times, int m,
                      float ce_weight, float *loss, float *grads) {
  if (!s || !features || !times || m <= 0) return B2P_ERR_INVALID_ARG;
  DevBuf X, T;
  cudaError_t e = cudaMalloc(&X.p, (size_t)m * kF * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&T.p, (size_t)m * kC * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(X.p, features, (size_t)m * kF * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(T.p, times, (size_t)m * kC * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e);
  int rc = run_fwd_bwd(s, X.p, T.p, m, ce_weight);
  if (rc) return rc;
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess && loss) e = cudaMemcpy(loss, s->loss, sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && grads) e = cudaMemcpy(grads, s->grads, kP * sizeof(float), cudaMemcpyDeviceToHost);
  return cuda_status(e);
}

int b2p_selector_train(b2p_selector s, const float *features, const float *times, int m, int epochs,
                       float lr, float ce_weight, float *final_loss) {
  if (!s || !features || !times || m <= 0 || epochs < 0) return B2P_ERR_INVALID_ARG;
  DevBuf X, T;
  cudaError_t e = cudaMalloc(&X.p, (size_t)m * kF * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&T.p, (size_t)m * kC * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(X.p, features, (size_t)m * kF * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(T.p, times, (size_t)m * kC * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    int rc = run_fwd_bwd(s, X.p, T.p, m, ce_weight);
    if (rc) return rc;
    ++s->step;
    const float c1 = 1.f - std::pow(b1, (float)s->step), c2 = 1.f - std::pow(b2, (float)s->step);
    mlp_adam_kernel<<<(kP + 255) / 256, 256>>>(s->params, s->grads, s->m1, s->m2, lr, b1, b2, eps, c1, c2);
  }
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess && final_loss) {
    int rc = run_fwd_bwd(s, X.p, T.p, m, ce_weight);
    if (rc) return rc;
    e = cudaMemcpy(final_loss, s->loss, sizeof(float), cudaMemcpyDeviceToHost);
  }
  return cuda_status(e);
}

int b2p_selector_predict(b2p_selector s, const float *features, int m, int *configs) {
  if (!s || !features || !configs || m <= 0) return B2P_ERR_INVALID_ARG;
  std::vector<unsigned long long> mk((size_t)m);
  for (int i = 0; i < m; ++i) mk[(size_t)i] = row_mask(features + (size_t)i * kF);
  DevBuf X;
  unsigned long long *dm = nullptr;
  int *dout = nullptr;
  cudaError_t e = cudaMalloc(&X.p, (size_t)m * kF * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dm, (size_t)m * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&dout, (size_t)m * sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(X.p, features, (size_t)m * kF * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dm, mk.data(), (size_t)m * sizeof(unsigned long long), cudaMemcpyHostToDevice);
  int rc = B2P_OK;
  if (e == cudaSuccess) {
    const size_t smem = (size_t)kP * sizeof(float);
    rc = ensure_dynamic_smem((const void *)mlp_predict_kernel, smem);
    if (!rc) {
      const int grid = std::min(m, 148 * 8);
      mlp_predict_kernel<<<grid, kH, smem>>>(X.p, dm, m, s->params, dout);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpy(configs, dout, (size_t)m * sizeof(int), cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(dm);
  cudaFree(dout);
  return rc ? rc : cuda_status(e);
}

int b2p_selector_get_params(b2p_selector s, float *params) {
  if (!s || !params) return B2P_ERR_INVALID_ARG;
  return cuda_status(cudaMemcpy(params, s->params, kP * sizeof(float), cudaMemcpyDeviceToHost));
}

int b2p_selector_set_params(b2p_selector s, const float *params) {
  if (!s || !params) return B2P_ERR_INVALID_ARG;
  s->step = 0;
  cudaMemset(s->m1, 0, kP * sizeof(float));
  cudaMemset(s->m2, 0, kP * sizeof(float));
  return cuda_status(cudaMemcpy(s->params, params, kP * sizeof(float), cudaMemcpyHostToDevice));
}

// File: magic[8], u32 param count, char gpu[64], char version[32], floats.
int b2p_selector_save(b2p_selector s, const char *path) {
  if (!s || !path) return B2P_ERR_INVALID_ARG;
  std::vector<float> h(kP);
  int rc = b2p_selector_get_params(s, h.data());
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) return B2P_ERR_IO;
  char gpu[64] = {0}, ver[32] = {0};
  snprintf(gpu, sizeof(gpu), "%s", device_info().name);
  snprintf(ver, sizeof(ver), "%s", b2p_version());
  const uint32_t np = kP;
  bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(&np, 4, 1, f) == 1 && fwrite(gpu, 1, 64, f) == 64 &&
            fwrite(ver, 1, 32, f) == 32 && fwrite(h.data(), sizeof(float), kP, f) == (size_t)kP;
  fclose(f);
  return ok ? B2P_OK : B2P_ERR_IO;
}

int b2p_selector_load(b2p_selector s, const char *path) {
  if (!s || !path) return B2P_ERR_INVALID_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) return B2P_ERR_IO;
  char magic[8], gpu[64], ver[32];
  uint32_t np = 0;
  std::vector<float> h(kP);
  bool ok = fread(magic, 1, 8, f) == 8 && fread(&np, 4, 1, f) == 1 && fread(gpu, 1, 64, f) == 64 &&
            fread(ver, 1, 32, f) == 32 && np == (uint32_t)kP &&
            fread(h.data(), sizeof(float), kP, f) == (size_t)kP;
  fclose(f);
  if (!ok || memcmp(magic, kMagic, 8) != 0) return B2P_ERR_IO;
  gpu[63] = 0;
  ver[31] = 0;
  // weights are only valid for the GPU model and library they were trained on
  if (strncmp(gpu, device_info().name, 63) != 0 || strncmp(ver, b2p_version(), 31) != 0)
    return B2P_ERR_IO;
  return b2p_selector_set_params(s, h.data());
}

int b2p_selector_install(b2p_selector s) {
  if (!s) {
    clear_auto_table();
    return B2P_OK;
  }
  // decisions over the table's grid of shapes, one batched inference launch
  AutoTable t;
  t.cfg.assign(AutoTable::size(), -1);
  std::vector<float> feats;
  std::vector<size_t> where;
  const int prims[7] = {B2P_PRIM_REDUCE, B2P_PRIM_SCAN, B2P_PRIM_COPY_IF, B2P_PRIM_HISTOGRAM,
                        B2P_PRIM_DOT, B2P_PRIM_SEG_REDUCE, B2P_PRIM_SEG_SCAN};
  for (int prim : prims)
    for (int dt = 0; dt < 7; ++dt)
      for (int lb = 0; lb < AutoTable::kLogSteps; ++lb)
        for (int sb = 0; sb < AutoTable::kSegBuckets; ++sb)
          for (int cb = 0; cb < AutoTable::kCvBuckets; ++cb) {
            const bool seg = prim == B2P_PRIM_SEG_REDUCE || prim == B2P_PRIM_SEG_SCAN;
            if (!seg && (sb || cb)) continue;
            if (seg && sb == 0) continue;
            const size_t n = (size_t)std::llround(std::exp2(lb / 4.0));
            const int64_t nseg = seg ? (int64_t)std::llround(std::exp2(2.0 * (sb - 1) + 1.0)) : 1;
            float f[kF];
            b2p_selector_features(prim, dt, n, nseg, (cb + 0.5) / 2.0, f);
            feats.insert(feats.end(), f, f + kF);
            where.push_back(AutoTable::index(prim, dt, lb, sb, cb));
          }
  std::vector<int> cfg(where.size());
  int rc = b2p_selector_predict(s, feats.data(), (int)where.size(), cfg.data());
  if (rc) return rc;
  for (size_t i = 0; i < where.size(); ++i) t.cfg[where[i]] = (int16_t)cfg[i];
  // segmented entries without segments fall back to bucket 1
  t.valid = true;
  install_auto_table(t);
  return B2P_OK;
}

}  // extern "C"
