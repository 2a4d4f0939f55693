// Seeded synthetic workloads for the benchmark, the autotuner and the tests
// (b2p_synth_fill / b2p_synth_segments in include/b2p.h).
//
// Counter-based: element i of stream k is a pure function of (seed, i, k),
// computed with the SplitMix64 finaliser (Steele, Lea, Flood 2014), so the
// output does not depend on the number of host threads.  Normal variates use
// the Box-Muller transform in double precision, rounded once to the storage
// type.  The truncated Zipf keys use an inverse-CDF table.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../../include/b2p.h"

namespace {

inline uint64_t mix(uint64_t seed, uint64_t i, uint64_t stream) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + (i + 1) * 0xD1B54A32D192ED03ull +
               (stream + 1) * 0x8CB92BA72F3D8DD7ull;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// uniform on (0, 1]
inline double unif(uint64_t seed, uint64_t i, uint64_t stream) {
  return (double)((mix(seed, i, stream) >> 11) + 1) * 0x1.0p-53;
}

inline double normal(uint64_t seed, uint64_t i, uint64_t s0) {
  const double u1 = unif(seed, i, s0), u2 = unif(seed, i, s0 + 1);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

inline uint16_t f32_to_bf16_rne(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);  // NaN stays NaN
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

inline float mixed_normal(uint64_t seed, uint64_t i, double frac, double scale) {
  if (frac > 0.0 && unif(seed, i, 3) <= frac) return (float)(scale * normal(seed, i, 4));
  return (float)normal(seed, i, 1);
}

}  // namespace

extern "C" int b2p_synth_fill(int kind, uint64_t seed, size_t n, double a, double b,
                              void *host_out) {
  if (!host_out && n) return B2P_ERR_INVALID_ARG;
  const long long N = (long long)n;
  switch (kind) {
  case 0: {
    int32_t *o = (int32_t *)host_out;
    const long long lo = (long long)a, span = (long long)b - lo + 1;
    if (span <= 0) return B2P_ERR_INVALID_ARG;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) o[i] = (int32_t)(lo + (long long)(mix(seed, i, 0) % (uint64_t)span));
    return B2P_OK;
  }
  case 1:
  case 2: {
    float *o = (float *)host_out;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
      float v = mixed_normal(seed, (uint64_t)i, a, b);
      o[i] = kind == 2 ? std::fabs(v) : v;
    }
    return B2P_OK;
  }
  case 3: {
    uint32_t *o = (uint32_t *)host_out;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) o[i] = (uint32_t)(mix(seed, i, 0) >> 32);
    return B2P_OK;
  }
  case 4: {
    const double s = a > 0 ? a : 1.2;
    double cdf[256];
    double acc = 0.0;
    for (int r = 1; r <= 256; ++r) {
      acc += std::pow((double)r, -s);
      cdf[r - 1] = acc;
    }
    for (int r = 0; r < 256; ++r) cdf[r] /= acc;
    cdf[255] = 1.0;
    uint8_t *o = (uint8_t *)host_out;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
      const double u = unif(seed, (uint64_t)i, 0);
      int k = (int)(std::lower_bound(cdf, cdf + 256, u) - cdf);
      o[i] = (uint8_t)(k > 255 ? 255 : k);
    }
    return B2P_OK;
  }
  case 5: {
    int64_t *o = (int64_t *)host_out;
    const long long lo = (long long)a, span = (long long)b - lo + 1;
    if (span <= 0) return B2P_ERR_INVALID_ARG;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) o[i] = (int64_t)(lo + (long long)(mix(seed, i, 0) % (uint64_t)span));
    return B2P_OK;
  }
  case 6:
  case 7: {
    uint16_t *o = (uint16_t *)host_out;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
      float v = mixed_normal(seed, (uint64_t)i, a, b);
      o[i] = f32_to_bf16_rne(kind == 7 ? std::fabs(v) : v);
    }
    return B2P_OK;
  }
  default:
    return B2P_ERR_INVALID_ARG;
  }
}

extern "C" int b2p_synth_segments(uint64_t seed, int64_t nseg, double log2max, uint64_t cap,
                                  int64_t *offsets, uint64_t *total) {
  if (nseg < 0 || !offsets) return B2P_ERR_INVALID_ARG;
  std::vector<double> len((size_t)nseg);
  double sum = 0.0;
  for (int64_t s = 0; s < nseg; ++s) {
    const double u = (double)(mix(seed, (uint64_t)s, 0) >> 11) * 0x1.0p-53;  // [0, 1)
    len[(size_t)s] = std::max(1.0, std::floor(std::exp2(log2max * u)));
    sum += len[(size_t)s];
  }
  if (cap > 0 && sum > (double)cap) {
    const double f = (double)cap / sum;
    for (auto &l : len) l = std::max(1.0, std::floor(l * f));
  }
  offsets[0] = 0;
  for (int64_t s = 0; s < nseg; ++s) offsets[s + 1] = offsets[s] + (int64_t)len[(size_t)s];
  // the max(1, .) floor can push the total past the cap: trim the longest segment
  if (cap > 0 && (uint64_t)offsets[nseg] > cap && nseg > 0) {
    const int64_t excess = offsets[nseg] - (int64_t)cap;
    size_t big = (size_t)(std::max_element(len.begin(), len.end()) - len.begin());
    len[big] = std::max(1.0, len[big] - (double)excess);
    for (int64_t s = 0; s < nseg; ++s) offsets[s + 1] = offsets[s] + (int64_t)len[(size_t)s];
  }
  if (total) *total = (uint64_t)offsets[nseg];
  return B2P_OK;
}
