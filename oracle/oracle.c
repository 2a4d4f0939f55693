/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the evaluation order that AdaptiveCpp's OpenMP
 * (host) backend uses for the data-parallel primitive path, plus FP64
 * reference results for every floating-point primitive.  It is the checker
 * for the CUDA library and the timed CPU baseline; nothing in the product
 * links, loads or calls it.
 *
 * Parity pins: the integer results are pinned against the known answers of
 * the reference's own tests (tests/pstl/{reduce,transform_reduce,
 * inclusive_scan,exclusive_scan,copy_if}.cpp, tests/sycl/reduction.cpp,
 * tests/sycl/atomic.cpp) through tests/test_oracle_golden.py.  The reference
 * itself is not compiled here: its OMP nd_range path needs a generated
 * config header, the runtime library and Boost.Fiber.
 *
 * Citations are paths inside the AdaptiveCpp source tree.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).  FP
 * contraction is disabled so that a*b+c is two roundings, as in the
 * reference's separate transform and combine calls.
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* dtype codes — identical to b2p_dtype in include/b2p.h */
enum { D_I32 = 0, D_I64 = 1, D_U32 = 2, D_U64 = 3, D_F32 = 4, D_BF16 = 5, D_F64 = 6 };
/* op codes — identical to b2p_op in include/b2p.h */
enum { OP_SUM = 0, OP_PROD = 1, OP_MIN = 2, OP_MAX = 3, OP_AND = 4, OP_OR = 5, OP_XOR = 6 };

static inline float bf16_to_f32(uint16_t h) {
  uint32_t u = ((uint32_t)h) << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * Combine operators.  Integer arithmetic is done in the unsigned type of the
 * same width so that overflow wraps (two's complement) instead of being UB;
 * the reference's int accumulation wraps the same way on every target.
 *
 * min/max follow sycl::minimum / sycl::maximum
 * (include/hipSYCL/sycl/libkernel/functional.hpp): (x < y) ? x : y and
 * (x < y) ? y : x.
 * ---------------------------------------------------------------------- */
#define OP_EXPR_INT(U, op, a, b)                                              \
  ((op) == OP_SUM   ? (U)((U)(a) + (U)(b))                                    \
   : (op) == OP_PROD ? (U)((U)(a) * (U)(b))                                   \
   : (op) == OP_AND  ? (U)((U)(a) & (U)(b))                                   \
   : (op) == OP_OR   ? (U)((U)(a) | (U)(b))                                   \
   : (U)((U)(a) ^ (U)(b)))

/* ------------------------------------------------------------------------
 * Known identities: include/hipSYCL/algorithms/numeric.hpp:35-53.
 *   plus -> T{}, multiplies -> T{1}, minimum -> numeric_limits<T>::max(),
 *   maximum -> numeric_limits<T>::min()   (for float: FLT_MIN, the smallest
 *   positive normal — a quirk of the reference that this oracle keeps).
 * bit_and / bit_or / bit_xor have no entry, so they take the unknown-identity
 * path with initialization flags (reduction_engine / wi_reducer.hpp:59-70).
 * ---------------------------------------------------------------------- */

/* Thread count and id inside a parallel region (1 and 0 without OpenMP). */
#define DEFINE_THREAD_IDS(NAME)                                                \
  static inline void NAME##_thread_ids(size_t *nt, size_t *tid) {              \
    *nt = (size_t)omp_get_num_threads_or_1();                                  \
    *tid = (size_t)omp_get_thread_num_or_0();                                  \
  }

static inline int omp_get_num_threads_or_1(void) {
#ifdef _OPENMP
  return omp_get_num_threads();
#else
  return 1;
#endif
}
static inline int omp_get_thread_num_or_0(void) {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

/* Generic reduce generator.  T = accumulation type, IN = input element type,
 * CVT converts one input element to T. */
#define DEFINE_REDUCE(NAME, T, IN, CVT, COMBINE, IDENT_SUM, IDENT_PROD,        \
                      IDENT_MIN, IDENT_MAX)                                    \
  DEFINE_THREAD_IDS(NAME)                                                      \
  static T NAME##_comb(int op, T a, T b) { return COMBINE(op, a, b); }         \
  static int NAME##_ident(int op, T *id) {                                     \
    switch (op) {                                                              \
    case OP_SUM: *id = IDENT_SUM; return 1;                                    \
    case OP_PROD: *id = IDENT_PROD; return 1;                                  \
    case OP_MIN: *id = IDENT_MIN; return 1;                                    \
    case OP_MAX: *id = IDENT_MAX; return 1;                                    \
    default: return 0;                                                         \
    }                                                                          \
  }                                                                            \
  /* group tree over 128 work-items with init flags:                          \
   * wg_model/group_reduction_algorithms.hpp:139-189 */                        \
  static void NAME##_tree(int op, T *loc, int *flg) {                          \
    for (int i = 64; i > 0; i /= 2)                                            \
      for (int l = 0; l < i; ++l) {                                            \
        if (flg[l] && flg[l + i]) {                                            \
          loc[l] = NAME##_comb(op, loc[l], loc[l + i]);                        \
        } else if (flg[l + i]) {                                               \
          loc[l] = loc[l + i];                                                 \
          flg[l] = 1;                                                          \
        }                                                                      \
      }                                                                        \
  }                                                                            \
  /* OMP-backend reduce: numeric.hpp:67-161 with util/memory_streaming.hpp    \
   * run_host (8 contiguous elements per work-item, :93-113), WG = 128        \
   * (:144), then dedicated 128-wide stage kernels                            \
   * (reduction_engine.hpp:123-191).  Returns 1 if the result is initialized. \
   * X2 non-NULL: binary transform X[i]*X2[i] (transform_reduce dot form,     \
   * numeric.hpp:170-192,215-223). */                                          \
  static int NAME##_omp_reduce(int op, const IN *x, const IN *x2, size_t n,   \
                               T *res) {                                       \
    T ident;                                                                   \
    int known = NAME##_ident(op, &ident);                                      \
    if (!known) memset(&ident, 0, sizeof(T));                                  \
    size_t items = (n + 127) / 128;                                            \
    size_t G = (items + 7) / 8;                                                \
    if (G > items) G = items;                                                  \
    T *part = (T *)malloc(sizeof(T) * (G ? G : 1));                            \
    int *pflag = (int *)malloc(sizeof(int) * (G ? G : 1));                     \
    _Pragma("omp parallel for schedule(static)")                               \
    for (size_t g = 0; g < G; ++g) {                                           \
      T loc[128];                                                              \
      int flg[128];                                                            \
      for (int l = 0; l < 128; ++l) {                                          \
        size_t gid = g * 128 + (size_t)l;                                      \
        T v = ident;                                                           \
        int init = known;                                                      \
        for (int i = 0; i < 8; ++i) {                                          \
          size_t pos = 8 * gid + (size_t)i;                                    \
          if (g != G - 1 || pos < n) {                                         \
            T e = x2 ? (T)(CVT(x[pos]) * CVT(x2[pos])) : CVT(x[pos]);          \
            if (init) v = NAME##_comb(op, v, e);                               \
            else { v = e; init = 1; }                                          \
          }                                                                    \
        }                                                                      \
        loc[l] = v;                                                            \
        flg[l] = init;                                                         \
      }                                                                        \
      NAME##_tree(op, loc, flg);                                               \
      part[g] = loc[0];                                                        \
      pflag[g] = flg[0];                                                       \
    }                                                                          \
    size_t m = G;                                                              \
    while (m > 1) {                                                            \
      size_t G2 = (m + 127) / 128;                                             \
      T *p2 = (T *)malloc(sizeof(T) * G2);                                     \
      int *f2 = (int *)malloc(sizeof(int) * G2);                               \
      for (size_t g = 0; g < G2; ++g) {                                        \
        T loc[128];                                                            \
        int flg[128];                                                          \
        for (int l = 0; l < 128; ++l) {                                        \
          size_t id = g * 128 + (size_t)l;                                     \
          T v = ident;                                                         \
          int init = known;                                                    \
          if (id < m && (known || pflag[id])) {                                \
            if (init) v = NAME##_comb(op, v, part[id]);                        \
            else { v = part[id]; init = 1; }                                   \
          }                                                                    \
          loc[l] = v;                                                          \
          flg[l] = init;                                                       \
        }                                                                      \
        NAME##_tree(op, loc, flg);                                             \
        p2[g] = loc[0];                                                        \
        f2[g] = flg[0];                                                        \
      }                                                                        \
      free(part);                                                              \
      free(pflag);                                                             \
      part = p2;                                                               \
      pflag = f2;                                                              \
      m = G2;                                                                  \
    }                                                                          \
    int ok = G ? pflag[0] : 0;                                                 \
    if (G) *res = part[0];                                                     \
    free(part);                                                                \
    free(pflag);                                                               \
    return ok;                                                                 \
  }                                                                            \
  /* OMP-backend scan: algorithms/scan/scan.hpp:26-32 (WG 1024 on OMP),       \
   * decoupled_lookback_scan.hpp:137-177 (one leader scans the 16*1024        \
   * tile sequentially into local memory, finds the tile's exclusive prefix,  \
   * then writes op(prefix, local[i]) -- one write per element), :219-257     \
   * (look-back; here the predecessor's inclusive prefix, so the carries     \
   * form the serial chain prefix[g] = op(prefix[g-1], agg[g]) whatever the   \
   * timing), :259-277 (exclusive = shifted inclusive with x[-1] := init;     \
   * out-of-range generator ids clamp to n-1, scan.hpp:58-66).  Threads take  \
   * tiles round-robin and each waits only for its predecessor's prefix,      \
   * which is published as soon as that tile's local scan is done. */         \
  static void NAME##_omp_scan(int op, int inclusive, const IN *x, T *y,       \
                              size_t n, const T *init) {                       \
    const size_t TILE = 16 * 1024;                                             \
    size_t ntiles = ((n + 15) / 16 + 1023) / 1024;                             \
    T *pre = (T *)malloc(sizeof(T) * ntiles);                                  \
    int *ready = (int *)calloc(ntiles, sizeof(int));                           \
    _Pragma("omp parallel")                                                    \
    {                                                                          \
      size_t nt = 1, tid = 0;                                                  \
      NAME##_thread_ids(&nt, &tid);                                            \
      T *loc = (T *)malloc(sizeof(T) * TILE);                                  \
      for (size_t g = tid; g < ntiles; g += nt) {                              \
        T cur;                                                                 \
        memset(&cur, 0, sizeof(T));                                            \
        for (size_t i = 0; i < TILE; ++i) {                                    \
          size_t gid = g * TILE + i;                                           \
          T e;                                                                 \
          if (inclusive) {                                                     \
            size_t src = gid < n ? gid : n - 1;                                \
            e = CVT(x[src]);                                                   \
            if (init && gid == 0) e = NAME##_comb(op, *init, e);               \
          } else {                                                             \
            if (gid == 0) e = *init;                                           \
            else {                                                             \
              size_t src = gid - 1 < n ? gid - 1 : n - 1;                      \
              e = CVT(x[src]);                                                 \
            }                                                                  \
          }                                                                    \
          cur = (i == 0) ? e : NAME##_comb(op, cur, e);                        \
          loc[i] = cur;                                                        \
        }                                                                      \
        if (g == 0) {                                                          \
          pre[0] = cur;                                                        \
        } else {                                                               \
          while (!__atomic_load_n(&ready[g - 1], __ATOMIC_ACQUIRE))            \
            __builtin_ia32_pause();                                            \
          pre[g] = NAME##_comb(op, pre[g - 1], cur);                           \
        }                                                                      \
        __atomic_store_n(&ready[g], 1, __ATOMIC_RELEASE);                      \
        size_t end = (g + 1) * TILE < n ? (g + 1) * TILE : n;                  \
        if (g == 0) {                                                          \
          for (size_t gid = 0; gid < end; ++gid) y[gid] = loc[gid];            \
        } else {                                                               \
          T p = pre[g - 1];                                                    \
          for (size_t gid = g * TILE; gid < end; ++gid)                        \
            y[gid] = NAME##_comb(op, p, loc[gid - g * TILE]);                  \
        }                                                                      \
      }                                                                        \
      free(loc);                                                               \
    }                                                                          \
    free(pre);                                                                 \
    free(ready);                                                               \
  }

#define COMB_INT(U) (U)
#define IDENT(x) (x)

/* integer combine helpers */
static inline int32_t comb_i32(int op, int32_t a, int32_t b) {
  if (op == OP_MIN) return (a < b) ? a : b;
  if (op == OP_MAX) return (a < b) ? b : a;
  return (int32_t)OP_EXPR_INT(uint32_t, op, a, b);
}
static inline int64_t comb_i64(int op, int64_t a, int64_t b) {
  if (op == OP_MIN) return (a < b) ? a : b;
  if (op == OP_MAX) return (a < b) ? b : a;
  return (int64_t)OP_EXPR_INT(uint64_t, op, a, b);
}
static inline uint32_t comb_u32(int op, uint32_t a, uint32_t b) {
  if (op == OP_MIN) return (a < b) ? a : b;
  if (op == OP_MAX) return (a < b) ? b : a;
  return OP_EXPR_INT(uint32_t, op, a, b);
}
static inline uint64_t comb_u64(int op, uint64_t a, uint64_t b) {
  if (op == OP_MIN) return (a < b) ? a : b;
  if (op == OP_MAX) return (a < b) ? b : a;
  return OP_EXPR_INT(uint64_t, op, a, b);
}
static inline float comb_f32(int op, float a, float b) {
  switch (op) {
  case OP_SUM: return a + b;
  case OP_PROD: return a * b;
  case OP_MIN: return (a < b) ? a : b;
  default: return (a < b) ? b : a;
  }
}
static inline double comb_f64(int op, double a, double b) {
  switch (op) {
  case OP_SUM: return a + b;
  case OP_PROD: return a * b;
  case OP_MIN: return (a < b) ? a : b;
  default: return (a < b) ? b : a;
  }
}

#define CVT_ID(v) (v)
#define CVT_BF16(v) bf16_to_f32(v)

DEFINE_REDUCE(i32, int32_t, int32_t, CVT_ID, comb_i32, 0, 1, INT32_MAX, INT32_MIN)
DEFINE_REDUCE(i64, int64_t, int64_t, CVT_ID, comb_i64, 0, 1, INT64_MAX, INT64_MIN)
DEFINE_REDUCE(u32, uint32_t, uint32_t, CVT_ID, comb_u32, 0u, 1u, UINT32_MAX, 0u)
DEFINE_REDUCE(u64, uint64_t, uint64_t, CVT_ID, comb_u64, 0u, 1u, UINT64_MAX, 0u)
DEFINE_REDUCE(f32, float, float, CVT_ID, comb_f32, 0.0f, 1.0f, FLT_MAX, FLT_MIN)
DEFINE_REDUCE(bf16, float, uint16_t, CVT_BF16, comb_f32, 0.0f, 1.0f, FLT_MAX, FLT_MIN)
DEFINE_REDUCE(f64, double, double, CVT_ID, comb_f64, 0.0, 1.0, DBL_MAX, DBL_MIN)

/* ------------------------------------------------------------------------
 * Public oracle entry points (ctypes).  Return 0 on success, -1 on a bad
 * dtype/op.  For n == 0 the output is left untouched, as the reference does
 * (numeric.hpp:165-169, 178-179).
 * ---------------------------------------------------------------------- */

/* hipsycl::algorithms::reduce / transform_reduce with a known-identity or
 * unknown-identity operator; *out = op(init, r) (reduction_descriptor.hpp:36-38).
 * For BF16 input, init/out are float. */
int orc_reduce(int dtype, int op, const void *x, size_t n, const void *init,
               void *out) {
  if (n == 0) return 0;
#define RED_CASE(D, NAME, T, IN)                                              \
  case D: {                                                                    \
    T r;                                                                       \
    int ok = NAME##_omp_reduce(op, (const IN *)x, NULL, n, &r);                \
    T iv = *(const T *)init;                                                   \
    *(T *)out = ok ? NAME##_comb(op, iv, r) : iv;                              \
    return 0;                                                                  \
  }
  switch (dtype) {
    RED_CASE(D_I32, i32, int32_t, int32_t)
    RED_CASE(D_I64, i64, int64_t, int64_t)
    RED_CASE(D_U32, u32, uint32_t, uint32_t)
    RED_CASE(D_U64, u64, uint64_t, uint64_t)
    RED_CASE(D_F32, f32, float, float)
    RED_CASE(D_BF16, bf16, float, uint16_t)
    RED_CASE(D_F64, f64, double, double)
  default: return -1;
  }
#undef RED_CASE
}

/* transform_reduce(first1, last1, first2, out, init) with plus/multiplies
 * (numeric.hpp:215-223): each work-item combines a[i]*b[i] rounded to the
 * accumulation type. */
int orc_dot(int dtype, const void *a, const void *b, size_t n, const void *init,
            void *out) {
  if (n == 0) return 0;
  switch (dtype) {
  case D_F32: {
    float r;
    f32_omp_reduce(OP_SUM, (const float *)a, (const float *)b, n, &r);
    *(float *)out = *(const float *)init + r;
    return 0;
  }
  case D_BF16: {
    float r;
    bf16_omp_reduce(OP_SUM, (const uint16_t *)a, (const uint16_t *)b, n, &r);
    *(float *)out = *(const float *)init + r;
    return 0;
  }
  case D_F64: {
    double r;
    f64_omp_reduce(OP_SUM, (const double *)a, (const double *)b, n, &r);
    *(double *)out = *(const double *)init + r;
    return 0;
  }
  default: return -1;
  }
}

/* inclusive_scan / exclusive_scan (numeric.hpp:251-297).  init may be NULL
 * for an inclusive scan without init.  For BF16 input, y and init are float. */
int orc_scan(int dtype, int op, int inclusive, const void *x, void *y, size_t n,
             const void *init) {
  if (n == 0) return 0;
  if (!inclusive && !init) return -1;
  switch (dtype) {
  case D_I32: i32_omp_scan(op, inclusive, (const int32_t *)x, (int32_t *)y, n, (const int32_t *)init); return 0;
  case D_I64: i64_omp_scan(op, inclusive, (const int64_t *)x, (int64_t *)y, n, (const int64_t *)init); return 0;
  case D_U32: u32_omp_scan(op, inclusive, (const uint32_t *)x, (uint32_t *)y, n, (const uint32_t *)init); return 0;
  case D_U64: u64_omp_scan(op, inclusive, (const uint64_t *)x, (uint64_t *)y, n, (const uint64_t *)init); return 0;
  case D_F32: f32_omp_scan(op, inclusive, (const float *)x, (float *)y, n, (const float *)init); return 0;
  case D_BF16: bf16_omp_scan(op, inclusive, (const uint16_t *)x, (float *)y, n, (const float *)init); return 0;
  case D_F64: f64_omp_scan(op, inclusive, (const double *)x, (double *)y, n, (const double *)init); return 0;
  default: return -1;
  }
}

/* copy_if (algorithms/algorithm.hpp:178-243): order-preserving compaction via
 * an exclusive size_t scan of predicate flags; count = excl[n-1] + pred(x[n-1]).
 * Predicate family used by the C-ABI: (x & mask) CMP rhs, with CMP codes
 * 0:<  1:<=  2:==  3:!=  4:>=  5:>.  Parallel: per-block counts, serial
 * offsets, per-block scatter — identical output to any correct compaction. */
static inline int pred_u32(uint32_t v, uint32_t mask, int cmp, uint32_t rhs) {
  uint32_t a = v & mask;
  switch (cmp) {
  case 0: return a < rhs;
  case 1: return a <= rhs;
  case 2: return a == rhs;
  case 3: return a != rhs;
  case 4: return a >= rhs;
  default: return a > rhs;
  }
}

int orc_copy_if_u32(const uint32_t *x, size_t n, uint32_t mask, int cmp,
                    uint32_t rhs, uint32_t *out, uint64_t *count) {
  if (n == 0) { if (count) *count = 0; return 0; }
  const size_t B = 1 << 16;
  size_t nb = (n + B - 1) / B;
  uint64_t *cnt = (uint64_t *)calloc(nb + 1, sizeof(uint64_t));
  _Pragma("omp parallel for schedule(static)")
  for (size_t b = 0; b < nb; ++b) {
    size_t end = (b + 1) * B < n ? (b + 1) * B : n;
    uint64_t c = 0;
    for (size_t i = b * B; i < end; ++i) c += pred_u32(x[i], mask, cmp, rhs);
    cnt[b + 1] = c;
  }
  for (size_t b = 0; b < nb; ++b) cnt[b + 1] += cnt[b];
  _Pragma("omp parallel for schedule(static)")
  for (size_t b = 0; b < nb; ++b) {
    size_t end = (b + 1) * B < n ? (b + 1) * B : n;
    uint64_t o = cnt[b];
    for (size_t i = b * B; i < end; ++i)
      if (pred_u32(x[i], mask, cmp, rhs)) out[o++] = x[i];
  }
  if (count) *count = cnt[nb];
  free(cnt);
  return 0;
}

/* Histogram through atomic_ref<uint32_t>::fetch_add(1) on bins[key]
 * (sycl/libkernel/atomic_ref.hpp:143-149): counts are added to the existing
 * bin values, modulo 2^32.  Keys >= nbins are skipped, matching the C-ABI. */
int orc_histogram_u8(const uint8_t *keys, size_t n, uint32_t *bins, int nbins) {
  int nt = orc_num_threads();
  uint32_t *loc = (uint32_t *)calloc((size_t)nt * 256, sizeof(uint32_t));
  _Pragma("omp parallel")
  {
#ifdef _OPENMP
    int t = omp_get_thread_num();
#else
    int t = 0;
#endif
    uint32_t *h = loc + (size_t)t * 256;
    _Pragma("omp for schedule(static)")
    for (size_t i = 0; i < n; ++i) h[keys[i]]++;
  }
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < nbins && k < 256; ++k) bins[k] += loc[(size_t)t * 256 + k];
  free(loc);
  return 0;
}

/* Segmented primitives: the reference has no segmented entry point; its
 * analogue is one reduce / inclusive_scan call per CSR segment.  Reduce uses
 * init = T{} (the reduce(q, s, first, last, out) overload, numeric.hpp:242-249)
 * and writes T{} for an empty segment. */
int orc_segmented_reduce(int dtype, int op, const void *x, const int64_t *offs,
                         int64_t nseg, void *out) {
  size_t es = (dtype == D_I64 || dtype == D_U64 || dtype == D_F64) ? 8 : (dtype == D_BF16 ? 2 : 4);
  size_t os = (dtype == D_BF16) ? 4 : es;
  char zero[8] = {0};
  if (op == OP_PROD) {
    if (dtype == D_F32 || dtype == D_BF16) { float one = 1.0f; memcpy(zero, &one, 4); }
    else if (dtype == D_F64) { double one = 1.0; memcpy(zero, &one, 8); }
    else if (es == 8) { int64_t one = 1; memcpy(zero, &one, 8); }
    else { int32_t one = 1; memcpy(zero, &one, 4); }
  }
  for (int64_t s = 0; s < nseg; ++s) {
    size_t b = (size_t)offs[s], e = (size_t)offs[s + 1];
    char *o = (char *)out + (size_t)s * os;
    memcpy(o, zero, os);
    if (e > b) {
      int rc = orc_reduce(dtype, op, (const char *)x + b * es, e - b, zero, o);
      if (rc) return rc;
    }
  }
  return 0;
}

int orc_segmented_scan(int dtype, int op, int inclusive, const void *x,
                       const int64_t *offs, int64_t nseg, void *y, const void *init) {
  size_t es = (dtype == D_I64 || dtype == D_U64 || dtype == D_F64) ? 8 : (dtype == D_BF16 ? 2 : 4);
  size_t os = (dtype == D_BF16) ? 4 : es;
  for (int64_t s = 0; s < nseg; ++s) {
    size_t b = (size_t)offs[s], e = (size_t)offs[s + 1];
    if (e > b) {
      int rc = orc_scan(dtype, op, inclusive, (const char *)x + b * es, (char *)y + b * os, e - b, init);
      if (rc) return rc;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * FP64 oracle.  Double-double (Ogita–Rump–Oishi Sum2 / Dot2, 2005) over the
 * exact fp32 (or bf16-rounded) input values.  A fp32 product is exact in
 * double, so Dot2 here only needs TwoSum.  Work is chunked at a fixed 2^16
 * granularity, so the result does not depend on the thread count.
 * ---------------------------------------------------------------------- */
typedef struct { double hi, lo; } dd_t;

static inline dd_t dd_add_d(dd_t a, double b) {
  double s = a.hi + b;
  double bp = s - a.hi;
  double e = (a.hi - (s - bp)) + (b - bp);
  dd_t r = {s, a.lo + e};
  return r;
}
static inline dd_t dd_add(dd_t a, dd_t b) {
  dd_t r = dd_add_d(a, b.hi);
  r.lo += b.lo;
  double s = r.hi + r.lo;
  double e = r.lo - (s - r.hi);
  r.hi = s;
  r.lo = e;
  return r;
}
static inline double elem_f64(int dtype, const void *x, size_t i) {
  switch (dtype) {
  case D_F32: return (double)((const float *)x)[i];
  case D_BF16: return (double)bf16_to_f32(((const uint16_t *)x)[i]);
  case D_F64: return ((const double *)x)[i];
  case D_I32: return (double)((const int32_t *)x)[i];
  case D_I64: return (double)((const int64_t *)x)[i];
  case D_U32: return (double)((const uint32_t *)x)[i];
  default: return (double)((const uint64_t *)x)[i];
  }
}

/* sum (b == NULL) or dot (b != NULL); also returns sum |x_i| (|a_i b_i|) */
int orc_fp64_sum(int dtype, const void *a, const void *b, size_t n, double init,
                 double *out_hi, double *out_lo, double *out_abs) {
  const size_t C = 1 << 16;
  size_t nc = (n + C - 1) / C;
  dd_t *part = (dd_t *)calloc(nc ? nc : 1, sizeof(dd_t));
  double *pabs = (double *)calloc(nc ? nc : 1, sizeof(double));
  _Pragma("omp parallel for schedule(static)")
  for (size_t c = 0; c < nc; ++c) {
    size_t end = (c + 1) * C < n ? (c + 1) * C : n;
    dd_t s = {0.0, 0.0};
    double sa = 0.0;
    for (size_t i = c * C; i < end; ++i) {
      double v = elem_f64(dtype, a, i);
      if (b) v *= elem_f64(dtype, b, i); /* exact for fp32/bf16 inputs */
      s = dd_add_d(s, v);
      sa += fabs(v);
    }
    part[c] = s;
    pabs[c] = sa;
  }
  dd_t tot = {init, 0.0};
  double ta = fabs(init);
  for (size_t c = 0; c < nc; ++c) { tot = dd_add(tot, part[c]); ta += pabs[c]; }
  free(part);
  free(pabs);
  if (out_hi) *out_hi = tot.hi;
  if (out_lo) *out_lo = tot.lo;
  if (out_abs) *out_abs = ta;
  return 0;
}

/* inclusive (or exclusive with init) prefix sums in double-double, rounded to
 * double per element. */
int orc_fp64_scan(int dtype, int inclusive, const void *x, size_t n, double init,
                  double *y) {
  const size_t C = 1 << 16;
  size_t nc = (n + C - 1) / C;
  dd_t *part = (dd_t *)calloc(nc + 1, sizeof(dd_t));
  _Pragma("omp parallel for schedule(static)")
  for (size_t c = 0; c < nc; ++c) {
    size_t end = (c + 1) * C < n ? (c + 1) * C : n;
    dd_t s = {0.0, 0.0};
    for (size_t i = c * C; i < end; ++i) s = dd_add_d(s, elem_f64(dtype, x, i));
    part[c + 1] = s;
  }
  part[0].hi = init;
  part[0].lo = 0.0;
  for (size_t c = 1; c <= nc; ++c) part[c] = dd_add(part[c - 1], part[c]);
  _Pragma("omp parallel for schedule(static)")
  for (size_t c = 0; c < nc; ++c) {
    size_t end = (c + 1) * C < n ? (c + 1) * C : n;
    dd_t s = part[c];
    for (size_t i = c * C; i < end; ++i) {
      double v = elem_f64(dtype, x, i);
      if (inclusive) {
        s = dd_add_d(s, v);
        y[i] = s.hi + s.lo;
      } else {
        y[i] = s.hi + s.lo;
        s = dd_add_d(s, v);
      }
    }
  }
  free(part);
  return 0;
}

/* Segmented FP64 oracle: per-segment double-double sum. */
int orc_fp64_segmented_sum(int dtype, const void *x, const int64_t *offs,
                           int64_t nseg, double *out) {
  _Pragma("omp parallel for schedule(dynamic, 16)")
  for (int64_t s = 0; s < nseg; ++s) {
    dd_t t = {0.0, 0.0};
    for (int64_t i = offs[s]; i < offs[s + 1]; ++i) t = dd_add_d(t, elem_f64(dtype, x, (size_t)i));
    out[s] = t.hi + t.lo;
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * Seeded synthetic inputs, bit-identical to the library's b2p_synth_fill
 * (include/b2p.h): SplitMix64 finaliser over (seed, index, stream), uniform
 * on (0, 1] from the top 53 bits, Box-Muller in double rounded once, bf16 by
 * round-to-nearest-even, truncated Zipf keys by an inverse-CDF table.  The
 * CPU baseline and the reference arm of the benchmark generate their inputs
 * with this, so that they load nothing but this library;
 * tests/test_oracle_golden.py checks that both generators agree.
 * ---------------------------------------------------------------------- */
static inline uint64_t syn_mix(uint64_t seed, uint64_t i, uint64_t stream) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + (i + 1) * 0xD1B54A32D192ED03ull +
               (stream + 1) * 0x8CB92BA72F3D8DD7ull;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline double syn_unif(uint64_t seed, uint64_t i, uint64_t stream) {
  return (double)((syn_mix(seed, i, stream) >> 11) + 1) * 0x1.0p-53;
}
static inline double syn_normal(uint64_t seed, uint64_t i, uint64_t s0) {
  const double u1 = syn_unif(seed, i, s0), u2 = syn_unif(seed, i, s0 + 1);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
static inline float syn_mixed_normal(uint64_t seed, uint64_t i, double frac, double scale) {
  if (frac > 0.0 && syn_unif(seed, i, 3) <= frac) return (float)(scale * syn_normal(seed, i, 4));
  return (float)syn_normal(seed, i, 1);
}
static inline uint16_t syn_bf16_rne(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

/* kinds as b2p_synth_fill: 0 int32 U[a,b], 1 fp32 N(0,1) with a fraction a
 * scaled by b, 2 |kind 1|, 3 uint32, 4 uint8 Zipf(a), 5 int64 U[a,b],
 * 6 / 7 bf16 bits of kinds 1 / 2.  Returns 0, or -1 for a bad kind. */
int orc_synth_fill(int kind, uint64_t seed, size_t n, double a, double b, void *out) {
  const long long N = (long long)n;
  switch (kind) {
  case 0:
  case 5: {
    const long long lo = (long long)a, span = (long long)b - lo + 1;
    if (span <= 0) return -1;
    _Pragma("omp parallel for schedule(static)")
    for (long long i = 0; i < N; ++i) {
      const long long v = lo + (long long)(syn_mix(seed, (uint64_t)i, 0) % (uint64_t)span);
      if (kind == 0) ((int32_t *)out)[i] = (int32_t)v;
      else ((int64_t *)out)[i] = (int64_t)v;
    }
    return 0;
  }
  case 1:
  case 2: {
    float *o = (float *)out;
    _Pragma("omp parallel for schedule(static)")
    for (long long i = 0; i < N; ++i) {
      float v = syn_mixed_normal(seed, (uint64_t)i, a, b);
      o[i] = kind == 2 ? fabsf(v) : v;
    }
    return 0;
  }
  case 3: {
    uint32_t *o = (uint32_t *)out;
    _Pragma("omp parallel for schedule(static)")
    for (long long i = 0; i < N; ++i) o[i] = (uint32_t)(syn_mix(seed, (uint64_t)i, 0) >> 32);
    return 0;
  }
  case 4: {
    const double s = a > 0 ? a : 1.2;
    double cdf[256], acc = 0.0;
    for (int r = 1; r <= 256; ++r) {
      acc += pow((double)r, -s);
      cdf[r - 1] = acc;
    }
    for (int r = 0; r < 256; ++r) cdf[r] /= acc;
    cdf[255] = 1.0;
    uint8_t *o = (uint8_t *)out;
    _Pragma("omp parallel for schedule(static)")
    for (long long i = 0; i < N; ++i) {
      const double u = syn_unif(seed, (uint64_t)i, 0);
      int lo = 0, hi = 256; /* first k with cdf[k] >= u */
      while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (cdf[mid] < u) lo = mid + 1;
        else hi = mid;
      }
      o[i] = (uint8_t)(lo > 255 ? 255 : lo);
    }
    return 0;
  }
  case 6:
  case 7: {
    uint16_t *o = (uint16_t *)out;
    _Pragma("omp parallel for schedule(static)")
    for (long long i = 0; i < N; ++i) {
      float v = syn_mixed_normal(seed, (uint64_t)i, a, b);
      o[i] = syn_bf16_rne(kind == 7 ? fabsf(v) : v);
    }
    return 0;
  }
  default:
    return -1;
  }
}
