// C++ drop-in layer tests (compiled with nvcc, run on one GPU): the
// algorithms library signatures, sycl::reduction in parallel_for, group
// algorithms, atomic_ref and the stdpar overloads.  The cases follow the
// reference's own tests (tests/pstl/{reduce,transform_reduce,
// inclusive_scan,exclusive_scan,copy_if,sort,merge}.cpp, tests/sycl/reduction.cpp,
// tests/sycl/group_functions/group_functions_{reduce,scan}.cpp,
// tests/sycl/atomic.cpp); expected values are computed here on the host.
// Prints one line per failure and "ALL PASSED <n>" at the end; exit code 0
// only when every check passed.
#include <hipSYCL_b2p/stdpar.hpp>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <functional>
#include <random>
#include <string>
#include <vector>

namespace alg = hipsycl::algorithms;

static int g_checks = 0, g_fail = 0;
#define CHECK(cond, ...)                         \
  do {                                           \
    ++g_checks;                                  \
    if (!(cond)) {                               \
      ++g_fail;                                  \
      std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
      std::printf(__VA_ARGS__);                  \
      std::printf("\n");                         \
    }                                            \
  } while (0)

template <class T>
static std::vector<T> from_dev(sycl::queue &q, const T *d, size_t n) {
  std::vector<T> h(n);
  if (n) q.memcpy(h.data(), d, n * sizeof(T)).wait();
  return h;
}
template <class T>
static T *to_dev(sycl::queue &q, const std::vector<T> &h) {
  T *d = sycl::malloc_device<T>(h.size() ? h.size() : 1, q);
  if (!h.empty()) q.memcpy(d, h.data(), h.size() * sizeof(T)).wait();
  return d;
}

// ------------------------------------------------------ algorithms library

static void test_algorithms(sycl::queue &q) {
  alg::util::allocation_cache cache{alg::util::allocation_type::device};
  for (size_t n : {0ul, 1ul, 127ul, 1000ul, 1000000ul}) {
    std::vector<int> h(n);
    std::iota(h.begin(), h.end(), 0);
    int *d = to_dev(q, h);
    int *out = sycl::malloc_shared<int>(1, q);
    *out = -7;
    {
      alg::util::allocation_group g{&cache, q.get_device()};
      alg::reduce(q, g, d, d + n, out, 10).wait();
      const long long ref = 10 + (long long)n * (n ? n - 1 : 0) / 2;
      if (n == 0) CHECK(*out == -7, "reduce n=0 touched *out");
      else CHECK(*out == (int)ref, "reduce iota n=%zu got %d want %lld", n, *out, ref);
    }
    {
      // user operator (generic kernels)
      alg::util::allocation_group g{&cache, q.get_device()};
      auto op = [] __host__ __device__(int a, int b) { return a > b ? a : b; };
      if (n) {
        alg::reduce(q, g, d, d + n, out, -1, op).wait();
        CHECK(*out == (int)n - 1, "reduce max lambda n=%zu got %d", n, *out);
      }
    }
    {
      // transform_reduce, unary transform (generic) and dot form on doubles
      alg::util::allocation_group g{&cache, q.get_device()};
      if (n) {
        long long *lo = sycl::malloc_shared<long long>(1, q);
        alg::transform_reduce(q, g, d, d + n, lo, 0ll, std::plus<long long>{},
                              [] __host__ __device__(int x) { return (long long)x * 2; })
            .wait();
        CHECK(*lo == (long long)n * (n - 1), "transform_reduce n=%zu got %lld", n, *lo);
        sycl::free(lo, q);
        std::vector<double> a(n), b(n);
        double ref = 0.5;
        for (size_t i = 0; i < n; ++i) {
          a[i] = (double)(i % 17) * 0.25;
          b[i] = 1.0 + (double)(i % 5);
          ref += a[i] * b[i];
        }
        double *da = to_dev(q, a), *db = to_dev(q, b), *dd = sycl::malloc_shared<double>(1, q);
        alg::transform_reduce(q, g, da, da + n, db, dd, 0.5).wait();
        CHECK(std::fabs(*dd - ref) <= 1e-9 * std::fabs(ref), "dot n=%zu got %.17g want %.17g", n, *dd, ref);
        sycl::free(da, q);
        sycl::free(db, q);
        sycl::free(dd, q);
      }
    }
    sycl::free(out, q);
    sycl::free(d, q);
  }

  // scans: iota and multiplies with init 3 (tests/pstl/inclusive_scan.cpp)
  for (size_t n : {0ul, 1ul, 127ul, 1000ul, 1ul << 20}) {
    std::vector<int> h(n);
    std::iota(h.begin(), h.end(), 0);
    int *d = to_dev(q, h);
    int *o = sycl::malloc_device<int>(n ? n : 1, q);
    alg::util::allocation_group g{&cache, q.get_device()};
    alg::inclusive_scan(q, g, d, d + n, o).wait();
    auto got = from_dev(q, o, n);
    std::vector<int> ref(n);
    std::inclusive_scan(h.begin(), h.end(), ref.begin());
    CHECK(got == ref, "inclusive_scan iota n=%zu", n);
    alg::exclusive_scan(q, g, d, d + n, o, 3).wait();
    got = from_dev(q, o, n);
    std::exclusive_scan(h.begin(), h.end(), ref.begin(), 3);
    CHECK(got == ref, "exclusive_scan iota init 3 n=%zu", n);
    std::vector<unsigned> hu(n);
    for (size_t i = 0; i < n; ++i) hu[i] = 1u + (unsigned)(i % 3);
    unsigned *du = to_dev(q, hu), *ou = sycl::malloc_device<unsigned>(n ? n : 1, q);
    alg::inclusive_scan(q, g, du, du + n, ou, std::multiplies<unsigned>{}, 3u).wait();
    auto gotu = from_dev(q, ou, n);
    std::vector<unsigned> refu(n);
    std::inclusive_scan(hu.begin(), hu.end(), refu.begin(), std::multiplies<unsigned>{}, 3u);
    CHECK(gotu == refu, "inclusive_scan multiplies init 3 n=%zu", n);
    // user operator with transform (generic kernels)
    alg::transform_exclusive_scan(q, g, du, du + n, ou, 5u, std::plus<unsigned>{},
                                  [] __host__ __device__(unsigned x) { return x * x; })
        .wait();
    gotu = from_dev(q, ou, n);
    std::transform_exclusive_scan(hu.begin(), hu.end(), refu.begin(), 5u, std::plus<unsigned>{},
                                  [](unsigned x) { return x * x; });
    CHECK(gotu == refu, "transform_exclusive_scan n=%zu", n);
    sycl::free(d, q);
    sycl::free(o, q);
    sycl::free(du, q);
    sycl::free(ou, q);
  }

  // copy_if: even predicate on none / all / half (tests/pstl/copy_if.cpp)
  for (int mode = 0; mode < 3; ++mode) {
    const size_t n = 1000;
    std::vector<int> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = mode == 0 ? 2 * (int)i + 1 : mode == 1 ? 2 * (int)i : (int)i;
    int *d = to_dev(q, h), *o = sycl::malloc_device<int>(n, q);
    size_t *cnt = sycl::malloc_shared<size_t>(1, q);
    alg::util::allocation_group g{&cache, q.get_device()};
    alg::copy_if(q, g, d, d + n, o, [] __host__ __device__(int x) { return x % 2 == 0; }, cnt).wait();
    std::vector<int> ref;
    for (int x : h)
      if (x % 2 == 0) ref.push_back(x);
    CHECK(*cnt == ref.size(), "copy_if lambda mode %d count %zu want %zu", mode, *cnt, ref.size());
    auto got = from_dev(q, o, ref.size());
    CHECK(got == ref, "copy_if lambda mode %d values", mode);
    // the same through the libb2p fast path predicate
    alg::copy_if(q, g, d, d + n, o, alg::mask_compare<int>{1, 0, B2P_CMP_EQ}, cnt).wait();
    CHECK(*cnt == ref.size(), "copy_if mask_compare mode %d count %zu", mode, *cnt);
    got = from_dev(q, o, ref.size());
    CHECK(got == ref, "copy_if mask_compare mode %d values", mode);
    sycl::free(d, q);
    sycl::free(o, q);
    sycl::free(cnt, q);
  }

  // empty input: completed event, count 0, even with a pending dependency
  {
    alg::util::allocation_group g{&cache, q.get_device()};
    size_t cnt = 99;
    int *nothing = nullptr;
    auto ev = alg::copy_if(q, g, nothing, nothing, nothing, [] __host__ __device__(int) { return true; }, &cnt);
    CHECK(cnt == 0 && ev.is_complete(), "copy_if empty");
  }
  // the reference's sycl::maximum<float> identity (numeric_limits<float>::min())
  {
    alg::util::allocation_group g{&cache, q.get_device()};
    float *neg = to_dev(q, std::vector<float>(1000, -2.5f));
    float *fo = sycl::malloc_shared<float>(1, q);
    alg::reduce(q, g, neg, neg + 1000, fo, -5.0f, sycl::maximum<float>{}).wait();
    CHECK(*fo == std::numeric_limits<float>::min(), "reduce maximum<float> identity got %g", *fo);
    alg::reduce(q, g, neg, neg + 1000, fo, -5.0f, sycl::maximum<>{}).wait();
    CHECK(*fo == -2.5f, "reduce maximum<> got %g", *fo);
    sycl::free(neg, q);
    sycl::free(fo, q);
  }
  // any_of / all_of / none_of with the reference's signatures (no scratch,
  // int flag; an empty range leaves *out alone)
  {
    const size_t n = (1ul << 23) + 11;
    std::vector<int> h(n);
    std::iota(h.begin(), h.end(), 0);
    int *d = to_dev(q, h);
    int *flag = sycl::malloc_shared<int>(1, q);
    for (long long needle : {0ll, 12345ll, (long long)n - 1, -1ll}) {
      auto eq = [needle] __host__ __device__(int x) { return (long long)x == needle; };
      auto lt = [needle] __host__ __device__(int x) { return (long long)x < needle + 1; };
      const bool found = needle >= 0;
      alg::any_of(q, d, d + n, flag, eq).wait();
      CHECK(*flag == (int)found, "any_of needle %lld got %d", needle, *flag);
      alg::none_of(q, d, d + n, flag, eq).wait();
      CHECK(*flag == (int)!found, "none_of needle %lld got %d", needle, *flag);
      alg::all_of(q, d, d + n, flag, lt).wait();
      CHECK(*flag == (int)(needle == (long long)n - 1), "all_of below %lld got %d", needle, *flag);
    }
    *flag = 42;
    alg::any_of(q, d, d, flag, [] __host__ __device__(int) { return true; }).wait();
    CHECK(*flag == 42, "any_of of an empty range touched *out");
    sycl::free(d, q);
    sycl::free(flag, q);
  }
  // the cache reuses its allocations
  {
    int *d = to_dev(q, std::vector<int>(5000, 1));
    int *o = sycl::malloc_shared<int>(1, q);
    for (int r = 0; r < 3; ++r) {
      alg::util::allocation_group g{&cache, q.get_device()};
      alg::reduce(q, g, d, d + 5000, o, 0).wait();
      CHECK(*o == 5000, "repeated reduce %d got %d", r, *o);
    }
    sycl::free(d, q);
    sycl::free(o, q);
  }
}

// ------------------------------------------------------- sycl::reduction

static void test_reduction(sycl::queue &q) {
  // tests/sycl/reduction.cpp: sums and maxima over iota
  for (size_t n : {20ul, 128ul, 1000ul, 1024ul, 16384ul, 262144ul}) {
    std::vector<int> h(n);
    std::iota(h.begin(), h.end(), 0);
    int *d = to_dev(q, h);
    int *sum = sycl::malloc_shared<int>(1, q), *mx = sycl::malloc_shared<int>(1, q);
    *sum = 0;
    *mx = 0;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(sum, sycl::plus<int>{}),
                   [=] __device__(sycl::id<1> i, auto &r) { r += d[i[0]]; })
        .wait();
    q.submit([&](sycl::handler &cgh) {
       cgh.parallel_for(sycl::range<1>(n), sycl::reduction(mx, sycl::maximum<int>{}),
                        [=] __device__(sycl::id<1> i, auto &r) { r.combine(d[i[0]]); });
     }).wait();
    const long long ref = (long long)n * (n - 1) / 2;
    CHECK(*sum == (int)ref, "reduction sum n=%zu got %d", n, *sum);
    CHECK(*mx == (int)n - 1, "reduction max n=%zu got %d", n, *mx);
    // without initialize_to_identity the old value takes part; with it not
    *sum = 100;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(sum, sycl::plus<int>{}),
                   [=] __device__(sycl::id<1> i, auto &r) { r += d[i[0]]; })
        .wait();
    CHECK(*sum == (int)(ref + 100), "reduction combine-with-old n=%zu got %d", n, *sum);
    *sum = 100;
    q.parallel_for(sycl::range<1>(n),
                   sycl::reduction(sum, sycl::plus<int>{}, sycl::property::reduction::initialize_to_identity{}),
                   [=] __device__(sycl::id<1> i, auto &r) { r += d[i[0]]; })
        .wait();
    CHECK(*sum == (int)ref, "reduction initialize_to_identity n=%zu got %d", n, *sum);
    // float sum, tolerance 1e-3 relative (reduction.cpp uses 0.001)
    float *fs = sycl::malloc_shared<float>(1, q);
    *fs = 0.f;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(fs, sycl::plus<float>{}),
                   [=] __device__(sycl::id<1> i, auto &r) { r += (float)(d[i[0]] % 7) * 0.5f; })
        .wait();
    double fref = 0;
    for (size_t i = 0; i < n; ++i) fref += (double)(h[i] % 7) * 0.5;
    CHECK(std::fabs(*fs - fref) <= 1e-3 * fref, "reduction float n=%zu got %g want %g", n, *fs, fref);
    // user operator without a known identity, explicit identity
    auto op = [] __host__ __device__(int a, int b) { return a < b ? a : b; };
    *mx = 5;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(mx, op),
                   [=] __device__(sycl::id<1> i, auto &r) { r.combine(d[i[0]] + 3); })
        .wait();
    CHECK(*mx == 3, "reduction unknown identity n=%zu got %d", n, *mx);
    *mx = 1000000;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(mx, 1 << 30, op),
                   [=] __device__(sycl::id<1> i, auto &r) { r.combine(d[i[0]] + 9); })
        .wait();
    CHECK(*mx == 9, "reduction given identity n=%zu got %d", n, *mx);
    sycl::free(fs, q);
    sycl::free(sum, q);
    sycl::free(mx, q);
    sycl::free(d, q);
  }
}

// ---------------------------------------------------------- group functions

static void test_group_functions(sycl::queue &q) {
  for (size_t wg : {25ul, 144ul, 256ul}) {
    const size_t groups = 7, n = wg * groups;
    std::vector<int> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = (int)((i * 37) % 101) - 50;
    int *d = to_dev(q, h);
    int *red = sycl::malloc_device<int>(n, q), *inc = sycl::malloc_device<int>(n, q),
        *exc = sycl::malloc_device<int>(n, q), *sred = sycl::malloc_device<int>(n, q),
        *sinc = sycl::malloc_device<int>(n, q), *sexc = sycl::malloc_device<int>(n, q);
    q.parallel_for(sycl::nd_range<1>(sycl::range<1>(n), sycl::range<1>(wg)), [=] __device__(sycl::nd_item<1> it) {
       const size_t i = it.get_global_id(0);
       auto g = it.get_group();
       auto sg = it.get_sub_group();
       red[i] = sycl::reduce_over_group(g, d[i], sycl::plus<int>{});
       inc[i] = sycl::inclusive_scan_over_group(g, d[i], sycl::plus<int>{});
       exc[i] = sycl::exclusive_scan_over_group(g, d[i], 10, sycl::plus<int>{});
       sred[i] = sycl::reduce_over_group(sg, d[i], sycl::maximum<int>{});
       sinc[i] = sycl::inclusive_scan_over_group(sg, d[i], sycl::plus<int>{});
       sexc[i] = sycl::exclusive_scan_over_group(sg, d[i], sycl::plus<int>{});
     }).wait();
    auto r = from_dev(q, red, n), a = from_dev(q, inc, n), e = from_dev(q, exc, n), sr = from_dev(q, sred, n),
         si = from_dev(q, sinc, n), se = from_dev(q, sexc, n);
    bool ok_r = true, ok_i = true, ok_e = true, ok_sr = true, ok_si = true, ok_se = true;
    for (size_t gi = 0; gi < groups; ++gi) {
      int tot = 0, run = 0;
      for (size_t l = 0; l < wg; ++l) tot += h[gi * wg + l];
      for (size_t l = 0; l < wg; ++l) {
        const size_t i = gi * wg + l;
        ok_r &= r[i] == tot;
        ok_e &= e[i] == 10 + run;
        run += h[i];
        ok_i &= a[i] == run;
      }
      for (size_t s0 = 0; s0 < wg; s0 += 32) {
        const size_t s1 = std::min(wg, s0 + 32);
        int mxv = h[gi * wg + s0], srun = 0;
        for (size_t l = s0; l < s1; ++l) mxv = std::max(mxv, h[gi * wg + l]);
        for (size_t l = s0; l < s1; ++l) {
          const size_t i = gi * wg + l;
          ok_sr &= sr[i] == mxv;
          ok_se &= se[i] == srun;
          srun += h[i];
          ok_si &= si[i] == srun;
        }
      }
    }
    CHECK(ok_r, "reduce_over_group wg=%zu", wg);
    CHECK(ok_i, "inclusive_scan_over_group wg=%zu", wg);
    CHECK(ok_e, "exclusive_scan_over_group wg=%zu", wg);
    CHECK(ok_sr, "reduce_over_group(sub_group) wg=%zu", wg);
    CHECK(ok_si, "inclusive_scan_over_group(sub_group) wg=%zu", wg);
    CHECK(ok_se, "exclusive_scan_over_group(sub_group) wg=%zu", wg);

    // joint algorithms: each group works on its own span of 3*wg+5 elements
    const size_t span = 3 * wg + 5, m = span * groups;
    std::vector<int> hj(m);
    for (size_t i = 0; i < m; ++i) hj[i] = (int)((i * 13) % 29) - 14;
    int *dj = to_dev(q, hj);
    int *jr = sycl::malloc_device<int>(groups, q), *ji = sycl::malloc_device<int>(m, q),
        *je = sycl::malloc_device<int>(m, q);
    q.parallel_for(sycl::nd_range<1>(sycl::range<1>(n), sycl::range<1>(wg)), [=] __device__(sycl::nd_item<1> it) {
       auto g = it.get_group();
       const size_t gi = it.get_group(0);
       const int *f = dj + gi * span;
       const int v = sycl::joint_reduce(g, f, f + span, 7, sycl::plus<int>{});
       if (it.get_local_id(0) == 0) jr[gi] = v;
       sycl::joint_inclusive_scan(g, f, f + span, ji + gi * span, sycl::plus<int>{});
       sycl::joint_exclusive_scan(g, f, f + span, je + gi * span, 2, sycl::plus<int>{});
     }).wait();
    auto hjr = from_dev(q, jr, groups), hji = from_dev(q, ji, m), hje = from_dev(q, je, m);
    bool ok_jr = true, ok_ji = true, ok_je = true;
    for (size_t gi = 0; gi < groups; ++gi) {
      int tot = 7, run = 0;
      for (size_t l = 0; l < span; ++l) tot += hj[gi * span + l];
      ok_jr &= hjr[gi] == tot;
      for (size_t l = 0; l < span; ++l) {
        const size_t i = gi * span + l;
        ok_je &= hje[i] == 2 + run;
        run += hj[i];
        ok_ji &= hji[i] == run;
      }
    }
    CHECK(ok_jr, "joint_reduce wg=%zu", wg);
    CHECK(ok_ji, "joint_inclusive_scan wg=%zu", wg);
    CHECK(ok_je, "joint_exclusive_scan wg=%zu", wg);
    for (int *p : {d, red, inc, exc, sred, sinc, sexc, dj, jr, ji, je}) sycl::free(p, q);
  }
}

// ---------------------------------------------------------------- atomics

static void test_atomics(sycl::queue &q) {
  // fetch_add from 2048 work-items (tests/sycl/atomic.cpp)
  unsigned *c = sycl::malloc_shared<unsigned>(4, q);
  for (int i = 0; i < 4; ++i) c[i] = 0;
  double *fd = sycl::malloc_shared<double>(1, q);
  *fd = 0;
  q.parallel_for(sycl::range<1>(2048), [=] __host__ __device__(sycl::id<1> i) {
     sycl::atomic_ref<unsigned, sycl::memory_order::relaxed, sycl::memory_scope::device> a(c[0]);
     a.fetch_add(1u);
     sycl::atomic_ref<unsigned, sycl::memory_order::relaxed, sycl::memory_scope::device> m(c[1]);
     m.fetch_max((unsigned)i[0]);
     sycl::atomic_ref<unsigned, sycl::memory_order::acq_rel, sycl::memory_scope::device> o(c[2]);
     o.fetch_or(1u << (i[0] % 32));
     sycl::atomic_ref<double, sycl::memory_order::relaxed, sycl::memory_scope::device> f(*fd);
     f.fetch_add(0.5);
   }).wait();
  CHECK(c[0] == 2048u, "atomic fetch_add got %u", c[0]);
  CHECK(c[1] == 2047u, "atomic fetch_max got %u", c[1]);
  CHECK(c[2] == 0xffffffffu, "atomic fetch_or got %x", c[2]);
  CHECK(*fd == 1024.0, "atomic double fetch_add got %g", *fd);
  // 256-bin histogram of uint8 keys with atomic_ref<unsigned>::fetch_add
  const size_t n = 1 << 20;
  std::vector<unsigned char> keys(n);
  for (size_t i = 0; i < n; ++i) keys[i] = (unsigned char)((i * 2654435761u) >> 13);
  unsigned char *dk = to_dev(q, keys);
  unsigned *bins = sycl::malloc_device<unsigned>(256, q);
  q.memset(bins, 0, 256 * sizeof(unsigned)).wait();
  q.parallel_for(sycl::range<1>(n), [=] __host__ __device__(sycl::id<1> i) {
     sycl::atomic_ref<unsigned, sycl::memory_order::relaxed, sycl::memory_scope::device> b(bins[dk[i[0]]]);
     b.fetch_add(1u);
   }).wait();
  auto hb = from_dev(q, bins, 256);
  std::vector<unsigned> ref(256, 0);
  for (auto k : keys) ++ref[k];
  CHECK(hb == ref, "atomic_ref histogram");
  sycl::free(c, q);
  sycl::free(fd, q);
  sycl::free(dk, q);
  sycl::free(bins, q);
}

// ------------------------------------------------------------------ stdpar

static void test_stdpar() {
  const auto &pol = b2p_stdpar::par_unseq;
  for (size_t n : {0ul, 1ul, 127ul, 1000ul, 1000000ul}) {
    std::vector<long long> v(n);
    std::iota(v.begin(), v.end(), 0);
    const long long ref = std::reduce(v.begin(), v.end(), 10ll);
    CHECK(std::reduce(pol, v.begin(), v.end(), 10ll) == ref, "stdpar reduce n=%zu", n);
    CHECK(std::reduce(pol, v.begin(), v.end()) == ref - 10, "stdpar reduce no init n=%zu", n);
    CHECK(std::reduce(pol, v.begin(), v.end(), 10ll, std::plus<>{}) == ref, "stdpar reduce op n=%zu", n);
    std::vector<double> a(n), b(n);
    for (size_t i = 0; i < n; ++i) {
      a[i] = (double)(i % 11);
      b[i] = 0.5 * (double)(i % 3);
    }
    const double dref = std::transform_reduce(a.begin(), a.end(), b.begin(), 1.0);
    const double dgot = std::transform_reduce(pol, a.begin(), a.end(), b.begin(), 1.0);
    CHECK(std::fabs(dgot - dref) <= 1e-9 * std::max(1.0, std::fabs(dref)), "stdpar transform_reduce n=%zu", n);
  }
  for (size_t n : {0ul, 1ul, 127ul, 1000ul, 1ul << 20}) {
    std::vector<int> v(n), out(n), ref(n);
    std::iota(v.begin(), v.end(), 0);
    std::inclusive_scan(v.begin(), v.end(), ref.begin());
    std::inclusive_scan(pol, v.begin(), v.end(), out.begin());
    CHECK(out == ref, "stdpar inclusive_scan n=%zu", n);
    std::exclusive_scan(v.begin(), v.end(), ref.begin(), 3);
    std::exclusive_scan(pol, v.begin(), v.end(), out.begin(), 3);
    CHECK(out == ref, "stdpar exclusive_scan n=%zu", n);
    std::vector<unsigned> u(n), uo(n), ur(n);
    for (size_t i = 0; i < n; ++i) u[i] = 1u + (unsigned)(i % 2);
    std::inclusive_scan(u.begin(), u.end(), ur.begin(), std::multiplies<unsigned>{}, 3u);
    std::inclusive_scan(pol, u.begin(), u.end(), uo.begin(), std::multiplies<unsigned>{}, 3u);
    CHECK(uo == ur, "stdpar inclusive_scan multiplies init 3 n=%zu", n);
    // transform scans (pstl-impl/numeric.hpp:469-576): a known operator, and a
    // user lambda without a known identity (generic kernels)
    auto sq = [] __host__ __device__(int x) { return (long long)x * x; };
    std::vector<long long> lo(n), lr(n);
    std::transform_inclusive_scan(v.begin(), v.end(), lr.begin(), std::plus<long long>{}, sq);
    std::transform_inclusive_scan(pol, v.begin(), v.end(), lo.begin(), std::plus<long long>{}, sq);
    CHECK(lo == lr, "stdpar transform_inclusive_scan n=%zu", n);
    auto keep_max = [] __host__ __device__(int a, int b) { return a < b ? b : a; };
    auto wave = [] __host__ __device__(int x) { return (x * 7919) % 1000 - 500; };
    std::transform_inclusive_scan(v.begin(), v.end(), ref.begin(), keep_max, wave, -600);
    std::transform_inclusive_scan(pol, v.begin(), v.end(), out.begin(), keep_max, wave, -600);
    CHECK(out == ref, "stdpar transform_inclusive_scan lambda op init n=%zu", n);
    std::transform_exclusive_scan(v.begin(), v.end(), ref.begin(), 11, keep_max, wave);
    std::transform_exclusive_scan(pol, v.begin(), v.end(), out.begin(), 11, keep_max, wave);
    CHECK(out == ref, "stdpar transform_exclusive_scan lambda op n=%zu", n);
  }
  for (int mode = 0; mode < 3; ++mode) {
    std::vector<int> v(1000), out(1000, -1), ref;
    for (int i = 0; i < 1000; ++i) v[i] = mode == 0 ? 2 * i + 1 : mode == 1 ? 2 * i : i;
    auto even = [] __host__ __device__(int x) { return x % 2 == 0; };
    for (int x : v)
      if (even(x)) ref.push_back(x);
    auto end = std::copy_if(pol, v.begin(), v.end(), out.begin(), even);
    CHECK((size_t)(end - out.begin()) == ref.size(), "stdpar copy_if mode %d count", mode);
    CHECK(std::equal(ref.begin(), ref.end(), out.begin()), "stdpar copy_if mode %d values", mode);
  }
  // managed (shared-USM) ranges: prefetched, and with par_unseq_async the
  // scans queue back to back until b2p_stdpar::sync()
  {
    const size_t n = (1u << 20) + 3;
    int *m = nullptr, *o1 = nullptr, *o2 = nullptr;
    CHECK(cudaMallocManaged(&m, n * sizeof(int)) == cudaSuccess, "cudaMallocManaged");
    cudaMallocManaged(&o1, n * sizeof(int));
    cudaMallocManaged(&o2, n * sizeof(int));
    for (size_t i = 0; i < n; ++i) m[i] = (int)(i % 13) - 6;
    std::vector<int> r1(n), r2(n);
    std::inclusive_scan(m, m + n, r1.begin());
    std::exclusive_scan(r1.begin(), r1.end(), r2.begin(), 4);
    const auto &apol = b2p_stdpar::par_unseq_async;
    std::inclusive_scan(apol, m, m + n, o1);
    std::exclusive_scan(apol, o1, o1 + n, o2, 4);  // ordered after the first on the thread's stream
    b2p_stdpar::sync();
    CHECK(std::equal(r1.begin(), r1.end(), o1), "stdpar async inclusive_scan (managed)");
    CHECK(std::equal(r2.begin(), r2.end(), o2), "stdpar async exclusive_scan after it (managed)");
    std::inclusive_scan(apol, m, m + n, o1);
    const long long red = std::reduce(pol, o1, o1 + n, 0ll);  // blocking, after the async scan
    CHECK(red == std::accumulate(r1.begin(), r1.end(), 0ll), "stdpar reduce after async scan");
    cudaFree(m);
    cudaFree(o1);
    cudaFree(o2);
  }
  // a batch: 8 consecutive non-blocking scans, each reading the previous
  // output, recorded into one CUDA graph and launched once at sync(); the
  // same batch again reuses the executable graph
  {
    const size_t n = (1u << 20) + 77;
    const int kCalls = 8;
    std::vector<int *> bufs(kCalls + 1, nullptr);
    for (auto &b : bufs) CHECK(cudaMallocManaged(&b, n * sizeof(int)) == cudaSuccess, "cudaMallocManaged");
    for (size_t i = 0; i < n; ++i) bufs[0][i] = (int)(i % 5) - 2;
    std::vector<std::vector<int>> ref(kCalls + 1, std::vector<int>(n));
    ref[0].assign(bufs[0], bufs[0] + n);
    for (int c = 0; c < kCalls; ++c) {
      if (c % 2 == 0) std::inclusive_scan(ref[c].begin(), ref[c].end(), ref[c + 1].begin());
      else std::exclusive_scan(ref[c].begin(), ref[c].end(), ref[c + 1].begin(), c);
    }
    const auto &apol = b2p_stdpar::par_unseq_async;
    for (int round = 0; round < 2; ++round) {
      const auto before = b2p_stdpar::batch_stats();
      for (int c = 0; c < kCalls; ++c) {
        if (c % 2 == 0) std::inclusive_scan(apol, bufs[c], bufs[c] + n, bufs[c + 1]);
        else std::exclusive_scan(apol, bufs[c], bufs[c] + n, bufs[c + 1], c);
      }
      b2p_stdpar::sync();
      const auto after = b2p_stdpar::batch_stats();
      CHECK(after.graph_launches == before.graph_launches + 1, "stdpar batch: one graph launch for %d calls (got %zu)",
            kCalls, after.graph_launches - before.graph_launches);
      CHECK(after.batched_calls == before.batched_calls + kCalls, "stdpar batch: %d calls in the graph", kCalls);
      for (int c = 1; c <= kCalls; ++c)
        CHECK(std::equal(ref[c].begin(), ref[c].end(), bufs[c]), "stdpar batch round %d call %d result", round, c);
      for (int c = 1; c <= kCalls; ++c) std::fill(bufs[c], bufs[c] + n, -1);
    }
    // a blocking call finalises the open batch before it runs
    std::inclusive_scan(apol, bufs[0], bufs[0] + n, bufs[1]);
    const long long red = std::reduce(b2p_stdpar::par_unseq, bufs[1], bufs[1] + n, 0ll);
    CHECK(red == std::accumulate(ref[1].begin(), ref[1].end(), 0ll), "stdpar reduce after a batched scan");
    for (auto b : bufs) cudaFree(b);
  }
  // any_of / all_of / none_of (algorithm.hpp:422-516, pstl-impl/algorithm.hpp:403-500)
  for (size_t n : {1ul, 1000ul, (1ul << 22) + 7}) {
    std::vector<int> v(n);
    std::iota(v.begin(), v.end(), 0);
    for (long long needle : {0ll, (long long)n / 2, (long long)n - 1, -5ll}) {
      auto eq = [needle] __host__ __device__(int x) { return (long long)x == needle; };
      auto ne = [needle] __host__ __device__(int x) { return (long long)x != needle; };
      CHECK(std::any_of(pol, v.begin(), v.end(), eq) == std::any_of(v.begin(), v.end(), eq),
            "stdpar any_of n=%zu needle=%lld", n, needle);
      CHECK(std::all_of(pol, v.begin(), v.end(), ne) == std::all_of(v.begin(), v.end(), ne),
            "stdpar all_of n=%zu needle=%lld", n, needle);
      CHECK(std::none_of(pol, v.begin(), v.end(), eq) == std::none_of(v.begin(), v.end(), eq),
            "stdpar none_of n=%zu needle=%lld", n, needle);
    }
  }
  {
    std::vector<int> e;
    auto any = [] __host__ __device__(int) { return true; };
    CHECK(!std::any_of(pol, e.begin(), e.end(), any) && std::all_of(pol, e.begin(), e.end(), any) &&
              std::none_of(pol, e.begin(), e.end(), any),
          "stdpar any/all/none of an empty range");
  }
  CHECK(!b2p_stdpar::offload_history().empty(), "stdpar offload history recorded");
}

// Median time of `reps` runs of f on the queue's stream (CUDA events).
template <class F>
static float median_ms(sycl::queue &q, F f, int reps = 7) {
  std::vector<float> t;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  f();
  q.wait();
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(a, q.cuda_stream());
    f();
    cudaEventRecord(b, q.cuda_stream());
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    t.push_back(ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::sort(t.begin(), t.end());
  return t[t.size() / 2];
}

// ------------------------------------------------------------ sort / merge
// tests/pstl/sort.cpp:24-75 and tests/pstl/merge.cpp:24-137 through the
// stdpar overloads (pageable std::vector ranges, staged), then the
// algorithms-library calls with user comparators on device memory: a key
// with a payload sorted and merged on the key alone must come out in
// std::stable_sort / std::merge order (stability), and sizes around the
// 2048-key tile of the kernels.

struct keyed {
  int key;
  int idx;
  bool operator==(const keyed &o) const { return key == o.key && idx == o.idx; }
};

static std::vector<int> sorted_random(int amount, int seed) {
  std::mt19937 gen(seed);
  std::uniform_int_distribution<int> dist;
  std::vector<int> d;
  for (int i = 0; i < amount; ++i) d.push_back(dist(gen));
  std::sort(d.begin(), d.end());
  return d;
}

static void test_sort_merge(sycl::queue &q) {
  const auto &pol = b2p_stdpar::par_unseq;
  {
    const std::pair<size_t, int> cases[] = {{0, 0}, {1, 1}, {1024, -1}, {1024, 1}, {1000, -1}, {1000, 1}};
    for (auto [n, sign] : cases) {
      std::vector<int> v(n);
      for (size_t i = 0; i < n; ++i) v[i] = sign * (int)i;
      std::vector<int> h = v;
      std::sort(pol, v.begin(), v.end());
      std::sort(h.begin(), h.end());
      CHECK(v == h && std::is_sorted(v.begin(), v.end()), "stdpar sort n=%zu sign %d", n, sign);
    }
  }
  {
    auto merge_case = [&](const char *name, const std::vector<int> &a, const std::vector<int> &b) {
      std::vector<int> out(a.size() + b.size(), -1), ref(a.size() + b.size());
      auto ret = std::merge(pol, a.begin(), a.end(), b.begin(), b.end(), out.begin());
      auto hret = std::merge(a.begin(), a.end(), b.begin(), b.end(), ref.begin());
      CHECK(out == ref, "stdpar merge %s", name);
      CHECK(ret - out.begin() == hret - ref.begin(), "stdpar merge %s return", name);
    };
    merge_case("empty", {}, {});
    merge_case("single 1 0", {2}, {});
    merge_case("single 0 1", {}, {3});
    merge_case("single 1 1", {2}, {3});
    std::vector<int> lo(1024), hi(1024);
    std::iota(lo.begin(), lo.end(), 0);
    std::iota(hi.begin(), hi.end(), 1024);
    merge_case("trivial", lo, hi);
    merge_case("trivial swapped", hi, lo);
    merge_case("same size", sorted_random(256, 123), sorted_random(256, 42));
    merge_case("same data", sorted_random(1024, 123), sorted_random(1024, 123));
    merge_case("v1 larger", sorted_random(1932, 123), sorted_random(1000, 42));
    merge_case("v2 larger", sorted_random(1000, 123), sorted_random(1932, 42));
  }
  alg::util::allocation_cache cache{alg::util::allocation_type::device};
  std::mt19937 gen(7);
  auto by_key = [] __host__ __device__(const keyed &x, const keyed &y) { return x.key < y.key; };
  for (size_t n : {2ul, 2047ul, 2048ul, 2049ul, 3 * 4096ul + 5, 1ul << 20}) {
    std::vector<keyed> h(n);
    std::uniform_int_distribution<int> dk(0, (int)std::max<size_t>(n / 16, 1));
    for (size_t i = 0; i < n; ++i) h[i] = {dk(gen), (int)i};
    keyed *d = to_dev(q, h);
    alg::sort(q, d, d + n, by_key).wait();
    std::stable_sort(h.begin(), h.end(), [](const keyed &x, const keyed &y) { return x.key < y.key; });
    CHECK(from_dev(q, d, n) == h, "algorithms::sort stable with a lambda comparator n=%zu", n);
    // merge two sorted halves (ties across the halves: a's first)
    const size_t n1 = n / 3;
    std::vector<keyed> a(h.begin(), h.begin() + n1), b(h.begin() + n1, h.end());
    for (auto &x : b) x.idx += 1 << 30;
    std::vector<keyed> ref(n);
    std::merge(a.begin(), a.end(), b.begin(), b.end(), ref.begin(),
               [](const keyed &x, const keyed &y) { return x.key < y.key; });
    keyed *da = to_dev(q, a), *db = to_dev(q, b), *dout = sycl::malloc_device<keyed>(n, q);
    {
      alg::util::allocation_group g{&cache, q.get_device()};
      alg::merge(q, g, da, da + n1, db, db + (n - n1), dout, by_key).wait();
    }
    CHECK(from_dev(q, dout, n) == ref, "algorithms::merge stable with a lambda comparator n=%zu", n);
    sycl::free(dout, q);
    sycl::free(db, q);
    sycl::free(da, q);
    sycl::free(d, q);
  }
  {
    const size_t n = 1ul << 24;
    std::vector<double> h(n);
    std::normal_distribution<double> nd;
    for (auto &v : h) v = nd(gen);
    double *d = to_dev(q, h);
    alg::sort(q, d, d + n, std::greater<>{}).wait();
    std::sort(h.begin(), h.end(), std::greater<>{});
    CHECK(from_dev(q, d, n) == h, "algorithms::sort f64 std::greater 2^24");
    sycl::free(d, q);
  }
  {
    const size_t n = 1ul << 24;
    std::vector<uint32_t> h(n);
    for (auto &v : h) v = (uint32_t)gen();
    uint32_t *d = to_dev(q, h), *w = to_dev(q, h);
    std::vector<uint32_t> ref = h;
    std::sort(ref.begin(), ref.end());
    alg::sort(q, d, d + n).wait();
    CHECK(from_dev(q, d, n) == ref, "algorithms::sort u32 2^24");
    // each run restores the random keys (a 64 MiB device copy) and sorts them
    const float t = median_ms(q, [&] {
      cudaMemcpyAsync(d, w, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, q.cuda_stream());
      alg::sort(q, d, d + n);
    }, 5);
    std::printf("TIMING u32 2^24 random sort (+ key restore copy): %.4f ms\n", t);
    CHECK(from_dev(q, d, n) == ref, "algorithms::sort u32 2^24 after timing");
    sycl::free(w, q);
    sycl::free(d, q);
  }
}

// ----------------------------------------------- workload configurations
// Config 1: 2^24 int32 U[-1000, 1000] (seed 0) through the entry points it
// names -- sycl::reduction in parallel_for, std::reduce and
// std::inclusive_scan on the stdpar policy -- bit-exact against a host sum /
// scan.  Config 3: hipsycl::algorithms::copy_if with a lambda predicate
// (x & 7) < 3 on 2^28 uint32 (seed 4), bit-exact and order-preserving.
// Config 2's fp32 values (seed 1) through sycl::reduction: within 1e-6 of a
// float64 host sum.

static void test_workload_configs(sycl::queue &q) {
  alg::util::allocation_cache cache{alg::util::allocation_type::device};
  {
    const size_t n = 1ul << 24;
    std::vector<int32_t> h(n);
    CHECK(b2p_synth_fill(0, 0, n, -1000, 1000, h.data()) == B2P_OK, "synth config 1");
    uint32_t wrap = 0;
    for (int32_t v : h) wrap += (uint32_t)v;
    const int32_t ref = (int32_t)wrap;
    int32_t *d = to_dev(q, h);
    int32_t *sum = sycl::malloc_shared<int32_t>(1, q);
    *sum = 0;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(sum, sycl::plus<int32_t>{}),
                   [=] __device__(sycl::id<1> i, auto &r) { r += d[i[0]]; })
        .wait();
    CHECK(*sum == ref, "config 1 sycl::reduction 2^24 got %d want %d", *sum, ref);
    const auto &pol = b2p_stdpar::par_unseq;
    const int32_t sr = std::reduce(pol, h.begin(), h.end(), (int32_t)0);
    CHECK(sr == ref, "config 1 std::reduce 2^24 got %d want %d", sr, ref);
    std::vector<int32_t> sc(n), scr(n);
    std::inclusive_scan(pol, h.begin(), h.end(), sc.begin());
    uint32_t run = 0;
    for (size_t i = 0; i < n; ++i) scr[i] = (int32_t)(run += (uint32_t)h[i]);
    CHECK(sc == scr, "config 1 std::inclusive_scan 2^24");
    sycl::free(sum, q);
    sycl::free(d, q);
  }
  {
    const size_t n = 1ul << 28;
    std::vector<float> h(n);
    CHECK(b2p_synth_fill(1, 1, n, 0.125, 1e-6, h.data()) == B2P_OK, "synth config 2");
    double ref = 0.0;
    for (float v : h) ref += (double)v;
    float *d = to_dev(q, h);
    float *sum = sycl::malloc_shared<float>(1, q);
    *sum = 0.f;
    q.parallel_for(sycl::range<1>(n), sycl::reduction(sum, sycl::plus<float>{}),
                   [=] __device__(sycl::id<1> i, auto &r) { r += d[i[0]]; })
        .wait();
    CHECK(std::fabs((double)*sum - ref) <= 1e-6 * std::fabs(ref), "fp32 sycl::reduction 2^28 got %.9g want %.9g",
          (double)*sum, ref);
    // the same sum through hipsycl::algorithms::reduce (libb2p's b2p_reduce)
    // and through a user transform
    float *r2 = sycl::malloc_shared<float>(1, q);
    {
      alg::util::allocation_group g{&cache, q.get_device()};
      alg::reduce(q, g, d, d + n, r2, 0.f, sycl::plus<float>{}).wait();
      CHECK(std::fabs((double)*r2 - ref) <= 1e-6 * std::fabs(ref), "fp32 algorithms::reduce 2^28");
      alg::transform_reduce(q, g, d, d + n, r2, 0.f, sycl::plus<float>{},
                            [] __host__ __device__(float v) { return 2.f * v; })
          .wait();
      CHECK(std::fabs((double)*r2 - 2.0 * ref) <= 2e-6 * std::fabs(ref), "fp32 transform_reduce(2x) 2^28");
      const float t_red = median_ms(q, [&] {
        q.parallel_for(sycl::range<1>(n), sycl::reduction(sum, sycl::plus<float>{}),
                       [=] __device__(sycl::id<1> i, auto &r) { r += d[i[0]]; });
      });
      const float t_lib = median_ms(q, [&] {
        alg::util::allocation_group g1{&cache, q.get_device()};
        alg::reduce(q, g1, d, d + n, r2, 0.f, sycl::plus<float>{});
      });
      std::printf("TIMING fp32 2^28 sum: sycl::reduction %.4f ms, b2p_reduce %.4f ms, ratio %.3f\n", t_red, t_lib,
                  t_red / t_lib);
      CHECK(t_red <= 1.25f * t_lib, "sycl::reduction 2^28 within 25%% of b2p_reduce (%.4f vs %.4f ms)", t_red, t_lib);
    }
    sycl::free(r2, q);
    sycl::free(sum, q);
    sycl::free(d, q);
  }
  {
    const size_t n = 1ul << 28;
    std::vector<uint32_t> h(n);
    CHECK(b2p_synth_fill(3, 4, n, 0, 0, h.data()) == B2P_OK, "synth config 3");
    std::vector<uint32_t> ref;
    ref.reserve(n / 2);
    for (uint32_t v : h)
      if ((v & 7u) < 3u) ref.push_back(v);
    uint32_t *d = to_dev(q, h);
    uint32_t *out = sycl::malloc_device<uint32_t>(n, q);
    size_t *cnt = sycl::malloc_shared<size_t>(1, q);
    *cnt = 0;
    {
      alg::util::allocation_group g{&cache, q.get_device()};
      alg::copy_if(q, g, d, d + n, out, [] __host__ __device__(uint32_t v) { return (v & 7u) < 3u; }, cnt).wait();
    }
    CHECK(*cnt == ref.size(), "config 3 lambda copy_if count %zu want %zu", *cnt, ref.size());
    std::vector<uint32_t> got = from_dev(q, out, ref.size());
    CHECK(got == ref, "config 3 lambda copy_if values");
    {
      // one allocation group per call, as a caller of the algorithms library
      // has: its scratch returns to the cache and the next call reuses it
      auto lam = [] __host__ __device__(uint32_t v) { return (v & 7u) < 3u; };
      const alg::mask_compare<uint32_t> mc{7u, 3u, B2P_CMP_LT};
      const float t_lam = median_ms(q, [&] {
        alg::util::allocation_group g{&cache, q.get_device()};
        alg::copy_if(q, g, d, d + n, out, lam, cnt);
      });
      const float t_lib = median_ms(q, [&] {
        alg::util::allocation_group g{&cache, q.get_device()};
        alg::copy_if(q, g, d, d + n, out, mc, cnt);
      });
      std::printf("TIMING u32 2^28 copy_if: lambda %.4f ms, b2p_copy_if %.4f ms, ratio %.3f\n", t_lam, t_lib,
                  t_lam / t_lib);
      CHECK(t_lam <= 1.25f * t_lib, "lambda copy_if 2^28 within 25%% of b2p_copy_if (%.4f vs %.4f ms)", t_lam, t_lib);
      q.wait();
      CHECK(*cnt == ref.size(), "copy_if count after timing");
    }
    sycl::free(cnt, q);
    sycl::free(out, q);
    sycl::free(d, q);
  }
}

// With arguments, only the named sections run (algorithms, reduction, group,
// atomics, stdpar, sort_merge, workload), in the order given.
int main(int argc, char **argv) {
  try {
    sycl::queue q;
    const std::vector<std::pair<std::string, std::function<void()>>> sections = {
        {"algorithms", [&] { test_algorithms(q); }},   {"reduction", [&] { test_reduction(q); }},
        {"group", [&] { test_group_functions(q); }},   {"atomics", [&] { test_atomics(q); }},
        {"stdpar", [&] { test_stdpar(); }},            {"sort_merge", [&] { test_sort_merge(q); }},
        {"workload", [&] { test_workload_configs(q); }}};
    if (argc < 2) {
      for (auto &sec : sections) sec.second();
    } else {
      for (int i = 1; i < argc; ++i)
        for (auto &sec : sections)
          if (sec.first == argv[i]) sec.second();
    }
  } catch (const std::exception &e) {
    std::printf("FAIL exception: %s\n", e.what());
    return 2;
  }
  if (g_fail) {
    std::printf("%d of %d checks FAILED\n", g_fail, g_checks);
    return 1;
  }
  std::printf("ALL PASSED %d\n", g_checks);
  return 0;
}
