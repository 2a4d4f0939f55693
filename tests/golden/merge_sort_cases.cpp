// Inputs and expected outputs of the merge and sort cases of AdaptiveCpp's
// tests/pstl/merge.cpp:46-137 and tests/pstl/sort.cpp:44-75: the sorted
// random inputs come from std::mt19937 with std::uniform_int_distribution<int>
// (libstdc++), the expected outputs from the serial std::merge / std::sort
// the reference tests compare against.  Built and run by make_merge_sort.py.
//
// Output: a sequence of records "name\n" + int64 count + count int32 values.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <random>
#include <string>
#include <vector>

static void put(const std::string &name, const std::vector<int> &v) {
  std::fwrite(name.data(), 1, name.size(), stdout);
  std::fputc('\n', stdout);
  const int64_t n = (int64_t)v.size();
  std::fwrite(&n, sizeof n, 1, stdout);
  if (n) std::fwrite(v.data(), sizeof(int), v.size(), stdout);
}

static std::vector<int> sorted_random(int amount, int seed) {
  std::mt19937 gen(seed);
  std::uniform_int_distribution<int> dist;
  std::vector<int> d;
  for (int i = 0; i < amount; ++i) d.push_back(dist(gen));
  std::sort(d.begin(), d.end());
  return d;
}

template <class F>
static std::vector<int> make(int n, F f) {
  std::vector<int> v(n);
  for (int i = 0; i < n; ++i) v[i] = f(i);
  return v;
}

static void merge_case(const std::string &name, const std::vector<int> &a, const std::vector<int> &b) {
  std::vector<int> out(a.size() + b.size());
  std::merge(a.begin(), a.end(), b.begin(), b.end(), out.begin());
  put("merge/" + name + "/a", a);
  put("merge/" + name + "/b", b);
  put("merge/" + name + "/out", out);
}

static void sort_case(const std::string &name, const std::vector<int> &x) {
  std::vector<int> out = x;
  std::sort(out.begin(), out.end());
  put("sort/" + name + "/in", x);
  put("sort/" + name + "/out", out);
}

int main() {
  merge_case("empty", {}, {});
  merge_case("single_1_0", make(1, [](int) { return 2; }), {});
  merge_case("single_0_1", {}, make(1, [](int) { return 3; }));
  merge_case("single_1_1", make(1, [](int) { return 2; }), make(1, [](int) { return 3; }));
  auto lo = make(1024, [](int i) { return i; });
  auto hi = make(1024, [](int i) { return i + 1024; });
  merge_case("trivial_ab", lo, hi);
  merge_case("trivial_ba", hi, lo);
  merge_case("same_size", sorted_random(256, 123), sorted_random(256, 42));
  merge_case("same_data", sorted_random(1024, 123), sorted_random(1024, 123));
  merge_case("v1_larger", sorted_random(1932, 123), sorted_random(1000, 42));
  merge_case("v2_larger", sorted_random(1000, 123), sorted_random(1932, 42));
  sort_case("empty", {});
  sort_case("single", make(1, [](int i) { return i; }));
  sort_case("pow2_descending", make(1024, [](int i) { return -i; }));
  sort_case("pow2_ascending", make(1024, [](int i) { return i; }));
  sort_case("non_pow2_descending", make(1000, [](int i) { return -i; }));
  sort_case("non_pow2_ascending", make(1000, [](int i) { return i; }));
  return 0;
}
