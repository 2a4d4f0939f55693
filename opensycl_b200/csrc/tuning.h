// Decision table of the learned schedule selector, consulted by
// B2P_CONFIG_AUTO.  Built once by b2p_selector_install with one batched
// inference launch over a grid of call shapes; a lookup is a table read.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace b2p {

struct AutoTable {
  bool valid = false;
  // grid: prim (7) x dtype (7) x log2 n in quarter steps over [0, 40)
  //       x log2 nseg bucket (8: 0,1..,>=2^14 in steps of 2) x cv bucket (4)
  static constexpr int kLogSteps = 160;
  static constexpr int kSegBuckets = 8;
  static constexpr int kCvBuckets = 4;
  std::vector<int16_t> cfg;  // size 7*7*kLogSteps*kSegBuckets*kCvBuckets

  static int log_bucket(size_t n) {
    double l = n ? std::log2((double)n) : 0.0;
    int b = (int)std::lround(l * 4.0);
    return b < 0 ? 0 : (b >= kLogSteps ? kLogSteps - 1 : b);
  }
  static int seg_bucket(int64_t nseg) {
    if (nseg <= 1) return 0;
    int b = 1 + (int)(std::log2((double)nseg) / 2.0);
    return b >= kSegBuckets ? kSegBuckets - 1 : b;
  }
  static int cv_bucket(double cv) {
    int b = (int)(cv * 2.0);
    return b < 0 ? 0 : (b >= kCvBuckets ? kCvBuckets - 1 : b);
  }
  static size_t index(int prim, int dtype, int lb, int sb, int cb) {
    return ((((size_t)prim * 7 + (size_t)dtype) * kLogSteps + (size_t)lb) * kSegBuckets + (size_t)sb) *
               kCvBuckets + (size_t)cb;
  }
  static size_t size() { return (size_t)7 * 7 * kLogSteps * kSegBuckets * kCvBuckets; }
  int lookup(int prim, int dtype, size_t n, int64_t nseg, double cv) const {
    if (prim < 0 || prim > 6 || dtype < 0 || dtype > 6 || cfg.size() != size()) return -1;
    return cfg[index(prim, dtype, log_bucket(n), seg_bucket(nseg), cv_bucket(cv))];
  }
};

void install_auto_table(const AutoTable &t);
void clear_auto_table();
int heuristic_config(int prim, int dtype, size_t n, int64_t nseg);
int tune_shape(int prim, int dtype, int op, size_t n, int64_t nseg, double cv, int reps,
               uint64_t seed, float *times_ms);

}  // namespace b2p
