// Per-tile phases shared by the scan kernels: a thread's total over its
// ITEMS consecutive elements of a swizzled shared tile, the emission of its
// scanned outputs, and the conversions between a tile carry (accumulator or
// FP64 for long fp32/bf16 sums) and a thread's running value.
#pragma once

#include "tile.cuh"

namespace b2p {

// ------------------------------------------------------- per-tile phases

// Thread total of this thread's ITEMS consecutive elements of the shared
// tile (blocked arrangement, 16-byte reads).
template <class P, int ITEMS>
__device__ __forceinline__ typename P::Acc thread_total(const char *buf, int count) {
  using In = typename P::In;
  constexpr int IPV = 16 / (int)sizeof(In);
  constexpr int VPT = ITEMS * (int)sizeof(In) / 16;
  const int first = threadIdx.x * ITEMS;
  typename P::Acc agg = P::identity();
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    const In *e = reinterpret_cast<const In *>(&w);
#pragma unroll
    for (int q = 0; q < IPV; ++q)
      if (first + k * IPV + q < count) P::add(agg, e[q]);
  }
  if constexpr (P::kCompensated) agg = df_norm(agg);
  return agg;
}

// Re-read the inputs and write the outputs one 16-byte vector at a time.
// With equal element sizes each output vector overwrites the input vector
// it came from, which only this thread reads.
template <class P, int ITEMS>
__device__ __forceinline__ void emit_scan(const char *buf, char *obuf, typename P::Acc run,
                                          bool inclusive) {
  using In = typename P::In;
  using Out = typename P::Out;
  constexpr int IPV = 16 / (int)sizeof(In);
  constexpr int OPV = 16 / (int)sizeof(Out);
  constexpr int VPT = ITEMS * (int)sizeof(In) / 16;
  constexpr int OUT_PER_IN = IPV / OPV;
#pragma unroll
  for (int k = 0; k < VPT; ++k) {
    const uint4 w = *reinterpret_cast<const uint4 *>(buf + swz(threadIdx.x * VPT + k) * 16);
    const In *e = reinterpret_cast<const In *>(&w);
#pragma unroll
    for (int m = 0; m < OUT_PER_IN; ++m) {
      uint4 o;
      Out *oe = reinterpret_cast<Out *>(&o);
#pragma unroll
      for (int q = 0; q < OPV; ++q) {
        const In xv = e[m * OPV + q];
        if (inclusive) {
          P::add(run, xv);
          oe[q] = P::finalize(run);
        } else {
          oe[q] = P::finalize(run);
          P::add(run, xv);
        }
      }
      *reinterpret_cast<uint4 *>(obuf + swz((threadIdx.x * VPT + k) * OUT_PER_IN + m) * 16) = o;
    }
  }
}

// Running value of a thread: carry (+) the thread's exclusive prefix.
template <class P, bool WIDE>
__device__ __forceinline__ typename P::Acc start_value(unsigned long long carry_bits,
                                                       typename P::Acc texcl) {
  if constexpr (WIDE) {
    const double c = F64Ops::unpack(carry_bits) + ((double)texcl.hi + (double)texcl.lo);
    const float h = (float)c;
    return DF{h, (float)(c - (double)h)};
  } else {
    return P::combine(P::unpack(carry_bits), texcl);
  }
}

template <class P, bool WIDE>
__device__ __forceinline__ unsigned long long publish_value(typename P::Acc a) {
  if constexpr (WIDE) return F64Ops::pack((double)a.hi + (double)a.lo);
  else return P::pack(a);
}

// (flag, value) pair of the segmented operator: f = a segment head lies in
// the span, v = the combination after the last head (of everything when
// f == 0).  (f1, v1) + (f2, v2) = (f1 | f2, f2 ? v2 : v1 + v2).
template <class P>
struct SegPair {
  typename P::Acc v;
  int f;
};

template <class P>
struct SegOps {
  using Pub = SegPair<P>;
  __device__ static Pub identity() { return Pub{P::identity(), 0}; }
  __device__ static Pub combine(Pub a, Pub b) {
    return Pub{b.f ? b.v : P::combine(a.v, b.v), a.f | b.f};
  }
};

template <class P>
__device__ __forceinline__ SegPair<P> shfl_up(SegPair<P> a, int d) {
  a.v = shfl_up(a.v, d);
  a.f = __shfl_up_sync(0xffffffffu, a.f, d);
  return a;
}

template <class P>
__device__ __forceinline__ SegPair<P> shfl_idx(SegPair<P> a, int src) {
  a.v = shfl_idx(a.v, src);
  a.f = __shfl_sync(0xffffffffu, a.f, src);
  return a;
}

// copy_if predicate: (bits of v & mask) CMP rhs, compared as unsigned.
template <class T>
__device__ __forceinline__ bool pred_bits(T v, unsigned long long mask, int cmp,
                                          unsigned long long rhs) {
  using U = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
  U u;
  memcpy(&u, &v, sizeof(T));
  const U a = u & (U)mask, r = (U)rhs;
  switch (cmp) {
  case B2P_CMP_LT: return a < r;
  case B2P_CMP_LE: return a <= r;
  case B2P_CMP_EQ: return a == r;
  case B2P_CMP_NE: return a != r;
  case B2P_CMP_GE: return a >= r;
  default: return a > r;
  }
}

}  // namespace b2p
