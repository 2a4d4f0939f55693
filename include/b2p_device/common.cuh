// Shared device-side building blocks of libb2p: element policies (how a
// dtype/op pair accumulates, combines and is published across tiles),
// compensated fp32 arithmetic, warp collectives and the PTX accessors used
// by the single-pass kernels.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "../b2p.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libb2p is built for sm_100a only"
#endif

namespace b2p {

constexpr int kWarp = 32;

// ------------------------------------------------------------------ PTX

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// 16-byte streaming load through the non-coherent path, no L1 allocation:
// the primitives read every input byte exactly once.
__device__ __forceinline__ uint4 ld_stream_v4(const void *p) {
  uint4 r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}

// 16-byte streaming store (evict-first): outputs are not re-read here.
__device__ __forceinline__ void st_stream_v4(void *p, uint4 v) {
  asm volatile("st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y),
               "r"(v.z), "r"(v.w)
               : "memory");
}

// Tile status word of the single-pass look-back: {payload, meta} read and
// written as ONE 128-bit access, so payload and flag are always seen
// together.  meta = (epoch << 8) | flags.
struct __align__(16) StatusWord {
  unsigned long long payload;
  unsigned long long meta;
};

constexpr unsigned long long kFlagAgg = 1;     // tile aggregate available
constexpr unsigned long long kFlagPrefix = 2;  // inclusive prefix available
constexpr unsigned long long kFlagError = 4;   // predecessor chain broken

__device__ __forceinline__ StatusWord ld_status(const StatusWord *p) {
  StatusWord r;
  asm volatile(
      "{\n .reg .b128 t;\n ld.relaxed.gpu.global.b128 t, [%2];\n mov.b128 {%0,%1}, t;\n}"
      : "=l"(r.payload), "=l"(r.meta)
      : "l"(p)
      : "memory");
  return r;
}

__device__ __forceinline__ void st_status(StatusWord *p, unsigned long long payload,
                                          unsigned long long meta) {
  asm volatile(
      "{\n .reg .b128 t;\n mov.b128 t, {%1,%2};\n st.relaxed.gpu.global.b128 [%0], t;\n}" ::"l"(p),
      "l"(payload), "l"(meta)
      : "memory");
}

// Per-call control block at the start of every scratch buffer.  Every
// launch that uses the scratch advances `epoch` (its last block does), and
// every word a launch writes into the scratch body is a StatusWord tagged
// with its epoch, so no launch can mistake another launch's words (of any
// primitive) for its own.
struct __align__(64) ScratchHeader {
  unsigned long long epoch;     // launches so far (56 bits used in tags)
  unsigned long long tile_ctr;  // dynamic tile ids (reset by the last block)
  unsigned int done_ctr;        // block arrivals, atomicInc-wrapped
  unsigned int error;           // sticky b2p_status of a device-side failure
  unsigned int pad[10];
};
constexpr size_t kHeaderBytes = 256;
// Fixed block of arrival counters right after the header (two-phase
// kernels).  Launches that use them leave them zero; nothing else writes
// there, so their position never overlaps another launch's data.
constexpr size_t kCounterSlots = 1024;
// Start of the per-launch body (epoch-tagged words) in every scratch buffer.
constexpr size_t kScratchPrefix = kHeaderBytes + kCounterSlots * 4;

// ------------------------------------------------------- double-float

struct DF {
  float hi, lo;
};

// Knuth TwoSum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
  s = __fadd_rn(a, b);
  float bp = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}

// Sum2 step (Ogita-Rump-Oishi): hi accumulates, lo collects exact errors.
__device__ __forceinline__ void df_accumulate(DF &a, float x) {
  float s, e;
  two_sum(a.hi, x, s, e);
  a.hi = s;
  a.lo = __fadd_rn(a.lo, e);
}

// (a.hi+a.lo) + (b.hi+b.lo), renormalised (|lo| <= ulp(hi)/2).
__device__ __forceinline__ DF df_add(DF a, DF b) {
  float s, e;
  two_sum(a.hi, b.hi, s, e);
  e = __fadd_rn(e, __fadd_rn(a.lo, b.lo));
  float h = __fadd_rn(s, e);
  float l = __fsub_rn(e, __fsub_rn(h, s));
  return DF{h, l};
}

__device__ __forceinline__ DF df_norm(DF a) {
  float h = __fadd_rn(a.hi, a.lo);
  float l = __fsub_rn(a.lo, __fsub_rn(h, a.hi));
  return DF{h, l};
}

__device__ __forceinline__ unsigned long long df_pack(DF a) {
  return (unsigned long long)__float_as_uint(a.hi) |
         ((unsigned long long)__float_as_uint(a.lo) << 32);
}
__device__ __forceinline__ DF df_unpack(unsigned long long v) {
  return DF{__uint_as_float((unsigned)(v & 0xffffffffu)), __uint_as_float((unsigned)(v >> 32))};
}

__device__ __forceinline__ float bf16_bits_to_f32(uint16_t h) {
  return __uint_as_float(((unsigned)h) << 16);
}

// ------------------------------------------------------- element policies
//
// A policy P describes one (storage type, operator) pair:
//   In        storage element read from memory
//   Acc       per-thread accumulator (<= 8 bytes)
//   Out       element written by scans / result of reductions
//   identity(), add(acc, x), combine(a, b), finalize(acc), from_out(v),
//   pack/unpack (64-bit payload for tile status words and partial slots).
// combine must be associative and commutative (all ops here are).

template <class T>
__device__ __forceinline__ unsigned long long to_bits64(T v) {
  unsigned long long r = 0;
  memcpy(&r, &v, sizeof(T));
  return r;
}
template <class T>
__device__ __forceinline__ T from_bits64(unsigned long long v) {
  T r;
  memcpy(&r, &v, sizeof(T));
  return r;
}

template <class T, int OP>
struct IntOp {
  __device__ static T identity() {
    if constexpr (OP == B2P_SUM || OP == B2P_OR || OP == B2P_XOR) return T(0);
    else if constexpr (OP == B2P_PROD) return T(1);
    else if constexpr (OP == B2P_AND) return T(~T(0));
    else if constexpr (OP == B2P_MIN) return T(((T)-1 > 0) ? ~T(0) : (T)(~(1ull << (sizeof(T) * 8 - 1))));
    else return T(((T)-1 > 0) ? T(0) : (T)(1ull << (sizeof(T) * 8 - 1)));
  }
  __device__ static T apply(T a, T b) {
    using U = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
    if constexpr (OP == B2P_SUM) return (T)((U)a + (U)b);
    else if constexpr (OP == B2P_PROD) return (T)((U)a * (U)b);
    else if constexpr (OP == B2P_MIN) return (a < b) ? a : b;
    else if constexpr (OP == B2P_MAX) return (a < b) ? b : a;
    else if constexpr (OP == B2P_AND) return a & b;
    else if constexpr (OP == B2P_OR) return a | b;
    else return a ^ b;
  }
};

template <class T, int OP>
struct IntPolicy {
  using In = T;
  using Acc = T;
  using Out = T;
  static constexpr bool kCompensated = false;
  __device__ static Acc identity() { return IntOp<T, OP>::identity(); }
  __device__ static Acc lift(In x) { return x; }
  __device__ static void add(Acc &a, In x) { a = IntOp<T, OP>::apply(a, x); }
  __device__ static Acc combine(Acc a, Acc b) { return IntOp<T, OP>::apply(a, b); }
  __device__ static Out finalize(Acc a) { return a; }
  __device__ static Acc from_out(Out v) { return v; }
  __device__ static unsigned long long pack(Acc a) { return to_bits64(a); }
  __device__ static Acc unpack(unsigned long long v) { return from_bits64<Acc>(v); }
};

// fp32 / bf16 / fp64 with PROD, MIN, MAX: plain arithmetic.  MIN/MAX follow
// sycl::minimum / sycl::maximum: (x < y) ? x : y and (x < y) ? y : x.
template <class S, class A, int OP>
struct FloatPlainPolicy {
  using In = S;
  using Acc = A;
  using Out = A;
  static constexpr bool kCompensated = false;
  __device__ static Acc identity() {
    if constexpr (OP == B2P_SUM) return A(0);
    else if constexpr (OP == B2P_PROD) return A(1);
    else if constexpr (OP == B2P_MIN) return A(INFINITY);
    else return A(-INFINITY);
  }
  __device__ static Acc lift(In x) {
    if constexpr (sizeof(In) == 2) return bf16_bits_to_f32(x);
    else return (A)x;
  }
  __device__ static Acc combine(Acc a, Acc b) {
    if constexpr (OP == B2P_SUM) return a + b;
    else if constexpr (OP == B2P_PROD) return a * b;
    else if constexpr (OP == B2P_MIN) return (a < b) ? a : b;
    else return (a < b) ? b : a;
  }
  __device__ static void add(Acc &a, In x) { a = combine(a, lift(x)); }
  __device__ static Out finalize(Acc a) { return a; }
  __device__ static Acc from_out(Out v) { return v; }
  __device__ static unsigned long long pack(Acc a) { return to_bits64(a); }
  __device__ static Acc unpack(unsigned long long v) { return from_bits64<Acc>(v); }
};

// fp32 / bf16 SUM: compensated (Sum2) accumulation, double-float combine.
template <class S>
struct FloatSumPolicy {
  using In = S;
  using Acc = DF;
  using Out = float;
  static constexpr bool kCompensated = true;
  __device__ static Acc identity() { return DF{0.f, 0.f}; }
  __device__ static float lift_f(In x) {
    if constexpr (sizeof(In) == 2) return bf16_bits_to_f32(x);
    else return x;
  }
  __device__ static Acc lift(In x) { return DF{lift_f(x), 0.f}; }
  __device__ static void add(Acc &a, In x) { df_accumulate(a, lift_f(x)); }
  __device__ static Acc combine(Acc a, Acc b) { return df_add(a, b); }
  __device__ static Out finalize(Acc a) { return __fadd_rn(a.hi, a.lo); }
  __device__ static Acc from_out(Out v) { return DF{v, 0.f}; }
  __device__ static unsigned long long pack(Acc a) { return df_pack(a); }
  __device__ static Acc unpack(unsigned long long v) { return df_unpack(v); }
};

// Policy selector for (dtype code, op code).
template <int DT, int OP>
struct PolicyOf;
#define B2P_INT_POLICY(DT, T)                                   \
  template <int OP>                                             \
  struct PolicyOf<DT, OP> {                                     \
    using type = IntPolicy<T, OP>;                              \
  };
B2P_INT_POLICY(B2P_I32, int32_t)
B2P_INT_POLICY(B2P_I64, long long)
B2P_INT_POLICY(B2P_U32, uint32_t)
B2P_INT_POLICY(B2P_U64, unsigned long long)
#undef B2P_INT_POLICY
template <int OP>
struct PolicyOf<B2P_F32, OP> {
  using type = typename std::conditional<OP == B2P_SUM, FloatSumPolicy<float>,
                                         FloatPlainPolicy<float, float, OP>>::type;
};
template <int OP>
struct PolicyOf<B2P_BF16, OP> {
  using type = typename std::conditional<OP == B2P_SUM, FloatSumPolicy<uint16_t>,
                                         FloatPlainPolicy<uint16_t, float, OP>>::type;
};
template <int OP>
struct PolicyOf<B2P_F64, OP> {
  using type = FloatPlainPolicy<double, double, OP>;
};

// ------------------------------------------------------- warp collectives

template <class A>
__device__ __forceinline__ A shfl_xor(A v, int m) {
  if constexpr (sizeof(A) == 4) {
    unsigned u;
    memcpy(&u, &v, 4);
    u = __shfl_xor_sync(0xffffffffu, u, m);
    memcpy(&v, &u, 4);
    return v;
  } else {
    unsigned long long u;
    memcpy(&u, &v, 8);
    u = __shfl_xor_sync(0xffffffffu, u, m);
    memcpy(&v, &u, 8);
    return v;
  }
}

template <class A>
__device__ __forceinline__ A shfl_up(A v, int d) {
  if constexpr (sizeof(A) == 4) {
    unsigned u;
    memcpy(&u, &v, 4);
    u = __shfl_up_sync(0xffffffffu, u, d);
    memcpy(&v, &u, 4);
    return v;
  } else {
    unsigned long long u;
    memcpy(&u, &v, 8);
    u = __shfl_up_sync(0xffffffffu, u, d);
    memcpy(&v, &u, 8);
    return v;
  }
}

template <class A>
__device__ __forceinline__ A shfl_idx(A v, int src) {
  if constexpr (sizeof(A) == 4) {
    unsigned u;
    memcpy(&u, &v, 4);
    u = __shfl_sync(0xffffffffu, u, src);
    memcpy(&v, &u, 4);
    return v;
  } else {
    unsigned long long u;
    memcpy(&u, &v, 8);
    u = __shfl_sync(0xffffffffu, u, src);
    memcpy(&v, &u, 8);
    return v;
  }
}

// Butterfly all-reduce: every lane ends with the same value, computed by the
// same fixed tree.  32-bit integer add/min/max/and/or/xor use redux.sync.
template <class P>
__device__ __forceinline__ typename P::Acc warp_allreduce(typename P::Acc a) {
  using A = typename P::Acc;
  if constexpr (std::is_same<P, IntPolicy<uint32_t, B2P_SUM>>::value ||
                std::is_same<P, IntPolicy<int32_t, B2P_SUM>>::value) {
    return (A)__reduce_add_sync(0xffffffffu, (unsigned)a);
  } else if constexpr (std::is_same<P, IntPolicy<uint32_t, B2P_MIN>>::value) {
    return __reduce_min_sync(0xffffffffu, a);
  } else if constexpr (std::is_same<P, IntPolicy<uint32_t, B2P_MAX>>::value) {
    return __reduce_max_sync(0xffffffffu, a);
  } else if constexpr (std::is_same<P, IntPolicy<int32_t, B2P_MIN>>::value) {
    return __reduce_min_sync(0xffffffffu, a);
  } else if constexpr (std::is_same<P, IntPolicy<int32_t, B2P_MAX>>::value) {
    return __reduce_max_sync(0xffffffffu, a);
  } else if constexpr (std::is_same<P, IntPolicy<uint32_t, B2P_AND>>::value ||
                       std::is_same<P, IntPolicy<int32_t, B2P_AND>>::value) {
    return (A)__reduce_and_sync(0xffffffffu, (unsigned)a);
  } else if constexpr (std::is_same<P, IntPolicy<uint32_t, B2P_OR>>::value ||
                       std::is_same<P, IntPolicy<int32_t, B2P_OR>>::value) {
    return (A)__reduce_or_sync(0xffffffffu, (unsigned)a);
  } else if constexpr (std::is_same<P, IntPolicy<uint32_t, B2P_XOR>>::value ||
                       std::is_same<P, IntPolicy<int32_t, B2P_XOR>>::value) {
    return (A)__reduce_xor_sync(0xffffffffu, (unsigned)a);
  } else {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) a = P::combine(a, shfl_xor(a, m));
    return a;
  }
}

// Inclusive warp scan (Kogge-Stone over shuffles).
template <class P>
__device__ __forceinline__ typename P::Acc warp_inclusive_scan(typename P::Acc a, int lane) {
#pragma unroll
  for (int d = 1; d < kWarp; d <<= 1) {
    typename P::Acc o = shfl_up(a, d);
    if (lane >= d) a = P::combine(o, a);
  }
  return a;
}

// ------------------------------------------------------- launch table

struct LaunchConfig {
  int block;
  int items;
  int grid_mode;
};

__host__ __device__ inline LaunchConfig describe_config(int c) {
  LaunchConfig lc;
  lc.grid_mode = c / 16;
  lc.block = 128 << ((c / 4) % 4);
  lc.items = 4 << (c % 4);
  return lc;
}

}  // namespace b2p
