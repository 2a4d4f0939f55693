// Sharded reduce, dot and scan over the ranks of an NCCL communicator, for C and
// C++ hosts (one process or thread per GPU; rank r holds the r-th shard of
// one logical array, rank order = element order).  The same single-exchange
// plan as the Python layer (opensycl_b200/sharded.py):
//   reduce  local reduce of the shard, all-gather of the P partials, combined
//           in rank order on the host (the same bits on every rank);
//   scan    local total (a reduce), all-gather of the P totals, then one
//           local scan whose init is the combination of the totals of the
//           ranks before (the carry).
// Each partial travels as 16 bytes: the 8-byte value and a present flag (an
// empty shard contributes nothing), gathered with one ncclAllGather on the
// caller's stream.  NCCL's functions are taken from the libnccl.so.2 already
// loaded in the process (or loaded on first use): the library does not link
// NCCL, and the communicator the caller passes must come from that same
// library.  b2p_shard_combine is the host combination on its own, for hosts
// that exchange the partials with another transport (MPI, gloo, sockets).
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.h"

namespace b2p {

namespace {

struct NcclApi {
  ncclResult_t (*all_gather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*count)(ncclComm_t, int *) = nullptr;
  ncclResult_t (*user_rank)(ncclComm_t, int *) = nullptr;
  bool ok = false;
};

const NcclApi &nccl_api() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    api.all_gather = reinterpret_cast<decltype(api.all_gather)>(dlsym(h, "ncclAllGather"));
    api.count = reinterpret_cast<decltype(api.count)>(dlsym(h, "ncclCommCount"));
    api.user_rank = reinterpret_cast<decltype(api.user_rank)>(dlsym(h, "ncclCommUserRank"));
    api.ok = api.all_gather && api.count && api.user_rank;
  });
  return api;
}

// a op b of the accumulator type A: integers wrap (unsigned arithmetic),
// floats are combined in double by the caller
template <class A>
A int_combine(int op, A a, A b) {
  using U = typename std::make_unsigned<A>::type;
  switch (op) {
  case B2P_SUM: return (A)((U)a + (U)b);
  case B2P_PROD: return (A)((U)a * (U)b);
  case B2P_MIN: return b < a ? b : a;
  case B2P_MAX: return a < b ? b : a;
  case B2P_AND: return a & b;
  case B2P_OR: return a | b;
  default: return a ^ b;
  }
}

double float_combine(int op, double a, double b) {
  switch (op) {
  case B2P_SUM: return a + b;
  case B2P_PROD: return a * b;
  case B2P_MIN: return b < a ? b : a;
  default: return a < b ? b : a;
  }
}

template <class A>
int fold_int(int op, const unsigned char *vals, const unsigned char *present, int count, size_t stride,
             const void *init, void *result) {
  bool have = init != nullptr;
  A r{};
  if (have) memcpy(&r, init, sizeof(A));
  for (int i = 0; i < count; ++i) {
    if (present && !present[(size_t)i * stride]) continue;
    A v;
    memcpy(&v, vals + (size_t)i * stride, sizeof(A));
    r = have ? int_combine<A>(op, r, v) : v;
    have = true;
  }
  if (!have) return B2P_ERR_INVALID_ARG;
  memcpy(result, &r, sizeof(A));
  return B2P_OK;
}

template <class A>
int fold_float(int op, const unsigned char *vals, const unsigned char *present, int count, size_t stride,
               const void *init, void *result) {
  bool have = init != nullptr;
  double r = 0.0;
  if (have) {
    A a;
    memcpy(&a, init, sizeof(A));
    r = (double)a;
  }
  for (int i = 0; i < count; ++i) {
    if (present && !present[(size_t)i * stride]) continue;
    A v;
    memcpy(&v, vals + (size_t)i * stride, sizeof(A));
    r = have ? float_combine(op, r, (double)v) : (double)v;
    have = true;
  }
  if (!have) return B2P_ERR_INVALID_ARG;
  const A out = (A)r;
  memcpy(result, &out, sizeof(A));
  return B2P_OK;
}

// init op v[0] op ... op v[count - 1] over the present entries; values of
// the accumulator type at vals + i * stride, present flags (when given) at
// present + i * stride.  B2P_ERR_INVALID_ARG when there is nothing to fold.
int fold(int dtype, int op, const unsigned char *vals, const unsigned char *present, int count, size_t stride,
         const void *init, void *result) {
  switch (dtype) {
  case B2P_I32: return fold_int<int32_t>(op, vals, present, count, stride, init, result);
  case B2P_I64: return fold_int<int64_t>(op, vals, present, count, stride, init, result);
  case B2P_U32: return fold_int<uint32_t>(op, vals, present, count, stride, init, result);
  case B2P_U64: return fold_int<uint64_t>(op, vals, present, count, stride, init, result);
  case B2P_F32:
  case B2P_BF16: return fold_float<float>(op, vals, present, count, stride, init, result);
  case B2P_F64: return fold_float<double>(op, vals, present, count, stride, init, result);
  default: return B2P_ERR_INVALID_ARG;
  }
}

bool op_ok(int dtype, int op) {
  if (dtype < B2P_I32 || dtype > B2P_F64 || op < B2P_SUM || op > B2P_XOR) return false;
  return !(dtype_is_float(dtype) && op > B2P_MAX);
}

constexpr size_t kEntry = 16;  // value (8 bytes) + present flag (8 bytes)

// Scratch of the sharded calls: the local primitive's scratch, then this
// rank's entry, then the gathered entries of `world` ranks.
size_t local_part(size_t n, int dtype, int prim) {
  const size_t b = b2p_scratch_bytes(prim, dtype, n, 0, B2P_CONFIG_AUTO);
  return (b + 255) / 256 * 256;
}

// The shard partial of every rank on the host: local reduce (or dot, when
// `b` is given) into this rank's entry, one all-gather, one copy back.
// entries: world * kEntry.
int gather_partials(int dtype, int op, const void *in, const void *b, size_t n, void *scratch, size_t scratch_bytes,
                    int config, ncclComm_t comm, int world, cudaStream_t st, std::vector<unsigned char> &entries) {
  const NcclApi &nc = nccl_api();
  const size_t base = std::max({local_part(n, dtype, B2P_PRIM_REDUCE), local_part(n, dtype, B2P_PRIM_SCAN),
                                local_part(n, dtype, B2P_PRIM_DOT)});
  if (scratch_bytes < base + 256 + kEntry * (size_t)world) return B2P_ERR_SCRATCH;
  unsigned char *mine = reinterpret_cast<unsigned char *>(scratch) + base;
  unsigned char *all = mine + 256;
  unsigned long long flag = n > 0 ? 1ull : 0ull;
  cudaError_t e = cudaMemsetAsync(mine, 0, kEntry, st);
  if (e != cudaSuccess) return cuda_status(e);
  if (n > 0) {
    const int rc = b ? b2p_dot(dtype, in, b, n, mine, nullptr, scratch, base, config, (b2p_stream)st)
                     : b2p_reduce(dtype, op, in, n, mine, nullptr, scratch, base, config, (b2p_stream)st);
    if (rc) return rc;
  }
  if ((e = cudaMemcpyAsync(mine + 8, &flag, 8, cudaMemcpyHostToDevice, st)) != cudaSuccess) return cuda_status(e);
  if (nc.all_gather(mine, all, kEntry, ncclUint8, comm, st) != ncclSuccess) return B2P_ERR_CUDA;
  entries.resize(kEntry * (size_t)world);
  if ((e = cudaMemcpyAsync(entries.data(), all, entries.size(), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return cuda_status(e);
  // the host buffers (flag, entries) are read and written by the copies above
  return cuda_status(cudaStreamSynchronize(st));
}

int comm_shape(void *nccl_comm, int *world, int *rank) {
  const NcclApi &nc = nccl_api();
  if (!nc.ok) return B2P_ERR_UNSUPPORTED;
  if (!nccl_comm) return B2P_ERR_INVALID_ARG;
  if (nc.count((ncclComm_t)nccl_comm, world) != ncclSuccess ||
      nc.user_rank((ncclComm_t)nccl_comm, rank) != ncclSuccess || *world < 1)
    return B2P_ERR_INVALID_ARG;
  return B2P_OK;
}

}  // namespace

}  // namespace b2p

using namespace b2p;

extern "C" int b2p_shard_combine(int dtype, int op, const void *values, int count, size_t stride,
                                 const void *init, void *result) {
  if (!op_ok(dtype, op) || count < 0 || !result || (count > 0 && !values) || stride < acc_size(dtype))
    return B2P_ERR_INVALID_ARG;
  return fold(dtype, op, reinterpret_cast<const unsigned char *>(values), nullptr, count, stride, init, result);
}

extern "C" size_t b2p_sharded_scratch_bytes(int dtype, size_t n, int world) {
  if (world < 1) return 0;
  return std::max({local_part(n, dtype, B2P_PRIM_REDUCE), local_part(n, dtype, B2P_PRIM_SCAN),
                   local_part(n, dtype, B2P_PRIM_DOT)}) +
         256 + kEntry * (size_t)world + 256;
}

extern "C" int b2p_sharded_reduce(int dtype, int op, const void *in, size_t n, void *out, const void *init,
                                  void *scratch, size_t scratch_bytes, int config, void *nccl_comm,
                                  b2p_stream stream) {
  CallScope cs("b2p_sharded_reduce", dtype, n, 0, (double)n * dtype_size(dtype), stream);
  if (!op_ok(dtype, op)) return cs.done(B2P_ERR_INVALID_ARG);
  int world = 0, rank = 0;
  int rc = comm_shape(nccl_comm, &world, &rank);
  if (rc) return cs.done(rc);
  if ((rc = check_pointer(out, acc_size(dtype)))) return cs.done(rc);
  if (!scratch) return cs.done(B2P_ERR_SCRATCH);
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<unsigned char> entries;
  if ((rc = gather_partials(dtype, op, in, nullptr, n, scratch, scratch_bytes, config, (ncclComm_t)nccl_comm, world,
                            st, entries)))
    return cs.done(rc);
  unsigned long long r = 0;
  rc = fold(dtype, op, entries.data(), entries.data() + 8, world, kEntry, init, &r);
  if (rc == B2P_ERR_INVALID_ARG) return cs.done(B2P_OK);  // every shard empty and no init: out untouched
  if (rc) return cs.done(rc);
  cudaError_t e = cudaMemcpyAsync(out, &r, acc_size(dtype), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // r is a host local
  return cs.done(cuda_status(e));
}

extern "C" int b2p_sharded_scan(int dtype, int op, int inclusive, const void *in, void *out, size_t n,
                                const void *init, void *scratch, size_t scratch_bytes, int config, void *nccl_comm,
                                b2p_stream stream) {
  CallScope cs("b2p_sharded_scan", dtype, n, 0, (double)n * (dtype_size(dtype) + acc_size(dtype)), stream);
  if (!op_ok(dtype, op)) return cs.done(B2P_ERR_INVALID_ARG);
  if (!inclusive && !init) return cs.done(B2P_ERR_INVALID_ARG);
  int world = 0, rank = 0;
  int rc = comm_shape(nccl_comm, &world, &rank);
  if (rc) return cs.done(rc);
  if (!scratch) return cs.done(B2P_ERR_SCRATCH);
  cudaStream_t st = (cudaStream_t)stream;
  if (world == 1)  // nothing to exchange
    return cs.done(b2p_scan(dtype, op, inclusive, in, out, n, init, scratch, scratch_bytes, config, stream));
  std::vector<unsigned char> entries;
  if ((rc = gather_partials(dtype, op, in, nullptr, n, scratch, scratch_bytes, config, (ncclComm_t)nccl_comm, world,
                            st, entries)))
    return cs.done(rc);
  if (n == 0) return cs.done(B2P_OK);
  // carry = init op totals of the ranks before this one
  unsigned long long carry = 0;
  rc = fold(dtype, op, entries.data(), entries.data() + 8, rank, kEntry, init, &carry);
  if (rc == B2P_ERR_INVALID_ARG)  // rank 0 of an inclusive scan without init (or all earlier shards empty)
    return cs.done(b2p_scan(dtype, op, inclusive, in, out, n, nullptr, scratch, scratch_bytes, config, stream));
  if (rc) return cs.done(rc);
  return cs.done(b2p_scan(dtype, op, inclusive, in, out, n, &carry, scratch, scratch_bytes, config, stream));
}

extern "C" int b2p_sharded_dot(int dtype, const void *a, const void *b, size_t n, void *out, const void *init,
                               void *scratch, size_t scratch_bytes, int config, void *nccl_comm, b2p_stream stream) {
  CallScope cs("b2p_sharded_dot", dtype, n, 0, 2.0 * (double)n * dtype_size(dtype), stream);
  if (dtype != B2P_F32 && dtype != B2P_BF16 && dtype != B2P_F64) return cs.done(B2P_ERR_UNSUPPORTED);
  int world = 0, rank = 0;
  int rc = comm_shape(nccl_comm, &world, &rank);
  if (rc) return cs.done(rc);
  if ((rc = check_pointer(out, acc_size(dtype)))) return cs.done(rc);
  if (!scratch) return cs.done(B2P_ERR_SCRATCH);
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<unsigned char> entries;
  if ((rc = gather_partials(dtype, B2P_SUM, a, b, n, scratch, scratch_bytes, config, (ncclComm_t)nccl_comm, world,
                            st, entries)))
    return cs.done(rc);
  unsigned long long r = 0;
  rc = fold(dtype, B2P_SUM, entries.data(), entries.data() + 8, world, kEntry, init, &r);
  if (rc == B2P_ERR_INVALID_ARG) return cs.done(B2P_OK);  // every shard empty and no init: out untouched
  if (rc) return cs.done(rc);
  cudaError_t e = cudaMemcpyAsync(out, &r, acc_size(dtype), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cs.done(cuda_status(e));
}
