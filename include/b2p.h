/*
 * b2p.h — C-ABI of the B200-native data-parallel primitive library
 * (libb2p.so).  Plain pointers and sizes; no C++ or torch types.
 *
 * Every entry point here replaces one AdaptiveCpp interface on the
 * data-parallel primitive path; the reference file:line it stands in for is
 * given beside it (paths inside the AdaptiveCpp source tree).  The C++
 * drop-in headers under include/hipSYCL_b2p/ wrap these calls behind the
 * reference's own signatures.
 *
 * Conventions
 *  - `stream` is a cudaStream_t (0 = legacy default stream).  Every compute
 *    call is asynchronous on that stream, like a SYCL submission; nothing
 *    blocks the host unless its comment says so.
 *  - Input/output pointers must be device-accessible (device, managed or
 *    mapped pinned host memory) and naturally aligned for their element
 *    type.  They are checked with cudaPointerGetAttributes; a pageable host
 *    pointer is rejected with B2P_ERR_INVALID_PTR (there is no CPU fallback).
 *  - `init` arguments are HOST pointers to one value of the accumulation
 *    type (fp32 for bf16 inputs); the value is captured at call time.
 *  - `scratch` is device memory of at least b2p_scratch_bytes(...) bytes,
 *    zero-filled once before its first use (b2p_scratch_init).  Every call
 *    leaves it ready for the next one, including calls whose device-side
 *    waits timed out.  One scratch buffer must not be used by two calls
 *    that can overlap on the GPU (same rule as the reference's
 *    util::allocation_group, algorithms/util/allocation_cache.hpp:129-142).
 *  - `config` selects a launch configuration: 0..B2P_NUM_CONFIGS-1 from the
 *    fixed table (b2p_config_describe), or B2P_CONFIG_AUTO to let the
 *    library choose (learned selector, falling back to the exhaustive tuner
 *    table, then to a fixed heuristic).  The configuration never changes an
 *    integer result; float results stay within the documented tolerance.
 *  - n == 0: outputs are left untouched and no kernel is launched, as in
 *    the reference (algorithms/numeric.hpp:165-169).
 *  - Every call that launches work opens an NVTX range named after it
 *    (b2p_reduce, b2p_scan, ...) for the duration of the host call.
 *
 * Environment (read once per process)
 *  - B2P_LOG_LEVEL: see b2p_log_level().  Errors are logged at level >= 1,
 *    one record per call (operation, dtype, n, segments, configuration,
 *    status) at 3, and at 4 the call is timed on its stream and the record
 *    adds milliseconds and GB/s.
 *  - B2P_CHECKED=1: the extent of every pointer argument (elements x size)
 *    must lie inside one device allocation, and segment offsets are copied
 *    to the host and checked (non-decreasing, inside the input); a failed
 *    check returns B2P_ERR_INVALID_PTR / B2P_ERR_INVALID_ARG before
 *    anything is launched.  Off by default (the offsets check synchronises
 *    the stream).
 *  - B2P_SELECTOR: how B2P_CONFIG_AUTO chooses: "learned" (default: the
 *    installed selector table, else the fixed heuristic), "heuristic", or
 *    the path of a selector weights file (b2p_selector_save) that is loaded
 *    and installed at the first AUTO call.
 *  - B2P_SCAN_CHUNK_MB (default 16) and B2P_SCAN_LOOKAHEAD (default 2):
 *    chunk size in MiB of input, and how many chunks the first phase runs
 *    ahead of the second, of the two-phase scan kernel (persistent grid
 *    modes 1 and 2 of the scan configurations that do not run the TMA
 *    pipeline).  They change timing only, never results.
 */
#ifndef B2P_H
#define B2P_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *b2p_stream; /* == cudaStream_t */

typedef enum b2p_status {
  B2P_OK = 0,
  B2P_ERR_INVALID_ARG = 1,  /* bad size, dtype, op, config or NULL */
  B2P_ERR_INVALID_PTR = 2,  /* pointer not device-accessible / misaligned */
  B2P_ERR_TIMEOUT = 3,      /* a bounded device-side wait gave up */
  B2P_ERR_CUDA = 4,         /* a CUDA runtime call failed */
  B2P_ERR_UNSUPPORTED = 5,  /* dtype/op combination not provided */
  B2P_ERR_SCRATCH = 6,      /* scratch NULL, too small or misaligned */
  B2P_ERR_NO_DEVICE = 7,    /* no CUDA device / not an sm_100 device */
  B2P_ERR_IO = 8            /* selector / tuner file could not be read */
} b2p_status;

typedef enum b2p_dtype {
  B2P_I32 = 0,
  B2P_I64 = 1,
  B2P_U32 = 2,
  B2P_U64 = 3,
  B2P_F32 = 4,
  B2P_BF16 = 5, /* bf16 storage; accumulates in fp32, fp32 init/output */
  B2P_F64 = 6
} b2p_dtype;

/* sycl::plus / multiplies / minimum / maximum / bit_and / bit_or / bit_xor
 * (sycl/libkernel/functional.hpp).  Floating-point dtypes take SUM, PROD,
 * MIN, MAX.  min/max use the true identities (+inf / -inf for floats);
 * the drop-in header folds the reference's identity table into init. */
typedef enum b2p_op {
  B2P_SUM = 0,
  B2P_PROD = 1,
  B2P_MIN = 2,
  B2P_MAX = 3,
  B2P_AND = 4,
  B2P_OR = 5,
  B2P_XOR = 6
} b2p_op;

/* primitive ids, used by the scratch query, the tuner and the selector */
typedef enum b2p_prim {
  B2P_PRIM_REDUCE = 0,
  B2P_PRIM_SCAN = 1,
  B2P_PRIM_COPY_IF = 2,
  B2P_PRIM_HISTOGRAM = 3,
  B2P_PRIM_DOT = 4,
  B2P_PRIM_SEG_REDUCE = 5,
  B2P_PRIM_SEG_SCAN = 6,
  B2P_PRIM_SORT = 7,  /* scratch sizing only */
  B2P_PRIM_MERGE = 8  /* scratch sizing only (n = total keys) */
} b2p_prim;

/* copy_if predicate family: (x & mask) CMP rhs on the element's bits */
typedef enum b2p_cmp {
  B2P_CMP_LT = 0,
  B2P_CMP_LE = 1,
  B2P_CMP_EQ = 2,
  B2P_CMP_NE = 3,
  B2P_CMP_GE = 4,
  B2P_CMP_GT = 5
} b2p_cmp;

#define B2P_NUM_CONFIGS 48
#define B2P_CONFIG_AUTO (-1)

/* ---------------------------------------------------------------- library */

/* Library version string, e.g. "0.1.0 sm_100a". */
const char *b2p_version(void);

/* Human-readable text for a status code. */
const char *b2p_status_string(int status);

/* Architecture the library's kernels were compiled for, as the CUDA runtime
 * reports it for one of them on the current device (cudaFuncGetAttributes:
 * binaryVersion 100 = sm_100a machine code, ptxVersion 0 when no PTX is
 * embedded).  Stands in for the reference's device/backend query
 * (sycl/device.hpp:66-69); the library has one target only. */
int b2p_kernel_arch(int *binary_version, int *ptx_version);

/* Configuration table entry c: threads per block {128,256,512,1024},
 * items per thread {4,8,16,32}, grid mode {0: one tile per block,
 * 1: persistent at full occupancy, 2: persistent at half occupancy}.
 * Replaces the fixed launch shapes of util/memory_streaming.hpp:30-47
 * (4*CUs groups of 128) and algorithms/scan/scan.hpp:26-32 (WG 128 / 1024).
 * Returns B2P_ERR_INVALID_ARG for c outside the table. */
int b2p_config_describe(int config, int *block, int *items, int *grid_mode);

/* Whether config c can run primitive `prim` on `dtype` (shared-memory
 * limits).  1 = valid, 0 = masked. */
int b2p_config_valid(int prim, int dtype, int config);

/* Scratch bytes needed by one call.  Replaces the allocation_group::obtain
 * requests of reduction_engine.hpp:295-351 and
 * decoupled_lookback_scan.hpp:36-47,581-582.  `n` is the element count
 * (total elements for segmented calls), `nseg` the segment count (0 for
 * non-segmented primitives).  An upper bound over every config when
 * config == B2P_CONFIG_AUTO. */
size_t b2p_scratch_bytes(int prim, int dtype, size_t n, int64_t nseg, int config);

/* Zero-fill scratch on `stream` (cudaMemsetAsync).  Required once per new
 * scratch buffer. */
int b2p_scratch_init(void *scratch, size_t scratch_bytes, b2p_stream stream);

/* ------------------------------------------------------------ primitives */

/* *out = op(init, x[0] op ... op x[n-1]); init == NULL: *out = op(*out, r)
 * (the no-initialize_to_identity form of sycl::reduction).
 * Replaces hipsycl::algorithms::reduce (algorithms/numeric.hpp:226-249),
 * its engine (numeric.hpp:67-161, reduction/reduction_engine.hpp:116-390)
 * and the sycl::reduction handler path (sycl/handler.hpp:799-897).
 * fp32/bf16 SUM accumulates with compensated (TwoSum) fp32 arithmetic and a
 * fixed, configuration-independent combination tree: the bits of a float
 * result do not depend on `config`. */
int b2p_reduce(int dtype, int op, const void *in, size_t n, void *out,
               const void *init, void *scratch, size_t scratch_bytes,
               int config, b2p_stream stream);

/* Size of the library-resident scratch area used by b2p_reduce_static,
 * and the largest element count that entry point accepts. */
#define B2P_STATIC_SCRATCH_BYTES (128u * 1024u)
#define B2P_STATIC_MAX_ELEMS ((size_t)1 << 34)

/* Allocation-free reduce: the same result as b2p_reduce for the same
 * arguments, but with no scratch argument.  No counterpart in the reference
 * (its reduce always obtains scratch from an allocation_group).
 *
 * For callers that cannot allocate device memory -- code running inside a
 * device-memory allocator or pool callback, real-time paths whose memory is
 * fixed at start-up, host runtimes that own the device heap.  It calls no
 * cudaMalloc, cudaFree or other allocating routine; its scratch is a
 * B2P_STATIC_SCRATCH_BYTES array inside the library, which every GPU that
 * loads the library keeps until the process exits.
 *  - Every call looks up that array's device address (cudaGetSymbolAddress,
 *    with the device current), so an address from an earlier context is
 *    never used.  The first call on each device, and the first after its
 *    context was rebuilt (cudaDeviceReset), also loads the library's module
 *    and every reduce kernel this entry point can launch -- a driver-side
 *    allocation.  Make that first call at start-up, before any stream
 *    capture and outside any allocator callback; later calls load nothing.
 *  - All calls on a device share the one array: calls that can overlap on
 *    the GPU (different streams without ordering) race and must not be
 *    issued.  Each call clears the array's counters before its launch,
 *    after its arguments were checked (a rejected call leaves the array as
 *    it was).
 *  - n > B2P_STATIC_MAX_ELEMS returns B2P_ERR_INVALID_ARG; a call whose
 *    scratch need exceeds the array returns B2P_ERR_SCRATCH. */
int b2p_reduce_static(int dtype, int op, const void *in, size_t n, void *out,
                      const void *init, b2p_stream stream);

/* *out = init + sum a[i]*b[i]  (transform_reduce with plus/multiplies,
 * algorithms/numeric.hpp:170-192,215-223).  dtype F32, BF16 (fp32 out) or
 * F64.  fp32 uses Dot2 (fma TwoProduct + TwoSum). */
int b2p_dot(int dtype, const void *a, const void *b, size_t n, void *out,
            const void *init, void *scratch, size_t scratch_bytes, int config,
            b2p_stream stream);

/* Inclusive (inclusive != 0) or exclusive scan of in[0..n) into out.
 * init may be NULL for an inclusive scan; an exclusive scan requires it.
 * in == out is allowed.  bf16 input writes fp32 output.
 * Replaces inclusive_scan / exclusive_scan (algorithms/numeric.hpp:253-297),
 * scanning::scan (algorithms/scan/scan.hpp:51-83) and the decoupled
 * look-back kernel (algorithms/scan/decoupled_lookback_scan.hpp:555-655).
 * Every look-back wait is bounded: on time-out the call records
 * B2P_ERR_TIMEOUT in scratch (read with b2p_device_error). */
int b2p_scan(int dtype, int op, int inclusive, const void *in, void *out,
             size_t n, const void *init, void *scratch, size_t scratch_bytes,
             int config, b2p_stream stream);

/* Order-preserving compaction of the elements with (x & mask) CMP rhs.
 * Element size 4 (dtype I32/U32/F32) or 8 (I64/U64/F64); mask/rhs are
 * compared on the unsigned bit pattern.  *num_copied (device-accessible,
 * may be NULL) receives the count.  `out` must have room for n elements
 * (the count is not known before the call); writes never go past n.
 * Replaces hipsycl::algorithms::copy_if (algorithms/algorithm.hpp:178-243). */
int b2p_copy_if(int dtype, const void *in, void *out, size_t n, uint64_t mask,
                int cmp, uint64_t rhs, uint64_t *num_copied, void *scratch,
                size_t scratch_bytes, int config, b2p_stream stream);

/* bins[k] += |{i : keys[i] == k}| for k < nbins (nbins <= 256), modulo 2^32;
 * keys >= nbins are skipped.  The accumulate-into-bins semantics are those
 * of a parallel_for that calls
 * sycl::atomic_ref<uint32_t,...>::fetch_add(1) on bins[key]
 * (sycl/libkernel/atomic_ref.hpp:143-149,253-260). */
int b2p_histogram_u8(const uint8_t *keys, size_t n, uint32_t *bins, int nbins,
                     int config, b2p_stream stream);

/* Per-segment reduce over CSR offsets (offsets[0..nseg], device-accessible,
 * non-decreasing): out[s] = init op x[offsets[s]] op ... ; empty segments
 * get init.  init == NULL means the identity.  One launch for all segments.
 * No reference function; its analogue is one reduce call per segment. */
int b2p_segmented_reduce(int dtype, int op, const void *in,
                         const int64_t *offsets, int64_t nseg, void *out,
                         const void *init, void *scratch, size_t scratch_bytes,
                         int config, b2p_stream stream);

/* Per-segment inclusive/exclusive scan over CSR offsets, one launch.
 * Exclusive scans start each segment at init (required); inclusive scans
 * apply init (may be NULL) to each segment's first element.
 * Analogue: one inclusive_scan call per segment (numeric.hpp:253-279). */
int b2p_segmented_scan(int dtype, int op, int inclusive, const void *in,
                       void *out, const int64_t *offsets, int64_t nseg,
                       const void *init, void *scratch, size_t scratch_bytes,
                       int config, b2p_stream stream);

/* The per-call analogue of the two functions above, for comparison: one
 * b2p_reduce (prim = B2P_PRIM_SEG_REDUCE) or inclusive b2p_scan
 * (B2P_PRIM_SEG_SCAN) call per non-empty segment, issued from a host loop
 * over HOST offsets; empty reduce segments get the identity.  This is what
 * the reference does for a batch of segments (numeric.hpp:226-279, one
 * call each).  scratch must fit the largest segment. */
int b2p_segmented_per_call(int prim, int dtype, int op, const void *in, void *out,
                           const int64_t *host_offsets, int64_t nseg, void *scratch,
                           size_t scratch_bytes, int config, b2p_stream stream);

/* Stable merge of the sorted ranges a[0..na) and b[0..nb) into
 * out[0..na+nb) (ascending, or descending when descending != 0; on equal
 * keys the elements of a come first).  dtype I32, I64, U32, U64, F32, F64;
 * floats compare with < (NaNs unordered).  One pass: merge-path tiles.
 * scratch: device memory of at least b2p_scratch_bytes(B2P_PRIM_MERGE,
 * dtype, na + nb, 0, B2P_CONFIG_AUTO) bytes (the tile starts; no
 * initialisation needed, and like b2p_sort's not a look-back scratch
 * buffer of the other primitives).
 * Replaces hipsycl::algorithms::merge (algorithms/algorithm.hpp:519-560,
 * algorithms/merge/merge.hpp:222-313) for these types with std::less /
 * std::greater. */
int b2p_merge(int dtype, const void *a, size_t na, const void *b, size_t nb, void *out, int descending,
              void *scratch, size_t scratch_bytes, b2p_stream stream);

/* Sort keys[0..n) in place, ascending (descending != 0: descending),
 * stable.  dtype as b2p_merge.  scratch: device memory of at least
 * b2p_scratch_bytes(B2P_PRIM_SORT, dtype, n, 0, B2P_CONFIG_AUTO) bytes (a
 * second array of n keys and the merge passes' tile starts; its contents
 * need no initialisation).  The sort
 * overwrites it with keys, so it must not be a scratch buffer that the
 * other primitives use for their look-back status words.  A merge
 * sort: tiles sorted in shared memory, then log2(n / tile) merge passes.
 * Replaces hipsycl::algorithms::sort (algorithms/algorithm.hpp:519-529,
 * algorithms/sort/bitonic_sort.hpp:69-110). */
int b2p_sort(int dtype, void *keys, size_t n, int descending, void *scratch, size_t scratch_bytes,
             b2p_stream stream);

/* ------------------------------------------------------------ sharded
 * One logical array spread over the ranks of an NCCL communicator (one
 * process or thread per GPU, rank r holding the r-th contiguous shard).  The
 * reference runs every algorithm on one sycl::queue, i.e. one device
 * (algorithms/numeric.hpp, algorithm.hpp); these calls extend its reduce
 * (numeric.hpp:170-236) and scans (numeric.hpp:251-327) across devices with
 * a single exchange: each rank's shard partial (16 bytes) is all-gathered
 * on `stream` and combined in rank order on the host, so every rank gets the
 * same bits.  `nccl_comm` is an ncclComm_t of the libnccl.so.2 loaded in
 * the process (libb2p resolves NCCL's functions there and does not link
 * it).  The calls return after their work is complete (they synchronise
 * `stream`).  scratch: b2p_sharded_scratch_bytes(dtype, n, world) bytes,
 * zero-filled once (b2p_scratch_init), not shared with overlapping calls.
 * B2P_ERR_UNSUPPORTED when no libnccl.so.2 can be loaded.  Every rank must
 * make the call: a rank that rejects its arguments returns before the
 * exchange, and the others then wait in NCCL until its timeout. */
size_t b2p_sharded_scratch_bytes(int dtype, size_t n, int world);

/* *out (device, accumulation type) = init op (the reduction of every rank's
 * shard); init NULL: nothing folded in.  Integers wrap; float partials are
 * combined in double.  A rank may hold an empty shard (n == 0); when every
 * shard is empty and init is NULL, *out is left untouched. */
int b2p_sharded_reduce(int dtype, int op, const void *in, size_t n, void *out, const void *init,
                       void *scratch, size_t scratch_bytes, int config, void *nccl_comm, b2p_stream stream);

/* *out = init + the dot product of the concatenated shards of a and b (each
 * rank passes its shard of both; dtype F32, BF16 or F64; the compensated
 * local dot of b2p_dot, partials combined in double). */
int b2p_sharded_dot(int dtype, const void *a, const void *b, size_t n, void *out, const void *init,
                    void *scratch, size_t scratch_bytes, int config, void *nccl_comm, b2p_stream stream);

/* This rank's part of the inclusive (or exclusive) scan of the concatenated
 * shards: out[i] as the one-device scan of the whole array would give it.
 * The local scan runs once, with the combination of init and the totals of
 * the ranks before as its init.  Exclusive scans need init. */
int b2p_sharded_scan(int dtype, int op, int inclusive, const void *in, void *out, size_t n, const void *init,
                     void *scratch, size_t scratch_bytes, int config, void *nccl_comm, b2p_stream stream);

/* Host-side combination of exchanged partials, for hosts that move them
 * with their own transport: *result = init op values[0] op ... op
 * values[count - 1] (HOST memory; entries of the accumulation type, `stride`
 * bytes apart; init NULL: nothing folded in).  The rank-order combination
 * b2p_sharded_reduce and b2p_sharded_scan (carry = the first `rank` totals)
 * use.  B2P_ERR_INVALID_ARG when count == 0 and init is NULL. */
int b2p_shard_combine(int dtype, int op, const void *values, int count, size_t stride, const void *init,
                      void *result);

/* Log level of the library's stderr records (0 none, 1 errors, 2 warnings,
 * 3 one line per call, 4 each call also timed on its stream, which makes
 * the call wait for its work).  Initialised from B2P_LOG_LEVEL, else
 * ACPP_DEBUG_LEVEL / HIPSYCL_DEBUG_LEVEL as the reference reads them
 * (common/debug.hpp:14-21,61); default 2. */
int b2p_log_level(void);
void b2p_set_log_level(int level);

/* Wait for `stream`, then read the sticky device error word kept in
 * `scratch` (B2P_OK or B2P_ERR_TIMEOUT); clear != 0 resets it.  scratch ==
 * NULL reads the library's own word for the calls that take no scratch
 * (b2p_histogram_u8) on the current device.  Blocks the host.  Stands in
 * for the reference's asynchronous error list (runtime/error.hpp) that
 * event::wait() rethrows. */
int b2p_device_error(void *scratch, b2p_stream stream, int clear);

/* Process-wide bound for every device-side wait, in nanoseconds
 * (default 2e9).  Returns the previous value. */
uint64_t b2p_set_wait_timeout_ns(uint64_t ns);

/* The current bound (read by the header-compiled kernels of the C++ layer,
 * which honour the same limit). */
uint64_t b2p_wait_timeout_ns(void);

/* Test hook: the scan tile with this index (-1 = none) never publishes its
 * status in the next scan/copy_if launches, so its successors' bounded waits
 * run out.  Used only by the time-out test. */
void b2p_debug_stall_tile(int64_t tile);

/* ------------------------------------------------ batched plans / graphs */

typedef struct b2p_plan_s *b2p_plan;

/* Build a plan for one segmented reduce (prim = B2P_PRIM_SEG_REDUCE) or
 * inclusive scan (B2P_PRIM_SEG_SCAN) over fixed buffers, choose its launch
 * configuration (config or B2P_CONFIG_AUTO), allocate its scratch and
 * capture the launch into a CUDA graph on `stream`.  Blocks while it
 * captures.  The buffers must outlive the plan. */
int b2p_plan_segmented(b2p_plan *plan, int prim, int dtype, int op,
                       const void *in, void *out, const int64_t *offsets,
                       int64_t nseg, size_t total_elems, int config,
                       b2p_stream stream);

/* Launch the plan's graph on `stream` (one cudaGraphLaunch). */
int b2p_plan_launch(b2p_plan plan, b2p_stream stream);

/* Configuration the plan uses. */
int b2p_plan_config(b2p_plan plan);

void b2p_plan_destroy(b2p_plan plan);

/* ------------------------------------------------- autotuner / selector */

/* Exhaustive autotuner: time every valid config for one shape on synthetic
 * device data (median of `reps` launches after one warm-up, CUDA events)
 * and write milliseconds to times_ms[B2P_NUM_CONFIGS] (+inf for masked
 * configs).  nseg/cv describe segment lengths for segmented primitives
 * (nseg <= 1 otherwise).  Allocates and frees its own device buffers.
 * Blocks the host. */
int b2p_tune_shape(int prim, int dtype, int op, size_t n, int64_t nseg,
                   double cv, int reps, uint64_t seed, float *times_ms);

/* Learned schedule selector: 11 -> 64 -> 64 -> 48 MLP (ReLU), fp32.
 * Feature vector (B2P_SEL_FEATURES floats): log2 n, dtype one-hot
 * {I32,I64,F32,BF16}, op one-hot {reduce,scan,copy_if,histogram},
 * log2(segment count), segment-length coefficient of variation. */
#define B2P_SEL_FEATURES 11
#define B2P_SEL_HIDDEN 64

typedef struct b2p_selector_s *b2p_selector;

int b2p_selector_create(b2p_selector *sel, uint64_t seed);
void b2p_selector_destroy(b2p_selector sel);

/* Features for one call shape. */
int b2p_selector_features(int prim, int dtype, size_t n, int64_t nseg,
                          double cv, float *features);

/* Train on `m` samples: features[m*11], times_ms[m*48] (+inf = masked).
 * Loss: expected normalised time  sum_c softmax(z)_c * t_c / min_c t_c,
 * plus `ce_weight` * cross-entropy to the fastest config.  Adam, full
 * batch, on the GPU with the library's own forward/backward kernels.
 * Writes the final loss.  Blocks the host. */
int b2p_selector_train(b2p_selector sel, const float *features,
                       const float *times_ms, int m, int epochs, float lr,
                       float ce_weight, float *final_loss);

/* Batched inference on the GPU: best config per row of features[m*11]
 * (masked configs excluded using each row's primitive and dtype). */
int b2p_selector_predict(b2p_selector sel, const float *features, int m,
                         int *configs);

/* One forward+backward pass (no update) for gradient checks: writes loss
 * and the gradient w.r.t. every parameter (b2p_selector_num_params floats,
 * in the order W1,b1,W2,b2,W3,b3; W stored row-major [out][in]). */
int b2p_selector_grad(b2p_selector sel, const float *features,
                      const float *times_ms, int m, float ce_weight,
                      float *loss, float *grads);

int b2p_selector_num_params(void);
int b2p_selector_get_params(b2p_selector sel, float *params);
int b2p_selector_set_params(b2p_selector sel, const float *params);

/* Persist / restore weights (versioned; keyed by GPU name and library
 * version: a mismatch returns B2P_ERR_IO and leaves the selector as is). */
int b2p_selector_save(b2p_selector sel, const char *path);
int b2p_selector_load(b2p_selector sel, const char *path);

/* Install `sel` as the process-wide selector used by B2P_CONFIG_AUTO (NULL
 * to remove it).  Precomputes its decisions over a grid of call shapes with
 * one batched inference launch, so that a call's lookup costs a table read. */
int b2p_selector_install(b2p_selector sel);

/* Fixed heuristic used when no selector and no tuner entry exist. */
int b2p_heuristic_config(int prim, int dtype, size_t n, int64_t nseg);

/* Configuration B2P_CONFIG_AUTO resolves to for this shape right now. */
int b2p_auto_config(int prim, int dtype, size_t n, int64_t nseg, double cv);

/* --------------------------------------------------- synthetic workloads */

/* Fill HOST memory with the seeded synthetic inputs used by the benchmark
 * (counter-based SplitMix64; Box–Muller in double, rounded once).  kind:
 *  0: int32 uniform [lo, hi]         (a = lo, b = hi)
 *  1: fp32 N(0,1), a fraction `a` replaced by `b` * N(0,1)
 *  2: fp32 |N(0,1)|, same replacement
 *  3: uint32 uniform [0, 2^32)
 *  4: uint8 truncated Zipf(s = a) over 256 ranks, key = rank - 1
 *  5: int64 uniform [lo, hi]         (a = lo, b = hi)
 *  6: bf16 bits of kind 1 values (RNE)
 *  7: bf16 bits of kind 2 values (RNE)
 * Multi-threaded (OpenMP); results do not depend on the thread count. */
int b2p_synth_fill(int kind, uint64_t seed, size_t n, double a, double b,
                   void *host_out);

/* CSR offsets for `nseg` segments with lengths max(1, floor(2^(log2max*u)))
 * scaled so that the total does not exceed `cap` (0 = no cap); writes
 * offsets[nseg+1] to host memory and returns the total through *total. */
int b2p_synth_segments(uint64_t seed, int64_t nseg, double log2max,
                       uint64_t cap, int64_t *offsets, uint64_t *total);

#ifdef __cplusplus
}
#endif

#endif /* B2P_H */
