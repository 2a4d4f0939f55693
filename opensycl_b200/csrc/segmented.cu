// Segmented reduce / scan in one persistent launch (implementation follows).
#include "common.cuh"
#include "internal.h"

namespace b2p {
size_t segmented_scratch_bytes(int dtype, size_t n, int64_t nseg, int config) {
  (void)dtype; (void)n; (void)nseg; (void)config;
  return kScratchPrefix;
}
bool segmented_config_valid(int dtype, int config) { (void)dtype; (void)config; return false; }
int launch_segmented(int, int, int, int, const void *, void *, const int64_t *, int64_t, size_t,
                     const void *, void *, size_t, int, cudaStream_t) {
  return B2P_ERR_UNSUPPORTED;
}
}  // namespace b2p
