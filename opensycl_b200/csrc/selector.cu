// Learned schedule selector and batched plans (implementation follows).
#include "common.cuh"
#include "internal.h"
#include "tuning.h"

extern "C" {
int b2p_selector_create(b2p_selector *sel, uint64_t) { if (sel) *sel = nullptr; return B2P_ERR_UNSUPPORTED; }
void b2p_selector_destroy(b2p_selector) {}
int b2p_selector_features(int, int, size_t, int64_t, double, float *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_train(b2p_selector, const float *, const float *, int, int, float, float, float *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_predict(b2p_selector, const float *, int, int *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_grad(b2p_selector, const float *, const float *, int, float, float *, float *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_num_params(void) { return 0; }
int b2p_selector_get_params(b2p_selector, float *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_set_params(b2p_selector, const float *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_save(b2p_selector, const char *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_load(b2p_selector, const char *) { return B2P_ERR_UNSUPPORTED; }
int b2p_selector_install(b2p_selector) { return B2P_ERR_UNSUPPORTED; }
int b2p_plan_segmented(b2p_plan *plan, int, int, int, const void *, void *, const int64_t *, int64_t, size_t, int, b2p_stream) { if (plan) *plan = nullptr; return B2P_ERR_UNSUPPORTED; }
int b2p_plan_launch(b2p_plan, b2p_stream) { return B2P_ERR_UNSUPPORTED; }
int b2p_plan_config(b2p_plan) { return -1; }
void b2p_plan_destroy(b2p_plan) {}
}
