// batch.cu — batched ensemble (work in progress in this build step).
#include "batch.cuh"

extern "C" {
int wcsph_batch_create(const wcsph_params*, const wcsph_batch_scene*, uint32_t, int, wcsph_batch** out) {
    if (out) *out = nullptr;
    return WCSPH_ERR_NOT_SUPPORTED;
}
int wcsph_batch_destroy(wcsph_batch*) { return WCSPH_OK; }
int wcsph_batch_step_n(wcsph_batch*, int, float) { return WCSPH_ERR_NOT_SUPPORTED; }
int wcsph_batch_time_steps(wcsph_batch*, int, float, float*) { return WCSPH_ERR_NOT_SUPPORTED; }
int wcsph_batch_get_state(wcsph_batch*, uint32_t, float*, float*) { return WCSPH_ERR_NOT_SUPPORTED; }
int wcsph_batch_metrics(wcsph_batch*, float*, float*) { return WCSPH_ERR_NOT_SUPPORTED; }
const char* wcsph_batch_last_error(const wcsph_batch*) { return "batch not built"; }
}
