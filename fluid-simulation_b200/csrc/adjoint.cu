// adjoint.cu — differentiable rollout (work in progress in this build step).
#include "simulator.cuh"
namespace wcsph {
float CUDASPHSimulator::rollout_forward(int, float, int, const float*) {
    throw Error(WCSPH_ERR_NOT_SUPPORTED, "rollout not built");
}
void CUDASPHSimulator::rollout_backward(float*, float*, float*) {
    throw Error(WCSPH_ERR_NOT_SUPPORTED, "rollout not built");
}
}  // namespace wcsph
