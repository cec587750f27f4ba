// Instantiation of the fused step kernels for (float, F_BUFF).
#include "rs_step_impl.cuh"

namespace rs {
template cudaError_t launch_form<float, F_BUFF>(bool, int, int, bool, int, int, const StepArgs &,
                                           const NbConsts<float> &, const BondConsts &, cudaStream_t);
}  // namespace rs
