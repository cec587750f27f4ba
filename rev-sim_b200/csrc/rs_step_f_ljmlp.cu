// Instantiation of the fused step kernels for (float, F_LJ_MLP).
#include "rs_step_impl.cuh"

namespace rs {
template cudaError_t launch_form<float, F_LJ_MLP>(bool, int, int, bool, int, int, const StepArgs &,
                                              const NbConsts<float> &, const BondConsts &, cudaStream_t);
}  // namespace rs
