// Instantiation of the fused step kernels for (double, F_BUFF).
#include "rs_step_impl.cuh"

namespace rs {
template cudaError_t launch_form<double, F_BUFF>(bool, int, int, bool, int, int, const StepArgs &,
                                           const NbConsts<double> &, const BondConsts &, cudaStream_t);
}  // namespace rs
