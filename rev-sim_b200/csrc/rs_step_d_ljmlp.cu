// Instantiation of the fused step kernels for (double, F_LJ_MLP).
#include "rs_step_impl.cuh"

namespace rs {
template cudaError_t launch_form<double, F_LJ_MLP>(bool, int, int, bool, int, int, const StepArgs &,
                                              const NbConsts<double> &, const BondConsts &, cudaStream_t);
}  // namespace rs
