// Instantiation of the half-shell step kernels for (F_BUFF).
#include "rs_half_impl.cuh"

namespace rs {
template cudaError_t launch_half_form<float, F_BUFF>(bool, int, int, int, const StepArgs &, const NbConsts<float> &,
                                               const BondConsts &, cudaStream_t);
}  // namespace rs
