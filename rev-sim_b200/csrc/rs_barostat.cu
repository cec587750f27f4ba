// rs_barostat.cu -- the molecule-centre scaling of a Monte-Carlo volume move
// (MonteCarloBarostatNoUnits / apply_coupling!, water.jl:789-865, through Molly's
// scale_coords!): one thread per molecule.  The energy of the current and the trial state
// comes from k_energy_grads (rs_energy.cu); the draws, the Metropolis decision and the step
// adaptation are per replica on the host (rs_api.cu, baro_attempt).
#include "rs_internal.h"

namespace rs {

namespace {

// Centre c = x_O + (d_H1 + d_H2) / 3 (minimum-image O->H vectors in the old box L), shift
// c (l - 1); every atom moves by the shift and is wrapped into the new box l L.  x is
// overwritten with the trial positions (the caller keeps a copy).
__global__ void k_baro_scale(int M, const int *mol_rep, const double *box_old, const double *lsc,
                             double *x) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= M) return;
    const int r = mol_rep[I];
    const double L = box_old[r], l = lsc[r], Ln = __dmul_rn(L, l);
    double *xm = x + 9 * (size_t)I;
    double sh[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const double d1 = vec1d(xm[u], xm[3 + u], L), d2 = vec1d(xm[u], xm[6 + u], L);
        const double c = __dadd_rn(xm[u], __ddiv_rn(__dadd_rn(d1, d2), 3.0));
        sh[u] = __dsub_rn(__dmul_rn(c, l), c);
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) xm[3 * k + u] = wrap1d(__dadd_rn(xm[3 * k + u], sh[u]), Ln);
}

// Molecules of replicas whose move was rejected get their saved positions back.
__global__ void k_baro_restore(int M, const int *mol_rep, const int *accepted, const double *xb,
                               double *x) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= M || accepted[mol_rep[I]]) return;
#pragma unroll
    for (int q = 0; q < 9; q++) x[9 * (size_t)I + q] = xb[9 * (size_t)I + q];
}

}  // namespace

cudaError_t launch_baro_scale(int M, const int *mol_rep, const double *box_old, const double *lsc,
                              double *x, cudaStream_t st) {
    if (M > 0) k_baro_scale<<<(M + 127) / 128, 128, 0, st>>>(M, mol_rep, box_old, lsc, x);
    return cudaGetLastError();
}

cudaError_t launch_baro_restore(int M, const int *mol_rep, const int *accepted, const double *xb,
                                double *x, cudaStream_t st) {
    if (M > 0) k_baro_restore<<<(M + 127) / 128, 128, 0, st>>>(M, mol_rep, accepted, xb, x);
    return cudaGetLastError();
}

}  // namespace rs
