// gas_internal.h -- host-side interface between the gas-in-water C ABI (gas_api.cu) and its
// kernels (gas_kernels.cu).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rs_internal.h"

namespace gs {

using rs::BondConsts;
using rs::FormConsts;

// One warp per atom; four atoms per CTA.
constexpr int kWarpsPerCta = 4;
constexpr int kThreads = 32 * kWarpsPerCta;
constexpr int kMaxP = 7;

// Site kinds: 0 water O, 1 water H, 2 gas O.  Atoms 0 .. nw3-1 are waters (O, H1, H2),
// the rest O2 pairs.
__host__ __device__ __forceinline__ int site_kind(int a, int nw3) {
    return a < nw3 ? (a % 3 == 0 ? 0 : 1) : 2;
}

// Non-bonded constants of one parameter vector in pair precision R.  Classes of the pair
// form: 0 water O - water O, 1 water O - gas, 2 gas - gas (mixed parameters in fc[class]).
// The class sums of dF/d(mixed parameter k) reach theta through the mixing factors:
// theta[iw[k]] gets fw[class][k] of it and theta[ig[k]] (ig >= 0) fg[class][k] (FP64).
template <typename R>
struct GasConstsT {
    R qq[3];            // k_e q_a q_b for (O,O), (O,H), (H,H)
    R krf, krf2, rc2, twoinvq;
    double crf_shift;
    FormConsts<R> fc[3];
    int on[3];
    double fw[3][4], fg[3][4];
    int iw[4], ig[4];
    int P, iq;
};
using GasConsts = GasConstsT<double>;

// Gather buffers: V4T<R>::T per atom (float4 in mixed precision, double4 in FP64) of the
// positions (pos) and of C/m (wgt); the FP64 state x, v, A-D stays authoritative.
struct GasArgs {
    int N, nw3;
    double L, invL;
    const int *rows;
    const int *cnt;
    int cap;
    const void *pos_in;
    void *pos_out;
    const void *wgt_in;
    void *wgt_out;
    const double4 *pos64_in;   // FP64 positions for the molecule's bonded terms (the same
    double4 *pos64_out;        // buffers as pos_in / pos_out in FP64)
    double *x, *v, *A, *B, *C, *D, *G, *F_out;
    const double *acoef_in;   // forces-only reverse mode: the contraction weights [3N]
    double *part;       // [N][P] dtheta partials (accumulated)
    int *status;
    double dt, c, s, mO, mH, sdO, sdH;
    uint64_t seed_cur, seed_next;
    int mode;           // rs::MODE_FORCES_ONLY, rs::MODE_FUSE_NEXT
    BondConsts bw;      // water bonds and angle
    double kb_g, r0_g;  // O2 bond
};

struct GasRowArgs {
    int N, nw3;
    double L, rc_nl2;
    const double *x;    // FP64 state [3N]
    int *rows, *cnt;
    int cap;
    int *status;
};

// mixed: pair arithmetic in FP32 (R = float), else FP64
void launch_gas_rows(const GasRowArgs &a, cudaStream_t st);
void launch_gas_step(bool mixed, int form, bool rev, const GasConstsT<float> &kf,
                     const GasConstsT<double> &kd, const GasArgs &a, cudaStream_t st);
// part 1 of a reverse step (diffusion.jl:1566-1572) for every atom, writing pos_out / wgt_out
void launch_gas_part1(bool mixed, const GasArgs &a, cudaStream_t st);
// pos[a] = pos64[a] = x[a]
void launch_gas_pack(bool mixed, int N, const double *x, void *pos, double4 *pos64, cudaStream_t st);
// wgt[a] = w[a] / m_a
void launch_gas_pack_w(bool mixed, int N, int nw3, const double *w, double mO, double mH, void *wgt,
                       cudaStream_t st);
// accumulators at a loss point from dl/dx g (diffusion.jl:1547-1550): A = B = g f1,
// C = 0, D = g f2 / f3, G = 0
void launch_gas_reset(int n3, const double *g, double f1, double f2, double f3, double *A,
                      double *B, double *C, double *D, double *G, cudaStream_t st);
// y += k x
void launch_gas_axpy(int n, double k, const double *x, double *y, cudaStream_t st);
// per-atom [E, dE/dtheta (P)] of the pairs j > i within the cutoff and the bonded terms
// (each bonded term on its first atom)
void launch_gas_energy(int form, const GasConsts &k, const GasArgs &a, double *epart,
                       cudaStream_t st);
// out[q] (+)= scale_q * sum_atoms epart[a][q] for q = 0..P in atom order; scale_0 = e_scale,
// scale_q>0 = g_scale; accumulate adds into out
void launch_gas_esum(int N, int P, const double *epart, double e_scale, double g_scale,
                     bool accumulate, double *out, cudaStream_t st);

}  // namespace gs
