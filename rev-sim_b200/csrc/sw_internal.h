// sw_internal.h -- host/kernel interface of the Stillinger-Weber diamond engine
// (sw_kernels.cu, sw_api.cu).  Not part of the public ABI.
//
// Decomposition.  The SW energy is written as a sum over centres c of a centre energy
//   E_c = sum_q 1/2 E2(d_q) + sum_{q<q'} E3(d_q, d_q'),
// d_q = x_{j_q} - x_c over the active neighbours j_q (r/sigma < a) of c in ascending
// index order.  Every 2-body term is split in halves between its two atoms and every
// 3-body term of diamond.jl:463-527 belongs to exactly one centre, so sum_c E_c is the
// reference energy.  Per centre and active slot q the terms kernel stores
//   T_{c,q} = dE_c / dd_q   (and its directional derivative along a tangent),
// and the gather kernel forms the gradient of atom e as
//   dE/dx_e = sum_q ( T_{j_q, slot of e in j_q} - T_{e,q} ),
// summed in a fixed order over the slots (a butterfly over the lanes that hold them;
// slots ascend with the neighbour index): an order that depends only on the positions,
// not on when the candidate list was built, so forward and reverse forces are
// bit-identical without storing the lists.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rs_internal.h"   // rs_device.cuh, the MLP table and backprop launchers

namespace rs {
namespace sw {

constexpr int CAND = 64;        // candidate-row capacity (r < a sigma + skin)
constexpr int ST_SKIN = 16;     // an atom moved more than skin/2 since the list build
constexpr int TERM_THREADS = 128;
constexpr int NP = 7;           // theta = [A, B, a, lambda, gamma, sigma, eps]
// The learned radial term: one MLP type (rs_mlp.cu) tabulated on [0, MLP_RC] with RBF width
// MLP_W, added to the 2-body term of every active pair with r < MLP_RC.
constexpr double MLP_RC = 0.25, MLP_W = 0.0125;

// Parameters in term precision R, plus the FP64 values that decide activity.
template <typename R>
struct SwConsts {
    R A, B, a, lam, gam, sig, eps;
    R half_eA;   // eps * A / 2
    R el;        // eps * lambda
    R isig;      // 1 / sigma
    R asig;      // a sigma
    double a64, sig64, lim2;   // lim2 = (a sigma)^2
    double lo2, hi2;   // (a sigma)^2 (1 -+ 1e-9)^2: r^2 below lo2 is active, above hi2 not
    R mlp_hinv;        // learned term: NG / MLP_RC, NG / (2 MLP_RC), (NG / MLP_RC)^2
    R mlp_hhalf, mlp_hinv2;
    double mlp_rc2;    // MLP_RC^2 (the term is on for r^2 < mlp_rc2, decided in FP64)
};

struct SwNlArgs {
    int N, n_cells;
    const double *x;
    const int *atom_rep, *rep_nc, *rep_cell_off, *rep_atom0, *rep_n;
    const double *rep_box;
    int *cell_of, *cell_cnt, *cell_start, *cell_fill;
    float4 *cell_pos;    // [N] cell-ordered FP32 positions, atom index in .w
    int *cand, *cand_n;
    double *x_nl;
    float rl2f;          // (a sigma + skin + 1e-4)^2
    int *status, *max_cnt;
};

enum TermMode {
    TM_VALUE = 0,   // T only (forward step, forces, stress)
    TM_REV = 1,     // T, its derivative along w = C / m, and the dtheta contraction with acoef
    TM_LOSS = 2,    // T, its derivative along S d, and the contraction with S d / V
};

struct SwTermArgs {
    const int *blk_rep, *blk_atom0, *blk_n;   // CTA -> replica, first centre, centres
    const double *rep_box, *rep_vol;
    const double *x, *x_nl;
    const int *cand, *cand_n;
    const double *C;       // TM_REV: accumulator C (w = C / m)
    const double *A;       // TM_REV: accumulator A (acoef = A dt^2 / (2 m))
    const double *S;       // TM_LOSS: [R * 9] dL/dsigma per replica
    double inv_m, acoef_scale;
    int *act_idx, *act_n;
    void *Tv, *Tt;         // [N * G] 4-vectors in R (x, y, z, unused)
    double *part;          // [n_blk * NP] dtheta partials, accumulated (may be null)
    double *wpart;         // [n_blk * 9] virial partials, written (may be null)
    const void *mlp_tab;   // learned term: [MLP_NG] cubic coefficients in R (null: off)
    double *mlp_adj;       // [R][MLP_NCOPY][MLP_NG][4] coefficient adjoints (with part)
    double half_skin2;
    int *status, *max_act;
};

enum GatherMode {
    GM_FORCES = 0,   // write F (and dl_dfi when tangents are present)
    GM_FWD = 1,      // forward B-A-O-A step
    GM_REV = 2,      // reverse: un-kick, B/A update, optionally the next step's part 1
    GM_LOSS = 3,     // dL/dx, dL/dv, and optionally the adjoint initialisation
};

struct SwGatherArgs {
    int N;
    const int *atom_rep, *rep_atom0;
    const double *rep_box, *rep_vol, *rep_sd;
    const int *act_idx, *act_n;
    const void *Tv, *Tt;
    double *x, *v, *F, *G, *A, *B, *C, *D;
    double *dLdx, *dLdv;
    const double *S, *vbar;
    double dt, c, s, m, dt2;
    const uint64_t *seed_cur, *seed_next;   // [R] per replica, null = no noise (s == 0)
    int fuse_next, init_adjoint, vel_term;
    int *status;
};

struct SwRedArgs {
    int R;
    const int *ablk_rep, *ablk_atom0, *ablk_n;   // atom blocks of 256 within one replica
    int n_ablk;
    const int *blk_rep;                          // term CTAs
    int n_blk;
    const int *rep_blk0, *rep_ablk0, *rep_n;     // [R + 1] first term / atom block per replica, [R] atoms
    const double *v;
    double *vpart, *kpart;                       // [n_ablk * 3], [n_ablk * 9]
    double *vbar;                                // [R * 3]
    const double *wpart;                         // [n_blk * 9]
    const double *rep_vol, *target;              // [R], [R * 9]
    double m, weight;
    int vel_term;
    double *sigma, *S, *loss, *loss_acc;         // [R*9], [R*9], [R], [R] (loss_acc may be null)
};

cudaError_t launch_sw_nlist(const SwNlArgs &a, cudaStream_t st);
template <typename R>
cudaError_t launch_sw_terms(int mode, int G, int n_blk, const SwTermArgs &a, const SwConsts<R> &p,
                            cudaStream_t st);
template <typename R>
cudaError_t launch_sw_gather(int mode, int G, bool tangent, const SwGatherArgs &a, cudaStream_t st);
cudaError_t launch_sw_stress(const SwRedArgs &a, cudaStream_t st);
cudaError_t launch_sw_part1(int N, const SwGatherArgs &a, cudaStream_t st);
cudaError_t launch_sw_noise(int N, const int *atom_rep, const int *rep_atom0, const double *rep_sd,
                            const uint64_t *seeds, double *xi, cudaStream_t st);
cudaError_t launch_sw_active_pairs(int N, int G, const int *act_idx, const int *act_n,
                                   int32_t *pairs, unsigned long long *count, long long max_pairs,
                                   cudaStream_t st);

}  // namespace sw
}  // namespace rs
