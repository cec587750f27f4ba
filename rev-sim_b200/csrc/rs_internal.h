// rs_internal.h -- host-side interface between the C-ABI layer (rs_api.cu) and the
// kernel launchers (rs_nlist.cu, rs_step.cu, rs_loss.cu).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <utility>
#include <cuda_runtime.h>

#include "rs_device.cuh"

namespace rs {

// Step kernels are launched chained (programmatic dependent launch; the kernel side is
// chain_enter) unless REVSIM_CHAIN=0 is set in the environment when the library first
// launches one.
inline bool chain_on() {
    static const bool on = [] {
        const char *e = std::getenv("REVSIM_CHAIN");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Launch of a kernel whose first statement is chain_enter(): with programmatic stream
// serialisation, so that it may be scheduled while the previous kernel in the stream runs.
template <typename... P, typename... A>
cudaError_t launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t st, A &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = chain_on() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Learned pair correction (rs_mlp.cu): 16 radial basis functions -> 64 -> 64 SiLU -> 1
// per element pair (O-O, O-H, H-H), tabulated on MLP_NG intervals of [0, cutoff].
constexpr int MLP_NRBF = 16, MLP_H = 64, MLP_NG = 1024, MLP_NT = 3;
constexpr int MLP_PER_TYPE = MLP_H * MLP_NRBF + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1;
constexpr int MLP_NPARAMS = MLP_NT * MLP_PER_TYPE;
constexpr double MLP_WIDTH = 0.05;
// Copies of the coefficient-adjoint accumulator per replica; CTA b adds into copy
// b % MLP_NCOPY, which spreads the atomics of the many pairs that share an interval.
constexpr int MLP_NCOPY = 16;

// Per-launch constants of the non-bonded terms, in pair precision R.
template <typename R>
struct NbConsts {
    R qq[3];      // k_e q_a q_b for (O,O), (O,H), (H,H)
    R krf;        // reaction-field k_rf
    R krf2;       // 2 k_rf
    R rc2;        // cutoff^2
    R twoinvq;    // 2 / q_O  (dF_c/dq_O = 2 F_c / q_O, water.jl:1247)
    FormConsts<R> fc;
    // F_LJ_MLP: interval table [MLP_NT][MLP_NG] of 4-vectors (cubic coefficients), the
    // accumulators of their adjoints [R][MLP_NCOPY][MLP_NT][MLP_NG][4] (reverse), and
    // MLP_NG / cutoff
    const void *mlp_tab;
    double *mlp_adj;
    R mlp_hinv;
};

// Constants of one pair form for the per-pair parameters t[0..nfp-1] (rs_api.cu).
template <typename R>
FormConsts<R> form_consts(int form, const double *t, int nfp);

struct BondConsts {
    double kb, r0, ka, th0;
};

// Register budget per thread of the step kernels (__maxnreg__), by precision, direction and
// loop form U.  FP32 (two entries per lane step in packed arithmetic): forward 128, reverse
// 168 (U = 1) and 200 (U = 2, 3); FP64 (one entry per step): 128, and 255 for U = 3.
#ifndef RS_NREG_F_FWD
#define RS_NREG_F_FWD 128
#endif
#ifndef RS_NREG_F_REV1
#define RS_NREG_F_REV1 168
#endif
#ifndef RS_NREG_F_REV2
#define RS_NREG_F_REV2 200
#endif
#ifndef RS_NREG_F_REV3
#define RS_NREG_F_REV3 200
#endif
constexpr int step_nreg(bool fp32, bool rev, int U) {
    return !fp32 ? (U == 3 ? 255 : 128)
                 : (!rev ? RS_NREG_F_FWD : (U == 3 ? RS_NREG_F_REV3 : (U == 1 ? RS_NREG_F_REV1 : RS_NREG_F_REV2)));
}
// The largest CTA a kernel of nreg registers per thread can be launched with: a CTA's warps
// are spread over the SM's four schedulers, each with a quarter (16,384) of the registers, a
// thread's registers allocated in units of 8.  128 registers: 512 threads; 168: 384; 200 or
// 255: 256.
constexpr int max_threads_for(int nreg) { return 32 * 4 * (16384 / (32 * ((nreg + 7) / 8 * 8))); }
constexpr int step_max_threads(bool fp32, bool rev, int U) { return max_threads_for(step_nreg(fp32, rev, U)); }
// Row entries of the FP32 step kernels' neighbour loop are loaded this many iterations ahead.
#ifndef RS_ROW_AHEAD
#define RS_ROW_AHEAD 1
#endif
// Half-shell pair kernels (k_water_half): forward 128, reverse 168 registers.
#ifndef RS_NREG_HALF_REV
#define RS_NREG_HALF_REV 168
#endif
constexpr int half_nreg(bool rev) { return rev ? RS_NREG_HALF_REV : RS_NREG_F_FWD; }
constexpr int half_max_threads(bool rev) { return max_threads_for(half_nreg(rev)); }

// Everything the step kernels read or write.
struct StepArgs {
    const int *blk_rep, *blk_mol0, *blk_nmol;
    const double *rep_box, *rep_sdO, *rep_sdH;
    const int *rep_atom0;
    const uint32_t *nbr;
    const int *nbr_cnt;
    int cap;
    double *x, *v, *A, *B, *C, *D, *G;
    const void *pos_in, *wgt_in;
    void *pos_out, *wgt_out;
    double *part;      // [M * P] dtheta partials per molecule (accumulated); [n_blk * P] per
                       // CTA in the half-shell kernels
    double *norm2;     // [M] (half-shell: [n_blk]) sum of dl_dfi^2 (deferred / clipped mode)
    int P;
    int *status;
    double *F_out;     // forces-only mode
    double dt, c, s, mO, mH, acoefO, acoefH;
    double dtm_O, dtm_H, invm_O, invm_H;   // dt / m and 1 / m of O and H (the exact integrator)
    const uint64_t *seed_cur, *seed_next;   // [n_replicas]
    // Caller-supplied noise of the current / next step, [3N] each (host_noise entry points);
    // when set it replaces the Philox draw of seed_cur / seed_next.
    const double *noise_cur, *noise_next;
    int mode;
    int exact;         // 1: the exactly reversible integrator (grid increments, rs_device.cuh)
    // Half-shell pair evaluation (FP32 kernels, rs_half.cu): each unordered molecule pair is
    // evaluated once, by its owner, which writes the partner's share into a slot; a second
    // kernel per step sums every molecule's own partial and its incoming slots in row order.
    const uint32_t *split;   // [M * cap]: owned entries from the front, incoming slots from the back
    const int *cnt_own, *cnt_inc;   // [M]
    float4 *slot_f;    // [M * cap * 3]: per owned entry and partner atom (F_x, F_y, F_z, G_x)
    float2 *slot_g;    // [M * cap * 3]: (G_y, G_z)
    float *own;        // [M * 36]: own forces, own VJP, bonded forces, bonded VJP (9 each)
};

// Owner of an unordered molecule pair {I, J}: I when I + J is odd and I < J, or I + J is even
// and I > J -- every molecule owns about half of its row whatever the index order.
__host__ __device__ __forceinline__ bool half_owns(int I, int J) {
    return ((I ^ J) & 1) ? I < J : I > J;
}

enum StepMode {
    MODE_FORCES_ONLY = 1,   // write F_out (and G / part in reverse), no integration
    MODE_FUSE_NEXT = 2,     // reverse: also run part 1 of the next reverse step
    MODE_DEFER_BA = 4,      // reverse: leave B, A for the clip pass, write norm2
};

struct NlistArgs {
    int M, n_cells;
    const double *x;
    const int *mol_rep, *rep_nc, *rep_cell_off, *cell_rep;
    const double *rep_box;
    int *cell_of_mol, *cell_cnt, *cell_start, *cell_fill, *cell_tmp, *cell_sorted;
    uint32_t *nbr;
    int *nbr_cnt;
    int cap;
    double rc_nl2;     // neighbour-list cutoff^2
    double rcand2;     // O-O candidate radius^2
    double rcand_near2;   // the same with the tighter O-H bound rnear (every O-H within it)
    double rext2;      // max intramolecular O-H distance^2
    double rnear2;     // O-H distance^2 bound under which one image shift per molecule pair holds
    double shift_box;  // boxes above this side may use one image shift per molecule pair
    float band;        // |FP32 d^2 - rc_nl^2| at or below which FP64 decides membership
    int *status;
    int *max_cnt;      // [0] running maximum of the row counts; [1] this build's count of
                       // molecules with an O-H distance above sqrt(rnear2)
    // Half-shell split of the rows (null: none): split, cnt_own, cnt_inc as in StepArgs;
    // ownpos [M * cap] scratch (compact owned index of each owned row entry).
    uint32_t *split;
    int *cnt_own, *cnt_inc, *ownpos;
};

struct RdfArgs {
    const double *x;
    const int *rep_atom0, *rep_nmol;
    const double *rep_box;
    int sel1, sel2;
    double x_min, step, width, cutoff;
    int n_grid, off;
    double *hist;      // [R * n_grid] raw sums, then h
    const double *dLdh; // [R * n_grid]
    double *dLdx;      // [3N]
};

// The RDF kernels form consecutive Gaussians by a recurrence whose ratio at a window's
// anchor is exp(-(2 e step + step^2) / width) with |e| <= exp_cutoff + 2 step; it must stay
// finite (exp overflows above ~709), so terms whose ratio exponent could exceed 700 are
// rejected when they are set.
inline bool rdf_term_recurrence_ok(double step, double width, double exp_cutoff) {
    const double worst = (2.0 * (exp_cutoff + 2.0 * step) * step + step * step) / width;
    return worst <= 700.0;
}

// Launchers (return cudaError_t of the launch).
cudaError_t launch_nlist(const NlistArgs &a, cudaStream_t st, int *n_kernels);
cudaError_t launch_export_pairs(const uint32_t *nbr, const int *nbr_cnt, int cap, int mol0,
                                int nmol, int32_t *pairs, unsigned long long *count,
                                long long max_pairs, cudaStream_t st);

// Half-shell step (two kernels, FP32, one image per molecule pair): rs_half.cu.
cudaError_t launch_half(bool rev, int form, int G, int n_blk, int threads, const StepArgs &a,
                        const NbConsts<float> &nb, const BondConsts &bc, cudaStream_t st);
template <typename R, int FORM>
cudaError_t launch_half_form(bool rev, int G, int n_blk, int threads, const StepArgs &a,
                             const NbConsts<R> &nb, const BondConsts &bc, cudaStream_t st);
// Fused step kernels: lanes per molecule G (8/16/32), entries per iteration unroll (1/2),
// shift = one periodic image per molecule pair (valid when every box side exceeds
// 2 (cutoff + 2 * max O-H distance)).
template <typename R>
cudaError_t launch_step(bool rev, int form, int G, int unroll, bool shift, int n_blk, int threads,
                        const StepArgs &a, const NbConsts<R> &nb, const BondConsts &bc,
                        cudaStream_t st);
template <typename R, int FORM>
cudaError_t launch_form(bool rev, int G, int unroll, bool shift, int n_blk, int threads,
                        const StepArgs &a, const NbConsts<R> &nb, const BondConsts &bc,
                        cudaStream_t st);

// Potential energy and its parameter gradient (rs_energy.cu), one thread per molecule.
struct EnergyArgs {
    int M, P, cap;
    const double *x;
    const int *mol_rep;
    const double *rep_box;
    const uint32_t *nbr;
    const int *nbr_cnt;
    double rc2, ke, krf, crf_shift;   // crf_shift = 1/rc + k_rf rc^2
    double qO, kb, r0, ka, th0;
    double form_p[4];                 // pair-form parameters, zero-padded
    const void *mlp_tab;              // F_LJ_MLP: interval table, adjoint accumulators, NG / rc
    double *mlp_adj;
    double mlp_hinv;
    double *part;                     // [M][P + 1]: energy, then dE/dtheta (classical)
    int grads;                        // 0: energy column only, no classical partials
    const double *adj_scale;          // per replica: MLP adjoints scaled by adj_mul adj_scale[r]
    double adj_mul;                   // (adj_scale null: unscaled)
};
cudaError_t launch_energy_grads(int form, int prec, const EnergyArgs &a, cudaStream_t st);

// The enthalpy-of-vaporisation loss term (loss_enth_vap, water.jl:738-755) from the energy
// partials: per replica U = sum of part[I][0] over its molecules (fixed-order tree),
// e = u_gas - U / n + rt - target, acc[r] += e^2, ev_acc[r] += e^2, k[r] = 2 e / n and, when
// grads, dgrad[r][p] += -k[r] * sum part[I][1 + p].
struct EnthArgs {
    int R, P, grads;
    const int *rep_atom0, *rep_nmol;
    const double *part;
    double u_gas, rt, target;
    double *acc, *ev_acc, *k, *dgrad;
};
cudaError_t launch_enth_finalize(const EnthArgs &a, cudaStream_t st);
// E[r] = the replica's sum of part[I][0] (fixed-order tree), r < R.
cudaError_t launch_rep_energy(int R, const int *rep_atom0, const int *rep_nmol, const double *part, int P,
                              double *E, cudaStream_t st);
// dLdx[i] += k[replica of atom i / 3] * F[i], i < 3N (dl_ev/dx = (2 e / n) F).
cudaError_t launch_enth_dldx(int N, const int *atom_rep, const double *k, const double *F, double *dLdx,
                             cudaStream_t st);

// Monte-Carlo volume move (rs_barostat.cu): molecule centres scaled by lsc[replica] about
// the origin, positions wrapped into the scaled box (in place); and the restore of the
// replicas whose move was rejected.
cudaError_t launch_baro_scale(int M, const int *mol_rep, const double *box_old, const double *lsc,
                              double *x, cudaStream_t st);
cudaError_t launch_baro_restore(int M, const int *mol_rep, const int *accepted, const double *xb,
                                double *x, cudaStream_t st);

size_t mlp_scratch_doubles();
// Node evaluation and interval table of the MLP for parameters theta (device, FP64).
// nt types (1..MLP_NT) of theta, RBF width w: the water model's three types at MLP_WIDTH by
// default; the Stillinger-Weber radial term uses one type.
cudaError_t launch_mlp_table(int prec, const double *theta, double rc, double *scratch, void *tab,
                             cudaStream_t st, int nt = MLP_NT, double w = MLP_WIDTH);
// Interval-coefficient adjoints (the sum of ncopy accumulators) -> dtheta [MLP_NPARAMS]
// (after launch_mlp_table with the same theta and scratch).
cudaError_t launch_mlp_backprop(const double *theta, double rc, const double *cadj, int ncopy,
                                double *scratch, double *dtheta, cudaStream_t st, int nt = MLP_NT,
                                double w = MLP_WIDTH);

// Node values -> interval table, the scratch's node arrays (0 u, 1 du, 2 au, 3 ad), and the
// coefficient adjoints -> node adjoints alone (rs_mlp.cu).
cudaError_t launch_mlp_table_from_nodes(int prec, double *scratch, double rc, void *tab, cudaStream_t st,
                                        int nt = MLP_NT);
double *mlp_scratch_nodes(double *scratch, int which);
cudaError_t launch_mlp_node_adjoints(const double *cadj, int ncopy, double rc, double *scratch, cudaStream_t st,
                                     int nt = MLP_NT);
// The network on the tensor cores (rs_mlp_tc.cu, BF16 operands, FP32 accumulation): u and
// du/dr at n distances per type (r null: the NG + 1 nodes of [0, rc]); the backward pass from
// node adjoints au, ad [nt][NG + 1] to dtheta [nt * MLP_PER_TYPE] (FP64), with its scratch.
size_t mlp_tc_scratch_bytes();
cudaError_t launch_mlp_tc_eval(const double *theta, int nt, double rc, double w, int n, const double *r,
                               double *u, double *du, cudaStream_t st);
cudaError_t launch_mlp_tc_backprop(const double *theta, int nt, double rc, double w, const double *au,
                                   const double *ad, void *scratch, double *dtheta, cudaStream_t st);

cudaError_t launch_pack(int N, int prec, const double *x, const double *C, double mO, double mH,
                        const int *atom_rep, const double *rep_box, void *pos, void *wgt,
                        cudaStream_t st);
cudaError_t launch_unintegrate(int M, int prec, const StepArgs &a, const int *mol_rep,
                               cudaStream_t st);
// Positions (wrapped into the replica's box) and velocities rounded to the exact
// integrator's grid, in place.
cudaError_t launch_quantize_state(int N, double *x, double *v, const int *atom_rep, const double *rep_box,
                                  cudaStream_t st);
cudaError_t launch_clip_post(int N, const StepArgs &a, const int *atom_rep, const double *scale,
                             cudaStream_t st);
cudaError_t launch_init_adjoint(int N, const double *g, double c, double *A, double *B, double *C,
                                double *D, double *G, cudaStream_t st);
cudaError_t launch_noise(int N, const int *atom_rep, const int *rep_atom0, const double *rep_sdO,
                         const double *rep_sdH, const uint64_t *seeds, double *xi,
                         cudaStream_t st);

cudaError_t launch_rdf(const RdfArgs &a, int R, int max_n1, int max_n2, bool grad,
                       cudaStream_t st);
cudaError_t launch_rdf_finalize(const RdfArgs &a, int R, const double *pre, const double *target,
                                int slice_start, int slice_stride, int n_target, int norm,
                                double weight, double *loss, double *dLdh, cudaStream_t st);

}  // namespace rs
