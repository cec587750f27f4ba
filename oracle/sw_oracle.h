/*
 * sw_oracle.h -- CPU FP64 restatement of the Stillinger-Weber diamond path of
 * greener-group/rev-sim `diamond/diamond.jl`: the SW 2- and 3-body energy and forces
 * (diamond.jl:309-381, 444-532), their parameter and position derivatives (the Enzyme
 * pullbacks of diamond.jl:1658-1697), the virial stress tensor and its loss
 * (diamond.jl:753-786) and the reverse pass with dL/dv (diamond.jl:1757-1878).
 *
 * TEST INFRASTRUCTURE ONLY (the checker), like revsim_oracle.h.  Parity of absolute
 * values is unpinned (the reference needs Julia + Enzyme + JAX); pinned by F = -dU/dx,
 * central differences and the reconstruction / loss identities (diamond.jl:1940-1942).
 *
 * Derivatives are taken by the complex step: every term is written on complex
 * arguments and f'(x) v = Im f(x + i h v) / h, exact to rounding for these analytic
 * expressions.  Parameters theta = [A, B, a, lambda, gamma, sigma, eps] (diamond.jl:53),
 * exponents p = 4, q = 0 (diamond.jl:1354).  Single-species cubic box.
 */
#ifndef REVSIM_SW_ORACLE_H
#define REVSIM_SW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_SW_NP 7

/* The learned radial term (the MLP of mlp_oracle.h with one type): u(r) on [0, 0.25 nm]
 * (a sigma = 0.252 nm at the initial parameters), RBF width 0.0125 nm (the water basis
 * scaled by 0.25 nm / 1 nm), added to the 2-body term of every pair with r / sigma < a and
 * r < ORC_SW_MLP_RC.  Its ORC_MLP_PER_TYPE parameters follow the 7 SW ones. */
#define ORC_SW_MLP_RC 0.25
#define ORC_SW_MLP_WIDTH 0.0125

typedef struct {
    int32_t n_atoms;
    double box;     /* cubic side, nm */
    double mass;    /* u (12.011) */
    double kB;      /* u nm^2 ps^-2 K^-1 */
    double temp;    /* K */
    int32_t mlp;    /* 1: add the learned radial term */
} orc_sw_system;

/* Stress loss: weight * sum_ab (sigma_ab - target_ab)^2 / 9 (target 0 in the reference). */
typedef struct {
    double weight;        /* gamma_sigma, 5e-8 in diamond.jl:57 */
    double target[9];
    int32_t vel_term;     /* 1: include the kinetic tensor (diamond.jl:773) */
} orc_sw_loss;

/* 7, plus ORC_MLP_PER_TYPE with the learned term. */
int32_t orc_sw_n_params(const orc_sw_system *s);
double orc_sw_energy(const orc_sw_system *s, const double *theta, const double *x);
/* Pairs i < j with r / sigma < a (the 2-body terms), ascending; returns the count. */
int64_t orc_sw_pairs(const orc_sw_system *s, const double *theta, const double *x,
                     int32_t *pairs, int64_t max_pairs);
void orc_sw_forces(const orc_sw_system *s, const double *theta, const double *x, double *F);
/* F, dl_dfi[b] = sum_a (w_a/m) . dF_a/dx_b, dF_dp [3N * 7] (the SW parameters; may be NULL). */
void orc_sw_forces_grads(const orc_sw_system *s, const double *theta, const double *x,
                         const double *w, double *F, double *dl_dfi, double *dF_dp);
/* sum_a acoef_a . dF_a/dtheta for every parameter (SW, then the learned term's): dtheta[P]. */
void orc_sw_contract(const orc_sw_system *s, const double *theta, const double *x,
                     const double *acoef, double *dtheta);
/* Stress tensor sigma [9] (row-major) = (K + W) / V. */
void orc_sw_stress(const orc_sw_system *s, const double *theta, const double *x, const double *v,
                   int32_t vel_term, double *sigma);
/* Loss and its gradients w.r.t. x [3N], v [3N] and theta [P] (any may be NULL). */
double orc_sw_loss_grad(const orc_sw_system *s, const double *theta, const orc_sw_loss *L,
                        const double *x, const double *v, double *dLdx, double *dLdv,
                        double *dLdp);
void orc_sw_noise(const orc_sw_system *s, uint64_t seed, double *xi);
/* Forward pass (B-A-O-A, diamond.jl:1439-1474).  A loss point is a step with
 * (n_steps - step) % n_steps_loss == 0 and step >= n_steps_buffer; at each one the state is
 * copied to snap_x/snap_v[k] (k = 0, 1, ... in time order) when snap_x != NULL and the
 * stress loss is accumulated when calc_loss.  Returns the mean loss over loss points. */
double orc_sw_forward_sim(const orc_sw_system *s, const double *theta, double *x, double *v,
                          const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, int32_t n_steps_buffer, double dt,
                          const orc_sw_loss *L, int32_t calc_loss, double *snap_x, double *snap_v);
/* Reverse pass over n_blocks loss blocks with the dL/dv accumulators of diamond.jl:1789-1793
 * and the block schedule of diamond.jl:1799-1868 (snapshots as written by the forward pass);
 * dl_dp [P]. */
double orc_sw_reverse_sim(const orc_sw_system *s, const double *theta, double *x, double *v,
                          const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, int32_t n_steps_trunc, int32_t n_blocks, double dt,
                          const double *snap_x, const double *snap_v, const orc_sw_loss *L,
                          double *dl_dp);

#ifdef __cplusplus
}
#endif
#endif
