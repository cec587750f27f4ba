/*
 * mlp_oracle.h -- CPU FP64 restatement of the learned pair correction (no reference
 * counterpart: the reference's learned terms are MACE-OFF / DimeNet++ through PyTorch /
 * JAX hooks, water_maceoff.jl:147-163; this MLP replaces them).  TEST INFRASTRUCTURE ONLY.
 *
 * Per element pair tau in {O-O, O-H, H-H} of different molecules within the cutoff rc:
 *   u_tau(r) = MLP_tau(phi(r)) * fc(r),  fc(r) = (cos(pi r / rc) + 1) / 2,
 *   phi_k(r) = exp(-(r - mu_k)^2 / (2 w^2)),  mu_k = k rc / 15 (k = 0..15),  w = 0.05 nm,
 *   MLP: h1 = silu(W1 phi + b1) (64), h2 = silu(W2 h1 + b2) (64), y = w3 . h2 + b3.
 * The simulated pair energy is the cubic Hermite interpolant of u_tau on NG uniform
 * intervals of [0, rc] through the node values u and derivatives u' (the engine's
 * tabulation, defined identically here); forces, second derivatives and the parameter
 * chain rule are those of the interpolant.  Parameters per type (5,313):
 * W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3; types in the order O-O, O-H, H-H.
 */
#ifndef REVSIM_MLP_ORACLE_H
#define REVSIM_MLP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MLP_NRBF 16
#define ORC_MLP_H 64
#define ORC_MLP_NG 1024
#define ORC_MLP_NT 3
#define ORC_MLP_PER_TYPE (ORC_MLP_H * ORC_MLP_NRBF + ORC_MLP_H + ORC_MLP_H * ORC_MLP_H + ORC_MLP_H + ORC_MLP_H + 1)
#define ORC_MLP_NPARAMS (ORC_MLP_NT * ORC_MLP_PER_TYPE)
#define ORC_MLP_WIDTH 0.05

/* Node values and r-derivatives u[t][g], du[t][g] (g = 0..NG) of u_tau for cutoff rc. */
void orc_mlp_nodes(const double *theta, double rc, double *u, double *du);
/* Interval cubic coefficients coef[t][g][4] (p(s) = c0 + c1 s + c2 s^2 + c3 s^3, s in [0,1]). */
void orc_mlp_table(const double *theta, double rc, double *coef);
/* Interpolated pair energy, radial force F = -du/dr and dF/dr at distance r < rc. */
void orc_mlp_pair(const double *coef, int32_t type, double rc, double r, double *u, double *F,
                  double *dF);
/* Adjoint of the interval coefficients -> dtheta (accumulated): the chain rule through the
 * Hermite coefficients, the node values and derivatives, and the MLP. */
void orc_mlp_backprop(const double *theta, double rc, const double *coef_adj, double *dtheta);
/* The same three for the first nt types of theta and RBF width w (the functions above are
 * nt = ORC_MLP_NT, w = ORC_MLP_WIDTH); the Stillinger-Weber path uses one type. */
void orc_mlp_nodes_n(const double *theta, int32_t nt, double rc, double w, double *u, double *du);
void orc_mlp_table_n(const double *theta, int32_t nt, double rc, double w, double *coef);
void orc_mlp_backprop_n(const double *theta, int32_t nt, double rc, double w, const double *coef_adj,
                        double *dtheta);
/* Xavier-uniform W1, W2; w3 Xavier-uniform times 0.01; zero biases; seeded. */
void orc_mlp_init(uint64_t seed, double *theta);

#ifdef __cplusplus
}
#endif
#endif
