/*
 * revsim_sw.h -- C ABI of the Stillinger-Weber diamond engine of librevsim.so (sm_100a).
 *
 * Replaces the reversible-simulation gradient of greener-group/rev-sim
 * diamond/diamond.jl for inter_type :sw and loss_type :stress:
 *   forward_sim(coords, velocities, noise_seeds, gamma, n_steps, n_steps_loss,
 *               n_steps_buffer, params_sw, params_gnn, dt, ...)      diamond.jl:1394-1538
 *   reverse_sim(coords, velocities, noise_seeds, gamma, n_steps, n_steps_loss,
 *               n_steps_trunc, n_steps_buffer, params_sw, params_gnn, dt, ...,
 *               fwd_loggers, loss_accum_fwd, ...)                    diamond.jl:1757-1878
 * and the pieces under them: forces_sw! (diamond.jl:444-532), sw_force_and_grads!
 * (diamond.jl:1658-1697), virial_stress_tensor / loss_stress_sw and their pullback
 * (diamond.jl:753-786 via loss_and_grads, diamond.jl:1342-1350).
 *
 * Parameters theta = [A, B, a, lambda, gamma, sigma, eps] (diamond.jl:53), exponents
 * p = 4, q = 0 (diamond.jl:1352-1356).  Units nm, ps, u, kJ/mol, K.  Several independent
 * replicas (cubic boxes of their own size and temperature) run in every launch; arrays of
 * atoms are the replicas' atoms back to back, FP64 AoS xyz.  Status codes and the
 * precision modes are those of revsim.h.  No call keeps a host pointer.
 */
#ifndef REVSIM_SW_H
#define REVSIM_SW_H

#include <stdint.h>

#include "revsim.h"

#ifdef __cplusplus
extern "C" {
#endif

#define REVSIM_SW_NPARAMS 7
/* The learned radial term (desc.mlp = 1): one MLP pair function of r on [0, 0.25 nm]
 * (16 Gaussian radial basis functions of width 0.0125 nm -> 64 -> 64 SiLU -> 1, times a
 * cosine cutoff; the layout of revsim.h's per-type MLP), tabulated as cubic Hermite segments
 * on 1,024 intervals and added to the 2-body term of every active pair with r < 0.25 nm.
 * Its REVSIM_SW_MLP_NPARAMS parameters follow the 7 SW ones in every theta / gradient
 * array (n_params = 7 + REVSIM_SW_MLP_NPARAMS).  It stands in for the reference's learned
 * GNN term (params_gnn of diamond.jl:1394, 1757). */
#define REVSIM_SW_MLP_NPARAMS 5313
#define REVSIM_SW_MLP_CUTOFF 0.25

typedef struct revsim_sw_handle revsim_sw_handle;

typedef struct {
    int32_t n_replicas;
    const int32_t *n_atoms;   /* [n_replicas] */
    const double *box;        /* [n_replicas] cubic side, nm (1.784 in diamond.jl:42) */
    const double *temp;       /* [n_replicas] K (298 in diamond.jl:52) */
    int32_t precision;        /* REVSIM_FP64 or REVSIM_MIXED (FP32 terms, FP64 state) */
    double mass;              /* u (12.011, diamond.jl:41) */
    double kB;                /* u nm^2 ps^-2 K^-1 */
    double skin;              /* candidate-list skin beyond a sigma, nm */
    int32_t n_steps_nf;       /* candidate-list rebuild interval, steps; halved (and the call
                                 rerun) whenever an atom moves more than skin / 2 between builds */
    int32_t device;
    int32_t mlp;              /* 1: add the learned radial term */
} revsim_sw_desc;

/* Stress loss weight * sum_ab (sigma_ab - target_ab)^2 / 9 per replica (diamond.jl:772-775). */
typedef struct {
    double weight;            /* gamma_sigma (5e-8, diamond.jl:57) */
    int32_t vel_term;         /* 1: sigma includes the kinetic tensor (diamond.jl:766-770) */
    const double *target;     /* [n_replicas * 9] row-major, NULL = zero (the reference) */
} revsim_sw_loss;

int32_t revsim_sw_create(const revsim_sw_desc *desc, revsim_sw_handle **out);
void revsim_sw_destroy(revsim_sw_handle *h);
const char *revsim_sw_last_error(const revsim_sw_handle *h);

/* theta [n_params]: StillingerWeber(A, B, 4, 0, a, lambda, gamma, sigma, eps),
 * diamond.jl:1352-1356, then the learned term's parameters when desc.mlp. */
int32_t revsim_sw_set_params(revsim_sw_handle *h, const double *theta, int32_t n);
/* x, v [3 N] (x is wrapped into each replica's box by the caller, as Molly keeps it). */
int32_t revsim_sw_set_state(revsim_sw_handle *h, const double *x, const double *v);
int32_t revsim_sw_get_state(revsim_sw_handle *h, double *x, double *v);
int32_t revsim_sw_set_loss(revsim_sw_handle *h, const revsim_sw_loss *loss);

/* forces_sw (diamond.jl:534-541): F [3 N]. */
int32_t revsim_sw_forces(revsim_sw_handle *h, double *F);
/* sw_force_and_grads! (diamond.jl:1658-1697): F, dl_dfi[b] = sum_a (w_a / m) . dF_a/dx_b
 * and dtheta [n_replicas * n_params] = sum_a acoef_a . dF_a/dtheta per replica (acoef may be NULL,
 * then dtheta is not written). */
int32_t revsim_sw_force_vjp(revsim_sw_handle *h, const double *w, const double *acoef, double *F,
                            double *dl_dfi, double *dtheta);
/* virial_stress_tensor (diamond.jl:753-770): sigma [n_replicas * 9]. */
int32_t revsim_sw_stress(revsim_sw_handle *h, int32_t vel_term, double *sigma);
/* loss_and_grads for :stress (diamond.jl:1342-1350): loss [n_replicas], dL/dx, dL/dv [3 N],
 * dL/dtheta [n_replicas * n_params]; any output may be NULL. */
int32_t revsim_sw_loss_grad(revsim_sw_handle *h, double *loss, double *dLdx, double *dLdv,
                            double *dLdtheta);
/* generate_noise! (diamond.jl:1387-1392) for one seed per replica: xi [3 N]. */
int32_t revsim_sw_noise(revsim_sw_handle *h, const uint64_t *seeds, double *xi);
/* Active SW pairs (r / sigma < a) as global atom indices i < j; returns the count in *n
 * (pairs holds min(*n, max_pairs) of them, unordered). */
int32_t revsim_sw_active_pairs(revsim_sw_handle *h, int32_t *pairs, int64_t max_pairs, int64_t *n);

/* forward_sim (diamond.jl:1394-1538) for :sw, :stress.  noise_seeds [n_steps * n_replicas],
 * step-major.  A loss point is a step with (n_steps - step) % n_steps_loss == 0 and
 * step >= n_steps_buffer; the state there is kept on the device for the reverse pass.
 * loss [n_replicas] = mean stress loss over the loss points when calc_loss (may be NULL);
 * *n_blocks (may be NULL) = number of loss points. */
int32_t revsim_sw_forward(revsim_sw_handle *h, const uint64_t *noise_seeds, double gamma,
                          int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_buffer, double dt,
                          int32_t calc_loss, double *loss, int32_t *n_blocks);
/* reverse_sim (diamond.jl:1757-1878) from the handle's state (the forward end state):
 * loss [n_replicas], dl_dtheta [n_replicas * n_params], each the mean over the loss blocks of
 * the forward pass run last on this handle with the same n_steps and n_steps_loss. */
int32_t revsim_sw_reverse(revsim_sw_handle *h, const uint64_t *noise_seeds, double gamma,
                          int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                          double *loss, double *dl_dtheta);

int32_t revsim_sw_stream(revsim_sw_handle *h, void **stream);
int32_t revsim_sw_launch_count(revsim_sw_handle *h, int64_t *n);
/* CUDA-event timing of the term and gather kernels of the step loops (0: off). */
int32_t revsim_sw_set_kernel_timing(revsim_sw_handle *h, int32_t on);
/* which: 0 reverse terms, 1 forward terms, 2 reverse gather, 3 forward gather:
 * total ms and launches since timing was switched on. */
int32_t revsim_sw_kernel_time(revsim_sw_handle *h, int32_t which, double *ms, int64_t *launches);
/* Lanes per centre of the terms kernel (16 or 32; 16 serves up to 16 active neighbours). */
int32_t revsim_sw_set_lanes(revsim_sw_handle *h, int32_t lanes);

#ifdef __cplusplus
}
#endif
#endif
