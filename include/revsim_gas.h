/*
 * revsim_gas.h -- C ABI of the B200 (sm_100a) gas-in-water reversible-simulation engine.
 *
 * The engine replaces the hot path of greener-group/rev-sim `diffusion/diffusion.jl`:
 * forward_sim (diffusion.jl:1181-1298, without the RAD gradient), reverse_sim
 * (diffusion.jl:1511-1616) and the force / force-gradient kernels they call (calc_F!
 * diffusion.jl:959-1057, calc_F_and_grads! diffusion.jl:1300-1509, the neighbour finder of
 * setup_system diffusion.jl:1133-1155), with the diffusion-coefficient loss
 * (calculate_D diffusion.jl:861-895, loss_fn_final 897-911), the enthalpy-of-
 * vaporisation loss (diffusion.jl:799-815) and the RDF loss of the water atoms
 * (diffusion.jl:759-774) at the loss points.
 *
 * The system: n_water flexible 3-site waters (atoms O, H1, H2) followed by n_gas two-site
 * O2 molecules (atoms O1, O2).  Pair forms between unlike sites by Lorentz-Berthelot mixing
 * (sigma arithmetic, eps geometric; Buckingham A, B, C arithmetic), reaction-field Coulomb
 * between water sites, fixed harmonic water bonds and angles and a fixed O2 bond.
 * Parameter vector (diffusion.jl:1629-1639):
 *   REVSIM_LJ:                  [sigma_w, eps_w, sigma_g, eps_g, q_O]
 *   REVSIM_DEXP / LJSC / BUFF:  [sigma_w, eps_w, sigma_g, eps_g, p5, p6, q_O]
 *   REVSIM_BUCK:                [A_w, B_w, C_w, A_g, B_g, C_g, q_O]
 *
 * Conventions as in revsim.h: FP64 AoS xyz host arrays copied in and out, int32 status
 * (REVSIM_OK or a negative REVSIM_ERR_*), one CUDA stream per handle, one host thread per
 * handle at a time.  All arithmetic is FP64 unless the descriptor asks for REVSIM_MIXED.
 */
#ifndef REVSIM_GAS_H
#define REVSIM_GAS_H

#include <stdint.h>

#include "revsim.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Loss terms (loss_type of diffusion.jl:823-834), bits of loss_type: :diff -> REVSIM_GAS_DIFF,
 * :rdf -> REVSIM_GAS_RDF, :ev -> REVSIM_GAS_EV; :diff_rdf_ev -> all three. */
#define REVSIM_GAS_DIFF 1
#define REVSIM_GAS_RDF 2
#define REVSIM_GAS_EV 4

typedef struct revsim_gas_handle revsim_gas_handle;

/* System description (replaces setup_system, diffusion.jl:1059-1179, and the constants of
 * diffusion.jl:29-52).  A zero field takes the reference's value. */
typedef struct {
    int32_t n_water, n_gas;   /* molecules */
    double box;               /* cubic side, nm (>= 2 nl_cutoff) */
    int32_t inter_type;       /* REVSIM_LJ .. REVSIM_BUFF */
    double temp;              /* K (295.15) */
    double m_O, m_H;          /* u; gas sites have mass m_O */
    double coulomb_const;     /* kJ mol^-1 nm e^-2 */
    double cutoff;            /* interaction cutoff, nm (1.0) */
    double nl_cutoff;         /* neighbour-list cutoff, nm (1.2) */
    int32_t n_steps_nf;       /* neighbour rebuild period (20) */
    double kB;                /* u nm^2 ps^-2 K^-1 */
    double kb_w, r0_w, ka_w, th0_w;  /* water bonds / angle (462750.4, 0.09572, 836.8,
                                        1.82421813418) */
    double kb_g, r0_g;        /* O2 bond (1640.4 * 4.184 * 100, 0.12074) */
    int32_t n_mol_ev;         /* molecules dividing U in the enthalpy term (n_water + n_gas) */
    int32_t device;           /* CUDA device ordinal */
    int32_t precision;        /* REVSIM_FP64 (0) or REVSIM_MIXED: FP32 pair arithmetic; state,
                                 bonded terms, integrator, adjoints and sums stay FP64 */
} revsim_gas_desc;

/* System(...) of setup_system. */
int32_t revsim_gas_create(const revsim_gas_desc *desc, revsim_gas_handle **out);
int32_t revsim_gas_destroy(revsim_gas_handle *h);
const char *revsim_gas_last_error(const revsim_gas_handle *h);

/* inter_n_params + 1 of diffusion.jl:157-162: 5 for REVSIM_LJ, 7 otherwise. */
int32_t revsim_gas_n_params(int32_t inter_type);

/* generate_inter / inject_atom_grads (diffusion.jl:126-155, 584-615). */
int32_t revsim_gas_set_params(revsim_gas_handle *h, const double *theta, int32_t n_params);
/* coords / velocities [3 N], N = 3 n_water + 2 n_gas. */
int32_t revsim_gas_set_state(revsim_gas_handle *h, const double *x, const double *v);
int32_t revsim_gas_get_state(revsim_gas_handle *h, double *x, double *v);

/* The RDF term: loss_rdf (diffusion.jl:759-774) over the water atoms, n_terms smoothed-RDF
 * terms (revsim_rdf_term of revsim.h, e.g. the O-O and O-H L1 terms against the Soper data of
 * read_rdf_data, diffusion.jl:673-686) with their targets [n_target] each, weighted
 * 0.05 / n_blocks (loss_weighting_rdf, diffusion.jl:51) at every loss point. */
int32_t revsim_gas_set_rdf(revsim_gas_handle *h, int32_t n_terms, const revsim_rdf_term *terms,
                           const double *const *targets);

/* calc_F! at the current state: F [3 N]. */
int32_t revsim_gas_forces(revsim_gas_handle *h, double *F);

/* calc_F_and_grads! at the current state (diffusion.jl:1300-1509): forces F [3 N], the VJP
 * dl_dfi [3 N] against dl_dfi_prev = w [3 N], and dl_dp [n_params] = sum_a acoef[a] .
 * dF_a/dtheta (the contraction of diffusion.jl:1576-1578 with acoef in place of
 * A dt^2 / 2m). */
int32_t revsim_gas_force_vjp(revsim_gas_handle *h, const double *w, const double *acoef,
                             double *F, double *dl_dfi, double *dl_dp);

/* potential_energy (diffusion.jl:804) at the current state and, when dEdp is non-NULL,
 * dE/dtheta [n_params]. */
int32_t revsim_gas_energy(revsim_gas_handle *h, double *E, double *dEdp);

/* forward_sim (diffusion.jl:1181-1298 without the RAD gradient): n_steps B-A-O-A steps from
 * the current state with noise_seeds[n_steps]; snapshots of x, v at step 0 and every loss
 * point and the gas centres at the loss points stay on the handle for revsim_gas_reverse.
 * When calc_loss, loss receives loss_fn_final and parts[4] = (D in m^2/s, l_diff, l_rdf,
 * l_ev); centres [n_blocks * n_gas * 3] (may be NULL) the centres of loss_accum. */
int32_t revsim_gas_forward(revsim_gas_handle *h, const uint64_t *noise_seeds, double gamma,
                           int32_t n_steps, int32_t n_steps_loss, double dt, int32_t loss_type,
                           int32_t calc_loss, double *loss, double *parts, double *centres);

/* reverse_sim (diffusion.jl:1511-1616) after revsim_gas_forward with the same noise_seeds,
 * gamma, n_steps, n_steps_loss and dt: loss, dl_dp [n_params], parts[4] as above.  It starts
 * from the forward's last snapshot (fwd_coords_logger[end], diffusion.jl:1557-1558) whatever
 * the current state, with the current parameters.  The state afterwards is the
 * reconstruction of the first block's start; the forward record is consumed. */
int32_t revsim_gas_reverse(revsim_gas_handle *h, const uint64_t *noise_seeds, double gamma,
                           int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc,
                           double dt, int32_t loss_type, double *loss, double *dl_dp,
                           double *parts);

/* Instrumentation: the handle's stream, kernels launched so far, and per-kernel CUDA-event
 * timing of the step kernels (which: 0 reverse step, 1 forward step). */
void *revsim_gas_stream(revsim_gas_handle *h);
int64_t revsim_gas_launch_count(const revsim_gas_handle *h);
int32_t revsim_gas_set_kernel_timing(revsim_gas_handle *h, int32_t enable);
int32_t revsim_gas_kernel_time(revsim_gas_handle *h, int32_t which, double *total_ms,
                               int64_t *launches);

#ifdef __cplusplus
}
#endif

#endif
