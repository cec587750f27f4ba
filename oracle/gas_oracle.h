/*
 * gas_oracle.h -- CPU FP64 restatement of the gas-in-water reversible-simulation gradient
 * of greener-group/rev-sim `diffusion/diffusion.jl`: n_water flexible 3-site waters
 * (atoms O, H1, H2) followed by n_gas two-site O2 molecules (atoms O1, O2), a pair form
 * between unlike sites by Lorentz-Berthelot mixing (diffusion.jl:165-430), reaction-field
 * Coulomb between water sites, fixed harmonic water bonds / angles and a fixed O2 bond
 * (diffusion.jl:1068-1118), Langevin B-A-O-A steps, and the diffusion-coefficient loss
 * from the mean-squared displacement of the gas centres at the loss points, whose gradient
 * is injected at every loss point of the reverse pass (diffusion.jl:817-947, 1511-1616).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load it; the product path (the CUDA library behind
 * include/revsim_gas.h) never calls into it.
 *
 * Parity status: the reference is Julia (Molly / Enzyme / Zygote) and cannot run here, and it
 * ships no golden vectors for this path, so absolute values are parity unpinned.  The
 * restatement is pinned by the reference's own assertions (diffusion.jl:1674-1675:
 * reconstruction < 1e-9 in FP64 when n_steps_trunc >= n_steps_loss, |L_rev - L_fwd| < 1e-7),
 * by central finite differences of forces, the force VJP, the dF/dtheta contraction and the
 * whole reverse gradient against the forward loss (the diffusion.jl:1659-1667 check), and by
 * F = -dU/dx.  Shared conventions with revsim_oracle.h (minimum image, wrap, Philox noise).
 *
 * Parameter vector (diffusion.jl:1629-1639, inject_atom_grads 584-615, extract_grads 617-671):
 *   LJ:             [sigma_w, eps_w, sigma_g, eps_g, q_O]
 *   dexp/ljsc/buff: [sigma_w, eps_w, sigma_g, eps_g, p5, p6, q_O]  (p5, p6 the form's own)
 *   buck:           [A_w, B_w, C_w, A_g, B_g, C_g, q_O]
 * H sites carry no pair form (eps = 0 / A = 0); gas sites no charge.
 */
#ifndef GAS_ORACLE_H
#define GAS_ORACLE_H

#include <stdint.h>

#include "revsim_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t n_water, n_gas;  /* molecules; atoms 3 n_water + 2 n_gas, waters first */
    double box;              /* cubic side, nm */
    double m_O, m_H;         /* u; gas sites have mass m_O (diffusion.jl:40-44) */
    int32_t inter_type;      /* ORC_* of revsim_oracle.h */
    double coulomb_const, crf_const, cutoff, nl_cutoff;
    int32_t n_steps_nf;      /* neighbour rebuild period (20) */
    double kB, temp;
    double kb_w, r0_w, ka_w, th0_w;  /* water bonds and angle (fixed) */
    double kb_g, r0_g;               /* O2 bond (fixed) */
    int32_t n_mol_ev;        /* molecules dividing U in the enthalpy term (all: diffusion.jl:804) */
} orc_gas_system;

/* Loss selection: bit 0 the diffusion term, bit 1 the RDF term, bit 2 the enthalpy-of-
 * vaporisation term (loss_type :diff, :rdf, :ev and their sums, diffusion.jl:823-834).  The
 * RDF term is loss_rdf (diffusion.jl:759-774) over the water atoms: the terms of an orc_loss
 * (revsim_oracle.h; e.g. the O-O and O-H L1 terms against the Soper data) evaluated as the
 * water restatement does for a box of n_water molecules, weighted 0.05 / n_blocks. */
enum { ORC_GAS_DIFF = 1, ORC_GAS_RDF = 2, ORC_GAS_EV = 4 };

int32_t orc_gas_n_params(int32_t inter_type);

/* Pairs i < j with min-image d^2 <= nl_cutoff^2, excluding the pairs inside one molecule
 * (eligible matrix of diffusion.jl:1133-1147).  Returns the total count; fills at most
 * max_pairs. */
int64_t orc_gas_neighbor_pairs(const orc_gas_system *s, const double *x, int32_t *pairs,
                               int64_t max_pairs);

/* calc_F! (diffusion.jl:959-1057). */
void orc_gas_forces(const orc_gas_system *s, const double *params, const double *x,
                    const int32_t *pairs, int64_t n_pairs, double *F);

/* calc_F_and_grads! (diffusion.jl:1300-1509): forces F, the VJP dl_dfi against
 * dl_dfi_prev = w (divided by the masses inside, as the reference does), and
 * dl_dp[p] += sum_a acoef[a] . dF_a/dtheta_p (the contraction of diffusion.jl:1576-1578). */
void orc_gas_forces_grads(const orc_gas_system *s, const double *params, const double *x,
                          const int32_t *pairs, int64_t n_pairs, const double *w,
                          const double *acoef, double *F, double *dl_dfi, double *dl_dp);

/* Potential energy over the pairs within the cutoff and the bonded terms; dE/dtheta when
 * dEdp is non-NULL. */
double orc_gas_energy(const orc_gas_system *s, const double *params, const double *x,
                      const int32_t *pairs, int64_t n_pairs, double *dEdp);

/* Langevin noise of every atom for one step seed (Philox normals x sqrt(kB T / m)). */
void orc_gas_noise(const orc_gas_system *s, uint64_t seed, double *xi);

/* Gas centres c1 + vector(c1, c2) / 2, wrapped (extract_gas_coords, diffusion.jl:836-844). */
void orc_gas_centres(const orc_gas_system *s, const double *x, double *c);

/* calculate_D (diffusion.jl:861-877, its Enzyme pullback 879-895) over n_frames frames of n_gas centres, in nm^2/ps;
 * its gradient with respect to every centre coordinate into dD_dgc when non-NULL. */
double orc_gas_diffusion_D(const double *gc, int32_t n_frames, int32_t n_gas, double box,
                           double loss_frequency, double *dD_dgc);

/* The loss of loss_fn_final (diffusion.jl:897-911) from the frames and, for the RDF and
 * enthalpy terms, their accumulated per-frame sums; out[0..3] = D (m^2/s), l_diff, l_rdf,
 * l_ev.  dl_dgc receives the gradient of l_diff with respect to the centres when non-NULL. */
double orc_gas_loss_final(int32_t loss_type, const double *gc, int32_t n_frames, int32_t n_gas,
                          double box, double loss_frequency, double ev_sum, double rdf_sum,
                          double *out, double *dl_dgc);

/* One loss point's enthalpy term l = 0.05 (dH - 46.92)^2 / n_blocks with its gradients
 * dl/dx (dLdx) and the direct dl/dtheta (added into dl_dp) when non-NULL. */
double orc_gas_ev_point(const orc_gas_system *s, const double *params, const double *x,
                        int32_t n_blocks, double *dLdx, double *dl_dp);

/* forward_sim (diffusion.jl:1181-1298) without the RAD gradient; rdf: the RDF terms (used
 * when loss_type has ORC_GAS_RDF).  snap_x / snap_v
 * [(n_blocks + 1) * 3N]: the state at step 0 and at every loss point; gc
 * [n_blocks * n_gas * 3] the gas centres at the loss points.  Returns the loss when
 * calc_loss, else 0; out[0..3] as orc_gas_loss_final. */
double orc_gas_forward_sim(const orc_gas_system *s, const double *params, double *x, double *v,
                           const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                           int32_t n_steps_loss, double dt, int32_t loss_type,
                           int32_t calc_loss, double *snap_x, double *snap_v, double *gc,
                           double *out, const orc_loss *rdf);

/* reverse_sim (diffusion.jl:1511-1616) from the final state in x, v (and the forward's
 * snapshots and centres): returns the loss; dl_dp [P]; out[0..3] as above.  After a
 * snapshot restore the neighbour pairs are rebuilt (the reference keeps its list; a rebuilt
 * list holds every pair within the cutoff, which the stale one does only while no pair has
 * moved 0.2 nm). */
double orc_gas_reverse_sim(const orc_gas_system *s, const double *params, double *x, double *v,
                           const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                           int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                           int32_t loss_type, const double *snap_x, const double *snap_v,
                           const double *gc, double *dl_dp, double *out, const orc_loss *rdf);

#ifdef __cplusplus
}
#endif

#endif
