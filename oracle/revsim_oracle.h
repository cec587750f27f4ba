/*
 * revsim_oracle.h -- CPU FP64 restatement of the reversible-simulation gradient
 * of greener-group/rev-sim `water/water.jl` (3-site flexible water, LJ-family pair
 * term + reaction-field Coulomb, harmonic bonds/angles, Langevin B-A-O-A steps,
 * reverse-time reconstruction with the A-D adjoint accumulators, smoothed-RDF loss).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/, the smoke
 * check and the CPU-baseline leg of bench.py load it.  The product path (the CUDA
 * library behind include/revsim.h) never calls into it.
 *
 * Parity status: the reference is Julia on Molly v0.21.1 / Enzyme / Zygote, and no
 * Julia toolchain exists on either machine, so the reference cannot be run and it
 * ships no golden vectors.  Absolute values are therefore "parity unpinned"; the
 * restatement is pinned instead by the reference's own self-consistency assertions
 * (water.jl:1613-1615: reconstruction < 1e-9 in FP64, |L_rev - L_fwd| < 1e-7),
 * by central finite differences of every derivative (the diffusion.jl:1659-1667
 * pattern) and by energy/force consistency (F = -dU/dx).
 *
 * Conventions restated from third-party Molly v0.21.1 (not vendored in the reference):
 *   vector(c1, c2): per-dimension minimum image, returns c2 - c1 (see orc_vec1d);
 *   wrap_coords: c - floor(c / L) * L;
 *   random_velocity_3D(m, T, k): three N(0, sqrt(k T / m)) draws;
 *   coulomb_const: passed in by the caller (Molly's coulombconst, kJ mol^-1 nm e^-2);
 *   neighbour set: pairs i<j of different molecules with min-image d^2 <= rc_nl^2.
 * All arithmetic is FP64 and compiled with -ffp-contract=off so that no fused
 * multiply-add changes the rounding of the reference's expressions.
 */
#ifndef REVSIM_ORACLE_H
#define REVSIM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pair forms, in the order of water.jl:121-150 (generate_inter). */
enum { ORC_LJ = 0, ORC_DEXP = 1, ORC_BUCK = 2, ORC_LJSC = 3, ORC_BUFF = 4 };

/* A water system: atoms ordered O, H1, H2 per molecule (tip3p.pdb order), bonds
 * (O,H1), (O,H2), angle (H1, O, H2) with O central.  Parameter vector layout
 * follows water.jl:1572-1582: [pair-form params..., q_O, k_b, r0, k_a, theta0]. */
typedef struct {
    int32_t n_mol;
    double box;            /* cubic side, nm */
    double m_O, m_H;       /* u */
    int32_t inter_type;    /* ORC_* */
    double coulomb_const;  /* kJ mol^-1 nm e^-2 */
    double crf_const;      /* reaction-field k_rf, water.jl:41 */
    double cutoff;         /* interaction cutoff, nm (1.0) */
    double nl_cutoff;      /* neighbour-list cutoff, nm (1.2) */
    int32_t n_steps_nf;    /* neighbour rebuild period (20) */
    double kB;             /* u nm^2 ps^-2 K^-1 */
    double temp;           /* K */
    int32_t mlp;           /* 1: add the learned pair correction of mlp_oracle.h; its
                              ORC_MLP_NPARAMS parameters follow the classical ones */
} orc_system;

/* One smoothed-RDF loss term (water.jl:631-711).  The grid is
 * x_k = x_min + step*k (k = 0..n_grid-1); each distance is smeared with
 * exp(-(x-d)^2 / width) truncated at |x-d| <= exp_cutoff and normalised per
 * distance; h_k = V / (4 pi n1 n2 step) * sum / x_k^2.
 * loss = weight * sum_t |h[slice_start + t*slice_stride] - target[t]|^norm. */
typedef struct {
    int32_t sel1, sel2;    /* 0 = O atoms, 1 = H atoms */
    double x_min, step, width, exp_cutoff;
    int32_t n_grid;
    int32_t slice_start, slice_stride, n_target;
    const double *target;
    int32_t norm;          /* 1 = L1 (reference), 2 = squared error */
    double weight;
} orc_rdf_term;

/* The loss of loss_fn (water.jl:757-769): the RDF terms, plus -- when enth_vap is set -- the
 * enthalpy-of-vaporisation term of loss_enth_vap (water.jl:738-755),
 * l_ev = (u_gas - U / n_mol + rt - target)^2, U the potential energy (the reference's values:
 * u_gas 3.69, rt 2.45, target 44.12 + 2.8 kJ/mol). */
typedef struct {
    int32_t n_terms;
    const orc_rdf_term *terms;
    int32_t enth_vap;
    double u_gas, rt, target;
} orc_loss;

int32_t orc_n_form_params(int32_t inter_type);
int32_t orc_n_params(int32_t inter_type);
/* Classical parameters plus the MLP's when s->mlp. */
int32_t orc_system_n_params(const orc_system *s);

/* Minimum-image component of Molly's vector(c1, c2): c2 - c1 folded by one box. */
double orc_vec1d(double c1, double c2, double L);
double orc_wrap1d(double c, double L);

/* Neighbour pairs (i<j, different molecules, d^2 <= nl_cutoff^2), sorted by (i, j).
 * Writes up to max_pairs pairs into pairs[2*k], pairs[2*k+1]; returns the count
 * (which may exceed max_pairs: then only max_pairs are written). */
int64_t orc_neighbor_pairs(const orc_system *s, const double *x, int32_t *pairs, int64_t max_pairs);

/* calc_F! (water.jl:877-975): total force F[3N] over the given pair list. */
void orc_forces(const orc_system *s, const double *params, const double *x,
                const int32_t *pairs, int64_t n_pairs, double *F);

/* calc_F_and_grads! (water.jl:1212-1433): forces F[3N], the force VJP
 * dl_dfi[b] = sum_a (w[a]/m_a) . dF_a/dx_b with w = dl_dfi_prev, and the parameter
 * Jacobian of the classical parameters dF_dp[3N * P] (row-major, index (3a+u)*P + p,
 * P = orc_n_params).  dF_dp may be NULL. */
void orc_forces_grads(const orc_system *s, const double *params, const double *x,
                      const int32_t *pairs, int64_t n_pairs, const double *w,
                      double *F, double *dl_dfi, double *dF_dp);

/* sum_a acoef_a . dF_a/dtheta for every parameter (classical and MLP): dtheta[P]. */
void orc_contract(const orc_system *s, const double *params, const double *x,
                  const int32_t *pairs, int64_t n_pairs, const double *acoef, double *dtheta);

/* Potential energy and its parameter gradient dEdp[P] (classical, then the MLP's): the
 * per-snapshot dE/dtheta of the reweighting estimator (water.jl:1176-1183). */
double orc_energy_grads(const orc_system *s, const double *params, const double *x,
                        const int32_t *pairs, int64_t n_pairs, double *dEdp);

/* Potential energy (pair form + reaction-field Coulomb + bonds + angles). */
double orc_energy(const orc_system *s, const double *params, const double *x,
                  const int32_t *pairs, int64_t n_pairs);

/* Per-step Langevin noise: xi[3a+u] = sqrt(kB T / m_a) * z, z ~ N(0,1) from
 * Philox4x32-10 keyed by the 64-bit step seed, counter (a, 0/1, 0, 0), Box-Muller. */
void orc_noise(const orc_system *s, uint64_t seed, double temp, double *xi);
/* Four N(0,1) draws for (seed, atom): Philox blocks 0 and 1 (the per-atom draw of orc_noise). */
void orc_philox_normals(uint64_t seed, uint32_t atom, double z[4]);
/* Building blocks shared with the gas-in-water restatement (gas_oracle.c).
 * orc_pair_form: F(r) (positive = repulsive), dF/dr and dF/dtheta of one pair form for
 * the per-pair parameters p (its own mixing of p with itself is exact), invr2 = 1/r2;
 * returns 0 when the iszero gate switches the form off.  orc_pair_form_energy: its
 * potential energy.  orc_angle_term: the harmonic angle's forces on the two outer
 * atoms for the arms a, b from the central atom (the central atom takes minus their
 * sum) and their tangents along (ta, tb); returns 0 when a x b = 0. */
int32_t orc_pair_form(int32_t type, const double *p, double r, double invr2, int32_t grads,
                      double *F, double *dFdr, double *g);
double orc_pair_form_energy(int32_t type, const double *p, double r);
int32_t orc_angle_term(const double a[3], const double b[3], const double ta[3],
                       const double tb[3], double ka, double th0, double Fi[3], double Fk[3],
                       double dFi[3], double dFk[3]);

/* RDF histogram of one term at positions x: writes h[n_grid]. */
void orc_rdf(const orc_system *s, const orc_rdf_term *t, const double *x, double *h);

/* The RDF terms' loss and dL/dx[3N] (dLdx may be NULL); ignores the enthalpy term. */
double orc_loss_grad(const orc_system *s, const orc_loss *L, const double *x, double *dLdx);

/* loss_and_grads (water.jl:771-786) at x: returns the loss; l_parts[2] (may be NULL) receives
 * its RDF and enthalpy parts, dLdx[3N] (may be NULL) dL/dx, and dl_dp[P] (may be NULL) the
 * direct parameter gradient.  With the enthalpy term, e = u_gas - U/n_mol + rt - target gives
 * dl_ev/dx = (2 e / n_mol) F and dl_ev/dtheta = -(2 e / n_mol) dU/dtheta (the RDF terms have
 * no direct parameter dependence).  U sums over a fresh neighbour list, as
 * enthalpy_vaporization's find_neighbors does (water.jl:743). */
double orc_loss_and_grads(const orc_system *s, const double *params, const orc_loss *L,
                          const double *x, double *l_parts, double *dLdx, double *dl_dp);

/* forward_sim (water.jl:977-1105, loop 1029-1045).  x, v are updated in place
 * (final state).  Snapshots of x and v are written every n_steps_log steps,
 * including step 0, into snap_x/snap_v [(n_steps/n_steps_log + 1) * 3N] if not NULL.
 * Returns the block-averaged loss (0 when calc_loss == 0); l_parts[2] (may be NULL) receives
 * its block-averaged RDF and enthalpy parts. */
double orc_forward_sim(const orc_system *s, const double *params, double *x, double *v,
                       const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                       int32_t n_steps_loss, double dt, int32_t n_steps_log,
                       const orc_loss *loss, int32_t calc_loss,
                       double *snap_x, double *snap_v, double *l_parts);

/* reverse_sim (water.jl:1435-1558).  x, v: final forward state on entry,
 * reconstructed initial state on exit.  dl_dp[P] receives the gradient (the adjoint terms
 * plus, with the enthalpy term, the direct dl/dtheta of every loss point, water.jl:1540).
 * Returns the block-averaged loss (l_parts as for orc_forward_sim); NaN on bad arguments. */
double orc_reverse_sim(const orc_system *s, const double *params, double *x, double *v,
                       const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                       int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                       int32_t n_steps_log, const double *snap_x, const double *snap_v,
                       double clip_norm_threshold, const orc_loss *loss, double *dl_dp,
                       double *l_parts);

/* orc_forward_sim / orc_reverse_sim with the caller's noise host_noise [n_steps][3N] (entry
 * step - 1 = generate_noise!'s xi of step `step`, water.jl:867-873) in place of the seeds'
 * Philox draws (water.jl:1033-1036, 1497-1498). */
double orc_forward_sim_hn(const orc_system *s, const double *params, double *x, double *v,
                          const double *host_noise, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, double dt, int32_t n_steps_log,
                          const orc_loss *loss, int32_t calc_loss,
                          double *snap_x, double *snap_v, double *l_parts);
double orc_reverse_sim_hn(const orc_system *s, const double *params, double *x, double *v,
                          const double *host_noise, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                          int32_t n_steps_log, const double *snap_x, const double *snap_v,
                          double clip_norm_threshold, const orc_loss *loss, double *dl_dp,
                          double *l_parts);

/* Monte-Carlo barostat: MonteCarloBarostatNoUnits and its apply_coupling!
 * (water.jl:789-865) as forward_sim runs it with use_barostat (water.jl:1009-1014,
 * 1043-1044): every n_steps steps, after the step's neighbour refresh, one volume move
 * dV = volume_scale (2 u1 - 1), molecule centres scaled by l = cbrt((V + dV) / V) with the
 * box, the energy of the trial state over the same pair list, and acceptance if
 * dW = dU + P dV N_A - n_mol kB T ln(v_scale) <= 0 or u2 < exp(-dW / (kB T)) (kJ/mol);
 * after every 10 attempts volume_scale shrinks by scale_increment below 25 % acceptance
 * and grows (up to max_volume_frac V) above 75 %.
 * Differences, each deliberate: the two uniforms of attempt k are
 * orc_barostat_uniform(seed, 2k) and (seed, 2k + 1), a counter-based stream, where the
 * reference draws Julia's global rand(); the molecule centre is the mean of the O atom and
 * the minimum-image positions of its H atoms (Molly's scale_coords! averages the stored,
 * wrapped positions, which differs only for a molecule split across the box face). */
typedef struct {
    double pressure;          /* bar (1.0 in water.jl:1011) */
    int32_t n_steps;          /* attempt period in steps (30) */
    double volume_scale;      /* nm^3 (box volume x 0.01 at construction) */
    double scale_increment;   /* 1.1 */
    double max_volume_frac;   /* 0.3 */
    uint64_t seed;
    int64_t n_attempted, n_accepted;   /* the adaptation window */
    int64_t n_draws;                   /* attempts so far (the draw counter) */
    int64_t n_accepted_total;
} orc_barostat;

/* Uniform in [0, 1) from draw k of the stream `seed` (splitmix64 of seed + k). */
double orc_barostat_uniform(uint64_t seed, uint64_t k);

/* One attempt on (x, s->box) with the given pair list; updates x, s->box and b; returns 1
 * when the move was accepted. */
int32_t orc_barostat_attempt(orc_system *s, const double *params, double *x, const int32_t *pairs,
                             int64_t n_pairs, orc_barostat *b);

/* forward_sim with use_barostat and calc_loss = false (the equilibration runs of train(),
 * water.jl:1642-1645): n_steps B-A-O-A steps, neighbour rebuild every n_steps_nf steps, a
 * barostat attempt every b->n_steps steps.  Updates x, v, s->box and b. */
void orc_forward_sim_barostat(orc_system *s, const double *params, double *x, double *v,
                              const uint64_t *noise_seeds, double gamma, int32_t n_steps, double dt,
                              orc_barostat *b);

/* Number of OpenMP threads used by the force loops (1 when built without OpenMP). */
int32_t orc_num_threads(void);
void orc_set_num_threads(int32_t n);

#ifdef __cplusplus
}
#endif
#endif
