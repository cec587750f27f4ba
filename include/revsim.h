/*
 * revsim.h -- C ABI of the B200 (sm_100a) reversible-simulation gradient engine.
 *
 * The engine replaces the hot path of greener-group/rev-sim `water/water.jl`:
 * forward_sim (water.jl:977-1105), reverse_sim (water.jl:1435-1558) and the force /
 * force-gradient kernels they call (calc_F! water.jl:877-975, calc_F_and_grads!
 * water.jl:1212-1433, Molly's CellListMapNeighborFinder, loss_and_grads
 * water.jl:771-787).  Plain C types only: host arrays are FP64 AoS xyz
 * (Julia's reinterpret(Float64, ::Vector{SVector{3,Float64}}) layout), copied in and
 * out; the library never keeps a host pointer.  Every entry point returns an int32
 * status (REVSIM_OK or a negative REVSIM_ERR_*); no C++ exception crosses the ABI.
 * A handle owns all device memory and one CUDA stream; calls on one handle must come
 * from one host thread at a time.
 *
 * A handle holds R >= 1 independent replicas (water boxes of their own size,
 * box side and temperature) that are stepped together in one launch per step.
 */
#ifndef REVSIM_H
#define REVSIM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define REVSIM_OK 0
#define REVSIM_ERR_BADARG (-1)
#define REVSIM_ERR_CUDA (-2)
#define REVSIM_ERR_NLIST_OVERFLOW (-3)
#define REVSIM_ERR_NAN (-4)
#define REVSIM_ERR_TIMEOUT (-5)
#define REVSIM_ERR_GEOMETRY (-6)
#define REVSIM_ERR_STATE (-7)
#define REVSIM_ERR_NOMEM (-8)

/* Pair forms, same order as generate_inter (water.jl:121-150). */
#define REVSIM_LJ 0
#define REVSIM_DEXP 1
#define REVSIM_BUCK 2
#define REVSIM_LJSC 3
#define REVSIM_BUFF 4

/* Arithmetic of the pair terms.  State (x, v), reverse reconstruction, the adjoint
 * accumulators and the parameter-gradient sum are FP64 in both modes. */
#define REVSIM_FP64 0
#define REVSIM_MIXED 1 /* FP32 pair / bonded-term arithmetic */

/* Neighbour lists used by the reverse pass. */
#define REVSIM_NL_CHECKPOINT 0 /* rebuilt from the forward pass's build positions */
#define REVSIM_NL_RECONSTRUCTED 1 /* rebuilt from reconstructed positions, water.jl:1504 */

typedef struct revsim_handle revsim_handle;

/* System description (replaces System(structure_file, ff; ...) at water.jl:980-991
 * and the constants of water.jl:27-48).  Water atoms are ordered O, H1, H2. */
typedef struct {
    int32_t n_replicas;
    const int32_t *n_mol;   /* [n_replicas] molecules per replica */
    const double *box;      /* [n_replicas] cubic box side, nm */
    const double *temp;     /* [n_replicas] K */
    int32_t inter_type;     /* REVSIM_LJ .. REVSIM_BUFF */
    int32_t precision;      /* REVSIM_FP64 or REVSIM_MIXED */
    double m_O, m_H;        /* u */
    double coulomb_const;   /* kJ mol^-1 nm e^-2 */
    double crf_const;       /* reaction-field k_rf, nm^-3 */
    double cutoff;          /* interaction cutoff, nm */
    double nl_cutoff;       /* neighbour-list cutoff, nm */
    double kB;              /* u nm^2 ps^-2 K^-1 */
    int32_t n_steps_nf;     /* neighbour rebuild period, steps */
    int32_t n_steps_log;    /* forward snapshot period, steps */
    int32_t nl_mode;        /* REVSIM_NL_CHECKPOINT or REVSIM_NL_RECONSTRUCTED */
    int32_t device;         /* CUDA device ordinal */
    int32_t mlp;            /* 1: add the learned pair correction (REVSIM_LJ only); its
                               REVSIM_MLP_NPARAMS parameters follow the classical ones */
} revsim_system_desc;

/* The learned pair correction (no reference counterpart; it takes the place of the
 * reference's PyTorch / JAX learned terms, water_maceoff.jl:147-163): per element pair
 * (O-O, O-H, H-H) of different molecules within the cutoff, u(r) = MLP(phi(r)) fc(r) with
 * 16 Gaussian radial basis functions (centres k rc/15, width 0.05 nm), 64 -> 64 SiLU ->
 * scalar, fc(r) = (cos(pi r / rc) + 1) / 2, tabulated on 1,024 intervals of [0, rc] and
 * interpolated with cubic Hermite segments.  Parameters per type: W1[64][16], b1[64],
 * W2[64][64], b2[64], w3[64], b3. */
#define REVSIM_MLP_NPARAMS 15939

/* Arithmetic of the learned term's network (no reference counterpart).  The interval table
 * is built from the network's value and r-derivative at its 1,025 nodes per type, and the
 * reverse pass carries the table's adjoints back to the weights; both run either in FP64
 * scalar kernels (REVSIM_MLP_FP64, the default) or on the tensor cores with BF16 operands
 * and FP32 accumulation (REVSIM_MLP_BF16_TC: the forward and r-tangent GEMMs, the backward
 * through both streams with the mixed second derivative d^2u/dr dtheta, and the weight-
 * gradient GEMMs over the node batch; parameters stay FP64; each operand is split into a
 * BF16 high part and a BF16 remainder, three MMAs per product, ~16 significant bits). */
#define REVSIM_MLP_FP64 0
#define REVSIM_MLP_BF16_TC 1

/* One smoothed-RDF loss term (rdf_differentiable + loss_rdf_part, water.jl:631-697):
 * grid x_k = x_min + step*k, k < n_grid; Gaussian exp(-(x-d)^2/width) truncated at
 * |x-d| <= exp_cutoff and normalised per distance; loss =
 * weight * sum_t |h[slice_start + t*slice_stride] - target_t|^norm (norm 1 or 2).
 * sel: 0 = O atoms, 1 = H atoms. */
typedef struct {
    int32_t sel1, sel2;
    double x_min, step, width, exp_cutoff;
    int32_t n_grid;
    int32_t slice_start, slice_stride, n_target;
    int32_t norm;
    double weight;
} revsim_rdf_term;

/* Create / destroy.  Replaces System construction + inject_atom_grads (water.jl:546-569). */
int32_t revsim_create(const revsim_system_desc *desc, revsim_handle **out);
void revsim_destroy(revsim_handle *h);
/* Last error message of this handle ("" when none); valid until the next call. */
const char *revsim_last_error(const revsim_handle *h);
/* Status of the device-side checks (bit flags) accumulated since the last call. */
int32_t revsim_device_status(revsim_handle *h, int32_t *flags);

/* Sizes: total atoms over replicas and the parameter count P of the pair form. */
int32_t revsim_sizes(const revsim_handle *h, int64_t *n_atoms, int32_t *n_params);

/* Parameters in the reference layout [pair form..., q_O, k_b, r0, k_a, theta0]
 * (water.jl:1572-1582, inject_si_grads water.jl:528-543). */
int32_t revsim_set_params(revsim_handle *h, const double *theta, int32_t n_params);

/* State of all replicas, concatenated: x, v [3 * n_atoms]. */
int32_t revsim_set_state(revsim_handle *h, const double *x, const double *v);
int32_t revsim_get_state(revsim_handle *h, double *x, double *v);

/* Loss terms and per-replica targets [n_replicas * n_target] for each term. */
int32_t revsim_set_loss(revsim_handle *h, int32_t n_terms, const revsim_rdf_term *terms,
                        const double *const *targets);

/* Neighbour pair set of one replica at the current positions (Molly
 * find_neighbors with the 1.2 nm CellListMap finder, water.jl:1025): pairs
 * (i, j), i < j, replica-local atom indices, in no particular order.  Writes
 * min(count, cap) pairs to pairs[2k], pairs[2k+1] and the total to *count. */
int32_t revsim_neighbor_pairs(revsim_handle *h, int32_t replica, int32_t *pairs, int64_t cap,
                              int64_t *count);

/* calc_F! (water.jl:877-975) at the current positions: F [3 * n_atoms]. */
int32_t revsim_forces(revsim_handle *h, double *F);

/* calc_F_and_grads! (water.jl:1212-1433) at the current positions with
 * dl_dfi_prev = w [3 n_atoms]: forces F, the force VJP dl_dfi [3 n_atoms] and the
 * contraction dtheta[r*P + p] = sum_{a in replica r} acoef[a] . dF_a/dtheta_p
 * (the reference's sum(A dt^2/(2m) dF_dp), water.jl:1517-1519). */
int32_t revsim_force_vjp(revsim_handle *h, const double *w, const double *acoef, double *F,
                         double *dl_dfi, double *dtheta);

/* The potential energy energy[n_replicas] and its parameter gradient dEdtheta
 * [n_replicas * P] at the current state (the Zygote gradient of potential_energy in
 * reweighting_sim, water.jl:1176-1183).  Either output may be NULL. */
int32_t revsim_energy_grad(revsim_handle *h, double *energy, double *dEdtheta);

/* generate_noise! (water.jl:867-873) for one step seed per replica: xi [3 n_atoms]. */
int32_t revsim_noise(revsim_handle *h, const uint64_t *seeds, double *xi);

/* loss_and_grads (water.jl:771-787): loss [n_replicas] and dL/dx [3 n_atoms]
 * (dLdx may be NULL). */
int32_t revsim_loss_grad(revsim_handle *h, double *loss, double *dLdx);

/* The enthalpy-of-vaporisation loss term of loss_fn's loss_type :enth_vap and :both
 * (enthalpy_vaporization / loss_enth_vap, water.jl:738-769): per replica
 * l_ev = (u_gas - U / n_molecules + rt - target)^2, U the potential energy over a neighbour
 * list built from the current positions, added to the RDF terms' loss (revsim_set_loss; no
 * terms = :enth_vap) at every loss point of revsim_forward, revsim_reverse, revsim_loss_grad
 * and revsim_loss_and_grads.  Its dL/dx is (2 e / n) F and its direct parameter gradient
 * -(2 e / n) dU/dtheta, e = u_gas - U/n + rt - target, which revsim_reverse adds at every
 * loss point (water.jl:1471, 1540).  enable 0 removes the term.  The reference's constants:
 * u_gas 3.69, rt 2.45, target 44.12 + 2.8 kJ/mol.  No counterpart function in the
 * reference, whose loss_type argument selects the same terms. */
int32_t revsim_set_enth_vap(revsim_handle *h, int32_t enable, double u_gas, double rt, double target);

/* Monte-Carlo barostat of forward_sim's use_barostat (MonteCarloBarostatNoUnits and its
 * apply_coupling!, water.jl:789-865, set up at water.jl:1009-1014): every n_steps forward
 * steps (counted over the revsim_forward calls since it was switched on, so a run split into
 * blocks keeps the reference's schedule), after the step's neighbour refresh, each replica
 * tries one volume move:
 * dV = volume_scale (2 u1 - 1), molecule centres (O plus the mean of the minimum-image O->H
 * vectors) scaled with the box by cbrt((V + dV) / V), the energy of the trial state over the
 * current neighbour rows, acceptance if dW = dU + P dV N_A - n_mol kB T ln((V + dV) / V) <= 0
 * or u2 < exp(-dW / (kB T)); after every 10 attempts volume_scale is divided by
 * scale_increment below 25 % acceptance and multiplied (up to max_volume_frac V) above 75 %.
 * u1, u2 of replica r's attempt k are draws 2k and 2k+1 of the stream seed + r (splitmix64;
 * the reference draws Julia's global rand()).  A forward pass with the barostat on is an
 * equilibration run: revsim_reverse refuses its record. */
typedef struct {
    double pressure;          /* bar (1.0 in water.jl:1011) */
    int32_t n_steps;          /* attempt period, steps (30) */
    double scale_factor;      /* initial volume_scale / box volume (0.01) */
    double scale_increment;   /* 1.1 */
    double max_volume_frac;   /* 0.3 */
    uint64_t seed;
} revsim_barostat_desc;

/* Switch the barostat on (desc) or off (NULL); switching it on resets volume_scale to
 * scale_factor x the current box volume and the attempt counters. */
int32_t revsim_set_barostat(revsim_handle *h, const revsim_barostat_desc *desc);

/* Per replica: box side (nm), volume_scale (nm^3), attempts and accepted moves so far (any
 * output may be NULL). */
int32_t revsim_barostat_state(revsim_handle *h, double *box, double *volume_scale,
                              int64_t *n_attempts, int64_t *n_accepted);

/* The boundary argument of forward_sim / reverse_sim (water.jl:977, 1435, 1001): new cubic box
 * sides [n_replicas], nm (each above 2 x nl_cutoff).  Invalidates the forward record. */
int32_t revsim_set_box(revsim_handle *h, const double *box);

/* The RDF and enthalpy parts [n_replicas] of the loss the last revsim_forward or
 * revsim_reverse returned (loss_accum_rdf and loss_accum_ev over n_blocks, water.jl:1548-1551);
 * zeros after a forward pass without loss.  Either output may be NULL. */
int32_t revsim_loss_parts(revsim_handle *h, double *l_rdf, double *l_ev);

/* loss_and_grads (water.jl:771-786) at the current state, all of its outputs: loss, l_rdf and
 * l_ev [n_replicas], dl_dc = dL/dx [3 n_atoms] and the direct parameter gradient
 * dl_dp [n_replicas][n_params] (zero without the enthalpy term).  Any output may be NULL. */
int32_t revsim_loss_and_grads(revsim_handle *h, double *loss, double *l_rdf, double *l_ev,
                              double *dLdx, double *dl_dp);

/* One RDF histogram h [n_grid] of term t for one replica. */
int32_t revsim_rdf(revsim_handle *h, int32_t term, int32_t replica, double *hist);

/* forward_sim (water.jl:977-1105, loop 1029-1045) from the current state.
 * noise_seeds [n_steps * n_replicas], step-major.  Keeps snapshots every
 * n_steps_log steps and the neighbour-build positions on the device for the
 * reverse pass.  loss_out [n_replicas] (block-averaged; may be NULL). */
int32_t revsim_forward(revsim_handle *h, const uint64_t *noise_seeds, double gamma,
                       int32_t n_steps, int32_t n_steps_loss, double dt, int32_t calc_loss,
                       double *loss_out);

/* reverse_sim (water.jl:1435-1558) from the current state (the forward end state).
 * loss_out [n_replicas], dl_dp_out [n_replicas * P]: block-averaged loss and
 * gradient per replica.  clip_norm_threshold may be +inf. */
int32_t revsim_reverse(revsim_handle *h, const uint64_t *noise_seeds, double gamma,
                       int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                       double clip_norm_threshold, double *loss_out, double *dl_dp_out);

/* forward_sim / reverse_sim with the caller's own noise in place of the engine's seeded
 * Philox draws: host_noise [n_steps][3 n_atoms] (step-major; within a step the replicas'
 * atoms concatenated, xyz), entry step-1 = the velocity noise xi that generate_noise!
 * (water.jl:867-873) returns for the seed of step `step` (Molly random_velocity_3D, nm/ps,
 * sd sqrt(kB T / m)), used as v = v c + xi s in the forward step (water.jl:1033-1036) and
 * v = (v - xi s) / c in the reverse un-integration (water.jl:1497-1498).  A Julia host passes
 * the noise it draws with Xoshiro(seed), so that the engine runs the reference's own
 * trajectory for gamma > 0.  The reverse pass must get the same array as the forward pass.
 * The array is copied to the device (8 * 3 n_atoms * n_steps bytes) and not retained.
 * Otherwise as revsim_forward / revsim_reverse. */
int32_t revsim_forward_noise(revsim_handle *h, const double *host_noise, double gamma,
                             int32_t n_steps, int32_t n_steps_loss, double dt, int32_t calc_loss,
                             double *loss_out);
int32_t revsim_reverse_noise(revsim_handle *h, const double *host_noise, double gamma,
                             int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc,
                             double dt, double clip_norm_threshold, double *loss_out,
                             double *dl_dp_out);

/* Integrator arithmetic (no counterpart in the reference, whose FP64 step water.jl:1032-1037
 * and inverse 1496-1502 rebuild the start state only to rounding, which the dynamics' chaos
 * amplifies: in FP64 to ~1e-8 nm over 1,000 steps, and in mixed precision until a position
 * crosses an FP32 rounding boundary, after which the two passes' forces differ).
 * REVSIM_INTEGRATOR_REFERENCE (default): the reference's arithmetic.  REVSIM_INTEGRATOR_EXACT:
 * positions, velocities and box sides on the grid of multiples of 2^-48 nm (nm/ps), every
 * increment of the step (kick F dt / m, half drifts v dt / 2, the O step's result) rounded to
 * it, so the reverse pass subtracts exactly what the forward pass added: with gamma = 0 the
 * trajectory is rebuilt bit for bit in both precisions, however long the run; with friction
 * the O step's inverse stays approximate.  The state and boxes are rounded to the grid at the
 * start of each forward pass (<= 2^-49 nm, ~2e-15 nm); boxes must be under 32 nm
 * (REVSIM_ERR_BADARG otherwise).  Invalidates the forward record. */
#define REVSIM_INTEGRATOR_REFERENCE 0
#define REVSIM_INTEGRATOR_EXACT 1
int32_t revsim_set_integrator(revsim_handle *h, int32_t mode);

/* CUDA-graph mode (no counterpart in the reference, whose step loop is water.jl:1029-1045 /
 * 1492-1521): with enable = 1 each revsim_forward* / revsim_reverse* pass is captured from the
 * handle's stream into a CUDA graph the first time it runs with a given set of arguments and
 * handle configuration, and replayed with one graph launch on later calls (the per-step seeds
 * or noise are copied to the device before the replay, so new seeds reuse the graph).  A
 * change of parameters, loss terms, box, launch shape or any device buffer recaptures it (an
 * update in place when the graph keeps its shape).  Passes with a host decision inside
 * (barostat attempts, gradient clipping), with the enthalpy term or with kernel timing on run
 * as plain launches.  Results are the same bits either way.  enable = 0 (the default) turns
 * it off.  revsim_graph_stats: captures and replays so far. */
int32_t revsim_set_graph_mode(revsim_handle *h, int32_t enable);
int32_t revsim_graph_stats(const revsim_handle *h, int64_t *captures, int64_t *replays);

/* The learned term's network arithmetic (REVSIM_MLP_FP64 or REVSIM_MLP_BF16_TC); rebuilds the
 * interval table from the current parameters.  REVSIM_ERR_STATE on a handle without the term. */
int32_t revsim_set_mlp_precision(revsim_handle *h, int32_t mode);
/* The network itself on the tensor cores (split BF16 operands, FP32 accumulation) at n
 * distances per type: r [3][n] nm (O-O, O-H, H-H rows; NULL = the table's nodes k rc / 1024,
 * n = 1025), u [3][n] = MLP(phi(r)) fc(r) and du [3][n] = du/dr (both NULL: not copied back),
 * ms (may be NULL) = the device time of the evaluation kernel.  For tests and for timing a
 * per-pair evaluation against the table. */
int32_t revsim_mlp_eval(revsim_handle *h, int32_t n, const double *r, double *u, double *du, double *ms);

/* Pair evaluation of the mixed-precision step kernels.  REVSIM_PAIRS_BOTH_SIDES (default):
 * each molecule's lanes evaluate its whole neighbour row, so every unordered pair is
 * evaluated twice and each molecule's forces are summed by its own lanes in one fused
 * kernel.  REVSIM_PAIRS_HALF_SHELL: each pair is evaluated once, by one of its molecules
 * (I when I + J is odd and I < J, or even and I > J), which writes the partner's share to a
 * slot; a second kernel per step sums each molecule's slots in row order (deterministic,
 * forward and reverse forces the same bits).  In effect only with FP32 pair arithmetic,
 * boxes above 2 (cutoff + 0.3 nm) + 0.02 nm and no barostat; otherwise the both-sides
 * kernels run.  REVSIM_ERR_STATE for an FP64 handle.  Invalidates the forward record.
 * revsim_get_pair_mode returns the requested mode and the one in effect. */
#define REVSIM_PAIRS_BOTH_SIDES 0
#define REVSIM_PAIRS_HALF_SHELL 1
int32_t revsim_set_pair_mode(revsim_handle *h, int32_t mode);
int32_t revsim_get_pair_mode(const revsim_handle *h, int32_t *requested, int32_t *active);

/* The handle's CUDA stream (a cudaStream_t), for callers that time with events. */
void *revsim_stream(revsim_handle *h);

/* Launch counters: number of engine kernel launches since the handle was created. */
int64_t revsim_launch_count(const revsim_handle *h);

/* Per-kernel timing of the step kernels (which = 0: fused reverse step, 1: fused
 * forward step): when enabled, each launch is bracketed by CUDA events on the handle's
 * stream; the summed milliseconds and the launch count are returned by
 * revsim_kernel_time. */
int32_t revsim_set_kernel_timing(revsim_handle *h, int32_t enable);
int32_t revsim_kernel_time(revsim_handle *h, int32_t which, double *total_ms, int64_t *launches);

/* Block shape of the step kernels (which = 0: reverse step, 1: forward step, -1: both):
 * lanes per molecule (8, 16 or 32), molecules per CTA, and the neighbour loop form
 * (1: one entry per lane per iteration, 2: two, 3: one with the next entry prefetched;
 * 3 allows at most 256 threads per CTA); 0 keeps the current value.  Lanes per molecule are
 * one setting for both kernels whatever `which` says (the order in which a molecule's
 * forces are summed depends on it, and the reverse pass rebuilds the trajectory only when
 * its forces are the forward pass's bits); a count the other kernel's shape does not allow
 * returns REVSIM_ERR_BADARG.  revsim_autotune times the allowed shapes on the current state
 * (CTAs of 64-512 threads, plus the molecule counts that spread the CTAs over every SM in
 * one wave of one or two per SM) and keeps the lane count with the smallest forward +
 * reverse time and, for it, each kernel's fastest shape. */
int32_t revsim_set_launch_shape(revsim_handle *h, int32_t which, int32_t lanes_per_mol,
                                int32_t mols_per_cta, int32_t unroll);
int32_t revsim_get_launch_shape(revsim_handle *h, int32_t which, int32_t *lanes_per_mol,
                                int32_t *mols_per_cta, int32_t *unroll);
int32_t revsim_autotune(revsim_handle *h, double dt);

/* Allocation-free loss and dL/dx for one water box, for callers that cannot let the
 * library allocate device memory (a host whose pool allocator owns all device
 * memory, a loop that must avoid the synchronisation cudaMalloc implies, a fully
 * pre-budgeted service).  No counterpart in the reference: it is the loss of
 * revsim_loss_grad for one term and one box, computed on caller-owned device
 * buffers: d_x [3 * 3 n_mol] positions (FP64, O H H per molecule), d_target
 * [n_target], outputs d_loss [1] and d_dLdx [3 * 3 n_mol], all on the current device,
 * ordered on `stream` (a cudaStream_t; NULL = legacy default stream).  Its scratch is
 * a fixed array inside the library (grids of at most 8192 points; a larger n_grid
 * returns REVSIM_ERR_BADARG); it calls no cudaMalloc or cudaFree.  The first call on
 * a device looks up that array's device address, so make it before any stream
 * capture; a cudaDeviceReset of that device invalidates the address, so do not call
 * this entry point again in a process that has reset the device.  All calls share the
 * array: calls that overlap on the GPU race.  On an error return the outputs are
 * undefined (they may be partly written). */
int32_t revsim_rdf_loss_grad_noalloc(const double *d_x, int32_t n_mol, double box,
                                     const revsim_rdf_term *term, const double *d_target,
                                     double *d_loss, double *d_dLdx, void *stream);

/* Instrumentation with no counterpart in the reference: the measured FP32 / FP64 fused
 * multiply-add throughput (TFLOP/s, 2 flops per FMA) of a device, the roofline
 * denominators of the FP32-pipe-bound step kernels and of the FP64 gas-in-water kernels. */
int32_t revsim_probe_fp32_tflops(int32_t device, double *tflops);
int32_t revsim_probe_fp64_tflops(int32_t device, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
