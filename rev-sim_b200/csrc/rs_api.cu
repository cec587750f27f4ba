// rs_api.cu -- the C ABI of include/revsim.h: handle, device memory and the
// forward / reverse drivers.
//
// Driver structure (host loop on one CUDA stream, one kernel per MD step):
//   forward_sim  (water.jl:977-1105): per step one fused force+integrate kernel; the
//                neighbour list is rebuilt every n_steps_nf steps and the build
//                positions are kept ("checkpoints"); snapshots of x, v every
//                n_steps_log steps; the loss every n_steps_loss steps.
//   reverse_sim  (water.jl:1435-1558): loss gradient at the end state, then per step
//                one fused kernel (force + VJP + dtheta + un-kick + B/A update + the
//                next step's un-integration); snapshot restores, loss blocks and
//                truncation exactly as the reference orders them.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "revsim.h"
#include "rs_internal.h"

using namespace rs;

namespace {

constexpr double kRext = 0.15;        // bound on intramolecular O-H distance, nm
// Tighter O-H bound under which the row build takes one periodic image per molecule pair
// (boxes above 2 (rc_nl + 2 kRnear) + 0.02 nm); a molecule beyond it sends the build back to
// per-atom-pair images (same rows either way).
constexpr double kRnear = 0.12;
constexpr double kTwoPow1o6 = 1.122462048309373;

int form_nparams(int f) {
    switch (f) {
        case REVSIM_LJ: return 2;
        case REVSIM_DEXP: return 4;
        case REVSIM_BUCK: return 3;
        case REVSIM_LJSC: return 4;
        case REVSIM_BUFF: return 4;
    }
    return -1;
}

struct Term {
    revsim_rdf_term t;
    int off;
    double *d_target = nullptr;   // [R * n_target]
    double *d_hist = nullptr;     // [R * n_grid + R]  (histogram, then pre[R])
    double *d_dLdh = nullptr;     // [R * n_grid]
};

}  // namespace

struct revsim_handle {
    std::string err;
    int dev = 0;
    cudaStream_t st = nullptr;

    int R = 0, M = 0, N = 0;
    std::vector<int> nmol, mol0, atom0;
    std::vector<double> box, temp;
    int form = 0, prec = 0, nl_mode = 0, nf = 20, nlog = 1000;
    double mO = 0, mH = 0, ke = 0, krf = 0, rc = 0, rc_nl = 0, kB = 0;

    std::vector<double> theta;
    int P = 0, NFp = 0;   // classical parameter count (the step kernels' partials)
    int Pt = 0;           // all parameters: classical, then the MLP's when mlp
    bool mlp = false;
    double *d_mlp_theta = nullptr, *d_mlp_adj = nullptr, *d_mlp_scratch = nullptr,
           *d_mlp_grad = nullptr;
    void *d_mlp_tab = nullptr;
    int mlp_mode = 0;           // 0: FP64 network evaluation, 1: BF16 tensor cores (rs_mlp_tc.cu)
    void *d_mlp_tc = nullptr;   // scratch of the tensor-core backward pass
    double *d_mlp_r = nullptr, *d_mlp_u = nullptr;   // revsim_mlp_eval buffers
    size_t mlp_eval_cap = 0;
    double *d_epart = nullptr;   // [M][P + 1] energy-gradient partials
    bool have_params = false, have_state = false;

    // Launch shapes of the step kernels, [0] reverse and [1] forward, each with its own
    // CTA -> (replica, first molecule, molecule count) table.
    struct Shape {
        int G = 32, mpc = 8, U = 1, n_blk = 0;
        int *d_blk_rep = nullptr, *d_blk_mol0 = nullptr, *d_blk_nmol = nullptr;
    } shp[2];
    bool shift_ok = false;   // one periodic image per molecule pair is exact for every box
    int cap = 0;

    // tables
    int *d_mol_rep = nullptr, *d_atom_rep = nullptr, *d_rep_atom0 = nullptr, *d_rep_nmol = nullptr;
    double *d_rep_box = nullptr, *d_rep_sdO = nullptr, *d_rep_sdH = nullptr;
    // cells
    std::vector<int> nc, cell_off;
    int n_cells = 0;
    int *d_rep_nc = nullptr, *d_rep_cell_off = nullptr;
    int *d_cell_of_mol = nullptr, *d_cell_cnt = nullptr, *d_cell_start = nullptr,
        *d_cell_fill = nullptr, *d_cell_tmp = nullptr, *d_cell_sorted = nullptr;
    uint32_t *d_nbr = nullptr;       // working rows [M * cap] (+ the split rows, mixed precision)
    int *d_nbr_cnt = nullptr;        // [M] (+ owned and incoming counts, mixed precision)
    // Half-shell pair evaluation (mixed precision; REVSIM_PAIRS_HALF_SHELL): requested, in
    // effect at the last forward pass, and its scratch (compact owned positions of the split,
    // per-entry partner slots, per-molecule own partials), sized for half_cap
    bool half_req = false, fwd_half = false;
    int *d_ownpos = nullptr;
    float4 *d_slot_f = nullptr;
    float2 *d_slot_g = nullptr;
    float *d_own = nullptr;
    int half_cap = 0;
    int *d_cell_rep = nullptr;
    float band = 2e-5f;
    // rows of every forward build, reused by the reverse pass (checkpoint mode)
    uint32_t *d_nbr_store = nullptr;
    int *d_cnt_store = nullptr;
    size_t store_slots = 0, store_cap = 0;
    // state
    double *d_x = nullptr, *d_v = nullptr, *d_A = nullptr, *d_B = nullptr, *d_C = nullptr,
           *d_D = nullptr, *d_G = nullptr, *d_F = nullptr, *d_x0 = nullptr, *d_v0 = nullptr;
    void *d_pos[2] = {nullptr, nullptr}, *d_wgt[2] = {nullptr, nullptr};
    double *d_part = nullptr, *d_norm2 = nullptr, *d_scale = nullptr;
    std::vector<int> mol_rep_h;     // replica of each molecule (host copy)
    int *d_status = nullptr, *d_maxcnt = nullptr;
    unsigned long long *d_count = nullptr;
    // trajectory store
    double *d_snap_x = nullptr, *d_snap_v = nullptr, *d_ckpt = nullptr;
    size_t snap_cap = 0, snapv_cap = 0, ckpt_cap = 0;
    bool fwd_valid = false;
    int fwd_steps = 0;
    uint64_t *d_seeds = nullptr;
    size_t seeds_cap = 0;
    // caller-supplied noise [n_steps][3N] of the host-noise entry points (use_noise: the
    // running pass reads it instead of drawing Philox noise from the seeds)
    double *d_noise = nullptr;
    size_t noise_cap = 0;
    bool use_noise = false;
    // loss
    std::vector<Term> terms;
    double *d_loss = nullptr, *d_loss_acc = nullptr, *d_dLdx = nullptr;
    // enthalpy-of-vaporisation term: per-replica l_ev sums, 2 e / n, direct dl/dtheta sums
    // [R][P], and the neighbour rows of its energy (built at each loss point)
    bool ev_on = false;
    double ev_ugas = 3.69, ev_rt = 2.45, ev_target = 44.12 + 2.8;
    double *d_ev_acc = nullptr, *d_ev_k = nullptr, *d_ev_grad = nullptr;
    uint32_t *d_nbr_ev = nullptr;
    int *d_cnt_ev = nullptr;
    int ev_cap = 0;
    int last_blocks = 1;   // loss points of the last forward / reverse (0: no loss computed)
    // Monte-Carlo barostat (forward passes only): per replica volume_scale, the adaptation
    // window, the draw counter and the accepted total; saved positions and the trial
    // scale / acceptance per replica on the device
    bool baro_on = false, fwd_baro = false;
    revsim_barostat_desc baro{};
    std::vector<double> baro_vs;
    std::vector<long long> baro_att, baro_acc, baro_draws, baro_acc_tot;
    long long baro_step = 0;   // forward steps since the barostat was switched on
    double *d_bx = nullptr, *d_lsc = nullptr, *d_repE = nullptr;
    int *d_bacc = nullptr;
    int cell_cap = 0;   // allocated cells (the cell grid follows the boxes)
    // CUDA-graph mode: each forward / reverse pass is captured once and replayed while its
    // key (pass arguments, the handle's configuration generation `gen` and the allocation
    // counter) is unchanged
    bool graph_on = false;
    bool exact = false;   // the exactly reversible integrator (REVSIM_INTEGRATOR_EXACT)
    unsigned long long gen = 0;
    struct GraphCache {
        std::vector<double> key;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ex = nullptr;
        long long launches = 0;
    } gc[2];
    long long graph_captures = 0, graph_replays = 0;
    // instrumentation
    long long launches = 0;
    bool ktime = false;
    std::vector<cudaEvent_t> ev[2];   // [0] reverse-step kernel, [1] forward-step kernel
    size_t ev_used[2] = {0, 0};
    double kt_ms[2] = {0.0, 0.0};
    long long kt_n[2] = {0, 0};
};

namespace {

int fail(revsim_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(h, REVSIM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Every device allocation or free moves this counter; a captured pass graph holds device
// addresses, so it is replayed only while the counter it was captured at still holds.
std::atomic<unsigned long long> g_alloc_gen{0};

template <typename T>
cudaError_t dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    g_alloc_gen++;
    return cudaMalloc((void **)p, sizeof(T) * n);
}

void dfree(void *p) {
    if (p) {
        g_alloc_gen++;
        cudaFree(p);
    }
}

}  // namespace

namespace rs {

// Constants of one pair form for the per-pair parameters t[0..nfp-1] (the water engine's
// O-O parameters, or the gas engine's mixed parameters of one site class).
template <typename R>
FormConsts<R> form_consts(int form, const double *t, int nfp) {
    FormConsts<R> fc;
    for (int i = 0; i < 4; i++) fc.p[i] = (R)(i < nfp ? t[i] : 0.0);
    for (int i = 0; i < 8; i++) fc.c[i] = (R)0;
    fc.on = 0;
    switch (form) {
        case REVSIM_LJ: {
            const double s = t[0], e = t[1];
            fc.on = e != 0.0;
            fc.c[0] = (R)(s * s);
            fc.c[1] = (R)(24 * e);
            fc.c[2] = (R)(144 * e / s);
            fc.c[3] = (R)(e != 0.0 ? 1.0 / e : 0.0);
            break;
        }
        case REVSIM_BUCK: {
            const double A = t[0], B = t[1], C = t[2];
            fc.on = A != 0.0;
            fc.c[0] = (R)(A * B);
            fc.c[1] = (R)(6 * C);
            fc.c[2] = (R)(A * B * B);
            fc.c[3] = (R)(42 * C);
            break;
        }
        case REVSIM_DEXP: {
            const double s = t[0], e = t[1], al = t[2], be = t[3];
            const double rm = s * kTwoPow1o6;
            fc.on = e != 0.0;
            fc.c[0] = (R)(1.0 / rm);
            fc.c[1] = (R)(e * al * be);
            fc.c[2] = (R)(1.0 / (al - be));
            fc.c[3] = (R)rm;
            fc.c[4] = (R)kTwoPow1o6;
            break;
        }
        case REVSIM_LJSC: {
            const double s = t[0], e = t[1], al = t[2], la = t[3];
            const double s6 = s * s * s * s * s * s;
            const double u = s6 * al * la * la;
            fc.on = e != 0.0;
            fc.c[0] = (R)s6;
            fc.c[1] = (R)u;
            fc.c[2] = (R)(24 * e);
            fc.c[3] = (R)(s6 * s6);
            fc.c[4] = (R)(e != 0.0 ? 1.0 / e : 0.0);
            fc.c[5] = (R)(6 * u / s);
            fc.c[6] = (R)(s6 * la * la);
            fc.c[7] = (R)(2 * s6 * al * la);
            break;
        }
        case REVSIM_BUFF: {
            fc.on = t[1] != 0.0;
            fc.c[0] = (R)kTwoPow1o6;
            break;
        }
    }
    return fc;
}

template FormConsts<float> form_consts<float>(int, const double *, int);
template FormConsts<double> form_consts<double>(int, const double *, int);

}  // namespace rs

namespace {

template <typename R>
NbConsts<R> nb_consts(const revsim_handle *h) {
    const double *t = h->theta.data();
    const int nfp = h->NFp;
    const double qO = t[nfp], qH = -qO / 2;
    NbConsts<R> nb;
    nb.qq[0] = (R)(h->ke * qO * qO);
    nb.qq[1] = (R)(h->ke * qO * qH);
    nb.qq[2] = (R)(h->ke * qH * qH);
    nb.krf = (R)h->krf;
    nb.krf2 = (R)(2 * h->krf);
    nb.rc2 = (R)(h->rc * h->rc);
    nb.twoinvq = (R)(2.0 / qO);
    nb.fc = form_consts<R>(h->form, t, nfp);
    nb.mlp_tab = h->d_mlp_tab;
    nb.mlp_adj = h->d_mlp_adj;
    nb.mlp_hinv = (R)(MLP_NG / h->rc);
    return nb;
}

BondConsts bond_consts(const revsim_handle *h) {
    const double *t = h->theta.data() + h->NFp;
    return BondConsts{t[1], t[2], t[3], t[4]};
}

StepArgs base_args(revsim_handle *h, bool rev) {
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    const revsim_handle::Shape &sh = h->shp[rev ? 0 : 1];
    a.blk_rep = sh.d_blk_rep;
    a.blk_mol0 = sh.d_blk_mol0;
    a.blk_nmol = sh.d_blk_nmol;
    a.rep_box = h->d_rep_box;
    a.rep_sdO = h->d_rep_sdO;
    a.rep_sdH = h->d_rep_sdH;
    a.rep_atom0 = h->d_rep_atom0;
    a.nbr = h->d_nbr;
    a.nbr_cnt = h->d_nbr_cnt;
    a.cap = h->cap;
    a.x = h->d_x;
    a.v = h->d_v;
    a.A = h->d_A;
    a.B = h->d_B;
    a.C = h->d_C;
    a.D = h->d_D;
    a.G = h->d_G;
    a.part = h->d_part;
    a.P = h->P;
    a.status = h->d_status;
    a.mO = h->mO;
    a.mH = h->mH;
    a.exact = h->exact ? 1 : 0;
    return a;
}

int set_cells(revsim_handle *h);

// The exact integrator's grid: box sides and then the state rounded to it (a no-op for a state
// already on it, e.g. the end state of a previous exact pass).
int quantize_for_exact(revsim_handle *h) {
    bool moved = false;
    for (int r = 0; r < h->R; r++) {
        const double q = qgrid(h->box[r]);
        moved = moved || q != h->box[r];
        h->box[r] = q;
    }
    if (moved) {
        CK(cudaMemcpyAsync(h->d_rep_box, h->box.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice, h->st));
        if (int rc = set_cells(h)) return rc;
        h->gen++;
    }
    CK(launch_quantize_state(h->N, h->d_x, h->d_v, h->d_atom_rep, h->d_rep_box, h->st));
    h->launches++;
    return REVSIM_OK;
}

// A row set: the rows [M * cap], then (mixed precision) the split rows [M * cap] of the
// half-shell kernels; counts [M], then (mixed precision) owned [M] and incoming [M] counts.
bool split_rows(const revsim_handle *h) { return h->prec == REVSIM_MIXED; }
size_t rows_set(const revsim_handle *h) { return (size_t)h->M * h->cap * (split_rows(h) ? 2 : 1); }
size_t cnts_set(const revsim_handle *h) { return (size_t)h->M * (split_rows(h) ? 3 : 1); }

// Half-shell pair evaluation in effect: requested, FP32 pair arithmetic, one periodic image
// per molecule pair in every box, and no barostat (whose box moves could end that).
bool half_eff(const revsim_handle *h) { return h->half_req && split_rows(h) && h->shift_ok && !h->baro_on; }

// The step kernels' dtheta partials and |dl_dfi|^2 sums (d_part, d_norm2): one slot per
// molecule for the both-sides kernels, one per CTA of the reverse block table for the
// half-shell kernels.  part_slots: the slots to clear; slot_owner: each slot's replica.
size_t part_slots(const revsim_handle *h) { return std::max((size_t)h->shp[0].n_blk, (size_t)h->M); }

int slot_owner(revsim_handle *h, std::vector<int> &owner) {
    if (!half_eff(h)) {
        owner = h->mol_rep_h;
        return REVSIM_OK;
    }
    owner.resize(h->shp[0].n_blk);
    if (cudaMemcpy(owner.data(), h->shp[0].d_blk_rep, sizeof(int) * owner.size(), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return REVSIM_ERR_CUDA;
    return REVSIM_OK;
}

void free_half(revsim_handle *h) {
    dfree(h->d_ownpos);
    dfree(h->d_slot_f);
    dfree(h->d_slot_g);
    dfree(h->d_own);
    h->d_ownpos = nullptr;
    h->d_slot_f = nullptr;
    h->d_slot_g = nullptr;
    h->d_own = nullptr;
    h->half_cap = 0;
}

int ensure_half(revsim_handle *h) {
    if (h->half_cap == h->cap && h->d_own) return REVSIM_OK;
    free_half(h);
    const size_t mc = (size_t)h->M * h->cap;
    CK(dalloc(&h->d_ownpos, mc));
    CK(dalloc(&h->d_slot_f, 3 * mc));
    CK(dalloc(&h->d_slot_g, 3 * mc));
    CK(dalloc(&h->d_own, (size_t)h->M * 36));
    h->half_cap = h->cap;
    return REVSIM_OK;
}

int launch_step_k(revsim_handle *h, bool rev, const StepArgs &a_in) {
    const revsim_handle::Shape &sh = h->shp[rev ? 0 : 1];
    StepArgs a = a_in;
    a.blk_rep = sh.d_blk_rep;
    a.blk_mol0 = sh.d_blk_mol0;
    a.blk_nmol = sh.d_blk_nmol;
    const int threads = sh.G * sh.mpc;
    const BondConsts bc = bond_consts(h);
    const bool timed = h->ktime && !(a.mode & MODE_FORCES_ONLY);
    const int which = rev ? 0 : 1;
    if (timed) {
        while (h->ev[which].size() < h->ev_used[which] + 2) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            h->ev[which].push_back(e);
        }
        CK(cudaEventRecord(h->ev[which][h->ev_used[which]], h->st));
    }
    cudaError_t e;
    if (half_eff(h)) {
        if (int rc = ensure_half(h)) return rc;
        a.split = a.nbr + (size_t)h->M * h->cap;
        a.cnt_own = a.nbr_cnt + h->M;
        a.cnt_inc = a.nbr_cnt + 2 * (size_t)h->M;
        a.slot_f = h->d_slot_f;
        a.slot_g = h->d_slot_g;
        a.own = h->d_own;
        e = launch_half(rev, h->mlp ? (int)F_LJ_MLP : h->form, sh.G, sh.n_blk, threads, a, nb_consts<float>(h), bc,
                        h->st);
        h->launches++;
    } else if (h->prec == REVSIM_MIXED)
        e = launch_step<float>(rev, h->mlp ? (int)F_LJ_MLP : h->form, sh.G, sh.U, h->shift_ok, sh.n_blk,
                               threads, a, nb_consts<float>(h), bc, h->st);
    else
        e = launch_step<double>(rev, h->mlp ? (int)F_LJ_MLP : h->form, sh.G, sh.U, h->shift_ok, sh.n_blk,
                                threads, a, nb_consts<double>(h), bc, h->st);
    h->launches++;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("step kernel: ") + cudaGetErrorString(e));
    if (timed) {
        CK(cudaEventRecord(h->ev[which][h->ev_used[which] + 1], h->st));
        h->ev_used[which] += 2;
    }
    return REVSIM_OK;
}

// CTA table of one direction (0 reverse, 1 forward): CTAs never straddle replicas, so
// the reverse kernel's per-CTA dtheta partials are per replica.
int build_block_table(revsim_handle *h, int dir) {
    revsim_handle::Shape &sh = h->shp[dir];
    std::vector<int> br, bm, bn;
    for (int r = 0; r < h->R; r++)
        for (int m = 0; m < h->nmol[r]; m += sh.mpc) {
            br.push_back(r);
            bm.push_back(h->mol0[r] + m);
            bn.push_back(std::min(sh.mpc, h->nmol[r] - m));
        }
    sh.n_blk = (int)br.size();
    dfree(sh.d_blk_rep);
    dfree(sh.d_blk_mol0);
    dfree(sh.d_blk_nmol);
    sh.d_blk_rep = sh.d_blk_mol0 = sh.d_blk_nmol = nullptr;
    CK(dalloc(&sh.d_blk_rep, br.size()));
    CK(dalloc(&sh.d_blk_mol0, br.size()));
    CK(dalloc(&sh.d_blk_nmol, br.size()));
    CK(cudaMemcpy(sh.d_blk_rep, br.data(), sizeof(int) * br.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(sh.d_blk_mol0, bm.data(), sizeof(int) * bm.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(sh.d_blk_nmol, bn.data(), sizeof(int) * bn.size(), cudaMemcpyHostToDevice));
    if (dir == 0) {
        dfree(h->d_part);
        dfree(h->d_norm2);
        h->d_part = h->d_norm2 = nullptr;
        // per molecule (both-sides kernels) or per CTA (half-shell kernels)
        const size_t slots = std::max(br.size(), (size_t)h->M);
        CK(dalloc(&h->d_part, slots * (size_t)std::max(h->P, 1)));
        CK(dalloc(&h->d_norm2, slots));
    }
    return REVSIM_OK;
}

int alloc_nbr(revsim_handle *h, int cap) {
    dfree(h->d_nbr);
    h->d_nbr = nullptr;
    dfree(h->d_nbr_store);
    dfree(h->d_cnt_store);
    h->d_nbr_store = nullptr;
    h->d_cnt_store = nullptr;
    h->store_slots = 0;
    free_half(h);
    h->cap = cap;
    CK(dalloc(&h->d_nbr, rows_set(h)));
    return REVSIM_OK;
}

// Rows of every forward build (n slots), kept for the reverse pass when memory allows.
void ensure_list_store(revsim_handle *h, size_t slots) {
    if (slots <= 1) return;
    if (h->d_nbr_store && h->store_slots >= slots && h->store_cap == (size_t)h->cap) return;
    dfree(h->d_nbr_store);
    dfree(h->d_cnt_store);
    h->d_nbr_store = nullptr;
    h->d_cnt_store = nullptr;
    h->store_slots = 0;
    uint32_t *p = nullptr;
    int *c = nullptr;
    if (cudaMalloc((void **)&p, sizeof(uint32_t) * rows_set(h) * slots) != cudaSuccess ||
        cudaMalloc((void **)&c, sizeof(int) * cnts_set(h) * slots) != cudaSuccess) {
        cudaGetLastError();   // clear the failed allocation; fall back to rebuilding
        dfree(p);
        dfree(c);
        return;
    }
    h->d_nbr_store = p;
    h->d_cnt_store = c;
    h->store_slots = slots;
    h->store_cap = h->cap;
}

// Neighbour list from positions xsrc (d_x or a checkpoint) into rows nbr / counts cnt
// (the working list when null).
int build_nlist(revsim_handle *h, const double *xsrc, uint32_t *nbr = nullptr, int *cnt = nullptr) {
    NlistArgs a;
    a.M = h->M;
    a.n_cells = h->n_cells;
    a.x = xsrc;
    a.mol_rep = h->d_mol_rep;
    a.rep_nc = h->d_rep_nc;
    a.rep_cell_off = h->d_rep_cell_off;
    a.rep_box = h->d_rep_box;
    a.cell_of_mol = h->d_cell_of_mol;
    a.cell_cnt = h->d_cell_cnt;
    a.cell_start = h->d_cell_start;
    a.cell_fill = h->d_cell_fill;
    a.cell_tmp = h->d_cell_tmp;
    a.cell_sorted = h->d_cell_sorted;
    a.nbr = nbr ? nbr : h->d_nbr;
    a.nbr_cnt = cnt ? cnt : h->d_nbr_cnt;
    a.cap = h->cap;
    a.cell_rep = h->d_cell_rep;
    a.band = h->band;
    a.rc_nl2 = h->rc_nl * h->rc_nl;
    const double rcand = h->rc_nl + 2 * kRext;
    a.rcand2 = rcand * rcand;
    a.rext2 = kRext * kRext;
    a.rnear2 = kRnear * kRnear;
    a.rcand_near2 = (h->rc_nl + 2 * kRnear) * (h->rc_nl + 2 * kRnear);
    a.shift_box = 2 * (h->rc_nl + 2 * kRnear) + 0.02;
    a.status = h->d_status;
    a.max_cnt = h->d_maxcnt;
    a.split = nullptr;
    a.cnt_own = a.cnt_inc = a.ownpos = nullptr;
    if (half_eff(h)) {
        if (int rc = ensure_half(h)) return rc;
        a.split = a.nbr + (size_t)h->M * h->cap;
        a.cnt_own = a.nbr_cnt + h->M;
        a.cnt_inc = a.nbr_cnt + 2 * (size_t)h->M;
        a.ownpos = h->d_ownpos;
    }
    int nk = 0;
    cudaError_t e = launch_nlist(a, h->st, &nk);
    h->launches += nk;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("nlist: ") + cudaGetErrorString(e));
    return REVSIM_OK;
}

int read_status(revsim_handle *h, int *flags) {
    int s = 0;
    CK(cudaMemcpyAsync(&s, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->st));
    *flags = s;
    return REVSIM_OK;
}

int status_code(revsim_handle *h, int s) {
    if (s & ST_NLIST_OVERFLOW) return fail(h, REVSIM_ERR_NLIST_OVERFLOW, "neighbour row capacity exceeded");
    if (s & ST_GEOMETRY)
        return fail(h, REVSIM_ERR_GEOMETRY, "an O-H distance exceeds the 0.15 nm molecule bound");
    if (s & ST_NAN) return fail(h, REVSIM_ERR_NAN, "non-finite force");
    if (s & ST_ROW_ASYM) return fail(h, REVSIM_ERR_STATE, "neighbour rows are not symmetric (half-shell split)");
    return REVSIM_OK;
}

// Grow the row capacity from the largest row seen (after a synchronising read).
int grow_cap(revsim_handle *h) {
    int mx = 0;
    CK(cudaMemcpy(&mx, h->d_maxcnt, sizeof(int), cudaMemcpyDeviceToHost));
    int ncap = std::max(h->cap * 5 / 4, (mx * 5 / 4 + 31) / 32 * 32);
    return alloc_nbr(h, ncap);
}

// Build at the current positions and make sure the rows fit.
int build_nlist_checked(revsim_handle *h, const double *xsrc) {
    for (int attempt = 0; attempt < 4; attempt++) {
        int rc = build_nlist(h, xsrc);
        if (rc) return rc;
        int s;
        rc = read_status(h, &s);
        if (rc) return rc;
        if (!(s & ST_NLIST_OVERFLOW)) return status_code(h, s);
        rc = grow_cap(h);
        if (rc) return rc;
    }
    return fail(h, REVSIM_ERR_NLIST_OVERFLOW, "neighbour rows keep overflowing");
}

int pack(revsim_handle *h, int buf, bool with_w) {
    cudaError_t e = launch_pack(h->N, h->prec, h->d_x, with_w ? h->d_C : nullptr, h->mO, h->mH,
                                h->d_atom_rep, h->d_rep_box, h->d_pos[buf], h->d_wgt[buf], h->st);
    h->launches++;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("pack: ") + cudaGetErrorString(e));
    return REVSIM_OK;
}

EnergyArgs energy_args(revsim_handle *h, const uint32_t *nbr, const int *cnt) {
    EnergyArgs a;
    std::memset(&a, 0, sizeof(a));
    a.M = h->M;
    a.P = h->P;
    a.cap = h->cap;
    a.x = h->d_x;
    a.mol_rep = h->d_mol_rep;
    a.rep_box = h->d_rep_box;
    a.nbr = nbr;
    a.nbr_cnt = cnt;
    a.rc2 = h->rc * h->rc;
    a.ke = h->ke;
    a.krf = h->krf;
    a.crf_shift = 1.0 / h->rc + h->krf * h->rc * h->rc;
    const double *t = h->theta.data();
    a.qO = t[h->NFp];
    a.kb = t[h->NFp + 1];
    a.r0 = t[h->NFp + 2];
    a.ka = t[h->NFp + 3];
    a.th0 = t[h->NFp + 4];
    for (int k = 0; k < 4; k++) a.form_p[k] = k < h->NFp ? t[k] : 0.0;
    a.mlp_tab = h->d_mlp_tab;
    a.mlp_hinv = MLP_NG / h->rc;
    a.part = h->d_epart;
    a.grads = 1;
    a.adj_mul = 1.0;
    return a;
}

// The enthalpy-of-vaporisation term at the current positions (enthalpy_vaporization and
// loss_enth_vap, water.jl:738-755): adds l_ev to acc and d_ev_acc; with grad_p adds the
// direct -(2 e / n) dU/dtheta to d_ev_grad (classical) and d_mlp_adj (MLP coefficient
// adjoints); with grad_x adds (2 e / n) F to d_dLdx.  U sums over rows built here from the
// current positions, as the reference's find_neighbors does (water.jl:743).
int enth_dev(revsim_handle *h, double *acc, double *ev_acc, bool grad_x, bool grad_p) {
    if (h->ev_cap != h->cap) {
        dfree(h->d_nbr_ev);
        dfree(h->d_cnt_ev);
        h->d_nbr_ev = nullptr;
        h->d_cnt_ev = nullptr;
        h->ev_cap = 0;
        CK(dalloc(&h->d_nbr_ev, rows_set(h)));
        CK(dalloc(&h->d_cnt_ev, cnts_set(h)));
        h->ev_cap = h->cap;
    }
    if (!h->d_epart) CK(dalloc(&h->d_epart, (size_t)h->M * (h->P + 1)));
    int rc = build_nlist(h, h->d_x, h->d_nbr_ev, h->d_cnt_ev);
    if (rc) return rc;
    const int form = h->mlp ? (int)F_LJ_MLP : h->form;
    EnergyArgs a = energy_args(h, h->d_nbr_ev, h->d_cnt_ev);
    a.grads = grad_p ? 1 : 0;
    CK(launch_energy_grads(form, h->prec, a, h->st));
    EnthArgs f;
    f.R = h->R;
    f.P = h->P;
    f.grads = grad_p ? 1 : 0;
    f.rep_atom0 = h->d_rep_atom0;
    f.rep_nmol = h->d_rep_nmol;
    f.part = h->d_epart;
    f.u_gas = h->ev_ugas;
    f.rt = h->ev_rt;
    f.target = h->ev_target;
    f.acc = acc;
    f.ev_acc = ev_acc;
    f.k = h->d_ev_k;
    f.dgrad = h->d_ev_grad;
    CK(launch_enth_finalize(f, h->st));
    h->launches += 2;
    if (grad_p && h->mlp) {
        // dU/dcoef scaled per replica by -(2 e / n) into the MLP coefficient adjoints
        a.grads = 0;
        a.mlp_adj = h->d_mlp_adj;
        a.adj_scale = h->d_ev_k;
        a.adj_mul = -1.0;
        CK(launch_energy_grads(form, h->prec, a, h->st));
        h->launches++;
    }
    if (grad_x) {
        if ((rc = pack(h, 0, false))) return rc;
        StepArgs s = base_args(h, false);
        s.nbr = h->d_nbr_ev;
        s.nbr_cnt = h->d_cnt_ev;
        s.cap = h->cap;
        s.pos_in = h->d_pos[0];
        s.F_out = h->d_F;
        s.mode = MODE_FORCES_ONLY;
        if ((rc = launch_step_k(h, false, s))) return rc;
        CK(launch_enth_dldx(h->N, h->d_atom_rep, h->d_ev_k, h->d_F, h->d_dLdx, h->st));
        h->launches++;
    }
    return REVSIM_OK;
}

// loss_fn / loss_and_grads at the current positions: adds the per-replica loss to acc
// (device [R]) and the enthalpy part to ev_acc (may be null); if grad writes dL/dx into
// d_dLdx; if grad_p adds the enthalpy term's direct parameter gradient to d_ev_grad /
// d_mlp_adj.
int loss_dev(revsim_handle *h, bool grad, double *acc, double *ev_acc = nullptr, bool grad_p = false) {
    if (grad) CK(cudaMemsetAsync(h->d_dLdx, 0, sizeof(double) * 3 * (size_t)h->N, h->st));
    for (Term &T : h->terms) {
        const revsim_rdf_term &t = T.t;
        RdfArgs a;
        a.x = h->d_x;
        a.rep_atom0 = h->d_rep_atom0;
        a.rep_nmol = h->d_rep_nmol;
        a.rep_box = h->d_rep_box;
        a.sel1 = t.sel1;
        a.sel2 = t.sel2;
        a.x_min = t.x_min;
        a.step = t.step;
        a.width = t.width;
        a.cutoff = t.exp_cutoff;
        a.n_grid = t.n_grid;
        a.off = T.off;
        a.hist = T.d_hist;
        a.dLdh = T.d_dLdh;
        a.dLdx = h->d_dLdx;
        int mx = *std::max_element(h->nmol.begin(), h->nmol.end());
        const int n1 = t.sel1 == 0 ? mx : 2 * mx, n2 = t.sel2 == 0 ? mx : 2 * mx;
        CK(cudaMemsetAsync(T.d_hist, 0, sizeof(double) * (size_t)h->R * t.n_grid, h->st));
        CK(launch_rdf(a, h->R, n1, n2, false, h->st));
        CK(launch_rdf_finalize(a, h->R, T.d_hist + (size_t)h->R * t.n_grid, T.d_target, t.slice_start,
                               t.slice_stride, t.n_target, t.norm, t.weight, acc, T.d_dLdh, h->st));
        h->launches += 2;
        if (grad) {
            CK(launch_rdf(a, h->R, n1, n2, true, h->st));
            h->launches++;
        }
    }
    if (h->ev_on) return enth_dev(h, acc, ev_acc, grad, grad_p);
    return REVSIM_OK;
}

bool has_loss(const revsim_handle *h) { return !h->terms.empty() || h->ev_on; }

int upload_seeds(revsim_handle *h, const uint64_t *seeds, size_t n) {
    if (n > h->seeds_cap) {
        dfree(h->d_seeds);
        h->d_seeds = nullptr;
        CK(dalloc(&h->d_seeds, n));
        h->seeds_cap = n;
    }
    if (n) CK(cudaMemcpyAsync(h->d_seeds, seeds, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, h->st));
    return REVSIM_OK;
}

int ensure_store(revsim_handle *h, double **p, size_t *cap, size_t n) {
    if (n > *cap) {
        dfree(*p);
        *p = nullptr;
        CK(dalloc(p, n));
        *cap = n;
    }
    return REVSIM_OK;
}

int check_ready(revsim_handle *h) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!h->have_params) return fail(h, REVSIM_ERR_STATE, "parameters not set");
    if (!h->have_state) return fail(h, REVSIM_ERR_STATE, "state not set");
    CK(cudaSetDevice(h->dev));
    return REVSIM_OK;
}

// Cell grid of every replica from its current box (cells of side >= half the candidate
// distance, at most 64 per side), the one-image rule and the FP32 row band; the cell arrays
// grow when a box does.
int set_cells(revsim_handle *h) {
    const double rcand = h->rc_nl + 2 * kRext;
    std::vector<int> nc(h->R), coff(h->R);
    int ncell = 0;
    double lmax = 0;
    h->shift_ok = true;
    for (int r = 0; r < h->R; r++) {
        nc[r] = std::min(64, std::max(1, (int)std::floor(h->box[r] / (rcand / 2))));
        coff[r] = ncell;
        ncell += nc[r] * nc[r] * nc[r];
        lmax = std::max(lmax, h->box[r]);
        if (!(h->box[r] > 2 * (h->rc + 2 * kRext) + 0.02)) h->shift_ok = false;
    }
    h->band = (float)(2e-5 * std::max(1.0, lmax / 4.0));
    if (nc == h->nc) return REVSIM_OK;
    h->gen++;
    if (ncell > h->cell_cap) {
        int **arrs[] = {&h->d_cell_cnt, &h->d_cell_start, &h->d_cell_fill, &h->d_cell_rep};
        for (int **a : arrs) {
            dfree(*a);
            *a = nullptr;
        }
        h->cell_cap = 0;
        for (int **a : arrs) CK(dalloc(a, ncell));
        h->cell_cap = ncell;
    }
    std::vector<int> cell_rep(ncell);
    for (int r = 0; r < h->R; r++)
        for (int c = 0; c < nc[r] * nc[r] * nc[r]; c++) cell_rep[coff[r] + c] = r;
    CK(cudaMemcpyAsync(h->d_rep_nc, nc.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_rep_cell_off, coff.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_cell_rep, cell_rep.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->nc = nc;
    h->cell_off = coff;
    h->n_cells = ncell;
    return REVSIM_OK;
}

// Potential energy per replica (FP64 kernel over the given rows, per-replica tree sums).
int replica_energies(revsim_handle *h, const uint32_t *nbr, const int *cnt, std::vector<double> &E) {
    if (!h->d_epart) CK(dalloc(&h->d_epart, (size_t)h->M * (h->P + 1)));
    EnergyArgs a = energy_args(h, nbr, cnt);
    a.grads = 0;
    CK(launch_energy_grads(h->mlp ? (int)F_LJ_MLP : h->form, h->prec, a, h->st));
    CK(launch_rep_energy(h->R, h->d_rep_atom0, h->d_rep_nmol, h->d_epart, h->P, h->d_repE, h->st));
    h->launches += 2;
    E.assign(h->R, 0.0);
    CK(cudaMemcpyAsync(E.data(), h->d_repE, sizeof(double) * h->R, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

uint64_t splitmix_draw(uint64_t seed, uint64_t k) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (k + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t seed, uint64_t k) { return (double)(splitmix_draw(seed, k) >> 11) * (1.0 / 9007199254740992.0); }

// One volume move per replica (apply_coupling!, water.jl:820-862) on the current state with
// the current rows; on any acceptance the gather buffer `buf` is repacked and the cell grid
// follows the new boxes.
int baro_attempt(revsim_handle *h, const uint32_t *nbr, const int *cnt, int buf) {
    const int R = h->R;
    const double kBarNa = 0.0602214076;   // 1 bar nm^3 x N_A, kJ/mol
    std::vector<double> E, Et, lsc(R), old(h->box);
    int rc = replica_energies(h, nbr, cnt, E);
    if (rc) return rc;
    std::vector<double> dV(R), u2(R);
    for (int r = 0; r < R; r++) {
        const uint64_t sr = h->baro.seed + (uint64_t)r, k = (uint64_t)h->baro_draws[r]++;
        const double u1 = uniform01(sr, 2 * k);
        u2[r] = uniform01(sr, 2 * k + 1);
        const double V = old[r] * old[r] * old[r];
        dV[r] = h->baro_vs[r] * (2 * u1 - 1);
        lsc[r] = std::cbrt((V + dV[r]) / V);
    }
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_bx, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_lsc, lsc.data(), sizeof(double) * R, cudaMemcpyHostToDevice, h->st));
    CK(launch_baro_scale(h->M, h->d_mol_rep, h->d_rep_box, h->d_lsc, h->d_x, h->st));
    h->launches++;
    std::vector<double> trial(R);
    for (int r = 0; r < R; r++) trial[r] = old[r] * lsc[r];
    CK(cudaMemcpyAsync(h->d_rep_box, trial.data(), sizeof(double) * R, cudaMemcpyHostToDevice, h->st));
    if ((rc = replica_energies(h, nbr, cnt, Et))) return rc;
    std::vector<int> acc(R);
    bool any = false;
    for (int r = 0; r < R; r++) {
        const double kT = h->kB * h->temp[r], V = old[r] * old[r] * old[r];
        const double dW = (Et[r] - E[r]) + h->baro.pressure * kBarNa * dV[r] -
                          h->nmol[r] * kT * std::log((V + dV[r]) / V);
        acc[r] = (dW <= 0.0 || u2[r] < std::exp(-dW / kT)) ? 1 : 0;
        any = any || acc[r];
        h->box[r] = acc[r] ? trial[r] : old[r];
        if (acc[r]) {
            h->baro_acc[r]++;
            h->baro_acc_tot[r]++;
        }
        if (++h->baro_att[r] >= 10) {
            if (h->baro_acc[r] < 0.25 * h->baro_att[r]) {
                h->baro_vs[r] /= h->baro.scale_increment;
                h->baro_att[r] = h->baro_acc[r] = 0;
            } else if (h->baro_acc[r] > 0.75 * h->baro_att[r]) {
                h->baro_vs[r] = std::min(h->baro_vs[r] * h->baro.scale_increment, V * h->baro.max_volume_frac);
                h->baro_att[r] = h->baro_acc[r] = 0;
            }
        }
    }
    CK(cudaMemcpyAsync(h->d_bacc, acc.data(), sizeof(int) * R, cudaMemcpyHostToDevice, h->st));
    CK(launch_baro_restore(h->M, h->d_mol_rep, h->d_bacc, h->d_bx, h->d_x, h->st));
    CK(cudaMemcpyAsync(h->d_rep_box, h->box.data(), sizeof(double) * R, cudaMemcpyHostToDevice, h->st));
    h->launches++;
    if (any) {
        if ((rc = set_cells(h))) return rc;
        if ((rc = pack(h, buf, false))) return rc;
    }
    return REVSIM_OK;
}

int forward_impl(revsim_handle *h, double gamma, int n_steps, int n_steps_loss, double dt, int calc_loss) {
    const double c = std::exp(-gamma * dt), s = std::sqrt(1 - c * c);
    const size_t n3 = 3 * (size_t)h->N;
    const int R = h->R;
    int rc;
    h->fwd_half = half_eff(h);
    if ((rc = pack(h, 0, false))) return rc;
    int cur = 0;
    const bool store = h->d_nbr_store != nullptr;
    uint32_t *nbr = store ? h->d_nbr_store : h->d_nbr;
    int *ncnt = store ? h->d_cnt_store : h->d_nbr_cnt;
    CK(cudaMemcpyAsync(h->d_ckpt, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    if ((rc = build_nlist(h, h->d_x, nbr, ncnt))) return rc;
    CK(cudaMemcpyAsync(h->d_snap_x, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_snap_v, h->d_v, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemsetAsync(h->d_loss_acc, 0, sizeof(double) * R, h->st));
    if (h->ev_on) CK(cudaMemsetAsync(h->d_ev_acc, 0, sizeof(double) * R, h->st));
    StepArgs a = base_args(h, false);
    a.dt = dt;
    a.dtm_O = dt / h->mO;
    a.dtm_H = dt / h->mH;
    a.invm_O = 1.0 / h->mO;
    a.invm_H = 1.0 / h->mH;
    a.c = c;
    a.s = s;
    for (int step = 1; step <= n_steps; step++) {
        a.cap = h->cap;
        a.nbr = nbr;
        a.nbr_cnt = ncnt;
        a.pos_in = h->d_pos[cur];
        a.pos_out = h->d_pos[cur ^ 1];
        a.seed_cur = h->d_seeds + (size_t)(step - 1) * R;
        a.noise_cur = h->use_noise ? h->d_noise + (size_t)(step - 1) * n3 : nullptr;
        if ((rc = launch_step_k(h, false, a))) return rc;
        cur ^= 1;
        if (step % h->nf == 0 && step < n_steps) {
            const size_t k = (size_t)(step / h->nf);
            CK(cudaMemcpyAsync(h->d_ckpt + k * n3, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                               h->st));
            if (store) {
                nbr = h->d_nbr_store + k * rows_set(h);
                ncnt = h->d_cnt_store + k * cnts_set(h);
            }
            if ((rc = build_nlist(h, h->d_x, nbr, ncnt))) return rc;
        }
        if (h->nlog > 0 && step % h->nlog == 0) {
            const size_t si = (size_t)(step / h->nlog) * n3;
            CK(cudaMemcpyAsync(h->d_snap_x + si, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
            CK(cudaMemcpyAsync(h->d_snap_v + si, h->d_v, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
        }
        if (calc_loss && has_loss(h) && step % n_steps_loss == 0)
            if ((rc = loss_dev(h, false, h->d_loss_acc, h->d_ev_acc))) return rc;
        // apply_coupling! (water.jl:1043-1044) after the step's loggers and loss
        if (h->baro_on && ++h->baro_step % h->baro.n_steps == 0)
            if ((rc = baro_attempt(h, nbr, ncnt, cur))) return rc;
    }
    return REVSIM_OK;
}

int mlp_zero_adj(revsim_handle *h) {
    if (!h->mlp || !h->d_mlp_adj) return REVSIM_OK;
    CK(cudaMemsetAsync(h->d_mlp_adj, 0, sizeof(double) * (size_t)h->R * MLP_NCOPY * MLP_NT * MLP_NG * 4, h->st));
    return REVSIM_OK;
}

int reverse_impl(revsim_handle *h, double gamma, int n_steps, int n_steps_loss, int n_steps_trunc,
                 double dt, double clip) {
    const double c = std::exp(-gamma * dt), s = std::sqrt(1 - c * c);
    const size_t n3 = 3 * (size_t)h->N;
    const int R = h->R;
    const bool clipping = std::isfinite(clip);
    int rc;
    // the reverse pass must evaluate pairs as the forward pass did (same force bits)
    if (half_eff(h) != h->fwd_half)
        return fail(h, REVSIM_ERR_STATE, "the pair evaluation mode changed since the forward pass");
    CK(cudaMemsetAsync(h->d_part, 0, sizeof(double) * part_slots(h) * h->P, h->st));
    if (int rc_ = mlp_zero_adj(h)) return rc_;
    CK(cudaMemsetAsync(h->d_loss_acc, 0, sizeof(double) * R, h->st));
    if (h->ev_on) {
        CK(cudaMemsetAsync(h->d_ev_acc, 0, sizeof(double) * R, h->st));
        CK(cudaMemsetAsync(h->d_ev_grad, 0, sizeof(double) * R * h->P, h->st));
    }
    if ((rc = loss_dev(h, true, h->d_loss_acc, h->d_ev_acc, true))) return rc;
    CK(launch_init_adjoint(h->N, h->d_dLdx, c, h->d_A, h->d_B, h->d_C, h->d_D, h->d_G, h->st));
    h->launches++;

    StepArgs a = base_args(h, true);
    a.dt = dt;
    a.dtm_O = dt / h->mO;
    a.dtm_H = dt / h->mH;
    a.invm_O = 1.0 / h->mO;
    a.invm_H = 1.0 / h->mH;
    a.c = c;
    a.s = s;
    const double dt2 = dt * dt;
    a.acoefO = dt2 / (2 * h->mO);
    a.acoefH = dt2 / (2 * h->mH);
    a.norm2 = clipping ? h->d_norm2 : nullptr;

    int cur = 0;
    long group = -1;
    bool pending = true;
    int trunc = 0;
    if (h->nl_mode == REVSIM_NL_RECONSTRUCTED)
        if ((rc = build_nlist(h, h->d_x))) return rc;
    std::vector<double> scale(2 * R);
    for (int step_n = n_steps; step_n >= 1; step_n--) {
        trunc++;
        const bool restore = h->nlog > 0 && (step_n - 1) % h->nlog == 0 && step_n > 1;
        const bool lossb = (step_n - 1) % n_steps_loss == 0 && step_n > 1;
        if (trunc <= n_steps_trunc) {
            const int m = step_n - 1;
            if (pending) {
                StepArgs u = a;
                u.seed_cur = h->d_seeds + (size_t)(step_n - 1) * R;
                u.noise_cur = h->use_noise ? h->d_noise + (size_t)(step_n - 1) * n3 : nullptr;
                u.pos_out = h->d_pos[cur];
                u.wgt_out = h->d_wgt[cur];
                CK(launch_unintegrate(h->M, h->prec, u, h->d_mol_rep, h->st));
                h->launches++;
            }
            if (h->nl_mode == REVSIM_NL_CHECKPOINT) {
                const long g = m / h->nf;
                if (g != group) {
                    if (h->d_nbr_store && (size_t)g < h->store_slots) {
                        a.nbr = h->d_nbr_store + (size_t)g * rows_set(h);
                        a.nbr_cnt = h->d_cnt_store + (size_t)g * cnts_set(h);
                    } else {
                        if ((rc = build_nlist(h, h->d_ckpt + (size_t)g * n3))) return rc;
                        a.nbr = h->d_nbr;
                        a.nbr_cnt = h->d_nbr_cnt;
                    }
                    group = g;
                }
            } else if (step_n % h->nf == 0) {
                if ((rc = build_nlist(h, h->d_x))) return rc;
            }
            const bool next_active = step_n > 1 && trunc + 1 <= n_steps_trunc && !restore && !lossb;
            const bool fuse = next_active && !clipping;
            a.cap = h->cap;
            if (h->nl_mode != REVSIM_NL_CHECKPOINT) {
                a.nbr = h->d_nbr;
                a.nbr_cnt = h->d_nbr_cnt;
            }
            a.pos_in = h->d_pos[cur];
            a.wgt_in = h->d_wgt[cur];
            a.pos_out = h->d_pos[cur ^ 1];
            a.wgt_out = h->d_wgt[cur ^ 1];
            a.seed_next = fuse ? h->d_seeds + (size_t)(step_n - 2) * R : nullptr;
            a.noise_next = fuse && h->use_noise ? h->d_noise + (size_t)(step_n - 2) * n3 : nullptr;
            a.mode = (fuse ? MODE_FUSE_NEXT : 0) | (clipping ? MODE_DEFER_BA : 0);
            if ((rc = launch_step_k(h, true, a))) return rc;
            if (clipping) {
                // Per-replica norm of dl_dfi from the per-slot sums (fixed order).
                std::vector<int> br;
                if ((rc = slot_owner(h, br))) return fail(h, rc, "block table copy failed");
                std::vector<double> n2(br.size());
                CK(cudaMemcpyAsync(n2.data(), h->d_norm2, sizeof(double) * n2.size(), cudaMemcpyDeviceToHost, h->st));
                CK(cudaStreamSynchronize(h->st));
                std::vector<double> acc(R, 0.0);
                for (size_t b = 0; b < br.size(); b++) acc[br[b]] += n2[b];
                for (int r = 0; r < R; r++) {
                    scale[2 * r] = std::sqrt(acc[r]);
                    scale[2 * r + 1] = clip;
                }
                CK(cudaMemcpyAsync(h->d_scale, scale.data(), sizeof(double) * 2 * R, cudaMemcpyHostToDevice, h->st));
                CK(launch_clip_post(h->N, a, h->d_atom_rep, h->d_scale, h->st));
                h->launches++;
            }
            if (fuse) {
                cur ^= 1;
                pending = false;
            } else {
                pending = true;
            }
        }
        if (restore && (trunc <= n_steps_trunc || lossb)) {
            const size_t si = (size_t)((step_n - 1) / h->nlog) * n3;
            CK(cudaMemcpyAsync(h->d_x, h->d_snap_x + si, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
            CK(cudaMemcpyAsync(h->d_v, h->d_snap_v + si, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
            pending = true;
        }
        if (lossb) {
            trunc = 0;
            if ((rc = loss_dev(h, true, h->d_loss_acc, h->d_ev_acc, true))) return rc;
            CK(launch_init_adjoint(h->N, h->d_dLdx, c, h->d_A, h->d_B, h->d_C, h->d_D, h->d_G, h->st));
            h->launches++;
            pending = true;
        }
    }
    return REVSIM_OK;
}

// Fold the per-launch event pairs recorded since the last call into the totals.
int collect_kernel_times(revsim_handle *h) {
    for (int w = 0; w < 2; w++) {
        for (size_t i = 0; i + 1 < h->ev_used[w]; i += 2) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->ev[w][i], h->ev[w][i + 1]));
            h->kt_ms[w] += ms;
            h->kt_n[w]++;
        }
        h->ev_used[w] = 0;
    }
    return REVSIM_OK;
}

// Sum the dtheta partials per replica (FP64, in slot order).
int reduce_part(revsim_handle *h, std::vector<double> &out) {
    std::vector<int> owner;
    if (int rc = slot_owner(h, owner)) return fail(h, rc, "block table copy failed");
    std::vector<double> part(owner.size() * h->P);
    CK(cudaMemcpyAsync(part.data(), h->d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    out.assign((size_t)h->R * h->P, 0.0);
    for (size_t b = 0; b < owner.size(); b++)
        for (int p = 0; p < h->P; p++) out[(size_t)owner[b] * h->P + p] += part[b * h->P + p];
    return REVSIM_OK;
}

void free_all(revsim_handle *h) {
    for (auto &sh : h->shp) {
        dfree(sh.d_blk_rep);
        dfree(sh.d_blk_mol0);
        dfree(sh.d_blk_nmol);
    }
    void *mptrs[] = {h->d_mlp_theta, h->d_mlp_adj, h->d_mlp_scratch, h->d_mlp_grad, h->d_mlp_tab,
                     h->d_epart, h->d_mlp_tc, h->d_mlp_r, h->d_mlp_u};
    for (void *p : mptrs) dfree(p);
    free_half(h);
    void *ptrs[] = {h->d_mol_rep, h->d_atom_rep,
                    h->d_rep_atom0, h->d_rep_nmol, h->d_rep_box, h->d_rep_sdO, h->d_rep_sdH,
                    h->d_rep_nc, h->d_rep_cell_off, h->d_cell_of_mol, h->d_cell_cnt, h->d_cell_start,
                    h->d_cell_fill, h->d_cell_tmp, h->d_cell_sorted, h->d_nbr, h->d_nbr_cnt, h->d_x,
                    h->d_v, h->d_A, h->d_B, h->d_C, h->d_D, h->d_G, h->d_F, h->d_x0, h->d_v0,
                    h->d_pos[0], h->d_pos[1], h->d_wgt[0], h->d_wgt[1], h->d_part, h->d_norm2,
                    h->d_scale, h->d_status, h->d_maxcnt, h->d_count, h->d_snap_x, h->d_snap_v,
                    h->d_ckpt, h->d_seeds, h->d_noise, h->d_loss, h->d_loss_acc, h->d_dLdx,
                    h->d_cell_rep, h->d_nbr_store, h->d_cnt_store, h->d_ev_acc, h->d_ev_k,
                    h->d_ev_grad, h->d_nbr_ev, h->d_cnt_ev, h->d_bx, h->d_lsc, h->d_bacc, h->d_repE};
    for (void *p : ptrs) dfree(p);
    for (Term &T : h->terms) {
        dfree(T.d_target);
        dfree(T.d_hist);
        dfree(T.d_dLdh);
    }
    for (int w = 0; w < 2; w++)
        for (cudaEvent_t e : h->ev[w]) cudaEventDestroy(e);
    for (auto &c : h->gc) {
        if (c.ex) cudaGraphExecDestroy(c.ex);
        if (c.g) cudaGraphDestroy(c.g);
    }
    if (h->st) cudaStreamDestroy(h->st);
}

}  // namespace

extern "C" {

int32_t revsim_create(const revsim_system_desc *d, revsim_handle **out) {
    if (!d || !out) return REVSIM_ERR_BADARG;
    *out = nullptr;
    revsim_handle *h = new (std::nothrow) revsim_handle();
    if (!h) return REVSIM_ERR_NOMEM;
    auto bad = [&](const char *m) {
        delete h;
        (void)m;
        return REVSIM_ERR_BADARG;
    };
    if (d->n_replicas < 1 || !d->n_mol || !d->box || !d->temp) return bad("replicas");
    if (form_nparams(d->inter_type) < 0) return bad("inter_type");
    if (d->precision != REVSIM_FP64 && d->precision != REVSIM_MIXED) return bad("precision");
    if (!(d->m_O > 0 && d->m_H > 0 && d->cutoff > 0 && d->nl_cutoff >= d->cutoff && d->kB > 0))
        return bad("constants");
    if (d->n_steps_nf < 1 || d->n_steps_log < 0) return bad("periods");
    h->R = d->n_replicas;
    long long M = 0;
    for (int r = 0; r < h->R; r++) {
        if (d->n_mol[r] < 1 || !(d->box[r] > 2 * d->nl_cutoff) || !(d->temp[r] >= 0)) return bad("replica");
        h->nmol.push_back(d->n_mol[r]);
        h->mol0.push_back((int)M);
        h->atom0.push_back((int)(3 * M));
        h->box.push_back(d->box[r]);
        h->temp.push_back(d->temp[r]);
        M += d->n_mol[r];
    }
    if (M >= (1LL << 23)) return bad("too many molecules");
    h->M = (int)M;
    h->N = 3 * h->M;
    h->form = d->inter_type;
    h->prec = d->precision;
    h->nl_mode = d->nl_mode;
    h->nf = d->n_steps_nf;
    h->nlog = d->n_steps_log;
    h->mO = d->m_O;
    h->mH = d->m_H;
    h->ke = d->coulomb_const;
    h->krf = d->crf_const;
    h->rc = d->cutoff;
    h->rc_nl = d->nl_cutoff;
    h->kB = d->kB;
    h->dev = d->device;
    h->NFp = form_nparams(h->form);
    h->P = h->NFp + 5;
    h->mlp = d->mlp != 0;
    if (h->mlp && h->form != REVSIM_LJ) return bad("the learned pair correction needs REVSIM_LJ");
    h->Pt = h->P + (h->mlp ? MLP_NPARAMS : 0);
    h->shift_ok = true;
    for (int r = 0; r < h->R; r++)
        if (!(h->box[r] > 2 * (h->rc + 2 * kRext) + 0.02)) h->shift_ok = false;

    if (cudaSetDevice(h->dev) != cudaSuccess || cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return REVSIM_ERR_CUDA;
    }
    auto cfail = [&](const char *what) {
        free_all(h);
        delete h;
        (void)what;
        return REVSIM_ERR_CUDA;
    };
    // replica tables
    const double rcand = h->rc_nl + 2 * kRext;
    std::vector<int> mol_rep(h->M), atom_rep(h->N), rep_nc(h->R), rep_coff(h->R);
    std::vector<double> sdO(h->R), sdH(h->R);
    int ncell = 0, cap = 32;
    for (int r = 0; r < h->R; r++) {
        for (int m = 0; m < h->nmol[r]; m++) mol_rep[h->mol0[r] + m] = r;
        for (int a = 0; a < 3 * h->nmol[r]; a++) atom_rep[h->atom0[r] + a] = r;
        int nc = std::max(1, (int)std::floor(h->box[r] / (rcand / 2)));
        nc = std::min(nc, 64);
        rep_nc[r] = nc;
        rep_coff[r] = ncell;
        ncell += nc * nc * nc;
        sdO[r] = std::sqrt(h->kB * h->temp[r] / h->mO);
        sdH[r] = std::sqrt(h->kB * h->temp[r] / h->mH);
        const double rho = h->nmol[r] / (h->box[r] * h->box[r] * h->box[r]);
        const double rr = h->rc_nl + 0.25;
        const double expect = 4.0 / 3.0 * 3.14159265358979 * rr * rr * rr * rho;
        cap = std::max(cap, (int)((expect * 1.5 + 32 + 31) / 32) * 32);
    }
    cap = std::min(cap, h->M);
    cap = std::max(cap, 32);
    h->nc = rep_nc;
    h->cell_off = rep_coff;
    h->n_cells = ncell;
    h->cell_cap = ncell;
    std::vector<int> cell_rep(ncell);
    double lmax = 0;
    for (int r = 0; r < h->R; r++) {
        for (int c = 0; c < rep_nc[r] * rep_nc[r] * rep_nc[r]; c++) cell_rep[rep_coff[r] + c] = r;
        lmax = std::max(lmax, h->box[r]);
    }
    // FP32 coordinates of a box of side L round to within L * 2^-24; the FP32 distance^2
    // near the 1.2 nm cutoff is then within ~6e-6 (L/8) of the FP64 value.
    h->band = (float)(2e-5 * std::max(1.0, lmax / 4.0));
    const size_t n3 = 3 * (size_t)h->N;
    const size_t v4 = h->prec == REVSIM_MIXED ? sizeof(float4) : sizeof(double4);
    h->mol_rep_h = mol_rep;
    bool ok = dalloc(&h->d_mol_rep, h->M) == cudaSuccess && dalloc(&h->d_atom_rep, h->N) == cudaSuccess &&
              dalloc(&h->d_rep_atom0, h->R) == cudaSuccess && dalloc(&h->d_rep_nmol, h->R) == cudaSuccess &&
              dalloc(&h->d_rep_box, h->R) == cudaSuccess && dalloc(&h->d_rep_sdO, h->R) == cudaSuccess &&
              dalloc(&h->d_rep_sdH, h->R) == cudaSuccess && dalloc(&h->d_rep_nc, h->R) == cudaSuccess &&
              dalloc(&h->d_rep_cell_off, h->R) == cudaSuccess &&
              dalloc(&h->d_cell_of_mol, h->M) == cudaSuccess && dalloc(&h->d_cell_cnt, ncell) == cudaSuccess &&
              dalloc(&h->d_cell_start, ncell) == cudaSuccess && dalloc(&h->d_cell_fill, ncell) == cudaSuccess &&
              dalloc(&h->d_cell_tmp, h->M) == cudaSuccess && dalloc(&h->d_cell_sorted, h->M) == cudaSuccess &&
              dalloc(&h->d_nbr_cnt, cnts_set(h)) == cudaSuccess && dalloc(&h->d_x, n3) == cudaSuccess &&
              dalloc(&h->d_v, n3) == cudaSuccess && dalloc(&h->d_A, n3) == cudaSuccess &&
              dalloc(&h->d_B, n3) == cudaSuccess && dalloc(&h->d_C, n3) == cudaSuccess &&
              dalloc(&h->d_D, n3) == cudaSuccess && dalloc(&h->d_G, n3) == cudaSuccess &&
              dalloc(&h->d_F, n3) == cudaSuccess && dalloc(&h->d_x0, n3) == cudaSuccess &&
              dalloc(&h->d_v0, n3) == cudaSuccess && dalloc(&h->d_dLdx, n3) == cudaSuccess &&
              cudaMalloc(&h->d_pos[0], v4 * h->N) == cudaSuccess && cudaMalloc(&h->d_pos[1], v4 * h->N) == cudaSuccess &&
              cudaMalloc(&h->d_wgt[0], v4 * h->N) == cudaSuccess && cudaMalloc(&h->d_wgt[1], v4 * h->N) == cudaSuccess &&
              dalloc(&h->d_scale, 2 * h->R) == cudaSuccess && dalloc(&h->d_status, 1) == cudaSuccess &&
              dalloc(&h->d_maxcnt, 2) == cudaSuccess && dalloc(&h->d_count, 1) == cudaSuccess &&
              dalloc(&h->d_loss, h->R) == cudaSuccess && dalloc(&h->d_loss_acc, h->R) == cudaSuccess &&
              dalloc(&h->d_cell_rep, ncell) == cudaSuccess;
    if (!ok) return cfail("alloc");
    std::vector<int> rep_nmol(h->nmol.begin(), h->nmol.end());
    ok = cudaMemcpy(h->d_mol_rep, mol_rep.data(), sizeof(int) * h->M, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_atom_rep, atom_rep.data(), sizeof(int) * h->N, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_atom0, h->atom0.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_nmol, rep_nmol.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_box, h->box.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_sdO, sdO.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_sdH, sdH.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_nc, rep_nc.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_rep_cell_off, rep_coff.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->d_cell_rep, cell_rep.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(h->d_status, 0, sizeof(int)) == cudaSuccess && cudaMemset(h->d_maxcnt, 0, 2 * sizeof(int)) == cudaSuccess &&
         cudaMemset(h->d_C, 0, sizeof(double) * n3) == cudaSuccess &&
         cudaMemset(h->d_A, 0, sizeof(double) * n3) == cudaSuccess;
    if (!ok) return cfail("upload");
    if (build_block_table(h, 0) != REVSIM_OK || build_block_table(h, 1) != REVSIM_OK ||
        alloc_nbr(h, cap) != REVSIM_OK)
        return cfail("tables");
    *out = h;
    return REVSIM_OK;
}

void revsim_destroy(revsim_handle *h) {
    if (!h) return;
    cudaSetDevice(h->dev);
    if (h->st) cudaStreamSynchronize(h->st);
    free_all(h);
    delete h;
}

const char *revsim_last_error(const revsim_handle *h) { return h ? h->err.c_str() : "null handle"; }

int32_t revsim_device_status(revsim_handle *h, int32_t *flags) {
    if (!h || !flags) return REVSIM_ERR_BADARG;
    int s = 0;
    int rc = read_status(h, &s);
    *flags = s;
    return rc;
}

int32_t revsim_sizes(const revsim_handle *h, int64_t *n_atoms, int32_t *n_params) {
    if (!h) return REVSIM_ERR_BADARG;
    if (n_atoms) *n_atoms = h->N;
    if (n_params) *n_params = h->Pt;
    return REVSIM_OK;
}

namespace {
// Upload the MLP parameters and rebuild the interval table.
// The interval table from the device copy of the MLP parameters, in the handle's network
// precision (FP64 scalar kernels, or BF16 tensor cores with FP32 accumulation).
int build_mlp_table(revsim_handle *h) {
    cudaError_t e;
    if (h->mlp_mode == 1) {
        e = launch_mlp_tc_eval(h->d_mlp_theta, MLP_NT, h->rc, MLP_WIDTH, MLP_NG + 1, nullptr,
                               mlp_scratch_nodes(h->d_mlp_scratch, 0), mlp_scratch_nodes(h->d_mlp_scratch, 1), h->st);
        if (e == cudaSuccess) e = launch_mlp_table_from_nodes(h->prec, h->d_mlp_scratch, h->rc, h->d_mlp_tab, h->st);
    } else {
        e = launch_mlp_table(h->prec, h->d_mlp_theta, h->rc, h->d_mlp_scratch, h->d_mlp_tab, h->st);
    }
    h->launches += 2;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("MLP table: ") + cudaGetErrorString(e));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int set_mlp(revsim_handle *h, const double *theta_mlp) {
    const size_t adj = (size_t)h->R * MLP_NCOPY * MLP_NT * MLP_NG * 4;
    if (!h->d_mlp_theta) {
        CK(dalloc(&h->d_mlp_theta, MLP_NPARAMS));
        CK(dalloc(&h->d_mlp_adj, adj));
        CK(dalloc(&h->d_mlp_scratch, mlp_scratch_doubles()));
        CK(dalloc(&h->d_mlp_grad, (size_t)h->R * MLP_NPARAMS));
        CK(dalloc((double **)&h->d_mlp_tab, (size_t)MLP_NT * MLP_NG * 4));
        CK(cudaMemset(h->d_mlp_adj, 0, sizeof(double) * adj));
    }
    CK(cudaMemcpyAsync(h->d_mlp_theta, theta_mlp, sizeof(double) * MLP_NPARAMS, cudaMemcpyHostToDevice, h->st));
    return build_mlp_table(h);
}

// The accumulated interval-coefficient adjoints of every replica -> dtheta_mlp [R][MLP_NPARAMS].
int mlp_grads(revsim_handle *h, std::vector<double> &out) {
    for (int r = 0; r < h->R; r++) {
        const double *cadj = h->d_mlp_adj + (size_t)r * MLP_NCOPY * MLP_NT * MLP_NG * 4;
        double *grad = h->d_mlp_grad + (size_t)r * MLP_NPARAMS;
        cudaError_t e;
        if (h->mlp_mode == 1) {
            e = launch_mlp_node_adjoints(cadj, MLP_NCOPY, h->rc, h->d_mlp_scratch, h->st);
            if (e == cudaSuccess)
                e = launch_mlp_tc_backprop(h->d_mlp_theta, MLP_NT, h->rc, MLP_WIDTH,
                                           mlp_scratch_nodes(h->d_mlp_scratch, 2),
                                           mlp_scratch_nodes(h->d_mlp_scratch, 3), h->d_mlp_tc, grad, h->st);
            h->launches += 4;
        } else {
            e = launch_mlp_backprop(h->d_mlp_theta, h->rc, cadj, MLP_NCOPY, h->d_mlp_scratch, grad, h->st);
            h->launches += 3;
        }
        if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("MLP backprop: ") + cudaGetErrorString(e));
    }
    out.resize((size_t)h->R * MLP_NPARAMS);
    CK(cudaMemcpyAsync(out.data(), h->d_mlp_grad, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

// Classical sums [R][P] and MLP gradients [R][MLP_NPARAMS] -> out [R][Pt], times scale.
void join_grads(const revsim_handle *h, const std::vector<double> &cl, const std::vector<double> &ml,
                double scale, double *out) {
    for (int r = 0; r < h->R; r++) {
        for (int p = 0; p < h->P; p++) out[(size_t)r * h->Pt + p] = cl[(size_t)r * h->P + p] * scale;
        if (h->mlp)
            for (int p = 0; p < MLP_NPARAMS; p++)
                out[(size_t)r * h->Pt + h->P + p] = ml[(size_t)r * MLP_NPARAMS + p] * scale;
    }
}
}  // namespace

int32_t revsim_set_params(revsim_handle *h, const double *theta, int32_t n) {
    if (!h || !theta) return REVSIM_ERR_BADARG;
    if (n != h->Pt) return fail(h, REVSIM_ERR_BADARG, "wrong parameter count");
    for (int i = 0; i < n; i++)
        if (!std::isfinite(theta[i])) return fail(h, REVSIM_ERR_BADARG, "non-finite parameter");
    if (theta[h->NFp] == 0.0) return fail(h, REVSIM_ERR_BADARG, "q_O must be non-zero");
    if (h->mlp) {
        CK(cudaSetDevice(h->dev));
        int rc = set_mlp(h, theta + h->P);
        if (rc) return rc;
    }
    // the classical parameters are kernel arguments: a captured graph holds them
    if (!h->have_params || !std::equal(h->theta.begin(), h->theta.end(), theta)) h->gen++;
    h->theta.assign(theta, theta + h->P);
    h->have_params = true;
    return REVSIM_OK;
}

int32_t revsim_set_state(revsim_handle *h, const double *x, const double *v) {
    if (!h || !x || !v) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_x, x, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v, v, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->have_state = true;
    return REVSIM_OK;
}

int32_t revsim_get_state(revsim_handle *h, double *x, double *v) {
    if (!h) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N;
    if (x) CK(cudaMemcpyAsync(x, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->st));
    if (v) CK(cudaMemcpyAsync(v, h->d_v, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int32_t revsim_set_loss(revsim_handle *h, int32_t n_terms, const revsim_rdf_term *terms,
                        const double *const *targets) {
    if (!h || n_terms < 0 || (n_terms > 0 && (!terms || !targets))) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    for (Term &T : h->terms) {
        dfree(T.d_target);
        dfree(T.d_hist);
        dfree(T.d_dLdh);
    }
    h->terms.clear();
    for (int i = 0; i < n_terms; i++) {
        const revsim_rdf_term &t = terms[i];
        if (t.n_grid < 1 || !(t.step > 0) || !(t.width > 0) || !(t.exp_cutoff >= 0) || t.n_target < 0 ||
            t.slice_start < 0 || (t.n_target > 0 && (t.slice_stride < 1 ||
                                                     t.slice_start + (long long)(t.n_target - 1) * t.slice_stride >= t.n_grid)) ||
            (t.norm != 1 && t.norm != 2) || (t.sel1 != 0 && t.sel1 != 1) || (t.sel2 != 0 && t.sel2 != 1) ||
            !targets[i])
            return fail(h, REVSIM_ERR_BADARG, "bad loss term");
        const double q = t.x_min / t.step;
        if (std::fabs(q - std::llround(q)) > 1e-6)
            return fail(h, REVSIM_ERR_BADARG, "x_min must be a multiple of step (water.jl:660)");
        if (!rdf_term_recurrence_ok(t.step, t.width, t.exp_cutoff))
            return fail(h, REVSIM_ERR_BADARG, "width too small for the grid step and window");
        Term T;
        T.t = t;
        T.off = (int)std::llround(q) - 1;
        if (dalloc(&T.d_target, (size_t)h->R * std::max(t.n_target, 1)) != cudaSuccess ||
            dalloc(&T.d_hist, (size_t)h->R * t.n_grid + h->R) != cudaSuccess ||
            dalloc(&T.d_dLdh, (size_t)h->R * t.n_grid) != cudaSuccess) {
            dfree(T.d_target);
            dfree(T.d_hist);
            dfree(T.d_dLdh);
            return fail(h, REVSIM_ERR_NOMEM, "loss buffers");
        }
        h->terms.push_back(T);
        if (t.n_target > 0)
            CK(cudaMemcpy(T.d_target, targets[i], sizeof(double) * (size_t)h->R * t.n_target, cudaMemcpyHostToDevice));
        std::vector<double> pre(h->R);
        for (int r = 0; r < h->R; r++) {
            const double n1 = t.sel1 == 0 ? h->nmol[r] : 2.0 * h->nmol[r];
            const double n2 = t.sel2 == 0 ? h->nmol[r] : 2.0 * h->nmol[r];
            const double V = h->box[r] * h->box[r] * h->box[r];
            pre[r] = V / (4 * 3.14159265358979323846 * n1 * n2 * t.step);
        }
        CK(cudaMemcpy(T.d_hist + (size_t)h->R * t.n_grid, pre.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice));
    }
    return REVSIM_OK;
}

int32_t revsim_neighbor_pairs(revsim_handle *h, int32_t replica, int32_t *pairs, int64_t cap,
                              int64_t *count) {
    if (!h || !count || replica < 0 || replica >= h->R || cap < 0 || (cap > 0 && !pairs)) return REVSIM_ERR_BADARG;
    if (!h->have_state) return fail(h, REVSIM_ERR_STATE, "state not set");
    CK(cudaSetDevice(h->dev));
    int rc = build_nlist_checked(h, h->d_x);
    if (rc) return rc;
    int32_t *d_pairs = nullptr;
    CK(dalloc(&d_pairs, 2 * (size_t)std::max<int64_t>(cap, 1)));
    CK(cudaMemsetAsync(h->d_count, 0, sizeof(unsigned long long), h->st));
    cudaError_t e = launch_export_pairs(h->d_nbr, h->d_nbr_cnt, h->cap, h->mol0[replica], h->nmol[replica],
                                        d_pairs, h->d_count, cap, h->st);
    h->launches++;
    unsigned long long n = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n, h->d_count, sizeof(n), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    const int64_t w = std::min<int64_t>((int64_t)n, cap);
    if (e == cudaSuccess && w > 0) e = cudaMemcpy(pairs, d_pairs, sizeof(int32_t) * 2 * w, cudaMemcpyDeviceToHost);
    cudaFree(d_pairs);
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, cudaGetErrorString(e));
    *count = (int64_t)n;
    return REVSIM_OK;
}

int32_t revsim_forces(revsim_handle *h, double *F) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!F) return fail(h, REVSIM_ERR_BADARG, "F is null");
    if ((rc = build_nlist_checked(h, h->d_x))) return rc;
    if ((rc = pack(h, 0, false))) return rc;
    StepArgs a = base_args(h, false);
    a.pos_in = h->d_pos[0];
    a.F_out = h->d_F;
    a.mode = MODE_FORCES_ONLY;
    if ((rc = launch_step_k(h, false, a))) return rc;
    CK(cudaMemcpyAsync(F, h->d_F, sizeof(double) * 3 * (size_t)h->N, cudaMemcpyDeviceToHost, h->st));
    int s;
    if ((rc = read_status(h, &s))) return rc;
    return status_code(h, s);
}

int32_t revsim_force_vjp(revsim_handle *h, const double *w, const double *acoef, double *F,
                         double *dl_dfi, double *dtheta) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!w || !acoef) return fail(h, REVSIM_ERR_BADARG, "null input");
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_C, w, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_A, acoef, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    if ((rc = build_nlist_checked(h, h->d_x))) return rc;
    if ((rc = pack(h, 0, true))) return rc;
    CK(cudaMemsetAsync(h->d_part, 0, sizeof(double) * part_slots(h) * h->P, h->st));
    if ((rc = mlp_zero_adj(h))) return rc;
    StepArgs a = base_args(h, true);
    a.pos_in = h->d_pos[0];
    a.wgt_in = h->d_wgt[0];
    a.F_out = h->d_F;
    a.acoefO = 1.0;
    a.acoefH = 1.0;
    a.mode = MODE_FORCES_ONLY;
    if ((rc = launch_step_k(h, true, a))) return rc;
    if (F) CK(cudaMemcpyAsync(F, h->d_F, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->st));
    if (dl_dfi) CK(cudaMemcpyAsync(dl_dfi, h->d_G, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->st));
    std::vector<double> th, thm;
    if ((rc = reduce_part(h, th))) return rc;
    if (h->mlp && (rc = mlp_grads(h, thm))) return rc;
    if (dtheta) join_grads(h, th, thm, 1.0, dtheta);
    int s;
    if ((rc = read_status(h, &s))) return rc;
    return status_code(h, s);
}

int32_t revsim_energy_grad(revsim_handle *h, double *energy, double *dEdtheta) {
    int rc = check_ready(h);
    if (rc) return rc;
    CK(cudaSetDevice(h->dev));
    if ((rc = build_nlist_checked(h, h->d_x))) return rc;
    if ((rc = mlp_zero_adj(h))) return rc;
    if (!h->d_epart) CK(dalloc(&h->d_epart, (size_t)h->M * (h->P + 1)));
    EnergyArgs a = energy_args(h, h->d_nbr, h->d_nbr_cnt);
    a.mlp_adj = h->mlp ? h->d_mlp_adj : nullptr;
    cudaError_t e = launch_energy_grads(h->mlp ? (int)F_LJ_MLP : h->form, h->prec, a, h->st);
    h->launches++;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("energy gradient: ") + cudaGetErrorString(e));
    std::vector<double> part((size_t)h->M * (h->P + 1));
    std::vector<int> mol_rep(h->M);
    CK(cudaMemcpyAsync(part.data(), h->d_epart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(mol_rep.data(), h->d_mol_rep, sizeof(int) * h->M, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    std::vector<double> E(h->R, 0.0), cl((size_t)h->R * h->P, 0.0), ml;
    for (int I = 0; I < h->M; I++) {
        const int r = mol_rep[I];
        E[r] += part[(size_t)I * (h->P + 1)];
        for (int p = 0; p < h->P; p++) cl[(size_t)r * h->P + p] += part[(size_t)I * (h->P + 1) + 1 + p];
    }
    if (h->mlp && (rc = mlp_grads(h, ml))) return rc;
    if (energy) std::memcpy(energy, E.data(), sizeof(double) * h->R);
    if (dEdtheta) join_grads(h, cl, ml, 1.0, dEdtheta);
    int s;
    if ((rc = read_status(h, &s))) return rc;
    return status_code(h, s);
}

int32_t revsim_noise(revsim_handle *h, const uint64_t *seeds, double *xi) {
    if (!h || !seeds || !xi) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    int rc = upload_seeds(h, seeds, h->R);
    if (rc) return rc;
    CK(launch_noise(h->N, h->d_atom_rep, h->d_rep_atom0, h->d_rep_sdO, h->d_rep_sdH, h->d_seeds, h->d_F, h->st));
    h->launches++;
    CK(cudaMemcpyAsync(xi, h->d_F, sizeof(double) * 3 * (size_t)h->N, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int32_t revsim_loss_grad(revsim_handle *h, double *loss, double *dLdx) {
    if (!h || !loss) return REVSIM_ERR_BADARG;
    if (!h->have_state) return fail(h, REVSIM_ERR_STATE, "state not set");
    CK(cudaSetDevice(h->dev));
    CK(cudaMemsetAsync(h->d_loss, 0, sizeof(double) * h->R, h->st));
    int rc = loss_dev(h, dLdx != nullptr, h->d_loss);
    if (rc) return rc;
    CK(cudaMemcpyAsync(loss, h->d_loss, sizeof(double) * h->R, cudaMemcpyDeviceToHost, h->st));
    if (dLdx) CK(cudaMemcpyAsync(dLdx, h->d_dLdx, sizeof(double) * 3 * (size_t)h->N, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int32_t revsim_set_barostat(revsim_handle *h, const revsim_barostat_desc *d) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!d) {
        h->baro_on = false;
        return REVSIM_OK;
    }
    if (!(d->pressure >= 0) || d->n_steps < 1 || !(d->scale_factor > 0) || !(d->scale_increment > 1) ||
        !(d->max_volume_frac > 0))
        return fail(h, REVSIM_ERR_BADARG, "bad barostat description");
    CK(cudaSetDevice(h->dev));
    if (!h->d_bx) {
        CK(dalloc(&h->d_bx, 3 * (size_t)h->N));
        CK(dalloc(&h->d_lsc, (size_t)h->R));
        CK(dalloc(&h->d_bacc, (size_t)h->R));
        CK(dalloc(&h->d_repE, (size_t)h->R));
    }
    h->baro = *d;
    h->baro_vs.resize(h->R);
    for (int r = 0; r < h->R; r++) h->baro_vs[r] = h->box[r] * h->box[r] * h->box[r] * d->scale_factor;
    h->baro_att.assign(h->R, 0);
    h->baro_acc.assign(h->R, 0);
    h->baro_draws.assign(h->R, 0);
    h->baro_acc_tot.assign(h->R, 0);
    h->baro_step = 0;
    h->baro_on = true;
    h->gen++;
    return REVSIM_OK;
}

int32_t revsim_barostat_state(revsim_handle *h, double *box, double *volume_scale, int64_t *n_attempts,
                              int64_t *n_accepted) {
    if (!h) return REVSIM_ERR_BADARG;
    for (int r = 0; r < h->R; r++) {
        const bool on = !h->baro_vs.empty();
        if (box) box[r] = h->box[r];
        if (volume_scale) volume_scale[r] = on ? h->baro_vs[r] : 0.0;
        if (n_attempts) n_attempts[r] = on ? h->baro_draws[r] : 0;
        if (n_accepted) n_accepted[r] = on ? h->baro_acc_tot[r] : 0;
    }
    return REVSIM_OK;
}

int32_t revsim_set_box(revsim_handle *h, const double *box) {
    if (!h || !box) return REVSIM_ERR_BADARG;
    for (int r = 0; r < h->R; r++) {
        if (!(box[r] > 2 * h->rc_nl) || !std::isfinite(box[r]))
            return fail(h, REVSIM_ERR_BADARG, "box side must exceed twice the neighbour cutoff");
        if (h->exact && !(box[r] < kGridMaxBox))
            return fail(h, REVSIM_ERR_BADARG, "the exact integrator needs boxes under 32 nm");
    }
    CK(cudaSetDevice(h->dev));
    const std::vector<double> old = h->box;
    h->box.assign(box, box + h->R);
    int rc = set_cells(h);
    if (rc) {
        h->box = old;
        return rc;
    }
    CK(cudaMemcpyAsync(h->d_rep_box, h->box.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->fwd_valid = false;
    h->gen++;
    return REVSIM_OK;
}

int32_t revsim_set_enth_vap(revsim_handle *h, int32_t enable, double u_gas, double rt, double target) {
    if (!h) return REVSIM_ERR_BADARG;
    if (enable && !(std::isfinite(u_gas) && std::isfinite(rt) && std::isfinite(target)))
        return fail(h, REVSIM_ERR_BADARG, "enthalpy constants must be finite");
    CK(cudaSetDevice(h->dev));
    if (enable && !h->d_ev_acc) {
        CK(dalloc(&h->d_ev_acc, 2 * (size_t)h->R));   // [0, R) runs, [R, 2R) revsim_loss_and_grads
        CK(dalloc(&h->d_ev_k, (size_t)h->R));
        CK(dalloc(&h->d_ev_grad, (size_t)h->R * h->P));
        CK(cudaMemset(h->d_ev_acc, 0, sizeof(double) * 2 * h->R));
    }
    h->ev_on = enable != 0;
    h->gen++;
    h->ev_ugas = u_gas;
    h->ev_rt = rt;
    h->ev_target = target;
    return REVSIM_OK;
}

int32_t revsim_loss_parts(revsim_handle *h, double *l_rdf, double *l_ev) {
    if (!h) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    std::vector<double> tot(h->R, 0.0), ev(h->R, 0.0);
    if (h->last_blocks > 0) {
        CK(cudaMemcpy(tot.data(), h->d_loss_acc, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
        if (h->ev_on) CK(cudaMemcpy(ev.data(), h->d_ev_acc, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
    }
    const double nb = std::max(1, h->last_blocks);
    for (int r = 0; r < h->R; r++) {
        if (l_rdf) l_rdf[r] = h->last_blocks > 0 ? (tot[r] - ev[r]) / nb : 0.0;
        if (l_ev) l_ev[r] = h->last_blocks > 0 ? ev[r] / nb : 0.0;
    }
    return REVSIM_OK;
}

int32_t revsim_loss_and_grads(revsim_handle *h, double *loss, double *l_rdf, double *l_ev, double *dLdx,
                              double *dl_dp) {
    int rc = check_ready(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->d_loss, 0, sizeof(double) * h->R, h->st));
    if (h->ev_on) {
        CK(cudaMemsetAsync(h->d_ev_acc + h->R, 0, sizeof(double) * h->R, h->st));
        CK(cudaMemsetAsync(h->d_ev_grad, 0, sizeof(double) * h->R * h->P, h->st));
    }
    if (h->ev_on && dl_dp && (rc = mlp_zero_adj(h))) return rc;
    double *ev1 = h->ev_on ? h->d_ev_acc + h->R : nullptr;   // this call's slot
    if ((rc = loss_dev(h, dLdx != nullptr, h->d_loss, ev1, dl_dp != nullptr))) return rc;
    std::vector<double> tot(h->R), ev(h->R, 0.0);
    CK(cudaMemcpyAsync(tot.data(), h->d_loss, sizeof(double) * h->R, cudaMemcpyDeviceToHost, h->st));
    if (h->ev_on) CK(cudaMemcpyAsync(ev.data(), h->d_ev_acc + h->R, sizeof(double) * h->R, cudaMemcpyDeviceToHost, h->st));
    if (dLdx) CK(cudaMemcpyAsync(dLdx, h->d_dLdx, sizeof(double) * 3 * (size_t)h->N, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int r = 0; r < h->R; r++) {
        if (loss) loss[r] = tot[r];
        if (l_rdf) l_rdf[r] = tot[r] - ev[r];
        if (l_ev) l_ev[r] = ev[r];
    }
    if (dl_dp) {
        std::vector<double> cl((size_t)h->R * h->P, 0.0), ml;
        if (h->ev_on) {
            CK(cudaMemcpy(cl.data(), h->d_ev_grad, sizeof(double) * cl.size(), cudaMemcpyDeviceToHost));
            if (h->mlp && (rc = mlp_grads(h, ml))) return rc;
        } else if (h->mlp) {
            ml.assign((size_t)h->R * (h->Pt - h->P), 0.0);
        }
        join_grads(h, cl, ml, 1.0, dl_dp);
    }
    int s;
    if ((rc = read_status(h, &s))) return rc;
    return status_code(h, s);
}

int32_t revsim_rdf(revsim_handle *h, int32_t term, int32_t replica, double *hist) {
    if (!h || !hist || term < 0 || term >= (int)h->terms.size() || replica < 0 || replica >= h->R)
        return REVSIM_ERR_BADARG;
    if (!h->have_state) return fail(h, REVSIM_ERR_STATE, "state not set");
    CK(cudaSetDevice(h->dev));
    std::vector<Term> keep = h->terms;
    const bool ev = h->ev_on;
    h->terms.assign(1, keep[term]);
    h->ev_on = false;
    CK(cudaMemsetAsync(h->d_loss, 0, sizeof(double) * h->R, h->st));
    int rc = loss_dev(h, false, h->d_loss);
    h->terms = keep;
    h->ev_on = ev;
    if (rc) return rc;
    const Term &T = h->terms[term];
    CK(cudaMemcpyAsync(hist, T.d_hist + (size_t)replica * T.t.n_grid, sizeof(double) * T.t.n_grid,
                       cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

}  // extern "C"

namespace {

// Noise of a pass: the per-step seeds (Philox draws on the device) or, from the host-noise
// entry points, the caller's noise [n_steps][3N] copied to the device.  The guard clears the
// host-noise switch when the pass returns, on every path.
struct NoiseGuard {
    revsim_handle *h;
    ~NoiseGuard() { h->use_noise = false; }
};

int upload_noise(revsim_handle *h, const uint64_t *seeds, const double *noise, int n_steps) {
    h->use_noise = false;
    if (!noise) return upload_seeds(h, seeds, (size_t)n_steps * h->R);
    const size_t n = (size_t)n_steps * 3 * (size_t)h->N;
    if (n > h->noise_cap) {
        dfree(h->d_noise);
        h->d_noise = nullptr;
        h->noise_cap = 0;
        CK(dalloc(&h->d_noise, n));
        h->noise_cap = n;
    }
    if (n) CK(cudaMemcpyAsync(h->d_noise, noise, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
    h->use_noise = true;
    return REVSIM_OK;
}

// A pass (dir 0 reverse, 1 forward) through the handle's CUDA graph: captured from the
// stream on the first call with a given key, replayed on later calls.  Passes with a host
// decision inside (barostat attempts, gradient clipping), with the enthalpy term (its energy
// rows are allocated on first use) or with per-launch timing run as plain launches.
template <typename F>
int run_graphed(revsim_handle *h, int dir, std::vector<double> key, F &&pass) {
    if (!h->graph_on || h->ktime || h->baro_on || h->ev_on) return pass();
    // nothing may be allocated while the stream is capturing
    if (half_eff(h))
        if (int rc = ensure_half(h)) return rc;
    key.push_back((double)h->gen);
    key.push_back((double)g_alloc_gen.load());
    revsim_handle::GraphCache &c = h->gc[dir];
    if (c.ex == nullptr || c.key != key) {
        const long long l0 = h->launches;
        CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        const int rc = pass();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->st, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            h->launches = l0;
            if (rc) return rc;
            return fail(h, REVSIM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        }
        // a graph of the same shape updates the executable in place; otherwise a new one
        bool updated = false;
        if (c.ex) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(c.ex, g, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();
                cudaGraphExecDestroy(c.ex);
                c.ex = nullptr;
            }
        }
        if (!updated) {
            const cudaError_t ie = cudaGraphInstantiate(&c.ex, g, 0);
            if (ie != cudaSuccess) {
                cudaGraphDestroy(g);
                c.ex = nullptr;
                return fail(h, REVSIM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
            }
        }
        if (c.g) cudaGraphDestroy(c.g);
        c.g = g;
        c.key = key;
        c.launches = h->launches - l0;
        h->launches = l0;
        h->graph_captures++;
    }
    CK(cudaGraphLaunch(c.ex, h->st));
    h->launches += c.launches;
    h->graph_replays++;
    return REVSIM_OK;
}

int32_t forward_entry(revsim_handle *h, const uint64_t *noise_seeds, const double *noise, double gamma,
                      int32_t n_steps, int32_t n_steps_loss, double dt, int32_t calc_loss, double *loss_out) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (n_steps < 0 || (n_steps > 0 && !noise_seeds && !noise) || !(dt > 0) || !(gamma >= 0))
        return fail(h, REVSIM_ERR_BADARG, "bad forward arguments");
    if (calc_loss && n_steps > 0 && n_steps_loss < 1) return fail(h, REVSIM_ERR_BADARG, "n_steps_loss < 1");
    const size_t n3 = 3 * (size_t)h->N;
    NoiseGuard guard{h};
    if ((rc = upload_noise(h, noise_seeds, noise, n_steps))) return rc;
    if (h->exact && (rc = quantize_for_exact(h))) return rc;
    const size_t n_snap = (h->nlog > 0 ? (size_t)n_steps / h->nlog : 0) + 1;
    const size_t n_ckpt = n_steps > 0 ? (size_t)(n_steps - 1) / h->nf + 1 : 1;
    if ((rc = ensure_store(h, &h->d_snap_x, &h->snap_cap, n_snap * n3))) return rc;
    if ((rc = ensure_store(h, &h->d_snap_v, &h->snapv_cap, n_snap * n3))) return rc;
    if ((rc = ensure_store(h, &h->d_ckpt, &h->ckpt_cap, n_ckpt * n3))) return rc;
    CK(cudaMemcpyAsync(h->d_x0, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v0, h->d_v, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemsetAsync(h->d_maxcnt, 0, sizeof(int), h->st));
    // the barostat changes the boxes: a retry starts from the boxes and barostat state of now
    const std::vector<double> box0 = h->box, vs0 = h->baro_vs;
    const std::vector<long long> att0 = h->baro_att, acc0 = h->baro_acc, dr0 = h->baro_draws,
                                 tot0 = h->baro_acc_tot;
    const long long bstep0 = h->baro_step;
    for (int attempt = 0; attempt < 3; attempt++) {
        if (h->nl_mode == REVSIM_NL_CHECKPOINT) ensure_list_store(h, n_ckpt);
        const std::vector<double> key = {gamma, (double)n_steps, (double)n_steps_loss, dt, (double)calc_loss,
                                         (double)h->use_noise};
        if ((rc = run_graphed(h, 1, key, [&] { return forward_impl(h, gamma, n_steps, n_steps_loss, dt, calc_loss); })))
            return rc;
        int s;
        if ((rc = read_status(h, &s))) return rc;
        if (!(s & ST_NLIST_OVERFLOW)) {
            if ((rc = status_code(h, s))) return rc;
            break;
        }
        if (attempt == 2) return status_code(h, s);
        if ((rc = grow_cap(h))) return rc;
        CK(cudaMemcpyAsync(h->d_x, h->d_x0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
        CK(cudaMemcpyAsync(h->d_v, h->d_v0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
        if (h->baro_on) {
            h->box = box0;
            h->baro_vs = vs0;
            h->baro_att = att0;
            h->baro_acc = acc0;
            h->baro_draws = dr0;
            h->baro_acc_tot = tot0;
            h->baro_step = bstep0;
            CK(cudaMemcpyAsync(h->d_rep_box, h->box.data(), sizeof(double) * h->R, cudaMemcpyHostToDevice, h->st));
            if ((rc = set_cells(h))) return rc;
        }
    }
    h->fwd_baro = h->baro_on;
    h->last_blocks = calc_loss ? (n_steps == 0 ? 1 : std::max(1, n_steps / std::max(1, n_steps_loss))) : 0;
    if (loss_out) {
        const int n_blocks = n_steps == 0 ? 1 : std::max(1, n_steps / std::max(1, n_steps_loss));
        std::vector<double> l(h->R);
        CK(cudaMemcpy(l.data(), h->d_loss_acc, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
        for (int r = 0; r < h->R; r++) loss_out[r] = calc_loss ? l[r] / n_blocks : 0.0;
    }
    if (h->ktime && (rc = collect_kernel_times(h))) return rc;
    h->fwd_valid = true;
    h->fwd_steps = n_steps;
    return REVSIM_OK;
}

int32_t reverse_entry(revsim_handle *h, const uint64_t *noise_seeds, const double *noise, double gamma,
                      int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                      double clip_norm_threshold, double *loss_out, double *dl_dp_out) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (n_steps_trunc > n_steps_loss)
        return fail(h, REVSIM_ERR_BADARG, "n_steps_trunc must not be greater than n_steps_loss");
    if (n_steps < 1 || n_steps_loss < 1 || (!noise_seeds && !noise) || !(dt > 0) || !(gamma >= 0) ||
        !(clip_norm_threshold > 0))
        return fail(h, REVSIM_ERR_BADARG, "bad reverse arguments");
    if (!has_loss(h)) return fail(h, REVSIM_ERR_STATE, "no loss set");
    if (h->fwd_baro)
        return fail(h, REVSIM_ERR_STATE, "the forward pass ran with the barostat (an equilibration run): "
                                         "no reverse record");
    const bool need_store = h->nl_mode == REVSIM_NL_CHECKPOINT || (h->nlog > 0 && n_steps > h->nlog);
    if (need_store && !(h->fwd_valid && h->fwd_steps == n_steps))
        return fail(h, REVSIM_ERR_STATE, "reverse needs the forward pass of the same n_steps");
    NoiseGuard guard{h};
    if ((rc = upload_noise(h, noise_seeds, noise, n_steps))) return rc;
    const std::vector<double> key = {gamma, (double)n_steps, (double)n_steps_loss, (double)n_steps_trunc, dt,
                                     clip_norm_threshold, (double)h->use_noise};
    auto pass = [&] { return reverse_impl(h, gamma, n_steps, n_steps_loss, n_steps_trunc, dt, clip_norm_threshold); };
    if ((rc = std::isfinite(clip_norm_threshold) ? pass() : run_graphed(h, 0, key, pass))) return rc;
    int s;
    if ((rc = read_status(h, &s))) return rc;
    if ((rc = status_code(h, s))) return rc;
    const int n_blocks = n_steps / n_steps_loss;
    std::vector<double> th, thm;
    if ((rc = reduce_part(h, th))) return rc;
    if (h->ev_on) {
        // the enthalpy term's direct dl/dtheta of every loss point (water.jl:1471, 1540)
        std::vector<double> d((size_t)h->R * h->P);
        CK(cudaMemcpy(d.data(), h->d_ev_grad, sizeof(double) * d.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < d.size(); i++) th[i] += d[i];
    }
    if (h->mlp && (rc = mlp_grads(h, thm))) return rc;
    if (dl_dp_out) join_grads(h, th, thm, 1.0 / n_blocks, dl_dp_out);
    h->last_blocks = n_blocks;
    if (loss_out) {
        std::vector<double> l(h->R);
        CK(cudaMemcpy(l.data(), h->d_loss_acc, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
        for (int r = 0; r < h->R; r++) loss_out[r] = l[r] / n_blocks;
    }
    if (h->ktime && (rc = collect_kernel_times(h))) return rc;
    return REVSIM_OK;
}

}  // namespace

extern "C" {

int32_t revsim_forward(revsim_handle *h, const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                       int32_t n_steps_loss, double dt, int32_t calc_loss, double *loss_out) {
    if (h && n_steps > 0 && !noise_seeds) return fail(h, REVSIM_ERR_BADARG, "bad forward arguments");
    return forward_entry(h, noise_seeds, nullptr, gamma, n_steps, n_steps_loss, dt, calc_loss, loss_out);
}

int32_t revsim_forward_noise(revsim_handle *h, const double *host_noise, double gamma, int32_t n_steps,
                             int32_t n_steps_loss, double dt, int32_t calc_loss, double *loss_out) {
    if (h && n_steps > 0 && !host_noise) return fail(h, REVSIM_ERR_BADARG, "bad forward arguments");
    return forward_entry(h, nullptr, host_noise, gamma, n_steps, n_steps_loss, dt, calc_loss, loss_out);
}

int32_t revsim_reverse(revsim_handle *h, const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                       int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                       double clip_norm_threshold, double *loss_out, double *dl_dp_out) {
    if (h && !noise_seeds) return fail(h, REVSIM_ERR_BADARG, "bad reverse arguments");
    return reverse_entry(h, noise_seeds, nullptr, gamma, n_steps, n_steps_loss, n_steps_trunc, dt,
                         clip_norm_threshold, loss_out, dl_dp_out);
}

int32_t revsim_reverse_noise(revsim_handle *h, const double *host_noise, double gamma, int32_t n_steps,
                             int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                             double clip_norm_threshold, double *loss_out, double *dl_dp_out) {
    if (h && !host_noise) return fail(h, REVSIM_ERR_BADARG, "bad reverse arguments");
    return reverse_entry(h, nullptr, host_noise, gamma, n_steps, n_steps_loss, n_steps_trunc, dt,
                         clip_norm_threshold, loss_out, dl_dp_out);
}

int32_t revsim_set_integrator(revsim_handle *h, int32_t mode) {
    if (!h) return REVSIM_ERR_BADARG;
    if (mode != REVSIM_INTEGRATOR_REFERENCE && mode != REVSIM_INTEGRATOR_EXACT)
        return fail(h, REVSIM_ERR_BADARG, "bad integrator");
    if (mode == REVSIM_INTEGRATOR_EXACT)
        for (int r = 0; r < h->R; r++)
            if (!(h->box[r] < kGridMaxBox))
                return fail(h, REVSIM_ERR_BADARG, "the exact integrator needs boxes under 32 nm");
    if (h->exact != (mode == REVSIM_INTEGRATOR_EXACT)) h->gen++;
    h->exact = mode == REVSIM_INTEGRATOR_EXACT;
    h->fwd_valid = false;
    return REVSIM_OK;
}

int32_t revsim_set_graph_mode(revsim_handle *h, int32_t enable) {
    if (!h) return REVSIM_ERR_BADARG;
    h->graph_on = enable != 0;
    return REVSIM_OK;
}

int32_t revsim_graph_stats(const revsim_handle *h, int64_t *captures, int64_t *replays) {
    if (!h) return REVSIM_ERR_BADARG;
    if (captures) *captures = h->graph_captures;
    if (replays) *replays = h->graph_replays;
    return REVSIM_OK;
}

int32_t revsim_set_mlp_precision(revsim_handle *h, int32_t mode) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!h->mlp) return fail(h, REVSIM_ERR_STATE, "the handle has no learned pair term");
    if (mode != REVSIM_MLP_FP64 && mode != REVSIM_MLP_BF16_TC) return fail(h, REVSIM_ERR_BADARG, "bad MLP precision");
    CK(cudaSetDevice(h->dev));
    if (mode == REVSIM_MLP_BF16_TC && !h->d_mlp_tc) {
        void *p = nullptr;
        g_alloc_gen++;
        CK(cudaMalloc(&p, mlp_tc_scratch_bytes()));
        h->d_mlp_tc = p;
    }
    h->mlp_mode = mode;
    if (h->have_params && h->d_mlp_theta) return build_mlp_table(h);
    return REVSIM_OK;
}

int32_t revsim_mlp_eval(revsim_handle *h, int32_t n, const double *r, double *u, double *du, double *ms) {
    if (!h || n < 1 || (!u != !du)) return REVSIM_ERR_BADARG;
    if (!h->mlp || !h->have_params || !h->d_mlp_theta) return fail(h, REVSIM_ERR_STATE, "no learned pair term set");
    CK(cudaSetDevice(h->dev));
    const size_t need = (size_t)MLP_NT * n;
    if (need > h->mlp_eval_cap) {
        dfree(h->d_mlp_r);
        dfree(h->d_mlp_u);
        h->d_mlp_r = h->d_mlp_u = nullptr;
        h->mlp_eval_cap = 0;
        CK(dalloc(&h->d_mlp_r, need));
        CK(dalloc(&h->d_mlp_u, 2 * need));
        h->mlp_eval_cap = need;
    }
    if (r) CK(cudaMemcpyAsync(h->d_mlp_r, r, sizeof(double) * need, cudaMemcpyHostToDevice, h->st));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, h->st));
    }
    CK(launch_mlp_tc_eval(h->d_mlp_theta, MLP_NT, h->rc, MLP_WIDTH, n, r ? h->d_mlp_r : nullptr, h->d_mlp_u,
                          h->d_mlp_u + need, h->st));
    h->launches++;
    if (ms) CK(cudaEventRecord(e1, h->st));
    if (u) {
        CK(cudaMemcpyAsync(u, h->d_mlp_u, sizeof(double) * need, cudaMemcpyDeviceToHost, h->st));
        CK(cudaMemcpyAsync(du, h->d_mlp_u + need, sizeof(double) * need, cudaMemcpyDeviceToHost, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    if (ms) {
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        *ms = t;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return REVSIM_OK;
}

void *revsim_stream(revsim_handle *h) { return h ? (void *)h->st : nullptr; }

int64_t revsim_launch_count(const revsim_handle *h) { return h ? h->launches : 0; }

int32_t revsim_set_kernel_timing(revsim_handle *h, int32_t enable) {
    if (!h) return REVSIM_ERR_BADARG;
    h->ktime = enable != 0;
    h->gen++;
    for (int w = 0; w < 2; w++) {
        h->kt_ms[w] = 0.0;
        h->kt_n[w] = 0;
        h->ev_used[w] = 0;
    }
    return REVSIM_OK;
}

int32_t revsim_kernel_time(revsim_handle *h, int32_t which, double *total_ms, int64_t *launches) {
    if (!h || which < 0 || which > 1) return REVSIM_ERR_BADARG;
    if (total_ms) *total_ms = h->kt_ms[which];
    if (launches) *launches = h->kt_n[which];
    return REVSIM_OK;
}

}  // extern "C"

namespace {

// An allowed shape of step kernel dir (0 reverse, 1 forward): lanes 8, 16 or 32, whole warps,
// at most 512 threads and no more than the kernel's register budget lets one CTA have.
bool shape_ok(const revsim_handle *h, int dir, int G, int m, int U) {
    const int thr = G * m;
    if (!((G == 8 || G == 16 || G == 32) && m >= 1 && thr <= 512 && thr % 32 == 0 && U >= 1 && U <= 3 &&
          !(U == 3 && thr > 256)))
        return false;
    if (half_eff(h) && thr > half_max_threads(dir == 0)) return false;
    return thr <= step_max_threads(h->prec == REVSIM_MIXED, dir == 0, U);
}

// Shape of one step kernel (dir 0 reverse, 1 forward), after shape_ok.
int set_shape_dir(revsim_handle *h, int dir, int G, int m, int U) {
    revsim_handle::Shape &sh = h->shp[dir];
    h->gen++;
    sh.G = G;
    sh.U = U;
    if (m != sh.mpc || !sh.d_blk_rep) {
        sh.mpc = m;
        int rc = build_block_table(h, dir);
        if (rc) return rc;
    }
    return REVSIM_OK;
}

}  // namespace

extern "C" {

int32_t revsim_set_pair_mode(revsim_handle *h, int32_t mode) {
    if (!h) return REVSIM_ERR_BADARG;
    if (mode != REVSIM_PAIRS_BOTH_SIDES && mode != REVSIM_PAIRS_HALF_SHELL)
        return fail(h, REVSIM_ERR_BADARG, "bad pair evaluation mode");
    if (mode == REVSIM_PAIRS_HALF_SHELL && !split_rows(h))
        return fail(h, REVSIM_ERR_STATE, "half-shell pair evaluation needs mixed precision");
    const bool want = mode == REVSIM_PAIRS_HALF_SHELL;
    if (want == h->half_req) return REVSIM_OK;
    h->half_req = want;
    h->gen++;
    h->fwd_valid = false;
    // the half-shell reverse kernel allows fewer threads per CTA: shrink a shape beyond it
    for (int dir = 0; dir < 2; dir++) {
        revsim_handle::Shape &sh = h->shp[dir];
        if (shape_ok(h, dir, sh.G, sh.mpc, sh.U)) continue;
        int m = sh.mpc;
        while (m > 1 && !shape_ok(h, dir, sh.G, m, 1)) m--;
        if (int rc = set_shape_dir(h, dir, sh.G, m, 1)) return rc;
    }
    return REVSIM_OK;
}

int32_t revsim_get_pair_mode(const revsim_handle *h, int32_t *requested, int32_t *active) {
    if (!h) return REVSIM_ERR_BADARG;
    if (requested) *requested = h->half_req ? REVSIM_PAIRS_HALF_SHELL : REVSIM_PAIRS_BOTH_SIDES;
    if (active) *active = half_eff(h) ? REVSIM_PAIRS_HALF_SHELL : REVSIM_PAIRS_BOTH_SIDES;
    return REVSIM_OK;
}

// Lanes per molecule are one setting for both step kernels: a lane's share of a neighbour
// row and the butterfly that sums the lanes depend on it, so forward and reverse forces are
// the same bits only when both kernels use the same count.
int32_t revsim_set_launch_shape(revsim_handle *h, int32_t which, int32_t lanes, int32_t mpc,
                                int32_t unroll) {
    if (!h || which < -1 || which > 1) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->st));
    int G[2], m[2], U[2];
    for (int dir = 0; dir < 2; dir++) {
        const revsim_handle::Shape &sh = h->shp[dir];
        const bool sel = which < 0 || which == dir;
        G[dir] = lanes ? lanes : sh.G;
        m[dir] = sel && mpc ? mpc : sh.mpc;
        U[dir] = sel && unroll ? unroll : sh.U;
        if (!shape_ok(h, dir, G[dir], m[dir], U[dir]))
            return fail(h, REVSIM_ERR_BADARG,
                        sel ? "unsupported launch shape"
                            : "lanes per molecule apply to both step kernels; the other kernel's "
                              "shape does not allow this count");
    }
    for (int dir = 0; dir < 2; dir++)
        if (int rc = set_shape_dir(h, dir, G[dir], m[dir], U[dir])) return rc;
    return REVSIM_OK;
}

int32_t revsim_get_launch_shape(revsim_handle *h, int32_t which, int32_t *lanes, int32_t *mpc,
                                int32_t *unroll) {
    if (!h || which < 0 || which > 1) return REVSIM_ERR_BADARG;
    if (lanes) *lanes = h->shp[which].G;
    if (mpc) *mpc = h->shp[which].mpc;
    if (unroll) *unroll = h->shp[which].U;
    return REVSIM_OK;
}

// Project autotuner: for every lanes-per-molecule count G (one setting for both kernels, so
// that forward and reverse forces agree bit for bit) it times the reverse and the forward
// step kernel (forces-only mode, on the current state) at every allowed (molecules per CTA,
// entries per iteration), and keeps the G with the smallest reverse + forward time and, for
// it, each kernel's fastest shape.
int32_t revsim_autotune(revsim_handle *h, double dt) {
    int rc = check_ready(h);
    if (rc) return rc;
    if ((rc = build_nlist_checked(h, h->d_x))) return rc;
    if ((rc = pack(h, 0, true))) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best_total = std::numeric_limits<double>::infinity();
    int bm[2] = {h->shp[0].mpc, h->shp[1].mpc}, bu[2] = {h->shp[0].U, h->shp[1].U}, bg = h->shp[0].G;
    int n_sm = 148;
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, h->dev));
    auto blocks_for = [&](int m) {
        long b = 0;
        for (int r = 0; r < h->R; r++) b += (h->nmol[r] + m - 1) / m;
        return b;
    };
    for (int G : {8, 16, 32}) {
        double tot = 0.0;
        int gm[2] = {0, 0}, gu[2] = {1, 1};
        // molecules per CTA: the fixed thread counts, plus the smallest counts (whole warps)
        // whose CTAs fit in one wave of one or two CTAs per SM, which spread the molecules
        // over every SM
        std::vector<int> mpcs;
        for (int threads : {64, 128, 192, 256, 384, 512})
            if (threads >= G && threads % G == 0) mpcs.push_back(threads / G);
        const int mstep = std::max(1, 32 / G);
        for (int k : {1, 2}) {
            int m = mstep;
            while (m * G <= 512 && blocks_for(m) > (long)k * n_sm) m += mstep;
            if (m * G <= 512 && std::find(mpcs.begin(), mpcs.end(), m) == mpcs.end()) mpcs.push_back(m);
        }
        for (int dir = 0; dir < 2 && !rc; dir++) {
            const bool rev = dir == 0;
            double best = std::numeric_limits<double>::infinity();
            for (int mpc : mpcs) {
                for (int U : {1, 2, 3}) {
                    if (!shape_ok(h, dir, G, mpc, U)) continue;
                    if ((rc = set_shape_dir(h, dir, G, mpc, U))) break;
                    StepArgs a = base_args(h, rev);
                    a.pos_in = h->d_pos[0];
                    a.wgt_in = h->d_wgt[0];
                    a.F_out = h->d_F;
                    a.acoefO = dt * dt / (2 * h->mO);
                    a.acoefH = dt * dt / (2 * h->mH);
                    a.mode = MODE_FORCES_ONLY;
                    for (int it = 0; it < 2 && !rc; it++) rc = launch_step_k(h, rev, a);
                    if (rc) break;
                    CK(cudaEventRecord(e0, h->st));
                    for (int it = 0; it < 10 && !rc; it++) rc = launch_step_k(h, rev, a);
                    if (rc) break;
                    CK(cudaEventRecord(e1, h->st));
                    CK(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    if (ms < best) {
                        best = ms;
                        gm[dir] = mpc;
                        gu[dir] = U;
                    }
                }
                if (rc) break;
            }
            tot += best;
        }
        if (rc) break;
        if (tot < best_total) {
            best_total = tot;
            bg = G;
            for (int d = 0; d < 2; d++) {
                bm[d] = gm[d];
                bu[d] = gu[d];
            }
        }
    }
    for (int dir = 0; dir < 2 && !rc; dir++) rc = set_shape_dir(h, dir, bg, bm[dir], bu[dir]);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

}  // extern "C"
