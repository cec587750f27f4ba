// sw_api.cu -- the C ABI of include/revsim_sw.h: handle, device memory and the forward /
// reverse drivers of the Stillinger-Weber diamond engine.
//
// Driver structure (host loop on one CUDA stream, two kernels per MD step):
//   forward_sim  (diamond.jl:1439-1474): terms kernel (T_{c,q} at x_{n-1}), gather kernel
//                (forces + B-A-O-A step); candidate list rebuilt every n_steps_nf steps;
//                at each loss point the state is copied to the device-side snapshot store
//                and the stress loss is accumulated (virial from the terms kernel, kinetic
//                tensor and loss in three small reductions).
//   reverse_sim  (diamond.jl:1799-1868): loss and gradient at the end state, then per
//                step the terms kernel (T, its derivative along C / m, dtheta contraction
//                with A dt^2 / (2m)) and the gather kernel (forces, dl_dfi, un-kick, B/A
//                update and the next step's un-integration with the D/C update); blocks,
//                truncation and snapshot restores as the reference orders them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "revsim_sw.h"
#include "sw_internal.h"

using namespace rs;
using namespace rs::sw;

static_assert(REVSIM_SW_MLP_NPARAMS == MLP_PER_TYPE, "one MLP type of rs_mlp.cu");

struct revsim_sw_handle {
    std::string err;
    int dev = 0;
    cudaStream_t st = nullptr;

    int R = 0, N = 0, G = 16, prec = 0, nf = 10;
    std::vector<int> nat, atom0;
    std::vector<double> box, temp;
    double mass = 0, kB = 0, skin = 0;
    double theta[NP] = {0, 0, 0, 0, 0, 0, 0};
    // learned radial term: its MLP parameters follow the 7 SW ones (Pt in all)
    bool mlp = false;
    int Pt = NP;
    std::vector<double> theta_mlp;
    double *d_mlp_theta = nullptr, *d_mlp_adj = nullptr, *d_mlp_scratch = nullptr,
           *d_mlp_grad = nullptr;
    void *d_mlp_tab = nullptr;
    bool have_params = false, have_state = false, have_loss = false;
    double weight = 0;
    int vel_term = 1;

    // tables
    int *d_atom_rep = nullptr, *d_rep_atom0 = nullptr, *d_rep_n = nullptr;
    double *d_rep_box = nullptr, *d_rep_vol = nullptr, *d_rep_sd = nullptr, *d_target = nullptr;
    int n_blk = 0, n_ablk = 0;
    int *d_blk_rep = nullptr, *d_blk_atom0 = nullptr, *d_blk_n = nullptr;
    int *d_ablk_rep = nullptr, *d_ablk_atom0 = nullptr, *d_ablk_n = nullptr;
    int *d_rep_blk0 = nullptr, *d_rep_ablk0 = nullptr;   // [R + 1] block ranges per replica
    // cells and candidate rows
    std::vector<int> nc, cell_off;
    int n_cells = 0;
    int *d_rep_nc = nullptr, *d_rep_cell_off = nullptr, *d_cell_of = nullptr, *d_cell_cnt = nullptr,
        *d_cell_start = nullptr, *d_cell_fill = nullptr;
    float4 *d_cell_pos = nullptr;
    int *d_cand = nullptr, *d_cand_n = nullptr;
    double *d_x_nl = nullptr;
    // active slots and slot gradients (sized for 32 lanes in FP64)
    int *d_act_idx = nullptr, *d_act_n = nullptr;
    void *d_Tv = nullptr, *d_Tt = nullptr;
    // state and adjoints
    double *d_x = nullptr, *d_v = nullptr, *d_F = nullptr, *d_G = nullptr, *d_A = nullptr,
           *d_B = nullptr, *d_C = nullptr, *d_D = nullptr, *d_dLdx = nullptr, *d_dLdv = nullptr,
           *d_x0 = nullptr, *d_v0 = nullptr;
    // reductions
    double *d_part = nullptr, *d_wpart = nullptr, *d_vpart = nullptr, *d_kpart = nullptr,
           *d_vbar = nullptr, *d_sigma = nullptr, *d_S = nullptr, *d_loss = nullptr,
           *d_loss_acc = nullptr;
    int *d_status = nullptr, *d_maxcnt = nullptr, *d_maxact = nullptr;
    // trajectory store
    double *d_snap_x = nullptr, *d_snap_v = nullptr;
    size_t snap_cap = 0;
    uint64_t *d_seeds = nullptr;
    size_t seeds_cap = 0;
    bool fwd_valid = false;
    int fwd_steps = 0, fwd_nloss = 0, fwd_blocks = 0;
    // instrumentation
    long long launches = 0;
    bool ktime = false;
    std::vector<cudaEvent_t> ev[4];
    size_t ev_used[4] = {0, 0, 0, 0};
    double kt_ms[4] = {0, 0, 0, 0};
    long long kt_n[4] = {0, 0, 0, 0};
};

namespace {

int fail(revsim_sw_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(h, REVSIM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define RC(call)                    \
    do {                            \
        int rc_ = (call);           \
        if (rc_) return rc_;        \
    } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    return cudaMalloc((void **)p, sizeof(T) * n);
}

void dfree(void *p) {
    if (p) cudaFree(p);
}

template <typename R>
SwConsts<R> consts(const revsim_sw_handle *h) {
    const double *t = h->theta;
    SwConsts<R> p;
    p.A = (R)t[0];
    p.B = (R)t[1];
    p.a = (R)t[2];
    p.lam = (R)t[3];
    p.gam = (R)t[4];
    p.sig = (R)t[5];
    p.eps = (R)t[6];
    p.half_eA = (R)(0.5 * t[6] * t[0]);
    p.el = (R)(t[6] * t[3]);
    p.isig = (R)(1.0 / t[5]);
    p.a64 = t[2];
    p.sig64 = t[5];
    const double lim = t[2] * t[5];
    p.asig = (R)lim;
    p.lim2 = lim * lim;
    p.lo2 = (lim * (1 - 1e-9)) * (lim * (1 - 1e-9));
    p.hi2 = (lim * (1 + 1e-9)) * (lim * (1 + 1e-9));
    p.mlp_hinv = (R)(MLP_NG / MLP_RC);
    p.mlp_hhalf = (R)(MLP_NG / (2 * MLP_RC));
    p.mlp_hinv2 = (R)((MLP_NG / MLP_RC) * (MLP_NG / MLP_RC));
    p.mlp_rc2 = MLP_RC * MLP_RC;
    return p;
}

int set_blocks(revsim_sw_handle *h) {
    const int gpb = TERM_THREADS / h->G;
    std::vector<int> br, ba, bn;
    for (int r = 0; r < h->R; r++)
        for (int i = 0; i < h->nat[r]; i += gpb) {
            br.push_back(r);
            ba.push_back(h->atom0[r] + i);
            bn.push_back(std::min(gpb, h->nat[r] - i));
        }
    h->n_blk = (int)br.size();
    std::vector<int> r0(h->R + 1, 0);
    for (int b = 0; b < h->n_blk; b++) r0[br[b] + 1] = b + 1;
    for (int r = 0; r < h->R; r++) r0[r + 1] = std::max(r0[r + 1], r0[r]);
    dfree(h->d_rep_blk0);
    CK(dalloc(&h->d_rep_blk0, h->R + 1));
    CK(cudaMemcpy(h->d_rep_blk0, r0.data(), sizeof(int) * (h->R + 1), cudaMemcpyHostToDevice));
    dfree(h->d_blk_rep);
    dfree(h->d_blk_atom0);
    dfree(h->d_blk_n);
    dfree(h->d_part);
    dfree(h->d_wpart);
    CK(dalloc(&h->d_blk_rep, br.size()));
    CK(dalloc(&h->d_blk_atom0, br.size()));
    CK(dalloc(&h->d_blk_n, br.size()));
    CK(dalloc(&h->d_part, br.size() * NP));
    CK(dalloc(&h->d_wpart, br.size() * 9));
    CK(cudaMemcpy(h->d_blk_rep, br.data(), sizeof(int) * br.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_blk_atom0, ba.data(), sizeof(int) * ba.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_blk_n, bn.data(), sizeof(int) * bn.size(), cudaMemcpyHostToDevice));
    return REVSIM_OK;
}

// Cells of side >= a sigma + skin, at least 3 per box side.
int set_cells(revsim_sw_handle *h) {
    const double rl = h->theta[2] * h->theta[5] + h->skin;
    if (!(rl > 0)) return fail(h, REVSIM_ERR_BADARG, "a * sigma + skin must be positive");
    std::vector<int> nc(h->R), off(h->R);
    int tot = 0;
    for (int r = 0; r < h->R; r++) {
        nc[r] = (int)std::floor(h->box[r] / rl);
        if (nc[r] < 3)
            return fail(h, REVSIM_ERR_BADARG,
                        "box side below 3 (a sigma + skin): replica " + std::to_string(r));
        nc[r] = std::min(nc[r], 64);
        off[r] = tot;
        tot += nc[r] * nc[r] * nc[r];
    }
    if (tot != h->n_cells) {
        dfree(h->d_cell_cnt);
        dfree(h->d_cell_start);
        dfree(h->d_cell_fill);
        CK(dalloc(&h->d_cell_cnt, tot));
        CK(dalloc(&h->d_cell_start, tot));
        CK(dalloc(&h->d_cell_fill, tot));
    }
    h->nc = nc;
    h->cell_off = off;
    h->n_cells = tot;
    CK(cudaMemcpy(h->d_rep_nc, nc.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_rep_cell_off, off.data(), sizeof(int) * h->R, cudaMemcpyHostToDevice));
    return REVSIM_OK;
}

void free_all(revsim_sw_handle *h) {
    void *ptrs[] = {h->d_atom_rep, h->d_rep_atom0, h->d_rep_n, h->d_rep_box, h->d_rep_vol,
                    h->d_rep_sd, h->d_target, h->d_blk_rep, h->d_blk_atom0, h->d_blk_n,
                    h->d_ablk_rep, h->d_ablk_atom0, h->d_ablk_n, h->d_rep_blk0, h->d_rep_ablk0,
                    h->d_rep_nc, h->d_rep_cell_off,
                    h->d_cell_of, h->d_cell_cnt, h->d_cell_start, h->d_cell_fill, h->d_cell_pos,
                    h->d_cand, h->d_cand_n, h->d_x_nl, h->d_act_idx, h->d_act_n, h->d_Tv, h->d_Tt,
                    h->d_x, h->d_v, h->d_F, h->d_G, h->d_A, h->d_B, h->d_C, h->d_D, h->d_dLdx,
                    h->d_dLdv, h->d_x0, h->d_v0, h->d_part, h->d_wpart, h->d_vpart, h->d_kpart,
                    h->d_vbar, h->d_sigma, h->d_S, h->d_loss, h->d_loss_acc, h->d_status,
                    h->d_maxcnt, h->d_maxact, h->d_snap_x, h->d_snap_v, h->d_seeds,
                    h->d_mlp_theta, h->d_mlp_adj, h->d_mlp_scratch, h->d_mlp_grad, h->d_mlp_tab};
    for (void *p : ptrs) dfree(p);
    for (auto &v : h->ev)
        for (cudaEvent_t e : v) cudaEventDestroy(e);
    if (h->st) cudaStreamDestroy(h->st);
}

int read_status(revsim_sw_handle *h, int *flags) {
    int s = 0;
    CK(cudaMemcpyAsync(&s, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->st));
    *flags = s;
    return REVSIM_OK;
}

int status_code(revsim_sw_handle *h, int s) {
    if (s & ST_NLIST_OVERFLOW) {
        int ma = 0;
        CK(cudaMemcpy(&ma, h->d_maxact, sizeof(int), cudaMemcpyDeviceToHost));
        if (ma > h->G)
            return fail(h, REVSIM_ERR_NLIST_OVERFLOW,
                        "a centre has " + std::to_string(ma) + " active neighbours, more than " +
                            std::to_string(h->G) + " lanes");
        return fail(h, REVSIM_ERR_NLIST_OVERFLOW, "candidate row capacity exceeded");
    }
    if (s & ST_SKIN)
        return fail(h, REVSIM_ERR_NLIST_OVERFLOW,
                    "an atom moved more than skin / 2 between candidate-list builds");
    if (s & ST_NAN) return fail(h, REVSIM_ERR_NAN, "non-finite force or gradient");
    return REVSIM_OK;
}

// True when the last status overflowed the 16-lane slots (the caller may retry with 32).
bool lane_overflow(revsim_sw_handle *h) {
    int ma = 0;
    if (cudaMemcpy(&ma, h->d_maxact, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    return ma > h->G && h->G < 32 && ma <= 32;
}

int build_list(revsim_sw_handle *h) {
    SwNlArgs a;
    a.N = h->N;
    a.n_cells = h->n_cells;
    a.x = h->d_x;
    a.atom_rep = h->d_atom_rep;
    a.rep_nc = h->d_rep_nc;
    a.rep_cell_off = h->d_rep_cell_off;
    a.rep_atom0 = h->d_rep_atom0;
    a.rep_n = h->d_rep_n;
    a.rep_box = h->d_rep_box;
    a.cell_of = h->d_cell_of;
    a.cell_cnt = h->d_cell_cnt;
    a.cell_start = h->d_cell_start;
    a.cell_fill = h->d_cell_fill;
    a.cell_pos = h->d_cell_pos;
    a.cand = h->d_cand;
    a.cand_n = h->d_cand_n;
    a.x_nl = h->d_x_nl;
    const double rl = h->theta[2] * h->theta[5] + h->skin + 1e-4;
    a.rl2f = (float)(rl * rl);
    a.status = h->d_status;
    a.max_cnt = h->d_maxcnt;
    cudaError_t e = launch_sw_nlist(a, h->st);
    h->launches += 4;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("candidate list: ") + cudaGetErrorString(e));
    return REVSIM_OK;
}

int ev_begin(revsim_sw_handle *h, int which) {
    if (!h->ktime || which < 0) return REVSIM_OK;
    while (h->ev[which].size() < h->ev_used[which] + 2) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        h->ev[which].push_back(e);
    }
    CK(cudaEventRecord(h->ev[which][h->ev_used[which]], h->st));
    return REVSIM_OK;
}

int ev_end(revsim_sw_handle *h, int which) {
    if (!h->ktime || which < 0) return REVSIM_OK;
    CK(cudaEventRecord(h->ev[which][h->ev_used[which] + 1], h->st));
    h->ev_used[which] += 2;
    return REVSIM_OK;
}

int collect_kernel_times(revsim_sw_handle *h) {
    for (int w = 0; w < 4; w++) {
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

// Terms kernel.  mode TM_VALUE / TM_REV / TM_LOSS; with_w: write the virial partials.
int terms(revsim_sw_handle *h, int mode, bool with_part, bool with_w, double acoef_scale,
          int which = -1) {
    SwTermArgs a;
    a.blk_rep = h->d_blk_rep;
    a.blk_atom0 = h->d_blk_atom0;
    a.blk_n = h->d_blk_n;
    a.rep_box = h->d_rep_box;
    a.rep_vol = h->d_rep_vol;
    a.x = h->d_x;
    a.x_nl = h->d_x_nl;
    a.cand = h->d_cand;
    a.cand_n = h->d_cand_n;
    a.C = h->d_C;
    a.A = h->d_A;
    a.S = h->d_S;
    a.inv_m = 1.0 / h->mass;
    a.acoef_scale = acoef_scale;
    a.act_idx = h->d_act_idx;
    a.act_n = h->d_act_n;
    a.Tv = h->d_Tv;
    a.Tt = h->d_Tt;
    a.part = with_part ? h->d_part : nullptr;
    a.wpart = with_w ? h->d_wpart : nullptr;
    a.mlp_tab = h->mlp ? h->d_mlp_tab : nullptr;
    a.mlp_adj = (h->mlp && with_part) ? h->d_mlp_adj : nullptr;
    a.half_skin2 = 0.25 * h->skin * h->skin;
    a.status = h->d_status;
    a.max_act = h->d_maxact;
    RC(ev_begin(h, which));
    cudaError_t e = h->prec == REVSIM_MIXED
                        ? launch_sw_terms<float>(mode, h->G, h->n_blk, a, consts<float>(h), h->st)
                        : launch_sw_terms<double>(mode, h->G, h->n_blk, a, consts<double>(h), h->st);
    h->launches++;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("terms kernel: ") + cudaGetErrorString(e));
    return ev_end(h, which);
}

SwGatherArgs gather_args(revsim_sw_handle *h, double dt, double gamma) {
    SwGatherArgs g;
    g.N = h->N;
    g.atom_rep = h->d_atom_rep;
    g.rep_atom0 = h->d_rep_atom0;
    g.rep_box = h->d_rep_box;
    g.rep_vol = h->d_rep_vol;
    g.rep_sd = h->d_rep_sd;
    g.act_idx = h->d_act_idx;
    g.act_n = h->d_act_n;
    g.Tv = h->d_Tv;
    g.Tt = h->d_Tt;
    g.x = h->d_x;
    g.v = h->d_v;
    g.F = h->d_F;
    g.G = h->d_G;
    g.A = h->d_A;
    g.B = h->d_B;
    g.C = h->d_C;
    g.D = h->d_D;
    g.dLdx = nullptr;
    g.dLdv = nullptr;
    g.S = h->d_S;
    g.vbar = h->d_vbar;
    g.dt = dt;
    g.c = std::exp(-gamma * dt);
    g.s = std::sqrt(1 - g.c * g.c);
    g.m = h->mass;
    g.dt2 = dt * dt;
    g.seed_cur = g.seed_next = nullptr;
    g.fuse_next = 0;
    g.init_adjoint = 0;
    g.vel_term = h->vel_term;
    g.status = h->d_status;
    return g;
}

int gather(revsim_sw_handle *h, int mode, bool tangent, const SwGatherArgs &g, int which = -1) {
    RC(ev_begin(h, which));
    cudaError_t e = h->prec == REVSIM_MIXED ? launch_sw_gather<float>(mode, h->G, tangent, g, h->st)
                                            : launch_sw_gather<double>(mode, h->G, tangent, g, h->st);
    h->launches += mode == GM_FORCES ? 1 : 2;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("gather kernel: ") + cudaGetErrorString(e));
    return ev_end(h, which);
}

// Stress at the current state: virial from the terms kernel, then sigma, the loss and
// S = dL/dsigma per replica; adds the loss to loss_acc when accumulate.
int stress(revsim_sw_handle *h, int vel_term, bool accumulate) {
    RC(terms(h, TM_VALUE, false, true, 0.0));
    SwRedArgs a;
    a.R = h->R;
    a.ablk_rep = h->d_ablk_rep;
    a.ablk_atom0 = h->d_ablk_atom0;
    a.ablk_n = h->d_ablk_n;
    a.n_ablk = h->n_ablk;
    a.blk_rep = h->d_blk_rep;
    a.n_blk = h->n_blk;
    a.rep_blk0 = h->d_rep_blk0;
    a.rep_ablk0 = h->d_rep_ablk0;
    a.rep_n = h->d_rep_n;
    a.v = h->d_v;
    a.vpart = h->d_vpart;
    a.kpart = h->d_kpart;
    a.vbar = h->d_vbar;
    a.wpart = h->d_wpart;
    a.rep_vol = h->d_rep_vol;
    a.target = h->d_target;
    a.m = h->mass;
    a.weight = h->weight;
    a.vel_term = vel_term;
    a.sigma = h->d_sigma;
    a.S = h->d_S;
    a.loss = h->d_loss;
    a.loss_acc = accumulate ? h->d_loss_acc : nullptr;
    cudaError_t e = launch_sw_stress(a, h->st);
    h->launches += 4;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("stress: ") + cudaGetErrorString(e));
    return REVSIM_OK;
}

// dL/dx, dL/dv and the direct dL/dtheta (added to the partials) after stress().
int loss_grad_dev(revsim_sw_handle *h, double dt, double gamma, bool init_adjoint, double *dLdx,
                  double *dLdv) {
    RC(terms(h, TM_LOSS, true, false, 0.0));
    SwGatherArgs g = gather_args(h, dt > 0 ? dt : 1.0, gamma);
    g.dLdx = dLdx;
    g.dLdv = dLdv;
    g.init_adjoint = init_adjoint ? 1 : 0;
    return gather(h, GM_LOSS, true, g);
}

int upload_seeds(revsim_sw_handle *h, const uint64_t *seeds, size_t n) {
    if (n > h->seeds_cap) {
        dfree(h->d_seeds);
        h->d_seeds = nullptr;
        CK(dalloc(&h->d_seeds, n));
        h->seeds_cap = n;
    }
    if (n) CK(cudaMemcpyAsync(h->d_seeds, seeds, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, h->st));
    return REVSIM_OK;
}

// Zero the dtheta partials (and the learned term's coefficient adjoints).
int zero_part(revsim_sw_handle *h) {
    CK(cudaMemsetAsync(h->d_part, 0, sizeof(double) * (size_t)h->n_blk * NP, h->st));
    if (h->mlp)
        CK(cudaMemsetAsync(h->d_mlp_adj, 0, sizeof(double) * (size_t)h->R * MLP_NCOPY * MLP_NG * 4, h->st));
    return REVSIM_OK;
}

int reduce_part(revsim_sw_handle *h, std::vector<double> &out);

// Per replica: the SW partials summed in block order, then the learned term's gradient
// backpropagated from its coefficient adjoints; out [R][Pt] = scale * (both).
int grads_out(revsim_sw_handle *h, double scale, double *out) {
    std::vector<double> sw;
    RC(reduce_part(h, sw));
    std::vector<double> ml;
    if (h->mlp) {
        for (int r = 0; r < h->R; r++) {
            cudaError_t e = launch_mlp_backprop(h->d_mlp_theta, MLP_RC,
                                                h->d_mlp_adj + (size_t)r * MLP_NCOPY * MLP_NG * 4, MLP_NCOPY,
                                                h->d_mlp_scratch, h->d_mlp_grad + (size_t)r * MLP_PER_TYPE,
                                                h->st, 1, MLP_W);
            h->launches += 3;
            if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("MLP backprop: ") + cudaGetErrorString(e));
        }
        ml.resize((size_t)h->R * MLP_PER_TYPE);
        CK(cudaMemcpyAsync(ml.data(), h->d_mlp_grad, sizeof(double) * ml.size(), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    for (int r = 0; r < h->R; r++) {
        for (int p = 0; p < NP; p++) out[(size_t)r * h->Pt + p] = scale * sw[(size_t)r * NP + p];
        if (h->mlp)
            for (int p = 0; p < MLP_PER_TYPE; p++)
                out[(size_t)r * h->Pt + NP + p] = scale * ml[(size_t)r * MLP_PER_TYPE + p];
    }
    return REVSIM_OK;
}

int reduce_part(revsim_sw_handle *h, std::vector<double> &out) {
    std::vector<double> part((size_t)h->n_blk * NP);
    std::vector<int> br(h->n_blk);
    CK(cudaMemcpyAsync(part.data(), h->d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(br.data(), h->d_blk_rep, sizeof(int) * h->n_blk, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    out.assign((size_t)h->R * NP, 0.0);
    for (int b = 0; b < h->n_blk; b++)
        for (int p = 0; p < NP; p++) out[(size_t)br[b] * NP + p] += part[(size_t)b * NP + p];
    return REVSIM_OK;
}

int n_loss_points(int n_steps, int n_steps_loss, int n_steps_buffer) {
    int n = 0;
    for (int s = 1; s <= n_steps; s++)
        if ((n_steps - s) % n_steps_loss == 0 && s >= n_steps_buffer) n++;
    return n;
}

int ensure_snaps(revsim_sw_handle *h, size_t n) {
    if (n <= h->snap_cap) return REVSIM_OK;
    dfree(h->d_snap_x);
    dfree(h->d_snap_v);
    h->d_snap_x = h->d_snap_v = nullptr;
    h->snap_cap = 0;
    if (dalloc(&h->d_snap_x, n * 3 * (size_t)h->N) != cudaSuccess ||
        dalloc(&h->d_snap_v, n * 3 * (size_t)h->N) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, REVSIM_ERR_NOMEM, "snapshot store does not fit on the device");
    }
    h->snap_cap = n;
    return REVSIM_OK;
}

int set_lanes(revsim_sw_handle *h, int lanes) {
    if (lanes != 16 && lanes != 32) return fail(h, REVSIM_ERR_BADARG, "lanes must be 16 or 32");
    h->G = lanes;
    return set_blocks(h);
}

int forward_impl(revsim_sw_handle *h, double gamma, int n_steps, int n_steps_loss,
                 int n_steps_buffer, double dt, bool calc_loss, int n_blocks) {
    const size_t n3 = 3 * (size_t)h->N;
    const double sn = std::sqrt(1 - std::exp(-2 * gamma * dt));
    CK(cudaMemsetAsync(h->d_loss_acc, 0, sizeof(double) * h->R, h->st));
    CK(cudaMemsetAsync(h->d_maxact, 0, sizeof(int), h->st));
    RC(build_list(h));
    int since = 0, k = 0;
    for (int step = 1; step <= n_steps; step++) {
        if (since == h->nf) {
            RC(build_list(h));
            since = 0;
        }
        RC(terms(h, TM_VALUE, false, false, 0.0, 1));
        SwGatherArgs g = gather_args(h, dt, gamma);
        g.seed_cur = sn != 0.0 ? h->d_seeds + (size_t)(step - 1) * h->R : nullptr;
        RC(gather(h, GM_FWD, false, g, 3));
        since++;
        if ((n_steps - step) % n_steps_loss == 0 && step >= n_steps_buffer) {
            CK(cudaMemcpyAsync(h->d_snap_x + (size_t)k * n3, h->d_x, sizeof(double) * n3,
                               cudaMemcpyDeviceToDevice, h->st));
            CK(cudaMemcpyAsync(h->d_snap_v + (size_t)k * n3, h->d_v, sizeof(double) * n3,
                               cudaMemcpyDeviceToDevice, h->st));
            k++;
            if (calc_loss) RC(stress(h, h->vel_term, true));
        }
    }
    (void)n_blocks;
    return REVSIM_OK;
}

int reverse_impl(revsim_sw_handle *h, double gamma, int n_steps, int n_steps_loss,
                 int n_steps_trunc, double dt) {
    const size_t n3 = 3 * (size_t)h->N;
    const int n_blocks = h->fwd_blocks;
    const double sn = std::sqrt(1 - std::exp(-2 * gamma * dt));
    CK(cudaMemsetAsync(h->d_loss_acc, 0, sizeof(double) * h->R, h->st));
    RC(zero_part(h));
    CK(cudaMemsetAsync(h->d_maxact, 0, sizeof(int), h->st));
    const double acoef_scale = dt * dt / (2 * h->mass);
    RC(build_list(h));
    RC(stress(h, h->vel_term, true));
    RC(loss_grad_dev(h, dt, gamma, true, nullptr, nullptr));
    for (int lc = 1; lc <= n_blocks; lc++) {
        const int step_start = n_steps - (lc - 1) * n_steps_loss;
        const int step_end = std::max(step_start - n_steps_trunc + 1, 1);
        {
            SwGatherArgs g = gather_args(h, dt, gamma);
            g.seed_cur = sn != 0.0 ? h->d_seeds + (size_t)(step_start - 1) * h->R : nullptr;
            cudaError_t e = launch_sw_part1(h->N, g, h->st);
            h->launches++;
            if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("part 1: ") + cudaGetErrorString(e));
        }
        RC(build_list(h));
        int since = 0;
        for (int step_n = step_start; step_n >= step_end; step_n--) {
            if (since == h->nf) {
                RC(build_list(h));
                since = 0;
            }
            RC(terms(h, TM_REV, true, false, acoef_scale, 0));
            SwGatherArgs g = gather_args(h, dt, gamma);
            g.fuse_next = step_n - 1 >= step_end ? 1 : 0;
            g.seed_next = (g.fuse_next && sn != 0.0) ? h->d_seeds + (size_t)(step_n - 2) * h->R : nullptr;
            RC(gather(h, GM_REV, true, g, 2));
            since++;
        }
        if (lc != n_blocks) {
            const size_t si = (size_t)(n_blocks - lc - 1) * n3;
            CK(cudaMemcpyAsync(h->d_x, h->d_snap_x + si, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
            CK(cudaMemcpyAsync(h->d_v, h->d_snap_v + si, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
            RC(build_list(h));
            RC(stress(h, h->vel_term, true));
            RC(loss_grad_dev(h, dt, gamma, true, nullptr, nullptr));
        }
    }
    return REVSIM_OK;
}

int save_state(revsim_sw_handle *h) {
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_x0, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v0, h->d_v, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    return REVSIM_OK;
}

int restore_state(revsim_sw_handle *h) {
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_x, h->d_x0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v, h->d_v0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->st));
    return REVSIM_OK;
}

// Run fn; if a centre had more active neighbours than 16 lanes hold, switch to 32 lanes,
// and if an atom left the candidate-list skin, halve the rebuild interval; then restore
// the state saved at entry and run it again.  Forces do not depend on when the lists were
// built (sw_internal.h), so a rerun gives the result the first run would have given.
template <typename Fn>
int with_lane_retry(revsim_sw_handle *h, Fn fn) {
    RC(save_state(h));
    for (int attempt = 0; attempt < 8; attempt++) {
        RC(fn());
        int s;
        RC(read_status(h, &s));
        if ((s & ST_NLIST_OVERFLOW) && lane_overflow(h)) {
            RC(set_lanes(h, 32));
            RC(restore_state(h));
            continue;
        }
        if ((s & ST_SKIN) && !(s & (ST_NLIST_OVERFLOW | ST_NAN)) && h->nf > 1) {
            h->nf = std::max(1, h->nf / 2);
            RC(restore_state(h));
            continue;
        }
        return status_code(h, s);
    }
    return fail(h, REVSIM_ERR_NLIST_OVERFLOW, "candidate lists keep failing");
}

int check_ready(revsim_sw_handle *h) {
    if (!h->have_params) return fail(h, REVSIM_ERR_STATE, "parameters not set");
    if (!h->have_state) return fail(h, REVSIM_ERR_STATE, "state not set");
    return REVSIM_OK;
}

}  // namespace

extern "C" {

int32_t revsim_sw_create(const revsim_sw_desc *d, revsim_sw_handle **out) {
    if (!d || !out) return REVSIM_ERR_BADARG;
    *out = nullptr;
    if (d->n_replicas < 1 || !d->n_atoms || !d->box || !d->temp) return REVSIM_ERR_BADARG;
    if (d->precision != REVSIM_FP64 && d->precision != REVSIM_MIXED) return REVSIM_ERR_BADARG;
    if (!(d->mass > 0) || !(d->kB > 0) || !(d->skin > 0) || d->n_steps_nf < 1) return REVSIM_ERR_BADARG;
    revsim_sw_handle *h = new (std::nothrow) revsim_sw_handle();
    if (!h) return REVSIM_ERR_NOMEM;
    h->R = d->n_replicas;
    long long N = 0;
    for (int r = 0; r < h->R; r++) {
        if (d->n_atoms[r] < 2 || !(d->box[r] > 0) || !(d->temp[r] >= 0)) {
            delete h;
            return REVSIM_ERR_BADARG;
        }
        h->nat.push_back(d->n_atoms[r]);
        h->atom0.push_back((int)N);
        h->box.push_back(d->box[r]);
        h->temp.push_back(d->temp[r]);
        N += d->n_atoms[r];
    }
    if (N > (1ll << 30)) {
        delete h;
        return REVSIM_ERR_BADARG;
    }
    h->N = (int)N;
    h->prec = d->precision;
    h->mass = d->mass;
    h->kB = d->kB;
    h->skin = d->skin;
    h->nf = d->n_steps_nf;
    h->dev = d->device;
    h->mlp = d->mlp != 0;
    h->Pt = NP + (h->mlp ? MLP_PER_TYPE : 0);
    int rc = [&]() -> int {
        CK(cudaSetDevice(h->dev));
        CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
        const int R = h->R;
        const size_t n3 = 3 * (size_t)h->N;
        std::vector<int> arep(h->N), rn(h->nat);
        std::vector<double> vol(R), sd(R);
        for (int r = 0; r < R; r++) {
            for (int i = 0; i < h->nat[r]; i++) arep[h->atom0[r] + i] = r;
            vol[r] = h->box[r] * h->box[r] * h->box[r];
            sd[r] = std::sqrt(h->kB * h->temp[r] / h->mass);
        }
        CK(dalloc(&h->d_atom_rep, h->N));
        CK(dalloc(&h->d_rep_atom0, R));
        CK(dalloc(&h->d_rep_n, R));
        CK(dalloc(&h->d_rep_box, R));
        CK(dalloc(&h->d_rep_vol, R));
        CK(dalloc(&h->d_rep_sd, R));
        CK(dalloc(&h->d_target, 9 * (size_t)R));
        CK(dalloc(&h->d_rep_nc, R));
        CK(dalloc(&h->d_rep_cell_off, R));
        CK(cudaMemcpy(h->d_atom_rep, arep.data(), sizeof(int) * h->N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_rep_atom0, h->atom0.data(), sizeof(int) * R, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_rep_n, rn.data(), sizeof(int) * R, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_rep_box, h->box.data(), sizeof(double) * R, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_rep_vol, vol.data(), sizeof(double) * R, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_rep_sd, sd.data(), sizeof(double) * R, cudaMemcpyHostToDevice));
        CK(cudaMemset(h->d_target, 0, sizeof(double) * 9 * R));
        // atom blocks of 256 within one replica
        std::vector<int> ar, aa, an;
        for (int r = 0; r < R; r++)
            for (int i = 0; i < h->nat[r]; i += 256) {
                ar.push_back(r);
                aa.push_back(h->atom0[r] + i);
                an.push_back(std::min(256, h->nat[r] - i));
            }
        h->n_ablk = (int)ar.size();
        std::vector<int> ra(R + 1, 0);
        for (int b = 0; b < h->n_ablk; b++) ra[ar[b] + 1] = b + 1;
        for (int r = 0; r < R; r++) ra[r + 1] = std::max(ra[r + 1], ra[r]);
        CK(dalloc(&h->d_rep_ablk0, R + 1));
        CK(cudaMemcpy(h->d_rep_ablk0, ra.data(), sizeof(int) * (R + 1), cudaMemcpyHostToDevice));
        CK(dalloc(&h->d_ablk_rep, ar.size()));
        CK(dalloc(&h->d_ablk_atom0, ar.size()));
        CK(dalloc(&h->d_ablk_n, ar.size()));
        CK(cudaMemcpy(h->d_ablk_rep, ar.data(), sizeof(int) * ar.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_ablk_atom0, aa.data(), sizeof(int) * aa.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_ablk_n, an.data(), sizeof(int) * an.size(), cudaMemcpyHostToDevice));
        CK(dalloc(&h->d_vpart, 3 * ar.size()));
        CK(dalloc(&h->d_kpart, 9 * ar.size()));
        CK(dalloc(&h->d_vbar, 3 * (size_t)R));
        CK(dalloc(&h->d_sigma, 9 * (size_t)R));
        CK(dalloc(&h->d_S, 9 * (size_t)R));
        CK(dalloc(&h->d_loss, R));
        CK(dalloc(&h->d_loss_acc, R));
        CK(dalloc(&h->d_cell_of, h->N));
        CK(dalloc(&h->d_cell_pos, h->N));
        CK(dalloc(&h->d_cand, (size_t)h->N * CAND));
        CK(dalloc(&h->d_cand_n, h->N));
        CK(dalloc(&h->d_x_nl, n3));
        CK(dalloc(&h->d_act_idx, (size_t)h->N * 32));
        CK(dalloc(&h->d_act_n, h->N));
        CK(dalloc((char **)&h->d_Tv, (size_t)h->N * 32 * 4 * sizeof(double)));
        CK(dalloc((char **)&h->d_Tt, (size_t)h->N * 32 * 4 * sizeof(double)));
        double **st[] = {&h->d_x, &h->d_v, &h->d_F, &h->d_G, &h->d_A, &h->d_B, &h->d_C,
                         &h->d_D, &h->d_dLdx, &h->d_dLdv, &h->d_x0, &h->d_v0};
        for (double **p : st) {
            CK(dalloc(p, n3));
            CK(cudaMemset(*p, 0, sizeof(double) * n3));
        }
        CK(dalloc(&h->d_status, 1));
        CK(dalloc(&h->d_maxcnt, 1));
        CK(dalloc(&h->d_maxact, 1));
        CK(cudaMemset(h->d_status, 0, sizeof(int)));
        CK(cudaMemset(h->d_maxcnt, 0, sizeof(int)));
        CK(cudaMemset(h->d_maxact, 0, sizeof(int)));
        RC(set_blocks(h));
        if (h->mlp) {
            CK(dalloc(&h->d_mlp_theta, (size_t)MLP_PER_TYPE));
            CK(dalloc(&h->d_mlp_adj, (size_t)R * MLP_NCOPY * MLP_NG * 4));
            CK(dalloc(&h->d_mlp_scratch, mlp_scratch_doubles()));
            CK(dalloc(&h->d_mlp_grad, (size_t)R * MLP_PER_TYPE));
            CK(dalloc((char **)&h->d_mlp_tab, (size_t)MLP_NG * 4 * sizeof(double)));
        }
        return REVSIM_OK;
    }();
    if (rc) {
        free_all(h);
        delete h;
        return rc;
    }
    *out = h;
    return REVSIM_OK;
}

void revsim_sw_destroy(revsim_sw_handle *h) {
    if (!h) return;
    cudaSetDevice(h->dev);
    if (h->st) cudaStreamSynchronize(h->st);
    free_all(h);
    delete h;
}

const char *revsim_sw_last_error(const revsim_sw_handle *h) { return h ? h->err.c_str() : "null handle"; }

int32_t revsim_sw_set_params(revsim_sw_handle *h, const double *theta, int32_t n) {
    if (!h || !theta) return REVSIM_ERR_BADARG;
    if (n != h->Pt)
        return fail(h, REVSIM_ERR_BADARG, h->mlp ? "theta must hold 7 + REVSIM_SW_MLP_NPARAMS values"
                                                 : "theta must hold 7 values");
    for (int i = 0; i < n; i++)
        if (!std::isfinite(theta[i])) return fail(h, REVSIM_ERR_BADARG, "non-finite parameter");
    if (!(theta[2] > 0) || !(theta[5] > 0)) return fail(h, REVSIM_ERR_BADARG, "a and sigma must be positive");
    CK(cudaSetDevice(h->dev));
    double old[NP];
    std::memcpy(old, h->theta, sizeof(old));
    std::memcpy(h->theta, theta, sizeof(old));
    int rc = set_cells(h);
    if (rc) {
        std::memcpy(h->theta, old, sizeof(old));
        return rc;
    }
    for (int r = 0; r < h->R; r++)
        if (!(theta[2] * theta[5] + h->skin < 0.5 * h->box[r])) {
            std::memcpy(h->theta, old, sizeof(old));
            return fail(h, REVSIM_ERR_BADARG, "a sigma + skin must stay below half the box side");
        }
    if (h->mlp) {
        std::vector<double> tm(theta + NP, theta + n);
        if (tm != h->theta_mlp) {
            CK(cudaMemcpyAsync(h->d_mlp_theta, tm.data(), sizeof(double) * tm.size(), cudaMemcpyHostToDevice, h->st));
            cudaError_t e = launch_mlp_table(h->prec, h->d_mlp_theta, MLP_RC, h->d_mlp_scratch, h->d_mlp_tab,
                                             h->st, 1, MLP_W);
            h->launches += 2;
            if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
            if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, std::string("MLP table: ") + cudaGetErrorString(e));
            h->theta_mlp = tm;
            h->fwd_valid = false;
        }
    }
    h->have_params = true;
    if (std::memcmp(old, h->theta, sizeof(old)) != 0) h->fwd_valid = false;
    return REVSIM_OK;
}

int32_t revsim_sw_set_state(revsim_sw_handle *h, const double *x, const double *v) {
    if (!h || !x || !v) return fail(h, REVSIM_ERR_BADARG, "null state");
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N;
    for (int r = 0; r < h->R; r++)
        for (size_t i = 3 * (size_t)h->atom0[r]; i < 3 * (size_t)(h->atom0[r] + h->nat[r]); i++)
            if (!std::isfinite(x[i]) || !std::isfinite(v[i]) || x[i] < 0 || !(x[i] <= h->box[r]))
                return fail(h, REVSIM_ERR_BADARG, "positions must be finite and inside the box");
    CK(cudaMemcpyAsync(h->d_x, x, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v, v, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->have_state = true;
    return REVSIM_OK;
}

int32_t revsim_sw_get_state(revsim_sw_handle *h, double *x, double *v) {
    if (!h) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N;
    if (x) CK(cudaMemcpyAsync(x, h->d_x, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->st));
    if (v) CK(cudaMemcpyAsync(v, h->d_v, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int32_t revsim_sw_set_loss(revsim_sw_handle *h, const revsim_sw_loss *L) {
    if (!h || !L || !std::isfinite(L->weight)) return fail(h, REVSIM_ERR_BADARG, "bad loss");
    CK(cudaSetDevice(h->dev));
    std::vector<double> t(9 * (size_t)h->R, 0.0);
    if (L->target) std::memcpy(t.data(), L->target, sizeof(double) * t.size());
    CK(cudaMemcpy(h->d_target, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice));
    h->weight = L->weight;
    h->vel_term = L->vel_term ? 1 : 0;
    h->have_loss = true;
    h->fwd_valid = false;
    return REVSIM_OK;
}

int32_t revsim_sw_forces(revsim_sw_handle *h, double *F) {
    if (!h || !F) return fail(h, REVSIM_ERR_BADARG, "null output");
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    RC(with_lane_retry(h, [&]() -> int {
        RC(build_list(h));
        RC(terms(h, TM_VALUE, false, false, 0.0));
        SwGatherArgs g = gather_args(h, 1.0, 0.0);
        return gather(h, GM_FORCES, false, g);
    }));
    CK(cudaMemcpy(F, h->d_F, sizeof(double) * 3 * (size_t)h->N, cudaMemcpyDeviceToHost));
    return REVSIM_OK;
}

int32_t revsim_sw_force_vjp(revsim_sw_handle *h, const double *w, const double *acoef, double *F,
                            double *dl_dfi, double *dtheta) {
    if (!h || !w) return fail(h, REVSIM_ERR_BADARG, "null input");
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_C, w, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    if (acoef) CK(cudaMemcpyAsync(h->d_A, acoef, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
    else CK(cudaMemsetAsync(h->d_A, 0, sizeof(double) * n3, h->st));
    RC(with_lane_retry(h, [&]() -> int {
        RC(zero_part(h));
        RC(build_list(h));
        RC(terms(h, TM_REV, true, false, 1.0));
        SwGatherArgs g = gather_args(h, 1.0, 0.0);
        return gather(h, GM_FORCES, true, g);
    }));
    if (F) CK(cudaMemcpy(F, h->d_F, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    if (dl_dfi) CK(cudaMemcpy(dl_dfi, h->d_G, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    if (dtheta && acoef) RC(grads_out(h, 1.0, dtheta));
    return REVSIM_OK;
}

int32_t revsim_sw_stress(revsim_sw_handle *h, int32_t vel_term, double *sigma) {
    if (!h || !sigma) return fail(h, REVSIM_ERR_BADARG, "null output");
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    RC(with_lane_retry(h, [&]() -> int {
        RC(build_list(h));
        return stress(h, vel_term ? 1 : 0, false);
    }));
    CK(cudaMemcpy(sigma, h->d_sigma, sizeof(double) * 9 * (size_t)h->R, cudaMemcpyDeviceToHost));
    return REVSIM_OK;
}

int32_t revsim_sw_loss_grad(revsim_sw_handle *h, double *loss, double *dLdx, double *dLdv,
                            double *dLdtheta) {
    if (!h) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    if (!h->have_loss) return fail(h, REVSIM_ERR_STATE, "loss not set");
    const size_t n3 = 3 * (size_t)h->N;
    RC(with_lane_retry(h, [&]() -> int {
        RC(zero_part(h));
        RC(build_list(h));
        RC(stress(h, h->vel_term, false));
        return loss_grad_dev(h, 1.0, 0.0, false, h->d_dLdx, h->d_dLdv);
    }));
    if (loss) CK(cudaMemcpy(loss, h->d_loss, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
    if (dLdx) CK(cudaMemcpy(dLdx, h->d_dLdx, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    if (dLdv) CK(cudaMemcpy(dLdv, h->d_dLdv, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    if (dLdtheta) RC(grads_out(h, 1.0, dLdtheta));
    return REVSIM_OK;
}

int32_t revsim_sw_noise(revsim_sw_handle *h, const uint64_t *seeds, double *xi) {
    if (!h || !seeds || !xi) return fail(h, REVSIM_ERR_BADARG, "null argument");
    CK(cudaSetDevice(h->dev));
    RC(upload_seeds(h, seeds, h->R));
    cudaError_t e = launch_sw_noise(h->N, h->d_atom_rep, h->d_rep_atom0, h->d_rep_sd, h->d_seeds,
                                    h->d_F, h->st);
    h->launches++;
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, cudaGetErrorString(e));
    CK(cudaMemcpyAsync(xi, h->d_F, sizeof(double) * 3 * (size_t)h->N, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int32_t revsim_sw_active_pairs(revsim_sw_handle *h, int32_t *pairs, int64_t max_pairs, int64_t *n) {
    if (!h || !n || max_pairs < 0 || (max_pairs > 0 && !pairs)) return fail(h, REVSIM_ERR_BADARG, "bad argument");
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    RC(with_lane_retry(h, [&]() -> int {
        RC(build_list(h));
        return terms(h, TM_VALUE, false, false, 0.0);
    }));
    unsigned long long *d_count = nullptr;
    int32_t *d_pairs = nullptr;
    CK(dalloc(&d_count, 1));
    CK(dalloc(&d_pairs, 2 * (size_t)std::max<int64_t>(max_pairs, 1)));
    CK(cudaMemset(d_count, 0, sizeof(unsigned long long)));
    cudaError_t e = launch_sw_active_pairs(h->N, h->G, h->d_act_idx, h->d_act_n, d_pairs, d_count,
                                           max_pairs, h->st);
    h->launches++;
    unsigned long long cnt = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e == cudaSuccess) e = cudaMemcpy(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && max_pairs > 0)
        e = cudaMemcpy(pairs, d_pairs, sizeof(int32_t) * 2 * std::min<int64_t>(max_pairs, (int64_t)cnt),
                       cudaMemcpyDeviceToHost);
    dfree(d_count);
    dfree(d_pairs);
    if (e != cudaSuccess) return fail(h, REVSIM_ERR_CUDA, cudaGetErrorString(e));
    *n = (int64_t)cnt;
    return REVSIM_OK;
}

int32_t revsim_sw_forward(revsim_sw_handle *h, const uint64_t *noise_seeds, double gamma,
                          int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_buffer, double dt,
                          int32_t calc_loss, double *loss, int32_t *n_blocks) {
    if (!h) return REVSIM_ERR_BADARG;
    if (n_steps < 0 || n_steps_loss < 1 || (n_steps > 0 && !noise_seeds) || !(dt > 0) || !(gamma >= 0))
        return fail(h, REVSIM_ERR_BADARG, "bad forward arguments");
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    if (calc_loss && !h->have_loss) return fail(h, REVSIM_ERR_STATE, "loss not set");
    const int nb = n_loss_points(n_steps, n_steps_loss, n_steps_buffer);
    RC(ensure_snaps(h, std::max(nb, 1)));
    RC(upload_seeds(h, noise_seeds, (size_t)n_steps * h->R));
    h->fwd_valid = false;
    RC(with_lane_retry(h, [&]() -> int {
        return forward_impl(h, gamma, n_steps, n_steps_loss, n_steps_buffer, dt, calc_loss != 0, nb);
    }));
    if (h->ktime) RC(collect_kernel_times(h));
    if (loss) {
        std::vector<double> l(h->R, 0.0);
        if (calc_loss && nb > 0) {
            CK(cudaMemcpy(l.data(), h->d_loss_acc, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
            for (double &x : l) x /= nb;
        }
        std::memcpy(loss, l.data(), sizeof(double) * h->R);
    }
    if (n_blocks) *n_blocks = nb;
    h->fwd_valid = nb > 0;
    h->fwd_steps = n_steps;
    h->fwd_nloss = n_steps_loss;
    h->fwd_blocks = nb;
    return REVSIM_OK;
}

int32_t revsim_sw_reverse(revsim_sw_handle *h, const uint64_t *noise_seeds, double gamma,
                          int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                          double *loss, double *dl_dtheta) {
    if (!h) return REVSIM_ERR_BADARG;
    if (n_steps < 1 || n_steps_loss < 1 || n_steps_trunc < 1 || !noise_seeds || !(dt > 0) || !(gamma >= 0))
        return fail(h, REVSIM_ERR_BADARG, "bad reverse arguments");
    CK(cudaSetDevice(h->dev));
    RC(check_ready(h));
    if (!h->have_loss) return fail(h, REVSIM_ERR_STATE, "loss not set");
    if (!h->fwd_valid || h->fwd_steps != n_steps || h->fwd_nloss != n_steps_loss)
        return fail(h, REVSIM_ERR_STATE, "reverse needs the forward pass of the same n_steps and n_steps_loss");
    RC(upload_seeds(h, noise_seeds, (size_t)n_steps * h->R));
    RC(with_lane_retry(h, [&]() -> int {
        return reverse_impl(h, gamma, n_steps, n_steps_loss, n_steps_trunc, dt);
    }));
    if (h->ktime) RC(collect_kernel_times(h));
    const int nb = h->fwd_blocks;
    if (loss) {
        CK(cudaMemcpy(loss, h->d_loss_acc, sizeof(double) * h->R, cudaMemcpyDeviceToHost));
        for (int r = 0; r < h->R; r++) loss[r] /= nb;
    }
    if (dl_dtheta) RC(grads_out(h, 1.0 / nb, dl_dtheta));
    h->fwd_valid = false;
    return REVSIM_OK;
}

int32_t revsim_sw_stream(revsim_sw_handle *h, void **stream) {
    if (!h || !stream) return REVSIM_ERR_BADARG;
    *stream = (void *)h->st;
    return REVSIM_OK;
}

int32_t revsim_sw_launch_count(revsim_sw_handle *h, int64_t *n) {
    if (!h || !n) return REVSIM_ERR_BADARG;
    *n = h->launches;
    return REVSIM_OK;
}

int32_t revsim_sw_set_kernel_timing(revsim_sw_handle *h, int32_t on) {
    if (!h) return REVSIM_ERR_BADARG;
    h->ktime = on != 0;
    for (int w = 0; w < 4; w++) {
        h->kt_ms[w] = 0.0;
        h->kt_n[w] = 0;
        h->ev_used[w] = 0;
    }
    return REVSIM_OK;
}

int32_t revsim_sw_kernel_time(revsim_sw_handle *h, int32_t which, double *ms, int64_t *launches) {
    if (!h || which < 0 || which > 3 || !ms || !launches) return REVSIM_ERR_BADARG;
    *ms = h->kt_ms[which];
    *launches = h->kt_n[which];
    return REVSIM_OK;
}

int32_t revsim_sw_set_lanes(revsim_sw_handle *h, int32_t lanes) {
    if (!h) return REVSIM_ERR_BADARG;
    CK(cudaSetDevice(h->dev));
    return set_lanes(h, lanes);
}

}  // extern "C"
