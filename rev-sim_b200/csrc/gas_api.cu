// gas_api.cu -- the C ABI of include/revsim_gas.h: handle, device memory and the forward /
// reverse drivers of the gas-in-water engine (diffusion/diffusion.jl).
//
// Driver structure (host loop on one CUDA stream, one fused kernel per MD step):
//   forward_sim (diffusion.jl:1181-1298): per step one force+integrate kernel; neighbour rows
//               rebuilt every n_steps_nf steps; x, v snapshots at step 0 and every loss
//               point; at a loss point with the enthalpy term the potential energy.  The
//               gas centres of the loss points are read from the snapshots afterwards and
//               the loss (calculate_D, loss_fn_final) is formed on the host.
//   reverse_sim (diffusion.jl:1511-1616): the centre gradient of every frame from the
//               forward's centres; per block from its end: accumulators from dl/dx of the
//               loss point, part 1 of the first step, then per step one fused kernel
//               (force + VJP + dtheta + un-kick + adjoint updates + part 1 of the next
//               step), then the snapshot restore of the next block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "gas_internal.h"
#include "revsim_gas.h"

using namespace gs;

struct revsim_gas_handle {
    std::string err;
    int dev = 0;
    cudaStream_t st = nullptr;
    int nw = 0, ng = 0, N = 0, nw3 = 0;
    double L = 0;
    int form = 0, P = 0, nf = 20, n_mol_ev = 0;
    double temp = 0, mO = 0, mH = 0, ke = 0, krf = 0, rc = 0, rc_nl = 0, kB = 0;
    BondConsts bw{};
    double kbg = 0, r0g = 0;
    std::vector<double> theta;
    bool have_params = false, have_state = false;
    GasConsts kc{};
    GasConstsT<float> kcf{};
    bool mixed = false;   // FP32 pair arithmetic (REVSIM_MIXED)
    int cap = 0, cur = 0;
    int *d_rows = nullptr, *d_cnt = nullptr, *d_status = nullptr;
    double *d_x = nullptr, *d_v = nullptr, *d_A = nullptr, *d_B = nullptr, *d_C = nullptr,
           *d_D = nullptr, *d_G = nullptr, *d_F = nullptr, *d_g = nullptr, *d_w = nullptr,
           *d_ac = nullptr, *d_part = nullptr, *d_epart = nullptr, *d_direct = nullptr,
           *d_gtail = nullptr, *d_Eloss = nullptr;
    size_t eloss_cap = 0;
    // gather buffers (32 B per atom: double4 in FP64, float4 in mixed precision) and the FP64
    // copy pos64 of the positions (aliases d_pos in FP64)
    void *d_pos[2] = {nullptr, nullptr}, *d_wgt[2] = {nullptr, nullptr};
    double4 *d_pos64[2] = {nullptr, nullptr};
    double4 *d_p64own[2] = {nullptr, nullptr};   // allocations of pos64 in mixed precision
    // forward record
    double *d_snap_x = nullptr, *d_snap_v = nullptr;
    size_t snap_cap = 0;   // snapshots
    bool fwd_valid = false;
    int fwd_steps = 0, fwd_nl = 0, fwd_blocks = 0;
    double fwd_dt = 0, fwd_gamma = 0;
    std::vector<double> centres, Eloss, Rloss;
    bool fwd_has_E = false, fwd_has_R = false;
    // RDF term of the water atoms: the terms, their targets and scratch (histogram with the
    // normaliser behind it, dL/dh), the one-box table {atom0, n_mol} / box, dL/dx of the
    // water atoms, and the per-loss-point losses of the forward pass
    struct RdfDev {
        revsim_rdf_term t;
        int off = 0;
        double *d_target = nullptr, *d_hist = nullptr, *d_dLdh = nullptr;
    };
    std::vector<RdfDev> rdf;
    int *d_rdf_int = nullptr;
    double *d_rdf_box = nullptr, *d_rdf_dx = nullptr, *d_rdf_tmp = nullptr, *d_rdf_loss = nullptr;
    size_t rdf_loss_cap = 0;
    // instrumentation
    long long launches = 0;
    bool ktime = false;
    std::vector<cudaEvent_t> ev[2];
    size_t ev_used[2] = {0, 0};
    double kt_ms[2] = {0.0, 0.0};
    long long kt_n[2] = {0, 0};
};

namespace {

constexpr double kDiffExp = 2.0e-9, kDiffWeight = 1e18;   // diffusion.jl:900-902
constexpr double kLossWeightEv = 0.05;                    // diffusion.jl:52
constexpr double kLossWeightRdf = 0.05;                   // diffusion.jl:51
constexpr double kUGas = 3.69, kRT = 2.45, kEvTarget = 44.12 + 2.8;   // diffusion.jl:800-813

int fail(revsim_gas_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(h, REVSIM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    return cudaMalloc((void **)p, sizeof(T) * n);
}

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

// Molly vector_1D and wrap_coords on the host (the centres of extract_gas_coords).
double vec1(double c1, double c2, double L) {
    if (c1 < c2) return (c2 - c1) < (c1 - c2 + L) ? (c2 - c1) : (c2 - c1 - L);
    return (c1 - c2) < (c2 - c1 + L) ? (c2 - c1) : (c2 - c1 + L);
}
double wrap(double c, double L) { return c - std::floor(c / L) * L; }

// Non-bonded constants and mixing factors of theta (inject_atom_grads diffusion.jl:584-615,
// the mixing of 169-170 / 272-274 and the dsigma_dsigmaw ... factors of 190-193, 296-297).
void set_consts(revsim_gas_handle *h) {
    const double *t = h->theta.data();
    GasConsts &k = h->kc;
    std::memset(&k, 0, sizeof(k));
    k.P = h->P;
    k.iq = h->P - 1;
    const double qO = t[k.iq], qH = -qO / 2;
    k.qq[0] = h->ke * qO * qO;
    k.qq[1] = h->ke * qO * qH;
    k.qq[2] = h->ke * qH * qH;
    k.krf = h->krf;
    k.krf2 = 2 * h->krf;
    k.rc2 = h->rc * h->rc;
    k.twoinvq = 2.0 / qO;
    k.crf_shift = 1.0 / h->rc + h->krf * h->rc * h->rc;
    const int nfp = form_nparams(h->form);
    double pc[3][4] = {};
    if (h->form == REVSIM_BUCK) {
        const double *w = t, *g = t + 3;
        for (int q = 0; q < 3; q++) {
            pc[0][q] = (w[q] + w[q]) / 2;
            pc[1][q] = (w[q] + g[q]) / 2;
            pc[2][q] = (g[q] + g[q]) / 2;
            k.iw[q] = q;
            k.ig[q] = q + 3;
            k.fw[0][q] = 1.0; k.fg[0][q] = 0.0;
            k.fw[1][q] = 0.5; k.fg[1][q] = 0.5;
            k.fw[2][q] = 0.0; k.fg[2][q] = 1.0;
        }
        k.iw[3] = 0;
        k.ig[3] = -1;
        k.on[0] = w[0] != 0.0;
        k.on[1] = w[0] != 0.0 && g[0] != 0.0;
        k.on[2] = g[0] != 0.0;
    } else {
        const double sw = t[0], ew = t[1], sg = t[2], eg = t[3];
        const double sig[3] = {(sw + sw) / 2, (sw + sg) / 2, (sg + sg) / 2};
        const double eps[3] = {std::sqrt(ew * ew), std::sqrt(ew * eg), std::sqrt(eg * eg)};
        for (int c = 0; c < 3; c++) {
            pc[c][0] = sig[c];
            pc[c][1] = eps[c];
            pc[c][2] = nfp > 2 ? t[4] : 0.0;
            pc[c][3] = nfp > 2 ? t[5] : 0.0;
        }
        k.iw[0] = 0; k.ig[0] = 2;
        k.iw[1] = 1; k.ig[1] = 3;
        k.iw[2] = 4; k.ig[2] = -1;
        k.iw[3] = 5; k.ig[3] = -1;
        k.fw[0][0] = 1.0; k.fg[0][0] = 0.0;
        k.fw[0][1] = 1.0; k.fg[0][1] = 0.0;
        k.fw[1][0] = 0.5; k.fg[1][0] = 0.5;
        k.fw[1][1] = eps[1] != 0.0 ? eg / (2 * eps[1]) : 0.0;
        k.fg[1][1] = eps[1] != 0.0 ? ew / (2 * eps[1]) : 0.0;
        k.fw[2][0] = 0.0; k.fg[2][0] = 1.0;
        k.fw[2][1] = 0.0; k.fg[2][1] = 1.0;
        for (int c = 0; c < 3; c++) {
            k.fw[c][2] = k.fw[c][3] = 1.0;
            k.fg[c][2] = k.fg[c][3] = 0.0;
        }
        k.on[0] = ew != 0.0;
        k.on[1] = ew != 0.0 && eg != 0.0;
        k.on[2] = eg != 0.0;
    }
    for (int c = 0; c < 3; c++) {
        k.fc[c] = rs::form_consts<double>(h->form, pc[c], nfp);
        k.fc[c].on = k.on[c];
    }
    // the same constants in FP32 for the mixed-precision pair arithmetic
    GasConstsT<float> &kf = h->kcf;
    std::memset(&kf, 0, sizeof(kf));
    for (int q = 0; q < 3; q++) kf.qq[q] = (float)k.qq[q];
    kf.krf = (float)k.krf;
    kf.krf2 = (float)k.krf2;
    kf.rc2 = (float)k.rc2;
    kf.twoinvq = (float)k.twoinvq;
    kf.crf_shift = k.crf_shift;
    for (int c = 0; c < 3; c++) {
        kf.fc[c] = rs::form_consts<float>(h->form, pc[c], nfp);
        kf.fc[c].on = k.on[c];
        kf.on[c] = k.on[c];
        for (int q = 0; q < 4; q++) {
            kf.fw[c][q] = k.fw[c][q];
            kf.fg[c][q] = k.fg[c][q];
        }
    }
    for (int q = 0; q < 4; q++) {
        kf.iw[q] = k.iw[q];
        kf.ig[q] = k.ig[q];
    }
    kf.P = k.P;
    kf.iq = k.iq;
}

GasArgs args(revsim_gas_handle *h) {
    GasArgs a;
    std::memset(&a, 0, sizeof(a));
    a.N = h->N;
    a.nw3 = h->nw3;
    a.L = h->L;
    a.invL = 1.0 / h->L;
    a.rows = h->d_rows;
    a.cnt = h->d_cnt;
    a.cap = h->cap;
    a.pos_in = h->d_pos[h->cur];
    a.pos_out = h->d_pos[h->cur ^ 1];
    a.wgt_in = h->d_wgt[h->cur];
    a.wgt_out = h->d_wgt[h->cur ^ 1];
    a.pos64_in = h->d_pos64[h->cur];
    a.pos64_out = h->d_pos64[h->cur ^ 1];
    a.x = h->d_x;
    a.v = h->d_v;
    a.A = h->d_A;
    a.B = h->d_B;
    a.C = h->d_C;
    a.D = h->d_D;
    a.G = h->d_G;
    a.F_out = h->d_F;
    a.acoef_in = nullptr;
    a.part = h->d_part;
    a.status = h->d_status;
    a.mO = h->mO;
    a.mH = h->mH;
    a.sdO = std::sqrt(h->kB * h->temp / h->mO);
    a.sdH = std::sqrt(h->kB * h->temp / h->mH);
    a.bw = h->bw;
    a.kb_g = h->kbg;
    a.r0_g = h->r0g;
    return a;
}

int rebuild(revsim_gas_handle *h) {
    GasRowArgs r;
    r.N = h->N;
    r.nw3 = h->nw3;
    r.L = h->L;
    r.rc_nl2 = h->rc_nl * h->rc_nl;
    r.x = h->d_x;
    r.rows = h->d_rows;
    r.cnt = h->d_cnt;
    r.cap = h->cap;
    r.status = h->d_status;
    launch_gas_rows(r, h->st);
    h->launches++;
    CK(cudaGetLastError());
    return REVSIM_OK;
}

int pack(revsim_gas_handle *h) {
    launch_gas_pack(h->mixed, h->N, h->d_x, h->d_pos[h->cur], h->d_pos64[h->cur], h->st);
    h->launches++;
    CK(cudaGetLastError());
    return REVSIM_OK;
}

// One step-kernel launch; timed (CUDA events, which 0 = reverse, 1 = forward) when kernel
// timing is on and `timed`.
int step(revsim_gas_handle *h, bool rev, const GasArgs &a, bool timed = true) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int w = rev ? 0 : 1;
    timed = timed && h->ktime;
    if (timed) {
        if (h->ev_used[w] + 2 > h->ev[w].size()) {
            for (int q = 0; q < 2; q++) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                h->ev[w].push_back(e);
            }
        }
        e0 = h->ev[w][h->ev_used[w]++];
        e1 = h->ev[w][h->ev_used[w]++];
        CK(cudaEventRecord(e0, h->st));
    }
    launch_gas_step(h->mixed, h->form, rev, h->kcf, h->kc, a, h->st);
    h->launches++;
    CK(cudaGetLastError());
    if (timed) CK(cudaEventRecord(e1, h->st));
    return REVSIM_OK;
}

int collect_timing(revsim_gas_handle *h) {
    for (int w = 0; w < 2; w++) {
        for (size_t q = 0; q + 1 < h->ev_used[w]; q += 2) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->ev[w][q], h->ev[w][q + 1]));
            h->kt_ms[w] += ms;
            h->kt_n[w]++;
        }
        h->ev_used[w] = 0;
    }
    return REVSIM_OK;
}

int check_status(revsim_gas_handle *h) {
    int s = 0;
    CK(cudaMemcpyAsync(&s, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (h->ktime) {
        int rc = collect_timing(h);
        if (rc) return rc;
    }
    if (s) {
        CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->st));
        if (s & rs::ST_NLIST_OVERFLOW)
            return fail(h, REVSIM_ERR_NLIST_OVERFLOW, "a neighbour row exceeded its capacity");
        if (s & rs::ST_NAN) return fail(h, REVSIM_ERR_NAN, "non-finite force");
        return fail(h, REVSIM_ERR_CUDA, "device status " + std::to_string(s));
    }
    return REVSIM_OK;
}

// Per-atom potential energy and parameter partials (into d_epart) at the current rows.
int energy_partials(revsim_gas_handle *h) {
    GasArgs a = args(h);
    launch_gas_energy(h->form, h->kc, a, h->d_epart, h->st);
    h->launches++;
    CK(cudaGetLastError());
    return REVSIM_OK;
}

// calculate_D (diffusion.jl:861-877) and its Enzyme pullback (879-895): the unwrapped
// displacement over n_frames / 2 frames from every start frame; its derivative is +1 for the
// end frame and -1 for the start frame (vector() has unit slopes, so coords_t's own slope
// cancels at every step).
double diffusion_D(const std::vector<double> &gc, int n_frames, int n_gas, double L, double lf,
                   std::vector<double> *grad) {
    const int ns = n_frames / 2;
    const size_t fsz = 3 * (size_t)n_gas;
    if (grad) grad->assign(fsz * (size_t)n_frames, 0.0);
    std::vector<double> ct(fsz);
    double D = 0.0;
    for (int stf = 0; stf < ns; stf++) {
        const double *c0 = gc.data() + fsz * stf;
        std::copy(c0, c0 + fsz, ct.begin());
        for (int j = stf + 1; j <= stf + ns; j++) {
            const double *cj = gc.data() + fsz * j;
            for (size_t e = 0; e < fsz; e++) ct[e] += vec1(ct[e], cj[e], L);
        }
        double msd = 0.0;
        for (int q = 0; q < n_gas; q++) {
            double d2 = 0.0;
            for (int u = 0; u < 3; u++) {
                const double d = ct[3 * q + u] - c0[3 * q + u];
                d2 += d * d;
            }
            msd += d2;
        }
        msd /= n_gas;
        D += msd / (ns * lf);
        if (grad) {
            const double k = 2.0 / ((double)n_gas * ns * lf * (6.0 * ns));
            double *ge = grad->data() + fsz * (stf + ns), *gs0 = grad->data() + fsz * stf;
            for (size_t e = 0; e < fsz; e++) {
                const double d = ct[e] - c0[e];
                ge[e] += k * d;
                gs0[e] -= k * d;
            }
        }
    }
    return D / (6 * ns);
}

// The forward's centres from the snapshots' gas atoms (extract_gas_coords, 836-844).
int read_centres(revsim_gas_handle *h) {
    const int nb = h->fwd_blocks;
    const size_t n3 = 3 * (size_t)h->N, gsz = 6 * (size_t)h->ng;
    h->centres.assign((size_t)nb * 3 * h->ng, 0.0);
    if (h->ng == 0 || nb == 0) return REVSIM_OK;
    std::vector<double> tail(gsz * (size_t)nb);
    CK(cudaMemcpy2DAsync(tail.data(), gsz * sizeof(double), h->d_snap_x + n3 + 3 * (size_t)h->nw3,
                         n3 * sizeof(double), gsz * sizeof(double), nb, cudaMemcpyDeviceToHost,
                         h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int b = 0; b < nb; b++)
        for (int q = 0; q < h->ng; q++) {
            const double *x1 = tail.data() + gsz * b + 6 * q, *x2 = x1 + 3;
            for (int u = 0; u < 3; u++)
                h->centres[(size_t)b * 3 * h->ng + 3 * q + u] = wrap(x1[u] + vec1(x1[u], x2[u], h->L) / 2, h->L);
        }
    return REVSIM_OK;
}

double ev_err(const revsim_gas_handle *h, double E) {
    return kUGas - E / h->n_mol_ev + kRT - kEvTarget;
}

int ensure_snapshots(revsim_gas_handle *h, size_t n_snap) {
    if (n_snap <= h->snap_cap) return REVSIM_OK;
    if (h->d_snap_x) cudaFree(h->d_snap_x);
    if (h->d_snap_v) cudaFree(h->d_snap_v);
    h->d_snap_x = h->d_snap_v = nullptr;
    h->snap_cap = 0;
    const size_t n3 = 3 * (size_t)h->N;
    if (dalloc(&h->d_snap_x, n_snap * n3) != cudaSuccess || dalloc(&h->d_snap_v, n_snap * n3) != cudaSuccess)
        return fail(h, REVSIM_ERR_NOMEM, "snapshot store");
    h->snap_cap = n_snap;
    return REVSIM_OK;
}

int ensure_eloss(revsim_gas_handle *h, size_t n) {
    if (n <= h->eloss_cap) return REVSIM_OK;
    if (h->d_Eloss) cudaFree(h->d_Eloss);
    h->d_Eloss = nullptr;
    h->eloss_cap = 0;
    if (dalloc(&h->d_Eloss, n * (size_t)(h->P + 1)) != cudaSuccess)
        return fail(h, REVSIM_ERR_NOMEM, "loss-point energies");
    h->eloss_cap = n;
    return REVSIM_OK;
}

void free_rdf(revsim_gas_handle *h) {
    for (auto &T : h->rdf) {
        if (T.d_target) cudaFree(T.d_target);
        if (T.d_hist) cudaFree(T.d_hist);
        if (T.d_dLdh) cudaFree(T.d_dLdh);
    }
    h->rdf.clear();
}

// Every RDF term at the current state (the water atoms 0 .. 3 n_water - 1, laid out O, H1, H2
// as the water engine's boxes): the summed term losses into *d_loss (accumulated) and, when
// grad, dL/dx of the water atoms into d_rdf_dx (accumulated).
int rdf_point(revsim_gas_handle *h, bool grad, double *d_loss) {
    for (auto &T : h->rdf) {
        const revsim_rdf_term &t = T.t;
        CK(cudaMemsetAsync(T.d_hist, 0, sizeof(double) * t.n_grid, h->st));
        rs::RdfArgs a;
        a.x = h->d_x;
        a.rep_atom0 = h->d_rdf_int;
        a.rep_nmol = h->d_rdf_int + 1;
        a.rep_box = h->d_rdf_box;
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
        a.dLdx = h->d_rdf_dx;
        const int n1 = t.sel1 == 0 ? h->nw : 2 * h->nw, n2 = t.sel2 == 0 ? h->nw : 2 * h->nw;
        CK(rs::launch_rdf(a, 1, n1, n2, false, h->st));
        CK(rs::launch_rdf_finalize(a, 1, T.d_hist + t.n_grid, T.d_target, t.slice_start, t.slice_stride,
                                   t.n_target, t.norm, t.weight, d_loss, T.d_dLdh, h->st));
        h->launches += 2;
        if (grad) {
            CK(rs::launch_rdf(a, 1, n1, n2, true, h->st));
            h->launches++;
        }
    }
    return REVSIM_OK;
}

// dl/dx of one loss point into d_g (enthalpy term, then the centre gradient of the frame
// halved onto the two sites of each gas molecule, diffusion.jl:1536-1539), the direct
// enthalpy dl/dtheta into d_direct; l_ev receives the point's enthalpy loss.
int point_grad(revsim_gas_handle *h, int loss_type, int n_blocks, double E, double R,
               const double *dgc_frame, double *l_ev, double *l_rdf) {
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemsetAsync(h->d_g, 0, n3 * sizeof(double), h->st));
    *l_ev = 0.0;
    *l_rdf = 0.0;
    if (loss_type & REVSIM_GAS_EV) {
        const double e = ev_err(h, E);
        *l_ev = e * e * kLossWeightEv / n_blocks;
        const double kk = 2 * e * kLossWeightEv / ((double)n_blocks * h->n_mol_ev);
        GasArgs a = args(h);
        a.mode = rs::MODE_FORCES_ONLY;
        int rc = step(h, false, a, false);
        if (rc) return rc;
        launch_gas_axpy((int)n3, kk, h->d_F, h->d_g, h->st);
        h->launches++;
        rc = energy_partials(h);
        if (rc) return rc;
        launch_gas_esum(h->N, h->P, h->d_epart, 0.0, -kk, true, h->d_direct, h->st);
        h->launches++;
        CK(cudaGetLastError());
    }
    if ((loss_type & REVSIM_GAS_RDF) && h->nw > 0) {
        // loss_and_grads_rdf_ev (diffusion.jl:922-947): 0.05 loss_rdf / n_blocks
        const double wr = kLossWeightRdf / n_blocks;
        *l_rdf = wr * R;
        CK(cudaMemsetAsync(h->d_rdf_dx, 0, 9 * (size_t)h->nw * sizeof(double), h->st));
        CK(cudaMemsetAsync(h->d_rdf_tmp, 0, sizeof(double), h->st));
        int rc = rdf_point(h, true, h->d_rdf_tmp);
        if (rc) return rc;
        launch_gas_axpy(9 * h->nw, wr, h->d_rdf_dx, h->d_g, h->st);
        h->launches++;
        CK(cudaGetLastError());
    }
    if (h->ng > 0 && dgc_frame) {
        std::vector<double> half(6 * (size_t)h->ng);
        for (int q = 0; q < h->ng; q++)
            for (int u = 0; u < 3; u++) {
                half[6 * q + u] = dgc_frame[3 * q + u] / 2;
                half[6 * q + 3 + u] = dgc_frame[3 * q + u] / 2;
            }
        // pageable source: the call returns once the data is staged
        CK(cudaMemcpyAsync(h->d_gtail, half.data(), half.size() * sizeof(double),
                           cudaMemcpyHostToDevice, h->st));
        launch_gas_axpy((int)half.size(), 1.0, h->d_gtail, h->d_g + 3 * (size_t)h->nw3, h->st);
        h->launches++;
        CK(cudaGetLastError());
    }
    return REVSIM_OK;
}

int reset_accums(revsim_gas_handle *h, double c) {
    // diffusion.jl:1547-1550, 1600-1604
    launch_gas_reset(3 * h->N, h->d_g, 1 + c, 1 + 2 * c + c * c, 2 * c, h->d_A, h->d_B, h->d_C,
                     h->d_D, h->d_G, h->st);
    h->launches++;
    CK(cudaGetLastError());
    return REVSIM_OK;
}

}  // namespace

extern "C" {

int32_t revsim_gas_n_params(int32_t inter_type) {
    if (form_nparams(inter_type) < 0) return -1;
    return inter_type == REVSIM_LJ ? 5 : 7;
}

const char *revsim_gas_last_error(const revsim_gas_handle *h) {
    return h ? h->err.c_str() : "null handle";
}

int32_t revsim_gas_destroy(revsim_gas_handle *h) {
    if (!h) return REVSIM_OK;
    cudaSetDevice(h->dev);
    if (h->st) cudaStreamSynchronize(h->st);
    void *bufs[] = {h->d_rows, h->d_cnt, h->d_status, h->d_x, h->d_v, h->d_A, h->d_B, h->d_C,
                    h->d_D, h->d_G, h->d_F, h->d_g, h->d_w, h->d_ac, h->d_part, h->d_epart,
                    h->d_direct, h->d_gtail, h->d_Eloss, h->d_pos[0], h->d_pos[1], h->d_wgt[0],
                    h->d_wgt[1], h->d_snap_x, h->d_snap_v, h->d_p64own[0], h->d_p64own[1]};
    for (void *p : bufs)
        if (p) cudaFree(p);
    free_rdf(h);
    void *rbufs[] = {h->d_rdf_int, h->d_rdf_box, h->d_rdf_dx, h->d_rdf_tmp, h->d_rdf_loss};
    for (void *p : rbufs)
        if (p) cudaFree(p);
    for (int w = 0; w < 2; w++)
        for (cudaEvent_t e : h->ev[w]) cudaEventDestroy(e);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return REVSIM_OK;
}

int32_t revsim_gas_create(const revsim_gas_desc *d, revsim_gas_handle **out) {
    if (!out) return REVSIM_ERR_BADARG;
    *out = nullptr;
    if (!d) return REVSIM_ERR_BADARG;
    revsim_gas_handle *h = new (std::nothrow) revsim_gas_handle();
    if (!h) return REVSIM_ERR_NOMEM;
    auto def = [](double v, double dv) { return v != 0.0 ? v : dv; };
    h->nw = d->n_water;
    h->ng = d->n_gas;
    h->form = d->inter_type;
    h->L = d->box;
    h->temp = def(d->temp, 295.15);
    h->mO = def(d->m_O, 15.99943);
    h->mH = def(d->m_H, 1.007947);
    h->ke = def(d->coulomb_const, 138.93545764438196);
    h->rc = def(d->cutoff, 1.0);
    h->rc_nl = def(d->nl_cutoff, 1.2);
    h->nf = d->n_steps_nf > 0 ? d->n_steps_nf : 20;
    h->kB = def(d->kB, 0.00831446261815324);
    h->krf = (1.0 / (h->rc * h->rc * h->rc)) * ((78.3 - 1) / (2 * 78.3 + 1));   // diffusion.jl:38
    h->bw = BondConsts{def(d->kb_w, 462750.4), def(d->r0_w, 0.09572), def(d->ka_w, 836.8),
                       def(d->th0_w, 1.82421813418)};
    h->kbg = def(d->kb_g, 1640.4 * 4.184 * 100);
    h->r0g = def(d->r0_g, 0.12074);
    h->n_mol_ev = d->n_mol_ev > 0 ? d->n_mol_ev : d->n_water + d->n_gas;
    h->dev = d->device;
    h->mixed = d->precision == REVSIM_MIXED;
    int rc0 = REVSIM_OK;
    if (d->precision != REVSIM_FP64 && d->precision != REVSIM_MIXED)
        rc0 = fail(h, REVSIM_ERR_BADARG, "precision must be REVSIM_FP64 or REVSIM_MIXED");
    else if (h->nw < 0 || h->ng < 0 || h->nw + h->ng < 1)
        rc0 = fail(h, REVSIM_ERR_BADARG, "need n_water, n_gas >= 0 and at least one molecule");
    else if (form_nparams(h->form) < 0)
        rc0 = fail(h, REVSIM_ERR_BADARG, "unknown inter_type");
    else if (!(h->L >= 2 * h->rc_nl) || !(h->rc_nl >= h->rc) || !(h->rc > 0))
        rc0 = fail(h, REVSIM_ERR_GEOMETRY, "need box >= 2 nl_cutoff and nl_cutoff >= cutoff > 0");
    else if (3.0 * h->nw + 2.0 * h->ng > 2.0e9)
        rc0 = fail(h, REVSIM_ERR_BADARG, "too many atoms");
    if (rc0) {
        delete h;
        return rc0;
    }
    h->nw3 = 3 * h->nw;
    h->N = h->nw3 + 2 * h->ng;
    h->P = revsim_gas_n_params(h->form);
    const double pi = 3.14159265358979323846;
    const double n_est = h->N / (h->L * h->L * h->L) * (4.0 / 3.0) * pi * h->rc_nl * h->rc_nl * h->rc_nl;
    h->cap = std::min(h->N, ((int)(2.0 * n_est) + 64 + 31) / 32 * 32);
    const size_t N = h->N, n3 = 3 * N;
    auto bad = [&](cudaError_t e) { return e != cudaSuccess; };
    if (bad(cudaSetDevice(h->dev)) || bad(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)) ||
        bad(dalloc(&h->d_rows, N * (size_t)h->cap)) || bad(dalloc(&h->d_cnt, N)) ||
        bad(dalloc(&h->d_status, 1)) || bad(dalloc(&h->d_x, n3)) || bad(dalloc(&h->d_v, n3)) ||
        bad(dalloc(&h->d_A, n3)) || bad(dalloc(&h->d_B, n3)) || bad(dalloc(&h->d_C, n3)) ||
        bad(dalloc(&h->d_D, n3)) || bad(dalloc(&h->d_G, n3)) || bad(dalloc(&h->d_F, n3)) ||
        bad(dalloc(&h->d_g, n3)) || bad(dalloc(&h->d_w, n3)) || bad(dalloc(&h->d_ac, n3)) ||
        bad(dalloc(&h->d_part, N * kMaxP)) || bad(dalloc(&h->d_epart, N * (kMaxP + 1))) ||
        bad(dalloc(&h->d_direct, kMaxP + 1)) || bad(dalloc(&h->d_gtail, 6 * (size_t)h->ng)) ||
        bad(dalloc((double4 **)&h->d_pos[0], N)) || bad(dalloc((double4 **)&h->d_pos[1], N)) ||
        bad(dalloc((double4 **)&h->d_wgt[0], N)) || bad(dalloc((double4 **)&h->d_wgt[1], N)) ||
        (h->mixed && (bad(dalloc(&h->d_p64own[0], N)) || bad(dalloc(&h->d_p64own[1], N)))) ||
        bad(dalloc(&h->d_rdf_int, 2)) ||
        bad(dalloc(&h->d_rdf_box, 1)) || bad(dalloc(&h->d_rdf_dx, 9 * (size_t)h->nw)) ||
        bad(dalloc(&h->d_rdf_tmp, 1)) || bad(cudaMemset(h->d_status, 0, sizeof(int))) ||
        bad(cudaMemset(h->d_wgt[0], 0, N * sizeof(double4))) ||
        bad(cudaMemset(h->d_wgt[1], 0, N * sizeof(double4)))) {
        cudaGetLastError();
        revsim_gas_destroy(h);
        return REVSIM_ERR_NOMEM;
    }
    for (int b = 0; b < 2; b++)
        h->d_pos64[b] = h->mixed ? h->d_p64own[b] : static_cast<double4 *>(h->d_pos[b]);
    const int tab[2] = {0, h->nw};
    if (bad(cudaMemcpy(h->d_rdf_int, tab, sizeof(tab), cudaMemcpyHostToDevice)) ||
        bad(cudaMemcpy(h->d_rdf_box, &h->L, sizeof(double), cudaMemcpyHostToDevice))) {
        cudaGetLastError();
        revsim_gas_destroy(h);
        return REVSIM_ERR_CUDA;
    }
    *out = h;
    return REVSIM_OK;
}

int32_t revsim_gas_set_rdf(revsim_gas_handle *h, int32_t n_terms, const revsim_rdf_term *terms,
                           const double *const *targets) {
    if (!h) return REVSIM_ERR_BADARG;
    if (n_terms < 0 || (n_terms > 0 && (!terms || !targets))) return fail(h, REVSIM_ERR_BADARG, "bad RDF terms");
    for (int i = 0; i < n_terms; i++) {
        const revsim_rdf_term &t = terms[i];
        if (t.n_grid < 1 || !(t.step > 0) || !(t.width > 0) || !(t.exp_cutoff >= 0) || t.n_target < 1 ||
            t.slice_start < 0 || t.slice_stride < 1 ||
            t.slice_start + (long long)(t.n_target - 1) * t.slice_stride >= t.n_grid ||
            (t.norm != 1 && t.norm != 2) || (t.sel1 != 0 && t.sel1 != 1) || (t.sel2 != 0 && t.sel2 != 1) ||
            !targets[i])
            return fail(h, REVSIM_ERR_BADARG, "bad RDF term");
        const double q = t.x_min / t.step;
        if (std::fabs(q - std::llround(q)) > 1e-6)
            return fail(h, REVSIM_ERR_BADARG, "x_min must be a multiple of step (diffusion.jl:709)");
        if (!rs::rdf_term_recurrence_ok(t.step, t.width, t.exp_cutoff))
            return fail(h, REVSIM_ERR_BADARG, "width too small for the grid step and window");
    }
    if (n_terms > 0 && h->nw < 1) return fail(h, REVSIM_ERR_BADARG, "the RDF term needs water molecules");
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->st));
    free_rdf(h);
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n_terms; i++) {
        const revsim_rdf_term &t = terms[i];
        revsim_gas_handle::RdfDev T;
        T.t = t;
        T.off = (int)std::llround(t.x_min / t.step) - 1;
        h->rdf.push_back(T);
        auto &D = h->rdf.back();
        if (dalloc(&D.d_target, t.n_target) != cudaSuccess || dalloc(&D.d_hist, (size_t)t.n_grid + 1) != cudaSuccess ||
            dalloc(&D.d_dLdh, t.n_grid) != cudaSuccess) {
            free_rdf(h);
            return fail(h, REVSIM_ERR_NOMEM, "RDF scratch");
        }
        // the normaliser V / (4 pi n1 n2 step) behind the histogram (rdf_differentiable, 725)
        const double n1 = t.sel1 == 0 ? h->nw : 2.0 * h->nw, n2 = t.sel2 == 0 ? h->nw : 2.0 * h->nw;
        const double pre = h->L * h->L * h->L / (4 * pi * n1 * n2 * t.step);
        CK(cudaMemcpy(D.d_target, targets[i], sizeof(double) * t.n_target, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(D.d_hist + t.n_grid, &pre, sizeof(double), cudaMemcpyHostToDevice));
    }
    return REVSIM_OK;
}

int32_t revsim_gas_set_params(revsim_gas_handle *h, const double *theta, int32_t n_params) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!theta || n_params != h->P)
        return fail(h, REVSIM_ERR_BADARG, "expected " + std::to_string(h->P) + " parameters");
    for (int p = 0; p < n_params; p++)
        if (!std::isfinite(theta[p])) return fail(h, REVSIM_ERR_BADARG, "non-finite parameter");
    if (theta[n_params - 1] == 0.0) return fail(h, REVSIM_ERR_BADARG, "q_O must be non-zero");
    h->theta.assign(theta, theta + n_params);
    set_consts(h);
    h->have_params = true;
    return REVSIM_OK;
}

int32_t revsim_gas_set_state(revsim_gas_handle *h, const double *x, const double *v) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!x || !v) return fail(h, REVSIM_ERR_BADARG, "null state");
    const size_t n3 = 3 * (size_t)h->N;
    for (size_t e = 0; e < n3; e++)
        if (!std::isfinite(x[e]) || !std::isfinite(v[e])) return fail(h, REVSIM_ERR_BADARG, "non-finite state");
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(h->d_x, x, n3 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v, v, n3 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->have_state = true;
    return REVSIM_OK;
}

int32_t revsim_gas_get_state(revsim_gas_handle *h, double *x, double *v) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!h->have_state) return fail(h, REVSIM_ERR_STATE, "no state");
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaSetDevice(h->dev));
    if (x) CK(cudaMemcpyAsync(x, h->d_x, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    if (v) CK(cudaMemcpyAsync(v, h->d_v, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return REVSIM_OK;
}

int32_t revsim_gas_forces(revsim_gas_handle *h, double *F) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!F) return fail(h, REVSIM_ERR_BADARG, "null output");
    if (!h->have_params || !h->have_state) return fail(h, REVSIM_ERR_STATE, "set parameters and state first");
    CK(cudaSetDevice(h->dev));
    int rc = pack(h);
    if (!rc) rc = rebuild(h);
    if (rc) return rc;
    GasArgs a = args(h);
    a.mode = rs::MODE_FORCES_ONLY;
    rc = step(h, false, a, false);
    if (rc) return rc;
    CK(cudaMemcpyAsync(F, h->d_F, 3 * (size_t)h->N * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    return check_status(h);
}

int32_t revsim_gas_force_vjp(revsim_gas_handle *h, const double *w, const double *acoef, double *F,
                             double *dl_dfi, double *dl_dp) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!w || !acoef || !F || !dl_dfi || !dl_dp) return fail(h, REVSIM_ERR_BADARG, "null argument");
    if (!h->have_params || !h->have_state) return fail(h, REVSIM_ERR_STATE, "set parameters and state first");
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N;
    CK(cudaMemcpyAsync(h->d_w, w, n3 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_ac, acoef, n3 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemsetAsync(h->d_part, 0, (size_t)h->N * h->P * sizeof(double), h->st));
    int rc = pack(h);
    if (!rc) rc = rebuild(h);
    if (rc) return rc;
    launch_gas_pack_w(h->mixed, h->N, h->nw3, h->d_w, h->mO, h->mH, h->d_wgt[h->cur], h->st);
    h->launches++;
    GasArgs a = args(h);
    a.mode = rs::MODE_FORCES_ONLY;
    a.acoef_in = h->d_ac;
    rc = step(h, true, a, false);
    if (rc) return rc;
    std::vector<double> part((size_t)h->N * h->P);
    CK(cudaMemcpyAsync(F, h->d_F, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(dl_dfi, h->d_G, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(part.data(), h->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    rc = check_status(h);
    if (rc) return rc;
    for (int p = 0; p < h->P; p++) dl_dp[p] = 0.0;
    for (int i = 0; i < h->N; i++)
        for (int p = 0; p < h->P; p++) dl_dp[p] += part[(size_t)i * h->P + p];
    return REVSIM_OK;
}

int32_t revsim_gas_energy(revsim_gas_handle *h, double *E, double *dEdp) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!E) return fail(h, REVSIM_ERR_BADARG, "null output");
    if (!h->have_params || !h->have_state) return fail(h, REVSIM_ERR_STATE, "set parameters and state first");
    CK(cudaSetDevice(h->dev));
    int rc = pack(h);
    if (!rc) rc = rebuild(h);
    if (!rc) rc = energy_partials(h);
    if (rc) return rc;
    launch_gas_esum(h->N, h->P, h->d_epart, 1.0, 1.0, false, h->d_direct, h->st);
    h->launches++;
    std::vector<double> out(h->P + 1);
    CK(cudaMemcpyAsync(out.data(), h->d_direct, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    rc = check_status(h);
    if (rc) return rc;
    *E = out[0];
    if (dEdp)
        for (int p = 0; p < h->P; p++) dEdp[p] = out[1 + p];
    return REVSIM_OK;
}

int32_t revsim_gas_forward(revsim_gas_handle *h, const uint64_t *seeds, double gamma, int32_t n_steps,
                           int32_t n_steps_loss, double dt, int32_t loss_type, int32_t calc_loss,
                           double *loss, double *parts, double *centres) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!h->have_params || !h->have_state) return fail(h, REVSIM_ERR_STATE, "set parameters and state first");
    if (n_steps < 0 || n_steps_loss < 1 || !(dt > 0) || !(gamma >= 0) || (n_steps > 0 && !seeds))
        return fail(h, REVSIM_ERR_BADARG, "bad step arguments");
    if (loss_type & ~(REVSIM_GAS_DIFF | REVSIM_GAS_RDF | REVSIM_GAS_EV))
        return fail(h, REVSIM_ERR_BADARG, "unknown loss_type bits");
    if ((loss_type & REVSIM_GAS_RDF) && h->rdf.empty())
        return fail(h, REVSIM_ERR_STATE, "the RDF loss needs revsim_gas_set_rdf first");
    const int n_blocks = n_steps == 0 ? 1 : n_steps / n_steps_loss;
    if (calc_loss && (loss_type & REVSIM_GAS_DIFF) && n_blocks < 2)
        return fail(h, REVSIM_ERR_BADARG, "the diffusion loss needs at least two loss points");
    if (calc_loss && (loss_type & REVSIM_GAS_DIFF) && h->ng < 1)
        return fail(h, REVSIM_ERR_BADARG, "the diffusion loss needs gas molecules");
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N;
    int rc = ensure_snapshots(h, (size_t)n_blocks + 1);
    if (!rc && calc_loss && (loss_type & REVSIM_GAS_EV)) rc = ensure_eloss(h, (size_t)n_blocks);
    if (rc) return rc;
    const bool want_R = calc_loss && (loss_type & REVSIM_GAS_RDF);
    if (want_R && h->rdf_loss_cap < (size_t)n_blocks) {
        if (h->d_rdf_loss) cudaFree(h->d_rdf_loss);
        h->d_rdf_loss = nullptr;
        h->rdf_loss_cap = 0;
        if (dalloc(&h->d_rdf_loss, (size_t)n_blocks) != cudaSuccess)
            return fail(h, REVSIM_ERR_NOMEM, "loss-point RDF losses");
        h->rdf_loss_cap = n_blocks;
    }
    if (want_R) CK(cudaMemsetAsync(h->d_rdf_loss, 0, sizeof(double) * n_blocks, h->st));
    h->fwd_valid = false;
    const double c = std::exp(-gamma * dt), sn = std::sqrt(1 - c * c);   // diffusion.jl:1216-1217
    h->cur = 0;
    rc = pack(h);
    if (!rc) rc = rebuild(h);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->d_snap_x, h->d_x, n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_snap_v, h->d_v, n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    const bool want_E = calc_loss && (loss_type & REVSIM_GAS_EV);
    for (int stp = 1; stp <= n_steps; stp++) {
        GasArgs a = args(h);
        a.dt = dt;
        a.c = c;
        a.s = sn;
        a.seed_cur = seeds[stp - 1];
        rc = step(h, false, a);
        if (rc) return rc;
        h->cur ^= 1;
        if (stp % h->nf == 0) {
            rc = rebuild(h);
            if (rc) return rc;
        }
        if (stp % n_steps_loss == 0) {
            const int k = stp / n_steps_loss;
            if (k <= n_blocks) {
                CK(cudaMemcpyAsync(h->d_snap_x + (size_t)k * n3, h->d_x, n3 * sizeof(double),
                                   cudaMemcpyDeviceToDevice, h->st));
                CK(cudaMemcpyAsync(h->d_snap_v + (size_t)k * n3, h->d_v, n3 * sizeof(double),
                                   cudaMemcpyDeviceToDevice, h->st));
                if (want_E) {
                    rc = energy_partials(h);
                    if (rc) return rc;
                    launch_gas_esum(h->N, h->P, h->d_epart, 1.0, 1.0, false,
                                    h->d_Eloss + (size_t)(k - 1) * (h->P + 1), h->st);
                    h->launches++;
                }
                if (want_R) {
                    rc = rdf_point(h, false, h->d_rdf_loss + (k - 1));
                    if (rc) return rc;
                }
            }
        }
        if (h->ktime && (stp & 1023) == 0) {
            rc = check_status(h);
            if (rc) return rc;
        }
    }
    rc = check_status(h);
    if (rc) return rc;
    h->fwd_steps = n_steps;
    h->fwd_nl = n_steps_loss;
    h->fwd_blocks = n_steps / n_steps_loss;
    h->fwd_dt = dt;
    h->fwd_gamma = gamma;
    rc = read_centres(h);
    if (rc) return rc;
    h->fwd_has_E = want_E;
    h->Eloss.assign(h->fwd_blocks, 0.0);
    if (want_E && h->fwd_blocks > 0) {
        std::vector<double> e((size_t)h->fwd_blocks * (h->P + 1));
        CK(cudaMemcpyAsync(e.data(), h->d_Eloss, e.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        for (int b = 0; b < h->fwd_blocks; b++) h->Eloss[b] = e[(size_t)b * (h->P + 1)];
    }
    h->fwd_has_R = want_R;
    h->Rloss.assign(h->fwd_blocks, 0.0);
    if (want_R && h->fwd_blocks > 0) {
        CK(cudaMemcpyAsync(h->Rloss.data(), h->d_rdf_loss, sizeof(double) * h->fwd_blocks,
                           cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    h->fwd_valid = true;
    if (centres) std::copy(h->centres.begin(), h->centres.end(), centres);
    double D = 0.0, l_diff = 0.0, l_ev = 0.0, l_rdf = 0.0;
    if (h->fwd_blocks >= 2 && h->ng > 0)
        D = diffusion_D(h->centres, h->fwd_blocks, h->ng, h->L, n_steps_loss * dt, nullptr) * 1e-6;
    if (calc_loss) {
        if (loss_type & REVSIM_GAS_DIFF) l_diff = kDiffWeight * (D - kDiffExp) * (D - kDiffExp);
        if (want_E) {
            double s = 0.0;
            for (int b = 0; b < h->fwd_blocks; b++) {
                const double e = ev_err(h, h->Eloss[b]);
                s += e * e;
            }
            l_ev = kLossWeightEv * s / n_blocks;
        }
        if (want_R) {
            double s = 0.0;
            for (int b = 0; b < h->fwd_blocks; b++) s += h->Rloss[b];
            l_rdf = kLossWeightRdf * s / n_blocks;
        }
    }
    if (loss) *loss = l_diff + l_rdf + l_ev;
    if (parts) {
        parts[0] = D;
        parts[1] = l_diff;
        parts[2] = l_rdf;
        parts[3] = l_ev;
    }
    return REVSIM_OK;
}

int32_t revsim_gas_reverse(revsim_gas_handle *h, const uint64_t *seeds, double gamma, int32_t n_steps,
                           int32_t n_steps_loss, int32_t n_steps_trunc, double dt, int32_t loss_type,
                           double *loss, double *dl_dp, double *parts) {
    if (!h) return REVSIM_ERR_BADARG;
    if (!dl_dp) return fail(h, REVSIM_ERR_BADARG, "null output");
    if (!h->fwd_valid) return fail(h, REVSIM_ERR_STATE, "no forward pass to reverse");
    if (n_steps != h->fwd_steps || n_steps_loss != h->fwd_nl || dt != h->fwd_dt || gamma != h->fwd_gamma)
        return fail(h, REVSIM_ERR_BADARG, "reverse arguments differ from the forward pass");
    if (n_steps < 1 || n_steps_trunc < 1 || !seeds) return fail(h, REVSIM_ERR_BADARG, "bad step arguments");
    if (loss_type & ~(REVSIM_GAS_DIFF | REVSIM_GAS_RDF | REVSIM_GAS_EV))
        return fail(h, REVSIM_ERR_BADARG, "unknown loss_type bits");
    const int n_blocks = n_steps / n_steps_loss;
    if (n_blocks < 1) return fail(h, REVSIM_ERR_BADARG, "no loss point to reverse from");
    if ((loss_type & REVSIM_GAS_DIFF) && (n_blocks < 2 || h->ng < 1))
        return fail(h, REVSIM_ERR_BADARG, "the diffusion loss needs two loss points and gas molecules");
    if ((loss_type & REVSIM_GAS_EV) && !h->fwd_has_E)
        return fail(h, REVSIM_ERR_STATE, "the forward pass did not record the enthalpy term");
    if ((loss_type & REVSIM_GAS_RDF) && (!h->fwd_has_R || h->rdf.empty()))
        return fail(h, REVSIM_ERR_STATE, "the forward pass did not record the RDF term");
    CK(cudaSetDevice(h->dev));
    const size_t n3 = 3 * (size_t)h->N, fsz = 3 * (size_t)h->ng;
    const double c = std::exp(-gamma * dt), sn = std::sqrt(1 - c * c);
    const double lf = n_steps_loss * dt;
    std::vector<double> dgc;
    double D = 0.0, l_diff = 0.0;
    if (n_blocks >= 2 && h->ng > 0) D = diffusion_D(h->centres, n_blocks, h->ng, h->L, lf, &dgc) * 1e-6;
    if (loss_type & REVSIM_GAS_DIFF) {
        l_diff = kDiffWeight * (D - kDiffExp) * (D - kDiffExp);
        const double dl_dD = kDiffWeight * 2 * (D - kDiffExp) * 1e-6;
        for (double &g : dgc) g *= dl_dD;
    } else {
        dgc.assign(fsz * (size_t)n_blocks, 0.0);
    }
    CK(cudaMemsetAsync(h->d_part, 0, (size_t)h->N * h->P * sizeof(double), h->st));
    CK(cudaMemsetAsync(h->d_direct, 0, (h->P + 1) * sizeof(double), h->st));
    // the end state (fwd_coords_logger[end], diffusion.jl:1557-1558)
    CK(cudaMemcpyAsync(h->d_x, h->d_snap_x + (size_t)n_blocks * n3, n3 * sizeof(double),
                       cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->d_v, h->d_snap_v + (size_t)n_blocks * n3, n3 * sizeof(double),
                       cudaMemcpyDeviceToDevice, h->st));
    h->cur = 0;
    int rc = pack(h);
    if (!rc) rc = rebuild(h);
    if (rc) return rc;
    double l_ev = 0.0, lp = 0.0, l_rdf = 0.0, lr = 0.0;
    rc = point_grad(h, loss_type, n_blocks, h->Eloss.empty() ? 0.0 : h->Eloss[n_blocks - 1],
                    h->Rloss.empty() ? 0.0 : h->Rloss[n_blocks - 1],
                    dgc.empty() ? nullptr : dgc.data() + fsz * (n_blocks - 1), &lp, &lr);
    if (!rc) rc = reset_accums(h, c);
    if (rc) return rc;
    l_ev += lp;
    l_rdf += lr;
    for (int lc = 1; lc <= n_blocks; lc++) {
        const int s_start = n_steps - (lc - 1) * n_steps_loss;
        const int s_end = std::max(s_start - n_steps_trunc + 1, 1);
        {
            // part 1 of the block's first step, in place
            GasArgs a = args(h);
            a.dt = dt;
            a.c = c;
            a.s = sn;
            a.seed_next = seeds[s_start - 1];
            a.pos_out = h->d_pos[h->cur];
            a.pos64_out = h->d_pos64[h->cur];
            a.wgt_out = h->d_wgt[h->cur];
            launch_gas_part1(h->mixed, a, h->st);
            h->launches++;
            CK(cudaGetLastError());
        }
        for (int sn_ = s_start; sn_ >= s_end; sn_--) {
            if (sn_ % h->nf == 0) {   // diffusion.jl:1574
                rc = rebuild(h);
                if (rc) return rc;
            }
            GasArgs a = args(h);
            a.dt = dt;
            a.c = c;
            a.s = sn;
            a.mode = sn_ > s_end ? rs::MODE_FUSE_NEXT : 0;
            a.seed_next = sn_ > s_end ? seeds[sn_ - 2] : 0;
            rc = step(h, true, a);
            if (rc) return rc;
            if (sn_ > s_end) h->cur ^= 1;
        }
        if (lc != n_blocks) {
            // snapshot restore and the loss point of the next block (diffusion.jl:1589-1605)
            const int k = n_blocks - lc;
            CK(cudaMemcpyAsync(h->d_x, h->d_snap_x + (size_t)k * n3, n3 * sizeof(double),
                               cudaMemcpyDeviceToDevice, h->st));
            CK(cudaMemcpyAsync(h->d_v, h->d_snap_v + (size_t)k * n3, n3 * sizeof(double),
                               cudaMemcpyDeviceToDevice, h->st));
            rc = pack(h);
            if (!rc) rc = rebuild(h);
            if (!rc)
                rc = point_grad(h, loss_type, n_blocks, h->Eloss.empty() ? 0.0 : h->Eloss[k - 1],
                                h->Rloss.empty() ? 0.0 : h->Rloss[k - 1],
                                dgc.empty() ? nullptr : dgc.data() + fsz * (k - 1), &lp, &lr);
            if (!rc) rc = reset_accums(h, c);
            if (rc) return rc;
            l_ev += lp;
            l_rdf += lr;
        }
        if (h->ktime) {
            rc = check_status(h);
            if (rc) return rc;
        }
    }
    std::vector<double> part((size_t)h->N * h->P), direct(h->P + 1);
    CK(cudaMemcpyAsync(part.data(), h->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(direct.data(), h->d_direct, direct.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    rc = check_status(h);
    if (rc) return rc;
    for (int p = 0; p < h->P; p++) dl_dp[p] = direct[1 + p];
    for (int i = 0; i < h->N; i++)
        for (int p = 0; p < h->P; p++) dl_dp[p] += part[(size_t)i * h->P + p];
    h->fwd_valid = false;
    if (loss) *loss = l_diff + l_rdf + l_ev;
    if (parts) {
        parts[0] = D;
        parts[1] = l_diff;
        parts[2] = l_rdf;
        parts[3] = l_ev;
    }
    return REVSIM_OK;
}

void *revsim_gas_stream(revsim_gas_handle *h) { return h ? (void *)h->st : nullptr; }

int64_t revsim_gas_launch_count(const revsim_gas_handle *h) { return h ? h->launches : 0; }

int32_t revsim_gas_set_kernel_timing(revsim_gas_handle *h, int32_t enable) {
    if (!h) return REVSIM_ERR_BADARG;
    h->ktime = enable != 0;
    h->kt_ms[0] = h->kt_ms[1] = 0.0;
    h->kt_n[0] = h->kt_n[1] = 0;
    h->ev_used[0] = h->ev_used[1] = 0;
    return REVSIM_OK;
}

int32_t revsim_gas_kernel_time(revsim_gas_handle *h, int32_t which, double *total_ms, int64_t *launches) {
    if (!h || which < 0 || which > 1) return REVSIM_ERR_BADARG;
    if (total_ms) *total_ms = h->kt_ms[which];
    if (launches) *launches = h->kt_n[which];
    return REVSIM_OK;
}

}  // extern "C"
