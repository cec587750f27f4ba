/*
 * sw_oracle.c -- CPU FP64 restatement of the Stillinger-Weber diamond path of
 * greener-group/rev-sim diamond/diamond.jl (see sw_oracle.h).  TEST INFRASTRUCTURE ONLY.
 *
 * Terms: a 2-body term for every pair with r/sigma < a; a 3-body term for every centre c
 * and every pair {j, k} of its neighbours with r/sigma < a (the reference enumerates each
 * triplet once with its three centres, diamond.jl:463-527, which is the same set).
 * Derivatives by complex step (sw_oracle.h).
 */
#include "sw_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "mlp_oracle.h"
#include "revsim_oracle.h"

typedef double complex cplx;
static const double kH = 1e-30;   /* complex-step size */

int32_t orc_sw_n_params(const orc_sw_system *s) { return ORC_SW_NP + (s->mlp ? ORC_MLP_PER_TYPE : 0); }

/* ---------------------------------------------------------- learned radial term */
static const double kMlpHinv = ORC_MLP_NG / ORC_SW_MLP_RC;

/* Interval coefficients [NG][4] of the learned term, or NULL without it. */
static double *mlp_coef(const orc_sw_system *s, const double *theta) {
    if (!s->mlp) return NULL;
    double *c = (double *)malloc(sizeof(double) * ORC_MLP_NG * 4);
    orc_mlp_table_n(theta + ORC_SW_NP, 1, ORC_SW_MLP_RC, ORC_SW_MLP_WIDTH, c);
    return c;
}

static inline int mlp_seg(double r) {
    int g = (int)floor(r * kMlpHinv);
    return g < 0 ? 0 : (g > ORC_MLP_NG - 1 ? ORC_MLP_NG - 1 : g);
}

static double mlp_e(const double *coef, double r) {
    const int g = mlp_seg(r);
    const double sv = r * kMlpHinv - g, *c = coef + 4 * g;
    return c[0] + sv * (c[1] + sv * (c[2] + sv * c[3]));
}

/* g_j = u'(r) d / r for d = x_j - x_i: u' is a cubic in r on the interval of the real
 * distance, so the complex step through it is exact. */
static void mlp_g(const cplx d[3], const double *coef, cplx gj[3]) {
    const cplx r = csqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const int g = mlp_seg(creal(r));
    const cplx sv = r * kMlpHinv - g;
    const double *c = coef + 4 * g;
    const cplx du = (c[1] + sv * (2.0 * c[2] + 3.0 * sv * c[3])) * kMlpHinv;
    for (int u = 0; u < 3; u++) gj[u] = du * d[u] / r;
}

/* adj[g][k] += wgt d u'(r) / dc_k = wgt k s^(k-1) / h  (k = 1..3; c_0 does not enter u'). */
static void mlp_adj(double r, double wgt, double *adj) {
    const int g = mlp_seg(r);
    const double sv = r * kMlpHinv - g, w = wgt * kMlpHinv;
    adj[4 * g + 1] += w;
    adj[4 * g + 2] += 2.0 * w * sv;
    adj[4 * g + 3] += 3.0 * w * sv * sv;
}

/* ----------------------------------------------------------------- terms */
/* 2-body gradient g_j = dE2/dx_j for d = x_j - x_i (g_i = -g_j), diamond.jl:348-356 and
 * 450-458: E2 = eps A (B s^-4 - 1) exp(1/(s - a)), s = r/sigma. */
static void sw2_g(const cplx d[3], const cplx p[ORC_SW_NP], cplx gj[3]) {
    const cplx A = p[0], B = p[1], a = p[2], sig = p[5], eps = p[6];
    const cplx r = csqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const cplx s = r / sig, sa = s - a;
    const cplx e = cexp(1.0 / sa);
    const cplx s2 = s * s, s4 = s2 * s2, s5 = s4 * s;
    const cplx dEds = -eps * A * e * (4.0 * B / s5 + (B / s4 - 1.0) / (sa * sa));
    const cplx f = dEds / sig / r;
    for (int u = 0; u < 3; u++) gj[u] = f * d[u];
}

static double sw2_e(const double d[3], const double *p) {
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), s = r / p[5];
    return p[6] * p[0] * (p[1] / (s * s * s * s) - 1.0) * exp(1.0 / (s - p[2]));
}

/* 3-body gradients for centre c with dj = x_j - x_c, dk = x_k - x_c (diamond.jl:360-379,
 * 479-491): E3 = eps lambda exp(gamma/(s1 - a) + gamma/(s2 - a)) (cos theta + 1/3)^2. */
static void sw3_g(const cplx dj[3], const cplx dk[3], const cplx p[ORC_SW_NP], cplx gj[3],
                  cplx gk[3]) {
    const cplx a = p[2], lam = p[3], gam = p[4], sig = p[5], eps = p[6];
    const cplx rj = csqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]);
    const cplx rk = csqrt(dk[0] * dk[0] + dk[1] * dk[1] + dk[2] * dk[2]);
    const cplx s1a = rj / sig - a, s2a = rk / sig - a;
    const cplx e = cexp(gam / s1a + gam / s2a);
    const cplx dot = dj[0] * dk[0] + dj[1] * dk[1] + dj[2] * dk[2];
    const cplx cth = dot / (rj * rk), c = cth + 1.0 / 3.0;
    const cplx dEds1 = eps * lam * c * c * e * (-gam / (s1a * s1a));
    const cplx dEds2 = eps * lam * c * c * e * (-gam / (s2a * s2a));
    const cplx dEdc = 2.0 * eps * lam * e * c;
    for (int u = 0; u < 3; u++) {
        const cplx dcj = dk[u] / (rj * rk) - cth * dj[u] / (rj * rj);
        const cplx dck = dj[u] / (rj * rk) - cth * dk[u] / (rk * rk);
        gj[u] = dEds1 / sig * dj[u] / rj + dEdc * dcj;
        gk[u] = dEds2 / sig * dk[u] / rk + dEdc * dck;
    }
}

static double sw3_e(const double dj[3], const double dk[3], const double *p) {
    const double rj = sqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]);
    const double rk = sqrt(dk[0] * dk[0] + dk[1] * dk[1] + dk[2] * dk[2]);
    const double c = (dj[0] * dk[0] + dj[1] * dk[1] + dj[2] * dk[2]) / (rj * rk) + 1.0 / 3.0;
    return p[6] * p[3] * exp(p[4] / (rj / p[5] - p[2]) + p[4] / (rk / p[5] - p[2])) * c * c;
}

/* --------------------------------------------------------------- neighbours */
typedef struct {
    int32_t n, cap;
    int32_t *cnt;    /* [n] */
    int32_t *idx;    /* [n * cap] */
    double *d;       /* [n * cap * 3] min-image x_j - x_i */
} nbrs;

static void mi3(const double *xi, const double *xj, double L, double *d) {
    for (int u = 0; u < 3; u++) d[u] = orc_vec1d(xi[u], xj[u], L);
}

static void build_nbrs(const orc_sw_system *s, const double *p, const double *x, nbrs *nb) {
    const int n = s->n_atoms;
    const double rc = p[2] * p[5];   /* a sigma: s < a  <=>  r < a sigma */
    nb->n = n;
    nb->cap = 64;
    nb->cnt = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    nb->idx = (int32_t *)malloc(sizeof(int32_t) * (size_t)n * nb->cap);
    nb->d = (double *)malloc(sizeof(double) * 3 * (size_t)n * nb->cap);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            double d[3];
            mi3(x + 3 * i, x + 3 * j, s->box, d);
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (r / p[5] < p[2] && nb->cnt[i] < nb->cap) {
                const int q = nb->cnt[i]++;
                nb->idx[i * nb->cap + q] = j;
                memcpy(nb->d + 3 * ((size_t)i * nb->cap + q), d, sizeof(d));
            }
            (void)rc;
        }
    }
}

static void free_nbrs(nbrs *nb) {
    free(nb->cnt);
    free(nb->idx);
    free(nb->d);
}

/* ------------------------------------------------------------------ visitor
 * Every term once, with real displacements.  mode selects the complex perturbation:
 *   0: none; 1: positions along tan[3N]; 2: parameter p_idx; 3: positions along
 *   u_a = S d_a (S = tan[0..8], d_a relative to the term's centre).
 * For each term the callback receives the atoms, their gradients (complex) and the
 * displacements of the atoms from the term's centre. */
typedef void (*term_cb)(void *ctx, int na, const int *atoms, const cplx (*g)[3],
                        const double (*dc)[3]);

static void visit_terms(const orc_sw_system *s, const double *theta, const double *coef,
                        const nbrs *nb, int mode, const double *tan, int p_idx, term_cb cb,
                        void *ctx) {
    cplx p[ORC_SW_NP];
    for (int q = 0; q < ORC_SW_NP; q++) p[q] = theta[q] + ((mode == 2 && q == p_idx) ? I * kH : 0.0);
    const int n = nb->n;
    for (int i = 0; i < n; i++) {
        const int ci = nb->cnt[i];
        for (int qa = 0; qa < ci; qa++) {
            const int j = nb->idx[i * nb->cap + qa];
            const double *dj = nb->d + 3 * ((size_t)i * nb->cap + qa);
            if (j > i) {   /* 2-body, centre i */
                cplx d[3], gj[3], g[2][3];
                double dc[2][3] = {{0, 0, 0}, {dj[0], dj[1], dj[2]}};
                for (int u = 0; u < 3; u++) {
                    double t = 0.0;
                    if (mode == 1) t = tan[3 * j + u] - tan[3 * i + u];
                    if (mode == 3) t = tan[3 * u] * dj[0] + tan[3 * u + 1] * dj[1] + tan[3 * u + 2] * dj[2];
                    d[u] = dj[u] + I * kH * t;
                }
                sw2_g(d, p, gj);
                if (coef && sqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]) < ORC_SW_MLP_RC) {
                    cplx gm[3];
                    mlp_g(d, coef, gm);
                    for (int u = 0; u < 3; u++) gj[u] += gm[u];
                }
                for (int u = 0; u < 3; u++) {
                    g[0][u] = -gj[u];
                    g[1][u] = gj[u];
                }
                const int atoms[2] = {i, j};
                cb(ctx, 2, atoms, g, dc);
            }
            for (int qb = qa + 1; qb < ci; qb++) {   /* 3-body, centre i, ends j < ... in list order */
                const int k = nb->idx[i * nb->cap + qb];
                const double *dk = nb->d + 3 * ((size_t)i * nb->cap + qb);
                cplx a[3], b[3], gj[3], gk[3], g[3][3];
                double dc[3][3] = {{0, 0, 0}, {dj[0], dj[1], dj[2]}, {dk[0], dk[1], dk[2]}};
                for (int u = 0; u < 3; u++) {
                    double ta = 0.0, tb = 0.0;
                    if (mode == 1) {
                        ta = tan[3 * j + u] - tan[3 * i + u];
                        tb = tan[3 * k + u] - tan[3 * i + u];
                    }
                    if (mode == 3) {
                        ta = tan[3 * u] * dj[0] + tan[3 * u + 1] * dj[1] + tan[3 * u + 2] * dj[2];
                        tb = tan[3 * u] * dk[0] + tan[3 * u + 1] * dk[1] + tan[3 * u + 2] * dk[2];
                    }
                    a[u] = dj[u] + I * kH * ta;
                    b[u] = dk[u] + I * kH * tb;
                }
                sw3_g(a, b, p, gj, gk);
                for (int u = 0; u < 3; u++) {
                    g[0][u] = -gj[u] - gk[u];
                    g[1][u] = gj[u];
                    g[2][u] = gk[u];
                }
                const int atoms[3] = {i, j, k};
                cb(ctx, 3, atoms, g, dc);
            }
        }
    }
}

/* ---------------------------------------------------------------- callbacks */
typedef struct { double *out; int imag; double scale; } acc_ctx;

/* out[3a+u] += scale * (imag ? Im(g)/h : Re(g)) */
static void cb_acc(void *vctx, int na, const int *atoms, const cplx (*g)[3], const double (*dc)[3]) {
    acc_ctx *c = (acc_ctx *)vctx;
    (void)dc;
    for (int q = 0; q < na; q++)
        for (int u = 0; u < 3; u++)
            c->out[3 * atoms[q] + u] += c->scale * (c->imag ? cimag(g[q][u]) / kH : creal(g[q][u]));
}

typedef struct { double W[9]; int imag; } vir_ctx;

/* W_ab += sum over the term's atoms of g_a d_b (g real part, or Im/h for a derivative) */
static void cb_vir(void *vctx, int na, const int *atoms, const cplx (*g)[3], const double (*dc)[3]) {
    vir_ctx *c = (vir_ctx *)vctx;
    (void)atoms;
    for (int q = 0; q < na; q++)
        for (int al = 0; al < 3; al++)
            for (int be = 0; be < 3; be++)
                c->W[3 * al + be] += (c->imag ? cimag(g[q][al]) / kH : creal(g[q][al])) * dc[q][be];
}

/* ----------------------------------------------------------------- public */
double orc_sw_energy(const orc_sw_system *s, const double *theta, const double *x) {
    nbrs nb;
    build_nbrs(s, theta, x, &nb);
    double *coef = mlp_coef(s, theta);
    double E = 0.0;
    for (int i = 0; i < nb.n; i++) {
        for (int qa = 0; qa < nb.cnt[i]; qa++) {
            const int j = nb.idx[i * nb.cap + qa];
            const double *dj = nb.d + 3 * ((size_t)i * nb.cap + qa);
            if (j > i) {
                E += sw2_e(dj, theta);
                const double r = sqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]);
                if (coef && r < ORC_SW_MLP_RC) E += mlp_e(coef, r);
            }
            for (int qb = qa + 1; qb < nb.cnt[i]; qb++)
                E += sw3_e(dj, nb.d + 3 * ((size_t)i * nb.cap + qb), theta);
        }
    }
    free(coef);
    free_nbrs(&nb);
    return E;
}

int64_t orc_sw_pairs(const orc_sw_system *s, const double *theta, const double *x,
                     int32_t *pairs, int64_t max_pairs) {
    nbrs nb;
    build_nbrs(s, theta, x, &nb);
    int64_t n = 0;
    for (int i = 0; i < nb.n; i++)
        for (int q = 0; q < nb.cnt[i]; q++) {
            const int j = nb.idx[i * nb.cap + q];
            if (j <= i) continue;
            if (n < max_pairs) {
                pairs[2 * n] = i;
                pairs[2 * n + 1] = j;
            }
            n++;
        }
    free_nbrs(&nb);
    return n;
}

void orc_sw_forces(const orc_sw_system *s, const double *theta, const double *x, double *F) {
    orc_sw_forces_grads(s, theta, x, NULL, F, NULL, NULL);
}

void orc_sw_forces_grads(const orc_sw_system *s, const double *theta, const double *x,
                         const double *w, double *F, double *dl_dfi, double *dF_dp) {
    const int n3 = 3 * s->n_atoms;
    nbrs nb;
    build_nbrs(s, theta, x, &nb);
    double *coef = mlp_coef(s, theta);
    memset(F, 0, sizeof(double) * n3);
    acc_ctx c = {F, 0, -1.0};
    visit_terms(s, theta, coef, &nb, 0, NULL, 0, cb_acc, &c);
    if (dl_dfi && w) {
        /* J (w/m): the tangent of F along w/m; J is symmetric (a Hessian) */
        double *t = (double *)malloc(sizeof(double) * n3);
        for (int e = 0; e < n3; e++) t[e] = w[e] / s->mass;
        memset(dl_dfi, 0, sizeof(double) * n3);
        acc_ctx cg = {dl_dfi, 1, -1.0};
        visit_terms(s, theta, coef, &nb, 1, t, 0, cb_acc, &cg);
        free(t);
    }
    if (dF_dp) {
        double *col = (double *)malloc(sizeof(double) * n3);
        for (int p = 0; p < ORC_SW_NP; p++) {
            memset(col, 0, sizeof(double) * n3);
            acc_ctx cp = {col, 1, -1.0};
            visit_terms(s, theta, coef, &nb, 2, NULL, p, cb_acc, &cp);
            for (int e = 0; e < n3; e++) dF_dp[e * ORC_SW_NP + p] = col[e];
        }
        free(col);
    }
    free(coef);
    free_nbrs(&nb);
}

/* Learned-term coefficient adjoints of sum_a acoef_a . dF_a/dc: per pair F_j = -g_j,
 * F_i = g_j, so the weight is -(acoef_j - acoef_i) . d / r. */
static void mlp_contract_adj(const orc_sw_system *s, const nbrs *nb, const double *acoef, double *adj) {
    for (int i = 0; i < nb->n; i++)
        for (int q = 0; q < nb->cnt[i]; q++) {
            const int j = nb->idx[i * nb->cap + q];
            if (j <= i) continue;
            const double *d = nb->d + 3 * ((size_t)i * nb->cap + q);
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (!(r < ORC_SW_MLP_RC)) continue;
            double zu = 0.0;
            for (int u = 0; u < 3; u++) zu += (acoef[3 * j + u] - acoef[3 * i + u]) * d[u] / r;
            mlp_adj(r, -zu, adj);
        }
    (void)s;
}

void orc_sw_contract(const orc_sw_system *s, const double *theta, const double *x,
                     const double *acoef, double *dtheta) {
    const int n3 = 3 * s->n_atoms, P = orc_sw_n_params(s);
    double *F = (double *)malloc(sizeof(double) * n3);
    double *J = (double *)malloc(sizeof(double) * n3 * ORC_SW_NP);
    orc_sw_forces_grads(s, theta, x, NULL, F, NULL, J);
    for (int p = 0; p < P; p++) dtheta[p] = 0.0;
    for (int p = 0; p < ORC_SW_NP; p++)
        for (int e = 0; e < n3; e++) dtheta[p] += acoef[e] * J[e * ORC_SW_NP + p];
    if (s->mlp) {
        nbrs nb;
        build_nbrs(s, theta, x, &nb);
        double *adj = (double *)calloc(ORC_MLP_NG * 4, sizeof(double));
        mlp_contract_adj(s, &nb, acoef, adj);
        orc_mlp_backprop_n(theta + ORC_SW_NP, 1, ORC_SW_MLP_RC, ORC_SW_MLP_WIDTH, adj, dtheta + ORC_SW_NP);
        free(adj);
        free_nbrs(&nb);
    }
    free(F);
    free(J);
}

/* Kinetic tensor -sum m (v - vbar)(v - vbar)^T (diamond.jl:754-756). */
static void kinetic(const orc_sw_system *s, const double *v, double K[9], double vbar[3]) {
    const int n = s->n_atoms;
    vbar[0] = vbar[1] = vbar[2] = 0.0;
    for (int a = 0; a < n; a++)
        for (int u = 0; u < 3; u++) vbar[u] += v[3 * a + u];
    for (int u = 0; u < 3; u++) vbar[u] /= n;
    for (int q = 0; q < 9; q++) K[q] = 0.0;
    for (int a = 0; a < n; a++)
        for (int al = 0; al < 3; al++)
            for (int be = 0; be < 3; be++)
                K[3 * al + be] -= s->mass * (v[3 * a + al] - vbar[al]) * (v[3 * a + be] - vbar[be]);
}

void orc_sw_stress(const orc_sw_system *s, const double *theta, const double *x, const double *v,
                   int32_t vel_term, double *sigma) {
    nbrs nb;
    build_nbrs(s, theta, x, &nb);
    double *coef = mlp_coef(s, theta);
    vir_ctx c;
    memset(&c, 0, sizeof(c));
    visit_terms(s, theta, coef, &nb, 0, NULL, 0, cb_vir, &c);
    free(coef);
    double K[9], vb[3];
    kinetic(s, v, K, vb);
    const double V = s->box * s->box * s->box;
    for (int q = 0; q < 9; q++) sigma[q] = ((vel_term ? K[q] : 0.0) + c.W[q]) / V;
    free_nbrs(&nb);
}

double orc_sw_loss_grad(const orc_sw_system *s, const double *theta, const orc_sw_loss *L,
                        const double *x, const double *v, double *dLdx, double *dLdv,
                        double *dLdp) {
    const int n = s->n_atoms, n3 = 3 * n;
    const double V = s->box * s->box * s->box;
    double sig[9];
    orc_sw_stress(s, theta, x, v, L->vel_term, sig);
    double loss = 0.0, S[9];
    for (int q = 0; q < 9; q++) {
        const double e = sig[q] - L->target[q];
        loss += e * e;
        S[q] = 2.0 * L->weight * e / 9.0;   /* dL/dsigma */
    }
    loss *= L->weight / 9.0;
    if (dLdv) {
        memset(dLdv, 0, sizeof(double) * n3);
        if (L->vel_term) {
            double K[9], vb[3];
            kinetic(s, v, K, vb);
            for (int a = 0; a < n; a++)
                for (int g = 0; g < 3; g++) {
                    double t = 0.0;
                    for (int b = 0; b < 3; b++)
                        t += (S[3 * g + b] + S[3 * b + g]) * (v[3 * a + b] - vb[b]);
                    dLdv[3 * a + g] = -s->mass * t / V;
                }
        }
    }
    if (dLdx || dLdp) {
        nbrs nb;
        build_nbrs(s, theta, x, &nb);
        double *coef = mlp_coef(s, theta);
        if (dLdx) {
            /* (1/V) [ H u + S^T g ], u_a = S d_a per term */
            memset(dLdx, 0, sizeof(double) * n3);
            acc_ctx ch = {dLdx, 1, 1.0 / V};
            visit_terms(s, theta, coef, &nb, 3, S, 0, cb_acc, &ch);
            double *g = (double *)calloc((size_t)n3, sizeof(double));
            acc_ctx cg = {g, 0, 1.0};
            visit_terms(s, theta, coef, &nb, 0, NULL, 0, cb_acc, &cg);
            for (int a = 0; a < n; a++)
                for (int gm = 0; gm < 3; gm++) {
                    double t = 0.0;
                    for (int al = 0; al < 3; al++) t += S[3 * al + gm] * g[3 * a + al];
                    dLdx[3 * a + gm] += t / V;
                }
            free(g);
        }
        if (dLdp) {
            for (int p = 0; p < ORC_SW_NP; p++) {
                vir_ctx c;
                memset(&c, 0, sizeof(c));
                c.imag = 1;
                visit_terms(s, theta, coef, &nb, 2, NULL, p, cb_vir, &c);
                double t = 0.0;
                for (int q = 0; q < 9; q++) t += S[q] * c.W[q];
                dLdp[p] = t / V;
            }
            if (coef) {
                /* W += g_j (x) d per pair: dL/dc = sum_ab S_ab d_a d_b / (r V) du'/dc */
                double *adj = (double *)calloc(ORC_MLP_NG * 4, sizeof(double));
                for (int i = 0; i < nb.n; i++)
                    for (int q = 0; q < nb.cnt[i]; q++) {
                        const int j = nb.idx[i * nb.cap + q];
                        if (j <= i) continue;
                        const double *d = nb.d + 3 * ((size_t)i * nb.cap + q);
                        const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                        if (!(r < ORC_SW_MLP_RC)) continue;
                        double t = 0.0;
                        for (int al = 0; al < 3; al++)
                            for (int be = 0; be < 3; be++) t += S[3 * al + be] * d[al] * d[be];
                        mlp_adj(r, t / (r * V), adj);
                    }
                for (int p = ORC_SW_NP; p < orc_sw_n_params(s); p++) dLdp[p] = 0.0;
                orc_mlp_backprop_n(theta + ORC_SW_NP, 1, ORC_SW_MLP_RC, ORC_SW_MLP_WIDTH, adj,
                                   dLdp + ORC_SW_NP);
                free(adj);
            }
        }
        free(coef);
        free_nbrs(&nb);
    }
    return loss;
}

void orc_sw_noise(const orc_sw_system *s, uint64_t seed, double *xi) {
    const double sd = sqrt(s->kB * s->temp / s->mass);
    for (int a = 0; a < s->n_atoms; a++) {
        double z[4];
        orc_philox_normals(seed, (uint32_t)a, z);
        for (int u = 0; u < 3; u++) xi[3 * a + u] = z[u] * sd;
    }
}

/* ------------------------------------------------------------------ drivers */
double orc_sw_forward_sim(const orc_sw_system *s, const double *theta, double *x, double *v,
                          const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, int32_t n_steps_buffer, double dt,
                          const orc_sw_loss *L, int32_t calc_loss, double *snap_x, double *snap_v) {
    const int n3 = 3 * s->n_atoms;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c);
    double *F = (double *)malloc(sizeof(double) * n3), *xi = (double *)malloc(sizeof(double) * n3);
    double loss = 0.0;
    int n_blocks = 0;
    for (int step = 1; step <= n_steps; step++) {
        orc_sw_forces(s, theta, x, F);
        for (int e = 0; e < n3; e++) v[e] = v[e] + F[e] * dt / s->mass;
        for (int e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        orc_sw_noise(s, noise_seeds[step - 1], xi);
        for (int e = 0; e < n3; e++) v[e] = v[e] * c + xi[e] * sn;
        for (int e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        for (int e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], s->box);
        if ((n_steps - step) % n_steps_loss == 0 && step >= n_steps_buffer) {
            if (snap_x) {
                memcpy(snap_x + (size_t)n_blocks * n3, x, sizeof(double) * n3);
                memcpy(snap_v + (size_t)n_blocks * n3, v, sizeof(double) * n3);
            }
            n_blocks++;
            if (calc_loss && L) loss += orc_sw_loss_grad(s, theta, L, x, v, NULL, NULL, NULL);
        }
    }
    free(F);
    free(xi);
    return n_blocks ? loss / n_blocks : 0.0;
}

/* Accumulators at a loss point with g = dL/dx, h = dL/dv (diamond.jl:1789-1793). */
static void sw_reset(int n3, double c, double dt, const double *g, const double *h, double *A,
                     double *B, double *C, double *D, double *G) {
    for (int e = 0; e < n3; e++) {
        A[e] = g[e] * (1 + c) + h[e] * c * 2 / dt;
        B[e] = g[e] * (1 + c) + h[e] * (c - 1) * 2 / dt;
        C[e] = h[e] * (1 + c) / dt;
        D[e] = g[e] * (1 + 2 * c + c * c) / (2 * c) + h[e] * (c - 1 / c) / dt;
        G[e] = 0.0;
    }
}

double orc_sw_reverse_sim(const orc_sw_system *s, const double *theta, double *x, double *v,
                          const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, int32_t n_steps_trunc, int32_t n_blocks, double dt,
                          const double *snap_x, const double *snap_v, const orc_sw_loss *L,
                          double *dl_dp) {
    if (n_blocks <= 0 || n_steps_loss <= 0 || n_steps_trunc <= 0) return NAN;
    const int n = s->n_atoms, n3 = 3 * n;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c), dt2 = dt * dt;
    double *buf = (double *)calloc((size_t)n3 * 11, sizeof(double));
    double *F = buf, *xi = buf + n3, *g = buf + 2 * n3, *h = buf + 3 * n3, *A = buf + 4 * n3;
    double *B = buf + 5 * n3, *C = buf + 6 * n3, *D = buf + 7 * n3, *G = buf + 8 * n3;
    double *acoef = buf + 9 * n3, *w = buf + 10 * n3;
    const int P = orc_sw_n_params(s);
    double *dp = (double *)malloc(sizeof(double) * P);
    double *adj = s->mlp ? (double *)calloc(ORC_MLP_NG * 4, sizeof(double)) : NULL;
    double *dF_dp = (double *)malloc(sizeof(double) * n3 * ORC_SW_NP);
    double loss = orc_sw_loss_grad(s, theta, L, x, v, g, h, dp);
    for (int p = 0; p < P; p++) dl_dp[p] = dp[p];
    sw_reset(n3, c, dt, g, h, A, B, C, D, G);
    for (int lc = 1; lc <= n_blocks; lc++) {   /* diamond.jl:1799-1868 */
        const int step_start = n_steps - (lc - 1) * n_steps_loss;
        const int step_end = step_start - n_steps_trunc + 1 > 1 ? step_start - n_steps_trunc + 1 : 1;
        for (int step_n = step_start; step_n >= step_end; step_n--) {
            for (int e = 0; e < n3; e++) x[e] = x[e] - v[e] * dt / 2;
            orc_sw_noise(s, noise_seeds[step_n - 1], xi);
            for (int e = 0; e < n3; e++) v[e] = (v[e] - xi[e] * sn) / c;
            for (int e = 0; e < n3; e++) x[e] = x[e] - v[e] * dt / 2;
            for (int e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], s->box);
            for (int e = 0; e < n3; e++) D[e] = c * D[e] + dt2 * G[e] * (1 + c) / 2;
            for (int e = 0; e < n3; e++) C[e] = C[e] + D[e];
            for (int e = 0; e < n3; e++) w[e] = C[e];
            orc_sw_forces_grads(s, theta, x, w, F, G, dF_dp);
            for (int e = 0; e < n3; e++) acoef[e] = A[e] * (dt2 / (2 * s->mass));
            for (int p = 0; p < ORC_SW_NP; p++) {
                double t = 0.0;
                for (int e = 0; e < n3; e++) t += acoef[e] * dF_dp[e * ORC_SW_NP + p];
                dl_dp[p] += t;
            }
            if (adj) {
                nbrs nb;
                build_nbrs(s, theta, x, &nb);
                mlp_contract_adj(s, &nb, acoef, adj);
                free_nbrs(&nb);
            }
            for (int e = 0; e < n3; e++) v[e] = v[e] - F[e] * dt / s->mass;
            for (int e = 0; e < n3; e++) B[e] = c * B[e] + dt2 * G[e];
            for (int e = 0; e < n3; e++) A[e] = A[e] + B[e];
        }
        if (lc != n_blocks) {
            const size_t si = (size_t)(n_blocks - lc - 1) * n3;
            memcpy(x, snap_x + si, sizeof(double) * n3);
            memcpy(v, snap_v + si, sizeof(double) * n3);
            loss += orc_sw_loss_grad(s, theta, L, x, v, g, h, dp);
            for (int p = 0; p < P; p++) dl_dp[p] += dp[p];
            sw_reset(n3, c, dt, g, h, A, B, C, D, G);
        }
    }
    if (adj) orc_mlp_backprop_n(theta + ORC_SW_NP, 1, ORC_SW_MLP_RC, ORC_SW_MLP_WIDTH, adj, dl_dp + ORC_SW_NP);
    for (int p = 0; p < P; p++) dl_dp[p] /= n_blocks;
    free(buf);
    free(dF_dp);
    free(dp);
    free(adj);
    return loss / n_blocks;
}
