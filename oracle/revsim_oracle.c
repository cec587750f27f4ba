/*
 * revsim_oracle.c -- CPU FP64 restatement of greener-group/rev-sim water/water.jl.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): loaded by tests/, the smoke check and the
 * CPU-baseline leg of bench.py; never by the product path.  Parity against absolute
 * reference outputs is unpinned (no Julia toolchain, no golden vectors in the
 * reference); pinned by the reference's self-consistency identities and central FD.
 * See revsim_oracle.h for the conventions restated from Molly v0.21.1.
 *
 * Build: gcc -O2 -fPIC -shared -fopenmp -ffp-contract=off (oracle/Makefile).
 */
#include "revsim_oracle.h"
#include "mlp_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

int32_t orc_num_threads(void) {
#ifdef _OPENMP
    return (int32_t)omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int32_t n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* water.jl:121-157 (generate_inter / inter_n_params): pair-form parameter counts. */
int32_t orc_n_form_params(int32_t t) {
    switch (t) {
        case ORC_LJ: return 2;   /* sigma, eps */
        case ORC_DEXP: return 4; /* sigma, eps, alpha, beta */
        case ORC_BUCK: return 3; /* A, B, C */
        case ORC_LJSC: return 4; /* sigma, eps, alpha, lambda */
        case ORC_BUFF: return 4; /* sigma, eps, delta, gamma */
        default: return -1;
    }
}

/* + q_O, k_b, r0, k_a, theta0 (water.jl:1572-1582, n_bonded_params = 4 at :48). */
int32_t orc_n_params(int32_t t) {
    int32_t n = orc_n_form_params(t);
    return n < 0 ? -1 : n + 5;
}

int32_t orc_system_n_params(const orc_system *s) {
    int32_t n = orc_n_params(s->inter_type);
    return n < 0 ? -1 : n + (s->mlp ? ORC_MLP_NPARAMS : 0);
}

/* The MLP's interval table for the parameters (NULL when the system has no MLP). */
static double *mlp_table(const orc_system *s, const double *params) {
    if (!s->mlp) return NULL;
    double *coef = (double *)malloc(sizeof(double) * ORC_MLP_NT * ORC_MLP_NG * 4);
    orc_mlp_table(params + orc_n_params(s->inter_type), s->cutoff, coef);
    return coef;
}

/* Molly vector_1D: displacement c2 - c1 folded to the nearer image. */
double orc_vec1d(double c1, double c2, double L) {
    if (c1 < c2)
        return (c2 - c1) < (c1 - c2 + L) ? (c2 - c1) : (c2 - c1 - L);
    else
        return (c1 - c2) < (c2 - c1 + L) ? (c2 - c1) : (c2 - c1 + L);
}

/* Molly wrap_coords for one component. */
double orc_wrap1d(double c, double L) { return c - floor(c / L) * L; }

static inline void vec3(const double *xi, const double *xj, double L, double *d) {
    d[0] = orc_vec1d(xi[0], xj[0], L);
    d[1] = orc_vec1d(xi[1], xj[1], L);
    d[2] = orc_vec1d(xi[2], xj[2], L);
}

static inline double sumsq3(const double *d) { return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]; }

static inline int is_O(int64_t a) { return (a % 3) == 0; }

/* ------------------------------------------------------------------------- */
/* Neighbour pairs (Molly CellListMapNeighborFinder semantics; eligible matrix of
 * diffusion.jl:1133-1147 excludes every intramolecular pair of a water). */
int64_t orc_neighbor_pairs(const orc_system *s, const double *x, int32_t *pairs, int64_t max_pairs) {
    const int64_t n = 3 * (int64_t)s->n_mol;
    const double rc2 = s->nl_cutoff * s->nl_cutoff;
    const double L = s->box;
    /* Rows i in parallel; per-row counts, then a prefix sum keeps the (i, j) order. */
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; i++) {
        int64_t c = 0;
        for (int64_t j = i + 1; j < n; j++) {
            if (i / 3 == j / 3) continue;
            double d[3];
            vec3(x + 3 * i, x + 3 * j, L, d);
            if (sumsq3(d) <= rc2) c++;
        }
        cnt[i + 1] = c;
    }
    for (int64_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    const int64_t total = cnt[n];
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; i++) {
        int64_t k = cnt[i];
        if (k >= max_pairs) continue;
        for (int64_t j = i + 1; j < n && k < max_pairs; j++) {
            if (i / 3 == j / 3) continue;
            double d[3];
            vec3(x + 3 * i, x + 3 * j, L, d);
            if (sumsq3(d) <= rc2) {
                pairs[2 * k] = (int32_t)i;
                pairs[2 * k + 1] = (int32_t)j;
                k++;
            }
        }
    }
    free(cnt);
    return total;
}

/* ------------------------------------------------------------------------- */
/* Pair forms.  Each returns the radial force F(r) (positive = repulsive; the force
 * on atom i is -F * dr/r with dr = x_j - x_i), dF/dr, and dF/dtheta for the form's
 * own parameters.  `grads` selects the force_grads_inter! arithmetic
 * (water.jl:172-407) instead of force_inter (water.jl:160-351). */

static const double two_pow_1o6 = 1.122462048309373; /* T(2^(1/6)), water.jl:47 */

/* Buffered 14-7 force (water.jl:336-351) on complex arguments, used for the
 * complex-step derivatives d/dr and d/dtheta (exact to rounding). */
static double complex buff_F(double complex r, double complex sig, double complex eps,
                             double complex del, double complex gam) {
    double complex rm = sig * two_pow_1o6;
    double complex s = r / rm;
    double complex s6 = s * s * s * s * s * s;
    double complex s7 = s6 * s;
    double complex g7 = (1.0 + gam) / (s7 + gam);
    double complex b = (1.0 + del) / (s + del);
    double complex b7 = b * b * b * b * b * b * b;
    return (7.0 * eps / rm) * b7 * ((1.0 / (s + del)) * (g7 - 2.0) + (1.0 / (s7 + gam)) * s6 * g7);
}

/* Returns 0 if the pair form is switched off for this pair (eps or A zero, the
 * iszero gates of water.jl:161,196,244,282,337). */
static int pair_form(int type, const double *p, double r, double invr2, int grads,
                     double *F, double *dFdr, double *g) {
    switch (type) {
        case ORC_LJ: { /* water.jl:160-193 */
            double sig = p[0], eps = p[1];
            if (eps == 0.0) return 0;
            double sm = (sig + sig) / 2, em = sqrt(eps * eps);
            double six = sm * sm * invr2;
            six = six * six * six;
            double twelve = six * six;
            *F = (24 * em / r) * (2 * twelve - six);
            if (!grads) return 1;
            *dFdr = -24 * em * invr2 * (26 * twelve - 7 * six);
            g[0] = (144 * em * invr2 / sm) * (4 * twelve - six) * r;
            g[1] = *F / em;
            return 1;
        }
        case ORC_DEXP: { /* water.jl:195-241 */
            double sig = p[0], eps = p[1], al = p[2], be = p[3];
            if (eps == 0.0) return 0;
            double sm = (sig + sig) / 2, em = sqrt(eps * eps);
            double rm = sm * two_pow_1o6;
            if (!grads) {
                double k1 = be * exp(al) / (al - be);
                double k2 = al * exp(be) / (al - be);
                *F = em * (al * k1 * exp(-al * r / rm) - be * k2 * exp(-be * r / rm)) / rm;
                return 1;
            }
            double e1 = exp(-al * r / rm) * exp(al) / (al - be);
            double e2 = exp(-be * r / rm) * exp(be) / (al - be);
            double eab = em * al * be;
            if (grads) *F = eab * (e1 - e2) / rm;
            *dFdr = -eab * (al * e1 - be * e2) / (rm * rm);
            double dFdrm = eab * ((al * r - rm) * e1 - (be * r - rm) * e2) / (rm * rm * rm);
            g[0] = dFdrm * two_pow_1o6;
            g[1] = (eab * (e1 - e2) / rm) / em;
            g[2] = -em * be * ((al * (al - be) * (r - rm) + be * rm) * e1 - (be * rm) * e2) / (rm * rm * (al - be));
            g[3] = em * al * ((al * rm) * e1 - (be * (be - al) * (r - rm) + al * rm) * e2) / (rm * rm * (al - be));
            return 1;
        }
        case ORC_BUCK: { /* water.jl:243-279 */
            double A = p[0], B = p[1], C = p[2];
            if (A == 0.0) return 0;
            double Am = (A + A) / 2, Bm = (B + B) / 2, Cm = (C + C) / 2;
            double invr7 = invr2 * invr2 * invr2 / r;
            double e = exp(-Bm * r);
            *F = Am * Bm * e - 6 * Cm * invr7;
            if (!grads) return 1;
            *dFdr = -Am * Bm * Bm * e + 42 * Cm * invr7 / r;
            g[0] = Bm * e;
            g[1] = Am * (1 - Bm * r) * e;
            g[2] = -6 * invr7;
            return 1;
        }
        case ORC_LJSC: { /* water.jl:281-334 with Molly LennardJonesSoftCore, p = 2 */
            double sig = p[0], eps = p[1], al = p[2], lam = p[3];
            if (eps == 0.0) return 0;
            double sm = (sig + sig) / 2, em = sqrt(eps * eps);
            double lp = lam * lam;              /* lambda^p, p = 2 */
            double s6fac = al * lp;             /* sigma6_fac = alpha * lambda^p */
            double s5 = sm * sm * sm * sm * sm, s6 = s5 * sm, s12 = s6 * s6;
            double r4 = r * r * r * r, r5 = r4 * r, r6 = r5 * r;
            double rsc6 = r6 + s6 * s6fac, rsc6m = r6 - s6 * s6fac;
            double rsc12 = rsc6 * rsc6, rsc24 = rsc12 * rsc12;
            double inv_rsc6 = 1.0 / rsc6;
            double inv_rsc = sqrt(cbrt(inv_rsc6));
            double six = s6 * inv_rsc6;
            double q = r * inv_rsc;
            *F = (24 * em * inv_rsc) * (2 * six * six - six) * (q * q * q * q * q);
            if (!grads) return 1;
            *dFdr = (24 * em * s6 * r4) * (rsc12 + 6 * rsc6 * rsc6m - 36 * r6 * s6 + 10 * s6 * rsc6) / rsc24;
            g[0] = -144 * em * r5 * s5 * (rsc6 * rsc6m + 2 * al * s12 * lp - 4 * r6 * s6) / rsc24;
            g[1] = *F / em;
            g[2] = 48 * em * r5 * s12 * lp * (rsc6 - 3 * s6) / rsc24;
            g[3] = 48 * em * r5 * s12 * al * 2 * lam * (rsc6 - 3 * s6) / rsc24;
            return 1;
        }
        case ORC_BUFF: { /* water.jl:336-407, derivatives by complex step */
            double sig = p[0], eps = p[1], del = p[2], gam = p[3];
            if (eps == 0.0) return 0;
            double sm = (sig + sig) / 2, em = sqrt(eps * eps);
            const double h = 1e-30;
            *F = creal(buff_F(r, sm, em, del, gam));
            if (!grads) return 1;
            *dFdr = cimag(buff_F(r + I * h, sm, em, del, gam)) / h;
            g[0] = cimag(buff_F(r, sm + I * h, em, del, gam)) / h;
            g[1] = cimag(buff_F(r, sm, em + I * h, del, gam)) / h;
            g[2] = cimag(buff_F(r, sm, em, del + I * h, gam)) / h;
            g[3] = cimag(buff_F(r, sm, em, del, gam + I * h)) / h;
            return 1;
        }
    }
    return 0;
}

int32_t orc_pair_form(int32_t type, const double *p, double r, double invr2, int32_t grads,
                      double *F, double *dFdr, double *g) {
    return pair_form(type, p, r, invr2, grads, F, dFdr, g);
}

/* Pair-form potential energy (Molly potential_energy for LJ / soft-core, and
 * water.jl:409-526 for the others); used by the FD consistency tests only. */
static double pair_form_energy(int type, const double *p, double r) {
    switch (type) {
        case ORC_LJ: {
            if (p[1] == 0.0) return 0.0;
            double sr6 = pow(p[0] / r, 6);
            return 4 * p[1] * (sr6 * sr6 - sr6);
        }
        case ORC_DEXP: {
            if (p[1] == 0.0) return 0.0;
            double rm = p[0] * two_pow_1o6, al = p[2], be = p[3];
            double k1 = be * exp(al) / (al - be), k2 = al * exp(be) / (al - be);
            return p[1] * (k1 * exp(-al * r / rm) - k2 * exp(-be * r / rm));
        }
        case ORC_BUCK: {
            if (p[0] == 0.0) return 0.0;
            return p[0] * exp(-p[1] * r) - p[2] / pow(r, 6);
        }
        case ORC_LJSC: {
            if (p[1] == 0.0) return 0.0;
            double s6 = pow(p[0], 6);
            double six = s6 / (pow(r, 6) + s6 * p[2] * p[3] * p[3]);
            return 4 * p[1] * (six * six - six);
        }
        case ORC_BUFF: {
            if (p[1] == 0.0) return 0.0;
            double rm = p[0] * two_pow_1o6, d = p[2], gm = p[3];
            double s = r / rm;
            return p[1] * pow((1 + d) / (s + d), 7) * ((1 + gm) / (pow(s, 7) + gm) - 2);
        }
    }
    return 0.0;
}

double orc_pair_form_energy(int32_t type, const double *p, double r) {
    return pair_form_energy(type, p, r);
}

/* The pair-form energies on complex parameters (the same expressions as
 * pair_form_energy): dE/dtheta_k = Im E(theta + i h e_k) / h, exact to rounding. */
static double complex cpow6(double complex z) {
    double complex z2 = z * z;
    return z2 * z2 * z2;
}

static double complex pair_form_energy_c(int type, const double complex *p, double r) {
    switch (type) {
        case ORC_LJ: {
            double complex sr6 = cpow6(p[0] / r);
            return 4 * p[1] * (sr6 * sr6 - sr6);
        }
        case ORC_DEXP: {
            double complex rm = p[0] * two_pow_1o6, al = p[2], be = p[3];
            double complex k1 = be * cexp(al) / (al - be), k2 = al * cexp(be) / (al - be);
            return p[1] * (k1 * cexp(-al * r / rm) - k2 * cexp(-be * r / rm));
        }
        case ORC_BUCK:
            return p[0] * cexp(-p[1] * r) - p[2] / pow(r, 6);
        case ORC_LJSC: {
            double complex s6 = cpow6(p[0]);
            double complex six = s6 / (pow(r, 6) + s6 * p[2] * p[3] * p[3]);
            return 4 * p[1] * (six * six - six);
        }
        case ORC_BUFF: {
            double complex rm = p[0] * two_pow_1o6, d = p[2], gm = p[3];
            double complex s = r / rm, b = (1 + d) / (s + d);
            double complex b7 = cpow6(b) * b, s7 = cpow6(s) * s;
            return p[1] * b7 * ((1 + gm) / (s7 + gm) - 2);
        }
    }
    return 0.0;
}

/* ------------------------------------------------------------------------- */
/* Forward-mode dual numbers for the angle-term Jacobian-vector product.  The
 * Hessian of a potential is symmetric, so J w (tangent of the force along w)
 * equals the reference's hand-expanded J^T w block (water.jl:1359-1419). */
typedef struct { double v, d; } dual;

static inline dual D(double v, double d) { dual r = {v, d}; return r; }
static inline dual dadd(dual a, dual b) { return D(a.v + b.v, a.d + b.d); }
static inline dual dsub(dual a, dual b) { return D(a.v - b.v, a.d - b.d); }
static inline dual dmul(dual a, dual b) { return D(a.v * b.v, a.d * b.v + a.v * b.d); }
static inline dual ddiv(dual a, dual b) { return D(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
static inline dual dsqrt(dual a) { double s = sqrt(a.v); return D(s, a.d / (2 * s)); }
static inline dual dacos(dual a) { return D(acos(a.v), -a.d / sqrt(1 - a.v * a.v)); }
static inline dual dneg(dual a) { return D(-a.v, -a.d); }

static inline void dcross(const dual *a, const dual *b, dual *c) {
    c[0] = dsub(dmul(a[1], b[2]), dmul(a[2], b[1]));
    c[1] = dsub(dmul(a[2], b[0]), dmul(a[0], b[2]));
    c[2] = dsub(dmul(a[0], b[1]), dmul(a[1], b[0]));
}
static inline dual ddot(const dual *a, const dual *b) {
    return dadd(dadd(dmul(a[0], b[0]), dmul(a[1], b[1])), dmul(a[2], b[2]));
}

/* Harmonic angle i-j-k (j central), water.jl:936-968 / 1316-1356.  Inputs: min-image
 * a = vector(x_j, x_i), b = vector(x_j, x_k) with tangents ta = w_i - w_j,
 * tb = w_k - w_j.  Outputs force on i, k (F_j = -F_i - F_k) with tangents, and the
 * unit-force directions p1d, p3d (for dF/dk_a, dF/dtheta0).  Returns 0 when the
 * cross product vanishes (the reference skips the angle). */
static int angle_term(const double *a_, const double *b_, const double *ta, const double *tb,
                      double ka, double th0, dual *Fi, dual *Fk, double *p1d_out,
                      double *p3d_out, double *disp_out) {
    dual a[3], b[3], cr[3], p1u[3], p3u[3], t[3];
    for (int u = 0; u < 3; u++) {
        a[u] = D(a_[u], ta ? ta[u] : 0.0);
        b[u] = D(b_[u], tb ? tb[u] : 0.0);
    }
    dual ra = dsqrt(ddot(a, a)), rb = dsqrt(ddot(b, b));
    dcross(a, b, cr);
    if (cr[0].v == 0.0 && cr[1].v == 0.0 && cr[2].v == 0.0) return 0;
    dcross(a, cr, p1u);
    dcross(b, cr, t);
    for (int u = 0; u < 3; u++) p3u[u] = dneg(t[u]);
    dual n1 = dsqrt(ddot(p1u, p1u)), n3 = dsqrt(ddot(p3u, p3u));
    dual cth = ddiv(ddot(a, b), dmul(ra, rb));
    dual th = dacos(cth);
    dual F = dmul(D(ka, 0.0), dsub(D(th0, 0.0), th));
    for (int u = 0; u < 3; u++) {
        dual p1d = ddiv(ddiv(p1u[u], n1), ra);
        dual p3d = ddiv(ddiv(p3u[u], n3), rb);
        Fi[u] = dmul(F, p1d);
        Fk[u] = dmul(F, p3d);
        if (p1d_out) p1d_out[u] = p1d.v;
        if (p3d_out) p3d_out[u] = p3d.v;
    }
    if (disp_out) *disp_out = th0 - th.v;
    return 1;
}

int32_t orc_angle_term(const double a[3], const double b[3], const double ta[3],
                       const double tb[3], double ka, double th0, double Fi[3], double Fk[3],
                       double dFi[3], double dFk[3]) {
    dual Fid[3], Fkd[3];
    if (!angle_term(a, b, ta, tb, ka, th0, Fid, Fkd, NULL, NULL, NULL)) return 0;
    for (int u = 0; u < 3; u++) {
        Fi[u] = Fid[u].v;
        Fk[u] = Fkd[u].v;
        dFi[u] = Fid[u].d;
        dFk[u] = Fkd[u].d;
    }
    return 1;
}

/* The complex-parameter energy for callers in this library (the gas restatement's
 * complex-step dE/dtheta through the mixing rules). */
double complex orc_pair_form_energy_cx(int32_t type, const double complex *p, double r) {
    return pair_form_energy_c(type, p, r);
}

/* ------------------------------------------------------------------------- */
typedef struct {
    int P, nf;             /* total and pair-form parameter counts */
    double qO, qH, kb, r0, ka, th0;
} wparams;

static wparams unpack(const orc_system *s, const double *params) {
    wparams w;
    w.nf = orc_n_form_params(s->inter_type);
    w.P = w.nf + 5;
    w.qO = params[w.nf];
    w.qH = -w.qO / 2;               /* water.jl:549 */
    w.kb = params[w.nf + 1];
    w.r0 = params[w.nf + 2];
    w.ka = params[w.nf + 3];
    w.th0 = params[w.nf + 4];
    return w;
}

static inline double charge(const wparams *w, int64_t a) { return is_O(a) ? w->qO : w->qH; }

static inline double mass(const orc_system *s, int64_t a) { return is_O(a) ? s->m_O : s->m_H; }

/* Core of calc_F! / calc_F_and_grads!.  wvec: dl_dfi_prev (NULL: forces only).
 * dF_dp: full Jacobian (may be NULL).  acoef/dl_dp: contraction
 * dl_dp[p] += sum_a acoef[a] . dF_a/dtheta_p (may be NULL). */
static void forces_core(const orc_system *s, const double *params, const double *x,
                        const int32_t *pairs, int64_t n_pairs, const double *wvec, int grads,
                        double *F, double *dl_dfi, double *dF_dp, const double *acoef,
                        double *dl_dp, const double *mlp_coef, double *mlp_adj) {
    const int64_t n = 3 * (int64_t)s->n_mol, n3 = 3 * n;
    const double L = s->box, rc2 = s->cutoff * s->cutoff;
    const double kc = s->coulomb_const, crf = s->crf_const;
    const wparams w = unpack(s, params);
    const int P = w.P, nf = w.nf, iq = nf;
    const int nthr = orc_num_threads();

    /* Per-thread scratch as in the reference ([3N, n_threads], water.jl:1215-1225). */
    double *Ft = (double *)calloc((size_t)n3 * nthr, sizeof(double));
    double *Gt = wvec ? (double *)calloc((size_t)n3 * nthr, sizeof(double)) : NULL;
    double *Pt = (double *)calloc((size_t)P * nthr, sizeof(double));
    double *Jt = dF_dp ? (double *)calloc((size_t)n3 * P * nthr, sizeof(double)) : NULL;
    const size_t NA = (size_t)ORC_MLP_NT * ORC_MLP_NG * 4;
    double *At = (mlp_coef && mlp_adj && acoef) ? (double *)calloc(NA * nthr, sizeof(double)) : NULL;
    const double mlp_hinv = ORC_MLP_NG / s->cutoff;

#pragma omp parallel
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
#else
        int tid = 0;
#endif
        double *Fl = Ft + (size_t)n3 * tid;
        double *Gl = Gt ? Gt + (size_t)n3 * tid : NULL;
        double *Pl = Pt + (size_t)P * tid;
        double *Jl = Jt ? Jt + (size_t)n3 * P * tid : NULL;
        double *Al = At ? At + NA * tid : NULL;

        /* Non-bonded: water.jl:892-913 (forces) and 1232-1277 (grads). */
#pragma omp for schedule(static)
        for (int64_t ni = 0; ni < n_pairs; ni++) {
            int64_t i = pairs[2 * ni], j = pairs[2 * ni + 1];
            double dr[3];
            vec3(x + 3 * i, x + 3 * j, L, dr);
            double r2 = sumsq3(dr);
            if (!(r2 <= rc2)) continue;
            double r = sqrt(r2), invr2 = 1.0 / r2, invr3 = invr2 / r;
            double ndr[3] = {dr[0] / r, dr[1] / r, dr[2] / r};
            double cpf = kc * charge(&w, i) * charge(&w, j);
            double Fc = cpf * (invr2 - 2 * crf * r);
            double Ftot = Fc, dFdr = -2 * cpf * (invr3 + crf);
            double g[8] = {0};
            int on = 0;
            if (is_O(i) && is_O(j)) {
                double Fp = 0.0, dFp = 0.0;
                on = pair_form(s->inter_type, params, r, invr2, grads, &Fp, &dFp, g);
                if (on) { Ftot += Fp; dFdr += dFp; }
            }
            int mt = 0, mg = 0;
            double ms = 0.0;
            if (mlp_coef) {
                /* learned pair correction (mlp_oracle.h): types O-O, O-H, H-H */
                double Fm, dFm;
                mt = (is_O(i) ? 0 : 1) + (is_O(j) ? 0 : 1);
                orc_mlp_pair(mlp_coef, mt, s->cutoff, r, NULL, &Fm, &dFm);
                Ftot += Fm;
                dFdr += dFm;
                const double q = r * mlp_hinv;
                mg = (int)floor(q);
                if (mg > ORC_MLP_NG - 1) mg = ORC_MLP_NG - 1;
                ms = q - mg;
            }
            double *Fi = Fl + 3 * i, *Fj = Fl + 3 * j;
            for (int u = 0; u < 3; u++) {
                Fi[u] -= Ftot * ndr[u];
                Fj[u] += Ftot * ndr[u];
            }
            if (!grads) continue;
            /* dF/dq_O of the Coulomb part: 2 F_c / q_O (water.jl:1247). */
            double gq = 2 * Fc / w.qO;
            if (Gl) {
                /* dl_term (water.jl:1263-1271): M = dF_i/dx_j; dl_dfi_j += (w_i/m_i - w_j/m_j) M. */
                double Fdr3 = Ftot * invr3, mi = mass(s, i), mj = mass(s, j);
                for (int uj = 0; uj < 3; uj++) {
                    double dl = 0.0;
                    for (int ui = 0; ui < 3; ui++) {
                        double drt = (ui == uj) ? dr[ui] * dr[ui] - r2 : dr[ui] * dr[uj];
                        double dft = -(dFdr * ndr[ui]) * ndr[uj] + Fdr3 * drt;
                        dl += wvec[3 * i + ui] * (dft / mi) - wvec[3 * j + ui] * (dft / mj);
                    }
                    Gl[3 * i + uj] -= dl;
                    Gl[3 * j + uj] += dl;
                }
            }
            if (acoef) {
                double t = 0.0;
                for (int u = 0; u < 3; u++) t += (acoef[3 * j + u] - acoef[3 * i + u]) * ndr[u];
                if (on)
                    for (int p = 0; p < nf; p++) Pl[p] += g[p] * t;
                Pl[iq] += gq * t;
                if (Al) {
                    /* F = -(c1 + 2 c2 s + 3 c3 s^2) / h on interval mg */
                    double *ca = Al + ((size_t)mt * ORC_MLP_NG + mg) * 4;
                    ca[1] += -mlp_hinv * t;
                    ca[2] += -2.0 * ms * mlp_hinv * t;
                    ca[3] += -3.0 * ms * ms * mlp_hinv * t;
                }
            }
            if (Jl) {
                for (int u = 0; u < 3; u++) {
                    if (on)
                        for (int p = 0; p < nf; p++) {
                            Jl[(3 * i + u) * P + p] -= g[p] * ndr[u];
                            Jl[(3 * j + u) * P + p] += g[p] * ndr[u];
                        }
                    Jl[(3 * i + u) * P + iq] -= gq * ndr[u];
                    Jl[(3 * j + u) * P + iq] += gq * ndr[u];
                }
            }
        }

        /* Bonds (O,H1), (O,H2): water.jl:915-934 and 1279-1314. */
#pragma omp for schedule(static)
        for (int64_t bi = 0; bi < 2 * (int64_t)s->n_mol; bi++) {
            int64_t i = 3 * (bi / 2), j = i + 1 + (bi % 2);
            double dr[3];
            vec3(x + 3 * i, x + 3 * j, L, dr);
            double r2 = sumsq3(dr), r = sqrt(r2);
            double ndr[3] = {dr[0] / r, dr[1] / r, dr[2] / r};
            double disp = r - w.r0;
            double Fb = -w.kb * disp;
            double *Fi = Fl + 3 * i, *Fj = Fl + 3 * j;
            for (int u = 0; u < 3; u++) {
                Fi[u] -= Fb * ndr[u];
                Fj[u] += Fb * ndr[u];
            }
            if (!grads) continue;
            if (Gl) {
                double Fdr3 = Fb / (r2 * r), mi = mass(s, i), mj = mass(s, j);
                for (int uj = 0; uj < 3; uj++) {
                    double dl = 0.0;
                    for (int ui = 0; ui < 3; ui++) {
                        double drt = (ui == uj) ? dr[ui] * dr[ui] - r2 : dr[ui] * dr[uj];
                        double dft = -(-w.kb * ndr[ui]) * ndr[uj] + Fdr3 * drt;
                        dl += wvec[3 * i + ui] * (dft / mi) - wvec[3 * j + ui] * (dft / mj);
                    }
                    Gl[3 * i + uj] -= dl;
                    Gl[3 * j + uj] += dl;
                }
            }
            /* dF_i/dk_b = disp * ndr, dF_i/dr0 = -k_b * ndr (water.jl:1298-1301). */
            if (acoef) {
                double t = 0.0;
                for (int u = 0; u < 3; u++) t += (acoef[3 * i + u] - acoef[3 * j + u]) * ndr[u];
                Pl[nf + 1] += disp * t;
                Pl[nf + 2] += -w.kb * t;
            }
            if (Jl) {
                for (int u = 0; u < 3; u++) {
                    Jl[(3 * i + u) * P + nf + 1] += disp * ndr[u];
                    Jl[(3 * j + u) * P + nf + 1] -= disp * ndr[u];
                    Jl[(3 * i + u) * P + nf + 2] += -w.kb * ndr[u];
                    Jl[(3 * j + u) * P + nf + 2] -= -w.kb * ndr[u];
                }
            }
        }

        /* Angles (H1, O, H2): water.jl:936-968 and 1316-1422. */
#pragma omp for schedule(static)
        for (int64_t m = 0; m < (int64_t)s->n_mol; m++) {
            int64_t i = 3 * m + 1, j = 3 * m, k = 3 * m + 2;
            double a[3], b[3];
            vec3(x + 3 * j, x + 3 * i, L, a);
            vec3(x + 3 * j, x + 3 * k, L, b);
            double ta[3], tb[3];
            const double *tap = NULL, *tbp = NULL;
            if (grads && Gl) {
                double mi = mass(s, i), mj = mass(s, j), mk = mass(s, k);
                for (int u = 0; u < 3; u++) {
                    ta[u] = wvec[3 * i + u] / mi - wvec[3 * j + u] / mj;
                    tb[u] = wvec[3 * k + u] / mk - wvec[3 * j + u] / mj;
                }
                tap = ta;
                tbp = tb;
            }
            dual Fi[3], Fk[3];
            double p1d[3], p3d[3], disp;
            if (!angle_term(a, b, tap, tbp, w.ka, w.th0, Fi, Fk, p1d, p3d, &disp)) continue;
            for (int u = 0; u < 3; u++) {
                Fl[3 * i + u] += Fi[u].v;
                Fl[3 * k + u] += Fk[u].v;
                Fl[3 * j + u] -= Fi[u].v + Fk[u].v;
            }
            if (!grads) continue;
            if (Gl) {
                /* The tangent of F along (w/m) is J (w/m); J is symmetric. */
                for (int u = 0; u < 3; u++) {
                    Gl[3 * i + u] += Fi[u].d;
                    Gl[3 * k + u] += Fk[u].d;
                    Gl[3 * j + u] -= Fi[u].d + Fk[u].d;
                }
            }
            if (acoef) {
                double t = 0.0;
                for (int u = 0; u < 3; u++)
                    t += acoef[3 * i + u] * p1d[u] + acoef[3 * k + u] * p3d[u] -
                         acoef[3 * j + u] * (p1d[u] + p3d[u]);
                Pl[nf + 3] += disp * t;
                Pl[nf + 4] += w.ka * t;
            }
            if (Jl) {
                for (int u = 0; u < 3; u++) {
                    Jl[(3 * i + u) * P + nf + 3] += disp * p1d[u];
                    Jl[(3 * k + u) * P + nf + 3] += disp * p3d[u];
                    Jl[(3 * j + u) * P + nf + 3] -= disp * (p1d[u] + p3d[u]);
                    Jl[(3 * i + u) * P + nf + 4] += w.ka * p1d[u];
                    Jl[(3 * k + u) * P + nf + 4] += w.ka * p3d[u];
                    Jl[(3 * j + u) * P + nf + 4] -= w.ka * (p1d[u] + p3d[u]);
                }
            }
        }

        /* Thread reduction (water.jl:970-972, 1424-1430). */
#pragma omp for schedule(static)
        for (int64_t e = 0; e < n3; e++) {
            double sf = 0.0, sg = 0.0;
            for (int t = 0; t < nthr; t++) {
                sf += Ft[(size_t)n3 * t + e];
                if (Gt) sg += Gt[(size_t)n3 * t + e];
            }
            F[e] = sf;
            if (dl_dfi && Gt) dl_dfi[e] = sg;
            if (dF_dp)
                for (int p = 0; p < P; p++) {
                    double sj = 0.0;
                    for (int t = 0; t < nthr; t++) sj += Jt[((size_t)n3 * t + e) * P + p];
                    dF_dp[e * P + p] = sj;
                }
        }
    }
    if (dl_dp)
        for (int t = 0; t < nthr; t++)
            for (int p = 0; p < P; p++) dl_dp[p] += Pt[(size_t)P * t + p];
    if (At)
        for (int t = 0; t < nthr; t++)
            for (size_t k = 0; k < NA; k++) mlp_adj[k] += At[NA * t + k];
    free(At);
    free(Ft);
    free(Gt);
    free(Pt);
    free(Jt);
}

void orc_forces(const orc_system *s, const double *params, const double *x,
                const int32_t *pairs, int64_t n_pairs, double *F) {
    double *coef = mlp_table(s, params);
    forces_core(s, params, x, pairs, n_pairs, NULL, 0, F, NULL, NULL, NULL, NULL, coef, NULL);
    free(coef);
}

void orc_forces_grads(const orc_system *s, const double *params, const double *x,
                      const int32_t *pairs, int64_t n_pairs, const double *w,
                      double *F, double *dl_dfi, double *dF_dp) {
    double *coef = mlp_table(s, params);
    forces_core(s, params, x, pairs, n_pairs, w, 1, F, dl_dfi, dF_dp, NULL, NULL, coef, NULL);
    free(coef);
}

void orc_contract(const orc_system *s, const double *params, const double *x,
                  const int32_t *pairs, int64_t n_pairs, const double *acoef, double *dtheta) {
    const int Pc = orc_n_params(s->inter_type), Pt = orc_system_n_params(s);
    double *coef = mlp_table(s, params);
    double *adj = coef ? (double *)calloc((size_t)ORC_MLP_NT * ORC_MLP_NG * 4, sizeof(double)) : NULL;
    double *F = (double *)malloc(sizeof(double) * 9 * (size_t)s->n_mol);
    for (int p = 0; p < Pt; p++) dtheta[p] = 0.0;
    forces_core(s, params, x, pairs, n_pairs, NULL, 1, F, NULL, NULL, acoef, dtheta, coef, adj);
    if (coef) orc_mlp_backprop(params + Pc, s->cutoff, adj, dtheta + Pc);
    free(F);
    free(coef);
    free(adj);
}

/* Potential energy: pair form + reaction-field Coulomb (Molly CoulombReactionField:
 * k q_i q_j (1/r + k_rf r^2 - c_rf), c_rf = 1/rc + k_rf rc^2) + bonds + angles. */
double orc_energy_grads(const orc_system *s, const double *params, const double *x,
                        const int32_t *pairs, int64_t n_pairs, double *dEdp) {
    const double L = s->box, rc = s->cutoff, rc2 = rc * rc;
    const double crf = s->crf_const, c_rf = 1.0 / rc + crf * rc * rc;
    const wparams w = unpack(s, params);
    const int Pc = w.P, Pt = orc_system_n_params(s), nf = w.nf;
    double *coef = mlp_table(s, params);
    double *adj = coef ? (double *)calloc((size_t)ORC_MLP_NT * ORC_MLP_NG * 4, sizeof(double)) : NULL;
    const double hinv = ORC_MLP_NG / rc, ch = 1e-30;
    for (int p = 0; p < Pt; p++) dEdp[p] = 0.0;
    double E = 0.0;
    for (int64_t ni = 0; ni < n_pairs; ni++) {
        int64_t i = pairs[2 * ni], j = pairs[2 * ni + 1];
        double dr[3];
        vec3(x + 3 * i, x + 3 * j, L, dr);
        double r2 = sumsq3(dr);
        if (!(r2 <= rc2)) continue;
        double r = sqrt(r2);
        double Ec = s->coulomb_const * charge(&w, i) * charge(&w, j) * (1.0 / r + crf * r2 - c_rf);
        E += Ec;
        dEdp[nf] += 2.0 * Ec / w.qO;
        if (is_O(i) && is_O(j)) {
            E += pair_form_energy(s->inter_type, params, r);
            /* the reference's iszero gate (eps, or A for Buckingham) switches the form off */
            if (params[s->inter_type == ORC_BUCK ? 0 : 1] != 0.0)
                for (int k = 0; k < nf; k++) {
                    double complex pc[4];
                    for (int q = 0; q < nf; q++) pc[q] = params[q] + (q == k ? I * ch : 0.0);
                    dEdp[k] += cimag(pair_form_energy_c(s->inter_type, pc, r)) / ch;
                }
        }
        if (coef) {
            const int t = (is_O(i) ? 0 : 1) + (is_O(j) ? 0 : 1);
            double um;
            orc_mlp_pair(coef, t, rc, r, &um, NULL, NULL);
            E += um;
            const double q = r * hinv;
            int g = (int)floor(q);
            if (g > ORC_MLP_NG - 1) g = ORC_MLP_NG - 1;
            const double sv = q - g;
            double *ca = adj + ((size_t)t * ORC_MLP_NG + g) * 4;
            ca[0] += 1.0;
            ca[1] += sv;
            ca[2] += sv * sv;
            ca[3] += sv * sv * sv;
        }
    }
    for (int64_t m = 0; m < s->n_mol; m++) {
        const double *xo = x + 9 * m;
        for (int h = 1; h <= 2; h++) {
            double dr[3];
            vec3(xo, xo + 3 * h, L, dr);
            double d = sqrt(sumsq3(dr)) - w.r0;
            E += 0.5 * w.kb * d * d;
            dEdp[nf + 1] += 0.5 * d * d;
            dEdp[nf + 2] += -w.kb * d;
        }
        double a[3], b[3];
        vec3(xo, xo + 3, L, a);
        vec3(xo, xo + 6, L, b);
        double c = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) / (sqrt(sumsq3(a)) * sqrt(sumsq3(b)));
        double th = acos(c) - w.th0;
        E += 0.5 * w.ka * th * th;
        dEdp[nf + 3] += 0.5 * th * th;
        dEdp[nf + 4] += -w.ka * th;
    }
    if (coef) orc_mlp_backprop(params + Pc, rc, adj, dEdp + Pc);
    free(coef);
    free(adj);
    return E;
}

double orc_energy(const orc_system *s, const double *params, const double *x,
                  const int32_t *pairs, int64_t n_pairs) {
    const double L = s->box, rc = s->cutoff, rc2 = rc * rc;
    const double crf = s->crf_const, c_rf = 1.0 / rc + crf * rc * rc;
    const wparams w = unpack(s, params);
    double *coef = mlp_table(s, params);
    double E = 0.0;
    for (int64_t ni = 0; ni < n_pairs; ni++) {
        int64_t i = pairs[2 * ni], j = pairs[2 * ni + 1];
        double dr[3];
        vec3(x + 3 * i, x + 3 * j, L, dr);
        double r2 = sumsq3(dr);
        if (!(r2 <= rc2)) continue;
        double r = sqrt(r2);
        E += s->coulomb_const * charge(&w, i) * charge(&w, j) * (1.0 / r + crf * r2 - c_rf);
        if (is_O(i) && is_O(j)) E += pair_form_energy(s->inter_type, params, r);
        if (coef) {
            double um;
            orc_mlp_pair(coef, (is_O(i) ? 0 : 1) + (is_O(j) ? 0 : 1), rc, r, &um, NULL, NULL);
            E += um;
        }
    }
    free(coef);
    for (int64_t m = 0; m < s->n_mol; m++) {
        const double *xo = x + 9 * m;
        for (int h = 1; h <= 2; h++) {
            double dr[3];
            vec3(xo, xo + 3 * h, L, dr);
            double d = sqrt(sumsq3(dr)) - w.r0;
            E += 0.5 * w.kb * d * d;
        }
        double a[3], b[3];
        vec3(xo, xo + 3, L, a);
        vec3(xo, xo + 6, L, b);
        double c = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) / (sqrt(sumsq3(a)) * sqrt(sumsq3(b)));
        double th = acos(c) - w.th0;
        E += 0.5 * w.ka * th * th;
    }
    return E;
}

/* ------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and Box-Muller normals. */
static inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* 53-bit uniform from two Philox words. */
static inline uint64_t bits53(uint32_t hi, uint32_t lo) {
    return (((uint64_t)hi << 21) ^ ((uint64_t)lo >> 11)) & ((1ull << 53) - 1);
}

/* Two N(0,1) draws for (seed, atom, blk): counter (atom, blk, 0, 0), key = seed;
 * u1 = (w + 1) 2^-53 in (0, 1], u2 = w' 2^-53 in [0, 1), Box-Muller. */
static void normals2(uint64_t seed, uint32_t atom, uint32_t blk, double z[2]) {
    uint32_t c[4] = {atom, blk, 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    double u1 = ((double)bits53(c[0], c[1]) + 1.0) * (1.0 / 9007199254740992.0);
    double u2 = (double)bits53(c[2], c[3]) * (1.0 / 9007199254740992.0);
    double rr = sqrt(-2.0 * log(u1));
    z[0] = rr * cos(2.0 * ORC_PI * u2);
    z[1] = rr * sin(2.0 * ORC_PI * u2);
}

void orc_philox_normals(uint64_t seed, uint32_t atom, double z[4]) {
    normals2(seed, atom, 0u, z);
    normals2(seed, atom, 1u, z + 2);
}

void orc_noise(const orc_system *s, uint64_t seed, double temp, double *xi) {
    const int64_t n = 3 * (int64_t)s->n_mol;
    for (int64_t a = 0; a < n; a++) {
        double z[4];
        normals2(seed, (uint32_t)a, 0u, z);
        normals2(seed, (uint32_t)a, 1u, z + 2);
        double sd = sqrt(s->kB * temp / mass(s, a));
        for (int u = 0; u < 3; u++) xi[3 * a + u] = z[u] * sd;
    }
}

/* ------------------------------------------------------------------------- */
/* Smoothed RDF (water.jl:631-691) and its analytic gradient (the Enzyme pullback
 * of water.jl:715-736 differentiates the same windowed sums). */
typedef struct {
    int64_t n1, n2;
    int64_t *idx1, *idx2;
    int64_t off;          /* Int(x_min / step) - 1, water.jl:660 */
    double pre;           /* V / (4 pi n1 n2 step) */
} rdf_ctx;

static void rdf_select(const orc_system *s, int sel, int64_t **idx, int64_t *cnt) {
    const int64_t n = 3 * (int64_t)s->n_mol;
    int64_t c = 0;
    *idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t a = 0; a < n; a++)
        if ((sel == 0) == is_O(a)) (*idx)[c++] = a;
    *cnt = c;
}

static inline double grid_x(const orc_rdf_term *t, int64_t k) { return t->x_min + t->step * (double)k; }

/* Grid window of the per-distance normaliser: 0-based [lo, hi] (water.jl:663-665). */
static inline void den_window(const orc_rdf_term *t, int64_t off, double d, int64_t *lo, int64_t *hi) {
    int64_t s = (int64_t)ceil((d - t->exp_cutoff) / t->step) - off;  /* 1-based */
    int64_t e = (int64_t)floor((d + t->exp_cutoff) / t->step) - off;
    if (s < 1) s = 1;
    if (e > t->n_grid) e = t->n_grid;
    *lo = s - 1;
    *hi = e - 1;
}

/* Histogram window: grid points with x - c <= d <= x + c (water.jl:676-688). */
static inline void hist_window(const orc_rdf_term *t, double d, int64_t *lo, int64_t *hi) {
    int64_t a = (int64_t)floor((d - t->exp_cutoff - t->x_min) / t->step) - 1;
    int64_t b = (int64_t)ceil((d + t->exp_cutoff - t->x_min) / t->step) + 1;
    if (a < 0) a = 0;
    if (b > t->n_grid - 1) b = t->n_grid - 1;
    while (a <= b && !(d <= grid_x(t, a) + t->exp_cutoff)) a++;
    while (b >= a && !(d >= grid_x(t, b) - t->exp_cutoff)) b--;
    *lo = a;
    *hi = b;
}

static void rdf_setup(const orc_system *s, const orc_rdf_term *t, rdf_ctx *c) {
    rdf_select(s, t->sel1, &c->idx1, &c->n1);
    rdf_select(s, t->sel2, &c->idx2, &c->n2);
    c->off = (int64_t)llround(t->x_min / t->step) - 1;
    double V = s->box * s->box * s->box;
    c->pre = V / (4 * ORC_PI * (double)c->n1 * (double)c->n2 * t->step);
}

static void rdf_free(rdf_ctx *c) {
    free(c->idx1);
    free(c->idx2);
}

/* sum_k over the normaliser window of g_k(d) and of dg_k/dd. */
static inline void rdf_den(const orc_rdf_term *t, int64_t off, double d, double *den, double *dden) {
    int64_t lo, hi;
    den_window(t, off, d, &lo, &hi);
    double s = 0.0, ds = 0.0;
    for (int64_t k = lo; k <= hi; k++) {
        double xk = grid_x(t, k), e = xk - d;
        double g = exp(-(e * e) / t->width);
        s += g;
        ds += g * 2 * e / t->width;
    }
    *den = s;
    *dden = ds;
}

void orc_rdf(const orc_system *s, const orc_rdf_term *t, const double *x, double *h) {
    rdf_ctx c;
    rdf_setup(s, t, &c);
    const double L = s->box;
    const int nthr = orc_num_threads();
    double *acc = (double *)calloc((size_t)t->n_grid * nthr, sizeof(double));
#pragma omp parallel
    {
#ifdef _OPENMP
        double *al = acc + (size_t)t->n_grid * omp_get_thread_num();
#else
        double *al = acc;
#endif
#pragma omp for schedule(static)
        for (int64_t a = 0; a < c.n1; a++) {
            for (int64_t b = 0; b < c.n2; b++) {
                double dr[3];
                vec3(x + 3 * c.idx1[a], x + 3 * c.idx2[b], L, dr);
                double d = sqrt(sumsq3(dr));
                if (d == 0.0) continue;
                int64_t lo, hi;
                hist_window(t, d, &lo, &hi);
                if (lo > hi) continue;
                double den, dden;
                rdf_den(t, c.off, d, &den, &dden);
                for (int64_t k = lo; k <= hi; k++) {
                    double e = grid_x(t, k) - d;
                    al[k] += exp(-(e * e) / t->width) / den;
                }
            }
        }
    }
    for (int64_t k = 0; k < t->n_grid; k++) {
        double sum = 0.0;
        for (int th = 0; th < nthr; th++) sum += acc[(size_t)t->n_grid * th + k];
        double xk = grid_x(t, k);
        h[k] = c.pre * sum / (xk * xk);
    }
    free(acc);
    rdf_free(&c);
}

double orc_loss_grad(const orc_system *s, const orc_loss *Ls, const double *x, double *dLdx) {
    const int64_t n3 = 9 * (int64_t)s->n_mol;
    const double L = s->box;
    double loss = 0.0;
    if (dLdx) memset(dLdx, 0, sizeof(double) * (size_t)n3);
    for (int ti = 0; ti < Ls->n_terms; ti++) {
        const orc_rdf_term *t = &Ls->terms[ti];
        double *h = (double *)malloc(sizeof(double) * (size_t)t->n_grid);
        double *dLdh = (double *)calloc((size_t)t->n_grid, sizeof(double));
        orc_rdf(s, t, x, h);
        double lt = 0.0;
        for (int q = 0; q < t->n_target; q++) {
            int64_t k = t->slice_start + (int64_t)q * t->slice_stride;
            double e = h[k] - t->target[q];
            if (t->norm == 1) {
                lt += fabs(e);
                dLdh[k] += t->weight * (e > 0 ? 1.0 : (e < 0 ? -1.0 : 0.0));
            } else {
                lt += e * e;
                dLdh[k] += t->weight * 2 * e;
            }
        }
        loss += t->weight * lt;
        if (dLdx) {
            rdf_ctx c;
            rdf_setup(s, t, &c);
            const int nthr = orc_num_threads();
            double *gacc = (double *)calloc((size_t)n3 * nthr, sizeof(double));
#pragma omp parallel
            {
#ifdef _OPENMP
            double *gl = gacc + (size_t)n3 * omp_get_thread_num();
#else
            double *gl = gacc;
#endif
#pragma omp for schedule(static)
            for (int64_t a = 0; a < c.n1; a++) {
                for (int64_t b = 0; b < c.n2; b++) {
                    int64_t ia = c.idx1[a], ib = c.idx2[b];
                    double dr[3];
                    vec3(x + 3 * ia, x + 3 * ib, L, dr);
                    double d = sqrt(sumsq3(dr));
                    if (d == 0.0) continue;
                    int64_t lo, hi;
                    hist_window(t, d, &lo, &hi);
                    if (lo > hi) continue;
                    double den, dden;
                    rdf_den(t, c.off, d, &den, &dden);
                    double dLdd = 0.0;
                    for (int64_t k = lo; k <= hi; k++) {
                        if (dLdh[k] == 0.0) continue;
                        double xk = grid_x(t, k), e = xk - d;
                        double g = exp(-(e * e) / t->width);
                        double gp = g * 2 * e / t->width;
                        dLdd += dLdh[k] * c.pre / (xk * xk) * (gp / den - g * dden / (den * den));
                    }
                    if (dLdd == 0.0) continue;
                    for (int u = 0; u < 3; u++) {
                        double gu = dLdd * dr[u] / d;
                        gl[3 * ib + u] += gu;
                        gl[3 * ia + u] -= gu;
                    }
                }
            }
            }
            for (int64_t e = 0; e < n3; e++)
                for (int th = 0; th < nthr; th++) dLdx[e] += gacc[(size_t)n3 * th + e];
            free(gacc);
            rdf_free(&c);
        }
        free(h);
        free(dLdh);
    }
    return loss;
}

double orc_loss_and_grads(const orc_system *s, const double *params, const orc_loss *Ls,
                          const double *x, double *l_parts, double *dLdx, double *dl_dp) {
    const int64_t n3 = 9 * (int64_t)s->n_mol;
    const int P = orc_system_n_params(s);
    /* loss_fn, water.jl:757-769 */
    const double l_rdf = orc_loss_grad(s, Ls, x, dLdx);
    double l_ev = 0.0;
    if (dl_dp)
        for (int p = 0; p < P; p++) dl_dp[p] = 0.0;
    if (Ls->enth_vap) {
        /* enthalpy_vaporization / loss_enth_vap, water.jl:738-755 */
        int64_t cap = 16 * (3 * (int64_t)s->n_mol) + 1024;
        int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
        int64_t np = orc_neighbor_pairs(s, x, pairs, cap);
        if (np > cap) {
            cap = np;
            pairs = (int32_t *)realloc(pairs, sizeof(int32_t) * 2 * (size_t)cap);
            np = orc_neighbor_pairs(s, x, pairs, cap);
        }
        double *dU = (double *)malloc(sizeof(double) * (size_t)P);
        const double U = orc_energy_grads(s, params, x, pairs, np, dU);
        const double e = Ls->u_gas - U / s->n_mol + Ls->rt - Ls->target;
        const double k = 2.0 * e / s->n_mol;   /* dl_ev/dU = -k */
        l_ev = e * e;
        if (dl_dp)
            for (int p = 0; p < P; p++) dl_dp[p] = -k * dU[p];
        if (dLdx) {
            double *F = (double *)malloc(sizeof(double) * (size_t)n3);
            orc_forces(s, params, x, pairs, np, F);
            for (int64_t i = 0; i < n3; i++) dLdx[i] += k * F[i];
            free(F);
        }
        free(dU);
        free(pairs);
    }
    if (l_parts) {
        l_parts[0] = l_rdf;
        l_parts[1] = l_ev;
    }
    return l_rdf + l_ev;
}

/* ------------------------------------------------------------------------- */
/* Rebuild the pair list into a growable buffer; returns the pair count. */
static int64_t rebuild_pairs(const orc_system *s, const double *x, int32_t **pairs, int64_t *cap) {
    int64_t cnt = orc_neighbor_pairs(s, x, *pairs, *cap);
    if (cnt > *cap) {
        *cap = cnt + cnt / 4 + 16;
        *pairs = (int32_t *)realloc(*pairs, sizeof(int32_t) * 2 * (size_t)(*cap));
        cnt = orc_neighbor_pairs(s, x, *pairs, *cap);
    }
    return cnt;
}

/* The noise of one step: the caller's array (host_noise [n_steps][3N], entry step - 1) when
 * given, else the Philox draw of the step's seed. */
static void step_noise(const orc_system *s, const uint64_t *noise_seeds, const double *host_noise,
                       int32_t step, int64_t n3, double *xi) {
    if (host_noise)
        memcpy(xi, host_noise + (size_t)(step - 1) * (size_t)n3, sizeof(double) * (size_t)n3);
    else
        orc_noise(s, noise_seeds[step - 1], s->temp, xi);
}

static double forward_sim_any(const orc_system *s, const double *params, double *x, double *v,
                              const uint64_t *noise_seeds, const double *host_noise, double gamma,
                              int32_t n_steps, int32_t n_steps_loss, double dt, int32_t n_steps_log,
                              const orc_loss *loss, int32_t calc_loss, double *snap_x,
                              double *snap_v, double *l_parts) {
    const int64_t n = 3 * (int64_t)s->n_mol, n3 = 3 * n;
    const double L = s->box;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c);   /* water.jl:1019-1020 */
    const int32_t n_blocks = (n_steps == 0) ? 1 : n_steps / n_steps_loss;
    double *F = (double *)malloc(sizeof(double) * (size_t)n3);
    double *xi = (double *)malloc(sizeof(double) * (size_t)n3);
    int64_t cap = 16 * n + 1024;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
    int64_t np = rebuild_pairs(s, x, &pairs, &cap);
    double *coef = mlp_table(s, params);
    if (snap_x) {
        memcpy(snap_x, x, sizeof(double) * (size_t)n3);
        memcpy(snap_v, v, sizeof(double) * (size_t)n3);
    }
    double loss_accum = 0.0, parts_accum[2] = {0.0, 0.0};
    /* water.jl:1029-1045 */
    for (int32_t step = 1; step <= n_steps; step++) {
        forces_core(s, params, x, pairs, np, NULL, 0, F, NULL, NULL, NULL, NULL, coef, NULL);
        for (int64_t a = 0; a < n; a++) {
            double m = mass(s, a);
            for (int u = 0; u < 3; u++) v[3 * a + u] = v[3 * a + u] + F[3 * a + u] * dt / m;
        }
        for (int64_t e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        step_noise(s, noise_seeds, host_noise, step, n3, xi);
        for (int64_t e = 0; e < n3; e++) v[e] = v[e] * c + xi[e] * sn;
        for (int64_t e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        for (int64_t e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], L);
        if (step % s->n_steps_nf == 0) np = rebuild_pairs(s, x, &pairs, &cap);
        if (snap_x && n_steps_log > 0 && step % n_steps_log == 0) {
            int64_t si = step / n_steps_log;
            memcpy(snap_x + si * n3, x, sizeof(double) * (size_t)n3);
            memcpy(snap_v + si * n3, v, sizeof(double) * (size_t)n3);
        }
        if (calc_loss && loss && step % n_steps_loss == 0) {
            double lp[2];
            loss_accum += orc_loss_and_grads(s, params, loss, x, lp, NULL, NULL);
            parts_accum[0] += lp[0];
            parts_accum[1] += lp[1];
        }
    }
    if (l_parts) {
        l_parts[0] = parts_accum[0] / n_blocks;
        l_parts[1] = parts_accum[1] / n_blocks;
    }
    free(coef);
    free(F);
    free(xi);
    free(pairs);
    return loss_accum / n_blocks;
}

static void reset_accums(int64_t n3, double c, const double *g, double *A, double *B,
                         double *C, double *D, double *dl_dfi) {
    /* water.jl:1480-1483, 1541-1545 */
    for (int64_t e = 0; e < n3; e++) {
        A[e] = g[e] * (1 + c);
        B[e] = g[e] * (1 + c);
        C[e] = 0.0;
        D[e] = g[e] * (1 + 2 * c + c * c) / (2 * c);
        dl_dfi[e] = 0.0;
    }
}

double orc_forward_sim(const orc_system *s, const double *params, double *x, double *v,
                       const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                       int32_t n_steps_loss, double dt, int32_t n_steps_log,
                       const orc_loss *loss, int32_t calc_loss,
                       double *snap_x, double *snap_v, double *l_parts) {
    return forward_sim_any(s, params, x, v, noise_seeds, NULL, gamma, n_steps, n_steps_loss, dt,
                           n_steps_log, loss, calc_loss, snap_x, snap_v, l_parts);
}

double orc_forward_sim_hn(const orc_system *s, const double *params, double *x, double *v,
                          const double *host_noise, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, double dt, int32_t n_steps_log,
                          const orc_loss *loss, int32_t calc_loss,
                          double *snap_x, double *snap_v, double *l_parts) {
    return forward_sim_any(s, params, x, v, NULL, host_noise, gamma, n_steps, n_steps_loss, dt,
                           n_steps_log, loss, calc_loss, snap_x, snap_v, l_parts);
}

static double reverse_sim_any(const orc_system *s, const double *params, double *x, double *v,
                              const uint64_t *noise_seeds, const double *host_noise, double gamma,
                              int32_t n_steps, int32_t n_steps_loss, int32_t n_steps_trunc,
                              double dt, int32_t n_steps_log, const double *snap_x,
                              const double *snap_v, double clip_norm_threshold,
                              const orc_loss *loss, double *dl_dp, double *l_parts) {
    if (n_steps_trunc > n_steps_loss || n_steps_loss <= 0) return NAN;  /* water.jl:1437-1439 */
    const int64_t n = 3 * (int64_t)s->n_mol, n3 = 3 * n;
    const double L = s->box;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c);
    const double dt2 = dt * dt;
    const int32_t n_blocks = n_steps / n_steps_loss;
    const int P = orc_system_n_params(s), Pc = orc_n_params(s->inter_type);
    double *coef = mlp_table(s, params);
    double *adj = coef ? (double *)calloc((size_t)ORC_MLP_NT * ORC_MLP_NG * 4, sizeof(double)) : NULL;
    double *buf = (double *)calloc((size_t)n3 * 9, sizeof(double));
    double *F = buf, *xi = buf + n3, *g = buf + 2 * n3, *A = buf + 3 * n3, *B = buf + 4 * n3;
    double *C = buf + 5 * n3, *Dd = buf + 6 * n3, *dl_dfi = buf + 7 * n3, *acoef = buf + 8 * n3;
    int64_t cap = 16 * n + 1024;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);

    for (int p = 0; p < P; p++) dl_dp[p] = 0.0;
    /* direct dl/dtheta of every loss point (water.jl:1471, 1540) */
    double *ddirect = (double *)calloc((size_t)P, sizeof(double));
    double *dblock = (double *)malloc(sizeof(double) * (size_t)P);
    double lp[2], parts_accum[2];
    double loss_accum = orc_loss_and_grads(s, params, loss, x, lp, g, dblock);   /* water.jl:1471 */
    parts_accum[0] = lp[0];
    parts_accum[1] = lp[1];
    for (int p = 0; p < P; p++) ddirect[p] += dblock[p];
    reset_accums(n3, c, g, A, B, C, Dd, dl_dfi);
    int64_t np = rebuild_pairs(s, x, &pairs, &cap);

    int32_t trunc_count = 0;
    for (int32_t step_n = n_steps; step_n >= 1; step_n--) {
        trunc_count++;
        if (trunc_count <= n_steps_trunc) {
            /* part 1, water.jl:1496-1502 */
            for (int64_t e = 0; e < n3; e++) x[e] = x[e] - v[e] * dt / 2;
            step_noise(s, noise_seeds, host_noise, step_n, n3, xi);
            for (int64_t e = 0; e < n3; e++) v[e] = (v[e] - xi[e] * sn) / c;
            for (int64_t e = 0; e < n3; e++) x[e] = x[e] - v[e] * dt / 2;
            for (int64_t e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], L);
            for (int64_t e = 0; e < n3; e++) Dd[e] = c * Dd[e] + dt2 * dl_dfi[e] * (1 + c) / 2;
            for (int64_t e = 0; e < n3; e++) C[e] = C[e] + Dd[e];
            if (step_n % s->n_steps_nf == 0) np = rebuild_pairs(s, x, &pairs, &cap);  /* :1504 */
            /* dF/dtheta is contracted with A dt^2 / (2m) on the fly (water.jl:1517-1519). */
            for (int64_t a = 0; a < n; a++) {
                double m = mass(s, a);
                for (int u = 0; u < 3; u++) acoef[3 * a + u] = A[3 * a + u] * (dt2 / (2 * m));
            }
            forces_core(s, params, x, pairs, np, C, 1, F, dl_dfi, NULL, acoef, dl_dp, coef, adj);
            /* part 2, water.jl:1511-1521 */
            double nrm = 0.0;
            for (int64_t e = 0; e < n3; e++) nrm += dl_dfi[e] * dl_dfi[e];
            nrm = sqrt(nrm);
            if (nrm > clip_norm_threshold)
                for (int64_t e = 0; e < n3; e++) dl_dfi[e] = dl_dfi[e] * clip_norm_threshold / nrm;
            for (int64_t a = 0; a < n; a++) {
                double m = mass(s, a);
                for (int u = 0; u < 3; u++) v[3 * a + u] = v[3 * a + u] - F[3 * a + u] * dt / m;
            }
            for (int64_t e = 0; e < n3; e++) B[e] = c * B[e] + dt2 * dl_dfi[e];
            for (int64_t e = 0; e < n3; e++) A[e] = A[e] + B[e];
        }
        /* part 3, water.jl:1525-1547; snapshots are indexed by the step they hold. */
        if (n_steps_log > 0 && (step_n - 1) % n_steps_log == 0 && step_n > 1) {
            if (trunc_count <= n_steps_trunc || (step_n - 1) % n_steps_loss == 0) {
                int64_t si = (step_n - 1) / n_steps_log;
                memcpy(x, snap_x + si * n3, sizeof(double) * (size_t)n3);
                memcpy(v, snap_v + si * n3, sizeof(double) * (size_t)n3);
            }
        }
        if ((step_n - 1) % n_steps_loss == 0 && step_n > 1) {
            trunc_count = 0;
            loss_accum += orc_loss_and_grads(s, params, loss, x, lp, g, dblock);
            parts_accum[0] += lp[0];
            parts_accum[1] += lp[1];
            for (int p = 0; p < P; p++) ddirect[p] += dblock[p];
            reset_accums(n3, c, g, A, B, C, Dd, dl_dfi);
        }
    }
    if (coef) orc_mlp_backprop(params + Pc, s->cutoff, adj, dl_dp + Pc);
    for (int p = 0; p < P; p++) dl_dp[p] = (dl_dp[p] + ddirect[p]) / n_blocks;
    if (l_parts) {
        l_parts[0] = parts_accum[0] / n_blocks;
        l_parts[1] = parts_accum[1] / n_blocks;
    }
    free(ddirect);
    free(dblock);
    free(coef);
    free(adj);
    free(buf);
    free(pairs);
    return loss_accum / n_blocks;
}

double orc_reverse_sim(const orc_system *s, const double *params, double *x, double *v,
                       const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                       int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                       int32_t n_steps_log, const double *snap_x, const double *snap_v,
                       double clip_norm_threshold, const orc_loss *loss, double *dl_dp,
                       double *l_parts) {
    return reverse_sim_any(s, params, x, v, noise_seeds, NULL, gamma, n_steps, n_steps_loss,
                           n_steps_trunc, dt, n_steps_log, snap_x, snap_v, clip_norm_threshold,
                           loss, dl_dp, l_parts);
}

double orc_reverse_sim_hn(const orc_system *s, const double *params, double *x, double *v,
                          const double *host_noise, double gamma, int32_t n_steps,
                          int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                          int32_t n_steps_log, const double *snap_x, const double *snap_v,
                          double clip_norm_threshold, const orc_loss *loss, double *dl_dp,
                          double *l_parts) {
    return reverse_sim_any(s, params, x, v, NULL, host_noise, gamma, n_steps, n_steps_loss,
                           n_steps_trunc, dt, n_steps_log, snap_x, snap_v, clip_norm_threshold,
                           loss, dl_dp, l_parts);
}

/* ------------------------------------------------------------------------- */
/* Monte-Carlo barostat, water.jl:789-865 (see revsim_oracle.h). */
static const double kBarNa = 0.0602214076;   /* 1 bar nm^3 x N_A in kJ/mol */

double orc_barostat_uniform(uint64_t seed, uint64_t k) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (k + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* Molecule centres scaled by l about the origin, atoms moved with their molecule and
 * wrapped into the scaled box (scale_coords!). */
static void scale_molecules(const orc_system *s, const double *x, double l, double *xt) {
    const double L = s->box, Ln = L * l;
    for (int64_t m = 0; m < s->n_mol; m++) {
        const double *xo = x + 9 * m;
        double d1[3], d2[3], sh[3];
        vec3(xo, xo + 3, L, d1);
        vec3(xo, xo + 6, L, d2);
        for (int u = 0; u < 3; u++) {
            const double c = xo[u] + (d1[u] + d2[u]) / 3.0;
            sh[u] = c * l - c;
        }
        for (int k = 0; k < 3; k++)
            for (int u = 0; u < 3; u++) xt[9 * m + 3 * k + u] = orc_wrap1d(xo[3 * k + u] + sh[u], Ln);
    }
}

int32_t orc_barostat_attempt(orc_system *s, const double *params, double *x, const int32_t *pairs,
                             int64_t n_pairs, orc_barostat *b) {
    const int64_t n3 = 9 * (int64_t)s->n_mol;
    const double kT = s->kB * s->temp;
    const double E = orc_energy(s, params, x, pairs, n_pairs);
    const double L = s->box, V = L * L * L;
    const double u1 = orc_barostat_uniform(b->seed, 2 * (uint64_t)b->n_draws);
    const double u2 = orc_barostat_uniform(b->seed, 2 * (uint64_t)b->n_draws + 1);
    b->n_draws++;
    const double dV = b->volume_scale * (2 * u1 - 1);
    const double v_scale = (V + dV) / V, l = cbrt(v_scale);
    double *xt = (double *)malloc(sizeof(double) * (size_t)n3);
    scale_molecules(s, x, l, xt);
    s->box = L * l;
    const double Et = orc_energy(s, params, xt, pairs, n_pairs);
    const double dW = (Et - E) + b->pressure * kBarNa * dV - s->n_mol * kT * log(v_scale);
    int32_t acc = 0;
    if (dW <= 0.0 || u2 < exp(-dW / kT)) {
        memcpy(x, xt, sizeof(double) * (size_t)n3);
        b->n_accepted++;
        b->n_accepted_total++;
        acc = 1;
    } else {
        s->box = L;
    }
    b->n_attempted++;
    if (b->n_attempted >= 10) {
        if (b->n_accepted < 0.25 * b->n_attempted) {
            b->volume_scale /= b->scale_increment;
            b->n_attempted = b->n_accepted = 0;
        } else if (b->n_accepted > 0.75 * b->n_attempted) {
            const double cap = V * b->max_volume_frac, vs = b->volume_scale * b->scale_increment;
            b->volume_scale = vs < cap ? vs : cap;
            b->n_attempted = b->n_accepted = 0;
        }
    }
    free(xt);
    return acc;
}

void orc_forward_sim_barostat(orc_system *s, const double *params, double *x, double *v,
                              const uint64_t *noise_seeds, double gamma, int32_t n_steps, double dt,
                              orc_barostat *b) {
    const int64_t n = 3 * (int64_t)s->n_mol, n3 = 3 * n;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c);
    double *F = (double *)malloc(sizeof(double) * (size_t)n3);
    double *xi = (double *)malloc(sizeof(double) * (size_t)n3);
    int64_t cap = 16 * n + 1024;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
    int64_t np = rebuild_pairs(s, x, &pairs, &cap);
    double *coef = mlp_table(s, params);
    for (int32_t step = 1; step <= n_steps; step++) {   /* water.jl:1029-1045 */
        forces_core(s, params, x, pairs, np, NULL, 0, F, NULL, NULL, NULL, NULL, coef, NULL);
        for (int64_t a = 0; a < n; a++) {
            const double m = mass(s, a);
            for (int u = 0; u < 3; u++) v[3 * a + u] = v[3 * a + u] + F[3 * a + u] * dt / m;
        }
        for (int64_t e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        orc_noise(s, noise_seeds[step - 1], s->temp, xi);
        for (int64_t e = 0; e < n3; e++) v[e] = v[e] * c + xi[e] * sn;
        for (int64_t e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        for (int64_t e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], s->box);
        if (step % s->n_steps_nf == 0) np = rebuild_pairs(s, x, &pairs, &cap);
        if (b && step % b->n_steps == 0) orc_barostat_attempt(s, params, x, pairs, np, b);
    }
    free(coef);
    free(F);
    free(xi);
    free(pairs);
}
