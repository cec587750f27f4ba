/*
 * gas_oracle.c -- CPU FP64 restatement of the gas-in-water reversible-simulation gradient
 * of greener-group/rev-sim diffusion/diffusion.jl (see gas_oracle.h).  TEST INFRASTRUCTURE
 * ONLY: the checker for the CUDA path, never called by it.
 */
#include "gas_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "revsim_oracle.h"

double complex orc_pair_form_energy_cx(int32_t type, const double complex *p, double r);

static const double kDiffExp = 2.0e-9;        /* D_exp, m^2 s^-1 (diffusion.jl:900) */
static const double kDiffWeight = 1e18;       /* loss_weight, m^-4 s^2 (diffusion.jl:902) */
static const double kLossWeightEv = 0.05;     /* loss_weighting_ev (diffusion.jl:52) */
static const double kLossWeightRdf = 0.05;    /* loss_weighting_rdf (diffusion.jl:51) */
static const double kUGas = 3.69, kRT = 2.45, kEvTarget = 44.12 + 2.8;   /* :800-813 */

static inline void vec3(const double *xi, const double *xj, double L, double *d) {
    d[0] = orc_vec1d(xi[0], xj[0], L);
    d[1] = orc_vec1d(xi[1], xj[1], L);
    d[2] = orc_vec1d(xi[2], xj[2], L);
}

static inline double sumsq3(const double *d) { return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]; }

static inline int64_t n_atoms(const orc_gas_system *s) {
    return 3 * (int64_t)s->n_water + 2 * (int64_t)s->n_gas;
}

/* 0: water O, 1: water H, 2: gas O */
static inline int kind(const orc_gas_system *s, int64_t a) {
    const int64_t nw3 = 3 * (int64_t)s->n_water;
    return a < nw3 ? (a % 3 == 0 ? 0 : 1) : 2;
}

static inline int64_t molecule(const orc_gas_system *s, int64_t a) {
    const int64_t nw3 = 3 * (int64_t)s->n_water;
    return a < nw3 ? a / 3 : s->n_water + (a - nw3) / 2;
}

static inline double amass(const orc_gas_system *s, int64_t a) {
    return kind(s, a) == 1 ? s->m_H : s->m_O;
}

int32_t orc_gas_n_params(int32_t t) {
    if (orc_n_form_params(t) < 0) return -1;
    return t == ORC_LJ ? 5 : 7;
}

/* ------------------------------------------------------------------------- */
/* Per-class pair-form parameters by the mixing rules (diffusion.jl:169-170, 272-274) and
 * the factors that carry dF/d(mixed k) onto theta (dsigma_dsigmaw ... of 190-193, 296-297).
 * Classes: 0 water O - water O, 1 water O - gas, 2 gas - gas. */
typedef struct {
    int type, P, nf, iq;
    double qO, qH;
    double pc[3][4];
    int on[3];
    double fw[3][4], fg[3][4];
    int iw[4], ig[4];
} gparams;

static gparams unpack(const orc_gas_system *s, const double *t) {
    gparams g;
    memset(&g, 0, sizeof(g));
    g.type = s->inter_type;
    g.nf = orc_n_form_params(s->inter_type);
    g.P = orc_gas_n_params(s->inter_type);
    g.iq = g.P - 1;
    g.qO = t[g.iq];
    g.qH = -g.qO / 2;
    if (g.type == ORC_BUCK) {
        const double *w = t, *q = t + 3;
        for (int k = 0; k < 3; k++) {
            g.pc[0][k] = (w[k] + w[k]) / 2;
            g.pc[1][k] = (w[k] + q[k]) / 2;
            g.pc[2][k] = (q[k] + q[k]) / 2;
            g.iw[k] = k;
            g.ig[k] = k + 3;
            g.fw[0][k] = 1.0; g.fg[0][k] = 0.0;
            g.fw[1][k] = 0.5; g.fg[1][k] = 0.5;
            g.fw[2][k] = 0.0; g.fg[2][k] = 1.0;
        }
        g.on[0] = w[0] != 0.0;
        g.on[1] = w[0] != 0.0 && q[0] != 0.0;
        g.on[2] = q[0] != 0.0;
    } else {
        const double sw = t[0], ew = t[1], sg = t[2], eg = t[3];
        const double sig[3] = {(sw + sw) / 2, (sw + sg) / 2, (sg + sg) / 2};
        const double eps[3] = {sqrt(ew * ew), sqrt(ew * eg), sqrt(eg * eg)};
        for (int c = 0; c < 3; c++) {
            g.pc[c][0] = sig[c];
            g.pc[c][1] = eps[c];
            g.pc[c][2] = g.nf > 2 ? t[4] : 0.0;
            g.pc[c][3] = g.nf > 2 ? t[5] : 0.0;
        }
        g.iw[0] = 0; g.ig[0] = 2;
        g.iw[1] = 1; g.ig[1] = 3;
        g.iw[2] = 4; g.ig[2] = -1;
        g.iw[3] = 5; g.ig[3] = -1;
        g.fw[0][0] = 1.0; g.fg[0][0] = 0.0;
        g.fw[0][1] = 1.0; g.fg[0][1] = 0.0;
        g.fw[1][0] = 0.5; g.fg[1][0] = 0.5;
        g.fw[1][1] = eps[1] != 0.0 ? eg / (2 * eps[1]) : 0.0;
        g.fg[1][1] = eps[1] != 0.0 ? ew / (2 * eps[1]) : 0.0;
        g.fw[2][0] = 0.0; g.fg[2][0] = 1.0;
        g.fw[2][1] = 0.0; g.fg[2][1] = 1.0;
        for (int c = 0; c < 3; c++) {
            g.fw[c][2] = g.fw[c][3] = 1.0;
            g.fg[c][2] = g.fg[c][3] = 0.0;
        }
        g.on[0] = ew != 0.0;
        g.on[1] = ew != 0.0 && eg != 0.0;
        g.on[2] = eg != 0.0;
    }
    return g;
}

static inline double charge(const gparams *g, int k) { return k == 0 ? g->qO : (k == 1 ? g->qH : 0.0); }

/* ------------------------------------------------------------------------- */
int64_t orc_gas_neighbor_pairs(const orc_gas_system *s, const double *x, int32_t *pairs,
                               int64_t max_pairs) {
    const int64_t n = n_atoms(s);
    const double rc2 = s->nl_cutoff * s->nl_cutoff, L = s->box;
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; i++) {
        int64_t c = 0;
        const int64_t mi = molecule(s, i);
        for (int64_t j = i + 1; j < n; j++) {
            if (molecule(s, j) == mi) continue;
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
        const int64_t mi = molecule(s, i);
        for (int64_t j = i + 1; j < n && k < max_pairs; j++) {
            if (molecule(s, j) == mi) continue;
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
/* One radial pair term with F(r), dF/dr on the displacement dr (from i to j): forces, and
 * when grads the VJP dl_dfi += (w_i/m_i - w_j/m_j) M as in diffusion.jl:1352-1363. */
static void radial(int64_t i, int64_t j, const double *dr, double r2, double F, double dFdr,
                   int grads, const double *w, double mi, double mj, double *Fl, double *Gl) {
    const double r = sqrt(r2);
    const double ndr[3] = {dr[0] / r, dr[1] / r, dr[2] / r};
    for (int u = 0; u < 3; u++) {
        Fl[3 * i + u] -= F * ndr[u];
        Fl[3 * j + u] += F * ndr[u];
    }
    if (!grads || !Gl) return;
    const double Fdr3 = F / (r2 * r);
    for (int uj = 0; uj < 3; uj++) {
        double dl = 0.0;
        for (int ui = 0; ui < 3; ui++) {
            double drt = (ui == uj) ? dr[ui] * dr[ui] - r2 : dr[ui] * dr[uj];
            double dft = -(dFdr * ndr[ui]) * ndr[uj] + Fdr3 * drt;
            dl += w[3 * i + ui] * (dft / mi) - w[3 * j + ui] * (dft / mj);
        }
        Gl[3 * i + uj] -= dl;
        Gl[3 * j + uj] += dl;
    }
}

static void forces_core(const orc_gas_system *s, const double *params, const double *x,
                        const int32_t *pairs, int64_t n_pairs, int grads, const double *w,
                        const double *acoef, double *F, double *dl_dfi, double *dl_dp) {
    const int64_t n = n_atoms(s), n3 = 3 * n;
    const double L = s->box, rc2 = s->cutoff * s->cutoff;
    const double kc = s->coulomb_const, crf = s->crf_const;
    const gparams g = unpack(s, params);
    const int P = g.P;
    const int nthr = orc_num_threads();
    double *Ft = (double *)calloc((size_t)n3 * nthr, sizeof(double));
    double *Gt = (grads && w) ? (double *)calloc((size_t)n3 * nthr, sizeof(double)) : NULL;
    double *Pt = (double *)calloc((size_t)P * nthr, sizeof(double));

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

        /* Non-bonded: diffusion.jl:974-995 (forces), 1320-1365 (grads). */
#pragma omp for schedule(static)
        for (int64_t ni = 0; ni < n_pairs; ni++) {
            const int64_t i = pairs[2 * ni], j = pairs[2 * ni + 1];
            double dr[3];
            vec3(x + 3 * i, x + 3 * j, L, dr);
            const double r2 = sumsq3(dr);
            if (!(r2 <= rc2)) continue;
            const int ki = kind(s, i), kj = kind(s, j);
            const double r = sqrt(r2), invr2 = 1.0 / r2, invr3 = invr2 / r;
            const double cpf = kc * charge(&g, ki) * charge(&g, kj);
            double Ftot = cpf * (invr2 - 2 * crf * r);
            double dFdr = -2 * cpf * (invr3 + crf);
            const double gq = 2 * Ftot / g.qO;
            double gf[4] = {0, 0, 0, 0};
            int cls = -1;
            if (ki != 1 && kj != 1) {
                cls = (ki == 2) + (kj == 2);
                double Fp = 0.0, dFp = 0.0;
                if (g.on[cls] && orc_pair_form(g.type, g.pc[cls], r, invr2, grads, &Fp, &dFp, gf)) {
                    Ftot += Fp;
                    dFdr += dFp;
                } else {
                    cls = -1;
                }
            }
            radial(i, j, dr, r2, Ftot, dFdr, grads, w, amass(s, i), amass(s, j), Fl, Gl);
            if (!grads || !acoef) continue;
            double t = 0.0;
            for (int u = 0; u < 3; u++) t += (acoef[3 * j + u] - acoef[3 * i + u]) * (dr[u] / r);
            if (cpf != 0.0) Pl[g.iq] += gq * t;
            if (cls >= 0)
                for (int k = 0; k < g.nf; k++) {
                    Pl[g.iw[k]] += gf[k] * g.fw[cls][k] * t;
                    if (g.ig[k] >= 0) Pl[g.ig[k]] += gf[k] * g.fg[cls][k] * t;
                }
        }

        /* Water bonds O-H1, O-H2 and the O2 bonds: diffusion.jl:997-1016, 1367-1397. */
        const int64_t nb = 2 * (int64_t)s->n_water + s->n_gas;
#pragma omp for schedule(static)
        for (int64_t bi = 0; bi < nb; bi++) {
            int64_t i, j;
            double kb, r0;
            if (bi < 2 * (int64_t)s->n_water) {
                i = 3 * (bi / 2);
                j = i + 1 + (bi % 2);
                kb = s->kb_w;
                r0 = s->r0_w;
            } else {
                i = 3 * (int64_t)s->n_water + 2 * (bi - 2 * (int64_t)s->n_water);
                j = i + 1;
                kb = s->kb_g;
                r0 = s->r0_g;
            }
            double dr[3];
            vec3(x + 3 * i, x + 3 * j, L, dr);
            const double r2 = sumsq3(dr), r = sqrt(r2);
            radial(i, j, dr, r2, -kb * (r - r0), -kb, grads, w, amass(s, i), amass(s, j), Fl, Gl);
        }

        /* Water angles H1-O-H2: diffusion.jl:1018-1050, 1399-1498. */
#pragma omp for schedule(static)
        for (int64_t m = 0; m < (int64_t)s->n_water; m++) {
            const int64_t i = 3 * m + 1, j = 3 * m, k = 3 * m + 2;
            double a[3], b[3], ta[3] = {0, 0, 0}, tb[3] = {0, 0, 0};
            vec3(x + 3 * j, x + 3 * i, L, a);
            vec3(x + 3 * j, x + 3 * k, L, b);
            if (grads && Gl)
                for (int u = 0; u < 3; u++) {
                    ta[u] = w[3 * i + u] / s->m_H - w[3 * j + u] / s->m_O;
                    tb[u] = w[3 * k + u] / s->m_H - w[3 * j + u] / s->m_O;
                }
            double Fi[3], Fk[3], dFi[3], dFk[3];
            if (!orc_angle_term(a, b, ta, tb, s->ka_w, s->th0_w, Fi, Fk, dFi, dFk)) continue;
            for (int u = 0; u < 3; u++) {
                Fl[3 * i + u] += Fi[u];
                Fl[3 * k + u] += Fk[u];
                Fl[3 * j + u] -= Fi[u] + Fk[u];
                if (grads && Gl) {
                    Gl[3 * i + u] += dFi[u];
                    Gl[3 * k + u] += dFk[u];
                    Gl[3 * j + u] -= dFi[u] + dFk[u];
                }
            }
        }

#pragma omp for schedule(static)
        for (int64_t e = 0; e < n3; e++) {
            double sf = 0.0, sg = 0.0;
            for (int t = 0; t < nthr; t++) {
                sf += Ft[(size_t)n3 * t + e];
                if (Gt) sg += Gt[(size_t)n3 * t + e];
            }
            F[e] = sf;
            if (dl_dfi && Gt) dl_dfi[e] = sg;
        }
    }
    if (dl_dp && grads && acoef)
        for (int t = 0; t < nthr; t++)
            for (int p = 0; p < P; p++) dl_dp[p] += Pt[(size_t)P * t + p];
    free(Ft);
    free(Gt);
    free(Pt);
}

void orc_gas_forces(const orc_gas_system *s, const double *params, const double *x,
                    const int32_t *pairs, int64_t n_pairs, double *F) {
    forces_core(s, params, x, pairs, n_pairs, 0, NULL, NULL, F, NULL, NULL);
}

void orc_gas_forces_grads(const orc_gas_system *s, const double *params, const double *x,
                          const int32_t *pairs, int64_t n_pairs, const double *w,
                          const double *acoef, double *F, double *dl_dfi, double *dl_dp) {
    forces_core(s, params, x, pairs, n_pairs, 1, w, acoef, F, dl_dfi, dl_dp);
}

/* ------------------------------------------------------------------------- */
/* Mixed parameters of one class on complex per-site parameters (for complex-step dE/dtheta). */
static void mix_c(int type, int cls, const double complex *t, double complex *pc) {
    if (type == ORC_BUCK) {
        const double complex *a = cls == 2 ? t + 3 : t, *b = cls == 0 ? t : t + 3;
        for (int k = 0; k < 3; k++) pc[k] = (a[k] + b[k]) / 2;
        pc[3] = 0.0;
    } else {
        const double complex sa = cls == 2 ? t[2] : t[0], sb = cls == 0 ? t[0] : t[2];
        const double complex ea = cls == 2 ? t[3] : t[1], eb = cls == 0 ? t[1] : t[3];
        pc[0] = (sa + sb) / 2;
        pc[1] = csqrt(ea * eb);
        pc[2] = t[4];
        pc[3] = t[5];
    }
}

double orc_gas_energy(const orc_gas_system *s, const double *params, const double *x,
                      const int32_t *pairs, int64_t n_pairs, double *dEdp) {
    const double L = s->box, rc = s->cutoff, rc2 = rc * rc;
    const double crf = s->crf_const, c_rf = 1.0 / rc + crf * rc * rc;
    const gparams g = unpack(s, params);
    const int P = g.P;
    const double ch = 1e-30;
    if (dEdp)
        for (int p = 0; p < P; p++) dEdp[p] = 0.0;
    double E = 0.0;
    for (int64_t ni = 0; ni < n_pairs; ni++) {
        const int64_t i = pairs[2 * ni], j = pairs[2 * ni + 1];
        double dr[3];
        vec3(x + 3 * i, x + 3 * j, L, dr);
        const double r2 = sumsq3(dr);
        if (!(r2 <= rc2)) continue;
        const double r = sqrt(r2);
        const int ki = kind(s, i), kj = kind(s, j);
        /* Molly CoulombReactionField energy */
        const double Ec = s->coulomb_const * charge(&g, ki) * charge(&g, kj) * (1.0 / r + crf * r2 - c_rf);
        E += Ec;
        if (dEdp && Ec != 0.0) dEdp[g.iq] += 2.0 * Ec / g.qO;
        if (ki == 1 || kj == 1) continue;
        const int cls = (ki == 2) + (kj == 2);
        if (!g.on[cls]) continue;
        E += orc_pair_form_energy(g.type, g.pc[cls], r);
        if (!dEdp) continue;
        for (int k = 0; k < P - 1; k++) {
            double complex tc[6], pc[4];
            for (int q = 0; q < P - 1; q++) tc[q] = params[q] + (q == k ? I * ch : 0.0);
            mix_c(g.type, cls, tc, pc);
            dEdp[k] += cimag(orc_pair_form_energy_cx(g.type, pc, r)) / ch;
        }
    }
    for (int64_t m = 0; m < s->n_water; m++) {
        const double *xo = x + 9 * m;
        for (int h = 1; h <= 2; h++) {
            double dr[3];
            vec3(xo, xo + 3 * h, L, dr);
            const double d = sqrt(sumsq3(dr)) - s->r0_w;
            E += 0.5 * s->kb_w * d * d;
        }
        double a[3], b[3];
        vec3(xo, xo + 3, L, a);
        vec3(xo, xo + 6, L, b);
        const double c = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) / (sqrt(sumsq3(a)) * sqrt(sumsq3(b)));
        const double th = acos(c) - s->th0_w;
        E += 0.5 * s->ka_w * th * th;
    }
    for (int64_t q = 0; q < s->n_gas; q++) {
        const double *xg = x + 9 * (int64_t)s->n_water + 6 * q;
        double dr[3];
        vec3(xg, xg + 3, L, dr);
        const double d = sqrt(sumsq3(dr)) - s->r0_g;
        E += 0.5 * s->kb_g * d * d;
    }
    return E;
}

/* ------------------------------------------------------------------------- */
void orc_gas_noise(const orc_gas_system *s, uint64_t seed, double *xi) {
    const int64_t n = n_atoms(s);
    for (int64_t a = 0; a < n; a++) {
        double z[4];
        orc_philox_normals(seed, (uint32_t)a, z);
        const double sd = sqrt(s->kB * s->temp / amass(s, a));
        for (int u = 0; u < 3; u++) xi[3 * a + u] = z[u] * sd;
    }
}

void orc_gas_centres(const orc_gas_system *s, const double *x, double *c) {
    const double L = s->box;
    for (int64_t q = 0; q < s->n_gas; q++) {
        const double *x1 = x + 9 * (int64_t)s->n_water + 6 * q, *x2 = x1 + 3;
        for (int u = 0; u < 3; u++) {
            const double cen = x1[u] + orc_vec1d(x1[u], x2[u], L) / 2;
            c[3 * q + u] = orc_wrap1d(cen, L);
        }
    }
}

double orc_gas_diffusion_D(const double *gc, int32_t n_frames, int32_t n_gas, double box,
                           double loss_frequency, double *dD_dgc) {
    const int32_t ns = n_frames / 2;
    const size_t fsz = 3 * (size_t)n_gas;
    if (dD_dgc) memset(dD_dgc, 0, sizeof(double) * fsz * (size_t)n_frames);
    double *ct = (double *)malloc(sizeof(double) * (fsz ? fsz : 1));
    double D = 0.0;
    for (int32_t st = 0; st < ns; st++) {
        const double *c0 = gc + fsz * st;
        memcpy(ct, c0, sizeof(double) * fsz);
        for (int32_t j = st + 1; j <= st + ns; j++) {
            const double *cj = gc + fsz * j;
            for (size_t e = 0; e < fsz; e++) ct[e] += orc_vec1d(ct[e], cj[e], box);
        }
        double msd = 0.0;
        for (int32_t q = 0; q < n_gas; q++) {
            double d2 = 0.0;
            for (int u = 0; u < 3; u++) {
                const double d = ct[3 * q + u] - c0[3 * q + u];
                d2 += d * d;
            }
            msd += d2;
        }
        msd /= n_gas;
        D += msd / (ns * loss_frequency);
        if (dD_dgc) {
            /* d ct_final / d frame(st + ns) = 1, / d earlier frames = 0; minus frame st */
            const double k = 2.0 / ((double)n_gas * ns * loss_frequency * (6.0 * ns));
            double *ge = dD_dgc + fsz * (st + ns), *gs = dD_dgc + fsz * st;
            for (size_t e = 0; e < fsz; e++) {
                const double d = ct[e] - c0[e];
                ge[e] += k * d;
                gs[e] -= k * d;
            }
        }
    }
    free(ct);
    return D / (6 * ns);
}

double orc_gas_loss_final(int32_t loss_type, const double *gc, int32_t n_frames, int32_t n_gas,
                          double box, double loss_frequency, double ev_sum, double rdf_sum,
                          double *out, double *dl_dgc) {
    const double D = orc_gas_diffusion_D(gc, n_frames, n_gas, box, loss_frequency, dl_dgc);
    const double Dc = D * 1e-6;
    double l_diff = 0.0;
    const size_t nc = 3 * (size_t)n_gas * (size_t)n_frames;
    if (loss_type & ORC_GAS_DIFF) {
        l_diff = kDiffWeight * (Dc - kDiffExp) * (Dc - kDiffExp);
        if (dl_dgc) {
            const double dl_dD = kDiffWeight * 2 * (Dc - kDiffExp) * 1e-6;
            for (size_t e = 0; e < nc; e++) dl_dgc[e] *= dl_dD;
        }
    } else if (dl_dgc) {
        memset(dl_dgc, 0, sizeof(double) * nc);
    }
    const double l_ev = (loss_type & ORC_GAS_EV) ? kLossWeightEv * ev_sum / n_frames : 0.0;
    const double l_rdf = (loss_type & ORC_GAS_RDF) ? kLossWeightRdf * rdf_sum / n_frames : 0.0;
    if (out) {
        out[0] = Dc;
        out[1] = l_diff;
        out[2] = l_rdf;
        out[3] = l_ev;
    }
    return l_diff + l_rdf + l_ev;
}

static int64_t rebuild(const orc_gas_system *s, const double *x, int32_t **pairs, int64_t *cap) {
    int64_t cnt = orc_gas_neighbor_pairs(s, x, *pairs, *cap);
    if (cnt > *cap) {
        *cap = cnt + cnt / 4 + 16;
        *pairs = (int32_t *)realloc(*pairs, sizeof(int32_t) * 2 * (size_t)(*cap));
        cnt = orc_gas_neighbor_pairs(s, x, *pairs, *cap);
    }
    return cnt;
}

/* (dH_vap - target)^2 of loss_enth_vap (diffusion.jl:799-815) and de/dU = -1/n. */
static double ev_raw(const orc_gas_system *s, const double *params, const double *x,
                     double *dEdp, double *e_out) {
    int64_t cap = 16 * n_atoms(s) + 1024;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
    const int64_t np = rebuild(s, x, &pairs, &cap);
    const double U = orc_gas_energy(s, params, x, pairs, np, dEdp);
    free(pairs);
    const double e = kUGas - U / s->n_mol_ev + kRT - kEvTarget;
    if (e_out) *e_out = e;
    return e * e;
}

double orc_gas_ev_point(const orc_gas_system *s, const double *params, const double *x,
                        int32_t n_blocks, double *dLdx, double *dl_dp) {
    const int P = orc_gas_n_params(s->inter_type);
    double dEdp[8], e;
    const double l = ev_raw(s, params, x, dl_dp ? dEdp : NULL, &e) * kLossWeightEv / n_blocks;
    /* dl/dU = -2 e w / (n_blocks n) */
    const double k = 2 * e * kLossWeightEv / ((double)n_blocks * s->n_mol_ev);
    if (dLdx) {
        const int64_t n3 = 3 * n_atoms(s);
        int64_t cap = 16 * n_atoms(s) + 1024;
        int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
        const int64_t np = rebuild(s, x, &pairs, &cap);
        double *F = (double *)malloc(sizeof(double) * (size_t)n3);
        orc_gas_forces(s, params, x, pairs, np, F);
        for (int64_t e3 = 0; e3 < n3; e3++) dLdx[e3] += k * F[e3];
        free(F);
        free(pairs);
    }
    if (dl_dp)
        for (int p = 0; p < P; p++) dl_dp[p] += -k * dEdp[p];
    return l;
}

/* loss_rdf of the water atoms (diffusion.jl:759-774) by the water restatement; its gradient
 * with respect to the water coordinates into dldx [9 n_water] when non-NULL. */
static double rdf_raw(const orc_gas_system *s, const orc_loss *rdf, const double *x, double *dldx) {
    orc_system ws;
    memset(&ws, 0, sizeof(ws));
    ws.n_mol = s->n_water;
    ws.box = s->box;
    orc_loss L = *rdf;
    L.enth_vap = 0;
    return orc_loss_grad(&ws, &L, x, dldx);
}

/* ------------------------------------------------------------------------- */
double orc_gas_forward_sim(const orc_gas_system *s, const double *params, double *x, double *v,
                           const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                           int32_t n_steps_loss, double dt, int32_t loss_type,
                           int32_t calc_loss, double *snap_x, double *snap_v, double *gc,
                           double *out, const orc_loss *rdf) {
    const int64_t n = n_atoms(s), n3 = 3 * n;
    const double L = s->box;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c);   /* diffusion.jl:1216-1217 */
    const int32_t n_blocks = (n_steps == 0) ? 1 : n_steps / n_steps_loss;
    const double lf = n_steps_loss * dt;
    double *F = (double *)malloc(sizeof(double) * (size_t)n3);
    double *xi = (double *)malloc(sizeof(double) * (size_t)n3);
    int64_t cap = 16 * n + 1024;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
    int64_t np = rebuild(s, x, &pairs, &cap);
    if (snap_x) {
        memcpy(snap_x, x, sizeof(double) * (size_t)n3);
        memcpy(snap_v, v, sizeof(double) * (size_t)n3);
    }
    double ev_sum = 0.0, rdf_sum = 0.0;
    /* diffusion.jl:1226-1240 */
    for (int32_t step = 1; step <= n_steps; step++) {
        orc_gas_forces(s, params, x, pairs, np, F);
        for (int64_t a = 0; a < n; a++) {
            const double m = amass(s, a);
            for (int u = 0; u < 3; u++) v[3 * a + u] = v[3 * a + u] + F[3 * a + u] * dt / m;
        }
        for (int64_t e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        orc_gas_noise(s, noise_seeds[step - 1], xi);
        for (int64_t e = 0; e < n3; e++) v[e] = v[e] * c + xi[e] * sn;
        for (int64_t e = 0; e < n3; e++) x[e] = x[e] + v[e] * dt / 2;
        for (int64_t e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], L);
        if (step % s->n_steps_nf == 0) np = rebuild(s, x, &pairs, &cap);
        if (step % n_steps_loss == 0) {
            const int64_t k = step / n_steps_loss;
            if (snap_x && k <= n_blocks) {
                memcpy(snap_x + k * n3, x, sizeof(double) * (size_t)n3);
                memcpy(snap_v + k * n3, v, sizeof(double) * (size_t)n3);
            }
            if (gc && k <= n_blocks) orc_gas_centres(s, x, gc + (k - 1) * 3 * (int64_t)s->n_gas);
            if (calc_loss && (loss_type & ORC_GAS_EV)) ev_sum += ev_raw(s, params, x, NULL, NULL);
            if (calc_loss && (loss_type & ORC_GAS_RDF) && rdf) rdf_sum += rdf_raw(s, rdf, x, NULL);
        }
    }
    double loss = 0.0;
    if (calc_loss && gc)
        loss = orc_gas_loss_final(loss_type, gc, n_blocks, s->n_gas, L, lf, ev_sum, rdf_sum, out, NULL);
    free(F);
    free(xi);
    free(pairs);
    return loss;
}

static void reset_accums(int64_t n3, double c, const double *g, double *A, double *B,
                         double *C, double *D, double *dl_dfi) {
    /* diffusion.jl:1547-1550, 1600-1604 */
    for (int64_t e = 0; e < n3; e++) {
        A[e] = g[e] * (1 + c);
        B[e] = g[e] * (1 + c);
        C[e] = 0.0;
        D[e] = g[e] * (1 + 2 * c + c * c) / (2 * c);
        dl_dfi[e] = 0.0;
    }
}

/* dl/dx at one loss point: the enthalpy term (when on) plus the centre gradient of the
 * frame split half and half onto the two sites of each gas molecule (diffusion.jl:1536-1539, 1596-1598). */
static double point_grad(const orc_gas_system *s, const double *params, const double *x,
                         int32_t loss_type, int32_t n_blocks, const double *dgc_frame,
                         double *g, double *dl_dp, const orc_loss *rdf, double *l_rdf) {
    const int64_t n3 = 3 * n_atoms(s);
    memset(g, 0, sizeof(double) * (size_t)n3);
    double l = 0.0;
    if (loss_type & ORC_GAS_EV) l = orc_gas_ev_point(s, params, x, n_blocks, g, dl_dp);
    *l_rdf = 0.0;
    if ((loss_type & ORC_GAS_RDF) && rdf) {
        const int64_t nw9 = 9 * (int64_t)s->n_water;
        double *t = (double *)malloc(sizeof(double) * (size_t)(nw9 ? nw9 : 1));
        const double w = kLossWeightRdf / n_blocks;
        *l_rdf = w * rdf_raw(s, rdf, x, t);
        for (int64_t e = 0; e < nw9; e++) g[e] += w * t[e];
        free(t);
    }
    double *gg = g + 9 * (int64_t)s->n_water;
    for (int64_t q = 0; q < s->n_gas; q++)
        for (int u = 0; u < 3; u++) {
            const double h = dgc_frame[3 * q + u] / 2;
            gg[6 * q + u] += h;
            gg[6 * q + 3 + u] += h;
        }
    return l;
}

double orc_gas_reverse_sim(const orc_gas_system *s, const double *params, double *x, double *v,
                           const uint64_t *noise_seeds, double gamma, int32_t n_steps,
                           int32_t n_steps_loss, int32_t n_steps_trunc, double dt,
                           int32_t loss_type, const double *snap_x, const double *snap_v,
                           const double *gc, double *dl_dp, double *out, const orc_loss *rdf) {
    const int64_t n = n_atoms(s), n3 = 3 * n;
    const double L = s->box;
    const double c = exp(-gamma * dt), sn = sqrt(1 - c * c), dt2 = dt * dt;
    const int32_t n_blocks = n_steps / n_steps_loss;
    const double lf = n_steps_loss * dt;
    const int P = orc_gas_n_params(s->inter_type);
    const size_t fsz = 3 * (size_t)s->n_gas;
    double *dgc = (double *)malloc(sizeof(double) * (fsz * (size_t)n_blocks + 1));
    double parts[4];
    const double l_diff = orc_gas_loss_final(loss_type & ORC_GAS_DIFF, gc, n_blocks, s->n_gas, L, lf,
                                             0.0, 0.0, parts, dgc);
    double *buf = (double *)calloc((size_t)n3 * 9, sizeof(double));
    double *F = buf, *xi = buf + n3, *g = buf + 2 * n3, *A = buf + 3 * n3, *B = buf + 4 * n3;
    double *C = buf + 5 * n3, *Dd = buf + 6 * n3, *dl_dfi = buf + 7 * n3, *acoef = buf + 8 * n3;
    int64_t cap = 16 * n + 1024;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (size_t)cap);
    for (int p = 0; p < P; p++) dl_dp[p] = 0.0;

    double lr_pt = 0.0, l_rdf = 0.0;
    double l_ev = point_grad(s, params, x, loss_type, n_blocks, dgc + fsz * (n_blocks - 1), g, dl_dp,
                             rdf, &lr_pt);
    l_rdf += lr_pt;
    reset_accums(n3, c, g, A, B, C, Dd, dl_dfi);
    memcpy(x, snap_x + (size_t)n_blocks * n3, sizeof(double) * (size_t)n3);
    memcpy(v, snap_v + (size_t)n_blocks * n3, sizeof(double) * (size_t)n3);
    int64_t np = rebuild(s, x, &pairs, &cap);

    for (int32_t lc = 1; lc <= n_blocks; lc++) {
        const int32_t s_start = n_steps - (lc - 1) * n_steps_loss;
        const int32_t s_end = s_start - n_steps_trunc + 1 > 1 ? s_start - n_steps_trunc + 1 : 1;
        for (int32_t step_n = s_start; step_n >= s_end; step_n--) {
            /* part 1, diffusion.jl:1566-1572 */
            for (int64_t e = 0; e < n3; e++) x[e] = x[e] - v[e] * dt / 2;
            orc_gas_noise(s, noise_seeds[step_n - 1], xi);
            for (int64_t e = 0; e < n3; e++) v[e] = (v[e] - xi[e] * sn) / c;
            for (int64_t e = 0; e < n3; e++) x[e] = x[e] - v[e] * dt / 2;
            for (int64_t e = 0; e < n3; e++) x[e] = orc_wrap1d(x[e], L);
            for (int64_t e = 0; e < n3; e++) Dd[e] = c * Dd[e] + dt2 * dl_dfi[e] * (1 + c) / 2;
            for (int64_t e = 0; e < n3; e++) C[e] = C[e] + Dd[e];
            if (step_n % s->n_steps_nf == 0) np = rebuild(s, x, &pairs, &cap);   /* :1574 */
            for (int64_t a = 0; a < n; a++) {
                const double m = amass(s, a);
                for (int u = 0; u < 3; u++) acoef[3 * a + u] = A[3 * a + u] * (dt2 / (2 * m));
            }
            orc_gas_forces_grads(s, params, x, pairs, np, C, acoef, F, dl_dfi, dl_dp);
            /* part 2, diffusion.jl:1579-1586 */
            for (int64_t a = 0; a < n; a++) {
                const double m = amass(s, a);
                for (int u = 0; u < 3; u++) v[3 * a + u] = v[3 * a + u] - F[3 * a + u] * dt / m;
            }
            for (int64_t e = 0; e < n3; e++) B[e] = c * B[e] + dt2 * dl_dfi[e];
            for (int64_t e = 0; e < n3; e++) A[e] = A[e] + B[e];
        }
        /* part 3, diffusion.jl:1589-1605 */
        if (lc != n_blocks) {
            const int32_t k = n_blocks - lc;
            memcpy(x, snap_x + (size_t)k * n3, sizeof(double) * (size_t)n3);
            memcpy(v, snap_v + (size_t)k * n3, sizeof(double) * (size_t)n3);
            np = rebuild(s, x, &pairs, &cap);
            l_ev += point_grad(s, params, x, loss_type, n_blocks, dgc + fsz * (k - 1), g, dl_dp, rdf,
                               &lr_pt);
            l_rdf += lr_pt;
            reset_accums(n3, c, g, A, B, C, Dd, dl_dfi);
        }
    }
    if (out) {
        out[0] = parts[0];
        out[1] = l_diff;
        out[2] = l_rdf;
        out[3] = l_ev;
    }
    free(dgc);
    free(buf);
    free(pairs);
    return l_diff + l_rdf + l_ev;
}
