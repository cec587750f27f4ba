/*
 * mlp_oracle.c -- FP64 restatement of the tabulated MLP pair correction (see mlp_oracle.h).
 * TEST INFRASTRUCTURE ONLY.
 */
#include "mlp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NR ORC_MLP_NRBF
#define H ORC_MLP_H
#define NG ORC_MLP_NG

typedef struct {
    const double *W1, *b1, *W2, *b2, *w3, *b3;
} mlp_view;

static mlp_view view(const double *theta, int t) {
    const double *p = theta + (size_t)t * ORC_MLP_PER_TYPE;
    mlp_view v;
    v.W1 = p;
    v.b1 = v.W1 + H * NR;
    v.W2 = v.b1 + H;
    v.b2 = v.W2 + H * H;
    v.w3 = v.b2 + H;
    v.b3 = v.w3 + H;
    return v;
}

static inline double sigm(double z) { return 1.0 / (1.0 + exp(-z)); }
static inline double silu(double z) { return z * sigm(z); }
static inline double silu1(double z) { double s = sigm(z); return s * (1.0 + z * (1.0 - s)); }
static inline double silu2(double z) { double s = sigm(z); return s * (1.0 - s) * (2.0 + z * (1.0 - 2.0 * s)); }

/* Activations of one node, value and r-tangent streams. */
typedef struct {
    double phi[NR], dphi[NR], z1[H], dz1[H], h1[H], dh1[H], z2[H], dz2[H], h2[H], dh2[H];
    double y, dy, fc, dfc;
} node_act;

static void node_forward(const mlp_view *m, double r, double rc, double w, node_act *a) {
    for (int k = 0; k < NR; k++) {
        const double mu = k * rc / (NR - 1), e = r - mu;
        a->phi[k] = exp(-e * e / (2 * w * w));
        a->dphi[k] = -e / (w * w) * a->phi[k];
    }
    for (int i = 0; i < H; i++) {
        double z = m->b1[i], dz = 0.0;
        for (int k = 0; k < NR; k++) {
            z += m->W1[i * NR + k] * a->phi[k];
            dz += m->W1[i * NR + k] * a->dphi[k];
        }
        a->z1[i] = z;
        a->dz1[i] = dz;
        a->h1[i] = silu(z);
        a->dh1[i] = silu1(z) * dz;
    }
    for (int i = 0; i < H; i++) {
        double z = m->b2[i], dz = 0.0;
        for (int j = 0; j < H; j++) {
            z += m->W2[i * H + j] * a->h1[j];
            dz += m->W2[i * H + j] * a->dh1[j];
        }
        a->z2[i] = z;
        a->dz2[i] = dz;
        a->h2[i] = silu(z);
        a->dh2[i] = silu1(z) * dz;
    }
    double y = m->b3[0], dy = 0.0;
    for (int i = 0; i < H; i++) {
        y += m->w3[i] * a->h2[i];
        dy += m->w3[i] * a->dh2[i];
    }
    a->y = y;
    a->dy = dy;
    const double x = M_PI * r / rc;
    a->fc = 0.5 * (cos(x) + 1.0);
    a->dfc = -0.5 * M_PI / rc * sin(x);
}

void orc_mlp_nodes_n(const double *theta, int32_t nt, double rc, double w, double *u, double *du) {
    for (int t = 0; t < nt; t++) {
        const mlp_view m = view(theta, t);
#pragma omp parallel for schedule(static)
        for (int g = 0; g <= NG; g++) {
            node_act a;
            node_forward(&m, g * (rc / NG), rc, w, &a);
            u[t * (NG + 1) + g] = a.y * a.fc;
            du[t * (NG + 1) + g] = a.dy * a.fc + a.y * a.dfc;
        }
    }
}

/* Hermite coefficients of interval g from the end values/derivatives (h = interval). */
static void hermite(double y0, double d0, double y1, double d1, double h, double c[4]) {
    c[0] = y0;
    c[1] = h * d0;
    c[2] = 3.0 * (y1 - y0) - h * (2.0 * d0 + d1);
    c[3] = 2.0 * (y0 - y1) + h * (d0 + d1);
}

void orc_mlp_nodes(const double *theta, double rc, double *u, double *du) {
    orc_mlp_nodes_n(theta, ORC_MLP_NT, rc, ORC_MLP_WIDTH, u, du);
}

void orc_mlp_table_n(const double *theta, int32_t nt, double rc, double w, double *coef) {
    double *u = (double *)malloc(sizeof(double) * nt * (NG + 1));
    double *du = (double *)malloc(sizeof(double) * nt * (NG + 1));
    orc_mlp_nodes_n(theta, nt, rc, w, u, du);
    const double h = rc / NG;
    for (int t = 0; t < nt; t++)
        for (int g = 0; g < NG; g++) {
            const int b = t * (NG + 1) + g;
            hermite(u[b], du[b], u[b + 1], du[b + 1], h, coef + ((size_t)t * NG + g) * 4);
        }
    free(u);
    free(du);
}

void orc_mlp_pair(const double *coef, int32_t type, double rc, double r, double *u, double *F,
                  double *dF) {
    const double h = rc / NG;
    double q = r / h;
    int g = (int)floor(q);
    if (g > NG - 1) g = NG - 1;
    if (g < 0) g = 0;
    const double s = q - g;
    const double *c = coef + ((size_t)type * NG + g) * 4;
    if (u) *u = c[0] + s * (c[1] + s * (c[2] + s * c[3]));
    const double d1 = (c[1] + s * (2.0 * c[2] + 3.0 * s * c[3])) / h;
    const double d2 = (2.0 * c[2] + 6.0 * s * c[3]) / (h * h);
    if (F) *F = -d1;
    if (dF) *dF = -d2;
}

void orc_mlp_table(const double *theta, double rc, double *coef) {
    orc_mlp_table_n(theta, ORC_MLP_NT, rc, ORC_MLP_WIDTH, coef);
}

void orc_mlp_backprop(const double *theta, double rc, const double *coef_adj, double *dtheta) {
    orc_mlp_backprop_n(theta, ORC_MLP_NT, rc, ORC_MLP_WIDTH, coef_adj, dtheta);
}

void orc_mlp_backprop_n(const double *theta, int32_t nt, double rc, double w, const double *coef_adj,
                        double *dtheta) {
    const double h = rc / NG;
    for (int t = 0; t < nt; t++) {
        const mlp_view m = view(theta, t);
        /* coefficient adjoints -> node value / derivative adjoints */
        double *au = (double *)calloc(NG + 1, sizeof(double));
        double *ad = (double *)calloc(NG + 1, sizeof(double));
        for (int g = 0; g < NG; g++) {
            const double *ca = coef_adj + ((size_t)t * NG + g) * 4;
            /* c0 = y0; c1 = h d0; c2 = 3(y1 - y0) - h(2 d0 + d1); c3 = 2(y0 - y1) + h(d0 + d1) */
            au[g] += ca[0] - 3.0 * ca[2] + 2.0 * ca[3];
            au[g + 1] += 3.0 * ca[2] - 2.0 * ca[3];
            ad[g] += h * ca[1] - 2.0 * h * ca[2] + h * ca[3];
            ad[g + 1] += -h * ca[2] + h * ca[3];
        }
        double *dW1 = dtheta + (size_t)t * ORC_MLP_PER_TYPE;
        double *db1 = dW1 + H * NR, *dW2 = db1 + H, *db2 = dW2 + H * H, *dw3 = db2 + H, *db3 = dw3 + H;
        for (int g = 0; g <= NG; g++) {
            if (au[g] == 0.0 && ad[g] == 0.0) continue;
            node_act a;
            node_forward(&m, g * h, rc, w, &a);
            /* u = y fc, u' = y' fc + y fc' */
            const double yb = au[g] * a.fc + ad[g] * a.dfc, dyb = ad[g] * a.fc;
            double z2b[H], dz2b[H], h1b[H], dh1b[H];
            db3[0] += yb;
            for (int i = 0; i < H; i++) {
                dw3[i] += yb * a.h2[i] + dyb * a.dh2[i];
                const double h2b = yb * m.w3[i], dh2b = dyb * m.w3[i];
                /* h2 = silu(z2), dh2 = silu'(z2) dz2 */
                z2b[i] = h2b * silu1(a.z2[i]) + dh2b * silu2(a.z2[i]) * a.dz2[i];
                dz2b[i] = dh2b * silu1(a.z2[i]);
                db2[i] += z2b[i];
            }
            for (int j = 0; j < H; j++) {
                double s1 = 0.0, s2 = 0.0;
                for (int i = 0; i < H; i++) {
                    dW2[i * H + j] += z2b[i] * a.h1[j] + dz2b[i] * a.dh1[j];
                    s1 += m.W2[i * H + j] * z2b[i];
                    s2 += m.W2[i * H + j] * dz2b[i];
                }
                h1b[j] = s1;
                dh1b[j] = s2;
            }
            for (int i = 0; i < H; i++) {
                const double z1b = h1b[i] * silu1(a.z1[i]) + dh1b[i] * silu2(a.z1[i]) * a.dz1[i];
                const double dz1b = dh1b[i] * silu1(a.z1[i]);
                db1[i] += z1b;
                for (int k = 0; k < NR; k++) dW1[i * NR + k] += z1b * a.phi[k] + dz1b * a.dphi[k];
            }
        }
        free(au);
        free(ad);
    }
}

/* splitmix64 -> uniform [0, 1) */
static double u01(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

void orc_mlp_init(uint64_t seed, double *theta) {
    uint64_t s = seed;
    memset(theta, 0, sizeof(double) * ORC_MLP_NPARAMS);
    for (int t = 0; t < ORC_MLP_NT; t++) {
        double *p = theta + (size_t)t * ORC_MLP_PER_TYPE;
        double *W1 = p, *W2 = p + H * NR + H, *w3 = W2 + H * H + H;
        const double a1 = sqrt(6.0 / (NR + H)), a2 = sqrt(6.0 / (H + H)), a3 = sqrt(6.0 / (H + 1));
        for (int i = 0; i < H * NR; i++) W1[i] = a1 * (2.0 * u01(&s) - 1.0);
        for (int i = 0; i < H * H; i++) W2[i] = a2 * (2.0 * u01(&s) - 1.0);
        for (int i = 0; i < H; i++) w3[i] = 0.01 * a3 * (2.0 * u01(&s) - 1.0);
    }
}
