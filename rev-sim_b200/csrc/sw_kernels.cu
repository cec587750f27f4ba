// sw_kernels.cu -- Stillinger-Weber diamond kernels (sm_100a): candidate-list build,
// per-centre terms with forward-mode tangents, deterministic gather + integrators,
// stress reductions.  Follows diamond/diamond.jl: SW terms 348-381 and 444-532, the
// Enzyme VJP and parameter pullback of sw_force_and_grads! 1658-1697, the stress
// tensor and loss 753-786, the forward step 1462-1467 and the reverse step 1801-1846.
// The decomposition into per-centre slot gradients is described in sw_internal.h.
#include "sw_internal.h"

namespace rs {
namespace sw {

namespace {

// ------------------------------------------------------------------ duals
// Forward-mode dual with K tangents (K = 0: a plain value).  Tangent 0 is the
// position direction (w or S d), tangents 1..3 are a, gamma, sigma.  Every value
// operation is the same rounding intrinsic whatever K is, so value parts are
// bit-identical between the forward (K = 0) and reverse (K = 4) kernels.
template <typename R, int K>
struct SD {
    R v;
    R d[K > 0 ? K : 1];
};

template <typename R, int K>
__device__ __forceinline__ SD<R, K> sdc(R v) {
    SD<R, K> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = R(0);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> operator+(const SD<R, K> &a, const SD<R, K> &b) {
    SD<R, K> r;
    r.v = xadd(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xadd(a.d[k], b.d[k]);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> operator-(const SD<R, K> &a, const SD<R, K> &b) {
    SD<R, K> r;
    r.v = xsub(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xsub(a.d[k], b.d[k]);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> operator*(const SD<R, K> &a, const SD<R, K> &b) {
    SD<R, K> r;
    r.v = xmul(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xfma(a.d[k], b.v, xmul(a.v, b.d[k]));
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> operator*(R a, const SD<R, K> &b) {
    SD<R, K> r;
    r.v = xmul(a, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xmul(a, b.d[k]);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> operator/(const SD<R, K> &a, const SD<R, K> &b) {
    SD<R, K> r;
    r.v = xdiv(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xdiv(xsub(a.d[k], xmul(r.v, b.d[k])), b.v);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> sd_exp(const SD<R, K> &a) {
    SD<R, K> r;
    r.v = xexp(a.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xmul(r.v, a.d[k]);
    return r;
}
__device__ __forceinline__ float xrcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double xrcp(double a) { return __drcp_rn(a); }

template <typename R, int K>
__device__ __forceinline__ SD<R, K> sd_inv(const SD<R, K> &a) {
    SD<R, K> r;
    r.v = xrcp(a.v);
    const R m = -xmul(r.v, r.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xmul(m, a.d[k]);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ SD<R, K> sd_neg(const SD<R, K> &a) {
    SD<R, K> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = -a.d[k];
    return r;
}

__device__ __forceinline__ double dist2(const double *xa, const double *xb, double L, double d[3]) {
    d[0] = vec1d(xa[0], xb[0], L);
    d[1] = vec1d(xa[1], xb[1], L);
    d[2] = vec1d(xa[2], xb[2], L);
    return __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2]));
}

// Sum NV per-thread doubles over the CTA in a fixed order; thread k < NV then adds (or
// writes) the total to out[k].
template <int NV>
__device__ __forceinline__ void cta_sum(double (*s_red)[9], const double *val, double *out,
                                        bool accumulate) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        v[k] = val[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] = __dadd_rn(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    }
    const int warp = threadIdx.x / 32, nw = blockDim.x / 32;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) s_red[warp][k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int w = 0; w < nw; w++) t = __dadd_rn(t, s_red[w][threadIdx.x]);
        out[threadIdx.x] = accumulate ? __dadd_rn(out[threadIdx.x], t) : t;
    }
    __syncthreads();
}

// ------------------------------------------------------------ candidate list
__global__ void k_cell_count(SwNlArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.N) return;
    const int r = a.atom_rep[e];
    const int nc = a.rep_nc[r];
    const double L = a.rep_box[r];
    int ci[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const double xu = a.x[3 * (size_t)e + u];
        a.x_nl[3 * (size_t)e + u] = xu;
        int cc = (int)floor(xu / L * nc);
        ci[u] = cc < 0 ? 0 : (cc >= nc ? nc - 1 : cc);
    }
    const int cell = a.rep_cell_off[r] + (ci[2] * nc + ci[1]) * nc + ci[0];
    a.cell_of[e] = cell;
    atomicAdd(a.cell_cnt + cell, 1);
}

__global__ void k_cell_scan(SwNlArgs a) {
    __shared__ int s_part[1024];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < a.n_cells; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < a.n_cells ? a.cell_cnt[i] : 0;
        s_part[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < blockDim.x; off <<= 1) {
            const int t = threadIdx.x >= off ? s_part[threadIdx.x - off] : 0;
            __syncthreads();
            s_part[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < a.n_cells) {
            a.cell_start[i] = s_carry + s_part[threadIdx.x] - v;
            a.cell_fill[i] = 0;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry += s_part[threadIdx.x];
        __syncthreads();
    }
}

// Cell-ordered FP32 copy of the positions with the atom index in .w: the candidate test
// streams one 16-byte load per atom.
__global__ void k_cell_fill(SwNlArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.N) return;
    const int c = a.cell_of[e];
    const double *x = a.x + 3 * (size_t)e;
    a.cell_pos[a.cell_start[c] + atomicAdd(a.cell_fill + c, 1)] =
        make_float4((float)x[0], (float)x[1], (float)x[2], __int_as_float(e));
}

// Candidate row of atom e: every other atom of its replica within a sigma + skin, ascending
// index.  The rows only need to hold every active pair (the terms kernel decides activity
// exactly, in FP64), so the test is FP32 with a 1e-4 nm margin.  Cells are at least that
// wide and number at least 3 per side, so the 27 cells around e are distinct and hold
// every candidate.  One warp per atom: lane l < 27 scans cell l, hits are collected in
// shared memory in any order, then each hit is written at its rank (distinct atoms).
constexpr int ROWS_WARPS = 8;
__global__ void __launch_bounds__(32 * ROWS_WARPS) k_rows(SwNlArgs a) {
    __shared__ int s_list[ROWS_WARPS][CAND];
    __shared__ int s_cnt[ROWS_WARPS];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int e = blockIdx.x * ROWS_WARPS + warp;
    if (e >= a.N) return;
    const int r = a.atom_rep[e];
    const int nc = a.rep_nc[r], off = a.rep_cell_off[r];
    const double L = a.rep_box[r];
    const int loc = a.cell_of[e] - off;
    const int cx = loc % nc, cy = (loc / nc) % nc, cz = loc / (nc * nc);
    const float xe0 = (float)a.x[3 * (size_t)e], xe1 = (float)a.x[3 * (size_t)e + 1],
                xe2 = (float)a.x[3 * (size_t)e + 2];
    const float Lf = (float)L, iLf = (float)(1.0 / L), rl2 = a.rl2f;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    if (lane < 27) {
        const int z = (cz + lane / 9 - 1 + nc) % nc;
        const int y = (cy + (lane / 3) % 3 - 1 + nc) % nc;
        const int xx = (cx + lane % 3 - 1 + nc) % nc;
        const int cell = off + (z * nc + y) * nc + xx;
        const int s0 = a.cell_start[cell], s1 = s0 + a.cell_cnt[cell];
        for (int q = s0; q < s1; q++) {
            const float4 pj = a.cell_pos[q];
            const int j = __float_as_int(pj.w);
            float dx = pj.x - xe0, dy = pj.y - xe1, dz = pj.z - xe2;
            dx -= Lf * rintf(dx * iLf);
            dy -= Lf * rintf(dy * iLf);
            dz -= Lf * rintf(dz * iLf);
            if (j != e && dx * dx + dy * dy + dz * dz < rl2) {
                const int k = atomicAdd(&s_cnt[warp], 1);
                if (k < CAND) s_list[warp][k] = j;
            }
        }
    }
    __syncwarp();
    const int cnt = s_cnt[warp];
    const int m = cnt < CAND ? cnt : CAND;
    int *out = a.cand + (size_t)e * CAND;
    for (int it = lane; it < m; it += 32) {
        const int v = s_list[warp][it];
        int rank = 0;
        for (int k = 0; k < m; k++) rank += s_list[warp][k] < v ? 1 : 0;
        out[rank] = v;
    }
    if (lane == 0) {
        if (cnt > CAND) atomicOr(a.status, ST_NLIST_OVERFLOW);
        a.cand_n[e] = m;
        atomicMax(a.max_cnt, cnt);
    }
}

// ------------------------------------------------------------------ terms
// One group of G lanes per centre c.  Phase 1: the candidates are tested in FP64
// (r / sigma < a, as diamond.jl:351) and the active ones compacted into slots in
// ascending index order.  Phase 2: lane q prepares slot q (unit vector, 3-body radial
// factor h = exp(gamma / (s - a)), its derivative factors, the 2-body radial
// derivative).  Phase 3: lane q sums over the other slots q' the 3-body gradient with
// respect to d_q; with u = d / r, cos = u_q . u_q', c3 = cos + 1/3,
//   dE3/dd_q = eps lambda h_q' c3 [ (c3 alpha_q - cos beta_q) u_q + beta_q u_q' ],
//   alpha_q = dh_q/ds / sigma,  beta_q = 2 h_q / r_q,
// so T_q = u_q (eps A g2_q / 2 + eps lambda S1) + eps lambda beta_q V with
// S1 = sum h_q' c3 (c3 alpha_q - cos beta_q), V = sum h_q' c3 u_q'.
template <typename R, int G, int MODE>
__global__ void __launch_bounds__(TERM_THREADS) k_terms(SwTermArgs t, SwConsts<R> p) {
    constexpr int K = MODE == TM_VALUE ? 0 : 4;
    constexpr int GPB = TERM_THREADS / G;
    using D = SD<R, K>;
    __shared__ double s_d[GPB][G][3];
    __shared__ R s_dd[GPB][G][3];
    __shared__ int s_j[GPB][G];
    // slot data read by the other lanes, in 4-vectors: (u, h), (u', h'_pos), (h'_a, h'_gamma,
    // h'_sigma, -) -- the unit vector, its position tangent (u does not depend on theta)
    // and the 3-body radial factor h with its tangents
    using V4 = typename V4T<R>::T;
    __shared__ V4 s_uh[GPB][G];
    __shared__ V4 s_ut[GPB][K > 0 ? G : 1];
    chain_enter();
    __shared__ V4 s_ht[GPB][K > 0 ? G : 1];
    __shared__ double s_red[TERM_THREADS / 32][9];

    const int lane = threadIdx.x % G, grp = threadIdx.x / G;
    const int gshift = (threadIdx.x % 32) / G * G;
    const unsigned gbits = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
    const unsigned gmask = gbits << gshift;
    const int b = blockIdx.x;
    const int rep = t.blk_rep[b];
    const bool live = grp < t.blk_n[b];
    const int c = t.blk_atom0[b] + grp;
    const double L = t.rep_box[rep];

    double xc[3] = {0.0, 0.0, 0.0}, wc[3] = {0.0, 0.0, 0.0}, ac[3] = {0.0, 0.0, 0.0};
    int nc = 0;
    if (live) {
#pragma unroll
        for (int u = 0; u < 3; u++) xc[u] = t.x[3 * (size_t)c + u];
        nc = t.cand_n[c];
        if (lane == 0) {
            double d[3];
            if (dist2(t.x_nl + 3 * (size_t)c, xc, L, d) > t.half_skin2) atomicOr(t.status, ST_SKIN);
        }
        if (MODE == TM_REV) {
#pragma unroll
            for (int u = 0; u < 3; u++) {
                wc[u] = __dmul_rn(t.C[3 * (size_t)c + u], t.inv_m);
                ac[u] = __dmul_rn(t.A[3 * (size_t)c + u], t.acoef_scale);
            }
        }
    }
    const double *S = MODE == TM_LOSS ? t.S + 9 * rep : nullptr;
    const double invV = MODE == TM_LOSS ? 1.0 / t.rep_vol[rep] : 0.0;

    // Phase 1: active slots.
    int n = 0;
    for (int k0 = 0; k0 < nc; k0 += G) {
        const int k = k0 + lane;
        bool act = false;
        double d[3] = {0.0, 0.0, 0.0};
        int j = -1;
        if (k < nc) {
            j = t.cand[(size_t)c * CAND + k];
            const double r2 = dist2(xc, t.x + 3 * (size_t)j, L, d);
            // r / sigma < a decided in FP64 as the reference rounds it; r^2 outside a
            // 1e-9 relative band around (a sigma)^2 decides it without the root.
            act = r2 < p.lo2 || (r2 <= p.hi2 && __ddiv_rn(__dsqrt_rn(r2), p.sig64) < p.a64);
        }
        const unsigned bal = (__ballot_sync(gmask, act) >> gshift) & gbits;
        if (act) {
            const int q = n + __popc(bal & ((1u << lane) - 1u));
            if (q < G) {
                s_j[grp][q] = j;
#pragma unroll
                for (int u = 0; u < 3; u++) s_d[grp][q][u] = d[u];
                if (MODE == TM_REV) {
#pragma unroll
                    for (int u = 0; u < 3; u++)
                        s_dd[grp][q][u] = (R)__dsub_rn(__dmul_rn(t.C[3 * (size_t)j + u], t.inv_m), wc[u]);
                } else if (MODE == TM_LOSS) {
#pragma unroll
                    for (int u = 0; u < 3; u++)
                        s_dd[grp][q][u] = (R)__dadd_rn(__dadd_rn(__dmul_rn(S[3 * u], d[0]),
                                                                  __dmul_rn(S[3 * u + 1], d[1])),
                                                       __dmul_rn(S[3 * u + 2], d[2]));
                }
            }
        }
        n += __popc(bal);
    }
    if (n > G) {
        if (lane == 0) atomicOr(t.status, ST_NLIST_OVERFLOW);
        n = G;
    }
    if (live && lane == 0) {
        t.act_n[c] = n;
        atomicMax(t.max_act, n);
    }
    __syncwarp(gmask);

    // Phase 2: per-slot quantities (u = d / r, h = exp(gamma / t), alpha = dh/ds / sigma,
    // beta = 2 h / r with s = r / sigma, t = s - a; t from an FP64 difference to keep its
    // digits near the cutoff).  Divisions are reciprocals.
    const bool own = lane < n;
    D u[3], alpha = sdc<R, K>(R(0)), beta = sdc<R, K>(R(0)), sD = sdc<R, K>(R(1)),
            itD = sdc<R, K>(R(0)), it2 = sdc<R, K>(R(0)), g2 = sdc<R, K>(R(0));
    R gB = R(0);
    D gm = sdc<R, K>(R(0));   // learned term: u'(r) / 2, the slot's half of the pair
    int mg = -1;              // its interval (-1: off) and position in it
    R msv = R(0);
#pragma unroll
    for (int k = 0; k < 3; k++) u[k] = sdc<R, K>(R(0));
    D gam = sdc<R, K>(p.gam), isig = sdc<R, K>(p.isig);
    if constexpr (K > 0) {
        gam.d[2] = R(1);
        isig.d[3] = -xmul(p.isig, p.isig);
    }
    if (own) {
        double d64[3];
#pragma unroll
        for (int k = 0; k < 3; k++) d64[k] = s_d[grp][lane][k];
        t.act_idx[(size_t)c * G + lane] = s_j[grp][lane];
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d64[0], d64[0]), __dmul_rn(d64[1], d64[1])),
                                    __dmul_rn(d64[2], d64[2]));
        const R r = xsqrt((R)r2), ir = xrcp(r);
        R rdot = R(0);
#pragma unroll
        for (int k = 0; k < 3; k++) u[k].v = xmul((R)d64[k], ir);
        sD.v = xmul(r, p.isig);
        // t = s - a = (r^2 - (a sigma)^2) / (sigma (r + a sigma)), the difference in FP64
        D tD = sdc<R, K>(xmul((R)__dsub_rn(r2, p.lim2), xrcp(xmul(p.sig, xadd(r, p.asig)))));
        D irD = sdc<R, K>(ir);
        if constexpr (K > 0) {
            // position tangent: r' = u . d'; u' = (d' - u r') / r; s' = r' / sigma;
            // parameter tangents: dt/da = -1, ds/dsigma = dt/dsigma = -s / sigma
            R dd[3];
#pragma unroll
            for (int k = 0; k < 3; k++) dd[k] = s_dd[grp][lane][k];
            rdot = xfma(u[0].v, dd[0], xfma(u[1].v, dd[1], xmul(u[2].v, dd[2])));
#pragma unroll
            for (int k = 0; k < 3; k++) u[k].d[0] = xmul(xsub(dd[k], xmul(u[k].v, rdot)), ir);
            sD.d[0] = xmul(rdot, p.isig);
            sD.d[3] = -xmul(sD.v, p.isig);
            tD.d[0] = sD.d[0];
            tD.d[1] = R(-1);
            tD.d[3] = sD.d[3];
            irD.d[0] = -xmul(rdot, xmul(ir, ir));
        }
        itD = sd_inv(tD);
        it2 = itD * itD;
        const D h = sd_exp(gam * itD);
        alpha = sd_neg(((gam * h) * it2) * isig);
        beta = R(2) * (h * irD);
        // 2-body: dE2/dr / (eps A) = e^{1/t} (-4 B s^-5 - (B s^-4 - 1) / t^2) / sigma
        // (diamond.jl:453), and its B derivative.
        const D e1 = sd_exp(itD);
        const D is = sd_inv(sD);
        const D is2 = is * is, is4 = is2 * is2, is5 = is4 * is;
        g2 = (e1 * sd_neg((R(4) * p.B) * is5 + ((p.B * is4) - sdc<R, K>(R(1))) * it2)) * isig;
        gB = xmul(xmul(e1.v, -xadd(xmul(R(4), is5.v), xmul(is4.v, it2.v))), p.isig);
        if (t.mlp_tab && r2 < p.mlp_rc2) {
            // u'/2 = (c1 + s (2 c2 + 3 s c3)) NG / (2 rc) on the cubic segment of interval
            // g, s = r NG / rc - g; its position tangent u''/2 r' = (c2 + 3 s c3) (NG/rc)^2 r'
            const R q = xmul(r, p.mlp_hinv);
            mg = min((int)q, MLP_NG - 1);
            msv = xsub(q, (R)mg);
            const V4 cc = reinterpret_cast<const V4 *>(t.mlp_tab)[mg];
            const R s3 = xmul(R(3), msv);
            gm.v = xmul(xfma(msv, xfma(s3, cc.w, xmul(R(2), cc.z)), cc.y), p.mlp_hhalf);
            if constexpr (K > 0) gm.d[0] = xmul(xmul(xfma(s3, cc.w, cc.z), p.mlp_hinv2), rdot);
        }
        V4 uh;
        uh.x = u[0].v;
        uh.y = u[1].v;
        uh.z = u[2].v;
        uh.w = h.v;
        s_uh[grp][lane] = uh;
        if constexpr (K > 0) {
            V4 ut, ht;
            ut.x = u[0].d[0];
            ut.y = u[1].d[0];
            ut.z = u[2].d[0];
            ut.w = h.d[0];
            ht.x = h.d[1];
            ht.y = h.d[2];
            ht.z = h.d[3];
            ht.w = R(0);
            s_ut[grp][lane] = ut;
            s_ht[grp][lane] = ht;
        }
    }
    __syncwarp(gmask);

    // Phase 3: 3-body sums over the other slots.  The value arithmetic is the same
    // sequence of rounded operations for every K; the tangents use that u and cos
    // depend on the position direction only (tangent 0), not on the parameters.
    D S1 = sdc<R, K>(R(0)), V[3];
#pragma unroll
    for (int k = 0; k < 3; k++) V[k] = sdc<R, K>(R(0));
    if (own) {
        const R third = R(1) / R(3);
        R ud[3] = {R(0), R(0), R(0)};
        if constexpr (K > 0) {
#pragma unroll
            for (int k = 0; k < 3; k++) ud[k] = u[k].d[0];
        }
        for (int q2 = 0; q2 < n; q2++) {
            // the slot itself enters with weight 0 (its terms are finite), which keeps the
            // lanes of a group on one path
            const R one = q2 == lane ? R(0) : R(1);
            const V4 uh2 = s_uh[grp][q2];
            const R u2[3] = {uh2.x, uh2.y, uh2.z};
            const R h2 = xmul(uh2.w, one);
            const R cs = xadd(xadd(xmul(u[0].v, u2[0]), xmul(u[1].v, u2[1])), xmul(u[2].v, u2[2]));
            const R c3 = xadd(cs, third);
            const R w = xmul(h2, c3);
            const R X = xsub(xmul(c3, alpha.v), xmul(cs, beta.v));
            S1.v = xadd(S1.v, xmul(w, X));
#pragma unroll
            for (int k = 0; k < 3; k++) V[k].v = xadd(V[k].v, xmul(w, u2[k]));
            if constexpr (K > 0) {
                const V4 ut2 = s_ut[grp][q2], ht2 = s_ht[grp][q2];
                const R u2d[3] = {ut2.x, ut2.y, ut2.z};
                const R h2d[4] = {ut2.w, ht2.x, ht2.y, ht2.z};
                const R csd = xfma(ud[0], u2[0], xfma(u[0].v, u2d[0], xfma(ud[1], u2[1], xfma(u[1].v, u2d[1],
                                   xfma(ud[2], u2[2], xmul(u[2].v, u2d[2]))))));
                R wd[K], Xd[K];
                wd[0] = xfma(xmul(h2d[0], one), c3, xmul(h2, csd));
                Xd[0] = xsub(xfma(csd, alpha.v, xmul(c3, alpha.d[0])), xfma(csd, beta.v, xmul(cs, beta.d[0])));
#pragma unroll
                for (int kk = 1; kk < K; kk++) {
                    wd[kk] = xmul(xmul(h2d[kk], one), c3);
                    Xd[kk] = xsub(xmul(c3, alpha.d[kk]), xmul(cs, beta.d[kk]));
                }
#pragma unroll
                for (int kk = 0; kk < K; kk++) S1.d[kk] = xfma(wd[kk], X, xfma(w, Xd[kk], S1.d[kk]));
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    V[k].d[0] = xfma(wd[0], u2[k], xfma(w, u2d[k], V[k].d[0]));
#pragma unroll
                    for (int kk = 1; kk < K; kk++) V[k].d[kk] = xfma(wd[kk], u2[k], V[k].d[kk]);
                }
            }
        }
    }
    double d64[3] = {0.0, 0.0, 0.0};
    if (own) {
#pragma unroll
        for (int k = 0; k < 3; k++) d64[k] = s_d[grp][lane][k];
    }
    D T[3];
    const D coef = (p.half_eA * g2 + p.el * S1) + gm;
    const D elb = p.el * beta;
#pragma unroll
    for (int k = 0; k < 3; k++) T[k] = u[k] * coef + elb * V[k];
    if (own) {
        using V4 = typename V4T<R>::T;
        V4 tv;
        tv.x = T[0].v;
        tv.y = T[1].v;
        tv.z = T[2].v;
        tv.w = R(0);
        reinterpret_cast<V4 *>(t.Tv)[(size_t)c * G + lane] = tv;
        if constexpr (K > 0) {
            V4 tt;
            tt.x = T[0].d[0];
            tt.y = T[1].d[0];
            tt.z = T[2].d[0];
            tt.w = R(0);
            reinterpret_cast<V4 *>(t.Tt)[(size_t)c * G + lane] = tt;
        }
    }

    // Parameter contraction sum_q z_q . dT_q/dtheta (theta order A, B, a, lambda, gamma,
    // sigma, eps); the linear parameters from the value parts.
    if constexpr (MODE != TM_VALUE) {
      if (t.part) {
        double con[NP] = {0, 0, 0, 0, 0, 0, 0};
        if (own) {
            R z[3];
            const int j = s_j[grp][lane];
            if (MODE == TM_REV) {
#pragma unroll
                for (int k = 0; k < 3; k++)
                    z[k] = (R)__dsub_rn(__dmul_rn(t.A[3 * (size_t)j + k], t.acoef_scale), ac[k]);
            } else {
#pragma unroll
                for (int k = 0; k < 3; k++)
                    z[k] = (R)__dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(S[3 * k], d64[0]),
                                                            __dmul_rn(S[3 * k + 1], d64[1])),
                                                  __dmul_rn(S[3 * k + 2], d64[2])),
                                        invV);
            }
            R zu = R(0), zT3 = R(0), zd[3] = {R(0), R(0), R(0)};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                zu = xfma(z[k], u[k].v, zu);
                zT3 = xfma(z[k], xfma(u[k].v, S1.v, xmul(beta.v, V[k].v)), zT3);
#pragma unroll
                for (int m = 0; m < 3; m++) zd[m] = xfma(z[k], T[k].d[1 + m], zd[m]);
            }
            const double sgn = MODE == TM_REV ? -1.0 : 1.0;
            const double half_g2zu = 0.5 * (double)g2.v * (double)zu;
            con[0] = sgn * (double)p.eps * half_g2zu;
            con[1] = sgn * (double)p.half_eA * (double)gB * (double)zu;
            con[2] = sgn * (double)zd[0];
            con[3] = sgn * (double)p.eps * (double)zT3;
            con[4] = sgn * (double)zd[1];
            con[5] = sgn * (double)zd[2];
            con[6] = sgn * ((double)p.A * half_g2zu + (double)p.lam * (double)zT3);
            if (t.mlp_adj && mg >= 0) {
                // z . dT/dc_k = zu k s^(k-1) NG / (2 rc), k = 1..3, into the replica's copy
                const double w = sgn * (double)zu * (double)p.mlp_hhalf, sv = (double)msv;
                double *ad = t.mlp_adj + (((size_t)rep * MLP_NCOPY + (size_t)(c % MLP_NCOPY)) * MLP_NG + mg) * 4;
                atomicAdd(ad + 1, w);
                atomicAdd(ad + 2, 2.0 * w * sv);
                atomicAdd(ad + 3, 3.0 * w * sv * sv);
            }
        }
        cta_sum<NP>(s_red, con, t.part + (size_t)b * NP, true);
      }
    }
    // Virial sum_q T_q (x) d_q (diamond.jl:757-769, as the strain derivative of the energy).
    if (t.wpart) {
        double w9[9];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int bb = 0; bb < 3; bb++) w9[3 * a + bb] = own ? __dmul_rn((double)T[a].v, d64[bb]) : 0.0;
        cta_sum<9>(s_red, w9, t.wpart + (size_t)b * 9, false);
    }
}

// ------------------------------------------------------------------ gather
__device__ __forceinline__ void part1(const SwGatherArgs &g, int e, int rep, const uint64_t *seeds) {
    // Un-integration of diamond.jl:1806-1812: x -= v dt/2; v = (v - xi s) / c; x -= v dt/2;
    // wrap; D = c D + dt^2 dl_dfi (1 + c) / 2; C += D.
    const double L = g.rep_box[rep];
    double xi[3] = {0.0, 0.0, 0.0};
    if (seeds) atom_noise(seeds[rep], (uint32_t)(e - g.rep_atom0[rep]), g.rep_sd[rep], xi);
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const size_t i = 3 * (size_t)e + u;
        double x = g.x[i], v = g.v[i];
        x = __dsub_rn(x, __ddiv_rn(__dmul_rn(v, g.dt), 2.0));
        v = __ddiv_rn(__dsub_rn(v, __dmul_rn(xi[u], g.s)), g.c);
        x = __dsub_rn(x, __ddiv_rn(__dmul_rn(v, g.dt), 2.0));
        g.x[i] = wrap1d(x, L);
        g.v[i] = v;
        const double Dn = __dadd_rn(__dmul_rn(g.c, g.D[i]),
                                    __ddiv_rn(__dmul_rn(__dmul_rn(g.dt2, g.G[i]), __dadd_rn(1.0, g.c)), 2.0));
        g.D[i] = Dn;
        g.C[i] = __dadd_rn(g.C[i], Dn);
    }
}

template <typename R, int G, bool TAN>
__global__ void __launch_bounds__(256) k_gather(SwGatherArgs g) {
    // G lanes per atom e: lane q reads slot q (T_{e,q}) and the matching slot of its
    // neighbour (T_{j_q, slot of e}); a butterfly sum over the lanes (every lane ends
    // with the same bits: each level adds two equal-order pairs) gives f = dE/dx_e and
    // tg, its derivative along the tangent (H w or H u).  Lane 0 writes F = -f and
    // G = -tg; k_finish integrates.
    chain_enter();
    const int lane = threadIdx.x % G;
    const int e = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G);
    const int gshift = (threadIdx.x % 32) / G * G;
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << gshift;
    using V4 = typename V4T<R>::T;
    const V4 *Tv = reinterpret_cast<const V4 *>(g.Tv);
    const V4 *Tt = reinterpret_cast<const V4 *>(g.Tt);
    const bool live = e < g.N;
    double f[3] = {0.0, 0.0, 0.0}, tg[3] = {0.0, 0.0, 0.0};
    if (live) {
        const int n = g.act_n[e];
        if (lane < n) {
            const int j = g.act_idx[(size_t)e * G + lane];
            const int nj = g.act_n[j];
            // the neighbour's whole slot row in G/4 16-byte loads, then compare
            const int4 *rj = reinterpret_cast<const int4 *>(g.act_idx + (size_t)j * G);
            int4 row[G / 4];
#pragma unroll
            for (int k = 0; k < G / 4; k++) row[k] = rj[k];
            int pos = -1;
#pragma unroll
            for (int k = 0; k < G / 4; k++) {
                if (4 * k + 0 < nj && row[k].x == e) pos = 4 * k + 0;
                if (4 * k + 1 < nj && row[k].y == e) pos = 4 * k + 1;
                if (4 * k + 2 < nj && row[k].z == e) pos = 4 * k + 2;
                if (4 * k + 3 < nj && row[k].w == e) pos = 4 * k + 3;
            }
            if (pos < 0) {
                atomicOr(g.status, ST_NLIST_OVERFLOW);
            } else {
                const size_t ie = (size_t)e * G + lane, ij = (size_t)j * G + pos;
                const V4 a = Tv[ij], b = Tv[ie];
                f[0] = __dsub_rn((double)a.x, (double)b.x);
                f[1] = __dsub_rn((double)a.y, (double)b.y);
                f[2] = __dsub_rn((double)a.z, (double)b.z);
                if (TAN) {
                    const V4 at = Tt[ij], bt = Tt[ie];
                    tg[0] = __dsub_rn((double)at.x, (double)bt.x);
                    tg[1] = __dsub_rn((double)at.y, (double)bt.y);
                    tg[2] = __dsub_rn((double)at.z, (double)bt.z);
                }
            }
        }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int u = 0; u < 3; u++) {
            f[u] = __dadd_rn(f[u], __shfl_xor_sync(gmask, f[u], o));
            if (TAN) tg[u] = __dadd_rn(tg[u], __shfl_xor_sync(gmask, tg[u], o));
        }
    }
    if (!live || lane != 0) return;
#pragma unroll
    for (int u = 0; u < 3; u++) {
        g.F[3 * (size_t)e + u] = -f[u];
        if (TAN) g.G[3 * (size_t)e + u] = -tg[u];
    }
    if (!(isfinite(f[0]) && isfinite(f[1]) && isfinite(f[2]) && isfinite(tg[0]) && isfinite(tg[1]) &&
          isfinite(tg[2])))
        atomicOr(g.status, ST_NAN);
}

// One thread per atom: the step (or loss) arithmetic after the gather.
template <int MODE>
__global__ void __launch_bounds__(256) k_finish(SwGatherArgs g) {
    chain_enter();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.N) return;
    double f[3], tg[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        f[u] = -g.F[3 * (size_t)e + u];
        tg[u] = MODE == GM_FWD ? 0.0 : -g.G[3 * (size_t)e + u];
    }
    const int rep = g.atom_rep[e];
    // f = dE/dx_e, tg = its derivative along the tangent (H w or H u).
    if (MODE == GM_FWD) {
        // diamond.jl:1462-1467
        const double L = g.rep_box[rep];
        double xi[3] = {0.0, 0.0, 0.0};
        if (g.seed_cur) atom_noise(g.seed_cur[rep], (uint32_t)(e - g.rep_atom0[rep]), g.rep_sd[rep], xi);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const size_t i = 3 * (size_t)e + u;
            const double F = -f[u];
            double v = __dadd_rn(g.v[i], __ddiv_rn(__dmul_rn(F, g.dt), g.m));
            double x = __dadd_rn(g.x[i], __ddiv_rn(__dmul_rn(v, g.dt), 2.0));
            v = __dadd_rn(__dmul_rn(v, g.c), __dmul_rn(xi[u], g.s));
            x = __dadd_rn(x, __ddiv_rn(__dmul_rn(v, g.dt), 2.0));
            g.x[i] = wrap1d(x, L);
            g.v[i] = v;
        }
        return;
    }
    if (MODE == GM_REV) {
        // diamond.jl:1838-1846: v -= F dt / m; B = c B + dt^2 dl_dfi; A += B
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const size_t i = 3 * (size_t)e + u;
            const double F = -f[u], Gn = -tg[u];
            g.v[i] = __dsub_rn(g.v[i], __ddiv_rn(__dmul_rn(F, g.dt), g.m));
            const double Bn = __dadd_rn(__dmul_rn(g.c, g.B[i]), __dmul_rn(g.dt2, Gn));
            g.B[i] = Bn;
            g.A[i] = __dadd_rn(g.A[i], Bn);
        }
        if (g.fuse_next) part1(g, e, rep, g.seed_next);
        return;
    }
    if (MODE == GM_LOSS) {
        // dL/dx = (H u + S^T dE/dx) / V,  dL/dv = -(m / V) (S + S^T)(v - vbar)
        const double *S = g.S + 9 * rep;
        const double V = g.rep_vol[rep];
        double gx[3], gv[3];
#pragma unroll
        for (int gm = 0; gm < 3; gm++) {
            double st = 0.0;
#pragma unroll
            for (int al = 0; al < 3; al++) st = __dadd_rn(st, __dmul_rn(S[3 * al + gm], f[al]));
            gx[gm] = __ddiv_rn(__dadd_rn(tg[gm], st), V);
            double tv = 0.0;
            if (g.vel_term) {
#pragma unroll
                for (int bb = 0; bb < 3; bb++)
                    tv = __dadd_rn(tv, __dmul_rn(__dadd_rn(S[3 * gm + bb], S[3 * bb + gm]),
                                                 __dsub_rn(g.v[3 * (size_t)e + bb], g.vbar[3 * rep + bb])));
            }
            gv[gm] = g.vel_term ? __ddiv_rn(__dmul_rn(-g.m, tv), V) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const size_t i = 3 * (size_t)e + u;
            if (g.dLdx) g.dLdx[i] = gx[u];
            if (g.dLdv) g.dLdv[i] = gv[u];
            if (g.init_adjoint) {
                // diamond.jl:1789-1793
                const double c = g.c, dt = g.dt;
                g.A[i] = __dadd_rn(__dmul_rn(gx[u], __dadd_rn(1.0, c)), __ddiv_rn(__dmul_rn(__dmul_rn(gv[u], c), 2.0), dt));
                g.B[i] = __dadd_rn(__dmul_rn(gx[u], __dadd_rn(1.0, c)),
                                   __ddiv_rn(__dmul_rn(__dmul_rn(gv[u], __dsub_rn(c, 1.0)), 2.0), dt));
                g.C[i] = __ddiv_rn(__dmul_rn(gv[u], __dadd_rn(1.0, c)), dt);
                g.D[i] = __dadd_rn(__ddiv_rn(__dmul_rn(gx[u], __dadd_rn(__dadd_rn(1.0, __dmul_rn(2.0, c)), __dmul_rn(c, c))),
                                             __dmul_rn(2.0, c)),
                                   __ddiv_rn(__dmul_rn(gv[u], __dsub_rn(c, __ddiv_rn(1.0, c))), dt));
                g.G[i] = 0.0;
            }
        }
    }
}

__global__ void k_part1(SwGatherArgs g) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.N) return;
    part1(g, e, g.atom_rep[e], g.seed_cur);
}

__global__ void k_noise(int N, const int *atom_rep, const int *rep_atom0, const double *rep_sd,
                        const uint64_t *seeds, double *xi) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= N) return;
    const int r = atom_rep[e];
    atom_noise(seeds[r], (uint32_t)(e - rep_atom0[r]), rep_sd[r], xi + 3 * (size_t)e);
}

// ------------------------------------------------------------- reductions
template <int NV>
__device__ __forceinline__ void block_sum256(double (*s)[256], double *v, double *out) {
#pragma unroll
    for (int k = 0; k < NV; k++) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
#pragma unroll
            for (int k = 0; k < NV; k++) s[k][threadIdx.x] = __dadd_rn(s[k][threadIdx.x], s[k][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x < NV) out[threadIdx.x] = s[threadIdx.x][0];
}

__global__ void __launch_bounds__(256) k_vsum(SwRedArgs a) {
    __shared__ double s[3][256];
    const int b = blockIdx.x;
    const int i = threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < a.ablk_n[b]) {
        const size_t e = (size_t)a.ablk_atom0[b] + i;
#pragma unroll
        for (int u = 0; u < 3; u++) v[u] = a.v[3 * e + u];
    }
    block_sum256<3>(s, v, a.vpart + 3 * (size_t)b);
}

// Per-replica sums of block partials: thread t adds blocks b0 + t, b0 + t + 256, ... in
// order, then a fixed tree over the threads.
template <int NV>
__device__ __forceinline__ void range_sum256(double (*s)[256], const double *part, int b0, int b1,
                                             double *out) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = 0.0;
    for (int b = b0 + threadIdx.x; b < b1; b += 256) {
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = __dadd_rn(v[k], part[(size_t)b * NV + k]);
    }
    block_sum256<NV>(s, v, out);
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_vbar(SwRedArgs a) {
    __shared__ double s[3][256];
    __shared__ double tot[3];
    const int r = blockIdx.x;
    range_sum256<3>(s, a.vpart, a.rep_ablk0[r], a.rep_ablk0[r + 1], tot);
    if (threadIdx.x < 3) a.vbar[3 * r + threadIdx.x] = __ddiv_rn(tot[threadIdx.x], (double)a.rep_n[r]);
}

__global__ void __launch_bounds__(256) k_kin(SwRedArgs a) {
    __shared__ double s[9][256];
    const int b = blockIdx.x;
    const int i = threadIdx.x;
    double k9[9];
#pragma unroll
    for (int k = 0; k < 9; k++) k9[k] = 0.0;
    if (i < a.ablk_n[b]) {
        const size_t e = (size_t)a.ablk_atom0[b] + i;
        const int r = a.ablk_rep[b];
        double dv[3];
#pragma unroll
        for (int u = 0; u < 3; u++) dv[u] = __dsub_rn(a.v[3 * e + u], a.vbar[3 * r + u]);
#pragma unroll
        for (int al = 0; al < 3; al++)
#pragma unroll
            for (int be = 0; be < 3; be++) k9[3 * al + be] = __dmul_rn(dv[al], dv[be]);
    }
    block_sum256<9>(s, k9, a.kpart + 9 * (size_t)b);
}

// sigma = (K + W) / V (diamond.jl:753-770); loss = weight sum (sigma - target)^2 / 9
// (diamond.jl:772-775); S = dL/dsigma.
__global__ void __launch_bounds__(256) k_loss_final(SwRedArgs a) {
    __shared__ double s[9][256];
    __shared__ double W[9], Kt[9];
    const int r = blockIdx.x;
    range_sum256<9>(s, a.wpart, a.rep_blk0[r], a.rep_blk0[r + 1], W);
    if (a.vel_term) range_sum256<9>(s, a.kpart, a.rep_ablk0[r], a.rep_ablk0[r + 1], Kt);
    if (threadIdx.x != 0) return;
    const double V = a.rep_vol[r];
    double l = 0.0;
    for (int k = 0; k < 9; k++) {
        const double K = a.vel_term ? __dmul_rn(-a.m, Kt[k]) : 0.0;
        const double sg = __ddiv_rn(__dadd_rn(K, W[k]), V);
        if (a.sigma) a.sigma[9 * r + k] = sg;
        const double e = __dsub_rn(sg, a.target[9 * r + k]);
        l = __dadd_rn(l, __dmul_rn(e, e));
        if (a.S) a.S[9 * r + k] = __ddiv_rn(__dmul_rn(__dmul_rn(2.0, a.weight), e), 9.0);
    }
    l = __dmul_rn(l, __ddiv_rn(a.weight, 9.0));
    if (a.loss) a.loss[r] = l;
    if (a.loss_acc) a.loss_acc[r] = __dadd_rn(a.loss_acc[r], l);
}

__global__ void k_active_pairs(int N, int G, const int *act_idx, const int *act_n, int32_t *pairs,
                               unsigned long long *count, long long max_pairs) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= N) return;
    for (int q = 0; q < act_n[e]; q++) {
        const int j = act_idx[(size_t)e * G + q];
        if (j <= e) continue;
        const unsigned long long k = atomicAdd(count, 1ull);
        if ((long long)k < max_pairs) {
            pairs[2 * k] = e;
            pairs[2 * k + 1] = j;
        }
    }
}

inline int nblk(int n, int t) { return (n + t - 1) / t; }

}  // namespace

// ------------------------------------------------------------------ launchers
cudaError_t launch_sw_nlist(const SwNlArgs &a, cudaStream_t st) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(a.cell_cnt, 0, sizeof(int) * a.n_cells, st))) return e;
    k_cell_count<<<nblk(a.N, 256), 256, 0, st>>>(a);
    k_cell_scan<<<1, 1024, 0, st>>>(a);
    k_cell_fill<<<nblk(a.N, 256), 256, 0, st>>>(a);
    k_rows<<<nblk(a.N, ROWS_WARPS), 32 * ROWS_WARPS, 0, st>>>(a);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_sw_terms(int mode, int G, int n_blk, const SwTermArgs &a, const SwConsts<R> &p,
                            cudaStream_t st) {
#define RS_TERMS(GG, MM) launch_chained(k_terms<R, GG, MM>, dim3(n_blk), dim3(TERM_THREADS), 0, st, a, p)
    if (G == 16) {
        if (mode == TM_VALUE) RS_TERMS(16, TM_VALUE);
        else if (mode == TM_REV) RS_TERMS(16, TM_REV);
        else RS_TERMS(16, TM_LOSS);
    } else if (G == 32) {
        if (mode == TM_VALUE) RS_TERMS(32, TM_VALUE);
        else if (mode == TM_REV) RS_TERMS(32, TM_REV);
        else RS_TERMS(32, TM_LOSS);
    } else {
        return cudaErrorInvalidValue;
    }
#undef RS_TERMS
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_sw_gather(int mode, int G, bool tangent, const SwGatherArgs &a, cudaStream_t st) {
    const int nb = (int)(((size_t)a.N * G + 255) / 256);
    const bool tan = tangent || mode == GM_REV || mode == GM_LOSS;
    if (G == 16) {
        if (tan) launch_chained(k_gather<R, 16, true>, dim3(nb), dim3(256), 0, st, a);
        else launch_chained(k_gather<R, 16, false>, dim3(nb), dim3(256), 0, st, a);
    } else if (G == 32) {
        if (tan) launch_chained(k_gather<R, 32, true>, dim3(nb), dim3(256), 0, st, a);
        else launch_chained(k_gather<R, 32, false>, dim3(nb), dim3(256), 0, st, a);
    } else {
        return cudaErrorInvalidValue;
    }
    const int na = nblk(a.N, 256);
    if (mode == GM_FWD) launch_chained(k_finish<GM_FWD>, dim3(na), dim3(256), 0, st, a);
    else if (mode == GM_REV) launch_chained(k_finish<GM_REV>, dim3(na), dim3(256), 0, st, a);
    else if (mode == GM_LOSS) launch_chained(k_finish<GM_LOSS>, dim3(na), dim3(256), 0, st, a);
    return cudaGetLastError();
}

cudaError_t launch_sw_stress(const SwRedArgs &a, cudaStream_t st) {
    k_vsum<<<a.n_ablk, 256, 0, st>>>(a);
    k_vbar<<<a.R, 256, 0, st>>>(a);
    k_kin<<<a.n_ablk, 256, 0, st>>>(a);
    k_loss_final<<<a.R, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sw_part1(int N, const SwGatherArgs &a, cudaStream_t st) {
    k_part1<<<nblk(N, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sw_noise(int N, const int *atom_rep, const int *rep_atom0, const double *rep_sd,
                            const uint64_t *seeds, double *xi, cudaStream_t st) {
    k_noise<<<nblk(N, 256), 256, 0, st>>>(N, atom_rep, rep_atom0, rep_sd, seeds, xi);
    return cudaGetLastError();
}

cudaError_t launch_sw_active_pairs(int N, int G, const int *act_idx, const int *act_n,
                                   int32_t *pairs, unsigned long long *count, long long max_pairs,
                                   cudaStream_t st) {
    k_active_pairs<<<nblk(N, 256), 256, 0, st>>>(N, G, act_idx, act_n, pairs, count, max_pairs);
    return cudaGetLastError();
}

template cudaError_t launch_sw_terms<float>(int, int, int, const SwTermArgs &, const SwConsts<float> &,
                                            cudaStream_t);
template cudaError_t launch_sw_terms<double>(int, int, int, const SwTermArgs &,
                                             const SwConsts<double> &, cudaStream_t);
template cudaError_t launch_sw_gather<float>(int, int, bool, const SwGatherArgs &, cudaStream_t);
template cudaError_t launch_sw_gather<double>(int, int, bool, const SwGatherArgs &, cudaStream_t);

}  // namespace sw
}  // namespace rs
