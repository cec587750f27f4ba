// gas_kernels.cu -- kernels of the gas-in-water engine (diffusion/diffusion.jl): neighbour
// rows, the fused forward and reverse step kernels, the energy and the small helpers.
//
// Work decomposition: one warp per atom.  The 32 lanes stride over the atom's neighbour row
// (every other atom within the list cutoff, both directions, grouped by site kind), test the
// entries against the cutoff, queue the ones inside per warp and evaluate them 32 at a time
// (see k_gas_step), accumulate the
// atom's force (and in reverse its VJP and the class sums of the parameter derivatives) in
// FP64 registers and combine them with a fixed xor butterfly; lane 0 adds the bonded terms of
// the atom's molecule and runs the atom's integrator update.  Each atom's sums are computed
// by one warp in a fixed order: no atomics, deterministic results.  Positions for the pair
// terms come from a double4 gather copy (pos_in) that the step writes into the other buffer
// (pos_out), so no warp reads a position another warp has already moved.
#include "gas_internal.h"
#include "rs_form_energy.cuh"
#include "rs_step_impl.cuh"

namespace gs {

using namespace rs;

namespace {

__device__ __forceinline__ double kind_mass(int k, double mO, double mH) { return k == 1 ? mH : mO; }

__device__ __forceinline__ double4 ld3(const double *x, int i) {
    const size_t b = 3 * (size_t)i;
    return make_double4(x[b], x[b + 1], x[b + 2], 0.0);
}

template <typename V4>
__device__ __forceinline__ V4 mk4(double a, double b, double c) {
    V4 r;
    r.x = a;
    r.y = b;
    r.z = c;
    r.w = 0;
    return r;
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Radial bond own atom -> partner (displacement d, own to partner): force on the own atom
// -(F/r) d with F = -k (r - r0), and in reverse the VJP M (w_p - w_o).
template <bool REV>
__device__ __forceinline__ void o2_bond(const double d[3], double kb, double r0, const double wo[3],
                                        const double wp[3], double f[3], double g[3]) {
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])),
                                __dmul_rn(d[2], d[2]));
    const double r = __dsqrt_rn(r2);
    const double rinv = __drcp_rn(r);
    const double F = -__dmul_rn(kb, __dsub_rn(r, r0));
    const double Fr = __dmul_rn(F, rinv);
#pragma unroll
    for (int u = 0; u < 3; u++) f[u] = __fma_rn(-Fr, d[u], f[u]);
    if (REV) {
        double e[3];
#pragma unroll
        for (int u = 0; u < 3; u++) e[u] = __dsub_rn(wp[u], wo[u]);
        const double s = __dmul_rn(rinv, __fma_rn(d[2], e[2], __fma_rn(d[1], e[1], __dmul_rn(d[0], e[0]))));
        const double k1 = __dmul_rn(__dmul_rn(__dsub_rn(-kb, Fr), s), rinv);
#pragma unroll
        for (int u = 0; u < 3; u++) g[u] = __dsub_rn(g[u], __fma_rn(k1, d[u], __dmul_rn(Fr, e[u])));
    }
}

// ------------------------------------------------------------------ neighbour rows
// Row of atom i: every atom j of another molecule with min-image d^2 <= rc_nl^2 (Molly's
// per-dimension rule), except water H - gas pairs, which carry no term (no charge on the
// gas, no pair form on H).  Grouped by site kind -- water O, then water H, then gas, each in
// ascending order (ballot compaction over that candidate order) -- so that the 32 lanes of
// a step kernel's warp mostly hold neighbours of one kind and take the same branches.
__device__ __forceinline__ int kind_order(int c, int nw3) {
    const int nw = nw3 / 3;
    if (c < nw) return 3 * c;                        // water O
    if (c < nw3) {                                   // water H1, H2
        const int q = c - nw;
        return 3 * (q >> 1) + 1 + (q & 1);
    }
    return c;                                        // gas
}

__global__ void __launch_bounds__(kThreads) k_gas_rows(GasRowArgs a) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (i >= a.N) return;
    const double4 pa = ld3(a.x, i);
    const int ka = site_kind(i, a.nw3);
    const int mi = i < a.nw3 ? i / 3 : (a.nw3 / 3) + (i - a.nw3) / 2;
    int n = 0;
    int *row = a.rows + (size_t)i * a.cap;
    for (int base = 0; base < a.N; base += 32) {
        const int cand = base + lane;
        const int j = cand < a.N ? kind_order(cand, a.nw3) : a.N;
        bool ok = false;
        if (j < a.N) {
            const int kb = site_kind(j, a.nw3);
            const int mj = j < a.nw3 ? j / 3 : (a.nw3 / 3) + (j - a.nw3) / 2;
            if (mj != mi && !((ka == 1 && kb == 2) || (ka == 2 && kb == 1))) {
                const double4 pb = ld3(a.x, j);
                const double d0 = vec1d(pa.x, pb.x, a.L), d1 = vec1d(pa.y, pb.y, a.L),
                             d2 = vec1d(pa.z, pb.z, a.L);
                const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)),
                                            __dmul_rn(d2, d2));
                ok = r2 <= a.rc_nl2;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const int k = n + __popc(m & ((1u << lane) - 1u));
            if (k < a.cap) row[k] = j;
        }
        n += __popc(m);
    }
    if (lane == 0) {
        a.cnt[i] = min(n, a.cap);
        if (n > a.cap) atomicOr(a.status, ST_NLIST_OVERFLOW);
    }
}

// ------------------------------------------------------------------ step kernels
// Register budget: the LJ reverse kernel at 5 CTAs per SM (96 registers, some spills), so
// that one warp per atom of the 2,675-atom diffusion box fits in one wave (at 128 registers
// 4 CTAs per SM held 2,368 of its warps and the rest ran as a second wave: 50.7 against
// 39.5 us per step); the other reverse forms (dual numbers, more live values) and the
// forward kernels (90 registers, 5 CTAs per SM) unconstrained.
template <int FORM, bool REV>
constexpr int gas_min_blocks() { return (REV && FORM == F_LJ) ? 5 : 1; }

// R: pair arithmetic (float in mixed precision, double in FP64).  The pair loop gathers
// V4T<R> positions and weights; the per-lane sums are R and are combined in FP64; the
// bonded terms and the integrator run in FP64 on the FP64 gather copy pos64.
template <typename R, int FORM, bool REV>
__global__ void __launch_bounds__(kThreads, gas_min_blocks<FORM, REV>()) k_gas_step(const GasConstsT<R> k, const GasArgs a) {
    using V4 = typename V4T<R>::T;
    constexpr int NP = FormInfo<FORM>::NP;
    chain_enter();
    const V4 *pos_in = static_cast<const V4 *>(a.pos_in);
    const V4 *wgt_in = static_cast<const V4 *>(a.wgt_in);
    const R L = (R)a.L, invL = (R)a.invL;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (i >= a.N) return;   // whole warps only
    const int ka = site_kind(i, a.nw3);
    const double ma = kind_mass(ka, a.mO, a.mH);
    const V4 pa = pos_in[i];
    V4 wa = mk4<V4>(0.0, 0.0, 0.0);
    R ca[3] = {R(0), R(0), R(0)};
    if (REV) {
        wa = wgt_in[i];
        const double cf = __ddiv_rn(__dmul_rn(a.dt, a.dt), __dmul_rn(2.0, ma));
#pragma unroll
        for (int u = 0; u < 3; u++)
            ca[u] = (R)(a.acoef_in ? a.acoef_in[3 * (size_t)i + u] : __dmul_rn(a.A[3 * (size_t)i + u], cf));
    }
    R fr[3] = {R(0), R(0), R(0)}, gr[3] = {R(0), R(0), R(0)};
    R accr[3][NP];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int q = 0; q < NP; q++) accr[c][q] = R(0);
    R thqr = R(0);
    const int n = a.cnt[i];
    const int *row = a.rows + (size_t)i * a.cap;
    // Pair terms of one row entry within the cutoff (displacement d, own atom to j).
    auto pair = [&](const int j, const R dx, const R dy, const R dz, const R r2) {
        const int kb = site_kind(j, a.nw3);
        const R rinv = xrsqrt(r2);
        const R r = xmul(r2, rinv);
        const R invr2 = xmul(rinv, rinv);
        R F = R(0), dF = R(0), Fc = R(0);
        const bool coul = ka != 2 && kb != 2;
        if (coul) {
            const int qi = (ka == 1) + (kb == 1);
            const R qq = qi == 0 ? k.qq[0] : qi == 1 ? k.qq[1] : k.qq[2];
            Fc = xmul(qq, xsub(invr2, xmul(k.krf2, r)));
            F = Fc;
            if (REV) dF = -xmul(xadd(qq, qq), xadd(xmul(invr2, rinv), k.krf));
        }
        R gf[4] = {R(0), R(0), R(0), R(0)};
        int cls = -1;
        if (ka != 1 && kb != 1) {
            cls = (ka == 2) + (kb == 2);
            if (cls == 0 ? k.on[0] : cls == 1 ? k.on[1] : k.on[2]) {
                // constant class indices keep the constants in the parameter bank
                R Ff = R(0), dFf = R(0);
                if (cls == 0)
                    pair_form<R, FORM, REV>(k.fc[0], r, rinv, invr2, Ff, dFf, gf);
                else if (cls == 1)
                    pair_form<R, FORM, REV>(k.fc[1], r, rinv, invr2, Ff, dFf, gf);
                else
                    pair_form<R, FORM, REV>(k.fc[2], r, rinv, invr2, Ff, dFf, gf);
                F = xadd(F, Ff);
                if (REV) dF = xadd(dF, dFf);
            } else {
                cls = -1;
            }
        }
        const R Fr = xmul(F, rinv);
        fr[0] = xfma(-Fr, dx, fr[0]);
        fr[1] = xfma(-Fr, dy, fr[1]);
        fr[2] = xfma(-Fr, dz, fr[2]);
        if (REV) {
            const V4 wb = wgt_in[j];
            const R ex = xsub(wb.x, wa.x), ey = xsub(wb.y, wa.y),
                         ez = xsub(wb.z, wa.z);
            const R s = xmul(rinv, xfma(dz, ez, xfma(dy, ey, xmul(dx, ex))));
            const R k1 = xmul(xmul(xsub(dF, Fr), s), rinv);
            gr[0] = xsub(gr[0], xfma(k1, dx, xmul(Fr, ex)));
            gr[1] = xsub(gr[1], xfma(k1, dy, xmul(Fr, ey)));
            gr[2] = xsub(gr[2], xfma(k1, dz, xmul(Fr, ez)));
            const R na = xmul(rinv, xfma(dz, ca[2], xfma(dy, ca[1], xmul(dx, ca[0]))));
            if (coul) thqr = xfma(-xmul(Fc, k.twoinvq), na, thqr);
#pragma unroll
            for (int c = 0; c < 3; c++)
                if (c == cls)
#pragma unroll
                    for (int q = 0; q < NP; q++) accr[c][q] = xfma(-gf[q], na, accr[c][q]);
        }
        };
    // Two phases per warp.  Phase 1: each lane loads GAS_U row entries (all loads issued
    // before any is used, so GAS_U neighbour gathers per lane are in flight), tests them
    // against the cutoff and pushes the ones inside (about 58 % at the list cutoff 1.2 nm)
    // onto a per-warp queue in shared memory.  Phase 2: while 32 or more are queued, all
    // lanes evaluate one each, so the pair arithmetic runs with full warps.  The queue is
    // processed last-in first-out in a fixed order (deterministic sums).
    constexpr int GAS_U = 4, QCAP = 32 * GAS_U + 32;
    __shared__ R s_d[kWarpsPerCta][4][QCAP];
    __shared__ int s_j[kWarpsPerCta][QCAP];
    const int w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int qn = 0;
    for (int base = 0; base < n; base += 32 * GAS_U) {
        int jj[GAS_U];
        V4 pb[GAS_U];
#pragma unroll
        for (int u = 0; u < GAS_U; u++) {
            const int e = base + 32 * u + lane;
            jj[u] = e < n ? row[e] : -1;
        }
#pragma unroll
        for (int u = 0; u < GAS_U; u++)
            if (jj[u] >= 0) pb[u] = pos_in[jj[u]];
#pragma unroll
        for (int u = 0; u < GAS_U; u++) {
            bool ok = false;
            R dx = R(0), dy = R(0), dz = R(0), r2 = R(0);
            if (jj[u] >= 0) {
                dx = vec_mi<R>(pa.x, pb[u].x, L, invL);
                dy = vec_mi<R>(pa.y, pb[u].y, L, invL);
                dz = vec_mi<R>(pa.z, pb[u].z, L, invL);
                r2 = xfma(dz, dz, xfma(dy, dy, xmul(dx, dx)));
                ok = r2 <= k.rc2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int q = qn + __popc(m & lt);
                s_j[w][q] = jj[u];
                s_d[w][0][q] = dx;
                s_d[w][1][q] = dy;
                s_d[w][2][q] = dz;
                s_d[w][3][q] = r2;
            }
            qn += __popc(m);
        }
        __syncwarp();
        while (qn >= 32) {
            const int q = qn - 32 + lane;
            pair(s_j[w][q], s_d[w][0][q], s_d[w][1][q], s_d[w][2][q], s_d[w][3][q]);
            qn -= 32;
        }
        __syncwarp();
    }
    if (lane < qn) pair(s_j[w][lane], s_d[w][0][lane], s_d[w][1][lane], s_d[w][2][lane], s_d[w][3][lane]);
    double f[3], g[3] = {0.0, 0.0, 0.0}, acc[3][NP], thq = 0.0;
#pragma unroll
    for (int u = 0; u < 3; u++) {
        f[u] = wsum((double)fr[u]);
        if (REV) g[u] = wsum((double)gr[u]);
    }
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int q = 0; q < NP; q++) acc[c][q] = 0.0;
    if (REV) {
        thq = wsum((double)thqr);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int q = 0; q < NP; q++) acc[c][q] = wsum((double)accr[c][q]);
    }
    if (lane != 0) return;

    // Every load of the atom's state is issued before its first store: the state arrays
    // are distinct, but the compiler cannot know that and would otherwise serialise the
    // three components behind the stores.  Forward: x and v, before the bonded terms.
    const size_t b = 3 * (size_t)i;
    const bool upd = !(a.mode & MODE_FORCES_ONLY);
    double xk[3] = {0.0, 0.0, 0.0}, vk[3] = {0.0, 0.0, 0.0};
    if (!REV && upd) {
#pragma unroll
        for (int u = 0; u < 3; u++) {
            vk[u] = a.v[b + u];
            xk[u] = a.x[b + u];
        }
    }

    // bonded terms of the atom's molecule (diffusion.jl:997-1050, 1367-1498)
    if (ka != 2) {
        const int m0 = i - i % 3, kk = i % 3;
        double xm[9], w9[9], ac9[9], Fb[9], Gb[9], tb[4];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const double4 p = a.pos64_in[m0 + q];
            xm[3 * q] = p.x;
            xm[3 * q + 1] = p.y;
            xm[3 * q + 2] = p.z;
            V4 w = mk4<V4>(0.0, 0.0, 0.0);
            if (REV) w = wgt_in[m0 + q];
            w9[3 * q] = w.x;
            w9[3 * q + 1] = w.y;
            w9[3 * q + 2] = w.z;
            ac9[3 * q] = ac9[3 * q + 1] = ac9[3 * q + 2] = 0.0;
        }
        bonded<double, REV>(xm, a.L, a.bw, w9, ac9, Fb, Gb, tb);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            f[u] = __dadd_rn(f[u], Fb[3 * kk + u]);
            if (REV) g[u] = __dadd_rn(g[u], Gb[3 * kk + u]);
        }
    } else {
        const int p = ((i - a.nw3) ^ 1) + a.nw3;
        const double4 pp = a.pos64_in[p], po = a.pos64_in[i];
        const double d[3] = {vec1d(po.x, pp.x, a.L), vec1d(po.y, pp.y, a.L), vec1d(po.z, pp.z, a.L)};
        double wo[3] = {0.0, 0.0, 0.0}, wp[3] = {0.0, 0.0, 0.0};
        if (REV) {
            const V4 w = wgt_in[p];
            wo[0] = wa.x; wo[1] = wa.y; wo[2] = wa.z;
            wp[0] = w.x; wp[1] = w.y; wp[2] = w.z;
        }
        o2_bond<REV>(d, a.kb_g, a.r0_g, wo, wp, f, g);
    }
    if (!isfinite(f[0]) || !isfinite(f[1]) || !isfinite(f[2])) atomicOr(a.status, ST_NAN);

    if (REV) {
        // dtheta of the atom: each parameter's contributions in (q, class) order, then the
        // charge term, with compile-time parameter indices so that the sums stay in
        // registers; the partials' loads all issued before their stores
        double *pt = a.part + (size_t)i * k.P;
        double old[kMaxP];
#pragma unroll
        for (int p = 0; p < kMaxP; p++) old[p] = p < k.P ? pt[p] : 0.0;
#pragma unroll
        for (int p = 0; p < kMaxP; p++) {
            double t = 0.0;
#pragma unroll
            for (int q = 0; q < NP; q++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    if (k.iw[q] == p) t = __fma_rn(k.fw[c][q], acc[c][q], t);
                    if (k.ig[q] == p) t = __fma_rn(k.fg[c][q], acc[c][q], t);
                }
            if (k.iq == p) t = __dadd_rn(t, thq);
            if (p < k.P) pt[p] = __dadd_rn(old[p], t);
        }
    }
    if (!upd) {
#pragma unroll
        for (int u = 0; u < 3; u++) {
            a.F_out[b + u] = f[u];
            if (REV) a.G[b + u] = g[u];
        }
        return;
    }
    const double sd = ka == 1 ? a.sdH : a.sdO;
    if (!REV) {
        // B-A-O-A (diffusion.jl:1228-1233)
        double xi[3] = {0.0, 0.0, 0.0};
        if (a.s != 0.0) atom_noise(a.seed_cur, (uint32_t)i, sd, xi);
        double xn[3];
#pragma unroll
        for (int u = 0; u < 3; u++) {
            double v = vk[u], x = xk[u];
            v = __dadd_rn(v, __ddiv_rn(__dmul_rn(f[u], a.dt), ma));
            x = __dadd_rn(x, __dmul_rn(__dmul_rn(v, a.dt), 0.5));
            v = __dadd_rn(__dmul_rn(v, a.c), __dmul_rn(xi[u], a.s));
            x = __dadd_rn(x, __dmul_rn(__dmul_rn(v, a.dt), 0.5));
            x = wrap1d(x, a.L);
            a.v[b + u] = v;
            a.x[b + u] = x;
            xn[u] = x;
        }
        static_cast<V4 *>(a.pos_out)[i] = mk4<V4>(xn[0], xn[1], xn[2]);
        a.pos64_out[i] = make_double4(xn[0], xn[1], xn[2], 0.0);
        return;
    }
    // reverse part 2 (diffusion.jl:1580-1586) and, fused, part 1 of the next step (1566-1572)
    const double dt2 = __dmul_rn(a.dt, a.dt);
    const bool fuse = (a.mode & MODE_FUSE_NEXT) != 0;
    double Bk[3], Ak[3], Dk[3] = {0.0, 0.0, 0.0}, Ck[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < 3; u++) {
        vk[u] = a.v[b + u];
        Bk[u] = a.B[b + u];
        Ak[u] = a.A[b + u];
        if (fuse) {
            xk[u] = a.x[b + u];
            Dk[u] = a.D[b + u];
            Ck[u] = a.C[b + u];
        }
    }
    double xi[3] = {0.0, 0.0, 0.0};
    if (fuse && a.s != 0.0) atom_noise(a.seed_next, (uint32_t)i, sd, xi);
    double xn[3], Cm[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const size_t e = b + u;
        a.G[e] = g[u];
        double v = __dsub_rn(vk[u], __ddiv_rn(__dmul_rn(f[u], a.dt), ma));
        const double B = __dadd_rn(__dmul_rn(a.c, Bk[u]), __dmul_rn(dt2, g[u]));
        a.B[e] = B;
        a.A[e] = __dadd_rn(Ak[u], B);
        if (fuse) {
            double x = xk[u];
            x = __dsub_rn(x, __dmul_rn(__dmul_rn(v, a.dt), 0.5));
            v = __ddiv_rn(__dsub_rn(v, __dmul_rn(xi[u], a.s)), a.c);
            x = __dsub_rn(x, __dmul_rn(__dmul_rn(v, a.dt), 0.5));
            x = wrap1d(x, a.L);
            const double D = __dadd_rn(__dmul_rn(a.c, Dk[u]),
                                       __ddiv_rn(__dmul_rn(__dmul_rn(dt2, g[u]), __dadd_rn(1.0, a.c)), 2.0));
            const double C = __dadd_rn(Ck[u], D);
            a.D[e] = D;
            a.C[e] = C;
            a.x[e] = x;
            xn[u] = x;
            Cm[u] = __ddiv_rn(C, ma);
        }
        a.v[e] = v;
    }
    if (fuse) {
        static_cast<V4 *>(a.pos_out)[i] = mk4<V4>(xn[0], xn[1], xn[2]);
        a.pos64_out[i] = make_double4(xn[0], xn[1], xn[2], 0.0);
        static_cast<V4 *>(a.wgt_out)[i] = mk4<V4>(Cm[0], Cm[1], Cm[2]);
    }
}

template <typename V4>
__global__ void k_gas_part1(const GasArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    const int ka = site_kind(i, a.nw3);
    const double ma = kind_mass(ka, a.mO, a.mH);
    const double dt2 = __dmul_rn(a.dt, a.dt);
    double xi[3] = {0.0, 0.0, 0.0};
    if (a.s != 0.0) atom_noise(a.seed_next, (uint32_t)i, ka == 1 ? a.sdH : a.sdO, xi);
    double xn[3], Cm[3];
    const size_t b = 3 * (size_t)i;
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const size_t e = b + u;
        double v = a.v[e], x = a.x[e];
        x = __dsub_rn(x, __dmul_rn(__dmul_rn(v, a.dt), 0.5));
        v = __ddiv_rn(__dsub_rn(v, __dmul_rn(xi[u], a.s)), a.c);
        x = __dsub_rn(x, __dmul_rn(__dmul_rn(v, a.dt), 0.5));
        x = wrap1d(x, a.L);
        const double D = __dadd_rn(__dmul_rn(a.c, a.D[e]),
                                   __ddiv_rn(__dmul_rn(__dmul_rn(dt2, a.G[e]), __dadd_rn(1.0, a.c)), 2.0));
        const double C = __dadd_rn(a.C[e], D);
        a.D[e] = D;
        a.C[e] = C;
        a.x[e] = x;
        a.v[e] = v;
        xn[u] = x;
        Cm[u] = __ddiv_rn(C, ma);
    }
    static_cast<V4 *>(a.pos_out)[i] = mk4<V4>(xn[0], xn[1], xn[2]);
    a.pos64_out[i] = make_double4(xn[0], xn[1], xn[2], 0.0);
    static_cast<V4 *>(a.wgt_out)[i] = mk4<V4>(Cm[0], Cm[1], Cm[2]);
}

template <typename V4>
__global__ void k_gas_pack(int N, const double *x, V4 *pos, double4 *pos64) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double4 p = ld3(x, i);
    pos[i] = mk4<V4>(p.x, p.y, p.z);
    pos64[i] = p;
}

template <typename V4>
__global__ void k_gas_pack_w(int N, int nw3, const double *w, double mO, double mH, V4 *wgt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double m = site_kind(i, nw3) == 1 ? mH : mO;
    const size_t b = 3 * (size_t)i;
    wgt[i] = mk4<V4>(__ddiv_rn(w[b], m), __ddiv_rn(w[b + 1], m), __ddiv_rn(w[b + 2], m));
}

__global__ void k_gas_reset(int n3, const double *g, double f1, double f2, double f3, double *A,
                            double *B, double *C, double *D, double *G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n3) return;
    const double ge = g[e];
    const double a = __dmul_rn(ge, f1);
    A[e] = a;
    B[e] = a;
    C[e] = 0.0;
    D[e] = __ddiv_rn(__dmul_rn(ge, f2), f3);
    G[e] = 0.0;
}

__global__ void k_gas_axpy(int n, double k, const double *x, double *y) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) y[e] = __fma_rn(k, x[e], y[e]);
}

// ------------------------------------------------------------------ energy
template <int FORM>
__global__ void __launch_bounds__(kThreads) k_gas_energy(const GasConsts k, const GasArgs a,
                                                         double *epart) {
    constexpr int NP = FormInfo<FORM>::NP;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (i >= a.N) return;
    const int ka = site_kind(i, a.nw3);
    const double4 pa = ld3(a.x, i);
    double E = 0.0, eq = 0.0;
    double acc[3][NP];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int q = 0; q < NP; q++) acc[c][q] = 0.0;
    const int n = a.cnt[i];
    const int *row = a.rows + (size_t)i * a.cap;
    for (int e = lane; e < n; e += 32) {
        const int j = row[e];
        if (j <= i) continue;
        const double4 pb = ld3(a.x, j);
        const double d0 = vec1d(pa.x, pb.x, a.L), d1 = vec1d(pa.y, pb.y, a.L), d2 = vec1d(pa.z, pb.z, a.L);
        const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
        if (!(r2 <= k.rc2)) continue;
        const double r = sqrt(r2);
        const int kb = site_kind(j, a.nw3);
        if (ka != 2 && kb != 2) {
            // Molly CoulombReactionField energy; dE/dq_O = 2 E_c / q_O
            const double Ec = k.qq[(ka == 1) + (kb == 1)] * (1.0 / r + k.krf * r2 - k.crf_shift);
            E += Ec;
            eq += Ec * k.twoinvq;
        }
        if (ka != 1 && kb != 1) {
            const int cls = (ka == 2) + (kb == 2);
            if (k.on[cls]) {
                const DualN<double, 4> Ef = form_energy<FORM>(cls == 0 ? k.fc[0].p : cls == 1 ? k.fc[1].p : k.fc[2].p, r);
                E += Ef.v;
#pragma unroll
                for (int c = 0; c < 3; c++)
                    if (c == cls)
#pragma unroll
                        for (int q = 0; q < NP; q++) acc[c][q] += Ef.d[q];
            }
        }
    }
    E = wsum(E);
    eq = wsum(eq);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int q = 0; q < NP; q++) acc[c][q] = wsum(acc[c][q]);
    if (lane != 0) return;
    // bonded terms on the molecule's first atom
    if (ka == 0) {
        double x[9];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const double4 p = ld3(a.x, i + q);
            x[3 * q] = p.x;
            x[3 * q + 1] = p.y;
            x[3 * q + 2] = p.z;
        }
        double dd[2][3];
        for (int h = 1; h <= 2; h++) {
            for (int u = 0; u < 3; u++) dd[h - 1][u] = vec1d(x[u], x[3 * h + u], a.L);
            const double bl = sqrt(dd[h - 1][0] * dd[h - 1][0] + dd[h - 1][1] * dd[h - 1][1] +
                                   dd[h - 1][2] * dd[h - 1][2]) - a.bw.r0;
            E += 0.5 * a.bw.kb * bl * bl;
        }
        const double *u1 = dd[0], *u2 = dd[1];
        const double cth = (u1[0] * u2[0] + u1[1] * u2[1] + u1[2] * u2[2]) /
                           (sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]) *
                            sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]));
        const double th = acos(cth) - a.bw.th0;
        E += 0.5 * a.bw.ka * th * th;
    } else if (ka == 2 && ((i - a.nw3) & 1) == 0) {
        const double4 pp = ld3(a.x, i + 1);
        const double d0 = vec1d(pa.x, pp.x, a.L), d1 = vec1d(pa.y, pp.y, a.L), d2 = vec1d(pa.z, pp.z, a.L);
        const double bl = sqrt(d0 * d0 + d1 * d1 + d2 * d2) - a.r0_g;
        E += 0.5 * a.kb_g * bl * bl;
    }
    double th[kMaxP];
#pragma unroll
    for (int p = 0; p < kMaxP; p++) th[p] = 0.0;
#pragma unroll
    for (int q = 0; q < NP; q++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            th[k.iw[q]] += k.fw[c][q] * acc[c][q];
            if (k.ig[q] >= 0) th[k.ig[q]] += k.fg[c][q] * acc[c][q];
        }
    th[k.iq] += eq;
    double *out = epart + (size_t)i * (k.P + 1);
    out[0] = E;
    for (int p = 0; p < k.P; p++) out[1 + p] = th[p];
}

// Single CTA: out[q] = scale * sum over atoms (strided per thread, then a fixed tree).
__global__ void __launch_bounds__(256) k_gas_esum(int N, int P, const double *epart, double e_scale,
                                                  double g_scale, int accumulate, double *out) {
    __shared__ double sh[256];
    for (int q = 0; q <= P; q++) {
        double s = 0.0;
        for (int a = threadIdx.x; a < N; a += 256) s += epart[(size_t)a * (P + 1) + q];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const double v = sh[0] * (q == 0 ? e_scale : g_scale);
            out[q] = accumulate ? out[q] + v : v;
        }
        __syncthreads();
    }
}

template <typename R, bool REV>
void step_form(int form, const GasConstsT<R> &k, const GasArgs &a, dim3 grid, cudaStream_t st) {
    switch (form) {
        case F_LJ: launch_chained(k_gas_step<R, F_LJ, REV>, grid, dim3(kThreads), 0, st, k, a); break;
        case F_DEXP: launch_chained(k_gas_step<R, F_DEXP, REV>, grid, dim3(kThreads), 0, st, k, a); break;
        case F_BUCK: launch_chained(k_gas_step<R, F_BUCK, REV>, grid, dim3(kThreads), 0, st, k, a); break;
        case F_LJSC: launch_chained(k_gas_step<R, F_LJSC, REV>, grid, dim3(kThreads), 0, st, k, a); break;
        case F_BUFF: launch_chained(k_gas_step<R, F_BUFF, REV>, grid, dim3(kThreads), 0, st, k, a); break;
    }
}

}  // namespace

void launch_gas_rows(const GasRowArgs &a, cudaStream_t st) {
    const int grid = (a.N + kWarpsPerCta - 1) / kWarpsPerCta;
    k_gas_rows<<<grid, kThreads, 0, st>>>(a);
}

void launch_gas_step(bool mixed, int form, bool rev, const GasConstsT<float> &kf,
                     const GasConstsT<double> &kd, const GasArgs &a, cudaStream_t st) {
    const dim3 grid((a.N + kWarpsPerCta - 1) / kWarpsPerCta);
    if (mixed) {
        if (rev)
            step_form<float, true>(form, kf, a, grid, st);
        else
            step_form<float, false>(form, kf, a, grid, st);
    } else {
        if (rev)
            step_form<double, true>(form, kd, a, grid, st);
        else
            step_form<double, false>(form, kd, a, grid, st);
    }
}

void launch_gas_part1(bool mixed, const GasArgs &a, cudaStream_t st) {
    if (mixed)
        k_gas_part1<float4><<<(a.N + 127) / 128, 128, 0, st>>>(a);
    else
        k_gas_part1<double4><<<(a.N + 127) / 128, 128, 0, st>>>(a);
}

void launch_gas_pack(bool mixed, int N, const double *x, void *pos, double4 *pos64, cudaStream_t st) {
    if (mixed)
        k_gas_pack<float4><<<(N + 127) / 128, 128, 0, st>>>(N, x, static_cast<float4 *>(pos), pos64);
    else
        k_gas_pack<double4><<<(N + 127) / 128, 128, 0, st>>>(N, x, static_cast<double4 *>(pos), pos64);
}

void launch_gas_pack_w(bool mixed, int N, int nw3, const double *w, double mO, double mH, void *wgt,
                       cudaStream_t st) {
    if (mixed)
        k_gas_pack_w<float4><<<(N + 127) / 128, 128, 0, st>>>(N, nw3, w, mO, mH, static_cast<float4 *>(wgt));
    else
        k_gas_pack_w<double4><<<(N + 127) / 128, 128, 0, st>>>(N, nw3, w, mO, mH, static_cast<double4 *>(wgt));
}

void launch_gas_reset(int n3, const double *g, double f1, double f2, double f3, double *A,
                      double *B, double *C, double *D, double *G, cudaStream_t st) {
    k_gas_reset<<<(n3 + 255) / 256, 256, 0, st>>>(n3, g, f1, f2, f3, A, B, C, D, G);
}

void launch_gas_axpy(int n, double k, const double *x, double *y, cudaStream_t st) {
    k_gas_axpy<<<(n + 255) / 256, 256, 0, st>>>(n, k, x, y);
}

void launch_gas_energy(int form, const GasConsts &k, const GasArgs &a, double *epart,
                       cudaStream_t st) {
    const dim3 grid((a.N + kWarpsPerCta - 1) / kWarpsPerCta);
    switch (form) {
        case F_LJ: k_gas_energy<F_LJ><<<grid, kThreads, 0, st>>>(k, a, epart); break;
        case F_DEXP: k_gas_energy<F_DEXP><<<grid, kThreads, 0, st>>>(k, a, epart); break;
        case F_BUCK: k_gas_energy<F_BUCK><<<grid, kThreads, 0, st>>>(k, a, epart); break;
        case F_LJSC: k_gas_energy<F_LJSC><<<grid, kThreads, 0, st>>>(k, a, epart); break;
        case F_BUFF: k_gas_energy<F_BUFF><<<grid, kThreads, 0, st>>>(k, a, epart); break;
    }
}

void launch_gas_esum(int N, int P, const double *epart, double e_scale, double g_scale,
                     bool accumulate, double *out, cudaStream_t st) {
    k_gas_esum<<<1, 256, 0, st>>>(N, P, epart, e_scale, g_scale, accumulate ? 1 : 0, out);
}

}  // namespace gs
