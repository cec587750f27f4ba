// rs_step_impl.cuh -- fused forward and reverse step kernels for flexible 3-site water
// (included by the per-precision, per-pair-form instantiation files rs_step_*.cu).
//
// Forward step (water.jl:1030-1037): calc_F! (non-bonded water.jl:892-913, bonds
// 915-934, angles 936-968) followed by the B-A-O-A update and the wrap.
// Reverse step (water.jl:1505-1521 and, fused, 1496-1502 of the next step):
// calc_F_and_grads! (water.jl:1212-1433) with the force VJP against
// dl_dfi_prev = accum_C, the contraction of dF/dtheta with A dt^2 / (2m)
// (water.jl:1517-1519, never materialised as a 3N x P matrix), the velocity
// un-kick, the B/A adjoint updates and the un-integration of the next step.
//
// Work decomposition: a group of G lanes owns one molecule; the lanes stride over
// the molecule's neighbour row (entries of 3 atoms each), accumulate the forces of
// the 3 own atoms in registers, and reduce them with a fixed xor butterfly.  Lanes
// 0..2 then finish one atom each (bonded terms in FP64, integrator in FP64).  Every
// atom's force is computed by exactly one group in a fixed order, so there are no
// atomics and the forward and reverse kernels produce bit-identical forces.
#pragma once

#include "rs_internal.h"
#include "rs_pack.cuh"

namespace rs {

namespace {

template <typename R>
__device__ __forceinline__ DualN<R, 1> d1(R v, R t) {
    DualN<R, 1> r;
    r.v = v;
    r.d[0] = t;
    return r;
}
template <typename R>
__device__ __forceinline__ DualN<R, 1> d1_sqrt(const DualN<R, 1> &a) {
    const R s = xsqrt(a.v);
    return d1(s, xdiv(a.d[0], xadd(s, s)));
}
__device__ __forceinline__ float r_acos(float c) { return acosf(c); }
__device__ __forceinline__ double r_acos(double c) { return acos(c); }
template <typename R>
__device__ __forceinline__ DualN<R, 1> d1_acos(const DualN<R, 1> &a) {
    return d1(r_acos(a.v), -xdiv(a.d[0], xsqrt(xsub(R(1), xmul(a.v, a.v)))));
}

// Harmonic angle H1-O-H2 (O central) of water.jl:936-968 / 1316-1356 on dual numbers:
// value = the reference's force construction (p1 = a x (a x b) / |.|, p3 = -b x (a x b) / |.|,
// F = k_a (theta0 - theta)), tangent along (w_H1 - w_O, w_H2 - w_O) = J w, which equals
// the reference's J^T w because the Hessian is symmetric.  Returns false when a x b = 0.
template <typename R>
__device__ __forceinline__ bool angle_term(const R a_[3], const R b_[3], const R ta[3],
                                           const R tb[3], R ka, R th0, DualN<R, 1> Fi[3],
                                           DualN<R, 1> Fk[3], R p1d[3], R p3d[3], R &disp) {
    using D = DualN<R, 1>;
    D a[3], b[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        a[u] = d1(a_[u], ta[u]);
        b[u] = d1(b_[u], tb[u]);
    }
    const D ra = d1_sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    const D rb = d1_sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    D cr[3], p1[3], p3[3];
    cr[0] = a[1] * b[2] - a[2] * b[1];
    cr[1] = a[2] * b[0] - a[0] * b[2];
    cr[2] = a[0] * b[1] - a[1] * b[0];
    if (cr[0].v == R(0) && cr[1].v == R(0) && cr[2].v == R(0)) return false;
    p1[0] = a[1] * cr[2] - a[2] * cr[1];
    p1[1] = a[2] * cr[0] - a[0] * cr[2];
    p1[2] = a[0] * cr[1] - a[1] * cr[0];
    const D zero = d1(R(0), R(0));
    p3[0] = zero - (b[1] * cr[2] - b[2] * cr[1]);
    p3[1] = zero - (b[2] * cr[0] - b[0] * cr[2]);
    p3[2] = zero - (b[0] * cr[1] - b[1] * cr[0]);
    const D n1 = d1_sqrt(p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2]);
    const D n3 = d1_sqrt(p3[0] * p3[0] + p3[1] * p3[1] + p3[2] * p3[2]);
    const D cth = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) / (ra * rb);
    const D th = d1_acos(cth);
    const D F = d1(ka, R(0)) * (d1(th0, R(0)) - th);
    const D s1 = n1 * ra, s3 = n3 * rb;
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const D q1 = p1[u] / s1;
        const D q3 = p3[u] / s3;
        Fi[u] = F * q1;
        Fk[u] = F * q3;
        p1d[u] = q1.v;
        p3d[u] = q3.v;
    }
    disp = xsub(th0, th.v);
    return true;
}

// Bonded terms of one molecule in pair precision R: forces Fb on (O, H1, H2); in
// reverse also the VJP Gb against w = C/m and the bonded dtheta contraction with
// acoef.  Intramolecular vectors and bond lengths come from the FP64 state (the
// displacement r - r0 is formed in FP64, so FP32 mode does not lose it to cancellation).
template <typename R, bool REV>
__device__ __forceinline__ void bonded(const double xm[9], double L, const BondConsts &bc,
                                       const R w[9], const R ac[9], R Fb[9], R Gb[9], R tb[4]) {
#pragma unroll
    for (int u = 0; u < 9; u++) {
        Fb[u] = R(0);
        Gb[u] = R(0);
    }
    tb[0] = tb[1] = tb[2] = tb[3] = R(0);
    const R kb = (R)bc.kb;
    R av[2][3];
    // Bonds (O, H1), (O, H2): radial pair with F(r) = -k_b (r - r0), F' = -k_b.
#pragma unroll
    for (int h = 1; h <= 2; h++) {
        double dd[3];
#pragma unroll
        for (int u = 0; u < 3; u++) dd[u] = vec1d(xm[u], xm[3 * h + u], L);
        const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dd[0], dd[0]), __dmul_rn(dd[1], dd[1])),
                                     __dmul_rn(dd[2], dd[2]));
        const double rd = __dsqrt_rn(r2d);
        const R disp = (R)__dsub_rn(rd, bc.r0);
        R dr[3];
#pragma unroll
        for (int u = 0; u < 3; u++) {
            dr[u] = (R)dd[u];
            av[h - 1][u] = dr[u];
        }
        const R rinv = xrsqrt((R)r2d);
        const R F = -xmul(kb, disp);
        const R Fr = xmul(F, rinv);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const R f = xmul(Fr, dr[u]);
            Fb[u] = xsub(Fb[u], f);
            Fb[3 * h + u] = xadd(Fb[3 * h + u], f);
        }
        if (REV) {
            // M delta with delta = w_H - w_O: -(F' - F/r) s n - (F/r) delta, s = n . delta
            R dl[3];
#pragma unroll
            for (int u = 0; u < 3; u++) dl[u] = xsub(w[3 * h + u], w[u]);
            const R s = xmul(rinv, xfma(dr[2], dl[2], xfma(dr[1], dl[1], xmul(dr[0], dl[0]))));
            const R k1 = xmul(xmul(xsub(-kb, Fr), s), rinv);
            R t = R(0);
#pragma unroll
            for (int u = 0; u < 3; u++) {
                const R m = -xfma(k1, dr[u], xmul(Fr, dl[u]));
                Gb[u] = xadd(Gb[u], m);
                Gb[3 * h + u] = xsub(Gb[3 * h + u], m);
                t = xfma(xsub(ac[u], ac[3 * h + u]), dr[u], t);
            }
            t = xmul(t, rinv);
            // dF_O/dk_b = disp n, dF_O/dr0 = -k_b n (water.jl:1298-1301)
            tb[0] = xfma(disp, t, tb[0]);
            tb[1] = xfma(-kb, t, tb[1]);
        }
    }
    // Angle H1-O-H2.
    R ta[3], tb3[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        ta[u] = REV ? xsub(w[3 + u], w[u]) : R(0);
        tb3[u] = REV ? xsub(w[6 + u], w[u]) : R(0);
    }
    DualN<R, 1> Fi[3], Fk[3];
    R p1d[3], p3d[3], disp;
    if (angle_term<R>(av[0], av[1], ta, tb3, (R)bc.ka, (R)bc.th0, Fi, Fk, p1d, p3d, disp)) {
        R t = R(0);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            Fb[3 + u] = xadd(Fb[3 + u], Fi[u].v);
            Fb[6 + u] = xadd(Fb[6 + u], Fk[u].v);
            Fb[u] = xsub(Fb[u], xadd(Fi[u].v, Fk[u].v));
            if (REV) {
                Gb[3 + u] = xadd(Gb[3 + u], Fi[u].d[0]);
                Gb[6 + u] = xadd(Gb[6 + u], Fk[u].d[0]);
                Gb[u] = xsub(Gb[u], xadd(Fi[u].d[0], Fk[u].d[0]));
                t = xadd(t, xsub(xfma(ac[3 + u], p1d[u], xmul(ac[6 + u], p3d[u])),
                                 xmul(ac[u], xadd(p1d[u], p3d[u]))));
            }
        }
        if (REV) {
            tb[2] = xmul(disp, t);           // dF/dk_a
            tb[3] = xmul((R)bc.ka, t);       // dF/dtheta0
        }
    }
}

template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <typename T>
__device__ __forceinline__ T pick3(int k, T a, T b, T c) {
    return k == 0 ? a : (k == 1 ? b : c);
}

__device__ __forceinline__ float r_rint(float v) { return rintf(v); }
__device__ __forceinline__ double r_rint(double v) { return rint(v); }

// Minimum-image component for the step kernels: d - L rint(d / L).  For every pair
// within the cutoff (|d| < L/2 - margin) it returns the same bits as Molly's rule
// (vec1d), one rounding of (c2 - c1) -/+ L; it differs only for pairs near L/2,
// which are far outside the cutoff.  Branch-free, unlike vec1d.
template <typename R>
__device__ __forceinline__ R vec_mi(R c1, R c2, R L, R invL) {
    const R d = xsub(c2, c1);
    return xfma(-r_rint(xmul(d, invL)), L, d);
}

// The learned pair correction's cubic segment at distance r of type QI (O-O, O-H, H-H):
// interval gi, offset sm in it, F contribution -d1 = -u'(r) = -(c1 + 2 c2 s + 3 c3 s^2) / h and
// dF/dr contribution -d2 = -(2 c2 + 6 c3 s) / h^2.
template <typename R, bool REV>
__device__ __forceinline__ void mlp_segment(const NbConsts<R> &nb, int QI, R r, int &gi, R &sm, R &d1,
                                            R &d2) {
    using V4m = typename V4T<R>::T;
    const R q = xmul(r, nb.mlp_hinv);
    gi = min((int)q, MLP_NG - 1);
    sm = xsub(q, (R)gi);
    const V4m cf = reinterpret_cast<const V4m *>(nb.mlp_tab)[QI * MLP_NG + gi];
    d1 = xmul(xfma(sm, xfma(xmul(R(3), sm), cf.w, xmul(R(2), cf.z)), cf.y), nb.mlp_hinv);
    d2 = R(0);
    if (REV) d2 = xmul(xmul(xfma(xmul(R(6), sm), cf.w, xmul(R(2), cf.z)), nb.mlp_hinv), nb.mlp_hinv);
}

// -(dF/dc_k) (n . acoef_a) for the interval's coefficients c1, c2, c3 (one in-cutoff pair).
template <typename R>
__device__ __forceinline__ void mlp_adjoint(double *madj, int QI, int gi, R na, R sm, R hinv) {
    const double v = (double)na * (double)hinv, s1 = (double)sm;
    double *adj = madj + ((size_t)QI * MLP_NG + gi) * 4;
    atomicAdd(adj + 1, v);
    atomicAdd(adj + 2, 2.0 * s1 * v);
    atomicAdd(adj + 3, 3.0 * s1 * s1 * v);
}

// The reverse kernels' charge contraction sum_slots (2 / q_O) (-A_c) (d . a) equals, per own
// atom, (2 / q_O) a . (F - F_form): the Coulomb share of the atom's pair force, known once the
// row is done.  So the slots only accumulate the O-O form's share F_form (one slot in nine), and
// the contraction is formed after the row -- except with the learned term, whose share is on
// every slot and which needs n . a per slot anyway.
__host__ __device__ constexpr bool charge_from_forces(int form) { return form != F_LJ_MLP; }

// The O-O Lennard-Jones form of pair_form on both halves of a register pair at once (the
// packed instructions round each half as the scalar ones do, so the halves carry the bits of
// pair_form<R, F_LJ>).  c[0] = sigma^2, c[1] = 24 eps, c[2] = 144 eps / sigma, c[3] = 1/eps.
template <typename R, bool GRAD>
__device__ __forceinline__ void lj_form2(const FormConsts<R> &fc, typename PkT<R>::T rinv,
                                         typename PkT<R>::T invr2, typename PkT<R>::T &F,
                                         typename PkT<R>::T &dF, typename PkT<R>::T g[2]) {
    using P = typename PkT<R>::T;
    P six = xmul(pk1(fc.c[0]), invr2);
    six = xmul(xmul(six, six), six);
    const P twelve = xmul(six, six);
    F = xmul(xmul(pk1(fc.c[1]), rinv), xsub(xadd(twelve, twelve), six));
    if (GRAD) {
        dF = xneg(xmul(xmul(pk1(fc.c[1]), invr2), xsub(xmul(pk1(R(26)), twelve), xmul(pk1(R(7)), six))));
        g[0] = xmul(xmul(pk1(fc.c[2]), rinv), xsub(xmul(pk1(R(4)), twelve), six));
        g[1] = xmul(F, pk1(fc.c[3]));
    }
}

// Two-entry form (FP32 kernels).  One (own atom KA, neighbour atom KB) slot of two neighbour
// entries at once: the .x halves of the displacement (dx, dy, dz), of the VJP differences
// (ex, ey, ez) = w_b - w_a, of the accumulators and of every intermediate belong to entry
// "x", the .y halves to entry "y" (rs_pack.cuh).  Evaluated unconditionally: pairs outside the
// neighbour mask or the cutoff contribute exact zeros, so the nine slots of an entry pair run
// as straight-line code with no divergence between the lanes of a warp.
//
// The slot works with A = F/r and B = (dF/dr - F/r) / r^2 of the radial force F(r): the force
// on the own atom is -A d, the force Jacobian is M = -(B d d^T + A I), so the VJP adds
// -(B (d . e) d + A e), and the contraction of dF/dtheta with the adjoint a is
// -(dF/dtheta / r) (d . a).  For the reaction-field Coulomb term F = qq (1/r^2 - 2 k_rf r),
// A = qq (1/r^3 - 2 k_rf) and B = -3 qq / r^5 in closed form (no separate r, dF or 1/r
// scaling of the dot products); the O-O form and the learned term add their own A and B.
// The accumulators receive -A and -B times the vectors ("mA", "mB").
template <typename R, int FORM, bool REV, int KA, int KB>
__device__ __forceinline__ void pair_term(bool bitx, bool bity, typename PkT<R>::T dx,
                                          typename PkT<R>::T dy, typename PkT<R>::T dz,
                                          typename PkT<R>::T ex, typename PkT<R>::T ey,
                                          typename PkT<R>::T ez, const R ca[3],
                                          const NbConsts<R> &nb, typename PkT<R>::T f[3],
                                          typename PkT<R>::T g[3], typename PkT<R>::T *th,
                                          typename PkT<R>::T fnc[3], double *madj) {
    using P = typename PkT<R>::T;
    constexpr int NF = FormInfo<FORM>::NP;
    constexpr int PF = FORM == F_LJ_MLP ? F_LJ : FORM;   // the O-O pair form
    constexpr int QI = (KA > 0) + (KB > 0);
    constexpr bool OO = KA == 0 && KB == 0;
    constexpr bool CHG_F = charge_from_forces(FORM);
    const P r2 = xfma(dz, dz, xfma(dy, dy, xmul(dx, dx)));
    const bool onx = bitx && r2.x <= nb.rc2;
    const bool ony = bity && r2.y <= nb.rc2;
    const R qq = nb.qq[QI];
    // dead slots: 1/r of r = 1 (finite) and a zero charge product
    const P rinv = xrsqrt(pk(onx ? r2.x : R(1), ony ? r2.y : R(1)));
    const P qz = pk(onx ? qq : R(0), ony ? qq : R(0));
    const P invr2 = xmul(rinv, rinv);
    const P rinv3 = xmul(invr2, rinv);
    const P mAc = xmul(qz, xsub(pk1(nb.krf2), rinv3));   // -A of the Coulomb term
    P mA = mAc;
    P mB = pk1(R(0));
    if (REV) mB = xmul(xmul(qz, pk1(R(3))), xmul(rinv3, invr2));   // 3 qq / r^5 = -B
    P gf[4];
    if (OO || FORM == F_LJ_MLP) {
        const P z = pk(onx ? R(1) : R(0), ony ? R(1) : R(0));
        const P r = xmul(pk(onx ? r2.x : R(1), ony ? r2.y : R(1)), rinv);
        P Ff = pk1(R(0)), dFf = pk1(R(0));
        bool have = false;
        if (OO && nb.fc.on) {
            have = true;
            if constexpr (PF == F_LJ) {
                lj_form2<R, REV>(nb.fc, rinv, invr2, Ff, dFf, gf);
            } else {
                // the other O-O forms per half with the scalar code
                R Fx, Fy, dFx = R(0), dFy = R(0), gx[4], gy[4];
                pair_form<R, PF, REV>(nb.fc, r.x, rinv.x, invr2.x, Fx, dFx, gx);
                pair_form<R, PF, REV>(nb.fc, r.y, rinv.y, invr2.y, Fy, dFy, gy);
                Ff = pk(Fx, Fy);
                if (REV) {
                    dFf = pk(dFx, dFy);
#pragma unroll
                    for (int p = 0; p < NF; p++) gf[p] = pk(gx[p], gy[p]);
                }
            }
        }
        int gix = 0, giy = 0;
        R smx = R(0), smy = R(0);
        if constexpr (FORM == F_LJ_MLP) {
            // the learned correction: F -= u'(r), dF/dr -= u''(r)
            R d1x, d1y, d2x, d2y;
            mlp_segment<R, REV>(nb, QI, r.x, gix, smx, d1x, d2x);
            mlp_segment<R, REV>(nb, QI, r.y, giy, smy, d1y, d2y);
            Ff = xsub(Ff, pk(d1x, d1y));
            if (REV) dFf = xsub(dFf, pk(d2x, d2y));
            have = true;
        }
        if (have) {
            Ff = xmul(Ff, z);
            const P Af = xmul(Ff, rinv);
            mA = xsub(mA, Af);
            if (REV) mB = xfma(xsub(Af, xmul(dFf, z)), invr2, mB);
            if (REV && CHG_F) {
                // the O-O form's share of the own-atom force, so that the Coulomb share is
                // known after the row (charge_contraction)
                fnc[0] = xfma(Af, dx, fnc[0]);
                fnc[1] = xfma(Af, dy, fnc[1]);
                fnc[2] = xfma(Af, dz, fnc[2]);
            }
        }
        if (REV) {
            const P dca = xfma(dz, pk1(ca[2]), xfma(dy, pk1(ca[1]), xmul(dx, pk1(ca[0]))));
            const P na = xmul(xmul(rinv, dca), z);   // n . a
            if (OO && nb.fc.on) {
#pragma unroll
                for (int p = 0; p < NF; p++) th[p] = xfma(xneg(gf[p]), na, th[p]);
            }
            if constexpr (FORM == F_LJ_MLP) {
                if (onx) mlp_adjoint<R>(madj, QI, gix, na.x, smx, nb.mlp_hinv);
                if (ony) mlp_adjoint<R>(madj, QI, giy, na.y, smy, nb.mlp_hinv);
            }
            // charge, per slot when the learned term is on: acoef . dF/dq_O = (2 / q_O) (-A_c) (d . a)
            if (!CHG_F) th[NF] = xfma(xmul(mAc, pk1(nb.twoinvq)), dca, th[NF]);
        }
    }
    // force on the own atom: -A d
    f[0] = xfma(mA, dx, f[0]);
    f[1] = xfma(mA, dy, f[1]);
    f[2] = xfma(mA, dz, f[2]);
    if (REV) {
        // VJP: -(B (d . e) d + A e)
        const P mt = xmul(mB, xfma(dz, ez, xfma(dy, ey, xmul(dx, ex))));
        g[0] = xfma(mt, dx, xfma(mA, ex, g[0]));
        g[1] = xfma(mt, dy, xfma(mA, ey, g[1]));
        g[2] = xfma(mt, dz, xfma(mA, ez, g[2]));
    }
}

// Displacement of one slot for both entries (FP32 kernels): cx / cy = the neighbour atom's
// gather coordinate in entry x / y, c = the own atom's; formed per half (the two results land
// in one register pair) and packed from there on.  The gather coordinates are offsets from
// per-molecule cell origins (gather_f32) and s carries the entries' origin differences (exact
// multiples of 0.5 nm).  SHIFT: s also carries one periodic image per molecule pair (chosen
// from the O-O vector) for all nine atom pairs, the minimum one for every pair within the
// cutoff whenever L > 2 (cutoff + 2 * max O-H distance); s stays exact, so d + s is the one
// rounding of a vector within the cutoff.  Otherwise the image is chosen per slot from d + s
// and applied to s first (s - L rint((d + s) / L), exact), then added to d.
template <typename R, bool SHIFT>
__device__ __forceinline__ typename PkT<R>::T slot_d(R c, R cx, R cy, typename PkT<R>::T s, R L, R invL) {
    using P = typename PkT<R>::T;
    const P d = pk(xsub(cx, c), xsub(cy, c));
    if (SHIFT) return xadd(d, s);
    const P q = xmul(xadd(d, s), pk1(invL));
    return xadd(d, xfma(pk(-r_rint(q.x), -r_rint(q.y)), pk1(L), s));
}

template <typename R>
__device__ __forceinline__ R image_shift(R d, R L, R hL) {
    return d > hL ? -L : (d < -hL ? L : R(0));
}

// The three slots of own atom KA against the three atoms of the two neighbour molecules
// (entry x: pbx, wbx; entry y: pby, wby).
template <typename R, int FORM, bool REV, bool SHIFT, int KA>
__device__ __forceinline__ void pair_row(uint32_t maskx, uint32_t masky, const typename V4T<R>::T &pa,
                                         const typename V4T<R>::T pbx[3],
                                         const typename V4T<R>::T pby[3],
                                         const typename V4T<R>::T &wa,
                                         const typename V4T<R>::T wbx[3],
                                         const typename V4T<R>::T wby[3], const R ca[3],
                                         const typename PkT<R>::T sh[3], R L, R invL,
                                         const NbConsts<R> &nb, typename PkT<R>::T f[3],
                                         typename PkT<R>::T g[3], typename PkT<R>::T *th,
                                         typename PkT<R>::T fnc[3], double *madj) {
    using P = typename PkT<R>::T;
#define RS_SLOT(KB)                                                                               \
    {                                                                                             \
        P ex = pk1(R(0)), ey = pk1(R(0)), ez = pk1(R(0));                                         \
        if (REV) {                                                                                \
            ex = pk(xsub(wbx[KB].x, wa.x), xsub(wby[KB].x, wa.x));                                \
            ey = pk(xsub(wbx[KB].y, wa.y), xsub(wby[KB].y, wa.y));                                \
            ez = pk(xsub(wbx[KB].z, wa.z), xsub(wby[KB].z, wa.z));                                \
        }                                                                                         \
        pair_term<R, FORM, REV, KA, KB>((maskx >> (3 * KA + KB)) & 1u, (masky >> (3 * KA + KB)) & 1u, \
                                        slot_d<R, SHIFT>(pa.x, pbx[KB].x, pby[KB].x, sh[0], L, invL), \
                                        slot_d<R, SHIFT>(pa.y, pbx[KB].y, pby[KB].y, sh[1], L, invL), \
                                        slot_d<R, SHIFT>(pa.z, pbx[KB].z, pby[KB].z, sh[2], L, invL), \
                                        ex, ey, ez, ca, nb, f, g, th, fnc, madj);                 \
    }
    RS_SLOT(0);
    RS_SLOT(1);
    RS_SLOT(2);
#undef RS_SLOT
}

// Single-entry form of the slots, used by the FP64 kernels (no packed FP64 arithmetic, and
// two entries per lane would exceed their registers).
// One (own atom KA, neighbour atom KB) interaction with displacement (dx, dy, dz),
// evaluated unconditionally: pairs outside the neighbour mask or the cutoff
// contribute exact zeros, so the nine slots of an entry run as straight-line code with
// no divergence between the lanes of a warp (each lane holds a different neighbour).
// Same A / B formulation as the two-entry form.
template <typename R, int FORM, bool REV, int KA, int KB>
__device__ __forceinline__ void pair_term1(bool bit, R dx, R dy, R dz,
                                          const typename V4T<R>::T &wa,
                                          const typename V4T<R>::T &wb, const R ca[3],
                                          const NbConsts<R> &nb, R f[3], R g[3], R *th,
                                          R fnc[3], double *madj) {
    constexpr int NF = FormInfo<FORM>::NP;
    constexpr int PF = FORM == F_LJ_MLP ? F_LJ : FORM;   // the O-O pair form
    constexpr int QI = (KA > 0) + (KB > 0);
    constexpr bool OO = KA == 0 && KB == 0;
    constexpr bool CHG_F = charge_from_forces(FORM);
    const R r2 = xfma(dz, dz, xfma(dy, dy, xmul(dx, dx)));
    const bool on = bit && r2 <= nb.rc2;
    const R r2s = on ? r2 : R(1);
    const R rinv = xrsqrt(r2s);
    const R qz = on ? nb.qq[QI] : R(0);
    const R invr2 = xmul(rinv, rinv);
    const R rinv3 = xmul(invr2, rinv);
    const R mAc = xmul(qz, xsub(nb.krf2, rinv3));   // -A of the Coulomb term
    R mA = mAc;
    R mB = R(0);
    if (REV) mB = xmul(xmul(qz, R(3)), xmul(rinv3, invr2));   // 3 qq / r^5 = -B
    R dca = R(0);
    if (REV && (OO || !CHG_F)) dca = xfma(dz, ca[2], xfma(dy, ca[1], xmul(dx, ca[0])));
    if (OO || FORM == F_LJ_MLP) {
        const R z = on ? R(1) : R(0);
        const R r = xmul(r2s, rinv);
        R Ff = R(0), dFf = R(0), gf[4];
        bool have = false;
        if (OO && nb.fc.on) {
            have = true;
            pair_form<R, PF, REV>(nb.fc, r, rinv, invr2, Ff, dFf, gf);
        }
        // Learned pair correction: the cubic segment of interval gi of type QI (O-O, O-H,
        // H-H), F -= u'(r) = (c1 + 2 c2 s + 3 c3 s^2) / h, dF/dr -= (2 c2 + 6 c3 s) / h^2.
        int gi = 0;
        R sm = R(0);
        if constexpr (FORM == F_LJ_MLP) {
            using V4m = typename V4T<R>::T;
            const R q = xmul(r, nb.mlp_hinv);
            gi = min((int)q, MLP_NG - 1);
            sm = xsub(q, (R)gi);
            const V4m cf = reinterpret_cast<const V4m *>(nb.mlp_tab)[QI * MLP_NG + gi];
            const R d1 = xmul(xfma(sm, xfma(xmul(R(3), sm), cf.w, xmul(R(2), cf.z)), cf.y), nb.mlp_hinv);
            Ff = xsub(Ff, d1);
            if (REV) {
                const R d2 = xmul(xmul(xfma(xmul(R(6), sm), cf.w, xmul(R(2), cf.z)), nb.mlp_hinv), nb.mlp_hinv);
                dFf = xsub(dFf, d2);
            }
            have = true;
        }
        if (have) {
            Ff = xmul(Ff, z);
            const R Af = xmul(Ff, rinv);
            mA = xsub(mA, Af);
            if (REV) mB = xfma(xsub(Af, xmul(dFf, z)), invr2, mB);
            if (REV && CHG_F) {
                fnc[0] = xfma(Af, dx, fnc[0]);
                fnc[1] = xfma(Af, dy, fnc[1]);
                fnc[2] = xfma(Af, dz, fnc[2]);
            }
        }
        if (REV) {
            const R na = xmul(xmul(rinv, dca), z);   // n . a
            if (OO && nb.fc.on) {
#pragma unroll
                for (int p = 0; p < NF; p++) th[p] = xfma(-gf[p], na, th[p]);
            }
            if constexpr (FORM == F_LJ_MLP) {
                // -(dF/dc_k) (n . acoef_a) for the interval's coefficients c1, c2, c3
                if (on) {
                    const double v = (double)na * (double)nb.mlp_hinv, s1 = (double)sm;
                    double *adj = madj + ((size_t)QI * MLP_NG + gi) * 4;
                    atomicAdd(adj + 1, v);
                    atomicAdd(adj + 2, 2.0 * s1 * v);
                    atomicAdd(adj + 3, 3.0 * s1 * s1 * v);
                }
            }
        }
    }
    // force on the own atom: -A d
    f[0] = xfma(mA, dx, f[0]);
    f[1] = xfma(mA, dy, f[1]);
    f[2] = xfma(mA, dz, f[2]);
    if (REV) {
        // VJP: -(B (d . e) d + A e), e = w_b - w_a
        const R ex = xsub(wb.x, wa.x), ey = xsub(wb.y, wa.y), ez = xsub(wb.z, wa.z);
        const R mt = xmul(mB, xfma(dz, ez, xfma(dy, ey, xmul(dx, ex))));
        g[0] = xfma(mt, dx, xfma(mA, ex, g[0]));
        g[1] = xfma(mt, dy, xfma(mA, ey, g[1]));
        g[2] = xfma(mt, dz, xfma(mA, ez, g[2]));
        // charge, per slot when the learned term is on: acoef . dF/dq_O = (2 / q_O) (-A_c) (d . a)
        if (!CHG_F) th[NF] = xfma(xmul(mAc, nb.twoinvq), dca, th[NF]);
    }
}

// Displacement of one slot.  SHIFT: one periodic image per molecule pair (chosen from
// the O-O vector) is applied to all nine atom pairs; d + s rounds exactly as Molly's
// (c2 - c1) -/+ L, and the image is the minimum one for every pair within the cutoff
// whenever L > 2 (cutoff + 2 * max O-H distance).  Otherwise per-slot vec_mi.
template <typename R, bool SHIFT>
__device__ __forceinline__ R slot_d1(R ca_, R cb_, R s, R L, R invL) {
    if (SHIFT) return xadd(xsub(cb_, ca_), s);
    return vec_mi(ca_, cb_, L, invL);
}

template <typename R, bool SHIFT>
__device__ __forceinline__ R image_shift1(R d, R L, R hL) {
    return d > hL ? -L : (d < -hL ? L : R(0));
}

template <typename R, int FORM, bool REV, bool SHIFT, int KA>
__device__ __forceinline__ void pair_row1(uint32_t mask, const typename V4T<R>::T &pa,
                                         const typename V4T<R>::T pb[3],
                                         const typename V4T<R>::T &wa,
                                         const typename V4T<R>::T wb[3], const R ca[3],
                                         const R sh[3], R L, R invL, const NbConsts<R> &nb,
                                         R f[3], R g[3], R *th, R fnc[3], double *madj) {
#define RS_SLOT(KB)                                                                             \
    pair_term1<R, FORM, REV, KA, KB>((mask >> (3 * KA + KB)) & 1u,                               \
                                    slot_d1<R, SHIFT>(pa.x, pb[KB].x, sh[0], L, invL),           \
                                    slot_d1<R, SHIFT>(pa.y, pb[KB].y, sh[1], L, invL),           \
                                    slot_d1<R, SHIFT>(pa.z, pb[KB].z, sh[2], L, invL), wa, wb[KB], \
                                    ca, nb, f, g, th, fnc, madj)
    RS_SLOT(0);
    RS_SLOT(1);
    RS_SLOT(2);
#undef RS_SLOT
}

// The per-atom update of a step after the pair, bonded and reduction phases: forces F and
// VJP Gv of atom k of molecule I (FP64 sums), then forces-only output, the forward B-A-O-A
// update or the reverse un-kick with the adjoint updates and the next step's part 1.
// n2 receives |Gv|^2, xn the new FP64 position when wpos.
template <typename R, bool REV>
__device__ __forceinline__ void atom_update(const StepArgs &a, int I, int k, int rep, double Ld,
                                            const double F[3], const double Gv[3], double &n2,
                                            double xn[3], bool &wpos) {
    using V4 = typename V4T<R>::T;
    const size_t ia = 3 * (size_t)I + k;
    const double m = k == 0 ? a.mO : a.mH;
    // The exact integrator multiplies by dt / m and 1 / m (its increments are rounded to the
    // grid, and forward and reverse use the same expression); the reference's arithmetic
    // divides as water.jl does.
    const double dtm = k == 0 ? a.dtm_O : a.dtm_H, invm = k == 0 ? a.invm_O : a.invm_H;
    if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) atomicOr(a.status, ST_NAN);
    const double xk[3] = {a.x[3 * ia], a.x[3 * ia + 1], a.x[3 * ia + 2]};
    if (a.mode & MODE_FORCES_ONLY) {
#pragma unroll
        for (int u = 0; u < 3; u++) {
            a.F_out[3 * ia + u] = F[u];
            if (REV) a.G[3 * ia + u] = Gv[u];
        }
    } else if (!REV) {
        // B-A-O-A (water.jl:1032-1037)
        const uint32_t la = (uint32_t)(ia - a.rep_atom0[rep]);
        // every load before the first store: the state arrays are distinct, but the compiler
        // cannot know that, and would otherwise serialise the three components
        const double vk[3] = {a.v[3 * ia], a.v[3 * ia + 1], a.v[3 * ia + 2]};
        double xi[3] = {0.0, 0.0, 0.0};
        if (a.s != 0.0) {
            if (a.noise_cur) {
#pragma unroll
                for (int u = 0; u < 3; u++) xi[u] = a.noise_cur[3 * ia + u];
            } else {
                atom_noise(a.seed_cur[rep], la, k == 0 ? a.rep_sdO[rep] : a.rep_sdH[rep], xi);
            }
        }
        const bool ex = a.exact != 0;
#pragma unroll
        for (int u = 0; u < 3; u++) {
            double v = vk[u], x = xk[u];
            const double kick = ex ? __dmul_rn(F[u], dtm) : __ddiv_rn(__dmul_rn(F[u], a.dt), m);
            v = __dadd_rn(v, ex ? qgrid(kick) : kick);
            const double h1 = __dmul_rn(__dmul_rn(v, a.dt), 0.5);
            x = __dadd_rn(x, ex ? qgrid(h1) : h1);
            v = __dadd_rn(__dmul_rn(v, a.c), __dmul_rn(xi[u], a.s));
            if (ex) v = qgrid(v);
            const double h2 = __dmul_rn(__dmul_rn(v, a.dt), 0.5);
            x = __dadd_rn(x, ex ? qgrid(h2) : h2);
            x = ex ? wrap_exact(x, Ld) : wrap1d(x, Ld);
            a.v[3 * ia + u] = v;
            a.x[3 * ia + u] = x;
            xn[u] = x;
        }
        wpos = true;
    } else {
        const double dt2 = __dmul_rn(a.dt, a.dt);
        const bool fuse = (a.mode & MODE_FUSE_NEXT) != 0;
        const bool defer = (a.mode & MODE_DEFER_BA) != 0;
        // every load before the first store (as in the forward branch)
        double vk[3], Bk[3], Ak[3], Dk[3], Ck[3];
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const size_t e = 3 * ia + u;
            vk[u] = a.v[e];
            if (!defer) {
                Bk[u] = a.B[e];
                Ak[u] = a.A[e];
            }
            if (fuse) {
                Dk[u] = a.D[e];
                Ck[u] = a.C[e];
            }
        }
        double xi[3] = {0.0, 0.0, 0.0};
        if (fuse && a.s != 0.0) {
            if (a.noise_next) {
#pragma unroll
                for (int u = 0; u < 3; u++) xi[u] = a.noise_next[3 * ia + u];
            } else {
                const uint32_t la = (uint32_t)(ia - a.rep_atom0[rep]);
                atom_noise(a.seed_next[rep], la, k == 0 ? a.rep_sdO[rep] : a.rep_sdH[rep], xi);
            }
        }
        double Cm[3];
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const size_t e = 3 * ia + u;
            a.G[e] = Gv[u];
            n2 = __dadd_rn(n2, __dmul_rn(Gv[u], Gv[u]));
            // v_{n-1} = v' - F dt / m (water.jl:1516)
            const double kick = a.exact ? __dmul_rn(F[u], dtm) : __ddiv_rn(__dmul_rn(F[u], a.dt), m);
            double v = __dsub_rn(vk[u], a.exact ? qgrid(kick) : kick);
            if (!defer) {
                // water.jl:1520-1521
                const double B = __dadd_rn(__dmul_rn(a.c, Bk[u]), __dmul_rn(dt2, Gv[u]));
                a.B[e] = B;
                a.A[e] = __dadd_rn(Ak[u], B);
            }
            if (fuse) {
                // part 1 of the next reverse step (water.jl:1496-1502)
                double x = xk[u];
                const double h2 = __dmul_rn(__dmul_rn(v, a.dt), 0.5);
                x = __dsub_rn(x, a.exact ? qgrid(h2) : h2);
                v = __dsub_rn(v, __dmul_rn(xi[u], a.s));
                if (a.c != 1.0) v = __ddiv_rn(v, a.c);   // v / 1 is v: the same bits at gamma = 0
                if (a.exact) v = qgrid(v);
                const double h1 = __dmul_rn(__dmul_rn(v, a.dt), 0.5);
                x = __dsub_rn(x, a.exact ? qgrid(h1) : h1);
                x = a.exact ? wrap_exact(x, Ld) : wrap1d(x, Ld);
                // (dt^2 G (1 + c)) / 2, the halving as the (exact) product with 0.5
                const double D = __dadd_rn(__dmul_rn(a.c, Dk[u]),
                                           __dmul_rn(__dmul_rn(__dmul_rn(dt2, Gv[u]), __dadd_rn(1.0, a.c)), 0.5));
                const double C = __dadd_rn(Ck[u], D);
                a.D[e] = D;
                a.C[e] = C;
                a.x[e] = x;
                xn[u] = x;
                Cm[u] = a.exact ? __dmul_rn(C, invm) : __ddiv_rn(C, m);
            }
            a.v[e] = v;
        }
        if (fuse) {
            V4 wo;
            wo.x = (R)Cm[0];
            wo.y = (R)Cm[1];
            wo.z = (R)Cm[2];
            wo.w = R(0);
            ((V4 *)a.wgt_out)[ia] = wo;
            wpos = true;
        }
    }
}

// Register budget per thread: step_nreg (rs_internal.h).
template <typename R, bool REV, int U>
constexpr int step_maxnreg() {
    return step_nreg(sizeof(R) == 4, REV, U);
}

// U = 1: one neighbour entry (FP32: entry pair) per lane per iteration; 2: two, all loads
// issued first; 3: one, with the next one's indices and coordinates loaded while the
// current one is computed (software pipelining; launched with at most 256 threads).  Every
// form sums a lane's entries in the same order, so at one lane count they give the same bits.
template <typename R, int FORM, int G, bool REV, bool SHIFT, int U>
__global__ void __maxnreg__((step_maxnreg<R, REV, U>())) k_water_step(StepArgs a, NbConsts<R> nb,
                                                                      BondConsts bc) {
    using V4 = typename V4T<R>::T;
    constexpr int NF = FormInfo<FORM>::NP;
    constexpr int NTH = NF + 1;
    // dynamic shared memory: [groups][22] bonded results (R): forces (9), VJP (9), dtheta (4)
    extern __shared__ double s_dyn[];
    chain_enter();

    const int grp = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int blk = blockIdx.x;
    const int rep = a.blk_rep[blk];
    const int I = a.blk_mol0[blk] + grp;
    const bool active = grp < a.blk_nmol[blk];
    const double Ld = a.rep_box[rep];
    const R L = (R)Ld;
    const R invL = (R)(1.0 / Ld);
    const V4 *__restrict__ pos = (const V4 *)a.pos_in;
    const V4 *__restrict__ wgt = (const V4 *)a.wgt_in;
    // this replica's accumulator of the learned term's interval-coefficient adjoints
    double *madj = FORM == F_LJ_MLP && REV
                       ? nb.mlp_adj + ((size_t)rep * MLP_NCOPY + (blk % MLP_NCOPY)) * MLP_NT * MLP_NG * 4
                       : nullptr;

    // FP32: two entries per lane step in packed arithmetic (rs_pack.cuh), accumulated in
    // the halves of f2, g2, th2 and combined after the row loop; FP64: one entry per step
    // into f, g, th.
    constexpr bool PACKED = sizeof(R) == 4;
    using P = typename PkT<R>::T;
    P f2[3][3], g2[3][3], th2[NTH], fnc2[3];
    R f[3][3], g[3][3], th[NTH], fnc[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) {
            f2[k][u] = pk1(R(0));
            g2[k][u] = pk1(R(0));
            f[k][u] = R(0);
            g[k][u] = R(0);
        }
#pragma unroll
    for (int p = 0; p < NTH; p++) {
        th2[p] = pk1(R(0));
        th[p] = R(0);
    }
#pragma unroll
    for (int u = 0; u < 3; u++) {
        fnc2[u] = pk1(R(0));
        fnc[u] = R(0);
    }

    V4 pa[3], wa[3];
    R ca[3][3];
    // Bonded terms first, by lane 0 of each group into shared memory, so that their
    // latency overlaps the neighbour loops of the other lanes and warps.
    R *s_bond = (R *)s_dyn + 22 * grp;
    if (active) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            pa[k] = pos[3 * I + k];
            if (REV) {
                wa[k] = wgt[3 * I + k];
                const double sc = k == 0 ? a.acoefO : a.acoefH;
#pragma unroll
                for (int u = 0; u < 3; u++) ca[k][u] = (R)__dmul_rn(a.A[9 * (size_t)I + 3 * k + u], sc);
            }
        }
        const uint32_t *__restrict__ row = a.nbr + (size_t)I * a.cap;
        const int cnt = min(a.nbr_cnt[I], a.cap);
        // padding entries (past the row end) read molecule 0 with an empty mask
        auto ent_at = [&](int e) { return e < cnt ? __ldg(row + e) : 0u; };
        // the lane's first row entries, loaded before the bonded terms so that their latency
        // overlaps lane 0's bonded arithmetic (entries lane + q G, q < 4 covers every loop form)
        uint32_t first[4];
#pragma unroll
        for (int q = 0; q < 4; q++) first[q] = ent_at(lane + q * G);
        if (lane == 0) {
            double xm[9];
#pragma unroll
            for (int u = 0; u < 9; u++) xm[u] = a.x[9 * (size_t)I + u];
            R w[9], ac[9];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                w[3 * k] = REV ? wa[k].x : R(0);
                w[3 * k + 1] = REV ? wa[k].y : R(0);
                w[3 * k + 2] = REV ? wa[k].z : R(0);
#pragma unroll
                for (int u = 0; u < 3; u++) ac[3 * k + u] = REV ? ca[k][u] : R(0);
            }
            R Fb[9], Gb[9], tb[4];
            bonded<R, REV>(xm, Ld, bc, w, ac, Fb, Gb, tb);
#pragma unroll
            for (int u = 0; u < 9; u++) {
                s_bond[u] = Fb[u];
                s_bond[9 + u] = Gb[u];
            }
#pragma unroll
            for (int q = 0; q < 4; q++) s_bond[18 + q] = tb[q];
        }
        const R hL = xmul(L, R(0.5));
        auto fetch = [&](uint32_t ent, V4 pbq[3], V4 wbq[3]) {
            const int J = (int)(ent & 0x7FFFFFu);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                pbq[k] = pos[3 * J + k];
                if (REV) wbq[k] = wgt[3 * J + k];
            }
        };
        if constexpr (PACKED) {
            // Entries e and e + G of the row as one pair (halves x and y); a lane takes the
            // pairs starting at lane, lane + 2G, lane + 4G, ...
            auto entry2 = [&](uint32_t ex, uint32_t ey, const V4 pbx[3], const V4 wbx[3], const V4 pby[3],
                              const V4 wby[3]) {
                // the entries' cell origins relative to the own molecule's (exact multiples of
                // 0.5 nm, gather_f32) and, with SHIFT, the periodic image from the O-O vector:
                // s = origin difference + image shift, exact, added to each slot's offset difference
                R ox[3], oy[3];
#pragma unroll
                for (int u = 0; u < 3; u++) {
                    ox[u] = xsub(pbx[u].w, pa[u].w);
                    oy[u] = xsub(pby[u].w, pa[u].w);
                }
                P sh[3] = {pk(ox[0], oy[0]), pk(ox[1], oy[1]), pk(ox[2], oy[2])};
                if (SHIFT) {
                    sh[0] = pk(xadd(ox[0], image_shift(xadd(xsub(pbx[0].x, pa[0].x), ox[0]), L, hL)),
                               xadd(oy[0], image_shift(xadd(xsub(pby[0].x, pa[0].x), oy[0]), L, hL)));
                    sh[1] = pk(xadd(ox[1], image_shift(xadd(xsub(pbx[0].y, pa[0].y), ox[1]), L, hL)),
                               xadd(oy[1], image_shift(xadd(xsub(pby[0].y, pa[0].y), oy[1]), L, hL)));
                    sh[2] = pk(xadd(ox[2], image_shift(xadd(xsub(pbx[0].z, pa[0].z), ox[2]), L, hL)),
                               xadd(oy[2], image_shift(xadd(xsub(pby[0].z, pa[0].z), oy[2]), L, hL)));
                }
                const uint32_t mx = ex >> 23, my = ey >> 23;
                pair_row<R, FORM, REV, SHIFT, 0>(mx, my, pa[0], pbx, pby, wa[0], wbx, wby, ca[0], sh, L, invL, nb,
                                                 f2[0], g2[0], th2, fnc2, madj);
                pair_row<R, FORM, REV, SHIFT, 1>(mx, my, pa[1], pbx, pby, wa[1], wbx, wby, ca[1], sh, L, invL, nb,
                                                 f2[1], g2[1], th2, fnc2, madj);
                pair_row<R, FORM, REV, SHIFT, 2>(mx, my, pa[2], pbx, pby, wa[2], wbx, wby, ca[2], sh, L, invL, nb,
                                                 f2[2], g2[2], th2, fnc2, madj);
            };
            if (U == 3) {
                // one entry pair per iteration, the next pair's indices and coordinates
                // loaded while the current pair is computed
                uint32_t nx = first[0], ny = first[1];
                V4 pnx[3], wnx[3], pny[3], wny[3];
                fetch(nx, pnx, wnx);
                fetch(ny, pny, wny);
                for (int e = lane; e < cnt; e += 2 * G) {
                    const uint32_t ex = nx, ey = ny;
                    V4 pbx[3], wbx[3], pby[3], wby[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        pbx[k] = pnx[k];
                        pby[k] = pny[k];
                        if (REV) {
                            wbx[k] = wnx[k];
                            wby[k] = wny[k];
                        }
                    }
                    if (e + 2 * G < cnt) {
                        nx = ent_at(e + 2 * G);
                        ny = ent_at(e + 3 * G);
                        fetch(nx, pnx, wnx);
                        fetch(ny, pny, wny);
                    }
                    entry2(ex, ey, pbx, wbx, pby, wby);
                }
            } else {
                // U entry pairs per lane per iteration: all their loads are issued first, and
                // the row entries are loaded RS_ROW_AHEAD iterations ahead
                constexpr int UP = U == 3 ? 1 : U;
                constexpr int D = RS_ROW_AHEAD;
                constexpr int STEP = 2 * U * G;
                uint32_t nx[D][UP], ny[D][UP];
#pragma unroll
                for (int d = 0; d < D; d++)
#pragma unroll
                    for (int q = 0; q < UP; q++) {
                        nx[d][q] = d == 0 ? first[2 * q] : ent_at(lane + d * STEP + 2 * q * G);
                        ny[d][q] = d == 0 ? first[2 * q + 1] : ent_at(lane + d * STEP + (2 * q + 1) * G);
                    }
                for (int e0 = lane; e0 < cnt; e0 += STEP) {
                    uint32_t ex[UP], ey[UP];
#pragma unroll
                    for (int q = 0; q < UP; q++) {
                        ex[q] = nx[0][q];
                        ey[q] = ny[0][q];
#pragma unroll
                        for (int d = 0; d + 1 < D; d++) {
                            nx[d][q] = nx[d + 1][q];
                            ny[d][q] = ny[d + 1][q];
                        }
                        nx[D - 1][q] = ent_at(e0 + D * STEP + 2 * q * G);
                        ny[D - 1][q] = ent_at(e0 + D * STEP + (2 * q + 1) * G);
                    }
                    V4 pbx[UP][3], wbx[UP][3], pby[UP][3], wby[UP][3];
#pragma unroll
                    for (int q = 0; q < UP; q++) {
                        fetch(ex[q], pbx[q], wbx[q]);
                        fetch(ey[q], pby[q], wby[q]);
                    }
#pragma unroll
                    for (int q = 0; q < UP; q++) entry2(ex[q], ey[q], pbx[q], wbx[q], pby[q], wby[q]);
                }
            }
        } else {
            // one neighbour entry: displacement image and the nine slots
            auto entry = [&](uint32_t ent, const V4 pbq[3], const V4 wbq[3]) {
                const uint32_t mask = ent >> 23;
                R sh[3] = {R(0), R(0), R(0)};
                if (SHIFT) {
                    sh[0] = image_shift1<R, SHIFT>(xsub(pbq[0].x, pa[0].x), L, hL);
                    sh[1] = image_shift1<R, SHIFT>(xsub(pbq[0].y, pa[0].y), L, hL);
                    sh[2] = image_shift1<R, SHIFT>(xsub(pbq[0].z, pa[0].z), L, hL);
                }
                pair_row1<R, FORM, REV, SHIFT, 0>(mask, pa[0], pbq, wa[0], wbq, ca[0], sh, L, invL, nb, f[0],
                                                  g[0], th, fnc, madj);
                pair_row1<R, FORM, REV, SHIFT, 1>(mask, pa[1], pbq, wa[1], wbq, ca[1], sh, L, invL, nb, f[1],
                                                  g[1], th, fnc, madj);
                pair_row1<R, FORM, REV, SHIFT, 2>(mask, pa[2], pbq, wa[2], wbq, ca[2], sh, L, invL, nb, f[2],
                                                  g[2], th, fnc, madj);
            };
            if (U == 3) {
                uint32_t ent_n = first[0];
                V4 pbn[3], wbn[3];
                fetch(ent_n, pbn, wbn);
                for (int e = lane; e < cnt; e += G) {
                    const uint32_t ent = ent_n;
                    V4 pbq[3], wbq[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        pbq[k] = pbn[k];
                        if (REV) wbq[k] = wbn[k];
                    }
                    ent_n = ent_at(e + G);
                    if (e + G < cnt) fetch(ent_n, pbn, wbn);
                    entry(ent, pbq, wbq);
                }
            } else {
                // U entries per lane per iteration: all their loads are issued first, and the
                // next iteration's row entries are loaded one iteration ahead
                constexpr int UE = U == 3 ? 1 : U;
                uint32_t nxt[UE];
#pragma unroll
                for (int q = 0; q < UE; q++) nxt[q] = first[q];
                for (int e0 = lane; e0 < cnt; e0 += U * G) {
                    uint32_t ent[UE];
#pragma unroll
                    for (int q = 0; q < UE; q++) {
                        ent[q] = nxt[q];
                        nxt[q] = ent_at(e0 + U * G + q * G);
                    }
                    V4 pb[UE][3], wb[UE][3];
#pragma unroll
                    for (int q = 0; q < UE; q++) fetch(ent[q], pb[q], wb[q]);
#pragma unroll
                    for (int q = 0; q < UE; q++) entry(ent[q], pb[q], wb[q]);
                }
            }
        }
    }

    // The charge contraction from the forces (charge_from_forces), per lane on its partial
    // sums: (2 / q_O) sum_k a_k . (F_k - F_form,k), F_form only on the O atom.
    if constexpr (REV && charge_from_forces(FORM)) {
        if (active) {
            if constexpr (PACKED) {
                P q = pk1(R(0));
#pragma unroll
                for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int u = 0; u < 3; u++)
                        q = xfma(pk1(ca[k][u]), k == 0 ? xadd(f2[0][u], fnc2[u]) : f2[k][u], q);
                th2[NF] = xfma(pk1(nb.twoinvq), q, th2[NF]);
            } else {
                R q = R(0);
#pragma unroll
                for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int u = 0; u < 3; u++)
                        q = xfma(ca[k][u], k == 0 ? xadd(f[0][u], fnc[u]) : f[k][u], q);
                th[NF] = xfma(nb.twoinvq, q, th[NF]);
            }
        }
    }

    // FP32: the lane's two halves.  Then a fixed butterfly over the group: every lane ends
    // with the same totals.
    if constexpr (PACKED) {
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int u = 0; u < 3; u++) {
                f[k][u] = xadd(f2[k][u].x, f2[k][u].y);
                g[k][u] = xadd(g2[k][u].x, g2[k][u].y);
            }
#pragma unroll
        for (int p = 0; p < NTH; p++) th[p] = xadd(th2[p].x, th2[p].y);
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) {
            f[k][u] = group_sum<G>(f[k][u]);
            if (REV) g[k][u] = group_sum<G>(g[k][u]);
        }
    if (REV) {
#pragma unroll
        for (int p = 0; p < NTH; p++) th[p] = group_sum<G>(th[p]);
    }
    // Every read of the molecule's FP64 state (bonded terms above) precedes the
    // per-atom writes below, and lane 0's bonded results are visible to lanes 1, 2.
    __syncwarp();

    double n2 = 0.0;
    double xn[3] = {0.0, 0.0, 0.0};   // new FP64 position of the lane's atom
    bool wpos = false;
    if (active && lane < 3) {
        const int k = lane;
        double F[3], Gv[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int u = 0; u < 3; u++) {
            F[u] = __dadd_rn((double)pick3(k, f[0][u], f[1][u], f[2][u]), (double)s_bond[3 * k + u]);
            if (REV)
                Gv[u] = __dadd_rn((double)pick3(k, g[0][u], g[1][u], g[2][u]), (double)s_bond[9 + 3 * k + u]);
        }
        atom_update<R, REV>(a, I, k, rep, Ld, F, Gv, n2, xn, wpos);
    }

    // Gather buffer of the next step: H atoms are written next to their O (lane 0 of
    // the group), so that molecules are contiguous (gather_coord).
    {
        const int src = (threadIdx.x & 31) - lane;
        const double o0 = __shfl_sync(0xffffffffu, xn[0], src);
        const double o1 = __shfl_sync(0xffffffffu, xn[1], src);
        const double o2 = __shfl_sync(0xffffffffu, xn[2], src);
        if (wpos) {
            const bool is_h = lane != 0;
            V4 po;
            if constexpr (sizeof(R) == 4) {
                const double xo[3] = {o0, o1, o2};
                po = gather_f32(xo, xn, lane, Ld);   // offsets from the molecule's cell origin
            } else {
                po.x = (R)gather_coord(o0, xn[0], is_h, Ld);
                po.y = (R)gather_coord(o1, xn[1], is_h, Ld);
                po.z = (R)gather_coord(o2, xn[2], is_h, Ld);
                po.w = R(0);
            }
            ((V4 *)a.pos_out)[3 * (size_t)I + lane] = po;
        }
    }

    if (REV) {
        // This molecule's dtheta contributions and |dl_dfi|^2, into its own slots: one group
        // per molecule and step, so every slot sums its steps in step order.
        const int P = a.P;
        // lanes 0..2 hold per-atom |G|^2; fold them into lane 0's in order
        const double n2a = __shfl_sync(0xffffffffu, n2, (threadIdx.x & 31) - lane + 1);
        const double n2b = __shfl_sync(0xffffffffu, n2, (threadIdx.x & 31) - lane + 2);
        if (active && lane == 0) {
            double *pm = a.part + (size_t)I * P;
#pragma unroll
            for (int p = 0; p < NTH; p++) pm[p] = __dadd_rn(pm[p], (double)th[p]);
#pragma unroll
            for (int q = 0; q < 4; q++) pm[NF + 1 + q] = __dadd_rn(pm[NF + 1 + q], (double)s_bond[18 + q]);
            if (a.norm2) a.norm2[I] = __dadd_rn(__dadd_rn(n2, n2a), n2b);
        }
    }
}

// Launch of one (precision, pair form): dispatch on lanes per molecule, image mode
// and entries per iteration.
template <typename R, int FORM, int G, bool SHIFT, int U>
cudaError_t launch_one(bool rev, int n_blk, int threads, const StepArgs &a, const NbConsts<R> &nb,
                       const BondConsts &bc, cudaStream_t st) {
    const size_t smem = sizeof(R) * 22 * (size_t)(threads / G);
    if (rev)
        return launch_chained(k_water_step<R, FORM, G, true, SHIFT, U>, dim3(n_blk), dim3(threads), smem,
                              st, a, nb, bc);
    return launch_chained(k_water_step<R, FORM, G, false, SHIFT, U>, dim3(n_blk), dim3(threads), smem, st,
                          a, nb, bc);
}

template <typename R, int FORM, int G, bool SHIFT>
cudaError_t launch_u(bool rev, int unroll, int n_blk, int threads, const StepArgs &a,
                     const NbConsts<R> &nb, const BondConsts &bc, cudaStream_t st) {
    switch (unroll) {
        case 1: return launch_one<R, FORM, G, SHIFT, 1>(rev, n_blk, threads, a, nb, bc, st);
        case 2: return launch_one<R, FORM, G, SHIFT, 2>(rev, n_blk, threads, a, nb, bc, st);
        case 3:
            if (threads > 256) return cudaErrorInvalidValue;
            return launch_one<R, FORM, G, SHIFT, 3>(rev, n_blk, threads, a, nb, bc, st);
    }
    return cudaErrorInvalidValue;
}

template <typename R, int FORM, int G>
cudaError_t launch_g(bool rev, bool shift, int unroll, int n_blk, int threads, const StepArgs &a,
                     const NbConsts<R> &nb, const BondConsts &bc, cudaStream_t st) {
    if (shift) return launch_u<R, FORM, G, true>(rev, unroll, n_blk, threads, a, nb, bc, st);
    return launch_u<R, FORM, G, false>(rev, unroll, n_blk, threads, a, nb, bc, st);
}

}  // namespace

template <typename R, int FORM>
cudaError_t launch_form(bool rev, int G, int unroll, bool shift, int n_blk, int threads,
                        const StepArgs &a, const NbConsts<R> &nb, const BondConsts &bc,
                        cudaStream_t st) {
    switch (G) {
        case 8: return launch_g<R, FORM, 8>(rev, shift, unroll, n_blk, threads, a, nb, bc, st);
        case 16: return launch_g<R, FORM, 16>(rev, shift, unroll, n_blk, threads, a, nb, bc, st);
        case 32: return launch_g<R, FORM, 32>(rev, shift, unroll, n_blk, threads, a, nb, bc, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace rs
