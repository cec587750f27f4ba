// rs_half_impl.cuh -- half-shell step kernels for the FP32 pair arithmetic (included by the
// per-pair-form instantiation files rs_half_*.cu).
//
// The fused step kernels (rs_step_impl.cuh) evaluate every unordered molecule pair twice,
// once from each side, so that each molecule's forces are summed by its own lanes with no
// atomics.  Here each pair is evaluated once, by its owner (half_owns, rs_internal.h):
//
//   k_water_half    the owner's lanes take the owned entries of its split row (rs_nlist.cu)
//                   in pairs, as the fused FP32 kernel does, and accumulate their own forces
//                   (and in reverse the VJP and the dtheta contraction) in registers; the
//                   partner's share of each entry -- the force with the opposite sign, and in
//                   reverse the VJP term with the opposite sign -- goes to the entry's slot;
//                   own partials and bonded terms go to a per-molecule record.
//   k_water_gather  the molecule's lanes sum the slots listed at the back of its split row,
//                   in row order, with a fixed butterfly, add the own partial and finish the
//                   atoms exactly as the fused kernel's epilogue does (atom_update).
//
// Pair terms are the fused kernel's (water.jl:892-913 forces, 1212-1433 VJP and dtheta): for
// the pair (a, b) the VJP of atom b is the negated VJP of atom a (the pair's second
// derivative block is symmetric and applied to w_a - w_b), and the two one-sided
// contractions -(dF/dtheta)(n . ca_a) and -(dF/dtheta)(-n . ca_b) sum to
// -(dF/dtheta) n . (ca_a - ca_b), which the owner takes once.  Forward and reverse kernels
// share the owned rows, the lane assignment, the arithmetic of the force terms and the
// gather order, so they give bit-identical forces (the reverse pass rebuilds the trajectory).
#pragma once

#include "rs_step_impl.cuh"

namespace rs {

namespace {

// One (own atom KA, partner atom KB) slot of two owned entries (halves x and y): as
// pair_term, with (cx, cy, cz) = ca_a - ca_b for the dtheta contraction, and the partner's
// share added to pf (forces) and pg (VJP).
template <int FORM, bool REV, int KA, int KB>
__device__ __forceinline__ void half_term(bool bitx, bool bity, float2 dx, float2 dy, float2 dz, float2 ex,
                                          float2 ey, float2 ez, float2 cx, float2 cy, float2 cz,
                                          const NbConsts<float> &nb, float2 f[3], float2 g[3], float2 *th,
                                          float2 pf[3], float2 pg[3], double *madj) {
    using R = float;
    using P = float2;
    constexpr int NF = FormInfo<FORM>::NP;
    constexpr int PF = FORM == F_LJ_MLP ? F_LJ : FORM;
    const P r2 = xfma(dz, dz, xfma(dy, dy, xmul(dx, dx)));
    const bool onx = bitx && r2.x <= nb.rc2;
    const bool ony = bity && r2.y <= nb.rc2;
    const P z = pk(onx ? R(1) : R(0), ony ? R(1) : R(0));
    const P r2s = pk(onx ? r2.x : R(1), ony ? r2.y : R(1));
    const P rinv = xrsqrt(r2s);
    const P r = xmul(r2s, rinv);
    const P invr2 = xmul(rinv, rinv);
    constexpr int QI = (KA > 0) + (KB > 0);
    const R qq = nb.qq[QI];
    const P Fc = xmul(pk1(qq), xsub(invr2, xmul(pk1(nb.krf2), r)));
    P F = Fc;
    P dF = pk1(R(0));
    P gf[4];
    if (REV) dF = xneg(xmul(pk1(xadd(qq, qq)), xadd(xmul(invr2, rinv), pk1(nb.krf))));
    if (KA == 0 && KB == 0) {
        if (nb.fc.on) {
            R Fx, Fy, dFx = R(0), dFy = R(0), gx[4], gy[4];
            pair_form<R, PF, REV>(nb.fc, r.x, rinv.x, invr2.x, Fx, dFx, gx);
            pair_form<R, PF, REV>(nb.fc, r.y, rinv.y, invr2.y, Fy, dFy, gy);
            F = xadd(F, pk(Fx, Fy));
            if (REV) {
                dF = xadd(dF, pk(dFx, dFy));
#pragma unroll
                for (int p = 0; p < NF; p++) gf[p] = pk(gx[p], gy[p]);
            }
        }
    }
    int gix = 0, giy = 0;
    R smx = R(0), smy = R(0);
    if constexpr (FORM == F_LJ_MLP) {
        R d1x, d1y, d2x, d2y;
        mlp_segment<R, REV>(nb, QI, r.x, gix, smx, d1x, d2x);
        mlp_segment<R, REV>(nb, QI, r.y, giy, smy, d1y, d2y);
        F = xsub(F, pk(d1x, d1y));
        if (REV) dF = xsub(dF, pk(d2x, d2y));
    }
    const P Fr = xmul(xmul(F, rinv), z);
    // own atom: -(F/r) d; partner: +(F/r) d
    const P mFr = xneg(Fr);
    f[0] = xfma(mFr, dx, f[0]);
    f[1] = xfma(mFr, dy, f[1]);
    f[2] = xfma(mFr, dz, f[2]);
    pf[0] = xfma(Fr, dx, pf[0]);
    pf[1] = xfma(Fr, dy, pf[1]);
    pf[2] = xfma(Fr, dz, pf[2]);
    if (REV) {
        // VJP of the own atom: -(k1 d + (F/r) e), e = w_b - w_a; the partner's is the negation
        const P s = xmul(rinv, xfma(dz, ez, xfma(dy, ey, xmul(dx, ex))));
        const P k1 = xmul(xmul(xsub(xmul(dF, z), Fr), s), rinv);
        const P t0 = xfma(k1, dx, xmul(Fr, ex));
        const P t1 = xfma(k1, dy, xmul(Fr, ey));
        const P t2 = xfma(k1, dz, xmul(Fr, ez));
        g[0] = xsub(g[0], t0);
        g[1] = xsub(g[1], t1);
        g[2] = xsub(g[2], t2);
        pg[0] = xadd(pg[0], t0);
        pg[1] = xadd(pg[1], t1);
        pg[2] = xadd(pg[2], t2);
        // dtheta: -(dF/dtheta_p) n . (ca_a - ca_b)
        const P na = xmul(xmul(rinv, xfma(dz, cz, xfma(dy, cy, xmul(dx, cx)))), z);
        th[NF] = xfma(xneg(xmul(Fc, pk1(nb.twoinvq))), na, th[NF]);
        if (KA == 0 && KB == 0) {
            if (nb.fc.on) {
#pragma unroll
                for (int p = 0; p < NF; p++) th[p] = xfma(xneg(gf[p]), na, th[p]);
            }
        }
        if constexpr (FORM == F_LJ_MLP) {
            if (onx) mlp_adjoint<R>(madj, QI, gix, na.x, smx, nb.mlp_hinv);
            if (ony) mlp_adjoint<R>(madj, QI, giy, na.y, smy, nb.mlp_hinv);
        }
    }
}

// Partner atom KB of two owned entries against the three own atoms.
template <int FORM, bool REV, int KB>
__device__ __forceinline__ void half_col(uint32_t mx, uint32_t my, const float4 pa[3], const float4 &pbx,
                                         const float4 &pby, const float4 wa[3], const float4 &wbx,
                                         const float4 &wby, const float ca[3][3], const float cbx[3],
                                         const float cby[3], const float2 sh[3], float L, float invL,
                                         const NbConsts<float> &nb, float2 f[3][3], float2 g[3][3], float2 *th,
                                         float2 pf[3], float2 pg[3], double *madj) {
    using P = float2;
#define RS_HSLOT(KA)                                                                                  \
    {                                                                                                 \
        P ex = pk1(0.f), ey = pk1(0.f), ez = pk1(0.f), cx = pk1(0.f), cy = pk1(0.f), cz = pk1(0.f);   \
        if (REV) {                                                                                    \
            ex = pk(xsub(wbx.x, wa[KA].x), xsub(wby.x, wa[KA].x));                                    \
            ey = pk(xsub(wbx.y, wa[KA].y), xsub(wby.y, wa[KA].y));                                    \
            ez = pk(xsub(wbx.z, wa[KA].z), xsub(wby.z, wa[KA].z));                                    \
            cx = pk(xsub(ca[KA][0], cbx[0]), xsub(ca[KA][0], cby[0]));                                \
            cy = pk(xsub(ca[KA][1], cbx[1]), xsub(ca[KA][1], cby[1]));                                \
            cz = pk(xsub(ca[KA][2], cbx[2]), xsub(ca[KA][2], cby[2]));                                \
        }                                                                                             \
        half_term<FORM, REV, KA, KB>((mx >> (3 * KA + KB)) & 1u, (my >> (3 * KA + KB)) & 1u,          \
                                     slot_d<float, true>(pa[KA].x, pbx.x, pby.x, sh[0], L, invL),     \
                                     slot_d<float, true>(pa[KA].y, pbx.y, pby.y, sh[1], L, invL),     \
                                     slot_d<float, true>(pa[KA].z, pbx.z, pby.z, sh[2], L, invL), ex, \
                                     ey, ez, cx, cy, cz, nb, f[KA], g[KA], th, pf, pg, madj);         \
    }
    RS_HSLOT(0);
    RS_HSLOT(1);
    RS_HSLOT(2);
#undef RS_HSLOT
}

template <int FORM, int G, bool REV>
__global__ void __maxnreg__((half_nreg(REV))) k_water_half(StepArgs a, NbConsts<float> nb,
                                                                          BondConsts bc) {
    using R = float;
    using V4 = float4;
    using P = float2;
    constexpr int NF = FormInfo<FORM>::NP;
    constexpr int NTH = NF + 1;
    // dynamic shared memory: [groups][P] dtheta (double), [groups] (unused here), then
    // [groups][22] bonded results (R): forces (9), VJP (9), dtheta (4)
    extern __shared__ double s_th[];
    chain_enter();

    const int grp = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int ngrp = blockDim.x / G;
    const int blk = blockIdx.x;
    const int rep = a.blk_rep[blk];
    const int I = a.blk_mol0[blk] + grp;
    const bool active = grp < a.blk_nmol[blk];
    const double Ld = a.rep_box[rep];
    const R L = (R)Ld;
    const R invL = (R)(1.0 / Ld);
    const V4 *__restrict__ pos = (const V4 *)a.pos_in;
    const V4 *__restrict__ wgt = (const V4 *)a.wgt_in;
    double *madj = FORM == F_LJ_MLP && REV
                       ? nb.mlp_adj + ((size_t)rep * MLP_NCOPY + (blk % MLP_NCOPY)) * MLP_NT * MLP_NG * 4
                       : nullptr;

    P f2[3][3], g2[3][3], th2[NTH];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) {
            f2[k][u] = pk1(R(0));
            g2[k][u] = pk1(R(0));
        }
#pragma unroll
    for (int p = 0; p < NTH; p++) th2[p] = pk1(R(0));

    V4 pa[3], wa[3];
    R ca[3][3];
    R *s_bond = (R *)(s_th + ngrp * (a.P + 1)) + 22 * grp;
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
        const uint32_t *__restrict__ row = a.split + (size_t)I * a.cap;
        const int cnt = a.cnt_own[I];
        const R hL = xmul(L, R(0.5));
        V4 *__restrict__ sf = a.slot_f + (size_t)I * a.cap * 3;
        float2 *__restrict__ sg = a.slot_g + (size_t)I * a.cap * 3;
        // owned entries e and e + G as one pair (halves x and y); a lane takes the pairs
        // starting at lane, lane + 2G, ...; a missing second entry is molecule 0 with an
        // empty mask (exact zeros) and writes no slot
        for (int e = lane; e < cnt; e += 2 * G) {
            const int e2 = e + G;
            const uint32_t ex = __ldg(row + e);
            const uint32_t ey = e2 < cnt ? __ldg(row + e2) : 0u;
            const int Jx = (int)(ex & 0x7FFFFFu), Jy = (int)(ey & 0x7FFFFFu);
            // the partner atoms' coordinates, weights and coefficients are loaded per partner
            // atom (RS_HCOL), the O coordinates first for the image shift
            const V4 pox = pos[3 * Jx], poy = pos[3 * Jy];
            // cell-origin differences (exact; gather_f32) plus the image shift from the O-O vector
            const R ox[3] = {xsub(pox.w, pa[0].w), xsub(pos[3 * Jx + 1].w, pa[1].w), xsub(pos[3 * Jx + 2].w, pa[2].w)};
            const R oy[3] = {xsub(poy.w, pa[0].w), xsub(pos[3 * Jy + 1].w, pa[1].w), xsub(pos[3 * Jy + 2].w, pa[2].w)};
            const P sh[3] = {pk(xadd(ox[0], image_shift(xadd(xsub(pox.x, pa[0].x), ox[0]), L, hL)),
                                xadd(oy[0], image_shift(xadd(xsub(poy.x, pa[0].x), oy[0]), L, hL))),
                             pk(xadd(ox[1], image_shift(xadd(xsub(pox.y, pa[0].y), ox[1]), L, hL)),
                                xadd(oy[1], image_shift(xadd(xsub(poy.y, pa[0].y), oy[1]), L, hL))),
                             pk(xadd(ox[2], image_shift(xadd(xsub(pox.z, pa[0].z), ox[2]), L, hL)),
                                xadd(oy[2], image_shift(xadd(xsub(poy.z, pa[0].z), oy[2]), L, hL)))};
            const uint32_t mx = ex >> 23, my = ey >> 23;
#define RS_HCOL(KB)                                                                                    \
    {                                                                                                  \
        const V4 pbx = KB == 0 ? pox : pos[3 * Jx + KB], pby = KB == 0 ? poy : pos[3 * Jy + KB];       \
        V4 wbx = {}, wby = {};                                                                         \
        if (REV) {                                                                                     \
            wbx = wgt[3 * Jx + KB];                                                                    \
            wby = wgt[3 * Jy + KB];                                                                    \
        }                                                                                              \
        P pf[3] = {pk1(R(0)), pk1(R(0)), pk1(R(0))}, pg[3] = {pk1(R(0)), pk1(R(0)), pk1(R(0))};        \
        R cbx[3] = {R(0), R(0), R(0)}, cby[3] = {R(0), R(0), R(0)};                                    \
        if (REV) {                                                                                     \
            const double sc = KB == 0 ? a.acoefO : a.acoefH;                                           \
            _Pragma("unroll") for (int u = 0; u < 3; u++) {                                            \
                cbx[u] = (R)__dmul_rn(a.A[9 * (size_t)Jx + 3 * KB + u], sc);                           \
                cby[u] = (R)__dmul_rn(a.A[9 * (size_t)Jy + 3 * KB + u], sc);                           \
            }                                                                                          \
        }                                                                                              \
        half_col<FORM, REV, KB>(mx, my, pa, pbx, pby, wa, wbx, wby, ca, cbx, cby, sh, L,                \
                                invL, nb, f2, g2, th2, pf, pg, madj);                                  \
        sf[3 * e + KB] = make_float4(pf[0].x, pf[1].x, pf[2].x, REV ? pg[0].x : R(0));                 \
        if (REV) sg[3 * e + KB] = make_float2(pg[1].x, pg[2].x);                                       \
        if (e2 < cnt) {                                                                                \
            sf[3 * e2 + KB] = make_float4(pf[0].y, pf[1].y, pf[2].y, REV ? pg[0].y : R(0));            \
            if (REV) sg[3 * e2 + KB] = make_float2(pg[1].y, pg[2].y);                                  \
        }                                                                                              \
    }
            RS_HCOL(0);
            RS_HCOL(1);
            RS_HCOL(2);
#undef RS_HCOL
        }
    }

    R f[3][3], g[3][3], th[NTH];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) {
            f[k][u] = group_sum<G>(xadd(f2[k][u].x, f2[k][u].y));
            g[k][u] = REV ? group_sum<G>(xadd(g2[k][u].x, g2[k][u].y)) : R(0);
        }
#pragma unroll
    for (int p = 0; p < NTH; p++) th[p] = REV ? group_sum<G>(xadd(th2[p].x, th2[p].y)) : R(0);
    __syncwarp();

    // own partial of atom `lane` (lanes 0..2): pair forces, pair VJP, bonded forces, bonded VJP
    if (active && lane < 3) {
        const int k = lane;
        float *o = a.own + (size_t)I * 36;
#pragma unroll
        for (int u = 0; u < 3; u++) {
            o[3 * k + u] = pick3(k, f[0][u], f[1][u], f[2][u]);
            o[18 + 3 * k + u] = s_bond[3 * k + u];
            if (REV) {
                o[9 + 3 * k + u] = pick3(k, g[0][u], g[1][u], g[2][u]);
                o[27 + 3 * k + u] = s_bond[9 + 3 * k + u];
            }
        }
    }

    if (REV) {
        // block reduction of the dtheta contributions (fixed order)
        const int P_ = a.P;
        double *sth = s_th;
        if (lane == 0) {
#pragma unroll
            for (int p = 0; p < NTH; p++) sth[grp * P_ + p] = active ? (double)th[p] : 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++) sth[grp * P_ + NF + 1 + q] = active ? (double)s_bond[18 + q] : 0.0;
        }
        __syncthreads();
        if (threadIdx.x < P_) {
            double s = 0.0;
            for (int q = 0; q < ngrp; q++) s = __dadd_rn(s, sth[q * P_ + threadIdx.x]);
            a.part[(size_t)blk * P_ + threadIdx.x] = __dadd_rn(a.part[(size_t)blk * P_ + threadIdx.x], s);
        }
    }
}

// Second kernel of a half-shell step: incoming slots, own partial, atom update.
template <int G, bool REV>
__global__ void __launch_bounds__(512) k_water_gather(StepArgs a) {
    using R = float;
    using V4 = float4;
    extern __shared__ double s_n2[];   // [groups] |dl_dfi|^2
    chain_enter();

    const int grp = threadIdx.x / G;
    const int lane = threadIdx.x % G;
    const int ngrp = blockDim.x / G;
    const int blk = blockIdx.x;
    const int rep = a.blk_rep[blk];
    const int I = a.blk_mol0[blk] + grp;
    const bool active = grp < a.blk_nmol[blk];
    const double Ld = a.rep_box[rep];

    R pf[3][3], pg[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) {
            pf[k][u] = R(0);
            pg[k][u] = R(0);
        }
    if (active) {
        const uint32_t *__restrict__ inc = a.split + (size_t)I * a.cap + (a.cap - 1);
        const int ci = a.cnt_inc[I];
        for (int q = lane; q < ci; q += G) {
            const size_t S = 3 * (size_t)__ldg(inc - q);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float4 v = a.slot_f[S + k];
                pf[k][0] = xadd(pf[k][0], v.x);
                pf[k][1] = xadd(pf[k][1], v.y);
                pf[k][2] = xadd(pf[k][2], v.z);
                if (REV) {
                    const float2 w = a.slot_g[S + k];
                    pg[k][0] = xadd(pg[k][0], v.w);
                    pg[k][1] = xadd(pg[k][1], w.x);
                    pg[k][2] = xadd(pg[k][2], w.y);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int u = 0; u < 3; u++) {
            pf[k][u] = group_sum<G>(pf[k][u]);
            if (REV) pg[k][u] = group_sum<G>(pg[k][u]);
        }
    __syncwarp();

    double n2 = 0.0;
    double xn[3] = {0.0, 0.0, 0.0};
    bool wpos = false;
    if (active && lane < 3) {
        const int k = lane;
        const float *o = a.own + (size_t)I * 36;
        double F[3], Gv[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int u = 0; u < 3; u++) {
            F[u] = __dadd_rn((double)xadd(o[3 * k + u], pick3(k, pf[0][u], pf[1][u], pf[2][u])),
                             (double)o[18 + 3 * k + u]);
            if (REV)
                Gv[u] = __dadd_rn((double)xadd(o[9 + 3 * k + u], pick3(k, pg[0][u], pg[1][u], pg[2][u])),
                                  (double)o[27 + 3 * k + u]);
        }
        atom_update<R, REV>(a, I, k, rep, Ld, F, Gv, n2, xn, wpos);
    }

    // gather buffer of the next step (as the fused kernel: H atoms next to their O)
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
        const double n2a = __shfl_sync(0xffffffffu, n2, (threadIdx.x & 31) - lane + 1);
        const double n2b = __shfl_sync(0xffffffffu, n2, (threadIdx.x & 31) - lane + 2);
        if (lane == 0) s_n2[grp] = active ? __dadd_rn(__dadd_rn(n2, n2a), n2b) : 0.0;
        __syncthreads();
        if (threadIdx.x == 0 && a.norm2) {
            double s = 0.0;
            for (int q = 0; q < ngrp; q++) s = __dadd_rn(s, s_n2[q]);
            a.norm2[blk] = s;
        }
    }
}

template <int FORM, int G>
cudaError_t launch_half_g(bool rev, int n_blk, int threads, const StepArgs &a, const NbConsts<float> &nb,
                          const BondConsts &bc, cudaStream_t st) {
    const int ngrp = threads / G;
    const size_t smem1 = sizeof(double) * (size_t)ngrp * (a.P + 1) + sizeof(float) * 22 * (size_t)ngrp;
    const size_t smem2 = sizeof(double) * (size_t)ngrp;
    cudaError_t e;
    if (rev) {
        e = launch_chained(k_water_half<FORM, G, true>, dim3(n_blk), dim3(threads), smem1, st, a, nb, bc);
        if (e != cudaSuccess) return e;
        return launch_chained(k_water_gather<G, true>, dim3(n_blk), dim3(threads), smem2, st, a);
    }
    e = launch_chained(k_water_half<FORM, G, false>, dim3(n_blk), dim3(threads), smem1, st, a, nb, bc);
    if (e != cudaSuccess) return e;
    return launch_chained(k_water_gather<G, false>, dim3(n_blk), dim3(threads), smem2, st, a);
}

}  // namespace

template <typename R, int FORM>
cudaError_t launch_half_form(bool rev, int G, int n_blk, int threads, const StepArgs &a, const NbConsts<R> &nb,
                             const BondConsts &bc, cudaStream_t st) {
    static_assert(sizeof(R) == 4, "half-shell kernels are FP32");
    switch (G) {
        case 8: return launch_half_g<FORM, 8>(rev, n_blk, threads, a, nb, bc, st);
        case 16: return launch_half_g<FORM, 16>(rev, n_blk, threads, a, nb, bc, st);
        case 32: return launch_half_g<FORM, 32>(rev, n_blk, threads, a, nb, bc, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace rs
