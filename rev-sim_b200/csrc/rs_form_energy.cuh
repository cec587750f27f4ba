// rs_form_energy.cuh -- pair-form potential energies on dual numbers whose tangents are
// the form's four per-pair parameters (used by the water and the gas-in-water energy
// kernels): Molly's LennardJones and LennardJonesSoftCore energies and the
// DoubleExponential, Buckingham and Buffered147 energies of water.jl:409-526 /
// diffusion.jl:486-581.
#pragma once

#include "rs_device.cuh"

namespace rs {

template <int K>
using DN = DualN<double, K>;

template <int K>
__device__ __forceinline__ DN<K> dexp_(const DN<K> &a) {
    DN<K> r;
    r.v = exp(a.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = r.v * a.d[k];
    return r;
}

template <int K>
__device__ __forceinline__ DN<K> pow6(const DN<K> &a) {
    const DN<K> a2 = a * a;
    return a2 * a2 * a2;
}

// Pair-form energy with tangents = form parameters p[0..3].
template <int FORM>
__device__ __forceinline__ DN<4> form_energy(const double *p, double r) {
    DN<4> P[4];
#pragma unroll
    for (int k = 0; k < 4; k++) P[k] = dn_var<double, 4>(p[k], k);
    const DN<4> one = dn_const<double, 4>(1.0), R = dn_const<double, 4>(r);
    constexpr double c216 = 1.122462048309373;
    if (FORM == F_LJ || FORM == F_LJ_MLP) {
        const DN<4> sr6 = pow6(P[0] / R);
        return dn_const<double, 4>(4.0) * P[1] * (sr6 * sr6 - sr6);
    } else if (FORM == F_DEXP) {
        const DN<4> rm = P[0] * dn_const<double, 4>(c216);
        const DN<4> k1 = P[3] * dexp_(P[2]) / (P[2] - P[3]), k2 = P[2] * dexp_(P[3]) / (P[2] - P[3]);
        const DN<4> x = R / rm;
        DN<4> na = P[2] * x, nb = P[3] * x;
        na.v = -na.v;
        nb.v = -nb.v;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            na.d[k] = -na.d[k];
            nb.d[k] = -nb.d[k];
        }
        return P[1] * (k1 * dexp_(na) - k2 * dexp_(nb));
    } else if (FORM == F_BUCK) {
        DN<4> e = P[1] * R;
        e.v = -e.v;
#pragma unroll
        for (int k = 0; k < 4; k++) e.d[k] = -e.d[k];
        const double r6 = r * r * r * r * r * r;
        return P[0] * dexp_(e) - P[2] / dn_const<double, 4>(r6);
    } else if (FORM == F_LJSC) {
        const double r6 = r * r * r * r * r * r;
        const DN<4> s6 = pow6(P[0]);
        const DN<4> six = s6 / (dn_const<double, 4>(r6) + s6 * P[2] * P[3] * P[3]);
        return dn_const<double, 4>(4.0) * P[1] * (six * six - six);
    } else {   // F_BUFF
        const DN<4> rm = P[0] * dn_const<double, 4>(c216);
        const DN<4> s = R / rm, b = (one + P[2]) / (s + P[2]);
        const DN<4> b7 = pow6(b) * b, s7 = pow6(s) * s;
        return P[1] * b7 * ((one + P[3]) / (s7 + P[3]) - dn_const<double, 4>(2.0));
    }
}

}  // namespace rs
