// rs_device.cuh -- device arithmetic shared by the water kernels (sm_100a).
//
// Reversibility needs the forward and reverse kernels to produce bit-identical
// forces for identical positions.  Every product, sum and fused multiply-add on
// the force path is therefore written with an explicit rounding intrinsic
// (__fmul_rn, __fadd_rn, __fmaf_rn, ...), which the compiler may neither contract
// nor reassociate, so the two kernels round identically whatever else they do.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace rs {

// Device status bits (OR-ed into one word; the host reads it after each call).
constexpr int ST_NLIST_OVERFLOW = 1;
constexpr int ST_NAN = 2;
constexpr int ST_GEOMETRY = 4;
constexpr int ST_CELL_OVERFLOW = 8;
constexpr int ST_ROW_ASYM = 64;   // half-shell split: a row member whose row lacks the owner

// ---------------------------------------------------------------- launch chaining
// Programmatic dependent launch of consecutive step kernels: a kernel launched with
// programmatic stream serialisation (launch_chained) waits here until the previous kernel in
// the stream has completed and its writes are visible, and then lets the next step kernel
// be scheduled, so that its CTAs become resident while this one runs and wait at the same
// point.  Called first, by every thread, before any read of device state or any write.
// Without the launch attribute both instructions return at once.
__device__ __forceinline__ void chain_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---------------------------------------------------------------- arithmetic
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float xsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float xexp(float a) { return expf(a); }
__device__ __forceinline__ double xexp(double a) { return exp(a); }

// 1/sqrt(r2): the MUFU reciprocal square root in FP32, IEEE sqrt + reciprocal in FP64.
__device__ __forceinline__ float xrsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ double xrsqrt(double a) { return __drcp_rn(__dsqrt_rn(a)); }

template <typename R> struct V4T;
template <> struct V4T<float> { using T = float4; };
template <> struct V4T<double> { using T = double4; };

// Molly vector_1D: c2 - c1 folded to the nearer periodic image (subtractions only,
// so the result is the same in every kernel and in the CPU restatement).
template <typename R>
__device__ __forceinline__ R vec1d(R c1, R c2, R L) {
    const R d = xsub(c2, c1);
    if (c1 < c2) return (d < xadd(xsub(c1, c2), L)) ? d : xsub(d, L);
    return (xsub(c1, c2) < xadd(d, L)) ? d : xadd(d, L);
}

// Molly wrap_coords: c - floor(c / L) * L, each operation rounded separately.
__device__ __forceinline__ double wrap1d(double c, double L) {
    return __dsub_rn(c, __dmul_rn(floor(__ddiv_rn(c, L)), L));
}

// Exactly reversible integration (revsim_set_integrator, REVSIM_INTEGRATOR_EXACT): positions,
// velocities and box sides are kept on the grid of multiples of 2^-48 (nm, nm/ps), and every
// increment of the velocity Verlet step (the kick F dt / m, each half drift v dt / 2) is
// rounded to that grid before it is added.  Sums of grid values below 2^5 in magnitude (box
// sides under 32 nm, speeds under 32 nm/ps) are exact in FP64, so the reverse pass, which subtracts the same increments computed from the
// same bits, restores the previous state exactly: with gamma = 0 the start state is rebuilt
// bit for bit however long the run (the reference's FP64 arithmetic rebuilds it to rounding
// that the dynamics' chaos amplifies).  With friction the O step v c + xi s is rounded to the
// grid too and its inverse is approximate, as in the reference.
constexpr double kGrid = 3.5527136788005009293556213378906e-15;   // 2^-48
constexpr double kGridInv = 281474976710656.0;                      // 2^48
constexpr double kGridMaxBox = 32.0;                                // 2^5 nm
__host__ __device__ __forceinline__ double qgrid(double y) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(rint(__dmul_rn(y, kGridInv)), kGrid);
#else
    return std::rint(y * kGridInv) * kGrid;
#endif
}

// Wrap into [0, L) exactly for grid values (c - k L, then one correction into the interval),
// so that the wrap of a reversed step undoes the forward wrap.
__device__ __forceinline__ double wrap_exact(double c, double L) {
    double w = __dsub_rn(c, __dmul_rn(floor(__ddiv_rn(c, L)), L));
    if (w < 0.0) w = __dadd_rn(w, L);
    else if (w >= L) w = __dsub_rn(w, L);
    return w;
}

// Coordinate written to the gather buffers read by the step kernels: an O as stored
// (wrapped into the box), an H as its O plus the minimum-image O->H vector, so that
// every molecule is contiguous in space and one periodic image per molecule pair
// serves all nine atom pairs.
__device__ __forceinline__ double gather_coord(double xo, double xa, bool is_h, double L) {
    return is_h ? __dadd_rn(xo, vec1d(xo, xa, L)) : xa;
}

// FP32 gather coordinates (the mixed-precision step kernels): each molecule's coordinates as
// FP32 offsets from an origin on a 0.5 nm grid (its O's cell), the origin's x, y, z in the
// w component of the molecule's O, H1, H2 entries.  An offset is at most ~0.6 nm, so it
// rounds to FP32 with an error of ~3e-8 nm where an absolute coordinate in a 4.5 nm box
// rounds with up to 2.4e-7 nm; two molecules' origins differ by an exact multiple of 0.5 nm.
// gather_origin: the grid point below the (wrapped) O coordinate xo, exactly.
__device__ __forceinline__ double gather_origin(double xo) { return __dmul_rn(floor(__dmul_rn(xo, 2.0)), 0.5); }

// Entry k (0: O, 1: H1, 2: H2) of a molecule whose O is at xo, the atom at xa.
__device__ __forceinline__ float4 gather_f32(const double xo[3], const double xa[3], int k, double L) {
    float4 r;
    const double o0 = gather_origin(xo[0]), o1 = gather_origin(xo[1]), o2 = gather_origin(xo[2]);
    r.x = (float)__dsub_rn(gather_coord(xo[0], xa[0], k != 0, L), o0);
    r.y = (float)__dsub_rn(gather_coord(xo[1], xa[1], k != 0, L), o1);
    r.z = (float)__dsub_rn(gather_coord(xo[2], xa[2], k != 0, L), o2);
    r.w = (float)(k == 0 ? o0 : (k == 1 ? o1 : o2));
    return r;
}

// ------------------------------------------------------------------ Philox
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11).
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__device__ __forceinline__ uint64_t bits53(uint32_t hi, uint32_t lo) {
    return (((uint64_t)hi << 21) ^ ((uint64_t)lo >> 11)) & ((1ull << 53) - 1);
}

// Two standard normals for (seed, atom, blk): u1 in (0,1], u2 in [0,1), Box-Muller.
__device__ __forceinline__ void normals2(uint64_t seed, uint32_t atom, uint32_t blk, double& z0,
                                         double& z1) {
    uint32_t c[4] = {atom, blk, 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = __dmul_rn((double)bits53(c[0], c[1]) + 1.0, 1.0 / 9007199254740992.0);
    const double u2 = __dmul_rn((double)bits53(c[2], c[3]), 1.0 / 9007199254740992.0);
    const double rr = sqrt(__dmul_rn(-2.0, log(u1)));
    const double ang = __dmul_rn(2.0 * 3.14159265358979323846, u2);
    double sn, cs;
    sincos(ang, &sn, &cs);
    z0 = __dmul_rn(rr, cs);
    z1 = __dmul_rn(rr, sn);
}

// Langevin noise of one atom: xi = sd * z, sd = sqrt(kB T / m) (Molly random_velocity_3D).
__device__ __forceinline__ void atom_noise(uint64_t seed, uint32_t atom, double sd, double xi[3]) {
    double z0, z1, z2, z3;
    normals2(seed, atom, 0u, z0, z1);
    normals2(seed, atom, 1u, z2, z3);
    xi[0] = __dmul_rn(z0, sd);
    xi[1] = __dmul_rn(z1, sd);
    xi[2] = __dmul_rn(z2, sd);
}

// -------------------------------------------------------------- pair forms
// Radial pair force F(r) (positive = repulsive), dF/dr and dF/dtheta_p for the
// O-O pair term (water.jl:160-407).  Only O carries the pair term in the water
// model, so the mixing rules reduce to the O parameters themselves.
enum Form { F_LJ = 0, F_DEXP = 1, F_BUCK = 2, F_LJSC = 3, F_BUFF = 4,
            F_LJ_MLP = 5 /* LJ plus the tabulated learned pair correction (rs_mlp.cu) */ };

template <int FORM> struct FormInfo;
template <> struct FormInfo<F_LJ> { static constexpr int NP = 2; };
template <> struct FormInfo<F_DEXP> { static constexpr int NP = 4; };
template <> struct FormInfo<F_BUCK> { static constexpr int NP = 3; };
template <> struct FormInfo<F_LJSC> { static constexpr int NP = 4; };
template <> struct FormInfo<F_BUFF> { static constexpr int NP = 4; };
template <> struct FormInfo<F_LJ_MLP> { static constexpr int NP = 2; };

// Precomputed per-launch constants of a pair form (host fills them from theta).
template <typename R>
struct FormConsts {
    R p[4];    // the form's own parameters
    R c[8];    // derived constants (see pair_form)
    int on;    // 0 when the iszero gate (eps or A == 0) switches the form off
};

// Multi-tangent dual number, used for the Buffered 14-7 derivatives.
template <typename R, int K>
struct DualN {
    R v;
    R d[K];
};

template <typename R, int K>
__device__ __forceinline__ DualN<R, K> dn_const(R v) {
    DualN<R, K> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = R(0);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ DualN<R, K> dn_var(R v, int k) {
    DualN<R, K> r = dn_const<R, K>(v);
    r.d[k] = R(1);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ DualN<R, K> operator+(const DualN<R, K>& a, const DualN<R, K>& b) {
    DualN<R, K> r;
    r.v = xadd(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xadd(a.d[k], b.d[k]);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ DualN<R, K> operator-(const DualN<R, K>& a, const DualN<R, K>& b) {
    DualN<R, K> r;
    r.v = xsub(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xsub(a.d[k], b.d[k]);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ DualN<R, K> operator*(const DualN<R, K>& a, const DualN<R, K>& b) {
    DualN<R, K> r;
    r.v = xmul(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xfma(a.d[k], b.v, xmul(a.v, b.d[k]));
    return r;
}
template <typename R, int K>
__device__ __forceinline__ DualN<R, K> operator/(const DualN<R, K>& a, const DualN<R, K>& b) {
    DualN<R, K> r;
    r.v = xdiv(a.v, b.v);
    const R ib = xdiv(R(1), b.v);
#pragma unroll
    for (int k = 0; k < K; k++) r.d[k] = xmul(xsub(a.d[k], xmul(r.v, b.d[k])), ib);
    return r;
}
template <typename R, int K>
__device__ __forceinline__ DualN<R, K> dn_pow7(const DualN<R, K>& a) {
    const DualN<R, K> a2 = a * a, a4 = a2 * a2;
    return a4 * a2 * a;
}

// Buffered 14-7 radial force (water.jl:336-351) on dual numbers.
template <typename T>
__device__ __forceinline__ T buff_force(const T& r, const T& sig, const T& eps, const T& del,
                                        const T& gam, const T& one, const T& two, const T& seven,
                                        const T& c216) {
    const T rm = sig * c216;
    const T s = r / rm;
    const T s2 = s * s, s3 = s2 * s, s6 = s3 * s3, s7 = s6 * s;
    const T g7 = (one + gam) / (s7 + gam);
    const T b7 = dn_pow7((one + del) / (s + del));
    return (seven * eps / rm) * b7 * ((one / (s + del)) * (g7 - two) + (one / (s7 + gam)) * s6 * g7);
}

// F, dF/dr and dF/dtheta of the O-O pair form.  `rinv`, `invr2` = 1/r, 1/r^2.
// Identical arithmetic for F whether or not GRAD is set.
template <typename R, int FORM, bool GRAD>
__device__ __forceinline__ void pair_form(const FormConsts<R>& fc, R r, R rinv, R invr2, R& F,
                                          R& dF, R* g) {
    if (FORM == F_LJ) {
        // c[0] = sigma^2, c[1] = 24 eps, c[2] = 144 eps / sigma, c[3] = 1/eps
        R six = xmul(fc.c[0], invr2);
        six = xmul(xmul(six, six), six);
        const R twelve = xmul(six, six);
        F = xmul(xmul(fc.c[1], rinv), xsub(xadd(twelve, twelve), six));
        if (GRAD) {
            dF = -xmul(xmul(fc.c[1], invr2), xsub(xmul(R(26), twelve), xmul(R(7), six)));
            g[0] = xmul(xmul(fc.c[2], rinv), xsub(xmul(R(4), twelve), six));
            g[1] = xmul(F, fc.c[3]);
        }
    } else if (FORM == F_BUCK) {
        // p = A, B, C; c[0] = A*B, c[1] = 6*C, c[2] = A*B*B, c[3] = 42*C
        const R e = xexp(-xmul(fc.p[1], r));
        const R invr7 = xmul(xmul(xmul(invr2, invr2), invr2), rinv);
        F = xsub(xmul(fc.c[0], e), xmul(fc.c[1], invr7));
        if (GRAD) {
            dF = xadd(-xmul(fc.c[2], e), xmul(xmul(fc.c[3], invr7), rinv));
            g[0] = xmul(fc.p[1], e);
            g[1] = xmul(xmul(fc.p[0], xsub(R(1), xmul(fc.p[1], r))), e);
            g[2] = xmul(R(-6), invr7);
        }
    } else if (FORM == F_DEXP) {
        // p = sigma, eps, alpha, beta; c[0] = 1/rm, c[1] = eps*alpha*beta, c[2] = 1/(alpha-beta),
        // c[3] = rm, c[4] = 2^(1/6)
        const R s = xmul(r, fc.c[0]);
        const R e1 = xmul(xexp(xmul(fc.p[2], xsub(R(1), s))), fc.c[2]);
        const R e2 = xmul(xexp(xmul(fc.p[3], xsub(R(1), s))), fc.c[2]);
        F = xmul(xmul(fc.c[1], xsub(e1, e2)), fc.c[0]);
        if (GRAD) {
            const R al = fc.p[2], be = fc.p[3], rm = fc.c[3], irm = fc.c[0];
            const R irm2 = xmul(irm, irm);
            dF = -xmul(xmul(fc.c[1], xsub(xmul(al, e1), xmul(be, e2))), irm2);
            const R dFdrm = xmul(xmul(fc.c[1], xsub(xmul(xsub(xmul(al, r), rm), e1),
                                                    xmul(xsub(xmul(be, r), rm), e2))),
                                 xmul(irm2, irm));
            g[0] = xmul(dFdrm, fc.c[4]);
            g[1] = xdiv(F, fc.p[1]);
            const R amb = xsub(al, be), rmr = xsub(r, rm);
            const R k = xmul(xmul(irm2, fc.c[2]), fc.p[1]);
            g[2] = -xmul(xmul(k, be), xsub(xmul(xadd(xmul(xmul(al, amb), rmr), xmul(be, rm)), e1),
                                           xmul(xmul(be, rm), e2)));
            // beta (beta - alpha) (r - rm) + alpha rm
            const R cb = xadd(xmul(xmul(be, -amb), rmr), xmul(al, rm));
            g[3] = xmul(xmul(k, al), xsub(xmul(xmul(al, rm), e1), xmul(cb, e2)));
        }
    } else if (FORM == F_LJSC) {
        // p = sigma, eps, alpha, lambda; with u = sigma^6 alpha lambda^2 and R = r^6 + u,
        // F = 24 eps r^5 (2 sigma^12 / R^3 - sigma^6 / R^2).
        // c[0] = sigma^6, c[1] = u, c[2] = 24 eps, c[3] = sigma^12, c[4] = 1/eps,
        // c[5] = 6 u / sigma, c[6] = u / alpha, c[7] = 2 u / lambda
        const R r2 = xmul(r, r), r4 = xmul(r2, r2), r5 = xmul(r4, r), r6 = xmul(r5, r);
        const R iR = xdiv(R(1), xadd(r6, fc.c[1]));
        const R iR2 = xmul(iR, iR), iR3 = xmul(iR2, iR);
        const R t = xsub(xmul(xadd(fc.c[3], fc.c[3]), iR3), xmul(fc.c[0], iR2));
        const R k = xmul(fc.c[2], r5);
        F = xmul(k, t);
        if (GRAD) {
            // dF/du = dF/dR = 24 eps r^5 (2 sigma^6 / R^3 - 6 sigma^12 / R^4)
            const R dFdu = xmul(k, xsub(xmul(xadd(fc.c[0], fc.c[0]), iR3),
                                        xmul(xmul(R(6), fc.c[3]), xmul(iR2, iR2))));
            dF = xadd(xmul(xmul(R(5), F), rinv), xmul(dFdu, xmul(R(6), r5)));
            // direct sigma dependence: 24 eps r^5 (24 sigma^11 / R^3 - 6 sigma^5 / R^2)
            const R isig = xdiv(R(1), fc.p[0]);
            const R dsig = xmul(k, xsub(xmul(xmul(R(24), xmul(fc.c[3], isig)), iR3),
                                        xmul(xmul(R(6), xmul(fc.c[0], isig)), iR2)));
            g[0] = xadd(dsig, xmul(dFdu, fc.c[5]));
            g[1] = xmul(F, fc.c[4]);
            g[2] = xmul(dFdu, fc.c[6]);
            g[3] = xmul(dFdu, fc.c[7]);
        }
    } else {  // F_BUFF
        if (!GRAD) {
            // The value arithmetic of DualN does not depend on the tangent count, so
            // this F is bit-identical to the GRAD path's res.v.
            using D1 = DualN<R, 1>;
            F = buff_force(dn_const<R, 1>(r), dn_const<R, 1>(fc.p[0]), dn_const<R, 1>(fc.p[1]),
                           dn_const<R, 1>(fc.p[2]), dn_const<R, 1>(fc.p[3]), dn_const<R, 1>(R(1)),
                           dn_const<R, 1>(R(2)), dn_const<R, 1>(R(7)), dn_const<R, 1>(fc.c[0]))
                    .v;
            (void)sizeof(D1);
        } else {
            using D5 = DualN<R, 5>;
            const D5 res = buff_force(dn_var<R, 5>(r, 0), dn_var<R, 5>(fc.p[0], 1),
                                      dn_var<R, 5>(fc.p[1], 2), dn_var<R, 5>(fc.p[2], 3),
                                      dn_var<R, 5>(fc.p[3], 4), dn_const<R, 5>(R(1)),
                                      dn_const<R, 5>(R(2)), dn_const<R, 5>(R(7)),
                                      dn_const<R, 5>(fc.c[0]));
            F = res.v;
            dF = res.d[0];
            g[0] = res.d[1];
            g[1] = res.d[2];
            g[2] = res.d[3];
            g[3] = res.d[4];
        }
    }
}

}  // namespace rs
