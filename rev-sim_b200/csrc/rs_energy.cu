// rs_energy.cu -- potential energy and its parameter gradient at the current state: the
// per-snapshot dE/dtheta of the reweighting estimator (reweighting_sim, water.jl:1107-1210;
// the Zygote gradient of potential_energy at water.jl:1176-1183).  FP64, once per loss point.
//
// One thread per molecule I sums the molecule pairs (I, J > I) of its neighbour row (each
// unordered pair once; the row's 9-bit mask gives the listed atom pairs), the pair-form
// energy on dual numbers whose tangents are the form's parameters, the reaction-field
// Coulomb energy (dE/dq_O = 2 E_c / q_O), its own two bonds and angle, and -- with the
// learned term -- the interval-coefficient adjoints (1, s, s^2, s^3) of each pair's Hermite
// segment, which the MLP backpropagation turns into dE/dtheta_mlp.  Per-molecule partials
// [E, dE/dtheta...] are summed per replica on the host in molecule order, or -- for the
// enthalpy-of-vaporisation loss term (loss_enth_vap, water.jl:738-755) -- on the device by
// k_enth_finalize, which also turns U into the loss and its coefficient 2 e / n.
#include "rs_form_energy.cuh"
#include "rs_internal.h"

namespace rs {

namespace {

// EG_LANES lanes per molecule stride its row; the per-lane sums are combined by a fixed
// xor butterfly (deterministic), and lane 0 adds the bonded terms and writes the partials.
constexpr int EG_LANES = 16, EG_THREADS = 128;

template <int FORM, typename V4>
__global__ void __launch_bounds__(EG_THREADS) k_energy_grads(EnergyArgs a) {
    const int Ig = (blockIdx.x * blockDim.x + threadIdx.x) / EG_LANES;
    const int lane = threadIdx.x % EG_LANES;
    // every lane of the warp reaches the butterfly: molecules past the end run empty
    const bool live = Ig < a.M;
    const int I = live ? Ig : a.M - 1;
    constexpr int NFm = FormInfo<FORM>::NP;
    const int rep = a.mol_rep[I];
    const double L = a.rep_box[rep];
    const double *x = a.x;
    const int P = a.P;   // classical parameters
    double acc[1 + 16];
#pragma unroll
    for (int k = 0; k < 17; k++) acc[k] = 0.0;
    const bool gate = a.form_p[FORM == F_BUCK ? 0 : 1] != 0.0;
    const double aw = a.adj_scale ? a.adj_mul * a.adj_scale[rep] : 1.0;
    const double qq[3] = {a.qO * a.qO, a.qO * (-0.5 * a.qO), 0.25 * a.qO * a.qO};
    double *madj = a.mlp_adj ? a.mlp_adj + ((size_t)rep * MLP_NCOPY + (I % MLP_NCOPY)) * MLP_NT * MLP_NG * 4
                             : nullptr;
    const uint32_t *row = a.nbr + (size_t)I * a.cap;
    const int cnt = live ? min(a.nbr_cnt[I], a.cap) : 0;
    for (int e = lane; e < cnt; e += EG_LANES) {
        const uint32_t ent = row[e];
        const int J = (int)(ent & 0x7FFFFFu);
        if (J <= I) continue;
        const uint32_t mask = ent >> 23;
        for (int ka = 0; ka < 3; ka++)
            for (int kb = 0; kb < 3; kb++) {
                if (!((mask >> (3 * ka + kb)) & 1u)) continue;
                const double *xi = x + 3 * (size_t)(3 * I + ka), *xj = x + 3 * (size_t)(3 * J + kb);
                const double d0 = vec1d(xi[0], xj[0], L), d1 = vec1d(xi[1], xj[1], L), d2 = vec1d(xi[2], xj[2], L);
                const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
                if (!(r2 <= a.rc2)) continue;
                const double r = sqrt(r2);
                const int QI = (ka > 0) + (kb > 0);
                const double Ec = a.ke * qq[QI] * (1.0 / r + a.krf * r2 - a.crf_shift);
                acc[0] += Ec;
                acc[1 + NFm] += 2.0 * Ec / a.qO;
                if (ka == 0 && kb == 0 && gate) {
                    if (a.grads) {
                        const DN<4> Ef = form_energy<FORM>(a.form_p, r);
                        acc[0] += Ef.v;
#pragma unroll
                        for (int k = 0; k < NFm; k++) acc[1 + k] += Ef.d[k];
                    } else {
                        acc[0] += form_energy<FORM>(a.form_p, r).v;
                    }
                }
                if (FORM == F_LJ_MLP) {
                    const double q = r * a.mlp_hinv;
                    const int g = min((int)q, MLP_NG - 1);
                    const double s = q - g;
                    const V4 c = reinterpret_cast<const V4 *>(a.mlp_tab)[QI * MLP_NG + g];
                    acc[0] += (double)c.x + s * ((double)c.y + s * ((double)c.z + s * (double)c.w));
                    if (madj) {
                        double *ad = madj + ((size_t)QI * MLP_NG + g) * 4;
                        atomicAdd(ad, aw);
                        atomicAdd(ad + 1, aw * s);
                        atomicAdd(ad + 2, aw * s * s);
                        atomicAdd(ad + 3, aw * s * s * s);
                    }
                }
            }
    }
    // fixed butterfly over the molecule's lanes
    const unsigned wmask = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 17; k++) {
        if (k > P) break;
#pragma unroll
        for (int o = EG_LANES / 2; o > 0; o >>= 1) acc[k] = __dadd_rn(acc[k], __shfl_xor_sync(wmask, acc[k], o));
    }
    if (lane != 0 || !live) return;
    // bonds (O, H1), (O, H2) and the angle H1-O-H2 (water.jl:915-968 energies)
    const double *xo = x + 9 * (size_t)I;
    double b[2][3];
    for (int h = 0; h < 2; h++) {
        for (int u = 0; u < 3; u++) b[h][u] = vec1d(xo[u], xo[3 * (h + 1) + u], L);
        const double d = sqrt(b[h][0] * b[h][0] + b[h][1] * b[h][1] + b[h][2] * b[h][2]) - a.r0;
        acc[0] += 0.5 * a.kb * d * d;
        acc[1 + NFm + 1] += 0.5 * d * d;
        acc[1 + NFm + 2] += -a.kb * d;
    }
    const double c = (b[0][0] * b[1][0] + b[0][1] * b[1][1] + b[0][2] * b[1][2]) /
                     (sqrt(b[0][0] * b[0][0] + b[0][1] * b[0][1] + b[0][2] * b[0][2]) *
                      sqrt(b[1][0] * b[1][0] + b[1][1] * b[1][1] + b[1][2] * b[1][2]));
    const double th = acos(fmin(1.0, fmax(-1.0, c))) - a.th0;
    acc[0] += 0.5 * a.ka * th * th;
    acc[1 + NFm + 3] += 0.5 * th * th;
    acc[1 + NFm + 4] += -a.ka * th;
    for (int k = 0; k <= (a.grads ? P : 0); k++) a.part[(size_t)I * (P + 1) + k] = acc[k];
}

constexpr int kEnthThreads = 256;

__global__ void __launch_bounds__(kEnthThreads) k_enth_finalize(EnthArgs a) {
    __shared__ double red[kEnthThreads];
    __shared__ double kr;
    const int r = blockIdx.x, t = threadIdx.x;
    const int m0 = a.rep_atom0[r] / 3, n = a.rep_nmol[r];
    const int ncol = a.grads ? a.P + 1 : 1;
    for (int col = 0; col < ncol; col++) {
        double s = 0.0;
        for (int I = t; I < n; I += kEnthThreads) s += a.part[(size_t)(m0 + I) * (a.P + 1) + col];
        red[t] = s;
        __syncthreads();
        for (int w = kEnthThreads / 2; w > 0; w >>= 1) {
            if (t < w) red[t] += red[t + w];
            __syncthreads();
        }
        if (t == 0) {
            if (col == 0) {
                // enthalpy_vaporization and loss_enth_vap, water.jl:738-755
                const double e = a.u_gas - red[0] / n + a.rt - a.target;
                a.acc[r] += e * e;
                if (a.ev_acc) a.ev_acc[r] += e * e;
                kr = 2.0 * e / n;
                a.k[r] = kr;
            } else {
                a.dgrad[(size_t)r * a.P + col - 1] += -kr * red[0];
            }
        }
        __syncthreads();
    }
}

// Per replica: the sum of the energy column of the partials (fixed-order tree).
__global__ void __launch_bounds__(kEnthThreads) k_rep_energy(const int *rep_atom0, const int *rep_nmol,
                                                             const double *part, int P, double *E) {
    __shared__ double red[kEnthThreads];
    const int r = blockIdx.x, t = threadIdx.x;
    const int m0 = rep_atom0[r] / 3, n = rep_nmol[r];
    double s = 0.0;
    for (int I = t; I < n; I += kEnthThreads) s += part[(size_t)(m0 + I) * (P + 1)];
    red[t] = s;
    __syncthreads();
    for (int w = kEnthThreads / 2; w > 0; w >>= 1) {
        if (t < w) red[t] += red[t + w];
        __syncthreads();
    }
    if (t == 0) E[r] = red[0];
}

__global__ void k_enth_dldx(int n3, const int *atom_rep, const double *k, const double *F, double *dLdx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3) dLdx[i] += k[atom_rep[i / 3]] * F[i];
}

template <int FORM>
cudaError_t launch_f(int prec, const EnergyArgs &a, cudaStream_t st) {
    const int per = EG_THREADS / EG_LANES, b = (a.M + per - 1) / per;
    if (prec == 1)
        k_energy_grads<FORM, float4><<<b, EG_THREADS, 0, st>>>(a);
    else
        k_energy_grads<FORM, double4><<<b, EG_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_enth_finalize(const EnthArgs &a, cudaStream_t st) {
    if (a.R > 0) k_enth_finalize<<<a.R, kEnthThreads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_rep_energy(int R, const int *rep_atom0, const int *rep_nmol, const double *part, int P,
                              double *E, cudaStream_t st) {
    if (R > 0) k_rep_energy<<<R, kEnthThreads, 0, st>>>(rep_atom0, rep_nmol, part, P, E);
    return cudaGetLastError();
}

cudaError_t launch_enth_dldx(int N, const int *atom_rep, const double *k, const double *F, double *dLdx,
                             cudaStream_t st) {
    const int n3 = 3 * N, t = 256;
    if (n3 > 0) k_enth_dldx<<<(n3 + t - 1) / t, t, 0, st>>>(n3, atom_rep, k, F, dLdx);
    return cudaGetLastError();
}

cudaError_t launch_energy_grads(int form, int prec, const EnergyArgs &a, cudaStream_t st) {
    switch (form) {
        case F_LJ: return launch_f<F_LJ>(prec, a, st);
        case F_DEXP: return launch_f<F_DEXP>(prec, a, st);
        case F_BUCK: return launch_f<F_BUCK>(prec, a, st);
        case F_LJSC: return launch_f<F_LJSC>(prec, a, st);
        case F_BUFF: return launch_f<F_BUFF>(prec, a, st);
        case F_LJ_MLP: return launch_f<F_LJ_MLP>(prec, a, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace rs
