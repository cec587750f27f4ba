// rs_step.cu -- per-atom kernels of the integrator and adjoint (pack, un-integrate,
// clip, adjoint initialisation, noise) and the step-kernel dispatch.  The fused
// step kernels themselves are in rs_step_impl.cuh, instantiated per precision and pair
// form by rs_step_{f,d}_<form>.cu so that they compile in parallel.
#include "rs_internal.h"

namespace rs {

namespace {

// ---------------------------------------------------------------- per atom
__global__ void k_pack_f(int N, const double *x, const double *C, double mO, double mH,
                         const int *atom_rep, const double *rep_box, float4 *pos, float4 *wgt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const bool is_h = (i % 3) != 0;
    const double m = is_h ? mH : mO;
    const double L = rep_box[atom_rep[i]];
    const double *xo = x + 9 * (size_t)(i / 3);
    pos[i] = gather_f32(xo, x + 3 * (size_t)i, i % 3, L);
    if (C)
        wgt[i] = make_float4((float)__ddiv_rn(C[3 * i], m), (float)__ddiv_rn(C[3 * i + 1], m),
                             (float)__ddiv_rn(C[3 * i + 2], m), 0.f);
}
__global__ void k_pack_d(int N, const double *x, const double *C, double mO, double mH,
                         const int *atom_rep, const double *rep_box, double4 *pos, double4 *wgt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const bool is_h = (i % 3) != 0;
    const double m = is_h ? mH : mO;
    const double L = rep_box[atom_rep[i]];
    const double *xo = x + 9 * (size_t)(i / 3);
    pos[i] = make_double4(gather_coord(xo[0], x[3 * i], is_h, L), gather_coord(xo[1], x[3 * i + 1], is_h, L),
                          gather_coord(xo[2], x[3 * i + 2], is_h, L), 0.0);
    if (C)
        wgt[i] = make_double4(__ddiv_rn(C[3 * i], m), __ddiv_rn(C[3 * i + 1], m),
                              __ddiv_rn(C[3 * i + 2], m), 0.0);
}

// Part 1 of a reverse step (water.jl:1496-1502), one thread per molecule; writes the
// gather buffers read by the next reverse-step kernel.
template <typename V4>
__global__ void k_unintegrate(int M, StepArgs a, const int *mol_rep) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= M) return;
    const int rep = mol_rep[I];
    const double Ld = a.rep_box[rep];
    const double dt2 = __dmul_rn(a.dt, a.dt);
    double xn[9];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int i = 3 * I + k;
        const bool isO = k == 0;
        const double m = isO ? a.mO : a.mH;
        double xi[3] = {0.0, 0.0, 0.0};
        if (a.s != 0.0) {
            if (a.noise_cur) {
#pragma unroll
                for (int u = 0; u < 3; u++) xi[u] = a.noise_cur[3 * (size_t)i + u];
            } else {
                atom_noise(a.seed_cur[rep], (uint32_t)(i - a.rep_atom0[rep]),
                           isO ? a.rep_sdO[rep] : a.rep_sdH[rep], xi);
            }
        }
        double Cm[3];
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const size_t e = 3 * (size_t)i + u;
            double x = a.x[e], v = a.v[e];
            const double h2 = __dmul_rn(__dmul_rn(v, a.dt), 0.5);
            x = __dsub_rn(x, a.exact ? qgrid(h2) : h2);
            v = __ddiv_rn(__dsub_rn(v, __dmul_rn(xi[u], a.s)), a.c);
            if (a.exact) v = qgrid(v);
            const double h1 = __dmul_rn(__dmul_rn(v, a.dt), 0.5);
            x = __dsub_rn(x, a.exact ? qgrid(h1) : h1);
            x = a.exact ? wrap_exact(x, Ld) : wrap1d(x, Ld);
            const double D = __dadd_rn(__dmul_rn(a.c, a.D[e]),
                                       __ddiv_rn(__dmul_rn(__dmul_rn(dt2, a.G[e]), __dadd_rn(1.0, a.c)), 2.0));
            const double C = __dadd_rn(a.C[e], D);
            a.x[e] = x;
            a.v[e] = v;
            a.D[e] = D;
            a.C[e] = C;
            xn[3 * k + u] = x;
            Cm[u] = __ddiv_rn(C, m);
        }
        using R = decltype(V4::x);
        V4 wo;
        wo.x = (R)Cm[0];
        wo.y = (R)Cm[1];
        wo.z = (R)Cm[2];
        wo.w = R(0);
        ((V4 *)a.wgt_out)[i] = wo;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        using R = decltype(V4::x);
        V4 po;
        if constexpr (sizeof(R) == 4) {
            po = gather_f32(xn, xn + 3 * k, k, Ld);
        } else {
            po.x = (R)gather_coord(xn[0], xn[3 * k], k != 0, Ld);
            po.y = (R)gather_coord(xn[1], xn[3 * k + 1], k != 0, Ld);
            po.z = (R)gather_coord(xn[2], xn[3 * k + 2], k != 0, Ld);
            po.w = R(0);
        }
        ((V4 *)a.pos_out)[3 * I + k] = po;
    }
}

__global__ void k_quantize_state(int N, double *x, double *v, const int *atom_rep, const double *rep_box) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double L = rep_box[atom_rep[i]];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const size_t e = 3 * (size_t)i + u;
        x[e] = wrap_exact(qgrid(x[e]), L);
        v[e] = qgrid(v[e]);
    }
}

// Clipping of dl_dfi by its norm (water.jl:1511-1515) and the deferred B/A updates.
__global__ void k_clip_post(int N, StepArgs a, const int *atom_rep, const double *scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int rep = atom_rep[i];
    const double nrm = scale[2 * rep], thr = scale[2 * rep + 1];
    const double dt2 = __dmul_rn(a.dt, a.dt);
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const size_t e = 3 * (size_t)i + u;
        double Gv = a.G[e];
        if (nrm > thr) Gv = __ddiv_rn(__dmul_rn(Gv, thr), nrm);
        a.G[e] = Gv;
        const double B = __dadd_rn(__dmul_rn(a.c, a.B[e]), __dmul_rn(dt2, Gv));
        a.B[e] = B;
        a.A[e] = __dadd_rn(a.A[e], B);
    }
}

// Adjoint accumulators at a loss point (water.jl:1480-1483, 1541-1545).
__global__ void k_init_adjoint(int n3, const double *g, double c, double *A, double *B, double *C,
                               double *D, double *G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n3) return;
    const double gv = g[e];
    const double opc = __dadd_rn(1.0, c);
    A[e] = __dmul_rn(gv, opc);
    B[e] = __dmul_rn(gv, opc);
    C[e] = 0.0;
    D[e] = __ddiv_rn(__dmul_rn(gv, __dadd_rn(__dadd_rn(1.0, __dmul_rn(2.0, c)), __dmul_rn(c, c))),
                     __dmul_rn(2.0, c));
    G[e] = 0.0;
}

__global__ void k_noise(int N, const int *atom_rep, const int *rep_atom0, const double *rep_sdO,
                        const double *rep_sdH, const uint64_t *seeds, double *xi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int rep = atom_rep[i];
    atom_noise(seeds[rep], (uint32_t)(i - rep_atom0[rep]), (i % 3 == 0) ? rep_sdO[rep] : rep_sdH[rep],
               xi + 3 * (size_t)i);
}

}  // namespace

template <typename R>
cudaError_t launch_step(bool rev, int form, int G, int unroll, bool shift, int n_blk, int threads,
                        const StepArgs &a, const NbConsts<R> &nb, const BondConsts &bc,
                        cudaStream_t st) {
    switch (form) {
        case F_LJ: return launch_form<R, F_LJ>(rev, G, unroll, shift, n_blk, threads, a, nb, bc, st);
        case F_DEXP: return launch_form<R, F_DEXP>(rev, G, unroll, shift, n_blk, threads, a, nb, bc, st);
        case F_BUCK: return launch_form<R, F_BUCK>(rev, G, unroll, shift, n_blk, threads, a, nb, bc, st);
        case F_LJSC: return launch_form<R, F_LJSC>(rev, G, unroll, shift, n_blk, threads, a, nb, bc, st);
        case F_BUFF: return launch_form<R, F_BUFF>(rev, G, unroll, shift, n_blk, threads, a, nb, bc, st);
        case F_LJ_MLP: return launch_form<R, F_LJ_MLP>(rev, G, unroll, shift, n_blk, threads, a, nb, bc, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_half(bool rev, int form, int G, int n_blk, int threads, const StepArgs &a,
                        const NbConsts<float> &nb, const BondConsts &bc, cudaStream_t st) {
    switch (form) {
        case F_LJ: return launch_half_form<float, F_LJ>(rev, G, n_blk, threads, a, nb, bc, st);
        case F_DEXP: return launch_half_form<float, F_DEXP>(rev, G, n_blk, threads, a, nb, bc, st);
        case F_BUCK: return launch_half_form<float, F_BUCK>(rev, G, n_blk, threads, a, nb, bc, st);
        case F_LJSC: return launch_half_form<float, F_LJSC>(rev, G, n_blk, threads, a, nb, bc, st);
        case F_BUFF: return launch_half_form<float, F_BUFF>(rev, G, n_blk, threads, a, nb, bc, st);
        case F_LJ_MLP: return launch_half_form<float, F_LJ_MLP>(rev, G, n_blk, threads, a, nb, bc, st);
    }
    return cudaErrorInvalidValue;
}

template cudaError_t launch_step<float>(bool, int, int, int, bool, int, int, const StepArgs &,
                                        const NbConsts<float> &, const BondConsts &, cudaStream_t);
template cudaError_t launch_step<double>(bool, int, int, int, bool, int, int, const StepArgs &,
                                         const NbConsts<double> &, const BondConsts &, cudaStream_t);

cudaError_t launch_pack(int N, int prec, const double *x, const double *C, double mO, double mH,
                        const int *atom_rep, const double *rep_box, void *pos, void *wgt,
                        cudaStream_t st) {
    const int t = 256, b = (N + t - 1) / t;
    if (prec == 1)
        k_pack_f<<<b, t, 0, st>>>(N, x, C, mO, mH, atom_rep, rep_box, (float4 *)pos, (float4 *)wgt);
    else
        k_pack_d<<<b, t, 0, st>>>(N, x, C, mO, mH, atom_rep, rep_box, (double4 *)pos, (double4 *)wgt);
    return cudaGetLastError();
}

cudaError_t launch_unintegrate(int M, int prec, const StepArgs &a, const int *mol_rep,
                               cudaStream_t st) {
    const int t = 128, b = (M + t - 1) / t;
    if (prec == 1)
        k_unintegrate<float4><<<b, t, 0, st>>>(M, a, mol_rep);
    else
        k_unintegrate<double4><<<b, t, 0, st>>>(M, a, mol_rep);
    return cudaGetLastError();
}

cudaError_t launch_quantize_state(int N, double *x, double *v, const int *atom_rep, const double *rep_box,
                                  cudaStream_t st) {
    const int t = 256, b = (N + t - 1) / t;
    k_quantize_state<<<b, t, 0, st>>>(N, x, v, atom_rep, rep_box);
    return cudaGetLastError();
}

cudaError_t launch_clip_post(int N, const StepArgs &a, const int *atom_rep, const double *scale,
                             cudaStream_t st) {
    const int t = 256, b = (N + t - 1) / t;
    k_clip_post<<<b, t, 0, st>>>(N, a, atom_rep, scale);
    return cudaGetLastError();
}

cudaError_t launch_init_adjoint(int N, const double *g, double c, double *A, double *B, double *C,
                                double *D, double *G, cudaStream_t st) {
    const int n3 = 3 * N, t = 256, b = (n3 + t - 1) / t;
    k_init_adjoint<<<b, t, 0, st>>>(n3, g, c, A, B, C, D, G);
    return cudaGetLastError();
}

cudaError_t launch_noise(int N, const int *atom_rep, const int *rep_atom0, const double *rep_sdO,
                         const double *rep_sdH, const uint64_t *seeds, double *xi,
                         cudaStream_t st) {
    const int t = 256, b = (N + t - 1) / t;
    k_noise<<<b, t, 0, st>>>(N, atom_rep, rep_atom0, rep_sdO, rep_sdH, seeds, xi);
    return cudaGetLastError();
}

}  // namespace rs
