// rs_mlp.cu -- the learned pair correction of the water model (no reference counterpart;
// it stands in for the reference's PyTorch / JAX learned terms, water_maceoff.jl:147-163).
//
// Per element pair tau in {O-O, O-H, H-H}: u_tau(r) = MLP_tau(phi(r)) fc(r), 16 Gaussian
// radial basis functions (centres k rc / 15, width 0.05 nm), 64 -> 64 SiLU, scalar output,
// fc(r) = (cos(pi r / rc) + 1) / 2.  The MLP depends on r alone, so it is evaluated once per
// parameter update at NG + 1 nodes of [0, rc] (value and r-derivative, FP64) and the step
// kernels interpolate each pair with the cubic Hermite segment of its interval (one
// 16- or 32-byte table load per pair).  The reverse pass accumulates the adjoints of the
// interval coefficients; k_mlp_* below carry them back to the weights once per pass.
// The same code serves the Stillinger-Weber path's learned radial term (one type, its own
// cutoff and width): the type count nt and width w are arguments.
#include "rs_internal.h"

namespace rs {

namespace {

constexpr int NR = MLP_NRBF, H = MLP_H, NG = MLP_NG;
constexpr int NA = 4 * H + 4;   // per-node activations: z1, dz1, z2, dz2, y, dy, fc, dfc

struct View {
    const double *W1, *b1, *W2, *b2, *w3, *b3;
};

__device__ __forceinline__ View view(const double *theta, int t) {
    View v;
    v.W1 = theta + (size_t)t * MLP_PER_TYPE;
    v.b1 = v.W1 + H * NR;
    v.W2 = v.b1 + H;
    v.b2 = v.W2 + H * H;
    v.w3 = v.b2 + H;
    v.b3 = v.w3 + H;
    return v;
}

__device__ __forceinline__ double sigm(double z) { return 1.0 / (1.0 + exp(-z)); }
__device__ __forceinline__ double silu0(double z) { return z * sigm(z); }
__device__ __forceinline__ double silu1(double z) {
    const double s = sigm(z);
    return s * (1.0 + z * (1.0 - s));
}
__device__ __forceinline__ double silu2(double z) {
    const double s = sigm(z);
    return s * (1.0 - s) * (2.0 + z * (1.0 - 2.0 * s));
}

__device__ __forceinline__ void rbf(double r, double rc, double w, int k, double &phi, double &dphi) {
    const double mu = k * rc / (NR - 1), e = r - mu;
    phi = exp(-e * e / (2.0 * w * w));
    dphi = -e / (w * w) * phi;
}

// Sum over the 64 threads of a block in a fixed tree.
__device__ __forceinline__ double block_sum64(double v, double *s) {
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 32; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    const double r = s[0];
    __syncthreads();
    return r;
}

// One block (64 threads = hidden units) per (node g, type t): value and r-tangent streams.
__global__ void __launch_bounds__(64) k_mlp_nodes(const double *theta, double rc, double w, double *act,
                                                  double *u, double *du) {
    __shared__ double s_phi[NR], s_dphi[NR], s_h1[H], s_dh1[H], s_red[H];
    const int g = blockIdx.x, t = blockIdx.y, i = threadIdx.x;
    const View m = view(theta, t);
    const double r = g * (rc / NG);
    if (i < NR) rbf(r, rc, w, i, s_phi[i], s_dphi[i]);
    __syncthreads();
    double z1 = m.b1[i], dz1 = 0.0;
    for (int k = 0; k < NR; k++) {
        z1 += m.W1[i * NR + k] * s_phi[k];
        dz1 += m.W1[i * NR + k] * s_dphi[k];
    }
    s_h1[i] = silu0(z1);
    s_dh1[i] = silu1(z1) * dz1;
    __syncthreads();
    double z2 = m.b2[i], dz2 = 0.0;
    for (int j = 0; j < H; j++) {
        z2 += m.W2[i * H + j] * s_h1[j];
        dz2 += m.W2[i * H + j] * s_dh1[j];
    }
    const double y = m.b3[0] + block_sum64(m.w3[i] * silu0(z2), s_red);
    const double dy = block_sum64(m.w3[i] * silu1(z2) * dz2, s_red);
    double *a = act + ((size_t)t * (NG + 1) + g) * NA;
    a[i] = z1;
    a[H + i] = dz1;
    a[2 * H + i] = z2;
    a[3 * H + i] = dz2;
    if (i == 0) {
        const double x = 3.14159265358979323846 * r / rc;
        const double fc = 0.5 * (cos(x) + 1.0), dfc = -0.5 * 3.14159265358979323846 / rc * sin(x);
        a[4 * H] = y;
        a[4 * H + 1] = dy;
        a[4 * H + 2] = fc;
        a[4 * H + 3] = dfc;
        u[t * (NG + 1) + g] = y * fc;
        du[t * (NG + 1) + g] = dy * fc + y * dfc;
    }
}

// Hermite coefficients of every interval: p(s) = c0 + c1 s + c2 s^2 + c3 s^3, s in [0, 1].
template <typename V4>
__global__ void k_mlp_coef(const double *u, const double *du, double rc, int nt, V4 *tab) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nt * NG) return;
    const int t = k / NG, g = k % NG;
    const double h = rc / NG;
    const double y0 = u[t * (NG + 1) + g], y1 = u[t * (NG + 1) + g + 1];
    const double d0 = du[t * (NG + 1) + g], d1 = du[t * (NG + 1) + g + 1];
    V4 c;
    c.x = y0;
    c.y = h * d0;
    c.z = 3.0 * (y1 - y0) - h * (2.0 * d0 + d1);
    c.w = 2.0 * (y0 - y1) + h * (d0 + d1);
    tab[k] = c;
}

// Coefficient adjoints (summed over the ncopy accumulators in order) -> node value /
// derivative adjoints (the transpose of k_mlp_coef).
__device__ __forceinline__ void sum_copies(const double *cadj, int ncopy, int nt, size_t off, double c[4]) {
    c[0] = c[1] = c[2] = c[3] = 0.0;
    for (int q = 0; q < ncopy; q++) {
        const double *p = cadj + (size_t)q * nt * NG * 4 + off;
        c[0] += p[0];
        c[1] += p[1];
        c[2] += p[2];
        c[3] += p[3];
    }
}

__global__ void k_mlp_adj_nodes(const double *cadj, int ncopy, int nt, double rc, double *au, double *ad) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nt * (NG + 1)) return;
    const int t = k / (NG + 1), g = k % (NG + 1);
    const double h = rc / NG;
    double a = 0.0, d = 0.0, c[4];
    if (g < NG) {
        sum_copies(cadj, ncopy, nt, ((size_t)t * NG + g) * 4, c);
        a += c[0] - 3.0 * c[2] + 2.0 * c[3];
        d += h * (c[1] - 2.0 * c[2] + c[3]);
    }
    if (g > 0) {
        sum_copies(cadj, ncopy, nt, ((size_t)t * NG + g - 1) * 4, c);
        a += 3.0 * c[2] - 2.0 * c[3];
        d += h * (c[3] - c[2]);
    }
    au[k] = a;
    ad[k] = d;
}

// Per node: adjoints of z2, dz2, z1, dz1 and of y, dy (reverse mode through both streams).
__global__ void __launch_bounds__(64) k_mlp_node_bwd(const double *theta, const double *act,
                                                     const double *au, const double *ad,
                                                     double *bwd) {
    __shared__ double s_z2b[H], s_dz2b[H];
    const int g = blockIdx.x, t = blockIdx.y, i = threadIdx.x;
    const View m = view(theta, t);
    const double *a = act + ((size_t)t * (NG + 1) + g) * NA;
    double *b = bwd + ((size_t)t * (NG + 1) + g) * NA;
    const int n = t * (NG + 1) + g;
    const double fc = a[4 * H + 2], dfc = a[4 * H + 3];
    // u = y fc, u' = y' fc + y fc'
    const double yb = au[n] * fc + ad[n] * dfc, dyb = ad[n] * fc;
    const double z2 = a[2 * H + i], dz2 = a[3 * H + i];
    const double h2b = yb * m.w3[i], dh2b = dyb * m.w3[i];
    s_z2b[i] = h2b * silu1(z2) + dh2b * silu2(z2) * dz2;
    s_dz2b[i] = dh2b * silu1(z2);
    __syncthreads();
    double h1b = 0.0, dh1b = 0.0;
    for (int q = 0; q < H; q++) {
        h1b += m.W2[q * H + i] * s_z2b[q];
        dh1b += m.W2[q * H + i] * s_dz2b[q];
    }
    const double z1 = a[i], dz1 = a[H + i];
    b[i] = h1b * silu1(z1) + dh1b * silu2(z1) * dz1;   // z1 adjoint
    b[H + i] = dh1b * silu1(z1);                        // dz1 adjoint
    b[2 * H + i] = s_z2b[i];
    b[3 * H + i] = s_dz2b[i];
    if (i == 0) {
        b[4 * H] = yb;
        b[4 * H + 1] = dyb;
    }
}

// One thread per parameter: sum over the nodes in order (deterministic).
__global__ void k_mlp_wgrad(double rc, double w, int nt, const double *act, const double *bwd,
                            double *dtheta) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nt * MLP_PER_TYPE) return;
    const int t = k / MLP_PER_TYPE, q = k % MLP_PER_TYPE;
    const double *A = act + (size_t)t * (NG + 1) * NA;
    const double *B = bwd + (size_t)t * (NG + 1) * NA;
    double s = 0.0;
    if (q < H * NR) {                              // W1[i][kk]
        const int i = q / NR, kk = q % NR;
        for (int g = 0; g <= NG; g++) {
            double phi, dphi;
            rbf(g * (rc / NG), rc, w, kk, phi, dphi);
            s += B[g * NA + i] * phi + B[g * NA + H + i] * dphi;
        }
    } else if (q < H * NR + H) {                   // b1[i]
        const int i = q - H * NR;
        for (int g = 0; g <= NG; g++) s += B[g * NA + i];
    } else if (q < H * NR + H + H * H) {           // W2[i][j]
        const int i = (q - H * NR - H) / H, j = (q - H * NR - H) % H;
        for (int g = 0; g <= NG; g++) {
            const double z1 = A[g * NA + j], dz1 = A[g * NA + H + j];
            s += B[g * NA + 2 * H + i] * silu0(z1) + B[g * NA + 3 * H + i] * silu1(z1) * dz1;
        }
    } else if (q < H * NR + H + H * H + H) {       // b2[i]
        const int i = q - H * NR - H - H * H;
        for (int g = 0; g <= NG; g++) s += B[g * NA + 2 * H + i];
    } else if (q < MLP_PER_TYPE - 1) {             // w3[i]
        const int i = q - H * NR - H - H * H - H;
        for (int g = 0; g <= NG; g++) {
            const double z2 = A[g * NA + 2 * H + i], dz2 = A[g * NA + 3 * H + i];
            s += B[g * NA + 4 * H] * silu0(z2) + B[g * NA + 4 * H + 1] * silu1(z2) * dz2;
        }
    } else {                                       // b3
        for (int g = 0; g <= NG; g++) s += B[g * NA + 4 * H];
    }
    dtheta[k] = s;
}

}  // namespace

// scratch layout: act [NT][NG+1][NA], bwd [NT][NG+1][NA], u, du, au, ad [NT][NG+1]
size_t mlp_scratch_doubles() { return (size_t)2 * MLP_NT * (NG + 1) * NA + 4 * (size_t)MLP_NT * (NG + 1); }

cudaError_t launch_mlp_table(int prec, const double *theta, double rc, double *scratch, void *tab,
                             cudaStream_t st, int nt, double w) {
    if (nt < 1 || nt > MLP_NT) return cudaErrorInvalidValue;
    const size_t S = (size_t)MLP_NT * (NG + 1) * NA, NN = (size_t)MLP_NT * (NG + 1);
    double *act = scratch, *u = scratch + 2 * S, *du = u + NN;
    k_mlp_nodes<<<dim3(NG + 1, nt), 64, 0, st>>>(theta, rc, w, act, u, du);
    const int n = nt * NG;
    if (prec == 1)
        k_mlp_coef<float4><<<(n + 255) / 256, 256, 0, st>>>(u, du, rc, nt, (float4 *)tab);
    else
        k_mlp_coef<double4><<<(n + 255) / 256, 256, 0, st>>>(u, du, rc, nt, (double4 *)tab);
    return cudaGetLastError();
}

// The tensor-core path (rs_mlp_tc.cu) shares the node arrays of this scratch: the interval
// table from node values computed elsewhere, and the node adjoints alone.
cudaError_t launch_mlp_table_from_nodes(int prec, double *scratch, double rc, void *tab, cudaStream_t st,
                                        int nt) {
    if (nt < 1 || nt > MLP_NT) return cudaErrorInvalidValue;
    const size_t S = (size_t)MLP_NT * (NG + 1) * NA, NN = (size_t)MLP_NT * (NG + 1);
    double *u = scratch + 2 * S, *du = u + NN;
    const int n = nt * NG;
    if (prec == 1)
        k_mlp_coef<float4><<<(n + 255) / 256, 256, 0, st>>>(u, du, rc, nt, (float4 *)tab);
    else
        k_mlp_coef<double4><<<(n + 255) / 256, 256, 0, st>>>(u, du, rc, nt, (double4 *)tab);
    return cudaGetLastError();
}

double *mlp_scratch_nodes(double *scratch, int which) {
    const size_t S = (size_t)MLP_NT * (NG + 1) * NA, NN = (size_t)MLP_NT * (NG + 1);
    return scratch + 2 * S + (size_t)which * NN;   // 0: u, 1: du, 2: au, 3: ad
}

cudaError_t launch_mlp_node_adjoints(const double *cadj, int ncopy, double rc, double *scratch, cudaStream_t st,
                                     int nt) {
    if (nt < 1 || nt > MLP_NT) return cudaErrorInvalidValue;
    const int nn = nt * (NG + 1);
    k_mlp_adj_nodes<<<(nn + 255) / 256, 256, 0, st>>>(cadj, ncopy, nt, rc, mlp_scratch_nodes(scratch, 2),
                                                        mlp_scratch_nodes(scratch, 3));
    return cudaGetLastError();
}

cudaError_t launch_mlp_backprop(const double *theta, double rc, const double *cadj, int ncopy,
                                double *scratch, double *dtheta, cudaStream_t st, int nt, double w) {
    if (nt < 1 || nt > MLP_NT) return cudaErrorInvalidValue;
    const size_t S = (size_t)MLP_NT * (NG + 1) * NA, NN = (size_t)MLP_NT * (NG + 1);
    double *act = scratch, *bwd = scratch + S;
    double *au = scratch + 2 * S + 2 * NN, *ad = au + NN;
    const int nn = nt * (NG + 1), np = nt * MLP_PER_TYPE;
    k_mlp_adj_nodes<<<(nn + 255) / 256, 256, 0, st>>>(cadj, ncopy, nt, rc, au, ad);
    k_mlp_node_bwd<<<dim3(NG + 1, nt), 64, 0, st>>>(theta, act, au, ad, bwd);
    k_mlp_wgrad<<<(np + 127) / 128, 128, 0, st>>>(rc, w, nt, act, bwd, dtheta);
    return cudaGetLastError();
}

}  // namespace rs
