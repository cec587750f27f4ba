// rs_mlp_tc.cu -- the learned pair correction's network on the tensor cores: BF16 operands,
// FP32 accumulation (mma.sync.m16n8k16 with bf16 inputs), for the node evaluation that builds
// the interval table and for its backward pass to the weights.
//
// Each FP32 operand x is split into two BF16 values, hi = bf16(x) and lo = bf16(x - hi), and
// each product is formed as A_lo B_hi + A_hi B_lo + A_hi B_hi (three MMAs, the small terms
// first): about 16 significant bits per operand instead of 8.  With plain BF16 operands the
// weight gradients, sums over the 1,025 nodes whose terms largely cancel, came out ~40 % off
// the FP64 result; split they agree to ~1e-4.
//
// Per element pair type t the network is u(r) = fc(r) (b3 + w3 . silu(W2 silu(W1 phi(r) + b1)
// + b2)) with 16 Gaussian radial basis functions phi (rs_mlp.cu).  Evaluated at many distances
// at once it is a chain of small GEMMs over a batch of rows (distances):
//   forward  Z1 = Phi W1^T (+ b1), Z2 = silu(Z1) W2^T (+ b2), and the r-tangent stream
//            dZ1 = dPhi W1^T, dZ2 = (silu'(Z1) o dZ1) W2^T, giving u and du/dr per row;
//   backward (adjoints au, ad of u and du/dr per node) Z2b, dZ2b elementwise, then
//            H1b = Z2b W2, dH1b = dZ2b W2, and Z1b = H1b o silu'(Z1) + dH1b o silu''(Z1) o dZ1
//            (the mixed second derivative d^2u / dr dtheta enters through silu''), dZ1b;
//   weights  gW2 = Z2b^T silu(Z1) + dZ2b^T (silu'(Z1) o dZ1), gW1 = Z1b^T Phi + dZ1b^T dPhi
//            (GEMMs whose reduction dimension is the node batch), and the bias / output-layer
//            sums.
// One warp owns a tile of 16 rows; the layer-1 C fragments become the layer-2 A fragments in
// registers.  Every sum has a fixed order (mma accumulation, fixed shuffle trees, per-tile and
// per-chunk partials reduced in index order in FP64), so the results are deterministic.
#include <algorithm>

#include <cuda_bf16.h>

#include "rs_internal.h"

namespace rs {

namespace {

constexpr int NR = MLP_NRBF, H = MLP_H, NG = MLP_NG;
constexpr int NODES = NG + 1;                    // nodes of one type
constexpr int NPAD = ((NODES + 79) / 80) * 80;   // 1040: 65 row tiles, 13 chunks of 80
constexpr int NTILE = NPAD / 16;
constexpr int CHUNK = 80, NCHUNK = NPAD / CHUNK;
constexpr int W1S = 12;   // shared-memory row stride of W1 in 32-bit words (8 used)
constexpr int W2S = 36;   // ... of W2 and W2^T (32 used)

struct TcWeights {        // one type's weights in shared memory, split hi / lo
    uint32_t w1[H * W1S], w1l[H * W1S];     // W1 [i][k] as bf16 pairs along k
    uint32_t w2[H * W2S], w2l[H * W2S];     // W2 [i][j] as bf16 pairs along j
    uint32_t w2t[H * W2S], w2tl[H * W2S];   // W2^T [j][i] as bf16 pairs along i
    float b1[H], b2[H], w3[H];
    float b3;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// x = hi + lo with hi = bf16(x): the remainder x - hi is exact in FP32.
__device__ __forceinline__ float bf16_rest(float x) {
    return x - __bfloat162float(__float2bfloat16_rn(x));
}

// Two consecutive elements (a, b) as split bf16 pairs.
struct Pair2 {
    uint32_t hi, lo;
};
__device__ __forceinline__ Pair2 split2(float a, float b) {
    return Pair2{pack_bf16(a, b), pack_bf16(bf16_rest(a), bf16_rest(b))};
}

// D = A B + D, m16n8k16, A 16x16 row-major bf16, B 16x8 column-major bf16, D FP32.
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// D += A B with split operands: A_lo B_hi + A_hi B_lo + A_hi B_hi.
__device__ __forceinline__ void mma3(float d[4], const uint32_t ah[4], const uint32_t al[4], uint32_t bh0,
                                     uint32_t bh1, uint32_t bl0, uint32_t bl1) {
    mma_bf16(d, al, bh0, bh1);
    mma_bf16(d, ah, bl0, bl1);
    mma_bf16(d, ah, bh0, bh1);
}

// An A fragment (four split pairs) from rows/columns already placed per the m16n8k16 layout.
__device__ __forceinline__ void frag_split(const Pair2 p[4], uint32_t ah[4], uint32_t al[4]) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        ah[q] = p[q].hi;
        al[q] = p[q].lo;
    }
}

__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu0(float z) { return z * sigm(z); }
__device__ __forceinline__ float silu1(float z) {
    const float s = sigm(z);
    return s * (1.f + z * (1.f - s));
}
__device__ __forceinline__ float silu2(float z) {
    const float s = sigm(z);
    return s * (1.f - s) * (2.f + z * (1.f - 2.f * s));
}

// Gaussian basis function k at r and its r-derivative (rs_mlp.cu: centres k rc / 15).
__device__ __forceinline__ void rbf_f(float r, float rc, float w, int k, float &phi, float &dphi) {
    const float mu = k * rc / (NR - 1), e = r - mu;
    phi = expf(-e * e / (2.f * w * w));
    dphi = -e / (w * w) * phi;
}

// Type t's weights (FP64 parameters) into shared memory as BF16 (matrices) and FP32.
__device__ void load_weights(const double *theta, int t, TcWeights &s) {
    const double *W1 = theta + (size_t)t * MLP_PER_TYPE;
    const double *b1 = W1 + H * NR, *W2 = b1 + H, *b2 = W2 + H * H, *w3 = b2 + H, *b3 = w3 + H;
    for (int q = threadIdx.x; q < H * NR / 2; q += blockDim.x) {
        const int i = q / (NR / 2), k2 = q % (NR / 2);
        const Pair2 w = split2((float)W1[i * NR + 2 * k2], (float)W1[i * NR + 2 * k2 + 1]);
        s.w1[i * W1S + k2] = w.hi;
        s.w1l[i * W1S + k2] = w.lo;
    }
    for (int q = threadIdx.x; q < H * H / 2; q += blockDim.x) {
        const int i = q / (H / 2), j2 = q % (H / 2);
        const Pair2 w = split2((float)W2[i * H + 2 * j2], (float)W2[i * H + 2 * j2 + 1]);
        const Pair2 t = split2((float)W2[(2 * j2) * H + i], (float)W2[(2 * j2 + 1) * H + i]);
        s.w2[i * W2S + j2] = w.hi;
        s.w2l[i * W2S + j2] = w.lo;
        s.w2t[i * W2S + j2] = t.hi;
        s.w2tl[i * W2S + j2] = t.lo;
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        s.b1[i] = (float)b1[i];
        s.b2[i] = (float)b2[i];
        s.w3[i] = (float)w3[i];
    }
    if (threadIdx.x == 0) s.b3 = (float)b3[0];
    __syncthreads();
}

// Forward of one 16-row tile: rows r0 (row g of the fragments) and r1 (row g + 8).  Leaves
// the layer C fragments z1, dz1, z2, dz2 [n-tile][4] and the row outputs y, dy (quad-reduced,
// for rows g and g + 8).
struct Fwd {
    float z1[8][4], dz1[8][4], z2[8][4], dz2[8][4];
    float y[2], dy[2];
};

__device__ __forceinline__ void tile_forward(const TcWeights &s, float r0, float r1, float rc, float w,
                                             Fwd &f) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    // layer-1 A fragments: phi and dphi of rows (r0, r1) at k = 2tq, 2tq+1, 2tq+8, 2tq+9
    float p[2][4], dp[2][4];
    const int ks[4] = {2 * tq, 2 * tq + 1, 2 * tq + 8, 2 * tq + 9};
#pragma unroll
    for (int q = 0; q < 4; q++) {
        rbf_f(r0, rc, w, ks[q], p[0][q], dp[0][q]);
        rbf_f(r1, rc, w, ks[q], p[1][q], dp[1][q]);
    }
    uint32_t a1h[4], a1l[4], da1h[4], da1l[4];
    {
        const Pair2 pa[4] = {split2(p[0][0], p[0][1]), split2(p[1][0], p[1][1]), split2(p[0][2], p[0][3]),
                             split2(p[1][2], p[1][3])};
        const Pair2 pd[4] = {split2(dp[0][0], dp[0][1]), split2(dp[1][0], dp[1][1]), split2(dp[0][2], dp[0][3]),
                             split2(dp[1][2], dp[1][3])};
        frag_split(pa, a1h, a1l);
        frag_split(pd, da1h, da1l);
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int o = (8 * j + g) * W1S + tq;
        const uint32_t b0 = s.w1[o], b1 = s.w1[o + 4], bl0 = s.w1l[o], bl1 = s.w1l[o + 4];
        const float bb0 = s.b1[8 * j + 2 * tq], bb1 = s.b1[8 * j + 2 * tq + 1];
        float c[4] = {bb0, bb1, bb0, bb1}, dc[4] = {0.f, 0.f, 0.f, 0.f};
        mma3(c, a1h, a1l, b0, b1, bl0, bl1);
        mma3(dc, da1h, da1l, b0, b1, bl0, bl1);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            f.z1[j][q] = c[q];
            f.dz1[j][q] = dc[q];
        }
    }
    // layer 2: A fragments from the layer-1 activations (two C tiles per k-tile)
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const float bb0 = s.b2[8 * j + 2 * tq], bb1 = s.b2[8 * j + 2 * tq + 1];
        f.z2[j][0] = bb0;
        f.z2[j][1] = bb1;
        f.z2[j][2] = bb0;
        f.z2[j][3] = bb1;
#pragma unroll
        for (int q = 0; q < 4; q++) f.dz2[j][q] = 0.f;
    }
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
        float h[2][4], dh[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float z = f.z1[2 * kt + u][q];
                h[u][q] = silu0(z);
                dh[u][q] = silu1(z) * f.dz1[2 * kt + u][q];
            }
        uint32_t ah[4], al[4], dah[4], dal[4];
        {
            const Pair2 ph[4] = {split2(h[0][0], h[0][1]), split2(h[0][2], h[0][3]), split2(h[1][0], h[1][1]),
                                 split2(h[1][2], h[1][3])};
            const Pair2 pd[4] = {split2(dh[0][0], dh[0][1]), split2(dh[0][2], dh[0][3]), split2(dh[1][0], dh[1][1]),
                                 split2(dh[1][2], dh[1][3])};
            frag_split(ph, ah, al);
            frag_split(pd, dah, dal);
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int o = (8 * j + g) * W2S + 8 * kt + tq;
            const uint32_t b0 = s.w2[o], b1 = s.w2[o + 4], bl0 = s.w2l[o], bl1 = s.w2l[o + 4];
            mma3(f.z2[j], ah, al, b0, b1, bl0, bl1);
            mma3(f.dz2[j], dah, dal, b0, b1, bl0, bl1);
        }
    }
    // outputs: y = b3 + w3 . silu(z2), dy = w3 . (silu'(z2) dz2), rows g and g + 8
    float y0 = 0.f, y1 = 0.f, d0 = 0.f, d1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const float wv = s.w3[8 * j + 2 * tq + c];
            y0 = fmaf(wv, silu0(f.z2[j][c]), y0);
            y1 = fmaf(wv, silu0(f.z2[j][2 + c]), y1);
            d0 = fmaf(wv, silu1(f.z2[j][c]) * f.dz2[j][c], d0);
            d1 = fmaf(wv, silu1(f.z2[j][2 + c]) * f.dz2[j][2 + c], d1);
        }
#pragma unroll
    for (int o = 1; o <= 2; o <<= 1) {
        y0 += __shfl_xor_sync(0xffffffffu, y0, o);
        y1 += __shfl_xor_sync(0xffffffffu, y1, o);
        d0 += __shfl_xor_sync(0xffffffffu, d0, o);
        d1 += __shfl_xor_sync(0xffffffffu, d1, o);
    }
    f.y[0] = y0 + s.b3;
    f.y[1] = y1 + s.b3;
    f.dy[0] = d0;
    f.dy[1] = d1;
}

__device__ __forceinline__ void cutoff(double r, double rc, double &fc, double &dfc) {
    const double x = 3.14159265358979323846 * r / rc;
    fc = 0.5 * (cos(x) + 1.0);
    dfc = -0.5 * 3.14159265358979323846 / rc * sin(x);
}

// u, du/dr at n distances per type (blockIdx.y = type): the nodes g rc / NG (r == null) or
// the given distances r[t * n + row].
__global__ void __launch_bounds__(128) k_mlp_tc_fwd(const double *theta, double rc, double w, int n,
                                                   const double *r, double *u, double *du) {
    __shared__ TcWeights s;
    const int t = blockIdx.y;
    load_weights(theta, t, s);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    const int ntile = (n + 15) / 16;
    for (int tile = blockIdx.x * 4 + warp; tile < ntile; tile += gridDim.x * 4) {
        const int row0 = tile * 16 + g, row1 = row0 + 8;
        const double rr0 = r ? (row0 < n ? r[(size_t)t * n + row0] : 0.0) : row0 * (rc / NG);
        const double rr1 = r ? (row1 < n ? r[(size_t)t * n + row1] : 0.0) : row1 * (rc / NG);
        Fwd f;
        tile_forward(s, (float)rr0, (float)rr1, (float)rc, (float)w, f);
        if (tq == 0) {
            const double rows[2] = {rr0, rr1};
            const int idx[2] = {row0, row1};
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (idx[h] >= n) continue;
                double fc, dfc;
                cutoff(rows[h], rc, fc, dfc);
                u[(size_t)t * n + idx[h]] = (double)f.y[h] * fc;
                du[(size_t)t * n + idx[h]] = (double)f.dy[h] * fc + (double)f.y[h] * dfc;
            }
        }
    }
}

// Scratch of the backward pass per type: transposed BF16 operands of the weight-gradient
// GEMMs [64][NPAD] (Z2b, dZ2b, H1 = silu(Z1), dH1, Z1b, dZ1b) and [16][NPAD] (Phi, dPhi),
// per-tile FP32 partials [NTILE][64] of b1, b2, w3 and [NTILE] of b3, per-chunk FP32 partials
// [NCHUNK][64][64] of W2 and [NCHUNK][64][16] of W1.
struct TcScratch {
    // [0]: hi parts, [1]: lo parts
    __nv_bfloat16 *z2b[2], *dz2b[2], *h1[2], *dh1[2], *z1b[2], *dz1b[2], *phi[2], *dphi[2];
    float *pb1, *pb2, *pw3, *pb3, *pW2, *pW1;
};

__host__ __device__ inline size_t tc_scratch_bytes_per_type() {
    const size_t b = 2 * sizeof(__nv_bfloat16) * ((size_t)6 * H * NPAD + 2 * (size_t)NR * NPAD) +
                     sizeof(float) * ((size_t)3 * NTILE * H + NTILE + (size_t)NCHUNK * H * H +
                                      (size_t)NCHUNK * H * NR);
    return (b + 255) / 256 * 256;
}

__host__ __device__ inline TcScratch tc_view(void *base, int t) {
    char *p = (char *)base + (size_t)t * tc_scratch_bytes_per_type();
    TcScratch s;
    auto take_b = [&](size_t n) {
        __nv_bfloat16 *q = (__nv_bfloat16 *)p;
        p += sizeof(__nv_bfloat16) * n;
        return q;
    };
    auto take_f = [&](size_t n) {
        float *q = (float *)p;
        p += sizeof(float) * n;
        return q;
    };
    for (int h = 0; h < 2; h++) {
        s.z2b[h] = take_b((size_t)H * NPAD);
        s.dz2b[h] = take_b((size_t)H * NPAD);
        s.h1[h] = take_b((size_t)H * NPAD);
        s.dh1[h] = take_b((size_t)H * NPAD);
        s.z1b[h] = take_b((size_t)H * NPAD);
        s.dz1b[h] = take_b((size_t)H * NPAD);
        s.phi[h] = take_b((size_t)NR * NPAD);
        s.dphi[h] = take_b((size_t)NR * NPAD);
    }
    s.pb1 = take_f((size_t)NTILE * H);
    s.pb2 = take_f((size_t)NTILE * H);
    s.pw3 = take_f((size_t)NTILE * H);
    s.pb3 = take_f(NTILE);
    s.pW2 = take_f((size_t)NCHUNK * H * H);
    s.pW1 = take_f((size_t)NCHUNK * H * NR);
    return s;
}

// Column sums over the 16 rows of a tile held by a warp's C fragments: v[j][0..1] (row g) +
// v[j][2..3] (row g + 8), summed over g by a fixed shuffle tree; lanes 0..3 hold columns
// 8j + 2 tq + {0, 1}.
__device__ __forceinline__ void col_sums(const float v[8][4], float out[8][2]) {
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
            float x = v[j][c] + v[j][2 + c];
#pragma unroll
            for (int o = 4; o <= 16; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            out[j][c] = x;
        }
}

// Backward, part 1: per 16-node tile, the forward recomputed, then the node adjoints
// (au, ad of u and du/dr, node-major [t][NODES]) carried through both streams to Z2b, dZ2b,
// Z1b, dZ1b; writes the weight-gradient GEMM operands (transposed, BF16) and the per-tile
// sums of the bias and output-layer gradients.
__global__ void __launch_bounds__(128) k_mlp_tc_bwd_nodes(const double *theta, double rc, double w,
                                                         const double *au, const double *ad,
                                                         void *scratch) {
    __shared__ TcWeights s;
    const int t = blockIdx.y;
    load_weights(theta, t, s);
    const TcScratch sc = tc_view(scratch, t);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    for (int tile = blockIdx.x * 4 + warp; tile < NTILE; tile += gridDim.x * 4) {
        const int row[2] = {tile * 16 + g, tile * 16 + g + 8};
        double rr[2];
        float yb[2], dyb[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            rr[h] = row[h] * (rc / NG);
            double fc, dfc;
            cutoff(rr[h], rc, fc, dfc);
            const double a = row[h] < NODES ? au[(size_t)t * NODES + row[h]] : 0.0;
            const double d = row[h] < NODES ? ad[(size_t)t * NODES + row[h]] : 0.0;
            // u = y fc, u' = y' fc + y fc'
            yb[h] = (float)(a * fc + d * dfc);
            dyb[h] = (float)(d * fc);
        }
        Fwd f;
        tile_forward(s, (float)rr[0], (float)rr[1], (float)rc, (float)w, f);
        // output layer: Z2b, dZ2b and the w3 terms
        float z2b[8][4], dz2b[8][4], g3[8][4];
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int h = q >> 1;
                const float wv = s.w3[8 * j + 2 * tq + (q & 1)];
                const float z = f.z2[j][q], dz = f.dz2[j][q];
                const float s1 = silu1(z);
                z2b[j][q] = yb[h] * wv * s1 + dyb[h] * wv * silu2(z) * dz;
                dz2b[j][q] = dyb[h] * wv * s1;
                g3[j][q] = yb[h] * silu0(z) + dyb[h] * s1 * dz;
            }
        // H1b = Z2b W2, dH1b = dZ2b W2 (B operand from W2^T)
        float h1b[8][4], dh1b[8][4];
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                h1b[j][q] = 0.f;
                dh1b[j][q] = 0.f;
            }
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            uint32_t ah[4], al[4], dah[4], dal[4];
            {
                const Pair2 pz[4] = {split2(z2b[2 * kt][0], z2b[2 * kt][1]), split2(z2b[2 * kt][2], z2b[2 * kt][3]),
                                     split2(z2b[2 * kt + 1][0], z2b[2 * kt + 1][1]),
                                     split2(z2b[2 * kt + 1][2], z2b[2 * kt + 1][3])};
                const Pair2 pd[4] = {split2(dz2b[2 * kt][0], dz2b[2 * kt][1]),
                                     split2(dz2b[2 * kt][2], dz2b[2 * kt][3]),
                                     split2(dz2b[2 * kt + 1][0], dz2b[2 * kt + 1][1]),
                                     split2(dz2b[2 * kt + 1][2], dz2b[2 * kt + 1][3])};
                frag_split(pz, ah, al);
                frag_split(pd, dah, dal);
            }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int o = (8 * j + g) * W2S + 8 * kt + tq;
                const uint32_t b0 = s.w2t[o], b1 = s.w2t[o + 4], bl0 = s.w2tl[o], bl1 = s.w2tl[o + 4];
                mma3(h1b[j], ah, al, b0, b1, bl0, bl1);
                mma3(dh1b[j], dah, dal, b0, b1, bl0, bl1);
            }
        }
        // hidden layer: Z1b (with the mixed second derivative through silu'') and dZ1b;
        // the transposed GEMM operands of the weight gradients
        float z1b[8][4], dz1b[8][4];
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float z = f.z1[j][q], dz = f.dz1[j][q];
                const float s1 = silu1(z);
                z1b[j][q] = h1b[j][q] * s1 + dh1b[j][q] * silu2(z) * dz;
                dz1b[j][q] = dh1b[j][q] * s1;
                const int rw = row[q >> 1], col = 8 * j + 2 * tq + (q & 1);
                const size_t o = (size_t)col * NPAD + rw;
                auto put = [&](__nv_bfloat16 *const dst[2], float x) {
                    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
                    dst[0][o] = hi;
                    dst[1][o] = __float2bfloat16_rn(x - __bfloat162float(hi));
                };
                put(sc.z2b, z2b[j][q]);
                put(sc.dz2b, dz2b[j][q]);
                put(sc.h1, silu0(z));
                put(sc.dh1, s1 * dz);
                put(sc.z1b, z1b[j][q]);
                put(sc.dz1b, dz1b[j][q]);
            }
        // basis functions of the tile's rows, transposed [k][node]
        if (lane < 16) {
            const int rw = tile * 16 + lane;
            const float rf = (float)(rw * (rc / NG));
#pragma unroll
            for (int k = 0; k < NR; k++) {
                float ph, dph;
                rbf_f(rf, (float)rc, (float)w, k, ph, dph);
                const size_t o = (size_t)k * NPAD + rw;
                const __nv_bfloat16 hp = __float2bfloat16_rn(ph), hd = __float2bfloat16_rn(dph);
                sc.phi[0][o] = hp;
                sc.phi[1][o] = __float2bfloat16_rn(ph - __bfloat162float(hp));
                sc.dphi[0][o] = hd;
                sc.dphi[1][o] = __float2bfloat16_rn(dph - __bfloat162float(hd));
            }
        }
        // per-tile sums of the bias and output-layer gradients
        float cs[8][2];
        col_sums(z1b, cs);
        if (g == 0)
#pragma unroll
            for (int j = 0; j < 8; j++)
#pragma unroll
                for (int c = 0; c < 2; c++) sc.pb1[(size_t)tile * H + 8 * j + 2 * tq + c] = cs[j][c];
        col_sums(z2b, cs);
        if (g == 0)
#pragma unroll
            for (int j = 0; j < 8; j++)
#pragma unroll
                for (int c = 0; c < 2; c++) sc.pb2[(size_t)tile * H + 8 * j + 2 * tq + c] = cs[j][c];
        col_sums(g3, cs);
        if (g == 0)
#pragma unroll
            for (int j = 0; j < 8; j++)
#pragma unroll
                for (int c = 0; c < 2; c++) sc.pw3[(size_t)tile * H + 8 * j + 2 * tq + c] = cs[j][c];
        // b3: sum of yb over the 16 rows (rows g and g + 8 from the lanes with tq == 0)
        float b = (tq == 0) ? yb[0] + yb[1] : 0.f;
#pragma unroll
        for (int o = 1; o <= 16; o <<= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
        if (lane == 0) sc.pb3[tile] = b;
    }
}

// Backward, part 2: the weight-gradient GEMMs over one chunk of 80 nodes per CTA
// (blockIdx.x) and type (blockIdx.y).  Warp w: gW2 columns 8w..8w+7 (all 64 rows) and the gW1
// tile (rows 16 (w / 2).., columns 8 (w % 2)..).  A operands Z2b^T, Z1b^T (M = unit, K = node),
// B operands silu(Z1), Phi (K = node, N = unit), read as bf16 pairs along the node dimension.
__global__ void __launch_bounds__(256) k_mlp_tc_wgrad(void *scratch) {
    const int t = blockIdx.y, ch = blockIdx.x;
    const TcScratch sc = tc_view(scratch, t);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    auto ld2 = [](const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); };
    float acc2[4][4], acc1[4];
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc2[m][q] = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) acc1[q] = 0.f;
    const int m1 = warp >> 1, n1 = warp & 1;
    for (int ks = 0; ks < CHUNK / 16; ks++) {
        const int k0 = ch * CHUNK + ks * 16;
        // B fragments (hi, lo): H1 / dH1 for columns 8 warp + g; Phi / dPhi for columns 8 n1 + g
        const size_t bo = (size_t)(8 * warp + g) * NPAD + k0 + 2 * tq;
        const size_t po = (size_t)(8 * n1 + g) * NPAD + k0 + 2 * tq;
        uint32_t bh[2][2], bd[2][2], bp[2][2], bq[2][2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            bh[h][0] = ld2(sc.h1[h] + bo);
            bh[h][1] = ld2(sc.h1[h] + bo + 8);
            bd[h][0] = ld2(sc.dh1[h] + bo);
            bd[h][1] = ld2(sc.dh1[h] + bo + 8);
            bp[h][0] = ld2(sc.phi[h] + po);
            bp[h][1] = ld2(sc.phi[h] + po + 8);
            bq[h][0] = ld2(sc.dphi[h] + po);
            bq[h][1] = ld2(sc.dphi[h] + po + 8);
        }
        auto afrag = [&](__nv_bfloat16 *const src[2], int m, uint32_t ah[4], uint32_t al[4]) {
            const size_t r0 = (size_t)(16 * m + g) * NPAD + k0 + 2 * tq, r1 = r0 + 8 * (size_t)NPAD;
            const size_t off[4] = {r0, r1, r0 + 8, r1 + 8};
#pragma unroll
            for (int q = 0; q < 4; q++) {
                ah[q] = ld2(src[0] + off[q]);
                al[q] = ld2(src[1] + off[q]);
            }
        };
#pragma unroll
        for (int m = 0; m < 4; m++) {
            uint32_t ah[4], al[4];
            afrag(sc.z2b, m, ah, al);
            mma3(acc2[m], ah, al, bh[0][0], bh[0][1], bh[1][0], bh[1][1]);
            afrag(sc.dz2b, m, ah, al);
            mma3(acc2[m], ah, al, bd[0][0], bd[0][1], bd[1][0], bd[1][1]);
        }
        {
            uint32_t ah[4], al[4];
            afrag(sc.z1b, m1, ah, al);
            mma3(acc1, ah, al, bp[0][0], bp[0][1], bp[1][0], bp[1][1]);
            afrag(sc.dz1b, m1, ah, al);
            mma3(acc1, ah, al, bq[0][0], bq[0][1], bq[1][0], bq[1][1]);
        }
    }
    // C fragment (row 16 m + g (+8), column 8 warp + 2 tq (+1)) -> per-chunk partials
    float *pW2 = sc.pW2 + (size_t)ch * H * H;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int i0 = 16 * m + g, j0 = 8 * warp + 2 * tq;
        pW2[i0 * H + j0] = acc2[m][0];
        pW2[i0 * H + j0 + 1] = acc2[m][1];
        pW2[(i0 + 8) * H + j0] = acc2[m][2];
        pW2[(i0 + 8) * H + j0 + 1] = acc2[m][3];
    }
    float *pW1 = sc.pW1 + (size_t)ch * H * NR;
    const int i0 = 16 * m1 + g, k0 = 8 * n1 + 2 * tq;
    pW1[i0 * NR + k0] = acc1[0];
    pW1[i0 * NR + k0 + 1] = acc1[1];
    pW1[(i0 + 8) * NR + k0] = acc1[2];
    pW1[(i0 + 8) * NR + k0 + 1] = acc1[3];
}

// Backward, part 3: every parameter's gradient in FP64, the partials summed in index order.
__global__ void k_mlp_tc_reduce(int nt, void *scratch, double *dtheta) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nt * MLP_PER_TYPE) return;
    const int t = k / MLP_PER_TYPE, q = k % MLP_PER_TYPE;
    const TcScratch sc = tc_view(scratch, t);
    double s = 0.0;
    if (q < H * NR) {
        for (int c = 0; c < NCHUNK; c++) s += (double)sc.pW1[(size_t)c * H * NR + q];
    } else if (q < H * NR + H) {
        const int i = q - H * NR;
        for (int b = 0; b < NTILE; b++) s += (double)sc.pb1[(size_t)b * H + i];
    } else if (q < H * NR + H + H * H) {
        const int e = q - H * NR - H;
        for (int c = 0; c < NCHUNK; c++) s += (double)sc.pW2[(size_t)c * H * H + e];
    } else if (q < H * NR + 2 * H + H * H) {
        const int i = q - H * NR - H - H * H;
        for (int b = 0; b < NTILE; b++) s += (double)sc.pb2[(size_t)b * H + i];
    } else if (q < MLP_PER_TYPE - 1) {
        const int i = q - H * NR - 2 * H - H * H;
        for (int b = 0; b < NTILE; b++) s += (double)sc.pw3[(size_t)b * H + i];
    } else {
        for (int b = 0; b < NTILE; b++) s += (double)sc.pb3[b];
    }
    dtheta[k] = s;
}

}  // namespace

size_t mlp_tc_scratch_bytes() { return (size_t)MLP_NT * tc_scratch_bytes_per_type(); }

cudaError_t launch_mlp_tc_eval(const double *theta, int nt, double rc, double w, int n, const double *r,
                               double *u, double *du, cudaStream_t st) {
    if (nt < 1 || nt > MLP_NT || n < 1) return cudaErrorInvalidValue;
    const int ntile = (n + 15) / 16;
    const int blocks = std::min((ntile + 3) / 4, 4 * 148);
    k_mlp_tc_fwd<<<dim3(blocks, nt), 128, 0, st>>>(theta, rc, w, n, r, u, du);
    return cudaGetLastError();
}

cudaError_t launch_mlp_tc_backprop(const double *theta, int nt, double rc, double w, const double *au,
                                   const double *ad, void *scratch, double *dtheta, cudaStream_t st) {
    if (nt < 1 || nt > MLP_NT) return cudaErrorInvalidValue;
    k_mlp_tc_bwd_nodes<<<dim3((NTILE + 3) / 4, nt), 128, 0, st>>>(theta, rc, w, au, ad, scratch);
    k_mlp_tc_wgrad<<<dim3(NCHUNK, nt), 256, 0, st>>>(scratch);
    const int np = nt * MLP_PER_TYPE;
    k_mlp_tc_reduce<<<(np + 255) / 256, 256, 0, st>>>(nt, scratch, dtheta);
    return cudaGetLastError();
}

}  // namespace rs
