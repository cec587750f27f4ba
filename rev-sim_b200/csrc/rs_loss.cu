// rs_loss.cu -- smoothed-RDF loss and its gradient on the device.
//
// rdf_differentiable (water.jl:631-691): every (set1, set2) atom pair at minimum-image
// distance d != 0 is smeared over the grid x_k = x_min + step*k with
// g_k(d) = exp(-(x_k - d)^2 / width), restricted to the window |x_k - d| <= cutoff and
// normalised by den(d) = sum of g_k over the index window [ceil((d-c)/step) - off,
// floor((d+c)/step) - off] (water.jl:660-667); h_k = V / (4 pi n1 n2 step) * sum / x_k^2.
// The loss (loss_rdf_part, water.jl:693-697) compares a strided slice of h with a
// target; the gradient is the analytic derivative of the same windowed sums (the
// quantity Enzyme differentiates in the reference's pullback, water.jl:715-736).
// One thread per ordered atom pair, shared-memory histogram, FP64 throughout; the window's
// Gaussians by a two-multiplication recurrence re-anchored on exp every 16 points.
#include <cmath>
#include <mutex>

#include "revsim.h"
#include "rs_internal.h"

namespace rs {

namespace {

__device__ __forceinline__ int rdf_atom(int sel, int atom0, int i) {
    return sel == 0 ? atom0 + 3 * i : atom0 + 3 * (i >> 1) + 1 + (i & 1);
}

__device__ __forceinline__ double grid_x(const RdfArgs &a, int k) {
    return __dadd_rn(a.x_min, __dmul_rn(a.step, (double)k));
}

// Normaliser window, 0-based inclusive.
__device__ __forceinline__ void den_window(const RdfArgs &a, double d, int &lo, int &hi) {
    long long s = (long long)ceil(__ddiv_rn(__dsub_rn(d, a.cutoff), a.step)) - a.off;
    long long e = (long long)floor(__ddiv_rn(__dadd_rn(d, a.cutoff), a.step)) - a.off;
    if (s < 1) s = 1;
    if (e > a.n_grid) e = a.n_grid;
    lo = (int)(s - 1);
    hi = (int)(e - 1);
}

// Histogram window: grid points with x - c <= d <= x + c.
__device__ __forceinline__ void hist_window(const RdfArgs &a, double d, int &lo, int &hi) {
    long long s = (long long)floor(__ddiv_rn(__dsub_rn(__dsub_rn(d, a.cutoff), a.x_min), a.step)) - 1;
    long long e = (long long)ceil(__ddiv_rn(__dsub_rn(__dadd_rn(d, a.cutoff), a.x_min), a.step)) + 1;
    if (s < 0) s = 0;
    if (e > a.n_grid - 1) e = a.n_grid - 1;
    int l = (int)s, h = (int)e;
    while (l <= h && !(d <= __dadd_rn(grid_x(a, l), a.cutoff))) l++;
    while (h >= l && !(d >= __dsub_rn(grid_x(a, h), a.cutoff))) h--;
    lo = l;
    hi = h;
}

// The Gaussians g_k = exp(-(x_k - d)^2 / width) of consecutive grid points by the recurrence
// g_{k+1} = g_k r_k, r_{k+1} = r_k q with r_k = exp(-(2 e_k step + step^2) / width) and
// q = exp(-2 step^2 / width): two multiplications per point instead of an exp.  The
// recurrence restarts from exp every kGaussAnchor points, which bounds the accumulated
// rounding at about kGaussAnchor^2 / 2 ulp (~1e-14 relative).
constexpr int kGaussAnchor = 16;

struct Gauss {
    double g, r;
};

__device__ __forceinline__ void gauss_anchor(const RdfArgs &a, double d, int k, double inv_w,
                                             Gauss &G) {
    const double e = __dsub_rn(grid_x(a, k), d);
    G.g = exp(-__dmul_rn(__dmul_rn(e, e), inv_w));
    G.r = exp(-__dmul_rn(__fma_rn(__dmul_rn(2.0, e), a.step, __dmul_rn(a.step, a.step)), inv_w));
}

__device__ __forceinline__ void gauss_next(Gauss &G, double q) {
    G.g = __dmul_rn(G.g, G.r);
    G.r = __dmul_rn(G.r, q);
}

__device__ __forceinline__ void den_sums(const RdfArgs &a, double d, double inv_w, double q,
                                         double &den, double &dden) {
    int lo, hi;
    den_window(a, d, lo, hi);
    double s = 0.0, ds = 0.0;
    Gauss G{0.0, 0.0};
    for (int k = lo; k <= hi; k++) {
        if (((k - lo) % kGaussAnchor) == 0) gauss_anchor(a, d, k, inv_w, G);
        const double e = __dsub_rn(grid_x(a, k), d);
        s = __dadd_rn(s, G.g);
        ds = __fma_rn(__dmul_rn(__dmul_rn(G.g, 2.0), e), inv_w, ds);
        gauss_next(G, q);
    }
    den = s;
    dden = ds;
}

template <bool GRAD>
__global__ void k_rdf(RdfArgs a, const double *pre) {
    extern __shared__ double s_hist[];
    const int r = blockIdx.y;
    const int nm = a.rep_nmol[r];
    const int atom0 = a.rep_atom0[r];
    const long long n1 = a.sel1 == 0 ? nm : 2LL * nm;
    const long long n2 = a.sel2 == 0 ? nm : 2LL * nm;
    const double L = a.rep_box[r];
    const bool use_smem = !GRAD && a.n_grid <= 6144;
    double *hist = a.hist + (size_t)r * a.n_grid;
    if (use_smem) {
        for (int k = threadIdx.x; k < a.n_grid; k += blockDim.x) s_hist[k] = 0.0;
        __syncthreads();
    }
    const double inv_w = __drcp_rn(a.width);
    const double q = exp(-__dmul_rn(__dmul_rn(2.0, __dmul_rn(a.step, a.step)), inv_w));
    const double dmin = __dsub_rn(__dsub_rn(a.x_min, a.cutoff), a.step);
    const double dmax = __dadd_rn(__dadd_rn(grid_x(a, a.n_grid - 1), a.cutoff), a.step);
    const long long total = n1 * n2;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total;
         p += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(p / n2), i2 = (int)(p % n2);
        const int ia = rdf_atom(a.sel1, atom0, i1), ib = rdf_atom(a.sel2, atom0, i2);
        const double *xa = a.x + 3 * (size_t)ia, *xb = a.x + 3 * (size_t)ib;
        double dr[3];
#pragma unroll
        for (int u = 0; u < 3; u++) dr[u] = vec1d(xa[u], xb[u], L);
        const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dr[0], dr[0]), __dmul_rn(dr[1], dr[1])),
                                              __dmul_rn(dr[2], dr[2])));
        if (d == 0.0 || d < dmin || d > dmax) continue;
        int lo, hi;
        hist_window(a, d, lo, hi);
        if (lo > hi) continue;
        double den, dden;
        den_sums(a, d, inv_w, q, den, dden);
        const double inv_den = __drcp_rn(den);
        Gauss G{0.0, 0.0};
        if (!GRAD) {
            for (int k = lo; k <= hi; k++) {
                if (((k - lo) % kGaussAnchor) == 0) gauss_anchor(a, d, k, inv_w, G);
                const double g = __dmul_rn(G.g, inv_den);
                if (use_smem)
                    atomicAdd(s_hist + k, g);
                else
                    atomicAdd(hist + k, g);
                gauss_next(G, q);
            }
        } else {
            const double *dLdh = a.dLdh + (size_t)r * a.n_grid;
            const double dd2 = __dmul_rn(dden, __dmul_rn(inv_den, inv_den));
            double dLdd = 0.0;
            for (int k = lo; k <= hi; k++) {
                if (((k - lo) % kGaussAnchor) == 0) gauss_anchor(a, d, k, inv_w, G);
                const double w = dLdh[k];
                if (w != 0.0) {
                    const double xk = grid_x(a, k), e = __dsub_rn(xk, d);
                    const double g = G.g;
                    const double gp = __dmul_rn(__dmul_rn(__dmul_rn(g, 2.0), e), inv_w);
                    const double t = __dsub_rn(__dmul_rn(gp, inv_den), __dmul_rn(g, dd2));
                    dLdd = __dadd_rn(dLdd, __dmul_rn(__ddiv_rn(__dmul_rn(w, pre[r]), __dmul_rn(xk, xk)), t));
                }
                gauss_next(G, q);
            }
            if (dLdd != 0.0) {
#pragma unroll
                for (int u = 0; u < 3; u++) {
                    const double gu = __ddiv_rn(__dmul_rn(dLdd, dr[u]), d);
                    atomicAdd(a.dLdx + 3 * (size_t)ib + u, gu);
                    atomicAdd(a.dLdx + 3 * (size_t)ia + u, -gu);
                }
            }
        }
    }
    if (use_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < a.n_grid; k += blockDim.x)
            if (s_hist[k] != 0.0) atomicAdd(hist + k, s_hist[k]);
    }
}

// h_k = pre * sum_k / x_k^2; loss += weight * sum |h - target|^norm over the slice;
// dL/dh at the slice points.  One CTA per replica.
__global__ void k_rdf_finalize(RdfArgs a, const double *pre, const double *target, int s0, int sd,
                               int nt, int norm, double weight, double *loss, double *dLdh) {
    const int r = blockIdx.x;
    double *h = a.hist + (size_t)r * a.n_grid;
    double *gh = dLdh + (size_t)r * a.n_grid;
    for (int k = threadIdx.x; k < a.n_grid; k += blockDim.x) {
        const double xk = grid_x(a, k);
        h[k] = __ddiv_rn(__dmul_rn(pre[r], h[k]), __dmul_rn(xk, xk));
        gh[k] = 0.0;
    }
    __syncthreads();
    __shared__ double s_l[256];
    double l = 0.0;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const int k = s0 + t * sd;
        const double e = __dsub_rn(h[k], target[(size_t)r * nt + t]);
        if (norm == 1) {
            l = __dadd_rn(l, fabs(e));
            gh[k] = weight * (e > 0.0 ? 1.0 : (e < 0.0 ? -1.0 : 0.0));
        } else {
            l = __dadd_rn(l, __dmul_rn(e, e));
            gh[k] = __dmul_rn(weight, __dmul_rn(2.0, e));
        }
    }
    s_l[threadIdx.x] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int t = 0; t < blockDim.x; t++) s = __dadd_rn(s, s_l[t]);
        loss[r] = __dadd_rn(loss[r], __dmul_rn(weight, s));
    }
}

}  // namespace

// pre [R] is stashed by the caller at a.hist + R*n_grid (scratch behind the histogram).
cudaError_t launch_rdf(const RdfArgs &a, int R, int max_n1, int max_n2, bool grad,
                       cudaStream_t st) {
    const long long pairs = (long long)max_n1 * max_n2;
    long long blocks = (pairs + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    const double *pre = a.hist + (size_t)R * a.n_grid;
    if (grad) {
        k_rdf<true><<<dim3((unsigned)blocks, R), 256, 0, st>>>(a, pre);
    } else {
        const size_t smem = a.n_grid <= 6144 ? sizeof(double) * a.n_grid : 0;
        k_rdf<false><<<dim3((unsigned)blocks, R), 256, smem, st>>>(a, pre);
    }
    return cudaGetLastError();
}

cudaError_t launch_rdf_finalize(const RdfArgs &a, int R, const double *pre, const double *target,
                                int slice_start, int slice_stride, int n_target, int norm,
                                double weight, double *loss, double *dLdh, cudaStream_t st) {
    k_rdf_finalize<<<R, 256, 0, st>>>(a, pre, target, slice_start, slice_stride, n_target, norm,
                                      weight, loss, dLdh);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free RDF loss and gradient for one water box.
//
// Some callers cannot let this library call cudaMalloc: a host that owns every byte
// of device memory through its own pool allocator (a Julia or Python framework that
// hands out device pointers), a loop that must not hit the device-wide
// synchronisation cudaMalloc/cudaFree imply, or a service whose memory is budgeted
// in full before it starts.  For them this entry point takes the caller's device
// buffers and keeps its scratch (the histogram, dL/dh, the normalisation constant
// and a one-box table, at most kNoallocMaxGrid grid points) in the file-scope
// array g_rdf_scratch, which every GPU that loads the library holds until the
// process exits.  Host code cannot use the array's name as a device address: the
// address is looked up once per device with cudaGetSymbolAddress, with that device
// current, on the first call that device sees (make that first call before any
// stream capture).  The looked-up address belongs to the device's current context: a
// cudaDeviceReset of that device invalidates it, so the entry point must not be called
// again in a process after it has reset the device.  All calls share the one array and
// leave the last call's values in it; each call clears what must start at zero, and calls
// that overlap on the GPU (concurrent streams, or several host threads on one device) race
// on it.  On an error return the outputs may be partly written.
namespace {

constexpr int kNoallocMaxGrid = 8192;
// layout (doubles): hist [kNoallocMaxGrid + 1] (the normaliser V / (4 pi n1 n2 step)
// sits right after the n_grid used entries) | dL/dh [kNoallocMaxGrid] | box [1] |
// {atom0, n_mol} as two ints [1]
constexpr int kNoallocDLdh = kNoallocMaxGrid + 1;
constexpr int kNoallocBox = 2 * kNoallocMaxGrid + 1;
constexpr int kNoallocInts = 2 * kNoallocMaxGrid + 2;
constexpr int kNoallocDoubles = 2 * kNoallocMaxGrid + 3;
static __device__ __align__(256) double g_rdf_scratch[kNoallocDoubles];

__global__ void k_noalloc_tables(double *s, int n_grid, double pre, double box, int n_mol) {
    s[n_grid] = pre;
    s[kNoallocBox] = box;
    int *t = reinterpret_cast<int *>(s + kNoallocInts);
    t[0] = 0;
    t[1] = n_mol;
}

std::mutex g_noalloc_mu;
double *g_noalloc_addr[256] = {};

}  // namespace

}  // namespace rs

extern "C" int32_t revsim_rdf_loss_grad_noalloc(const double *d_x, int32_t n_mol, double box,
                                                const revsim_rdf_term *t, const double *d_target,
                                                double *d_loss, double *d_dLdx, void *stream) {
    using namespace rs;
    if (!d_x || !t || !d_target || !d_loss || !d_dLdx || n_mol < 1 || !(box > 0)) return REVSIM_ERR_BADARG;
    if (t->n_grid < 1 || t->n_grid > kNoallocMaxGrid) return REVSIM_ERR_BADARG;   // beyond the scratch size
    if (!(t->step > 0) || !(t->width > 0) || !(t->exp_cutoff >= 0) || t->n_target < 1 || t->slice_start < 0 ||
        t->slice_stride < 1 || t->slice_start + (long long)(t->n_target - 1) * t->slice_stride >= t->n_grid ||
        (t->norm != 1 && t->norm != 2) || (t->sel1 != 0 && t->sel1 != 1) || (t->sel2 != 0 && t->sel2 != 1))
        return REVSIM_ERR_BADARG;
    const double q = t->x_min / t->step;
    if (std::fabs(q - std::llround(q)) > 1e-6) return REVSIM_ERR_BADARG;
    if (!rdf_term_recurrence_ok(t->step, t->width, t->exp_cutoff)) return REVSIM_ERR_BADARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return REVSIM_ERR_CUDA;
    double *s = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_rdf_scratch) != cudaSuccess || !p) return REVSIM_ERR_CUDA;
            g_noalloc_addr[dev] = static_cast<double *>(p);
        }
        s = g_noalloc_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double n1 = t->sel1 == 0 ? n_mol : 2.0 * n_mol;
    const double n2 = t->sel2 == 0 ? n_mol : 2.0 * n_mol;
    const double pre = box * box * box / (4 * 3.14159265358979323846 * n1 * n2 * t->step);
    k_noalloc_tables<<<1, 1, 0, st>>>(s, t->n_grid, pre, box, n_mol);
    if (cudaGetLastError() != cudaSuccess) return REVSIM_ERR_CUDA;
    if (cudaMemsetAsync(s, 0, sizeof(double) * t->n_grid, st) != cudaSuccess ||
        cudaMemsetAsync(d_loss, 0, sizeof(double), st) != cudaSuccess ||
        cudaMemsetAsync(d_dLdx, 0, sizeof(double) * 9 * (size_t)n_mol, st) != cudaSuccess)
        return REVSIM_ERR_CUDA;
    RdfArgs a;
    a.x = d_x;
    a.rep_atom0 = reinterpret_cast<const int *>(s + kNoallocInts);
    a.rep_nmol = a.rep_atom0 + 1;
    a.rep_box = s + kNoallocBox;
    a.sel1 = t->sel1;
    a.sel2 = t->sel2;
    a.x_min = t->x_min;
    a.step = t->step;
    a.width = t->width;
    a.cutoff = t->exp_cutoff;
    a.n_grid = t->n_grid;
    a.off = (int)std::llround(q) - 1;
    a.hist = s;
    a.dLdh = s + kNoallocDLdh;
    a.dLdx = d_dLdx;
    if (launch_rdf(a, 1, (int)n1, (int)n2, false, st) != cudaSuccess ||
        launch_rdf_finalize(a, 1, s + t->n_grid, d_target, t->slice_start, t->slice_stride, t->n_target,
                            t->norm, t->weight, d_loss, s + kNoallocDLdh, st) != cudaSuccess ||
        launch_rdf(a, 1, (int)n1, (int)n2, true, st) != cudaSuccess)
        return REVSIM_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? REVSIM_OK : REVSIM_ERR_CUDA;
}

