// rs_nlist.cu -- cell-list neighbour build for water (replaces Molly's
// CellListMapNeighborFinder, configured at water.jl:980-991 and rebuilt every
// n_steps_nf steps at water.jl:1025,1038,1504).
//
// The reference keeps an atom-pair list: pairs i<j of different molecules whose
// minimum-image distance is <= 1.2 nm (eligible matrix of diffusion.jl:1133-1147).
// Here the same pair set is stored blocked by molecule: row I lists every molecule
// J != I with at least one listed atom pair, as a 32-bit entry J | mask << 23 whose
// 9-bit mask marks which of the 3x3 atom pairs (own atom a, neighbour atom b; bit
// 3a+b) are in the reference's set.  Rows hold both directions, so each step kernel
// gathers a whole molecule (3 positions) per entry and accumulates the forces of its
// own molecule with no atomics.  Membership distances are FP64, each product and sum
// rounded separately, exactly as the CPU restatement computes them.
#include <algorithm>

#include "rs_internal.h"

namespace rs {

namespace {

__device__ __forceinline__ double dist2_fp64(const double *xa, const double *xb, double L) {
    const double dx = vec1d(xa[0], xb[0], L);
    const double dy = vec1d(xa[1], xb[1], L);
    const double dz = vec1d(xa[2], xb[2], L);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Cell of molecule I (by its O atom), written to cell_of_mol, with the O-H checks:
// molecules are matched by O-O distance with a margin of two O-H lengths.
__device__ __forceinline__ int mol_cell(const NlistArgs &a, int I) {
    const int r = a.mol_rep[I];
    const int nc = a.rep_nc[r];
    const double L = a.rep_box[r];
    const double *xo = a.x + 9 * (size_t)I;
    int ci[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        int c = (int)floor(xo[u] / L * nc);
        ci[u] = c < 0 ? 0 : (c >= nc ? nc - 1 : c);
    }
    const int cell = a.rep_cell_off[r] + (ci[2] * nc + ci[1]) * nc + ci[0];
    a.cell_of_mol[I] = cell;
    const double d1 = dist2_fp64(xo, xo + 3, L), d2 = dist2_fp64(xo, xo + 6, L);
    if (d1 > a.rext2 || d2 > a.rext2) atomicOr(a.status, ST_GEOMETRY);
    if (!(d1 <= a.rnear2 && d2 <= a.rnear2)) atomicAdd(a.max_cnt + 1, 1);
    return cell;
}

// Cell of each molecule and the per-cell counts.
__global__ void k_cell_count(NlistArgs a) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= a.M) return;
    atomicAdd(a.cell_cnt + mol_cell(a, I), 1);
}

// The four cell passes (count, scan, fill, sort) in one CTA, for systems of up to
// kCellsOneM molecules in up to kCellsOneC cells: counts, starts and fill cursors in shared
// memory, each pass separated by a barrier.  Same cells, starts and order as the four kernels.
constexpr int kCellsOneM = 8192, kCellsOneC = 4096;

__global__ void __launch_bounds__(1024) k_cells_one(NlistArgs a) {
    extern __shared__ int s_cell[];   // [3][n_cells]: counts, starts, fill cursors
    __shared__ int s_part[1024];
    int *s_cnt = s_cell, *s_start = s_cell + a.n_cells, *s_fill = s_cell + 2 * a.n_cells;
    const int t = threadIdx.x, nt = blockDim.x;
    for (int c = t; c < a.n_cells; c += nt) {
        s_cnt[c] = 0;
        s_fill[c] = 0;
    }
    if (t == 0) a.max_cnt[1] = 0;
    __syncthreads();
    for (int I = t; I < a.M; I += nt) atomicAdd(s_cnt + mol_cell(a, I), 1);
    __syncthreads();
    // exclusive scan: thread t takes the k consecutive cells from t k
    const int k = (a.n_cells + nt - 1) / nt;
    int sum = 0;
    for (int j = 0; j < k; j++) {
        const int c = t * k + j;
        if (c < a.n_cells) sum += s_cnt[c];
    }
    s_part[t] = sum;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        const int v = t >= off ? s_part[t - off] : 0;
        __syncthreads();
        s_part[t] += v;
        __syncthreads();
    }
    int run = s_part[t] - sum;
    for (int j = 0; j < k; j++) {
        const int c = t * k + j;
        if (c < a.n_cells) {
            s_start[c] = run;
            a.cell_start[c] = run;
            a.cell_cnt[c] = s_cnt[c];
            run += s_cnt[c];
        }
    }
    __syncthreads();
    for (int I = t; I < a.M; I += nt) {
        const int c = a.cell_of_mol[I];
        a.cell_tmp[s_start[c] + atomicAdd(s_fill + c, 1)] = I;
    }
    __syncthreads();
    for (int I = t; I < a.M; I += nt) {
        const int c = a.cell_of_mol[I];
        const int s0 = s_start[c], n = s_cnt[c];
        int rank = 0;
        for (int q = 0; q < n; q++) rank += a.cell_tmp[s0 + q] < I;
        a.cell_sorted[s0 + rank] = I;
    }
}

// Exclusive scan of the cell counts (one CTA; cells are few).
__global__ void k_cell_scan(NlistArgs a) {
    __shared__ int s_part[1024];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < a.n_cells; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < a.n_cells ? a.cell_cnt[i] : 0;
        s_part[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < blockDim.x; off <<= 1) {
            const int t = threadIdx.x >= off ? s_part[threadIdx.x - off] : 0;
            __syncthreads();
            s_part[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < a.n_cells) {
            a.cell_start[i] = s_carry + s_part[threadIdx.x] - v;
            a.cell_fill[i] = 0;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry += s_part[threadIdx.x];
        __syncthreads();
    }
}

__global__ void k_cell_fill(NlistArgs a) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= a.M) return;
    const int c = a.cell_of_mol[I];
    a.cell_tmp[a.cell_start[c] + atomicAdd(a.cell_fill + c, 1)] = I;
}

// Order each cell by molecule index, so that the rows are a deterministic
// function of the positions (the forward and reverse passes rebuild identical lists).
__global__ void k_cell_sort(NlistArgs a) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= a.M) return;
    const int c = a.cell_of_mol[I];
    const int s = a.cell_start[c], n = a.cell_cnt[c];
    int rank = 0;
    for (int t = 0; t < n; t++) rank += a.cell_tmp[s + t] < I;
    a.cell_sorted[s + rank] = I;
}

// Rows of the molecules of one home cell (up to eight CTAs of sixteen warps per cell, so
// that a warp has at most one home molecule in all but the fullest cells: the build's time
// is that of its slowest warp).  The CTA stages the neighbourhood -- the members of the
// surrounding cells, in the canonical cell order and index order within a cell -- with all
// three atoms in FP32 in shared memory, in chunks of up to kRowChunk molecules.  Each warp
// takes one home molecule at a time: an FP32 O-O test against the candidate radius (with a
// margin far above FP32 error) selects candidate molecules, an FP32 test classifies each of
// the nine atom pairs as clearly inside / clearly outside the list cutoff, and the few pairs
// within `band` of the cutoff are decided by the exact FP64 Molly arithmetic (dist2_fp64),
// so the set is bit-identical to the all-FP64 test.  Entries are appended in candidate order.
//
// Periodic images.  The FP64 test takes each atom pair's own minimum image.  The FP32 test
// sees whole molecules (each H placed at its O plus the O-H minimum image, as the step
// kernels' gather buffer holds them; the state wraps every atom on its own): the home
// molecule made whole in FP64, the staged candidates in FP32 (within 1e-6 nm of that).  When every O-H
// distance is at most r_near (counted by k_cell_count) and the box side L exceeds
// 2 (rc_nl + 2 r_near) + 0.02 nm, the FP32 test shifts all three atoms of the candidate by
// the image of the O-O vector instead: an atom pair whose own image differs has a component
// beyond L/2 after that shift, so both distances exceed L/2 - 2 r_near > rc_nl + 0.01 nm and
// the pair is outside either way; every other pair gets the same vector up to FP32 rounding
// (|d^2 error| < 5e-6 L/4.5 nm, a quarter of `band`).  The rows are the same bits with
// either form; the shifted form saves the 27 per-component image selections.
constexpr int kRowChunk = 2048;
constexpr int kCandBatch = 256;

__device__ __forceinline__ float mi_f(float d, float L, float hL) {
    return d > hL ? d - L : (d < -hL ? d + L : d);
}

__global__ void __launch_bounds__(512) k_rows(NlistArgs a) {
    extern __shared__ float s_c[];              // [9][kRowChunk] coordinates
    int *s_idx = (int *)(s_c + 9 * kRowChunk);   // [kRowChunk] molecule ids
    __shared__ int s_off[126], s_start[125];
    __shared__ int s_kbuf[16 * kCandBatch];      // per warp: candidates passing the O-O test
    const int c_home = blockIdx.x;
    const int r = a.cell_rep[c_home];
    const int nc = a.rep_nc[r];
    const int off0 = a.rep_cell_off[r];
    const double Ld = a.rep_box[r];
    const float L = (float)Ld, hL = 0.5f * (float)Ld;
    const bool one_image = Ld > a.shift_box && a.max_cnt[1] == 0;
    const int hs = a.cell_start[c_home], hn = a.cell_cnt[c_home];
    // gridDim.y CTAs share a home cell: CTA y takes every gridDim.y-th group of nwarp home
    // molecules (each stages the whole neighbourhood)
    if ((int)blockIdx.y * (int)(blockDim.x >> 5) >= hn) return;
    const int cl = c_home - off0;
    const int cx = cl % nc, cy = (cl / nc) % nc, cz = cl / (nc * nc);
    const int span = nc >= 5 ? 5 : nc;
    const int ncell = span * span * span;
    // neighbourhood cells in canonical order, their member counts and first members,
    // loaded by one thread per cell; the exclusive prefix of the counts in shared memory
    if (threadIdx.x < ncell) {
        const int t = threadIdx.x;
        const int dz = t / (span * span), dy = (t / span) % span, dx = t % span;
        const int z = nc >= 5 ? (cz + dz - 2 + nc) % nc : dz;
        const int y = nc >= 5 ? (cy + dy - 2 + nc) % nc : dy;
        const int x = nc >= 5 ? (cx + dx - 2 + nc) % nc : dx;
        const int c = off0 + (z * nc + y) * nc + x;
        s_off[t + 1] = a.cell_cnt[c];
        s_start[t] = a.cell_start[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s_off[0] = 0;
        for (int t = 1; t <= ncell; t++) s_off[t] += s_off[t - 1];
    }
    __syncthreads();
    const int total = s_off[ncell];
    // the home cell's place in the neighbourhood order (its members are staged in index
    // order there, so home molecule hi is staged candidate s_off[tc] + hi)
    const int tc = nc >= 5 ? (2 * span + 2) * span + 2 : (cz * span + cy) * span + cx;
    const int lane = threadIdx.x & 31;
    const int nwarp = (int)gridDim.y * (int)(blockDim.x >> 5);               // warps per home cell
    const int warp = (int)blockIdx.y * (int)(blockDim.x >> 5) + (threadIdx.x >> 5);
    // an atom pair within rc_nl needs an O-O distance within rc_nl + 2 (largest O-H)
    const float rcand2 = (float)(a.max_cnt[1] == 0 ? a.rcand_near2 : a.rcand2) + 1e-3f;
    const float rc2f = (float)a.rc_nl2;
    const float band = a.band;
    // per home molecule state kept across chunks (a warp owns the same molecules in
    // every chunk: home members warp, warp + nwarp, ...)
    constexpr int kMaxHome = 1;   // home molecules per warp per staging pass (the split gives
                                  // warps for twice the mean count; fuller cells restage)
    for (int h0 = 0; h0 < hn; h0 += nwarp * kMaxHome) {
        int cnt[kMaxHome];
#pragma unroll
        for (int q = 0; q < kMaxHome; q++) cnt[q] = 0;
        for (int c0 = 0; c0 < total; c0 += kRowChunk) {
            const int cn = min(kRowChunk, total - c0);
            __syncthreads();
            for (int k = threadIdx.x; k < cn; k += blockDim.x) {
                const int g = c0 + k;
                // the cell t with s_off[t] <= g < s_off[t + 1]
                int t = 0, t1 = ncell;
                while (t1 - t > 1) {
                    const int mid = (t + t1) >> 1;
                    if (s_off[mid] <= g) t = mid;
                    else t1 = mid;
                }
                const int J = a.cell_sorted[s_start[t] + (g - s_off[t])];
                s_idx[k] = J;
                const double *xj = a.x + 9 * (size_t)J;
#pragma unroll
                for (int u = 0; u < 3; u++) {
                    // whole molecule in FP32: H = O + minimum image of (H - O)
                    const float o = (float)xj[u];
                    s_c[u * kRowChunk + k] = o;
                    s_c[(3 + u) * kRowChunk + k] = o + mi_f((float)xj[3 + u] - o, L, hL);
                    s_c[(6 + u) * kRowChunk + k] = o + mi_f((float)xj[6 + u] - o, L, hL);
                }
            }
            __syncthreads();
#pragma unroll 1
            for (int q = 0; q < kMaxHome; q++) {
                const int hi = h0 + q * nwarp + warp;
                if (hi >= hn) break;
                const int I = a.cell_sorted[hs + hi];
                const int kself = s_off[tc] + hi - c0;   // the home molecule in this chunk
                float xi[9];
#pragma unroll
                for (int u = 0; u < 9; u++)
                    xi[u] = (float)gather_coord(a.x[9 * (size_t)I + u % 3], a.x[9 * (size_t)I + u], u >= 3, Ld);
                uint32_t *row = a.nbr + (size_t)I * a.cap;
                // in batches of kCandBatch candidates: the O-O test first, compacting the
                // passing candidates (in order) for the nine-pair test, so the lanes of the
                // second pass are all busy
                int *s_k = s_kbuf + (threadIdx.x >> 5) * kCandBatch;
                for (int b0 = 0; b0 < cn; b0 += kCandBatch) {
                    const int b1 = min(b0 + kCandBatch, cn);
                    int nk = 0;
                    auto oo_pass = [&](int k) {
                        if (k >= b1) return false;
                        const float ox = mi_f(s_c[k] - xi[0], L, hL);
                        const float oy = mi_f(s_c[kRowChunk + k] - xi[1], L, hL);
                        const float oz = mi_f(s_c[2 * kRowChunk + k] - xi[2], L, hL);
                        return k != kself && ox * ox + oy * oy + oz * oz <= rcand2;
                    };
                    // two candidates per lane per step (independent chains), compacted in order
                    const unsigned below = (1u << lane) - 1u;
                    for (int base = b0; base < b1; base += 64) {
                        const bool p0 = oo_pass(base + lane), p1 = oo_pass(base + 32 + lane);
                        const unsigned bal0 = __ballot_sync(0xffffffffu, p0);
                        const unsigned bal1 = __ballot_sync(0xffffffffu, p1);
                        if (p0) s_k[nk + __popc(bal0 & below)] = base + lane;
                        nk += __popc(bal0);
                        if (p1) s_k[nk + __popc(bal1 & below)] = base + 32 + lane;
                        nk += __popc(bal1);
                    }
                    __syncwarp();
                    for (int base = 0; base < nk; base += 32) {
                        const int idx = base + lane;
                        uint32_t ent = 0;
                        if (idx < nk) {
                            const int k = s_k[idx];
                            const int J = s_idx[k];
                            uint32_t mask = 0, near = 0;
                            float cb[9];
                            if (one_image) {
#pragma unroll
                                for (int u = 0; u < 3; u++) {
                                    const float d = s_c[u * kRowChunk + k] - xi[u];
                                    const float sft = d > hL ? -L : (d < -hL ? L : 0.f);
#pragma unroll
                                    for (int kb = 0; kb < 3; kb++)
                                        cb[3 * kb + u] = s_c[(3 * kb + u) * kRowChunk + k] + sft;
                                }
                            }
#pragma unroll
                            for (int ka = 0; ka < 3; ka++)
#pragma unroll
                                for (int kb = 0; kb < 3; kb++) {
                                    float dx, dy, dz;
                                    if (one_image) {
                                        dx = cb[3 * kb] - xi[3 * ka];
                                        dy = cb[3 * kb + 1] - xi[3 * ka + 1];
                                        dz = cb[3 * kb + 2] - xi[3 * ka + 2];
                                    } else {
                                        dx = mi_f(s_c[(3 * kb) * kRowChunk + k] - xi[3 * ka], L, hL);
                                        dy = mi_f(s_c[(3 * kb + 1) * kRowChunk + k] - xi[3 * ka + 1], L, hL);
                                        dz = mi_f(s_c[(3 * kb + 2) * kRowChunk + k] - xi[3 * ka + 2], L, hL);
                                    }
                                    const float d2 = dx * dx + dy * dy + dz * dz;
                                    mask |= (d2 < rc2f ? 1u : 0u) << (3 * ka + kb);
                                    near |= (fabsf(d2 - rc2f) <= band ? 1u : 0u) << (3 * ka + kb);
                                }
                            // the nine tests above are straight-line code; the rare pairs
                            // within `band` of the cutoff are decided here in FP64
                            while (near) {
                                const int b = __ffs(near) - 1;
                                near &= near - 1u;
                                const bool in = dist2_fp64(a.x + 9 * (size_t)I + 3 * (b / 3),
                                                           a.x + 9 * (size_t)J + 3 * (b % 3), Ld) <= a.rc_nl2;
                                mask = in ? (mask | (1u << b)) : (mask & ~(1u << b));
                            }
                            if (mask) ent = (uint32_t)J | (mask << 23);
                        }
                        const unsigned bal = __ballot_sync(0xffffffffu, ent != 0);
                        if (ent) {
                            const int pos = cnt[q] + __popc(bal & ((1u << lane) - 1u));
                            if (pos < a.cap) row[pos] = ent;
                        }
                        cnt[q] += __popc(bal);
                    }
                    __syncwarp();
                }
            }
        }
#pragma unroll 1
        for (int q = 0; q < kMaxHome; q++) {
            const int hi = h0 + q * nwarp + warp;
            if (hi >= hn) break;
            if (lane == 0) {
                const int I = a.cell_sorted[hs + hi];
                a.nbr_cnt[I] = cnt[q];
                if (cnt[q] > a.cap) atomicOr(a.status, ST_NLIST_OVERFLOW);
                atomicMax(a.max_cnt, cnt[q]);
            }
        }
    }
}

// Half-shell split of the rows.  Row order is the candidate order of k_rows: by the
// neighbourhood position t of the neighbour's cell relative to the row owner's cell (the
// canonical cell index when the grid has fewer than five cells a side), then by molecule
// index.  The key (t << 23) | K is therefore increasing along every row.
__device__ __forceinline__ uint32_t row_key(const NlistArgs &a, int nc, int off0, int cx, int cy, int cz,
                                            int K) {
    const int cl = a.cell_of_mol[K] - off0;
    const int kx = cl % nc, ky = (cl / nc) % nc, kz = cl / (nc * nc);
    int t;
    if (nc >= 5) {
        const int dx = (kx - cx + 2 + nc) % nc, dy = (ky - cy + 2 + nc) % nc, dz = (kz - cz + 2 + nc) % nc;
        t = (dz * 5 + dy) * 5 + dx;
    } else {
        t = cl;
    }
    return ((uint32_t)t << 23) | (uint32_t)K;
}

// Owned entries of each row, compacted in row order to the front of its split row; the
// compact index of each owned entry in ownpos.  One warp per row.
__global__ void k_split_own(NlistArgs a) {
    const int I = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (I >= a.M) return;
    const int n = min(a.nbr_cnt[I], a.cap);
    const uint32_t *row = a.nbr + (size_t)I * a.cap;
    uint32_t *out = a.split + (size_t)I * a.cap;
    int *op = a.ownpos + (size_t)I * a.cap;
    int c = 0;
    for (int base = 0; base < n; base += 32) {
        const int e = base + lane;
        uint32_t ent = 0;
        bool own = false;
        if (e < n) {
            ent = row[e];
            own = half_owns(I, (int)(ent & 0x7FFFFFu));
        }
        const unsigned bal = __ballot_sync(0xffffffffu, own);
        if (own) {
            const int p = c + __popc(bal & ((1u << lane) - 1u));
            out[p] = ent;
            op[e] = p;
        }
        c += __popc(bal);
    }
    if (lane == 0) a.cnt_own[I] = c;
}

// Incoming slots of each row: for every entry I that owns the pair, the slot I * cap + p'
// where I's owned entry of this molecule sits at compact index p' (found by binary search
// on the row key in I's row).  Written from the back of the split row, in row order, so
// that the owned entries (front) and the incoming slots (back) share the row's capacity.
__global__ void k_split_inc(NlistArgs a) {
    const int J = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (J >= a.M) return;
    const int n = min(a.nbr_cnt[J], a.cap);
    const uint32_t *row = a.nbr + (size_t)J * a.cap;
    uint32_t *out = a.split + (size_t)J * a.cap + (a.cap - 1);
    const int r = a.mol_rep[J];
    const int nc = a.rep_nc[r], off0 = a.rep_cell_off[r];
    int c = 0;
    for (int base = 0; base < n; base += 32) {
        const int e = base + lane;
        bool inc = false;
        uint32_t slot = 0;
        if (e < n) {
            const int I = (int)(row[e] & 0x7FFFFFu);
            if (!half_owns(J, I)) {
                inc = true;
                const int cl = a.cell_of_mol[I] - off0;
                const int cx = cl % nc, cy = (cl / nc) % nc, cz = cl / (nc * nc);
                const uint32_t target = row_key(a, nc, off0, cx, cy, cz, J);
                const uint32_t *ri = a.nbr + (size_t)I * a.cap;
                const int ni = min(a.nbr_cnt[I], a.cap);
                int lo = 0, hi = ni;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (row_key(a, nc, off0, cx, cy, cz, (int)(ri[mid] & 0x7FFFFFu)) < target) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < ni && (int)(ri[lo] & 0x7FFFFFu) == J) {
                    slot = (uint32_t)((size_t)I * a.cap + a.ownpos[(size_t)I * a.cap + lo]);
                } else {
                    atomicOr(a.status, ST_ROW_ASYM);
                    slot = (uint32_t)((size_t)I * a.cap);   // a valid slot; the status fails the call
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, inc);
        if (inc) out[-(c + __popc(bal & ((1u << lane) - 1u)))] = slot;
        c += __popc(bal);
    }
    if (lane == 0) a.cnt_inc[J] = c;
}

// Atom pairs (i < j, replica-local indices) of one replica's rows.
__global__ void k_export_pairs(const uint32_t *nbr, const int *nbr_cnt, int cap, int mol0,
                               int nmol, int32_t *pairs, unsigned long long *count,
                               long long max_pairs) {
    const int I = blockIdx.y * gridDim.x + blockIdx.x;
    if (I >= nmol) return;
    const int Ig = mol0 + I;
    const int n = min(nbr_cnt[Ig], cap);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const uint32_t ent = nbr[(size_t)Ig * cap + e];
        const int J = (int)(ent & 0x7FFFFFu) - mol0;
        if (J <= I) continue;
        const uint32_t mask = ent >> 23;
        for (int b = 0; b < 9; b++) {
            if (!((mask >> b) & 1u)) continue;
            const unsigned long long k = atomicAdd(count, 1ull);
            if ((long long)k < max_pairs) {
                pairs[2 * k] = 3 * I + b / 3;
                pairs[2 * k + 1] = 3 * J + b % 3;
            }
        }
    }
}

}  // namespace

cudaError_t launch_nlist(const NlistArgs &a, cudaStream_t st, int *n_kernels) {
    int nk = 0;
    if (a.M <= kCellsOneM && a.n_cells <= kCellsOneC) {
        k_cells_one<<<1, 1024, 3 * sizeof(int) * a.n_cells, st>>>(a);
        nk += 1;
    } else {
        cudaMemsetAsync(a.cell_cnt, 0, sizeof(int) * a.n_cells, st);
        cudaMemsetAsync(a.max_cnt + 1, 0, sizeof(int), st);
        const int t = 256, b = (a.M + t - 1) / t;
        k_cell_count<<<b, t, 0, st>>>(a);
        k_cell_scan<<<1, 1024, 0, st>>>(a);
        k_cell_fill<<<b, t, 0, st>>>(a);
        k_cell_sort<<<b, t, 0, st>>>(a);
        nk += 4;
    }
    const size_t smem = (9 * sizeof(float) + sizeof(int)) * kRowChunk;
    cudaFuncSetAttribute(k_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // home molecules per cell over the 16 warps of a CTA: split a cell over up to 8 CTAs,
    // with warps for twice the mean count, so that the fullest cells of a Poisson-like
    // occupancy still give a warp one home molecule (CTAs beyond a cell's count exit at once)
    const int per_cell = (a.M + a.n_cells - 1) / a.n_cells;
    const int split = std::min(8, std::max(1, (2 * per_cell + 15) / 16));
    k_rows<<<dim3(a.n_cells, split), 512, smem, st>>>(a);
    nk += 1;
    if (a.split) {
        const int wb = (a.M + 7) / 8;   // one warp per row, eight per CTA
        k_split_own<<<wb, 256, 0, st>>>(a);
        k_split_inc<<<wb, 256, 0, st>>>(a);
        nk += 2;
    }
    if (n_kernels) *n_kernels = nk;
    return cudaGetLastError();
}

cudaError_t launch_export_pairs(const uint32_t *nbr, const int *nbr_cnt, int cap, int mol0,
                                int nmol, int32_t *pairs, unsigned long long *count,
                                long long max_pairs, cudaStream_t st) {
    if (nmol <= 0) return cudaSuccess;
    const int gx = nmol < 65535 ? nmol : 65535;
    const int gy = (nmol + gx - 1) / gx;
    k_export_pairs<<<dim3(gx, gy), 128, 0, st>>>(nbr, nbr_cnt, cap, mol0, nmol, pairs, count,
                                                 max_pairs);
    return cudaGetLastError();
}

}  // namespace rs
