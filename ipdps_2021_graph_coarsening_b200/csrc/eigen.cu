// eigen.cu -- Fiedler-vector power iteration of one level.
//
// Reference: cmg/eigensolve_kokkos.h:102-206 (sgp_power_iter, normLap = 0):
//   d = rowsum(A); gb = max(2 d_i, 2); u -= (u.1^)1^; u /= |u|; v = u
//   while |dot - lastDot| > tol && iter < 1e14 / n:
//     u = v; y = A u; v = (gb - d) u + y; v -= (v.1^)1^; v /= |v|; dot = u.v
// and eigensolve_kokkos.h:1556-1559 (prolongation fine[i] = coarse[vcmap[i]]).
//
// One persistent cooperative kernel runs every iteration of a level.  The
// deflation, normalisation and dot product are folded into the SpMV pass:
// the pass stores the raw iterate r = (gb - d) u + A u and accumulates
// S1 = sum r, S2 = sum r^2, S3 = sum u r, S4 = sum u, S5 = sum u^2; then
//   mu = S1 / n, |r - mu|^2 = S2 - mu S1, dot = (S3 - mu S4) / |r - mu|
// and the next pass reads u_j = (r_j - mu) / |r - mu| on the fly.  One grid
// barrier per iteration; the reference issues ~8 kernels and 4 reductions.
// Per-block partial sums are combined in a fixed order, so results are
// reproducible run to run.
//
// Rows are processed by groups of G lanes (G from the level's mean degree);
// rows longer than the heavy threshold by a whole block.  V is the vector
// storage type: double (plain FP64) or float (mixed precision: FP32 storage,
// gathers and row sums; FP64 reductions, deflation and normalisation).
#include <math.h>
#include <string.h>

#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kPIThreads = 512;
constexpr int kNP = 5;

struct PIArgs {
    uint32_t n;
    const uint32_t *rp;
    const uint32_t *col;
    const void *w;
    const uint32_t *heavy;        // rows with degree > heavy_T, ascending
    const uint32_t *n_heavy_ptr;
    uint32_t heavy_T;
    const uint32_t *cpre;         // [n+1] prefix of per-row cost (0 for heavy rows): warp row ranges
    const uint32_t *cpre_all;     // [n+1] prefix of per-row cost of all rows: block row ranges
    const double *x_in;
    const uint32_t *vcmap;
    void *va;
    void *vb;
    double *out;
    double *partials;             // [2][gridDim][kNP]
    double tol;
    uint64_t iter_max;
    double stall_factor;          // > 0: stop when |d dot| has not improved by this factor in stall_window iterations
    uint32_t stall_window;
    double *res;                  // [0] niter [1] dot [2] gb [3] lambda [4] capped [5] stalled
};

__device__ __forceinline__ void grid_barrier(cg::grid_group &g) {
    if (gridDim.x == 1) __syncthreads();
    else g.sync();
}

template <typename V>
__device__ __forceinline__ double vld(const V *p, uint32_t i) { return (double)p[i]; }

// reduce per-block partials (all blocks compute the same totals, same order)
__device__ __forceinline__ void reduce_partials(const double *part, double (&S)[kNP], double *sm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (wid == 0) {
        double acc[kNP];
#pragma unroll
        for (int k = 0; k < kNP; k++) acc[k] = 0;
        for (uint32_t b = lane; b < gridDim.x; b += 32)
#pragma unroll
            for (int k = 0; k < kNP; k++) acc[k] += part[(size_t)b * kNP + k];
#pragma unroll
        for (int k = 0; k < kNP; k++) acc[k] = warp_sum(acc[k]);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < kNP; k++) sm[k] = acc[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kNP; k++) S[k] = sm[k];
    __syncthreads();
}

// Weighted degree of row i (sum of weights; row length for unit weights).
template <int G, typename W>
__device__ __forceinline__ double row_degree_group(const PIArgs &a, uint32_t i, uint32_t lane, unsigned gm) {
    const uint32_t b = a.rp[i], e = a.rp[i + 1];
    const W *w = (const W *)a.w;
    if (!w) return (double)(e - b);
    uint64_t s = 0;
    for (uint32_t j = b + lane; j < e; j += G) s += (uint64_t)__ldg(w + j);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(gm, s, o);
    return (double)s;
}

// acc += sum_j w_j src[col_j] and dsum += sum_j w_j over j = j0, j0 + s, ... < e.
// Four entries per lane are in flight (destination loads, weight loads, then
// the four gathers), so a warp keeps 4x the memory requests outstanding of a
// one-at-a-time loop; the summation order is fixed for a given stride.
template <typename W, typename V, typename ACC>
__device__ __forceinline__ void row_accum(const uint32_t *__restrict__ col, const W *__restrict__ w, const V *src,
                                          uint32_t j, uint32_t e, uint32_t s, ACC &acc, uint64_t &dsum) {
    // every trip issues up to four predicated entries, the last partial trip
    // included, so a row costs ceil(len / 4s) dependent-load rounds
    if (w) {
        for (; j < e; j += 4 * s) {
            const bool p1 = j + s < e, p2 = j + 2 * s < e, p3 = j + 3 * s < e;
            const uint32_t c0 = __ldg(col + j);
            const uint32_t c1 = p1 ? __ldg(col + j + s) : 0u;
            const uint32_t c2 = p2 ? __ldg(col + j + 2 * s) : 0u;
            const uint32_t c3 = p3 ? __ldg(col + j + 3 * s) : 0u;
            const W w0 = __ldg(w + j);
            const W w1 = p1 ? __ldg(w + j + s) : (W)0;
            const W w2 = p2 ? __ldg(w + j + 2 * s) : (W)0;
            const W w3 = p3 ? __ldg(w + j + 3 * s) : (W)0;
            const V x0 = src[c0];
            const V x1 = p1 ? src[c1] : (V)0;
            const V x2 = p2 ? src[c2] : (V)0;
            const V x3 = p3 ? src[c3] : (V)0;
            acc += (ACC)((V)w0 * x0);
            acc += (ACC)((V)w1 * x1);
            acc += (ACC)((V)w2 * x2);
            acc += (ACC)((V)w3 * x3);
            dsum += (uint64_t)w0 + (uint64_t)w1 + (uint64_t)w2 + (uint64_t)w3;
        }
    } else {
        for (; j < e; j += 4 * s) {
            const bool p1 = j + s < e, p2 = j + 2 * s < e, p3 = j + 3 * s < e;
            const uint32_t c0 = __ldg(col + j);
            const uint32_t c1 = p1 ? __ldg(col + j + s) : 0u;
            const uint32_t c2 = p2 ? __ldg(col + j + 2 * s) : 0u;
            const uint32_t c3 = p3 ? __ldg(col + j + 3 * s) : 0u;
            const V x0 = src[c0];
            const V x1 = p1 ? src[c1] : (V)0;
            const V x2 = p2 ? src[c2] : (V)0;
            const V x3 = p3 ? src[c3] : (V)0;
            acc += (ACC)x0;
            acc += (ACC)x1;
            acc += (ACC)x2;
            acc += (ACC)x3;
        }
    }
}

// first index i in [lo, hi] with pre[i] >= t (pre non-decreasing)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *pre, uint32_t lo, uint32_t hi, uint64_t t) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if ((uint64_t)pre[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <int G>
__device__ __forceinline__ unsigned pi_group_mask() {
    if (G == 32) return 0xFFFFFFFFu;
    const unsigned lane = threadIdx.x & 31;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
}

// block-wide deterministic sum of two values, result broadcast to all threads
__device__ __forceinline__ void block_sum2(double &x, double &y, double *sm) {
    double v[2] = {x, y};
    block_sum_d<2>(v, sm);
    if (threadIdx.x == 0) { sm[200] = v[0]; sm[201] = v[1]; }
    __syncthreads();
    x = sm[200];
    y = sm[201];
    __syncthreads();
}

template <int G, typename W, typename V>
__global__ void __launch_bounds__(kPIThreads, 2) k_power_iter(PIArgs a) {
    cg::grid_group grid = cg::this_grid();
    // [0, 160): block_sum_d scratch (5 x 32), [200, 202): broadcast, [210, 226): warp maxima
    __shared__ double sm[256];
    const uint32_t n = a.n;
    const W *w = (const W *)a.w;
    const unsigned gm = pi_group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    const uint32_t n_heavy = *a.n_heavy_ptr;
    const uint32_t T = a.heavy_T;
    // Work split, fixed for the whole launch: block b owns the rows whose
    // cost prefix (all rows) starts in the b-th equal share; inside the block,
    // heavy rows are processed by all threads and the remaining rows are cut
    // into equal-cost contiguous ranges, one per warp.
    const uint64_t call = a.cpre_all[n];
    const uint32_t B0 = lower_bound_u32(a.cpre_all, 0, n, call * blockIdx.x / gridDim.x);
    const uint32_t B1 = blockIdx.x + 1 == gridDim.x ? n
                                                    : lower_bound_u32(a.cpre_all, 0, n, call * (blockIdx.x + 1) / gridDim.x);
    const uint32_t h0 = lower_bound_u32(a.heavy, 0, n_heavy, B0);
    const uint32_t h1 = lower_bound_u32(a.heavy, 0, n_heavy, B1);
    const uint32_t wk = threadIdx.x >> 5, nwk = blockDim.x >> 5;
    const uint64_t clo = a.cpre[B0], chi = a.cpre[B1];
    const uint32_t w_r0 = lower_bound_u32(a.cpre, B0, B1, clo + (chi - clo) * wk / nwk);
    const uint32_t w_r1 = wk + 1 == nwk ? B1 : lower_bound_u32(a.cpre, B0, B1, clo + (chi - clo) * (wk + 1) / nwk);
    V *va = (V *)a.va, *vb = (V *)a.vb;
    double *part0 = a.partials, *part1 = a.partials + (size_t)gridDim.x * kNP;

    // ---- phase 0a: prolongate / load the start vector, weighted degrees
    double p_sum = 0, p_maxd = 0;
    for (uint64_t i64 = gid; i64 < n; i64 += ngroups) {
        const uint32_t i = (uint32_t)i64;
        const uint32_t deg = a.rp[i + 1] - a.rp[i];
        double d = deg > T ? 0.0 : row_degree_group<G, W>(a, i, lane, gm);
        if (lane == 0) {
            double x = a.vcmap ? a.x_in[a.vcmap[i]] : a.x_in[i];
            V xs = (V)x;
            va[i] = xs;
            p_sum += (double)xs;
            if (deg <= T && d > p_maxd) p_maxd = d;
        }
    }
    for (uint32_t h = blockIdx.x; h < n_heavy; h += gridDim.x) {
        const uint32_t i = a.heavy[h];
        const uint32_t b = a.rp[i], e = a.rp[i + 1];
        double d;
        if (!w) {
            d = (double)(e - b);
        } else {
            double s = 0;
            for (uint32_t j = b + threadIdx.x; j < e; j += blockDim.x) s += (double)__ldg(w + j);
            double z = 0;
            block_sum2(s, z, sm);
            d = s;
        }
        if (threadIdx.x == 0 && d > p_maxd) p_maxd = d;
    }
    {
        double v2[2] = {p_sum, 0};
        block_sum_d<2>(v2, sm);
        double mx = warp_max(p_maxd);
        if ((threadIdx.x & 31) == 0) sm[210 + (threadIdx.x >> 5)] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) m = sm[210 + k] > m ? sm[210 + k] : m;
            part0[(size_t)blockIdx.x * kNP + 0] = v2[0];
            part0[(size_t)blockIdx.x * kNP + 1] = m;
        }
    }
    grid_barrier(grid);
    double S1 = 0, maxd = 0;
    {
        const int lane32 = threadIdx.x & 31;
        if (threadIdx.x < 32) {
            double s = 0, m = 0;
            for (uint32_t b = lane32; b < gridDim.x; b += 32) {
                s += part0[(size_t)b * kNP + 0];
                double x = part0[(size_t)b * kNP + 1];
                m = x > m ? x : m;
            }
            s = warp_sum(s);
            m = warp_max(m);
            if (lane32 == 0) { sm[0] = s; sm[1] = m; }
        }
        __syncthreads();
        S1 = sm[0];
        maxd = sm[1];
        __syncthreads();
    }
    double gb = 2.0 * maxd;
    if (gb < 2.0) gb = 2.0;
    double mu = S1 / (double)n;
    // ---- phase 0b: norm of the deflated start vector
    double p_sq = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        double x = (double)va[i] - mu;
        p_sq += x * x;
    }
    {
        double v2[2] = {p_sq, 0};
        block_sum_d<2>(v2, sm);
        if (threadIdx.x == 0) part1[(size_t)blockIdx.x * kNP + 0] = v2[0];
    }
    grid_barrier(grid);
    double inv_nu;
    {
        if (threadIdx.x < 32) {
            double s = 0;
            for (uint32_t b = threadIdx.x; b < gridDim.x; b += 32) s += part1[(size_t)b * kNP + 0];
            s = warp_sum(s);
            if (threadIdx.x == 0) sm[0] = s;
        }
        __syncthreads();
        inv_nu = 1.0 / sqrt(sm[0]);
        __syncthreads();
    }

    // ---- iterations
    double dot = 0, last = 1;
    double best_delta = 1e300;
    uint64_t best_at = 0;
    uint64_t niter = 0;
    int stalled = 0;
    V *src = va, *dst = vb;
    while (true) {
        if (!(fabs(dot - last) > a.tol && niter < a.iter_max)) break;
        if (a.stall_factor > 0 && niter > 2 && niter - best_at > a.stall_window) { stalled = 1; break; }
        double P[kNP] = {0, 0, 0, 0, 0};
        // normal rows: this warp's cost-balanced contiguous range, G lanes per row
        for (uint32_t i = w_r0 + (threadIdx.x & 31) / G; i < w_r1; i += 32 / G) {
            const uint32_t b = a.rp[i], e = a.rp[i + 1];
            if (e - b > T) continue;   // group-uniform
            V acc = 0;
            uint64_t dsum = 0;
            row_accum<W, V, V>(a.col, w, src, b + lane, e, G, acc, dsum);
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) {
                acc += __shfl_xor_sync(gm, acc, o);
                if (w) dsum += __shfl_xor_sync(gm, dsum, o);
            }
            if (lane == 0) {
                const double d = w ? (double)dsum : (double)(e - b);
                const double ui = ((double)src[i] - mu) * inv_nu;
                const double r = (gb - d) * ui + ((double)acc - mu * d) * inv_nu;
                const V rs = (V)r;
                dst[i] = rs;
                const double rd = (double)rs;
                P[0] += rd; P[1] += rd * rd; P[2] += ui * rd; P[3] += ui; P[4] += ui * ui;
            }
        }
        // heavy rows of this block's range: all threads on one row
        for (uint32_t h = h0; h < h1; h++) {
            const uint32_t i = a.heavy[h];
            const uint32_t b = a.rp[i], e = a.rp[i + 1];
            double acc = 0;
            uint64_t dsum_i = 0;
            row_accum<W, V, double>(a.col, w, src, b + threadIdx.x, e, blockDim.x, acc, dsum_i);
            double dsum = (double)dsum_i;   // exact: weighted degrees stay below 2^53
            block_sum2(acc, dsum, sm);
            if (threadIdx.x == 0) {
                const double d = w ? dsum : (double)(e - b);
                const double ui = ((double)src[i] - mu) * inv_nu;
                const double r = (gb - d) * ui + (acc - mu * d) * inv_nu;
                const V rs = (V)r;
                dst[i] = rs;
                const double rd = (double)rs;
                P[0] += rd; P[1] += rd * rd; P[2] += ui * rd; P[3] += ui; P[4] += ui * ui;
            }
        }
        block_sum_d<kNP>(P, sm);
        double *part = (niter & 1) ? part1 : part0;
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < kNP; k++) part[(size_t)blockIdx.x * kNP + k] = P[k];
        grid_barrier(grid);
        double S[kNP];
        reduce_partials(part, S, sm);
        const double mu_n = S[0] / (double)n;
        const double nsq = S[1] - mu_n * S[0];
        const double inv_nu_n = 1.0 / sqrt(nsq);
        last = dot;
        dot = (S[2] - mu_n * S[3]) * inv_nu_n;
        niter++;
        const double delta = fabs(dot - last);
        if (niter > 2 && delta < best_delta * a.stall_factor) { best_delta = delta; best_at = niter; }
        if (!(fabs(dot - last) > a.tol && niter < a.iter_max) ||
            (a.stall_factor > 0 && niter > 2 && niter - best_at > a.stall_window)) {
            // the reference returns u of the last iteration: (src - mu) / nu
            for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
                 i += (uint64_t)gridDim.x * blockDim.x)
                a.out[i] = ((double)src[i] - mu) * inv_nu;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                a.res[0] = (double)niter;
                a.res[1] = dot;
                a.res[2] = gb;
                a.res[3] = (gb * S[4] - S[2]) / S[4];
                a.res[4] = niter >= a.iter_max ? 1.0 : 0.0;
                a.res[5] = (fabs(dot - last) > a.tol && niter < a.iter_max) ? 1.0 : 0.0;
            }
            return;
        }
        mu = mu_n;
        inv_nu = inv_nu_n;
        V *t = src; src = dst; dst = t;
    }
    // loop exit before any iteration (not reachable: |0 - 1| > tol)
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        a.out[i] = ((double)src[i] - mu) * inv_nu;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.res[0] = (double)niter; a.res[1] = dot; a.res[2] = gb; a.res[3] = 0; a.res[4] = 0;
        a.res[5] = stalled;
    }
}

// ----------------------------------------------------------- residual --
// |L x - lambda x|^2 partial sums per block (x unit-norm FP64 vector).
template <typename W>
__global__ void __launch_bounds__(256) k_residual(uint32_t n, const uint32_t *__restrict__ rp,
                                                 const uint32_t *__restrict__ col, const W *__restrict__ w,
                                                 const double *__restrict__ x, double lambda, double *part) {
    __shared__ double sm[96];
    double s[2] = {0, 0};
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = wid; i < n; i += nw) {
        double acc = 0, d = 0;
        for (uint32_t j = rp[i] + lane; j < rp[i + 1]; j += 32) {
            double wt = w ? (double)w[j] : 1.0;
            acc += wt * x[col[j]];
            d += wt;
        }
        acc = warp_sum(acc);
        d = warp_sum(d);
        if (lane == 0) {
            double r = d * x[i] - acc - lambda * x[i];
            s[0] += r * r;
            s[1] += x[i] * x[i];
        }
    }
    block_sum_d<2>(s, sm);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = s[0]; part[2 * blockIdx.x + 1] = s[1]; }
}

__global__ void k_sum_pairs(const double *part, uint32_t nb, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0, b = 0;
        for (uint32_t i = 0; i < nb; i++) { a += part[2 * i]; b += part[2 * i + 1]; }
        out[0] = a; out[1] = b;
    }
}

__global__ void k_heavy_flags(uint32_t n, const uint32_t *rp, uint32_t T, uint8_t *f) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = (rp[i + 1] - rp[i]) > T ? 1 : 0;
}

// per-row cost used to give every warp an equal share: entries plus a fixed
// row overhead; heavy rows (handled by whole blocks) cost nothing here
__global__ void k_row_cost(uint32_t n, const uint32_t *rp, uint32_t T, uint32_t shift, uint32_t *cost,
                           uint32_t *cost_all) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t len = rp[i + 1] - rp[i];
    uint32_t c = ((len + 8u) >> shift) + 1u;
    cost[i] = len > T ? 0u : c;
    cost_all[i] = c;
}

static int pi_lanes(double avg) { return avg <= 4 ? 4 : avg <= 8 ? 8 : avg <= 16 ? 16 : 32; }

static uint32_t pi_grid(const Context &C, uint32_t n, int G) {
    const uint64_t maxg = (uint64_t)2 * C.num_sms;   // two resident blocks per SM (launch bounds)
    const uint64_t want = cdiv((uint64_t)n * G, kPIThreads * 4ull);
    uint32_t grid = (uint32_t)(want < maxg ? want : maxg);
    return grid < 1 ? 1 : grid;
}

template <int G, typename W, typename V>
static int launch_pi(Context &C, PIArgs &a, uint32_t grid) {
    const void *k = (const void *)k_power_iter<G, W, V>;
    int per_sm = 0;
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kPIThreads, 0));
    if (per_sm < 1) {
        set_error("power-iteration kernel does not fit on an SM");
        return SGP_B200_ERR_DEVICE;
    }
    if ((uint64_t)grid > (uint64_t)per_sm * C.num_sms) grid = per_sm * C.num_sms;
    SGPB_TRY(dalloc_t(C, &a.partials, (size_t)2 * grid * kNP));
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kPIThreads), args, 0, C.stream));
    C.kernel_launches++;
    return SGP_B200_OK;
}

template <typename W, typename V>
static int launch_pi_w(Context &C, PIArgs &a, int G, uint32_t grid) {
    if (G == 4) return launch_pi<4, W, V>(C, a, grid);
    if (G == 8) return launch_pi<8, W, V>(C, a, grid);
    if (G == 16) return launch_pi<16, W, V>(C, a, grid);
    return launch_pi<32, W, V>(C, a, grid);
}

static int run_pi(Context &C, const Level &L, PIArgs a, int mixed, double *res_d, double res_h[6], float *ms) {
    const int G = pi_lanes(L.n ? (double)L.m / L.n : 0);
    const uint32_t grid = pi_grid(C, L.n, G);
    a.res = res_d;
    int rc;
    cudaEvent_t e0, e1;
    SGPB_CUDA(cudaEventCreate(&e0));
    SGPB_CUDA(cudaEventCreate(&e1));
    // partials are allocated inside launch_pi; the events bracket the launch only
    SGPB_CUDA(cudaEventRecord(e0, C.stream));
    if (mixed) {
        float *va, *vb;
        SGPB_TRY(dalloc_t(C, &va, L.n));
        SGPB_TRY(dalloc_t(C, &vb, L.n));
        a.va = va; a.vb = vb;
        if (L.wbytes == 8) rc = launch_pi_w<unsigned long long, float>(C, a, G, grid);
        else rc = launch_pi_w<uint32_t, float>(C, a, G, grid);
    } else {
        double *va, *vb;
        SGPB_TRY(dalloc_t(C, &va, L.n));
        SGPB_TRY(dalloc_t(C, &vb, L.n));
        a.va = va; a.vb = vb;
        if (L.wbytes == 8) rc = launch_pi_w<unsigned long long, double>(C, a, G, grid);
        else rc = launch_pi_w<uint32_t, double>(C, a, G, grid);
    }
    cudaEventRecord(e1, C.stream);
    if (rc != SGP_B200_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
    SGPB_CUDA(cudaGetLastError());
    SGPB_CUDA(cudaMemcpyAsync(C.h_pinned, res_d, 6 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    memcpy(res_h, C.h_pinned, 6 * sizeof(double));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms += t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return SGP_B200_OK;
}

int power_iter_level(Context &C, const Level &L, const double *x_in, const uint32_t *vcmap, double *x_out,
                     const PowerIterOpts &o, PowerIterResult *res, int want_residual) {
    const uint32_t n = L.n;
    if (n == 0) { *res = PowerIterResult(); return SGP_B200_OK; }
    const double avg = (double)L.m / n;
    PIArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n; a.rp = L.rp; a.col = L.col; a.w = L.w;
    // Rows longer than one warp's share of the entries (and than 64 G) are
    // processed by a whole block; the rest are split into cost-balanced
    // contiguous ranges, one per warp.
    const int G = pi_lanes(avg);
    const uint64_t nwarps = (uint64_t)pi_grid(C, n, G) * (kPIThreads / 32);
    uint64_t T = L.m / nwarps;
    if (T < 64ull * G) T = 64ull * G;
    if (T > 0xFFFFFFFFull) T = 0xFFFFFFFFull;
    a.heavy_T = (uint32_t)T;
    uint8_t *flags;
    uint32_t *heavy, *nh, *cost, *cpre, *cost_all, *cpre_all;
    SGPB_TRY(dalloc_t(C, &flags, n));
    SGPB_TRY(dalloc_t(C, &heavy, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &nh, 1));
    SGPB_TRY(dalloc_t(C, &cost, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &cpre, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &cost_all, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &cpre_all, (size_t)n + 1));
    k_heavy_flags<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, a.heavy_T, flags);
    const uint32_t shift = (L.m + 9ull * n < 0xFFFFFFF0ull) ? 0u : 4u;   // keep the cost total in 32 bits
    k_row_cost<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, a.heavy_T, shift, cost, cost_all);
    C.kernel_launches += 2;
    SGPB_TRY(compact_flags(C, flags, n, heavy, nh));
    SGPB_TRY(scan_u32(C, cost, cpre, n, nullptr));
    SGPB_TRY(scan_u32(C, cost_all, cpre_all, n, nullptr));
    a.heavy = heavy; a.n_heavy_ptr = nh; a.cpre = cpre; a.cpre_all = cpre_all;
    a.x_in = x_in; a.vcmap = vcmap; a.out = x_out;
    // the reference's cap (eigensolve_kokkos.h:153) is 1e14 / n, unbounded in
    // practice for small levels; a default budget of 5e6 iterations turns a
    // non-converging level into a reported cap instead of an endless kernel.
    uint64_t imax = 100000000000000ULL / (uint64_t)n;
    const uint64_t cap = o.iter_cap ? o.iter_cap : 5000000ULL;
    if (imax > cap) imax = cap;
    a.iter_max = imax;
    a.tol = o.tol;
    double *res_d;
    SGPB_TRY(dalloc_t(C, &res_d, 8));
    double rh[6];
    float kms = 0;
    uint64_t total_iters = 0;
    // Mixed precision: FP32 vector storage and gathers under the reference's
    // stopping rule.  When |d dot| stops shrinking before reaching tol (the
    // FP32 noise floor), the FP32 iterate seeds FP64 iterations that finish
    // the level at the requested tolerance.  Levels below 4096 vertices are
    // latency-bound and run in FP64 directly.
    bool done = false;
    if (o.mixed && n >= 4096) {
        a.stall_factor = 0.5;
        a.stall_window = 64;
        SGPB_TRY(run_pi(C, L, a, 1, res_d, rh, &kms));
        total_iters += (uint64_t)rh[0];
        done = rh[5] == 0.0;
        a.x_in = x_out;
        a.vcmap = nullptr;
        a.stall_factor = 0;
        a.iter_max = imax > total_iters ? imax - total_iters : 1;
    }
    if (!done) {
        SGPB_TRY(run_pi(C, L, a, 0, res_d, rh, &kms));
        total_iters += (uint64_t)rh[0];
    }
    res->niter = total_iters;
    res->dot = rh[1];
    res->gb = rh[2];
    res->lambda = rh[3];
    res->capped = rh[4] != 0.0;
    res->resid = 0;
    res->kernel_ms = kms;
    if (want_residual) {
        uint32_t nb = C.num_sms * 4;
        double *part, *out2;
        SGPB_TRY(dalloc_t(C, &part, 2 * (size_t)nb));
        SGPB_TRY(dalloc_t(C, &out2, 2));
        if (L.wbytes == 8)
            k_residual<unsigned long long><<<nb, 256, 0, C.stream>>>(n, L.rp, L.col, (const unsigned long long *)L.w,
                                                                     x_out, res->lambda, part);
        else
            k_residual<uint32_t><<<nb, 256, 0, C.stream>>>(n, L.rp, L.col, (const uint32_t *)L.w, x_out, res->lambda,
                                                           part);
        k_sum_pairs<<<1, 32, 0, C.stream>>>(part, nb, out2);
        C.kernel_launches += 2;
        SGPB_CUDA(cudaGetLastError());
        SGPB_CUDA(cudaMemcpyAsync(C.h_pinned, out2, 2 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
        SGPB_CUDA(cudaStreamSynchronize(C.stream));
        double r2 = ((double *)C.h_pinned)[0], x2 = ((double *)C.h_pinned)[1];
        res->resid = sqrt(r2 / (x2 > 0 ? x2 : 1)) / (res->gb > 0 ? res->gb : 1);
    }
    return SGP_B200_OK;
}

}  // namespace sgpb
