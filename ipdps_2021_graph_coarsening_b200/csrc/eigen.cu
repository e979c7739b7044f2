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
// SpMV mapping.  Block b owns an equal share of the rows' cost (entries plus
// a per-row overhead).  Inside the block, rows longer than one warp's share
// (and empty rows) are processed by all threads; the other rows are cut into
// equal-cost contiguous ranges, one per warp, and each warp streams its
// entries in tiles of 128 (four consecutive entries per lane, 16-byte vector
// loads of destinations and weights), recovers row ids from a window of row
// offsets in shared memory, and combines rows across lanes with a segmented
// warp scan.  Every lane carries four entries whatever the row lengths, so
// short-row graphs (grids, the finest R-MAT level) stream as well as dense
// coarse levels.
//
// Precision.  The iterate is stored and gathered in FP64 (V = double).  MX
// selects the SpMV arithmetic: false -- FP64 row sums of w_ij x_j (plain);
// true -- mixed precision: the Laplacian is applied in edge-difference form,
// (L x)_i = sum_j w_ij (x_i - x_j), each difference rounded to FP32 and the
// products and row sums formed in FP32, while the shift gb u_i, the
// deflation, the normalisation, the dot product and the stopping test stay
// FP64.  The FP32 rounding then scales with |x_i - x_j| instead of with the
// shifted iterate (about gb |u_i|), which keeps the mixed recurrence on the
// FP64 trajectory: an FP32-stored iterate would add a relative noise of
// about 6e-8 per element and iteration, and the shifted power iteration
// amplifies such noise by roughly gb / (lambda_3 - lambda_2).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kPIThreads = 512;
constexpr int kPIWarps = kPIThreads / 32;
constexpr int kNP = 5;
constexpr int kTile = 128;        // entries per warp tile
constexpr int kWin = kTile + 1;   // row offsets per window

struct PIArgs {
    uint32_t n;
    uint64_t m;
    const uint32_t *rp;
    const uint32_t *col;
    const void *w;
    int vec_ok;                   // col / w 16-byte aligned: vector loads allowed
    const uint32_t *heavy;        // rows handled block-wide (long or empty), ascending
    const uint32_t *n_heavy_ptr;
    uint32_t heavy_T;
    const uint32_t *hseg;         // [n+1] prefix of the segment counts of block-wide rows (0 for the others)
    const uint32_t *seg_row;      // row of each segment
    double *hpart;                // sum of each segment
    uint32_t seg_shift;           // segments of 2^seg_shift entries
    const uint32_t *cpre;         // [n+1] prefix of per-row cost, heavy rows 0: warp ranges
    const uint32_t *cpre_all;     // [n+1] prefix of per-row cost of all rows: block ranges
    double *deg;                  // [n] weighted degree (written in phase 0)
    const double *x_in;
    const uint32_t *vcmap;
    void *va;
    void *vb;
    double *out;
    double *partials;             // [2][gridDim][kNP]
    double tol;
    uint64_t iter_max;
    double *res;                  // [0] niter [1] dot [2] gb [3] lambda [4] capped
    const uint32_t *inv;          // relabelled copy: new id -> level vertex id (null: identity)
    uint32_t kcache;              // leading iterate entries: shared-memory copy, or the L1 hub prefix
    int cache_ok;                 // host: 2 shared-memory copy when it fits, 3 L1 hub prefix, 0 none
    int normlap;                  // refine_alg 1: lazy random walk (I + D^-1 A) / 2, no deflation in the loop
    // column panels (mode 6): the warp rows' entries regrouped panel by panel
    uint32_t P;                   // panels
    uint32_t PW;                  // iterate entries per panel (one block's shared-memory copy)
    const uint32_t *poff;         // [P*n+1] entry offsets, panel-major: panel p row i = [poff[p*n+i], poff[p*n+i+1])
    const uint16_t *pcol;         // destination minus p*PW
    const void *pw;               // weights (same width as w), null when unweighted
    void *yacc;                   // [n] row sums over the panels so far (iterate type)
    uint32_t *err;                // staged rows (mode 7): set when a bulk copy did not complete in time
};

// dynamic shared memory for the iterate cache, per block (two blocks per SM)
constexpr size_t kCacheBytesRows = 96 * 1024;
constexpr size_t kCacheBytesStream = 48 * 1024;
// iterate bytes of a relabelled level gathered with L1 evict-last priority
constexpr size_t kSplitBytes = 128 * 1024;
// the hub prefix in bytes: kSplitBytes, or SGPB_PI_SPLIT_KB (a tuning knob)
static size_t split_bytes() {
    static const size_t v = [] {
        const char *s = getenv("SGPB_PI_SPLIT_KB");
        const long kb = s ? atol(s) : 0;
        return kb > 0 && kb <= 256 ? (size_t)kb * 1024 : kSplitBytes;
    }();
    return v;
}
// dynamic shared memory for one column panel of the iterate, per block
constexpr size_t kPanelBytes = 96 * 1024;
constexpr uint32_t kMaxPanels = 31;
// rows above one warp's share of the cost / kHeavyDiv* are cut into segments
// of 2^kSegShift entries that the block's warps share
constexpr uint64_t kHeavyDivRows = 16;
constexpr uint64_t kHeavyDivStream = 64;
constexpr uint32_t kSegShift = 10;

// The iterate of a small level as the SpMV gathers it: entries below k (all
// of them) come from the block's shared-memory copy.
template <typename V>
struct XView {
    const V *g;
    const V *s;
    uint32_t k;
    __device__ __forceinline__ V operator[](uint32_t c) const { return c < k ? s[c] : g[c]; }
};

// Gathers of a hub-first relabelled level through L1 only for its leading k
// entries (the most referenced vertices, densely packed): those are loaded
// with L1 evict-last priority, all others bypass L1 allocation, so the other
// gathers cannot push the hub lines out of L1.
__device__ __forceinline__ double ld_hub(const double *p) {
    double v;
    asm volatile("ld.global.L1::evict_last.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_tail(const double *p) {
    double v;
    asm volatile("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
template <typename V>
struct SplitView {
    const V *g;
    uint32_t k;
    __device__ __forceinline__ V operator[](uint32_t c) const { return c < k ? ld_hub(g + c) : ld_tail(g + c); }
};

// iterate sources of the SpMV gathers
constexpr int kCacheNone = 0, kCachePrefix = 1, kCacheSplit = 2;

__device__ __forceinline__ void grid_barrier(cg::grid_group &g) {
    if (gridDim.x == 1) __syncthreads();
    else g.sync();
}

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

// first index i in [lo, hi] with pre[i] >= t (pre non-decreasing)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *pre, uint32_t lo, uint32_t hi, uint64_t t) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if ((uint64_t)pre[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Streaming loads of the matrix (destinations, weights): read-only and read
// once per iteration, so they bypass L1 allocation and leave L1 to the
// gathered vector entries (NA = true).
template <bool NA>
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) {
    if (NA) {
        uint32_t v;
        asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
        return v;
    }
    return __ldg(p);
}
// narrow weights of a relabelled copy (levels whose weights fit 8 / 16 bits)
template <bool NA>
__device__ __forceinline__ uint16_t ld_stream(const uint16_t *p) {
    if (NA) {
        unsigned short v;
        asm("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(v) : "l"(p));
        return v;
    }
    return __ldg(p);
}
template <bool NA>
__device__ __forceinline__ uint8_t ld_stream(const uint8_t *p) {
    if (NA) {
        unsigned short v;
        asm("ld.global.nc.L1::no_allocate.u8 %0, [%1];" : "=h"(v) : "l"(p));
        return (uint8_t)v;
    }
    return __ldg(p);
}
template <bool NA>
__device__ __forceinline__ unsigned long long ld_stream(const unsigned long long *p) {
    if (NA) {
        unsigned long long v;
        asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
        return v;
    }
    return __ldg(p);
}

// One SpMV term of row i for destination value xj and weight wt (weighted:
// HAS_W): plain, w_ij x_j in the iterate type; mixed (MX), the edge
// difference w_ij (x_i - x_j) with the difference rounded to FP32 and the
// product formed in FP32.
template <bool MX, typename ACC, typename V, typename W>
__device__ __forceinline__ ACC spmv_term(bool HAS_W, V xi, V xj, W wt) {
    if constexpr (MX) {
        const float dx = (float)(xi - xj);
        return HAS_W ? (float)wt * dx : dx;
    } else {
        return (ACC)(HAS_W ? (V)wt * xj : xj);
    }
}

// acc += sum_j term(w_j, src[col_j]) (and dsum += sum_j w_j) over the row
// entries j = j0, j0 + 32, ... < e of one warp (j0 = row start + lane): U
// predicated entries in flight per lane, destinations and weights first,
// then the U gathers.  xi: the row's own iterate value (used when MX).
template <int U, bool NA, bool MX, typename W, typename V, typename ACC, typename S>
__device__ __forceinline__ void warp_row_accum(const uint32_t *__restrict__ col, const W *__restrict__ w,
                                               const S &src, uint32_t j, uint32_t e, V xi, ACC &acc,
                                               uint64_t &dsum) {
    for (; j < e; j += 32 * U) {
        uint32_t c[U];
        ACC x[U];
#pragma unroll
        for (int k = 0; k < U; k++) c[k] = (j + 32 * k < e) ? ld_stream<NA>(col + j + 32 * k) : 0u;
        if (w) {
            W wt[U];
#pragma unroll
            for (int k = 0; k < U; k++) wt[k] = (j + 32 * k < e) ? ld_stream<NA>(w + j + 32 * k) : (W)0;
#pragma unroll
            for (int k = 0; k < U; k++) {
                x[k] = (j + 32 * k < e) ? spmv_term<MX, ACC>(true, xi, src[c[k]], wt[k]) : (ACC)0;
                dsum += (uint64_t)wt[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < U; k++) x[k] = (j + 32 * k < e) ? spmv_term<MX, ACC>(false, xi, src[c[k]], (W)0) : (ACC)0;
        }
#pragma unroll
        for (int k = 0; k < U; k++) acc += x[k];
    }
}

// One warp, rows [r0, r1) one after another, 128-entry trips (4 per lane),
// software-pipelined: the destinations and weights of the next trip (in the
// same row or the next processed row) are loaded before the gathers of the
// current trip, so DRAM latency overlaps the L2 gathers; a row's own value
// and weighted degree are loaded with its first trip (by every lane when MX,
// whose terms use it).  Rows for which skip(len) holds are left out.
// fin(i, sum, d, xi) on lane 0 once per row.
template <bool NA, bool MX, typename W, typename V, typename ACC, typename S, typename Skip, typename Fin>
__device__ __forceinline__ void warp_rows_pipelined(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                                                    const W *__restrict__ w, const S &src, const double *deg,
                                                    uint32_t r0, uint32_t r1, Skip skip, Fin &fin) {
    const unsigned lane = threadIdx.x & 31;
    // find the first processed row at or after i; returns r1 when none
    auto advance = [&](uint32_t i, uint32_t &b, uint32_t &e) -> uint32_t {
        for (; i < r1; i++) {
            b = rp[i];
            e = rp[i + 1];
            if (!skip(e - b)) return i;
        }
        return r1;
    };
    uint32_t cb = 0, ce = 0;
    uint32_t ci = advance(r0, cb, ce);
    if (ci >= r1) return;
    uint32_t cj = cb;   // base of the current trip
    uint32_t c_cur[4];
    W w_cur[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t j = cj + lane + 32 * k;
        c_cur[k] = j < ce ? ld_stream<NA>(col + j) : 0u;
        if (w) w_cur[k] = j < ce ? ld_stream<NA>(w + j) : (W)0;
    }
    double cx = 0, cd = 0;   // own value and weighted degree of row ci (lane 0; cx on every lane when MX)
    if (MX || lane == 0) cx = (double)src[ci];
    if (lane == 0) cd = w ? deg[ci] : (double)(ce - cb);
    ACC acc = 0;
    while (true) {
        // position of the next trip
        uint32_t ni = ci, nb = cb, ne = ce, nj = cj + 128;
        const bool row_ends = nj >= ce;
        if (row_ends) {
            ni = advance(ci + 1, nb, ne);
            nj = nb;
        }
        const bool have_next = ni < r1;
        uint32_t c_nxt[4];
        W w_nxt[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t j = nj + lane + 32 * k;
            const bool ok = have_next && j < ne;
            c_nxt[k] = ok ? ld_stream<NA>(col + j) : 0u;
            if (w) w_nxt[k] = ok ? ld_stream<NA>(w + j) : (W)0;
        }
        double nx = cx, nd = cd;
        if (row_ends && have_next) {
            if (MX || lane == 0) nx = (double)src[ni];
            if (lane == 0) nd = w ? deg[ni] : (double)(ne - nb);
        }
        // gathers of the current trip
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const bool ok = cj + lane + 32 * k < ce;
            if constexpr (MX) {
                if (ok) acc += spmv_term<true, ACC>(w != nullptr, (V)cx, src[c_cur[k]], w ? w_cur[k] : (W)0);
            } else {
                V x = ok ? src[c_cur[k]] : (V)0;
                if (w) x *= (V)w_cur[k];
                acc += (ACC)x;
            }
        }
        if (row_ends) {
            const ACC t = warp_sum(acc);
            if (lane == 0) fin(ci, t, cd, cx);
            acc = 0;
        }
        if (!have_next) break;
        ci = ni; cb = nb; ce = ne; cj = nj;
        cx = nx; cd = nd;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            c_cur[k] = c_nxt[k];
            if (w) w_cur[k] = w_nxt[k];
        }
    }
}

// four consecutive destinations (and weights) starting at p
template <bool NA>
__device__ __forceinline__ uint4 ld_stream4(const uint32_t *p) {
    if (NA) {
        uint4 v;
        asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                     : "l"(p));
        return v;
    }
    return __ldg(reinterpret_cast<const uint4 *>(p));
}

template <bool NA, typename W>
__device__ __forceinline__ void load4(const uint32_t *__restrict__ col, const W *__restrict__ w, uint32_t p,
                                      uint64_t m, bool vec, uint32_t (&c)[4], W (&wt)[4]) {
    if (vec && (uint64_t)p + 3 < m) {
        const uint4 v = ld_stream4<NA>(col + p);
        c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
        if (w) {
            if (sizeof(W) == 1) {   // four bytes at a 4-byte boundary (p is a multiple of 4)
                const uint32_t q = ld_stream<NA>(reinterpret_cast<const uint32_t *>(w + p));
                wt[0] = (W)(q & 0xFFu); wt[1] = (W)((q >> 8) & 0xFFu);
                wt[2] = (W)((q >> 16) & 0xFFu); wt[3] = (W)(q >> 24);
            } else if (sizeof(W) == 2) {   // four halves at an 8-byte boundary
                const unsigned long long q = ld_stream<NA>(reinterpret_cast<const unsigned long long *>(w + p));
                wt[0] = (W)(q & 0xFFFFu); wt[1] = (W)((q >> 16) & 0xFFFFu);
                wt[2] = (W)((q >> 32) & 0xFFFFu); wt[3] = (W)(q >> 48);
            } else if (sizeof(W) == 4) {
                const uint4 q = ld_stream4<NA>(reinterpret_cast<const uint32_t *>(w + p));
                wt[0] = (W)q.x; wt[1] = (W)q.y; wt[2] = (W)q.z; wt[3] = (W)q.w;
            } else {
                const uint4 q0 = ld_stream4<NA>(reinterpret_cast<const uint32_t *>(w + p));
                const uint4 q1 = ld_stream4<NA>(reinterpret_cast<const uint32_t *>(w + p + 2));
                wt[0] = (W)(((unsigned long long)q0.y << 32) | q0.x);
                wt[1] = (W)(((unsigned long long)q0.w << 32) | q0.z);
                wt[2] = (W)(((unsigned long long)q1.y << 32) | q1.x);
                wt[3] = (W)(((unsigned long long)q1.w << 32) | q1.z);
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const bool ok = (uint64_t)p + k < m;
            c[k] = ok ? ld_stream<NA>(col + p + k) : 0u;
            if (w) wt[k] = ok ? ld_stream<NA>(w + p + k) : (W)0;
        }
    }
}

// Stream the rows [ra, rb) (all non-empty, none block-wide) through one warp.
// fin(i, sum, degree, own value) is called exactly once per row, by one lane.
// win: this warp's kWin-entry shared-memory window of row offsets.
template <bool NA, bool MX, typename W, typename V, typename ACC, typename S, typename Fin>
__device__ __forceinline__ void warp_stream(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                                            const W *__restrict__ w, const S &src, uint64_t m, bool vec,
                                            uint32_t ra, uint32_t rb, const double *deg, uint32_t *win, V *winx,
                                            double *wind, Fin &fin) {
    const unsigned lane = threadIdx.x & 31;
    if (ra >= rb) return;
    const uint32_t Ea = rp[ra], Eb = rp[rb];
    uint32_t cur = ra;   // row holding the first entry of the tile
    ACC carry = 0;       // its partial sum from earlier tiles
    for (uint32_t c = Ea & ~3u; c < Eb; c += kTile) {
        // window: win[j] = rp[cur + j] (clamped at rb); rows are non-empty, so
        // the <= 128 entries of a tile lie in rows cur .. cur + 127.  The rows'
        // own iterate values (and weighted degrees) are staged alongside, so
        // finalising a row needs no dependent global load.
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t r = cur + lane * 4 + q;
            win[lane * 4 + q] = rp[r < rb ? r : rb];
            const uint32_t rr = r < rb ? r : rb - 1;
            winx[lane * 4 + q] = src[rr];
            if (w) wind[lane * 4 + q] = deg[rr];
        }
        if (lane == 0) {
            const uint32_t r = cur + kTile;
            win[kTile] = rp[r < rb ? r : rb];
        }
        const uint32_t p = c + 4 * lane;
        uint32_t cc[4];
        W ww[4];
        load4<NA, W>(col, w, p, m, vec, cc, ww);
        V xg[4];
        bool valid[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            valid[k] = (p + k >= Ea) && (p + k < Eb);
            xg[k] = valid[k] ? src[cc[k]] : (V)0;
        }
        __syncwarp();
        const uint32_t first = (Ea > c ? Ea : c);
        const unsigned lane_first = (first - c) >> 2;
        // row slot (offset from cur) of each valid entry
        uint32_t slot[4] = {0, 0, 0, 0};
        int nvalid = 0;
        {
            uint32_t s = 0;
            bool have = false;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (!valid[k]) continue;
                const uint32_t q = p + k;
                if (!have) {
                    uint32_t lo = 0, hi = kTile;   // largest j with win[j] <= q
                    while (lo < hi) {
                        uint32_t mid = (lo + hi + 1) >> 1;
                        if (win[mid] <= q) lo = mid;
                        else hi = mid - 1;
                    }
                    s = lo;
                    have = true;
                } else {
                    while (s < kTile && win[s + 1] <= q) s++;
                }
                slot[k] = s;
                nvalid++;
            }
        }
        // the entries' terms (mixed: edge differences to the row's own value)
        ACC prod[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if constexpr (MX) prod[k] = valid[k] ? spmv_term<true, ACC>(w != nullptr, winx[slot[k]], xg[k], w ? ww[k] : (W)0) : (ACC)0;
            else prod[k] = (ACC)(w ? (V)ww[k] * xg[k] : xg[k]);
        }
        // row slot s of this tile is complete with sum t
        auto done = [&](uint32_t s, ACC t) {
            fin(cur + s, t, w ? wind[s] : (double)(win[s + 1] - win[s]), (double)winx[s]);
        };
        // lane-local runs: A = first run, B = last run, middle runs complete here
        ACC A = 0, B = 0, run = 0;
        uint32_t s0 = 0, s3 = 0, rs = 0;
        bool started = false, multi = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!valid[k]) continue;
            if (!started) {
                started = true;
                rs = slot[k];
                s0 = rs;
                run = (ACC)prod[k];
            } else if (slot[k] != rs) {
                if (!multi) {
                    A = run;
                    multi = true;
                } else {
                    done(rs, run);   // middle run
                }
                rs = slot[k];
                run = (ACC)prod[k];
            } else {
                run += (ACC)prod[k];
            }
        }
        s3 = rs;
        B = run;
        if (!multi) A = B;
        if (lane == lane_first && nvalid) {
            A += carry;
            if (!multi) B = A;
        }
        // segmented inclusive scan over lanes of the last-run sums
        const bool lv = nvalid > 0;
        const uint32_t prev_s3 = __shfl_up_sync(0xFFFFFFFFu, s3, 1);
        const int prev_v = __shfl_up_sync(0xFFFFFFFFu, (int)lv, 1);
        const bool cont_prev = lv && lane > 0 && prev_v && lane != lane_first && prev_s3 == s0;
        ACC Sc = lv ? B : (ACC)0;
        int F = (!lv || multi || !cont_prev) ? 1 : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const ACC t = __shfl_up_sync(0xFFFFFFFFu, Sc, d);
            const int tf = __shfl_up_sync(0xFFFFFFFFu, F, d);
            if (lane >= (unsigned)d) {
                if (!F) Sc += t;
                F |= tf;
            }
        }
        const ACC S_prev = __shfl_up_sync(0xFFFFFFFFu, Sc, 1);
        const uint32_t next_s0 = __shfl_down_sync(0xFFFFFFFFu, s0, 1);
        const int next_v = __shfl_down_sync(0xFFFFFFFFu, (int)lv, 1);
        // first run of a multi-run lane ends here
        if (lv && multi) done(s0, A + (cont_prev ? S_prev : (ACC)0));
        // last run: ends here unless the next lane or the next tile continues it
        const bool next_cont = lane < 31 && next_v && next_s0 == s3;
        const bool tile_cont = lane == 31 && lv && win[s3 + 1] > c + kTile;
        if (lv && !next_cont && !tile_cont) done(s3, Sc);
        // next tile starts in row cur + s3 of lane 31 (continued) or the row after
        const int tc = __shfl_sync(0xFFFFFFFFu, (int)tile_cont, 31);
        const uint32_t s31 = __shfl_sync(0xFFFFFFFFu, s3, 31);
        const ACC S31 = __shfl_sync(0xFFFFFFFFu, Sc, 31);
        __syncwarp();
        if (tc) {
            cur += s31;
            carry = S31;
        } else {
            cur += s31 + 1;
            carry = 0;
        }
    }
}

// ------------------------------------------ staged warp rows (MODE 7) --
// The matrix stream of a warp's rows is copied into a per-warp ring of
// shared-memory chunks by 1-D bulk copies (cp.async.bulk, completion counted
// on an mbarrier per slot), issued by lane 0 ahead of use.  The warp then
// reads destinations and weights from shared memory, so its registers hold
// only the gathers: eight per lane in flight instead of four plus the
// prefetched stream.  Chunks are kStageCh consecutive entries at multiples of
// kStageCh in the level's arrays (16-byte aligned); the arrays of a level
// that runs this mode are padded by kStagePad entries, so every chunk copy
// is in bounds.  Only this GPU's own memory is read, and no copy uses cluster
// multicast.
constexpr uint32_t kStageCh = kStagePad;
constexpr int kStageU = 8;                       // entries per lane per trip (32 * 8 = kStageCh)
constexpr uint32_t kStageWaitLimit = 1u << 22;   // bounded mbarrier polls before giving up
template <typename W>
struct StageCfg {
    static constexpr uint32_t R = sizeof(W) == 8 ? 2 : (sizeof(W) == 4 ? 3 : 4);   // ring slots per warp
    // destinations, weights, mbarriers, chunk ids; 16-byte multiple
    static constexpr size_t warp_bytes = ((size_t)R * kStageCh * (4 + sizeof(W)) + 12 * R + 15) & ~(size_t)15;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase of the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity) {
    for (uint32_t k = 0; k < kStageWaitLimit; k++)
        if (mbar_test(b, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(b))
                 : "memory");
}
// generic-proxy reads of a slot are ordered before the next bulk copy into it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// A warp's ring in dynamic shared memory: slot s holds chunk ids[s].  Copies
// are numbered in issue order (seq): slot = seq % R, and the phase parity of
// a copy is (seq / R) & 1.  seq persists across the iterations of a launch
// (the barriers are set up once, by stage_init).
template <typename W>
struct StageRing {
    uint32_t *col;   // [R][kStageCh]
    W *w;            // [R][kStageCh]
    uint64_t *bar;   // [R]
    uint32_t *ids;   // [R]
};

template <typename W>
__device__ __forceinline__ StageRing<W> stage_ring(unsigned char *base, uint32_t warp) {
    constexpr uint32_t R = StageCfg<W>::R;
    unsigned char *p = base + (size_t)warp * StageCfg<W>::warp_bytes;
    StageRing<W> r;
    r.col = (uint32_t *)p;
    r.w = (W *)(p + (size_t)R * kStageCh * 4);
    r.bar = (uint64_t *)(p + (size_t)R * kStageCh * (4 + sizeof(W)));
    r.ids = (uint32_t *)(r.bar + R);
    return r;
}

template <typename W>
__device__ __forceinline__ void stage_init(const StageRing<W> &r) {
    if ((threadIdx.x & 31) == 0) {
        for (uint32_t s = 0; s < StageCfg<W>::R; s++) mbar_init(&r.bar[s]);
        mbar_fence_init();
    }
    __syncwarp();
}

// One warp, rows [r0, r1) (rows with skip(len) left out), one after another
// in trips of up to kStageCh entries of one row (kStageU per lane), the
// destinations and weights read from the ring.  fin(i, sum, d, xi) on lane 0
// once per row.  seq: the warp's copy counter (in/out).  Returns false when a
// copy did not complete within the wait limit, or the ring's bookkeeping
// failed a check (the caller reports the error); every copy issued has then
// been waited for once more, with the same limit.
template <bool MX, typename W, typename V, typename ACC, typename S, typename Skip, typename Fin>
__device__ __forceinline__ bool warp_rows_staged(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                                                 const W *__restrict__ w, const S &src, const double *deg,
                                                 uint32_t r0, uint32_t r1, Skip skip, Fin &fin,
                                                 const StageRing<W> &ring, uint32_t &seq) {
    constexpr uint32_t R = StageCfg<W>::R;
    const unsigned lane = threadIdx.x & 31;
    // producer: the chunks of the processed rows of [r0, r1), in order, each
    // once; [pc, pend) are the current producer row's chunks not yet issued
    uint32_t pr = r0, pc = 0, pend = 0;
    auto prod_next = [&]() -> bool {
        while (pc >= pend) {
            if (pr >= r1) return false;
            const uint32_t b = rp[pr], e = rp[pr + 1];
            pr++;
            if (skip(e - b)) continue;
            pend = (e + kStageCh - 1) / kStageCh;
            if (pc < b / kStageCh) pc = b / kStageCh;
        }
        return true;
    };
    uint32_t iss = seq, rel = seq;   // copies [rel, iss) hold chunks not yet consumed
    auto fill = [&]() {
        __syncwarp();   // every lane is done reading the released slots
        while (iss - rel < R && prod_next()) {
            const uint32_t slot = iss % R;
            if (lane == 0) {
                ring.ids[slot] = pc;
                fence_proxy_async();
                const uint32_t bytes = kStageCh * 4 + (w ? kStageCh * (uint32_t)sizeof(W) : 0u);
                mbar_expect_tx(&ring.bar[slot], bytes);
                bulk_load(ring.col + (size_t)slot * kStageCh, col + (size_t)pc * kStageCh, kStageCh * 4,
                          &ring.bar[slot]);
                if (w)
                    bulk_load(ring.w + (size_t)slot * kStageCh, w + (size_t)pc * kStageCh,
                              kStageCh * (uint32_t)sizeof(W), &ring.bar[slot]);
            }
            pc++;
            iss++;
        }
        __syncwarp();   // ids[] visible to every lane
    };
    // consumer: the current row ci = [cb, ce), entry j, own value cx, degree cd
    auto next_row = [&](uint32_t i, uint32_t &b, uint32_t &e) -> uint32_t {
        for (; i < r1; i++) {
            b = rp[i];
            e = rp[i + 1];
            if (!skip(e - b)) return i;
        }
        return r1;
    };
    uint32_t cb = 0, ce = 0;
    uint32_t ci = next_row(r0, cb, ce);
    double cx = 0, cd = 0;
    if (ci < r1) {
        if (MX || lane == 0) cx = (double)src[ci];
        if (lane == 0) cd = w ? deg[ci] : (double)(ce - cb);
    }
    uint32_t cseq = seq;   // the copy holding the chunk of entry j
    uint32_t j = cb;
    ACC acc = 0;
    bool ok = true;
    while (ci < r1) {
        const uint32_t tend = ce - j > kStageCh ? j + kStageCh : ce;
        const uint32_t c0 = j / kStageCh, c1 = (tend - 1) / kStageCh;
        // the copies before the one holding c0 are consumed: release them
        fill();
        while (cseq < iss && ring.ids[cseq % R] != c0) {
            cseq++;
            rel = cseq;
            fill();
        }
        // the trip's chunks are copies cseq (and cseq + 1), issued in order
        if (cseq >= iss || (c1 != c0 && (cseq + 1 >= iss || ring.ids[(cseq + 1) % R] != c1))) { ok = false; break; }
        if (!mbar_wait(&ring.bar[cseq % R], (cseq / R) & 1u)) { ok = false; break; }
        if (c1 != c0 && !mbar_wait(&ring.bar[(cseq + 1) % R], ((cseq + 1) / R) & 1u)) { ok = false; break; }
        // the next processed row's own value and degree load during the gathers
        const bool row_ends = tend == ce;
        uint32_t ni = ci, nb = cb, ne = ce;
        double nx = cx, nd = cd;
        if (row_ends) {
            ni = next_row(ci + 1, nb, ne);
            if (ni < r1) {
                if (MX || lane == 0) nx = (double)src[ni];
                if (lane == 0) nd = w ? deg[ni] : (double)(ne - nb);
            }
        }
        uint32_t c[kStageU];
        W wt[kStageU];
#pragma unroll
        for (int k = 0; k < kStageU; k++) {
            const uint32_t e = j + lane + 32 * k;
            const uint32_t slot = (e / kStageCh == c0 ? cseq : cseq + 1) % R;
            const uint32_t off = slot * kStageCh + e % kStageCh;
            c[k] = e < tend ? ring.col[off] : 0u;
            wt[k] = (w && e < tend) ? ring.w[off] : (W)0;
        }
        V x[kStageU];
#pragma unroll
        for (int k = 0; k < kStageU; k++) x[k] = (j + lane + 32 * k < tend) ? src[c[k]] : (V)0;
#pragma unroll
        for (int k = 0; k < kStageU; k++) {
            if (j + lane + 32 * k < tend) {
                if constexpr (MX) acc += spmv_term<true, ACC>(w != nullptr, (V)cx, x[k], wt[k]);
                else acc += (ACC)(w ? (V)wt[k] * x[k] : x[k]);
            }
        }
        if (row_ends) {
            const ACC t = warp_sum(acc);
            if (lane == 0) fin(ci, t, cd, cx);
            acc = 0;
            ci = ni; cb = nb; ce = ne; cx = nx; cd = nd;
            j = cb;
        } else {
            j = tend;
        }
    }
    if (!ok) {
        // every copy issued lands before the ring is given up
        for (uint32_t q = rel; q < iss; q++) mbar_wait(&ring.bar[q % R], (q / R) & 1u);
    }
    seq = iss;
    __syncwarp();
    return ok;
}

// Destinations of four consecutive panel entries (16-bit, panel-relative).
template <bool NA>
__device__ __forceinline__ void ld_pcol4(const uint16_t *p, uint32_t (&c)[4]) {
    uint32_t lo, hi;
    if (NA) {
        asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(lo), "=r"(hi) : "l"(p));
    } else {
        const uint2 v = __ldg(reinterpret_cast<const uint2 *>(p));
        lo = v.x; hi = v.y;
    }
    c[0] = lo & 0xFFFFu; c[1] = lo >> 16; c[2] = hi & 0xFFFFu; c[3] = hi >> 16;
}

// One warp, the up to 32 rows [g, g + gl) restricted to one column panel:
// each row's sum of w_ij * x_j over its entries in the panel (x_j read from
// the block's shared-memory copy xs of the panel) is added to yacc[row], or
// stored there on the first panel.  Entries are taken 128 per trip, four
// consecutive ones per lane; a trip's per-row sums are formed by runs inside
// each lane and a segmented scan across lanes, and each row slot receives at
// most one addition per trip, so the order of additions is fixed by the data.
// win: 33 words of this warp's shared memory; ysm: 32 accumulators.
template <bool NA, typename W, typename V, typename ACC>
__device__ __forceinline__ void panel_rows32(const uint32_t *__restrict__ offp, const uint16_t *__restrict__ pcol,
                                             const W *__restrict__ pw, const V *xs, uint32_t g, uint32_t gl,
                                             bool first, uint32_t *win, ACC *ysm, ACC *yacc) {
    const unsigned lane = threadIdx.x & 31;
    win[lane] = offp[g + (lane < gl ? lane : gl)];
    if (lane == 0) win[32] = offp[g + gl];
    ysm[lane] = (ACC)0;
    const ACC yprev = (!first && lane < gl) ? yacc[g + lane] : (ACC)0;
    __syncwarp();
    const uint32_t E0 = win[0], E1 = win[32];
    for (uint32_t c = E0 & ~3u; c < E1; c += 128) {
        const uint32_t q0 = c + 4 * lane;
        uint32_t cc[4] = {0, 0, 0, 0};
        W ww[4] = {0, 0, 0, 0};
        if (q0 < E1) {
            ld_pcol4<NA>(pcol + q0, cc);
            if (pw) {
                if (sizeof(W) == 4) {
                    const uint4 v = ld_stream4<NA>(reinterpret_cast<const uint32_t *>(pw + q0));
                    ww[0] = (W)v.x; ww[1] = (W)v.y; ww[2] = (W)v.z; ww[3] = (W)v.w;
                } else {
#pragma unroll
                    for (int k = 0; k < 4; k++) ww[k] = ld_stream<NA>(pw + q0 + k);
                }
            }
        }
        bool valid[4];
        V prod[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            valid[k] = q0 + k >= E0 && q0 + k < E1;
            const V x = xs[valid[k] ? cc[k] : 0u];   // entries outside the group may be padding
            prod[k] = valid[k] ? (pw ? (V)ww[k] * x : x) : (V)0;
        }
        // row slot of each valid entry: the last s with win[s] <= q (empty
        // rows share their start with the next row, so they are passed over)
        uint32_t sl[4] = {0, 0, 0, 0};
        {
            uint32_t s = 0;
            bool have = false;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (!valid[k]) continue;
                const uint32_t q = q0 + k;
                if (!have) {
                    uint32_t lo = 0, hi = gl - 1;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi + 1) >> 1;
                        if (win[mid] <= q) lo = mid;
                        else hi = mid - 1;
                    }
                    s = lo;
                    have = true;
                } else {
                    while (win[s + 1] <= q) s++;
                }
                sl[k] = s;
            }
        }
        // runs of equal slots inside the lane: the first (hs, A) and the last
        // (ts, B); runs in between belong to rows that start and end here
        ACC A = 0, B = 0, run = 0;
        uint32_t hs = 0xFFFFFFFEu, ts = 0xFFFFFFFFu, rs = 0;
        bool lv = false, multi = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!valid[k]) continue;
            if (!lv) {
                lv = true;
                rs = hs = sl[k];
                run = (ACC)prod[k];
            } else if (sl[k] != rs) {
                if (!multi) {
                    A = run;
                    multi = true;
                } else {
                    ysm[rs] += run;
                }
                rs = sl[k];
                run = (ACC)prod[k];
            } else {
                run += (ACC)prod[k];
            }
        }
        if (lv) { ts = rs; B = run; }
        // segmented inclusive scan of the last runs across lanes: a lane
        // continues its predecessor when its first slot is the predecessor's
        // last slot and it holds a single run
        const uint32_t prev_ts = __shfl_up_sync(0xFFFFFFFFu, ts, 1);
        const bool cont_prev = lv && lane > 0 && prev_ts == hs;
        ACC S = lv ? B : (ACC)0;
        int F = (!lv || multi || !cont_prev) ? 1 : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const ACC t = __shfl_up_sync(0xFFFFFFFFu, S, d);
            const int tf = __shfl_up_sync(0xFFFFFFFFu, F, d);
            if (lane >= (unsigned)d) {
                if (!F) S += t;
                F |= tf;
            }
        }
        const ACC Sprev = __shfl_up_sync(0xFFFFFFFFu, S, 1);
        const uint32_t next_hs = __shfl_down_sync(0xFFFFFFFFu, hs, 1);
        const bool cont_next = lane < 31 && next_hs == ts;
        if (multi) ysm[hs] += A + (cont_prev ? Sprev : (ACC)0);
        if (lv && !cont_next) ysm[ts] += S;
        __syncwarp();
    }
    if (lane < gl) yacc[g + lane] = yprev + ysm[lane];
    __syncwarp();
}

// The next raw iterate value r_i of row i from u_i = (x_i - mu) / nu and
// its row sum acc (plain: sum_j w_ij x_j; MX: sum_j w_ij (x_i - x_j)):
// shifted Laplacian r = (gb - d) u + A u = gb u - L u, or the lazy random
// walk r = u / 2 + (A u)_i / (2 d) of the normalized variant (r = u / 2 for
// an isolated vertex).  All in FP64.
template <bool MX>
__device__ __forceinline__ double next_value(int normlap, double gb, double mu, double inv_nu, double ui, double acc,
                                             double d) {
    if constexpr (MX) {
        const double lu = acc * inv_nu;   // (L u)_i; the mean cancels in the differences
        return normlap ? (d > 0 ? ui - 0.5 * lu / d : 0.5 * ui) : gb * ui - lu;
    } else {
        const double au = (acc - mu * d) * inv_nu;   // (A u)_i
        return normlap ? 0.5 * ui + (d > 0 ? 0.5 * au / d : 0.0) : (gb - d) * ui + au;
    }
}

template <int CACHE, typename V>
__device__ __forceinline__ auto make_src(const V *g, const V *s, uint32_t k) {
    if constexpr (CACHE == kCachePrefix) return XView<V>{g, s, k};
    else if constexpr (CACHE == kCacheSplit) return SplitView<V>{g, k};
    else return g;
}

// MODE 0: normal rows streamed in warp tiles (short-row levels); MODE 4: one
// warp per row with 4 loads in flight per lane; MODE 5: one warp per row,
// trips software-pipelined across rows (dense levels); MODE 6: column panels;
// MODE 7: one warp per row, the matrix stream staged in shared memory by bulk
// copies (dense levels of a padded relabelled copy).
// NA: matrix loads bypass L1 allocation.  CACHE: kCachePrefix -- gathers read
// the block's shared-memory copy of a small level's iterate; kCacheSplit --
// gathers below kcache (the hub prefix of a relabelled level) use L1
// evict-last priority, the others bypass L1 allocation.  MX: mixed-precision
// arithmetic (FP32 edge-difference row sums; never with column panels).
template <typename W, typename V, int MODE, bool NA, int CACHE, bool MX>
__global__ void __launch_bounds__(kPIThreads, 2) k_power_iter(PIArgs a) {
    constexpr bool STREAM = MODE == 0;
    cg::grid_group grid = cg::this_grid();
    // [0, 160): block_sum_d scratch (5 x 32), [200, 202): broadcast, [210, 226): warp maxima
    __shared__ double sm[256];
    constexpr bool WIN = MODE == 0 || MODE == 6;   // row-offset windows: streaming and panels only
    __shared__ uint32_t swin[WIN ? kPIWarps : 1][kWin + 3];
    // per-row staging of the stream windows (unused by the warp-row variants)
    __shared__ V swinx[STREAM ? kPIWarps : 1][kTile];
    __shared__ double swind[STREAM ? kPIWarps : 1][kTile];
    static_assert(sizeof(V) == 8, "the iterate is stored in FP64");
    static_assert(!(MX && MODE == 6), "column panels have no mixed-precision form");
    typedef typename std::conditional<MX, float, double>::type ACC;
    // panels: per-warp row sums of a 32-row group, group counters (two, used
    // by alternate panels so one can be reset while the other is in use)
    constexpr bool PANEL = MODE == 6;
    __shared__ ACC sysm[PANEL ? kPIWarps : 1][32];
    __shared__ uint32_t s_grp[2];
    __shared__ uint32_t s_seg;   // next block-wide-row segment
    if (threadIdx.x < 2) s_grp[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_seg = 0;   // first read after the phase-0 barriers
    const uint32_t n = a.n;
    const W *w = (const W *)a.w;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t n_heavy = *a.n_heavy_ptr;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    constexpr bool STAGED = MODE == 7;
    StageRing<W> ring;
    uint32_t stage_seq = 0;
    if constexpr (STAGED) {
        ring = stage_ring<W>(dyn_smem, threadIdx.x >> 5);
        stage_init(ring);
    }
    // Work split, fixed for the whole launch: block b owns the rows whose
    // cost prefix (all rows) starts in the b-th equal share; inside the block,
    // block-wide rows are processed by all threads and the remaining rows are
    // cut into equal-cost contiguous ranges, one per warp.
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
    const uint32_t wh0 = lower_bound_u32(a.heavy, h0, h1, w_r0);
    const uint32_t wh1 = lower_bound_u32(a.heavy, h0, h1, w_r1);
    V *va = (V *)a.va, *vb = (V *)a.vb;
    double *part0 = a.partials, *part1 = a.partials + (size_t)gridDim.x * kNP;
    const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;

    // ---- phase 0a: prolongate / load the start vector, weighted degrees
    double p_sum = 0, p_maxd = 0, p_xd = 0, p_d = 0;   // p_xd, p_d: D-weighted mean (normlap)
    for (uint64_t i64 = gwarp; i64 < n; i64 += nwarps) {
        const uint32_t i = (uint32_t)i64;
        const uint32_t b = a.rp[i], e = a.rp[i + 1];
        double d = (double)(e - b);
        if (w && e - b <= a.heavy_T) {
            uint64_t s = 0;
            for (uint32_t j = b + lane; j < e; j += 32) s += (uint64_t)__ldg(w + j);
            d = (double)warp_sum(s);
        }
        if (lane == 0) {
            const uint32_t o = a.inv ? a.inv[i] : i;
            const double x = a.vcmap ? a.x_in[a.vcmap[o]] : a.x_in[o];
            const V xs = (V)x;
            va[i] = xs;
            p_sum += (double)xs;
            if (!w || e - b <= a.heavy_T) {
                a.deg[i] = d;
                if (d > p_maxd) p_maxd = d;
                p_xd += (double)xs * d;
                p_d += d;
            }
        }
    }
    if (w) {
        for (uint32_t h = blockIdx.x; h < n_heavy; h += gridDim.x) {
            const uint32_t i = a.heavy[h];
            const uint32_t b = a.rp[i], e = a.rp[i + 1];
            if (e - b <= a.heavy_T) continue;   // empty rows were done above (block-uniform)
            uint64_t s = 0;
            for (uint32_t j = b + threadIdx.x; j < e; j += blockDim.x) s += (uint64_t)__ldg(w + j);
            double sd = (double)s, z = 0;
            block_sum2(sd, z, sm);
            if (threadIdx.x == 0) {
                a.deg[i] = sd;
                if (sd > p_maxd) p_maxd = sd;
                const uint32_t o = a.inv ? a.inv[i] : i;
                const V xs = (V)(a.vcmap ? a.x_in[a.vcmap[o]] : a.x_in[o]);
                p_xd += (double)xs * sd;
                p_d += sd;
            }
        }
    }
    {
        double v3[3] = {p_sum, p_xd, p_d};
        block_sum_d<3>(v3, sm);
        double mx = warp_max(p_maxd);
        if ((threadIdx.x & 31) == 0) sm[210 + (threadIdx.x >> 5)] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) m = sm[210 + k] > m ? sm[210 + k] : m;
            part0[(size_t)blockIdx.x * kNP + 0] = v3[0];
            part0[(size_t)blockIdx.x * kNP + 1] = m;
            part0[(size_t)blockIdx.x * kNP + 2] = v3[1];
            part0[(size_t)blockIdx.x * kNP + 3] = v3[2];
        }
    }
    grid_barrier(grid);
    double S1 = 0, maxd = 0, Sxd = 0, Sd = 0;
    {
        if (threadIdx.x < 32) {
            double s = 0, m = 0, xd = 0, dd = 0;
            for (uint32_t b = lane; b < gridDim.x; b += 32) {
                s += part0[(size_t)b * kNP + 0];
                double x = part0[(size_t)b * kNP + 1];
                m = x > m ? x : m;
                xd += part0[(size_t)b * kNP + 2];
                dd += part0[(size_t)b * kNP + 3];
            }
            s = warp_sum(s);
            m = warp_max(m);
            xd = warp_sum(xd);
            dd = warp_sum(dd);
            if (lane == 0) { sm[0] = s; sm[1] = m; sm[2] = xd; sm[3] = dd; }
        }
        __syncthreads();
        S1 = sm[0];
        maxd = sm[1];
        Sxd = sm[2];
        Sd = sm[3];
        __syncthreads();
    }
    double gb = 2.0 * maxd;
    if (gb < 2.0) gb = 2.0;
    // the start vector is orthogonalised against the constant vector (mean)
    // or, for the normalized Laplacian, D-orthogonalised (degree-weighted mean)
    double mu = a.normlap ? (Sd > 0 ? Sxd / Sd : 0.0) : S1 / (double)n;
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
    uint64_t niter = 0;
    V *src = va, *dst = vb;
    uint32_t panel_seq = 0;   // panels processed so far: selects the group counter
    uint32_t *win = swin[WIN ? wk : 0];
    V *winx = swinx[STREAM ? wk : 0];
    double *wind = swind[STREAM ? wk : 0];
    V *xs = reinterpret_cast<V *>(dyn_smem);
    const uint32_t kc = a.kcache < n ? a.kcache : n;
    while (true) {
        double P[kNP] = {0, 0, 0, 0, 0};
        // refresh the shared-memory copy of the leading iterate entries
        if (CACHE == kCachePrefix && kc) {
            for (uint32_t c = threadIdx.x; c < kc; c += blockDim.x) xs[c] = src[c];
            __syncthreads();
        }
        const auto xv = make_src<CACHE, V>(src, xs, kc);
        // finalise row i from its row sum acc (plain: sum_j w_ij src_j; MX:
        // sum_j w_ij (src_i - src_j)), its weighted degree d and its own raw
        // iterate value xi
        auto fin = [&](uint32_t i, ACC acc, double d, double xi) {
            const double ui = (xi - mu) * inv_nu;
            const double r = next_value<MX>(a.normlap, gb, mu, inv_nu, ui, (double)acc, d);
            const V rs = (V)r;
            dst[i] = rs;
            const double rd = (double)rs;
            P[0] += rd; P[1] += rd * rd; P[2] += ui * rd; P[3] += ui; P[4] += ui * ui;
        };
        // this warp's rows
        if (STREAM) {
            // in segments between block-wide rows
            uint32_t seg = w_r0;
            for (uint32_t h = wh0; h < wh1; h++) {
                const uint32_t hr = a.heavy[h];
                warp_stream<NA, MX, W, V, ACC>(a.rp, a.col, w, xv, a.m, a.vec_ok, seg, hr, a.deg, win, winx, wind,
                                               fin);
                seg = hr + 1;
            }
            warp_stream<NA, MX, W, V, ACC>(a.rp, a.col, w, xv, a.m, a.vec_ok, seg, w_r1, a.deg, win, winx, wind, fin);
        } else if (PANEL) {
            // column panels: the block copies panel p of the iterate into
            // shared memory, then its warps take 32-row groups of the block's
            // rows from a shared counter and add each row's panel sum to yacc
            ACC *yacc = (ACC *)a.yacc;
            const W *pw = (const W *)a.pw;
            const uint32_t ngroups = (B1 - B0 + 31) / 32;
            const bool vec = ((uintptr_t)src & 15u) == 0;
            constexpr uint32_t VPER = 16 / sizeof(V);
            for (uint32_t p = 0; p < a.P; p++, panel_seq++) {
                const uint32_t base = p * a.PW;
                const uint32_t len = n - base < a.PW ? n - base : a.PW;
                __syncthreads();   // every warp is done with the previous panel
                if (vec) {
                    const uint32_t nv = len / VPER;
                    const uint4 *s4 = reinterpret_cast<const uint4 *>(src + base);
                    uint4 *d4 = reinterpret_cast<uint4 *>(xs);
                    for (uint32_t c = threadIdx.x; c < nv; c += blockDim.x) d4[c] = __ldcg(s4 + c);
                    for (uint32_t c = nv * VPER + threadIdx.x; c < len; c += blockDim.x) xs[c] = __ldcg(src + base + c);
                } else {
                    for (uint32_t c = threadIdx.x; c < len; c += blockDim.x) xs[c] = __ldcg(src + base + c);
                }
                if (threadIdx.x == 0) s_grp[(panel_seq + 1) & 1] = 0;
                __syncthreads();
                const uint32_t *offp = a.poff + (size_t)p * n;
                uint32_t *ctr = &s_grp[panel_seq & 1];
                while (true) {
                    uint32_t k = 0;
                    if (lane == 0) k = atomicAdd(ctr, 1u);
                    k = __shfl_sync(0xFFFFFFFFu, k, 0);
                    if (k >= ngroups) break;
                    const uint32_t g = B0 + 32 * k;
                    const uint32_t gl = B1 - g < 32 ? B1 - g : 32;
                    panel_rows32<NA, W, V, ACC>(offp, a.pcol, pw, xs, g, gl, p == 0, win, sysm[PANEL ? wk : 0], yacc);
                }
            }
            __syncthreads();   // yacc holds every row of the block
            for (uint32_t i = B0 + threadIdx.x; i < B1; i += blockDim.x) {
                const uint32_t b = a.rp[i], e = a.rp[i + 1];
                if (e - b > a.heavy_T || e == b) continue;   // block-wide rows
                fin(i, yacc[i], w ? a.deg[i] : (double)(e - b), (double)src[i]);
            }
        } else if (MODE == 5) {
            const uint32_t T = a.heavy_T;
            auto skip = [T](uint32_t len) { return len > T || len == 0; };
            warp_rows_pipelined<NA, MX, W, V, ACC>(a.rp, a.col, w, xv, a.deg, w_r0, w_r1, skip, fin);
        } else if constexpr (STAGED) {
            const uint32_t T = a.heavy_T;
            auto skip = [T](uint32_t len) { return len > T || len == 0; };
            if (!warp_rows_staged<MX, W, V, ACC>(a.rp, a.col, w, xv, a.deg, w_r0, w_r1, skip, fin, ring, stage_seq) &&
                lane == 0) {
                atomicExch(a.err, 1u);
                __threadfence();
            }
        } else {
            uint32_t e = w_r0 < w_r1 ? a.rp[w_r0] : 0;
            for (uint32_t i = w_r0; i < w_r1; i++) {
                const uint32_t b = e;
                e = a.rp[i + 1];
                if (e - b > a.heavy_T || e == b) continue;   // block-wide rows
                // the row's own value is loaded before its entries so the
                // latency overlaps; the weighted degree is summed on the way
                const double xi = (MX || lane == 0) ? (double)src[i] : 0.0;
                ACC acc = 0;
                uint64_t ds = 0;
                warp_row_accum<(MODE == 8 ? 8 : 4), NA, MX, W, V, ACC>(a.col, w, xv, b + lane, e, (V)xi, acc, ds);
                acc = warp_sum(acc);
                if (w) ds = warp_sum(ds);
                if (lane == 0) fin(i, acc, w ? (double)ds : (double)(e - b), xi);
            }
        }
        // block-wide rows of this block's range: their segments of 2^seg_shift
        // entries are taken by the warps from a shared counter as they finish
        // their own rows; each segment's sum goes to its own slot, and the
        // slots of a row are added in order once all are written
        {
            const uint32_t sg0 = a.hseg[B0], sg1 = a.hseg[B1];
            while (true) {
                uint32_t k = 0;
                if (lane == 0) k = atomicAdd(&s_seg, 1u);
                const uint32_t sg = sg0 + __shfl_sync(0xFFFFFFFFu, k, 0);
                if (sg >= sg1) break;
                const uint32_t i = a.seg_row[sg];
                const uint32_t e = a.rp[i + 1];
                const uint32_t b = a.rp[i] + ((sg - a.hseg[i]) << a.seg_shift);
                const uint32_t e2 = e - b > (1u << a.seg_shift) ? b + (1u << a.seg_shift) : e;
                const V xi = MX ? src[i] : (V)0;
                ACC acc = 0;
                uint64_t ds = 0;
                warp_row_accum<8, NA, MX, W, V, ACC>(a.col, w, xv, b + lane, e2, xi, acc, ds);
                acc = warp_sum(acc);
                if (lane == 0) a.hpart[sg] = (double)acc;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_seg = 0;
        for (uint32_t h = h0 + threadIdx.x; h < h1; h += blockDim.x) {
            const uint32_t i = a.heavy[h];
            const uint32_t b = a.rp[i], e = a.rp[i + 1];
            double acc = 0;
            for (uint32_t sg = a.hseg[i]; sg < a.hseg[i + 1]; sg++) acc += a.hpart[sg];
            const double d = w ? (e > b ? a.deg[i] : 0.0) : (double)(e - b);
            const double ui = ((double)src[i] - mu) * inv_nu;
            const double r = next_value<MX>(a.normlap, gb, mu, inv_nu, ui, acc, d);
            const V rs = (V)r;
            dst[i] = rs;
            const double rd = (double)rs;
            P[0] += rd; P[1] += rd * rd; P[2] += ui * rd; P[3] += ui; P[4] += ui * ui;
        }
        block_sum_d<kNP>(P, sm);
        double *part = (niter & 1) ? part1 : part0;
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < kNP; k++) part[(size_t)blockIdx.x * kNP + k] = P[k];
        grid_barrier(grid);
        double S[kNP];
        reduce_partials(part, S, sm);
        const double mu_n = a.normlap ? 0.0 : S[0] / (double)n;   // no deflation in the normalized loop
        const double nsq = S[1] - mu_n * S[0];
        const double inv_nu_n = 1.0 / sqrt(nsq);
        last = dot;
        dot = (S[2] - mu_n * S[3]) * inv_nu_n;
        niter++;
        const double delta = fabs(dot - last);
        if (STAGED && *(volatile uint32_t *)a.err) {
            // a bulk copy did not complete: every block leaves here (the flag
            // was set before the barrier), the host reports the error
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                a.res[0] = (double)niter;
                a.res[5] = 1.0;
            }
            return;
        }
        if (!(delta > a.tol && niter < a.iter_max)) {
            // the reference returns u of the last iteration: (src - mu) / nu
            for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
                 i += (uint64_t)gridDim.x * blockDim.x)
                a.out[a.inv ? a.inv[i] : i] = ((double)src[i] - mu) * inv_nu;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                a.res[0] = (double)niter;
                a.res[1] = dot;
                a.res[2] = gb;
                // eigenvalue: of L from the shifted operator, or of the
                // random-walk Laplacian from the lazy walk's quotient
                a.res[3] = a.normlap ? 2.0 * (1.0 - S[2] / S[4]) : (gb * S[4] - S[2]) / S[4];
                a.res[4] = niter >= a.iter_max ? 1.0 : 0.0;
                a.res[5] = 0.0;
            }
            return;
        }
        mu = mu_n;
        inv_nu = inv_nu_n;
        V *t = src; src = dst; dst = t;
    }
}

// ------------------------------------------------------- small levels --
// A small level (the coarsest levels, which often need the most
// iterations) runs here: one block stages
// the whole level (offsets, destinations, weights), its weighted degrees and
// both iterate buffers in shared memory, one thread per row, and each
// iteration costs three block barriers.  Same recurrence, stopping rule and
// result as k_power_iter.
constexpr int kSmallThreads = 1024;
constexpr uint64_t kSmallCost = 32768;   // m + 8n of the largest level run here
constexpr size_t kSmallSmemBytes = 200 * 1024;

template <typename W, typename V>
static size_t small_level_bytes(uint32_t n, uint64_t m, bool weighted) {
    size_t b = ((size_t)n + 1) * 4 + (size_t)m * 4;
    b = (b + 15) & ~(size_t)15;
    if (weighted) b = (b + (size_t)m * sizeof(W) + 15) & ~(size_t)15;
    b += (size_t)n * 8;                              // degrees
    b += 2 * (((size_t)n * sizeof(V) + 15) & ~(size_t)15);
    return b;
}

// The whole computation of one small level by the calling block: the level
// (offsets, destinations, weights, degrees) and both iterates are staged in
// shared memory.  Every small level runs it inside the chained kernel
// (single partitions and batches alike), in FP64 also in a mixed-precision
// partition (these levels are latency-bound).
template <typename W, typename V>
__device__ __forceinline__ void small_level(const PIArgs &a) {
    typedef double ACC;
    __shared__ double sm[256];
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const uint32_t n = a.n;
    const uint64_t m = a.m;
    const W *wg = (const W *)a.w;
    unsigned char *p = dyn_smem;
    uint32_t *rp = (uint32_t *)p;
    p += ((size_t)n + 1) * 4;
    uint32_t *col = (uint32_t *)p;
    p += (size_t)m * 4;
    p = (unsigned char *)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    W *w = nullptr;
    if (wg) {
        w = (W *)p;
        p += (size_t)m * sizeof(W);
        p = (unsigned char *)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    }
    double *deg = (double *)p;
    p += (size_t)n * 8;
    V *xa = (V *)p;
    p += ((size_t)n * sizeof(V) + 15) & ~(size_t)15;
    V *xb = (V *)p;
    for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x) rp[i] = a.rp[i];
    for (uint64_t j = threadIdx.x; j < m; j += blockDim.x) {
        col[j] = a.col[j];
        if (wg) w[j] = wg[j];
    }
    __syncthreads();
    // phase 0: prolongation, weighted degrees, shift
    double p_sum = 0, p_maxd = 0, p_xd = 0, p_d = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t b = rp[i], e = rp[i + 1];
        double d = (double)(e - b);
        if (wg) {
            uint64_t s = 0;
            for (uint32_t j = b; j < e; j++) s += (uint64_t)w[j];
            d = (double)s;
        }
        deg[i] = d;
        p_maxd = d > p_maxd ? d : p_maxd;
        const V xs = (V)(a.vcmap ? a.x_in[a.vcmap[i]] : a.x_in[i]);
        xa[i] = xs;
        p_sum += (double)xs;
        p_xd += (double)xs * d;
        p_d += d;
    }
    double v2[3] = {p_sum, p_xd, p_d};
    block_sum_d<3>(v2, sm);
    {
        const double mx = warp_max(p_maxd);
        if ((threadIdx.x & 31) == 0) sm[210 + (threadIdx.x >> 5)] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mxd = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) mxd = sm[210 + k] > mxd ? sm[210 + k] : mxd;
        sm[200] = v2[0];
        sm[201] = mxd;
        sm[202] = v2[1];
        sm[203] = v2[2];
    }
    __syncthreads();
    const double S1 = sm[200];
    double gb = 2.0 * sm[201];
    if (gb < 2.0) gb = 2.0;
    double mu = a.normlap ? (sm[203] > 0 ? sm[202] / sm[203] : 0.0) : S1 / (double)n;
    __syncthreads();
    double p_sq = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = (double)xa[i] - mu;
        p_sq += x * x;
    }
    double q2[2] = {p_sq, 0};
    block_sum_d<2>(q2, sm);
    if (threadIdx.x == 0) sm[200] = q2[0];
    __syncthreads();
    double inv_nu = 1.0 / sqrt(sm[200]);
    __syncthreads();
    double dot = 0, last = 1;
    uint64_t niter = 0;
    V *src = xa, *dst = xb;
    // rows of at least 8 entries on average: one warp per row, else one thread
    const bool warp_rows = m >= 8ull * n;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    while (true) {
        double P[kNP] = {0, 0, 0, 0, 0};
        auto fin = [&](uint32_t i, ACC acc) {
            const double d = deg[i];
            const double ui = ((double)src[i] - mu) * inv_nu;
            const double au = ((double)acc - mu * d) * inv_nu;
            const double r = a.normlap ? 0.5 * ui + (d > 0 ? 0.5 * au / d : 0.0) : (gb - d) * ui + au;
            const V rs = (V)r;
            dst[i] = rs;
            const double rd = (double)rs;
            P[0] += rd; P[1] += rd * rd; P[2] += ui * rd; P[3] += ui; P[4] += ui * ui;
        };
        if (warp_rows) {
            for (uint32_t i = wid; i < n; i += nwarps) {
                const uint32_t b = rp[i], e = rp[i + 1];
                ACC acc = 0;
                for (uint32_t j = b + lane; j < e; j += 32) {
                    const V x = src[col[j]];
                    acc += (ACC)(wg ? (V)w[j] * x : x);
                }
                acc = warp_sum(acc);
                if (lane == 0) fin(i, acc);
            }
        } else {
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint32_t b = rp[i], e = rp[i + 1];
                ACC acc = 0;
                for (uint32_t j = b; j < e; j++) {
                    const V x = src[col[j]];
                    acc += (ACC)(wg ? (V)w[j] * x : x);
                }
                fin(i, acc);
            }
        }
        block_sum_d<kNP>(P, sm);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < kNP; k++) sm[200 + k] = P[k];
        __syncthreads();
        double S[kNP];
#pragma unroll
        for (int k = 0; k < kNP; k++) S[k] = sm[200 + k];
        __syncthreads();
        const double mu_n = a.normlap ? 0.0 : S[0] / (double)n;   // no deflation in the normalized loop
        const double nsq = S[1] - mu_n * S[0];
        const double inv_nu_n = 1.0 / sqrt(nsq);
        last = dot;
        dot = (S[2] - mu_n * S[3]) * inv_nu_n;
        niter++;
        const double delta = fabs(dot - last);
        if (!(delta > a.tol && niter < a.iter_max)) {
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) a.out[i] = ((double)src[i] - mu) * inv_nu;
            if (threadIdx.x == 0) {
                a.res[0] = (double)niter;
                a.res[1] = dot;
                a.res[2] = gb;
                // eigenvalue: of L from the shifted operator, or of the
                // random-walk Laplacian from the lazy walk's quotient
                a.res[3] = a.normlap ? 2.0 * (1.0 - S[2] / S[4]) : (gb * S[4] - S[2]) / S[4];
                a.res[4] = niter >= a.iter_max ? 1.0 : 0.0;
                a.res[5] = 0.0;
            }
            return;
        }
        mu = mu_n;
        inv_nu = inv_nu_n;
        V *t = src; src = dst; dst = t;
    }
}

template <typename W, typename V>
__global__ void __launch_bounds__(kSmallThreads, 1) k_power_iter_small(PIArgs a) {
    small_level<W, V>(a);
}

// A chain: the consecutive small levels of one hierarchy from its coarsest
// level up, each level reading the previous one's result through its vcmap.
struct PIChainDesc {
    PIArgs a;
    int wbytes;   // 0, 4 or 8
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Work queue over chains (the host orders them largest first): each block
// takes the next chain from a counter and runs its levels in order, so one
// launch iterates the small levels of a whole batch of hierarchies, one block
// per SM.  Each level is the single-level kernel's computation; res[6] of a
// level is its duration in ms by the device's global timer.
__global__ void __launch_bounds__(kSmallThreads, 1) k_power_iter_chains(const PIChainDesc *__restrict__ lev,
                                                                        const uint2 *__restrict__ chains,
                                                                        uint32_t nchains, uint32_t *next) {
    __shared__ uint32_t item;
    while (true) {
        __syncthreads();   // the previous chain is done with item
        if (threadIdx.x == 0) item = atomicAdd(next, 1u);
        __syncthreads();
        const uint32_t c = item;
        if (c >= nchains) return;
        const uint2 ch = chains[c];
        for (uint32_t k = 0; k < ch.y; k++) {
            const PIChainDesc &d = lev[ch.x + k];
            const unsigned long long t0 = global_ns();
            if (d.wbytes == 8) small_level<unsigned long long, double>(d.a);
            else small_level<uint32_t, double>(d.a);
            // the result is visible to the next level, and shared memory free
            __syncthreads();
            if (threadIdx.x == 0) d.a.res[6] = (double)(global_ns() - t0) * 1e-6;
        }
    }
}

// --------------------------------------------------- mid-size levels --
// Levels too large for one block's shared memory but small enough that the
// cooperative kernel's grid barriers dominate (about 13 us per iteration
// whatever the level's size) run on a cluster of kMidCTAs blocks: the
// iterate stays in global memory (L2-resident at these sizes), the five sums
// of an iteration are exchanged through distributed shared memory, and one
// cluster barrier per iteration replaces the grid barrier.  Clusters take
// chains of consecutive mid-size levels (one hierarchy each, coarsest first)
// from a work queue, so one launch iterates these levels of a whole batch of
// hierarchies, a cluster per hierarchy at a time.  The recurrence, stopping
// rule and result are the cooperative kernel's; the work split (rows by
// entry count over the cluster's blocks, then over their warps, CSR
// streaming) depends only on the level.
constexpr int kMidCTAs = 8;
constexpr int kMidThreads = 512;
constexpr int kMidWarps = kMidThreads / 32;
// m + 8n of the largest level run here by default: above it one level on the
// whole GPU is faster (measured on grids: at 2^17 both take ~12 us per
// iteration; at 3*10^5, 26 vs 9 us); batches raise it (options.cluster_max_log2)
constexpr uint64_t kMidCost = 1ull << 17;

struct MidLevelDesc {
    uint32_t n;
    uint64_t m;
    const uint32_t *rp;
    const uint32_t *col;
    const void *w;
    int wbytes;              // 0, 4 or 8
    int mixed;               // FP32 edge-difference arithmetic
    int normlap;
    int vec_ok;              // col / w 16-byte aligned
    const double *x_in;      // start vector, read through vcmap when set
    const uint32_t *vcmap;
    double *out;             // normalised result (n)
    double *va, *vb, *deg;   // iterate buffers and weighted degrees (n each)
    double tol;
    uint64_t iter_max;
    double *res;             // [0] niter [1] dot [2] gb [3] lambda [4] capped [6] ms
};

// first row i in [lo, hi] with rp[i] >= t
__device__ __forceinline__ uint32_t rows_at(const uint32_t *rp, uint32_t lo, uint32_t hi, uint64_t t) {
    return lower_bound_u32(rp, lo, hi, t);
}

// Cluster-wide sums of NV values: every block adds its partials to slot
// `buf` of its shared memory; after the cluster barrier lane r < kMidCTAs of
// the first warp reads block r's slot, lane 0 adds them in rank order and
// broadcasts through shared memory, so every block holds the same totals
// (and only kMidCTAs remote reads per value and block cross the cluster).
template <int CL, int NV>
__device__ __forceinline__ void cluster_sum(double (&v)[NV], double (*slot)[8], int buf, double *sm,
                                            cg::cluster_group &cl) {
    block_sum_d<NV>(v, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) slot[buf][k] = v[k];
    cl.sync();
    if (threadIdx.x < 32) {
        const unsigned lane = threadIdx.x;
        double mine[NV];
        const double *rs = cl.map_shared_rank(&slot[buf][0], lane < (unsigned)CL ? lane : 0u);
#pragma unroll
        for (int k = 0; k < NV; k++) mine[k] = lane < (unsigned)CL ? rs[k] : 0.0;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = 0;
            for (int r = 0; r < CL; r++) t += __shfl_sync(0xFFFFFFFFu, mine[k], r);
            if (lane == 0) sm[220 + k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = sm[220 + k];
    __syncthreads();   // sm is reused by the next sum
}

template <typename W, bool MX, int CL>
__device__ __forceinline__ void mid_level(const MidLevelDesc &d, cg::cluster_group &cl, double *sm,
                                          double (*slot)[8], uint32_t *win, double *winx, double *wind) {
    typedef typename std::conditional<MX, float, double>::type ACC;
    const uint32_t n = d.n;
    const uint64_t m = d.m;
    const uint32_t *rp = d.rp;
    const W *w = (const W *)d.w;
    const unsigned rank = cl.block_rank();
    const unsigned lane = threadIdx.x & 31, wk = threadIdx.x >> 5;
    // rows of this block and of this warp: equal shares of the entries
    const uint32_t R0 = rank == 0 ? 0u : rows_at(rp, 0, n, m * rank / CL);
    const uint32_t R1 = rank + 1 == (uint32_t)CL ? n : rows_at(rp, 0, n, m * (rank + 1) / CL);
    const uint64_t E0 = rp[R0], E1 = rp[R1];
    const uint32_t w0 = wk == 0 ? R0 : rows_at(rp, R0, R1, E0 + (E1 - E0) * wk / kMidWarps);
    const uint32_t w1 = wk + 1 == kMidWarps ? R1 : rows_at(rp, R0, R1, E0 + (E1 - E0) * (wk + 1) / kMidWarps);
    // ---- phase 0: start vector (prolongated), weighted degrees, shift
    double p[4] = {0, 0, 0, 0};   // sum x, sum x d, sum d (normlap mean), max d
    bool empty_rows = false;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t b = rp[i], e = rp[i + 1];
        double dg = (double)(e - b);
        if (w) {
            uint64_t sw = 0;
            for (uint32_t j = b + lane; j < e; j += 32) sw += (uint64_t)__ldg(w + j);
            dg = (double)warp_sum(sw);
        }
        empty_rows |= e == b;
        if (lane == 0) {
            const double x = d.vcmap ? d.x_in[d.vcmap[i]] : d.x_in[i];
            d.va[i] = x;
            d.deg[i] = dg;
            p[0] += x;
            p[1] += x * dg;
            p[2] += dg;
            p[3] = dg > p[3] ? dg : p[3];
        }
    }
    double mx = warp_max(p[3]);
    if (lane == 0) sm[210 + wk] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < kMidWarps; k++) t = sm[210 + k] > t ? sm[210 + k] : t;
        slot[1][4] = t;
    }
    double s3[3] = {p[0], p[1], p[2]};
    block_sum_d<3>(s3, sm);
    if (threadIdx.x == 0) { slot[1][0] = s3[0]; slot[1][1] = s3[1]; slot[1][2] = s3[2]; }
    cl.sync();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0, mxd = 0;
        for (int r = 0; r < CL; r++) {
            const double *rs = cl.map_shared_rank(&slot[1][0], r);
            a += rs[0];
            b += rs[1];
            c += rs[2];
            mxd = rs[4] > mxd ? rs[4] : mxd;
        }
        sm[220] = a; sm[221] = b; sm[222] = c; sm[223] = mxd;
    }
    __syncthreads();
    const double S0 = sm[220], Sxd = sm[221], Sd = sm[222], maxd = sm[223];
    __syncthreads();
    double gb = 2.0 * maxd;
    if (gb < 2.0) gb = 2.0;
    double mu = d.normlap ? (Sd > 0 ? Sxd / Sd : 0.0) : S0 / (double)n;
    double q[1] = {0};
    for (uint32_t i = R0 + threadIdx.x; i < R1; i += blockDim.x) {
        const double x = d.va[i] - mu;
        q[0] += x * x;
    }
    cluster_sum<CL, 1>(q, slot, 0, sm, cl);
    double inv_nu = 1.0 / sqrt(q[0]);
    // ---- iterations
    double dot = 0, last = 1;
    uint64_t niter = 0;
    double *src = d.va, *dst = d.vb;
    while (true) {
        double P[kNP] = {0, 0, 0, 0, 0};
        auto fin = [&](uint32_t i, ACC acc, double dg, double xi) {
            const double ui = (xi - mu) * inv_nu;
            const double r = next_value<MX>(d.normlap, gb, mu, inv_nu, ui, (double)acc, dg);
            dst[i] = r;
            P[0] += r; P[1] += r * r; P[2] += ui * r; P[3] += ui; P[4] += ui * ui;
        };
        if (w1 > w0)
            warp_stream<true, MX, W, double, ACC>(rp, d.col, w, (const double *)src, m, d.vec_ok != 0, w0, w1,
                                                  d.deg, win, winx, wind, fin);
        // rows without entries are not streamed: r = (gb - 0) u_i (u_i / 2
        // for the normalized walk)
        if (empty_rows && lane == 0)
            for (uint32_t i = w0; i < w1; i++)
                if (rp[i] == rp[i + 1]) fin(i, (ACC)0, 0.0, src[i]);
        // consecutive exchanges alternate slots (phase 0 used 1, then 0)
        cluster_sum<CL, kNP>(P, slot, (int)((niter + 1) & 1), sm, cl);
        const double mu_n = d.normlap ? 0.0 : P[0] / (double)n;
        const double nsq = P[1] - mu_n * P[0];
        const double inv_nu_n = 1.0 / sqrt(nsq);
        last = dot;
        dot = (P[2] - mu_n * P[3]) * inv_nu_n;
        niter++;
        const double delta = fabs(dot - last);
        if (!(delta > d.tol && niter < d.iter_max)) {
            for (uint32_t i = R0 + threadIdx.x; i < R1; i += blockDim.x) d.out[i] = (src[i] - mu) * inv_nu;
            if (rank == 0 && threadIdx.x == 0) {
                d.res[0] = (double)niter;
                d.res[1] = dot;
                d.res[2] = gb;
                d.res[3] = d.normlap ? 2.0 * (1.0 - P[2] / P[4]) : (gb * P[4] - P[2]) / P[4];
                d.res[4] = niter >= d.iter_max ? 1.0 : 0.0;
            }
            break;
        }
        mu = mu_n;
        inv_nu = inv_nu_n;
        double *t = src; src = dst; dst = t;
    }
}

// CL blocks per cluster, set at launch (cudaLaunchAttributeClusterDimension)
template <int CL>
__global__ void __launch_bounds__(kMidThreads, 1)
    k_power_iter_mid(const MidLevelDesc *__restrict__ lev, const uint2 *__restrict__ chains, uint32_t nchains,
                     uint32_t *next) {
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double sm[256];
    __shared__ double slot[2][8];
    __shared__ uint32_t swin[kMidWarps][kWin + 3];
    __shared__ double swinx[kMidWarps][kTile];
    __shared__ double swind[kMidWarps][kTile];
    __shared__ uint32_t item;
    const unsigned wk = threadIdx.x >> 5;
    while (true) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) item = atomicAdd(next, 1u);
        cl.sync();
        if (threadIdx.x == 0) sm[230] = (double)*cl.map_shared_rank(&item, 0);
        __syncthreads();
        const uint32_t c = (uint32_t)sm[230];
        // every block has read rank 0's `item` before any block can exit (a
        // block's shared memory must not be read after it has exited) or
        // rank 0 writes the next one
        cl.sync();
        if (c >= nchains) return;
        const uint2 ch = chains[c];
        for (uint32_t k = 0; k < ch.y; k++) {
            const MidLevelDesc &dsc = lev[ch.x + k];
            const unsigned long long t0 = global_ns();
            if (dsc.wbytes == 8) {
                if (dsc.mixed) mid_level<unsigned long long, true, CL>(dsc, cl, sm, slot, swin[wk], swinx[wk], swind[wk]);
                else mid_level<unsigned long long, false, CL>(dsc, cl, sm, slot, swin[wk], swinx[wk], swind[wk]);
            } else {
                if (dsc.mixed) mid_level<uint32_t, true, CL>(dsc, cl, sm, slot, swin[wk], swinx[wk], swind[wk]);
                else mid_level<uint32_t, false, CL>(dsc, cl, sm, slot, swin[wk], swinx[wk], swind[wk]);
            }
            // every block's part of the result is written before the next
            // level reads it, and every read of another block's slots is done
            cl.sync();
            if (cl.block_rank() == 0 && threadIdx.x == 0) dsc.res[6] = (double)(global_ns() - t0) * 1e-6;
        }
    }
}

// ----------------------------------------------------------- residual --
// |L x - lambda x|^2 partial sums per block (x unit-norm FP64 vector).
// normlap: the random-walk Laplacian I - D^-1 A instead of L = D - A.
// ||L x - lambda x||^2 and ||x||^2 of the finest level (the reference's
// eigenvalue log, eigensolve_kokkos.h:60-98, computes the same residual
// vector): one warp per row with four entries per lane in flight; rows of
// more than kResLongT entries are left to k_residual_long.
constexpr uint32_t kResLongT = 8192;

__device__ __forceinline__ double residual_term(int normlap, double xi, double acc, double d, double lambda) {
    return normlap ? xi - (d > 0 ? acc / d : 0.0) - lambda * xi : d * xi - acc - lambda * xi;
}

template <typename W>
__global__ void __launch_bounds__(256) k_residual(uint32_t n, const uint32_t *__restrict__ rp,
                                                 const uint32_t *__restrict__ col, const W *__restrict__ w,
                                                 const double *__restrict__ x, double lambda, int normlap,
                                                 double *part) {
    __shared__ double sm[96];
    double s[2] = {0, 0};
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = wid; i < n; i += nw) {
        const uint32_t b = rp[i], e = rp[i + 1];
        if (e - b > kResLongT) continue;   // warp-uniform: k_residual_long
        double acc = 0, d = 0;
        for (uint32_t j0 = b + lane; j0 < e; j0 += 128) {
            uint32_t c[4];
            double wt[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t j = j0 + 32 * k;
                c[k] = j < e ? col[j] : 0u;
                wt[k] = j < e ? (w ? (double)w[j] : 1.0) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (j0 + 32 * k < e) {
                    acc += wt[k] * x[c[k]];
                    d += wt[k];
                }
            }
        }
        acc = warp_sum(acc);
        d = warp_sum(d);
        if (lane == 0) {
            const double r = residual_term(normlap, x[i], acc, d, lambda);
            s[0] += r * r;
            s[1] += x[i] * x[i];
        }
    }
    block_sum_d<2>(s, sm);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = s[0]; part[2 * blockIdx.x + 1] = s[1]; }
}

// the rows of more than kResLongT entries (ascending list), a block each;
// lres[2 r], lres[2 r + 1] = r_i^2, x_i^2 of list entry r
template <typename W>
__global__ void __launch_bounds__(1024) k_residual_long(const uint32_t *__restrict__ rp,
                                                       const uint32_t *__restrict__ col, const W *__restrict__ w,
                                                       const double *__restrict__ x, double lambda, int normlap,
                                                       const uint32_t *__restrict__ list,
                                                       const uint32_t *__restrict__ cnt, double *lres) {
    __shared__ double sm[96];
    const uint32_t nl = *cnt;
    for (uint32_t r = blockIdx.x; r < nl; r += gridDim.x) {
        const uint32_t i = list[r];
        const uint32_t b = rp[i], e = rp[i + 1];
        double v[2] = {0, 0};
        for (uint32_t j0 = b + threadIdx.x; j0 < e; j0 += 4 * blockDim.x) {
            uint32_t c[4];
            double wt[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t j = j0 + k * blockDim.x;
                c[k] = j < e ? col[j] : 0u;
                wt[k] = j < e ? (w ? (double)w[j] : 1.0) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (j0 + k * blockDim.x < e) {
                    v[0] += wt[k] * x[c[k]];
                    v[1] += wt[k];
                }
            }
        }
        block_sum_d<2>(v, sm);   // ends with a barrier: sm is free for the next row
        if (threadIdx.x == 0) {
            const double t = residual_term(normlap, x[i], v[0], v[1], lambda);
            lres[2 * (size_t)r] = t * t;
            lres[2 * (size_t)r + 1] = x[i] * x[i];
        }
    }
}

__global__ void k_long_flags(uint32_t n, const uint32_t *rp, uint32_t T, uint8_t *f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = rp[i + 1] - rp[i] > T ? 1 : 0;
}

// the block partials in block order, then the long rows in ascending order
__global__ void k_sum_pairs(const double *part, uint32_t nb, const double *lres, const uint32_t *lcnt, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0, b = 0;
        for (uint32_t i = 0; i < nb; i++) { a += part[2 * i]; b += part[2 * i + 1]; }
        const uint32_t nl = lcnt ? *lcnt : 0u;
        for (uint32_t r = 0; r < nl; r++) { a += lres[2 * (size_t)r]; b += lres[2 * (size_t)r + 1]; }
        out[0] = a; out[1] = b;
    }
}

// block-wide rows: longer than T, or empty
__global__ void k_heavy_flags(uint32_t n, const uint32_t *rp, uint32_t T, uint8_t *f) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        uint32_t len = rp[i + 1] - rp[i];
        f[i] = (len > T || len == 0) ? 1 : 0;
    }
}

// Per-row cost used to give every block and warp an equal share: the row's
// entries rounded up to whole trips of 2^qs entries (the warp-row variants
// spend one trip on any row up to 128 entries; streaming has qs = 0) plus a
// fixed row overhead; block-wide rows cost nothing in the warp prefix.
__global__ void k_row_cost(uint32_t n, const uint32_t *rp, uint32_t T, uint32_t qs, uint32_t over, uint32_t shift,
                           uint32_t *cost, uint32_t *cost_all) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t len = rp[i + 1] - rp[i];
    const uint64_t trips = ((uint64_t)len + (1u << qs) - 1) >> qs;
    const uint32_t c = (uint32_t)(((trips << qs) + over) >> shift) + 1u;
    cost[i] = (len > T || len == 0) ? 0u : c;
    cost_all[i] = c;
}

// Segments of the block-wide rows: cnt[i] = segments of 2^shift entries of
// row i when it is longer than T, else 0.
__global__ void k_seg_counts(uint32_t n, const uint32_t *rp, uint32_t T, uint32_t shift, uint32_t *cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t len = rp[i + 1] - rp[i];
    cnt[i] = len > T ? (uint32_t)(((uint64_t)len + (1u << shift) - 1) >> shift) : 0u;
}

__global__ void k_seg_rows(uint32_t n, const uint32_t *hseg, uint32_t *seg_row) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t s = hseg[i]; s < hseg[i + 1]; s++) seg_row[s] = i;
}

// ------------------------------------------------------ column panels --
// Number of entries of a row below key (the row ascending by destination).
__device__ __forceinline__ uint32_t row_count_below(const uint32_t *col, uint32_t b, uint32_t e, uint32_t key) {
    uint32_t lo = b, hi = e;
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (col[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo - b;
}

// Lane l <= P of the warp holding row i gets the number of the row's entries
// in panels below l (0 for block-wide rows, which the panels leave out).
__device__ __forceinline__ uint32_t panel_bounds(const uint32_t *rp, const uint32_t *col, uint32_t i, uint32_t T,
                                                 uint32_t PW, uint32_t P, uint32_t &b, bool &skip) {
    const unsigned lane = threadIdx.x & 31;
    b = rp[i];
    const uint32_t e = rp[i + 1];
    skip = e - b > T || e == b;
    if (skip || lane > P) return 0;
    if (lane == P) return e - b;
    return lane == 0 ? 0u : row_count_below(col, b, e, lane * PW);
}

// cnt[p*n + i] = entries of warp row i in panel p (P <= 31)
__global__ void k_panel_count(uint32_t n, const uint32_t *rp, const uint32_t *col, uint32_t T, uint32_t PW,
                              uint32_t P, uint32_t *cnt) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        const uint32_t i = (uint32_t)r;
        uint32_t b;
        bool skip;
        const uint32_t lb = panel_bounds(rp, col, i, T, PW, P, b, skip);
        const uint32_t nb = __shfl_down_sync(0xFFFFFFFFu, lb, 1);
        if (lane < P) cnt[(size_t)lane * n + i] = skip ? 0u : nb - lb;
    }
}

// copy each warp row's panel segments to their panel-major places
template <typename W>
__global__ void k_panel_scatter(uint32_t n, const uint32_t *rp, const uint32_t *col, const W *w, uint32_t T,
                                uint32_t PW, uint32_t P, const uint32_t *off, uint16_t *pcol, W *pw) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        const uint32_t i = (uint32_t)r;
        uint32_t b;
        bool skip;
        const uint32_t lb = panel_bounds(rp, col, i, T, PW, P, b, skip);
        if (skip) continue;   // warp-uniform
        for (uint32_t p = 0; p < P; p++) {
            const uint32_t s0 = __shfl_sync(0xFFFFFFFFu, lb, p);
            const uint32_t s1 = __shfl_sync(0xFFFFFFFFu, lb, p + 1);
            const uint32_t d = off[(size_t)p * n + i];
            for (uint32_t k = s0 + lane; k < s1; k += 32) {
                pcol[d + k - s0] = (uint16_t)(col[b + k] - p * PW);
                if (w) pw[d + k - s0] = w[b + k];
            }
        }
    }
}

// *bad = 1 when some row is not ascending by destination
__global__ void k_rows_sorted(uint32_t n, const uint32_t *rp, const uint32_t *col, uint32_t *bad) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    bool ok = true;
    for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        const uint32_t b = rp[r], e = rp[r + 1];
        for (uint32_t j = b + lane; j + 1 < e; j += 32) ok = ok && col[j] <= col[j + 1];
    }
    if (__any_sync(0xFFFFFFFFu, !ok) && lane == 0) atomicOr(bad, 1u);
}

struct PanelLayout {
    uint32_t P = 0, PW = 0;
    uint32_t *off = nullptr;
    uint16_t *col = nullptr;
    void *w = nullptr;
    void *yacc = nullptr;
};

// Regroup the warp rows of L (rows of at most T entries) by column panel of
// kPanelBytes / vbytes iterate entries.  Leaves out->P = 0 when the level
// needs more than kMaxPanels panels.
static int build_panels(Context &C, const Level &L, uint32_t T, size_t vbytes, PanelLayout *out) {
    const uint32_t n = L.n;
    const uint32_t PW = (uint32_t)(kPanelBytes / vbytes);
    const uint32_t P = (uint32_t)cdiv(n, PW);
    *out = PanelLayout();
    if (P == 0 || P > kMaxPanels || (uint64_t)P * n >= 0xFFFFFFFFull) return SGP_B200_OK;
    uint32_t *cnt, *off, total = 0;
    const size_t pn = (size_t)P * n;
    SGPB_TRY(dalloc_t(C, &cnt, pn + 1));
    SGPB_TRY(dalloc_t(C, &off, pn + 1));
    uint32_t g = cdiv(n, 8);
    if (g > (uint32_t)C.num_sms * 16) g = C.num_sms * 16;
    k_panel_count<<<g, 256, 0, C.stream>>>(n, L.rp, L.col, T, PW, P, cnt);
    C.kernel_launches++;
    SGPB_TRY(scan_u32(C, cnt, off, (uint32_t)pn, nullptr));
    SGPB_TRY(read_u32(C, off + pn, &total));
    uint16_t *pcol;
    SGPB_TRY(dalloc_t(C, &pcol, (size_t)total + 256));
    void *pw = nullptr;
    if (L.w) {
        SGPB_TRY(dalloc(C, &pw, ((size_t)total + 256) * L.wbytes));
        if (L.wbytes == 8)
            k_panel_scatter<unsigned long long><<<g, 256, 0, C.stream>>>(n, L.rp, L.col, (const unsigned long long *)L.w,
                                                                         T, PW, P, off, pcol, (unsigned long long *)pw);
        else
            k_panel_scatter<uint32_t><<<g, 256, 0, C.stream>>>(n, L.rp, L.col, (const uint32_t *)L.w, T, PW, P, off,
                                                               pcol, (uint32_t *)pw);
    } else {
        k_panel_scatter<uint32_t><<<g, 256, 0, C.stream>>>(n, L.rp, L.col, nullptr, T, PW, P, off, pcol, nullptr);
    }
    C.kernel_launches++;
    SGPB_CUDA(cudaGetLastError());
    void *yacc;
    SGPB_TRY(dalloc(C, &yacc, (size_t)n * vbytes));
    out->P = P; out->PW = PW; out->off = off; out->col = pcol; out->w = pw; out->yacc = yacc;
    return SGP_B200_OK;
}

static uint32_t pi_grid(const Context &C, uint64_t n, uint64_t m, uint32_t units) {
    const uint64_t maxg = (uint64_t)2 * C.num_sms;   // two resident blocks per SM (launch bounds)
    // `units` cost units per thread (16 by the built-in rule): mid-size
    // levels are latency-bound, and more warps shorten each warp's serial
    // chain of rows (a 50k-vertex Erdos-Renyi graph: 63 -> 31 ms going from 64
    // to 16); levels large enough to fill the GPU are unaffected
    const uint64_t want = cdiv(m + 8 * n, (uint64_t)kPIThreads * units);
    uint64_t grid = want < maxg ? want : maxg;
    if (C.grid_cap && grid > C.grid_cap) grid = C.grid_cap;
    return (uint32_t)(grid < 1 ? 1 : grid);
}

// mean degree above which a level uses one warp per row
constexpr double kStreamMaxAvgDegree = 64.0;

// SpMV variant of a level: column panels when a panel layout was built for
// it, else CSR streaming below kStreamMaxAvgDegree and pipelined warp rows
// above; SGPB_PI_MODE = stream | row4 | rowp | panel overrides the rule.
struct PIVariant {
    int mode;   // 0 stream, 4 warp rows, 5 pipelined warp rows, 6 column panels, 7 staged warp rows
    bool na;
};
// Staged warp rows (mode 7) run only when SGPB_PI_MODE=staged asks for them,
// on a relabelled copy (whose arrays are padded for whole chunks): their ring
// of shared memory takes L1 capacity from the hub prefix of the gathers, and
// R-MAT scale 22's level 1 went from 173.5 to 393.7 ms with them.
static PIVariant pi_variant(const PIArgs &a) {
    PIVariant v;
    v.mode = (a.n && (double)a.m / a.n <= kStreamMaxAvgDegree) ? 0 : 5;
    v.na = true;
    if (const char *s = getenv("SGPB_PI_MODE")) {
        if (!strcmp(s, "stream")) v.mode = 0;
        else if (!strcmp(s, "row4")) v.mode = 4;
        else if (!strcmp(s, "rowp")) v.mode = 5;
        else if (!strcmp(s, "staged") && a.cache_ok == 3 && a.vec_ok) v.mode = 7;
    }
    if (a.P) v.mode = 6;
    return v;
}

// whether a level gets a column-panel layout (SGPB_PI_MODE=panel; rows
// ascending by destination, in the level's own numbering).  Off by default:
// on R-MAT levels the per-panel block barriers cost more than the shared-
// memory gathers save (measured 2x slower than pipelined warp rows).
// Levels whose layout would need more than kMaxPanels panels (or 2^32
// panel-row offsets) keep their rule variant.
static bool panels_wanted(const Level &L, const PIArgs &a) {
    if (a.inv || L.n == 0) return false;
    const char *s = getenv("SGPB_PI_MODE");
    if (!s || strcmp(s, "panel")) return false;
    const uint64_t P = cdiv((uint64_t)L.n, (uint64_t)(kPanelBytes / sizeof(double)));
    return P <= kMaxPanels && P * L.n < 0xFFFFFFFFull;
}

template <typename W, typename V, int CACHE, bool MX>
static const void *pi_kernel_c(int mode) {
    if (mode == 0) return (const void *)k_power_iter<W, V, 0, true, CACHE, MX>;
    if (mode == 5) return (const void *)k_power_iter<W, V, 5, true, CACHE, MX>;
    if constexpr (CACHE == kCacheSplit)
        if (mode == 7) return (const void *)k_power_iter<W, V, 7, true, kCacheSplit, MX>;
    if constexpr (sizeof(W) >= 4 && !MX)
        if (mode == 6) return (const void *)k_power_iter<W, V, 6, true, kCacheNone, false>;
    return (const void *)k_power_iter<W, V, 4, true, CACHE, MX>;
}

template <typename W, typename V, bool MX>
static int launch_pi(Context &C, PIArgs &a, uint32_t grid, int mode) {
    if (mode == 6 && !a.P) {   // column panels need their layout
        set_error("power iteration: column-panel variant without a panel layout");
        return SGP_B200_ERR_INVALID;
    }
    PIVariant var;
    var.mode = a.P ? 6 : mode;
    var.na = true;
    const size_t cache_bytes = var.mode == 0 ? kCacheBytesStream : kCacheBytesRows;
    const uint64_t kmax = cache_bytes / sizeof(V);
    // cache_ok: 2 = the whole iterate in shared memory when it fits, 3 =
    // relabelled copy (L1 policy by hub prefix), 0 = off
    a.kcache = (a.cache_ok == 2 && a.n <= kmax) ? (uint32_t)a.n : 0u;
    const bool split = a.cache_ok == 3 && var.mode != 6;
    if (split) a.kcache = (uint32_t)(a.n < split_bytes() / sizeof(V) ? a.n : split_bytes() / sizeof(V));
    if (var.mode == 6) a.kcache = 0;
    const void *k = nullptr;
    if constexpr (sizeof(W) < 4) {
        // narrow weights exist only in relabelled copies, which use the split
        if (!split) {
            set_error("narrow weights outside a relabelled copy");
            return SGP_B200_ERR_INVALID;
        }
        k = pi_kernel_c<W, V, kCacheSplit, MX>(var.mode);
    } else {
        k = split ? pi_kernel_c<W, V, kCacheSplit, MX>(var.mode)
                  : a.kcache ? pi_kernel_c<W, V, kCachePrefix, MX>(var.mode)
                             : pi_kernel_c<W, V, kCacheNone, MX>(var.mode);
    }
    const size_t dyn = var.mode == 7   ? (size_t)kPIWarps * StageCfg<W>::warp_bytes
                       : var.mode == 6 ? (size_t)a.PW * sizeof(V)
                       : split         ? 0
                                       : (size_t)a.kcache * sizeof(V);
    if (var.mode == 7)
        SGPB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    else if (var.mode == 6)
        SGPB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelBytes));
    else if (a.kcache && !split)
        SGPB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cache_bytes));
    int per_sm = 0;
    // shared-memory carveout preference in percent (SGPB_PI_CARVEOUT; -1 =
    // the driver's choice)
    if (const char *cv = getenv("SGPB_PI_CARVEOUT"))
        SGPB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, atoi(cv)));
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kPIThreads, dyn));
    if (per_sm < 1) {
        set_error("power-iteration kernel does not fit on an SM");
        return SGP_B200_ERR_DEVICE;
    }
    if ((uint64_t)grid > (uint64_t)per_sm * C.num_sms) grid = per_sm * C.num_sms;
    SGPB_TRY(dalloc_t(C, &a.partials, (size_t)2 * grid * kNP));
    SGPB_TRY(dalloc_t(C, &a.err, 1));
    SGPB_TRY(dzero(C, a.err, sizeof(uint32_t)));
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kPIThreads), args, dyn, C.stream));
    C.kernel_launches++;
    return SGP_B200_OK;
}

// Runs one level's iterations: the one-block shared-memory kernel for small
// levels, else the cooperative kernel (column panels when a layout is given).
// mixed: FP32 edge-difference arithmetic (never with panels or small levels).
static int run_pi(Context &C, const Level &L, PIArgs a, bool mixed, const PanelLayout *panels, double *res_d,
                  double res_h[5], float *ms, uint32_t grid, int mode) {
    a.res = res_d;
    a.P = 0;
    if (panels) {
        a.P = panels->P; a.PW = panels->PW; a.poff = panels->off; a.pcol = panels->col; a.pw = panels->w;
        a.yacc = panels->yacc;
    }
    int rc;
    cudaEvent_t e0, e1;
    SGPB_CUDA(cudaEventCreate(&e0));
    SGPB_CUDA(cudaEventCreate(&e1));
    // levels of at most kSmallCost cost units that fit in shared memory (not
    // when SGPB_PI_MODE forces a variant of the main kernel)
    const char *forced = getenv("SGPB_PI_MODE");
    const bool small = !mixed && !(forced && *forced) && !a.P && !a.inv && L.m + 8ull * L.n <= kSmallCost &&
                       (L.wbytes == 0 || L.wbytes == 4 || L.wbytes == 8) &&
                       small_level_bytes<unsigned long long, double>(L.n, L.m, L.w != nullptr) <= kSmallSmemBytes;
    if (small) {
        auto launch_small = [&](auto wtag) -> int {
            using Wt = decltype(wtag);
            const size_t bytes = small_level_bytes<Wt, double>(L.n, L.m, L.w != nullptr);
            const void *k = (const void *)k_power_iter_small<Wt, double>;
            // the limit is a property of the function, shared by every host
            // thread (batch workers): always the same bound, never this
            // launch's size, so no thread lowers it under another's launch
            SGPB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmemBytes));
            SGPB_CUDA(cudaEventRecord(e0, C.stream));
            k_power_iter_small<Wt, double><<<1, kSmallThreads, bytes, C.stream>>>(a);
            C.kernel_launches++;
            return SGP_B200_OK;
        };
        rc = L.wbytes == 8 ? launch_small((unsigned long long)0) : launch_small((uint32_t)0);
    } else {
        double *va, *vb;
        SGPB_TRY(dalloc_t(C, &va, L.n));
        SGPB_TRY(dalloc_t(C, &vb, L.n));
        a.va = va; a.vb = vb;
        // partials are allocated inside launch_pi; the events bracket the launch
        SGPB_CUDA(cudaEventRecord(e0, C.stream));
        auto go = [&](auto mx) -> int {
            constexpr bool M = decltype(mx)::value;
            if (L.wbytes == 8) return launch_pi<unsigned long long, double, M>(C, a, grid, mode);
            if (L.wbytes == 2) return launch_pi<uint16_t, double, M>(C, a, grid, mode);
            if (L.wbytes == 1) return launch_pi<uint8_t, double, M>(C, a, grid, mode);
            return launch_pi<uint32_t, double, M>(C, a, grid, mode);
        };
        rc = mixed ? go(std::true_type()) : go(std::false_type());
    }
    cudaEventRecord(e1, C.stream);
    if (rc != SGP_B200_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
    SGPB_CUDA(cudaGetLastError());
    SGPB_CUDA(cudaMemcpyAsync(C.h_pinned, res_d, 6 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    memcpy(res_h, C.h_pinned, 5 * sizeof(double));
    if (!small && ((const double *)C.h_pinned)[5] != 0.0) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        set_error("power iteration: a staged bulk copy of the matrix did not complete within its wait limit");
        return SGP_B200_ERR_DEVICE;
    }
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms += t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return SGP_B200_OK;
}

__global__ void k_max_deg(uint32_t n, const uint32_t *rp, uint32_t *out) {
    uint32_t mx = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t d = rp[i + 1] - rp[i];
        mx = d > mx ? d : mx;
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(out, mx);
}

int hub_first_copy(Context &C, const Level &L, uint32_t **perm_out, uint32_t **inv_out, Level *out);

// the reference's cap (eigensolve_kokkos.h:153) is 1e14 / n, unbounded in
// practice for small levels; a default budget of 5e6 iterations turns a
// non-converging level into a reported cap instead of an endless kernel.
static uint64_t iter_budget(uint32_t n, const PowerIterOpts &o) {
    uint64_t imax = 100000000000000ULL / (uint64_t)n;
    const uint64_t cap = o.iter_cap ? o.iter_cap : 5000000ULL;
    return imax > cap ? cap : imax;
}

// The work split of a level for variant t.mode (0 streaming, 5 or 7 warp
// rows, 6 panels): rows longer than a warp's cost share / t.heavy_div are
// block-wide (cut into 2^kSegShift-entry segments shared by the block's
// warps), the others are cut into equal-cost warp ranges; per-row costs
// count whole trips of the variant plus a row overhead.  Sets a.heavy_T,
// a.heavy, a.n_heavy_ptr, a.hseg, a.seg_row, a.hpart, a.cpre, a.cpre_all
// and allocates a.deg.
static int setup_split(Context &C, const Level &L, const PITune &t, PIArgs &a) {
    const uint32_t n = L.n;
    const int mode = t.mode;
    const uint64_t nwarps = (uint64_t)pi_grid(C, n, L.m, t.units) * kPIWarps;
    uint64_t T = (L.m + 8ull * n) / nwarps / (t.heavy_div ? t.heavy_div : 1);
    if (T < 4ull * kTile) T = 4ull * kTile;
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
    SGPB_TRY(dalloc_t(C, &a.deg, (size_t)n + 1));
    k_heavy_flags<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, a.heavy_T, flags);
    // the cost total is kept in 32 bits
    const uint32_t qs = (mode == 4 || mode == 5) ? 7u : mode == 7 ? 8u : 0u;   // trip of 128 / 256 entries
    const uint32_t over = (mode == 4 || mode == 5 || mode == 7) ? 32u : 8u;
    uint32_t shift = 0;
    while ((L.m + ((1ull << qs) + over + 1) * (uint64_t)n) >> shift >= 0xFFFFFFF0ull) shift++;
    k_row_cost<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, a.heavy_T, qs, over, shift, cost, cost_all);
    C.kernel_launches += 2;
    SGPB_TRY(compact_flags(C, flags, n, heavy, nh));
    {
        // rows longer than T have more than 512 entries: at most m / 512 of them
        const uint64_t max_segs = (L.m >> kSegShift) + L.m / (4ull * kTile) + 1;
        uint32_t *segc, *hseg, *seg_row;
        double *hpart;
        SGPB_TRY(dalloc_t(C, &segc, (size_t)n + 1));
        SGPB_TRY(dalloc_t(C, &hseg, (size_t)n + 1));
        SGPB_TRY(dalloc_t(C, &seg_row, max_segs));
        SGPB_TRY(dalloc_t(C, &hpart, max_segs));
        k_seg_counts<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, a.heavy_T, kSegShift, segc);
        SGPB_TRY(scan_u32(C, segc, hseg, n, nullptr));
        k_seg_rows<<<cdiv(n, 256), 256, 0, C.stream>>>(n, hseg, seg_row);
        C.kernel_launches += 2;
        a.hseg = hseg; a.seg_row = seg_row; a.hpart = hpart; a.seg_shift = kSegShift;
    }
    SGPB_TRY(scan_u32(C, cost, cpre, n, nullptr));
    SGPB_TRY(scan_u32(C, cost_all, cpre_all, n, nullptr));
    a.heavy = heavy; a.n_heavy_ptr = nh; a.cpre = cpre; a.cpre_all = cpre_all;
    return SGP_B200_OK;
}

// levels below this cost (entries + 8 per vertex) keep the built-in rule
constexpr uint64_t kTuneMinCost = 1ull << 18;
constexpr uint64_t kTuneIters = 10;   // trial iterations per candidate split

// Shape of a level for the autotuner's cache: weight width, relabelled copy
// or not, arithmetic, and the octave of the vertex count and the half octave
// of the mean degree.
static std::string tune_key(const Level &L, const PIArgs &a, bool mixed) {
    const double avg = L.n ? (double)L.m / L.n : 0;
    int ln = 0;
    while ((1ull << (ln + 1)) <= L.n) ln++;
    const int ld = avg >= 1 ? (int)floor(2.0 * log2(avg)) : 0;
    char k[96];
    snprintf(k, sizeof(k), "w%d_r%d_x%d_n%d_d%d", L.wbytes, a.cache_ok == 3 ? 1 : 0, mixed ? 1 : 0, ln, ld);
    return k;
}

// The first time a level of this shape is met on this device: run each
// candidate split for kTuneIters iterations from the level's start vector
// (into a scratch output, so the level's own run is untouched) and keep the
// fastest.  Candidates: both variants where the mean degree leaves the choice
// open (8 .. 512), long-row divisors of half, one and two times the rule's,
// then grid units of 8 and 32 for the best of those.  `t` holds the rule on
// entry and the choice on return.
static int autotune_level(Context &C, const Level &L, const PIArgs &a0, bool mixed, const PowerIterOpts &o,
                          PITune &t) {
    const std::string key = tune_key(L, a0, mixed);
    if (tune_lookup(C, key, &t)) return SGP_B200_OK;
    tune_lock();
    struct Unlock {
        ~Unlock() { tune_unlock(); }
    } unlock;
    if (tune_lookup(C, key, &t)) return SGP_B200_OK;   // tuned by another thread meanwhile
    const PITune rule = t;
    double *scratch, *res_d;
    SGPB_TRY(dalloc_t(C, &scratch, L.n));
    SGPB_TRY(dalloc_t(C, &res_d, 8));
    auto trial = [&](const PITune &c, double *ms) -> int {
        PIArgs a = a0;
        SGPB_TRY(setup_split(C, L, c, a));
        a.out = scratch;
        a.iter_max = kTuneIters;
        a.tol = -1.0;   // run exactly kTuneIters iterations
        double rh[5];
        float k = 0;
        SGPB_TRY(run_pi(C, L, a, mixed, nullptr, res_d, rh, &k, pi_grid(C, L.n, L.m, c.units), c.mode));
        *ms = k;
        return SGP_B200_OK;
    };
    const double avg = (double)L.m / L.n;
    std::vector<int> modes;
    if (avg >= 8.0 && avg <= 512.0) modes = {0, 5};
    else modes = {rule.mode};
    PITune best = rule;
    double best_ms = 1e300, rule_ms = 0;
    for (int m : modes) {
        const uint32_t base = (uint32_t)(m == 0 ? kHeavyDivStream : kHeavyDivRows);
        for (uint32_t div : {base / 2, base, base * 2}) {
            PITune c;
            c.mode = m;
            c.heavy_div = div;
            c.units = 16;
            double ms = 0;
            SGPB_TRY(trial(c, &ms));
            if (c.mode == rule.mode && c.heavy_div == rule.heavy_div && c.units == rule.units) rule_ms = ms;
            if (ms < best_ms) { best_ms = ms; best = c; }
        }
    }
    for (uint32_t u : {8u, 32u}) {
        PITune c = best;
        c.units = u;
        double ms = 0;
        SGPB_TRY(trial(c, &ms));
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    (void)o;
    t = best;
    tune_store(C, key, best, best_ms, rule_ms);
    return SGP_B200_OK;
}

int power_iter_level(Context &C, const Level &Lin, const double *x_in, const uint32_t *vcmap, double *x_out,
                     const PowerIterOpts &o, PowerIterResult *res, int want_residual) {
    const uint32_t n = Lin.n;
    if (n == 0) { *res = PowerIterResult(); return SGP_B200_OK; }
    if (power_iter_small_ok(Lin, o)) {
        // one block in shared memory: a chain of one level, none of the
        // row-cost tables of the multi-block kernel
        PIChain ch;
        ch.x0 = x_in;
        PIChainLevel cl;
        cl.L = &Lin;
        cl.vcmap = vcmap;
        cl.x_out = x_out;
        ch.lev.push_back(cl);
        SGPB_TRY(power_iter_chains(C, {&ch}, o));
        *res = ch.lev[0].res;
        if (want_residual) SGPB_TRY(level_residual(C, Lin, x_out, o.normlap, res));
        return SGP_B200_OK;
    }
    if (power_iter_mid_ok(Lin, o)) {
        // one cluster: a mid-size chain of one level
        PIChain ch;
        ch.x0 = x_in;
        PIChainLevel cl;
        cl.L = &Lin;
        cl.vcmap = vcmap;
        cl.x_out = x_out;
        ch.lev.push_back(cl);
        SGPB_TRY(power_iter_mid_chains(C, {&ch}, o));
        *res = ch.lev[0].res;
        if (want_residual) SGPB_TRY(level_residual(C, Lin, x_out, o.normlap, res));
        return SGP_B200_OK;
    }
    PIArgs a;
    memset(&a, 0, sizeof(a));
    // A level whose whole iterate fits in 96 KB keeps it in shared memory.
    // Skewed levels larger than the L1 hub prefix iterate on a hub-first
    // relabelled copy: the most referenced entries then sit densely at the
    // front of the iterate and are gathered with L1 evict-last priority while
    // all other gathers bypass L1 allocation (measured on R-MAT scale 22
    // level 1: 206 -> 187 ms).  SGPB_PI_RELABEL=0 turns the copy off.
    a.cache_ok = 2;
    Level L = Lin;
    {
        const double avg = (double)Lin.m / n;
        bool relabel = o.allow_relabel && n > kSplitBytes / sizeof(double) && avg >= 8.0;
        const char *rs = getenv("SGPB_PI_RELABEL");
        if (rs && atoi(rs) == 0) relabel = false;
        if (relabel) {
            uint32_t *mx, hmx = 0;
            SGPB_TRY(dalloc_t(C, &mx, 1));
            SGPB_TRY(dzero(C, mx, 4));
            uint32_t blocks = cdiv(n, 256);
            if (blocks > (uint32_t)C.num_sms * 8) blocks = C.num_sms * 8;
            k_max_deg<<<blocks, 256, 0, C.stream>>>(n, Lin.rp, mx);
            C.kernel_launches++;
            SGPB_TRY(read_u32(C, mx, &hmx));
            relabel = hmx >= 8.0 * avg;
        }
        if (relabel) {
            uint32_t *perm = nullptr, *inv = nullptr;
            SGPB_TRY(hub_first_copy(C, Lin, &perm, &inv, &L));
            a.inv = inv;
            a.cache_ok = 3;
        }
    }
    a.n = n; a.m = L.m; a.rp = L.rp; a.col = L.col; a.w = L.w;
    a.normlap = o.normlap;
    a.vec_ok = (((uintptr_t)L.col | (uintptr_t)L.w) & 15u) == 0;
    // mixed-precision arithmetic for levels of at least 4096 vertices (the
    // smaller ones are latency-bound and run in FP64)
    const bool mixed = o.mixed && n >= 4096;
    // the variant decides the heavy-row threshold and the cost model
    bool want_panels = !mixed && panels_wanted(L, a);
    if (want_panels && !L.sorted) {
        uint32_t *bad, hbad = 0;
        SGPB_TRY(dalloc_t(C, &bad, 1));
        SGPB_TRY(dzero(C, bad, 4));
        uint32_t g = cdiv(n, 8);
        if (g > (uint32_t)C.num_sms * 16) g = C.num_sms * 16;
        k_rows_sorted<<<g, 256, 0, C.stream>>>(n, L.rp, L.col, bad);
        C.kernel_launches++;
        SGPB_TRY(read_u32(C, bad, &hbad));
        want_panels = hbad == 0;
    }
    const int rule_mode = want_panels ? 6 : pi_variant(a).mode;
    a.x_in = x_in; a.vcmap = vcmap;
    // the work split: the built-in rule, or the autotuner's choice for
    // levels of this shape on this device (trial iterations the first time)
    PITune tune;
    tune.mode = rule_mode;
    tune.heavy_div = (uint32_t)(rule_mode == 0 ? kHeavyDivStream : kHeavyDivRows);
    tune.units = 16;
    const char *forced = getenv("SGPB_PI_MODE");
    if (!want_panels && !(forced && *forced) && (rule_mode == 0 || rule_mode == 5) && autotune_enabled() &&
        L.m + 8ull * n >= kTuneMinCost)
        SGPB_TRY(autotune_level(C, L, a, mixed, o, tune));
    SGPB_TRY(setup_split(C, L, tune, a));
    a.out = x_out;
    const uint64_t imax = iter_budget(n, o);
    a.iter_max = imax;
    a.tol = o.tol;
    double *res_d;
    SGPB_TRY(dalloc_t(C, &res_d, 8));
    double rh[5];
    float kms = 0;
    PanelLayout panels;
    if (want_panels) SGPB_TRY(build_panels(C, L, a.heavy_T, sizeof(double), &panels));
    SGPB_TRY(run_pi(C, L, a, mixed, want_panels ? &panels : nullptr, res_d, rh, &kms, pi_grid(C, n, L.m, tune.units),
                    tune.mode));
    const uint64_t total_iters = (uint64_t)rh[0];
    res->niter = total_iters;
    res->dot = rh[1];
    res->gb = rh[2];
    res->lambda = rh[3];
    res->capped = rh[4] != 0.0;
    res->resid = 0;
    res->kernel_ms = kms;
    // the result is in the level's own numbering: use the level itself
    if (want_residual) SGPB_TRY(level_residual(C, Lin, x_out, o.normlap, res));
    return SGP_B200_OK;
}

int level_residual(Context &C, const Level &L, const double *x, int normlap, PowerIterResult *res) {
    const uint32_t n = L.n;
    uint32_t nb = C.num_sms * 4;
    double *part, *out2;
    SGPB_TRY(dalloc_t(C, &part, 2 * (size_t)nb));
    SGPB_TRY(dalloc_t(C, &out2, 2));
    // rows of more than kResLongT entries: an ascending list, a block each
    double *lres = nullptr;
    uint32_t *lcnt = nullptr, *llist = nullptr;
    if (L.m > kResLongT && n) {
        uint8_t *flags;
        const uint64_t maxl = L.m / kResLongT + 1;
        SGPB_TRY(dalloc_t(C, &flags, n));
        SGPB_TRY(dalloc_t(C, &llist, (size_t)n + 1));
        SGPB_TRY(dalloc_t(C, &lcnt, 1));
        SGPB_TRY(dalloc_t(C, &lres, 2 * maxl));
        k_long_flags<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, kResLongT, flags);
        C.kernel_launches++;
        SGPB_TRY(compact_flags(C, flags, n, llist, lcnt));
    }
    const uint32_t gl = (uint32_t)(L.m / kResLongT + 1 < (uint64_t)C.num_sms * 2 ? L.m / kResLongT + 1
                                                                                 : (uint64_t)C.num_sms * 2);
    if (L.wbytes == 8) {
        k_residual<unsigned long long><<<nb, 256, 0, C.stream>>>(n, L.rp, L.col, (const unsigned long long *)L.w, x,
                                                                 res->lambda, normlap, part);
        if (lcnt)
            k_residual_long<unsigned long long><<<gl, 1024, 0, C.stream>>>(
                L.rp, L.col, (const unsigned long long *)L.w, x, res->lambda, normlap, llist, lcnt, lres);
    } else {
        k_residual<uint32_t><<<nb, 256, 0, C.stream>>>(n, L.rp, L.col, (const uint32_t *)L.w, x, res->lambda,
                                                       normlap, part);
        if (lcnt)
            k_residual_long<uint32_t><<<gl, 1024, 0, C.stream>>>(L.rp, L.col, (const uint32_t *)L.w, x, res->lambda,
                                                                 normlap, llist, lcnt, lres);
    }
    k_sum_pairs<<<1, 32, 0, C.stream>>>(part, nb, lres, lcnt, out2);
    C.kernel_launches += lcnt ? 3 : 2;
    SGPB_CUDA(cudaGetLastError());
    SGPB_CUDA(cudaMemcpyAsync(C.h_pinned, out2, 2 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    double r2 = ((double *)C.h_pinned)[0], x2 = ((double *)C.h_pinned)[1];
    const double scale = normlap ? 2.0 : (res->gb > 0 ? res->gb : 1);   // bound on the spectrum
    res->resid = sqrt(r2 / (x2 > 0 ? x2 : 1)) / scale;
    return SGP_B200_OK;
}

bool power_iter_small_ok(const Level &L, const PowerIterOpts &o) {
    const char *forced = getenv("SGPB_PI_MODE");
    if (forced && *forced) return false;
    if (L.n == 0 || L.m + 8ull * L.n > kSmallCost) return false;
    if (!(L.wbytes == 0 || L.wbytes == 4 || L.wbytes == 8)) return false;
    return small_level_bytes<unsigned long long, double>(L.n, L.m, L.w != nullptr) <= kSmallSmemBytes;
}

int power_iter_chains(Context &C, const std::vector<PIChain *> &chains, const PowerIterOpts &o) {
    std::vector<PIChainDesc> h;
    std::vector<std::pair<uint64_t, uint2>> order;   // (cost, chain) for largest-first
    size_t bytes = 0;
    for (PIChain *ch : chains) {
        if (!ch || ch->lev.empty()) continue;
        uint2 c = make_uint2((uint32_t)h.size(), (uint32_t)ch->lev.size());
        uint64_t cost = 0;
        for (size_t k = 0; k < ch->lev.size(); k++) {
            const PIChainLevel &cl = ch->lev[k];
            const Level &L = *cl.L;
            if (!power_iter_small_ok(L, o)) {
                set_error("level of %u vertices and %llu entries is not a small level", L.n,
                          (unsigned long long)L.m);
                return SGP_B200_ERR_INVALID;
            }
            PIChainDesc d;
            memset(&d, 0, sizeof(d));
            d.a.n = L.n; d.a.m = L.m; d.a.rp = L.rp; d.a.col = L.col; d.a.w = L.w;
            d.a.x_in = k == 0 ? ch->x0 : ch->lev[k - 1].x_out;
            d.a.vcmap = cl.vcmap;
            d.a.out = cl.x_out;
            d.a.tol = o.tol;
            d.a.iter_max = iter_budget(L.n, o);
            d.a.normlap = o.normlap;
            d.wbytes = L.wbytes;
            h.push_back(d);
            cost += L.m + 8ull * L.n;
            const size_t b = L.wbytes == 8 ? small_level_bytes<unsigned long long, double>(L.n, L.m, L.w != nullptr)
                                           : small_level_bytes<uint32_t, double>(L.n, L.m, L.w != nullptr);
            bytes = b > bytes ? b : bytes;
        }
        order.push_back({cost, c});
    }
    if (h.empty()) return SGP_B200_OK;
    std::stable_sort(order.begin(), order.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    std::vector<uint2> hc(order.size());
    for (size_t i = 0; i < order.size(); i++) hc[i] = order[i].second;
    double *res_d;
    SGPB_TRY(dalloc_t(C, &res_d, 8 * h.size()));
    for (size_t i = 0; i < h.size(); i++) h[i].a.res = res_d + 8 * i;
    PIChainDesc *lev_d;
    uint2 *ch_d;
    uint32_t *next;
    SGPB_TRY(dalloc_t(C, &lev_d, h.size()));
    SGPB_TRY(dalloc_t(C, &ch_d, hc.size()));
    SGPB_TRY(dalloc_t(C, &next, 1));
    SGPB_CUDA(cudaMemcpyAsync(lev_d, h.data(), sizeof(PIChainDesc) * h.size(), cudaMemcpyHostToDevice, C.stream));
    SGPB_CUDA(cudaMemcpyAsync(ch_d, hc.data(), sizeof(uint2) * hc.size(), cudaMemcpyHostToDevice, C.stream));
    SGPB_TRY(dzero(C, next, 4));
    // one fixed bound for every launch (host threads share the attribute)
    SGPB_CUDA(cudaFuncSetAttribute(k_power_iter_chains, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kSmallSmemBytes));
    const uint32_t grid = (uint32_t)(hc.size() < (size_t)C.num_sms ? hc.size() : (size_t)C.num_sms);
    k_power_iter_chains<<<grid, kSmallThreads, bytes, C.stream>>>(lev_d, ch_d, (uint32_t)hc.size(), next);
    C.kernel_launches++;
    SGPB_CUDA(cudaGetLastError());
    std::vector<double> rh(8 * h.size());
    SGPB_CUDA(cudaMemcpyAsync(rh.data(), res_d, sizeof(double) * rh.size(), cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    size_t i = 0;
    for (PIChain *ch : chains) {
        if (!ch) continue;
        for (PIChainLevel &cl : ch->lev) {
            const double *r = &rh[8 * i++];
            cl.res = PowerIterResult();
            cl.res.niter = (uint64_t)r[0];
            cl.res.dot = r[1];
            cl.res.gb = r[2];
            cl.res.lambda = r[3];
            cl.res.capped = r[4] != 0.0;
            cl.res.kernel_ms = (float)r[6];
        }
    }
    return SGP_B200_OK;
}

bool power_iter_mid_ok(const Level &L, const PowerIterOpts &o) {
    const char *forced = getenv("SGPB_PI_MODE");
    if (forced && *forced) return false;
    if (const char *e = getenv("SGPB_PI_MID"))
        if (atoi(e) == 0) return false;
    if (L.n == 0 || power_iter_small_ok(L, o)) return false;
    if (!(L.wbytes == 0 || L.wbytes == 4 || L.wbytes == 8)) return false;
    return L.m + 8ull * L.n <= (o.mid_limit ? o.mid_limit : kMidCost);
}

int power_iter_mid_chains(Context &C, const std::vector<PIChain *> &chains, const PowerIterOpts &o) {
    std::vector<MidLevelDesc> h;
    std::vector<std::pair<uint64_t, uint2>> order;   // (cost, chain) for largest-first
    for (PIChain *ch : chains) {
        if (!ch || ch->lev.empty()) continue;
        uint2 c = make_uint2((uint32_t)h.size(), (uint32_t)ch->lev.size());
        uint64_t cost = 0;
        for (size_t k = 0; k < ch->lev.size(); k++) {
            const PIChainLevel &cl = ch->lev[k];
            const Level &L = *cl.L;
            if (!power_iter_mid_ok(L, o)) {
                set_error("level of %u vertices and %llu entries is not a mid-size level", L.n,
                          (unsigned long long)L.m);
                return SGP_B200_ERR_INVALID;
            }
            MidLevelDesc d;
            memset(&d, 0, sizeof(d));
            d.n = L.n; d.m = L.m; d.rp = L.rp; d.col = L.col; d.w = L.w; d.wbytes = L.wbytes;
            d.mixed = o.mixed && L.n >= 4096;
            d.normlap = o.normlap;
            d.vec_ok = (((uintptr_t)L.col | (uintptr_t)L.w) & 15u) == 0;
            d.x_in = k == 0 ? ch->x0 : ch->lev[k - 1].x_out;
            d.vcmap = cl.vcmap;
            d.out = cl.x_out;
            SGPB_TRY(dalloc_t(C, &d.va, L.n));
            SGPB_TRY(dalloc_t(C, &d.vb, L.n));
            SGPB_TRY(dalloc_t(C, &d.deg, L.n));
            d.tol = o.tol;
            d.iter_max = iter_budget(L.n, o);
            h.push_back(d);
            cost += L.m + 8ull * L.n;
        }
        order.push_back({cost, c});
    }
    if (h.empty()) return SGP_B200_OK;
    std::stable_sort(order.begin(), order.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    std::vector<uint2> hc(order.size());
    for (size_t i = 0; i < order.size(); i++) hc[i] = order[i].second;
    double *res_d;
    SGPB_TRY(dalloc_t(C, &res_d, 8 * h.size()));
    for (size_t i = 0; i < h.size(); i++) h[i].res = res_d + 8 * i;
    MidLevelDesc *lev_d;
    uint2 *ch_d;
    uint32_t *next;
    SGPB_TRY(dalloc_t(C, &lev_d, h.size()));
    SGPB_TRY(dalloc_t(C, &ch_d, hc.size()));
    SGPB_TRY(dalloc_t(C, &next, 1));
    SGPB_CUDA(cudaMemcpyAsync(lev_d, h.data(), sizeof(MidLevelDesc) * h.size(), cudaMemcpyHostToDevice, C.stream));
    SGPB_CUDA(cudaMemcpyAsync(ch_d, hc.data(), sizeof(uint2) * hc.size(), cudaMemcpyHostToDevice, C.stream));
    SGPB_TRY(dzero(C, next, 4));
    // as many clusters as fit at once (the queue balances the rest); CL
    // blocks a cluster: 8 for single partitions (latency of each level), 2
    // for batches (more hierarchies iterate at once)
    const int CLn = o.mid_blocks ? o.mid_blocks : kMidCTAs;
    auto launch = [&](auto tag) -> int {
        constexpr int CL = decltype(tag)::value;
        const void *k = (const void *)k_power_iter_mid<CL>;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3(CL);
        cfg.blockDim = dim3(kMidThreads);
        cfg.stream = C.stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int max_clusters = 0;
        SGPB_CUDA(cudaOccupancyMaxActiveClusters(&max_clusters, k, &cfg));
        if (max_clusters < 1) {
            set_error("the mid-size power-iteration cluster does not fit on the device");
            return SGP_B200_ERR_DEVICE;
        }
        const uint32_t nclu = (uint32_t)(hc.size() < (size_t)max_clusters ? hc.size() : (size_t)max_clusters);
        cfg.gridDim = dim3(nclu * CL);
        const uint32_t nch = (uint32_t)hc.size();
        SGPB_CUDA(cudaLaunchKernelEx(&cfg, k_power_iter_mid<CL>, (const MidLevelDesc *)lev_d, (const uint2 *)ch_d, nch,
                                     next));
        return SGP_B200_OK;
    };
    if (CLn == 2) SGPB_TRY(launch(std::integral_constant<int, 2>()));
    else if (CLn == 8) SGPB_TRY(launch(std::integral_constant<int, 8>()));
    else {
        set_error("cluster_blocks must be 2 or 8 (got %d)", CLn);
        return SGP_B200_ERR_INVALID;
    }
    C.kernel_launches++;
    SGPB_CUDA(cudaGetLastError());
    std::vector<double> rh(8 * h.size());
    SGPB_CUDA(cudaMemcpyAsync(rh.data(), res_d, sizeof(double) * rh.size(), cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    size_t i = 0;
    for (PIChain *ch : chains) {
        if (!ch) continue;
        for (PIChainLevel &cl : ch->lev) {
            const double *r = &rh[8 * i++];
            cl.res = PowerIterResult();
            cl.res.niter = (uint64_t)r[0];
            cl.res.dot = r[1];
            cl.res.gb = r[2];
            cl.res.lambda = r[3];
            cl.res.capped = r[4] != 0.0;
            cl.res.kernel_ms = (float)r[6];
        }
    }
    return SGP_B200_OK;
}

}  // namespace sgpb
