// coarsen_alt.cu -- the reference's alternative coarseners (the HEC
// mapping is hec.cu), chosen by sgp_b200_options_t.coarsener:
//
//   MATCH  heavy-edge matching: cmg/heuristics.h:1584-1740 (sgp_coarsen_match
//          as built with PUREMATCH: proposal rounds along the heaviest edge,
//          retries along the heaviest unmatched edge, singletons at the end)
//   MIS2   aggregation around a distance-2 maximal independent set:
//          heuristics.h:8-80 (mis_2) and :218-310 (sgp_coarsen_mis_2)
//   GOSH   aggregation around high-degree cluster centres: heuristics.h:81-216
//          (GOSH_clusters) and :312-365 (sgp_coarsen_GOSH)
//   HEC_V3 HEC's heavy neighbours with the pointer-jumping map construction
//          of heuristics.h:766-834 (parallel_map_construct_v3)
//   GOSH_V2 high-degree roots, three joining passes, then the HEC map rounds
//          with those aggregates prefilled: heuristics.h:444-560
//
// The reference draws its random keys from a time-seeded pool, numbers
// aggregates with atomic counters and resolves some races by timing.  Here a
// vertex's random key is a hash of (level seed, vertex) made unique by the
// vertex id, every conflict is resolved by a max-key rule, neighbours are
// scanned in row order where the reference takes "any", and aggregates are
// numbered by ascending root vertex -- so each mapping is a pure function of
// (graph, seed), and oracle/sgpar_oracle.c restates it exactly.
#include <cooperative_groups.h>

#include "common.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace sgpb {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// A strict total order on vertices from the level seed: the high 32 bits of
// the HEC priority hash, then the id.
__device__ __host__ __forceinline__ uint64_t match_ord(uint64_t seed, uint32_t u) {
    return (prio_key(seed, u) & 0xFFFFFFFF00000000ull) | u;
}

// ---------------------------------------------------------------- MATCH --
// Initial heavy neighbour (heuristics.h:1616-1640): level 1 of an unweighted
// graph a uniformly random neighbour; otherwise the first neighbour of
// maximum weight in row order.  A vertex without neighbours points to itself.
template <int G, typename W>
__global__ void __launch_bounds__(256) k_match_hn0(uint32_t n, const uint32_t *__restrict__ rp,
                                                   const uint32_t *__restrict__ col, const W *__restrict__ w,
                                                   int random_level, uint64_t seed, uint32_t *__restrict__ hn) {
    const unsigned gm = group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t ng = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; u < n; u += ng) {
        const uint32_t b = rp[u], e = rp[u + 1];
        if (b == e) {
            if (lane == 0) hn[u] = (uint32_t)u;
            continue;
        }
        if (random_level) {
            if (lane == 0) hn[u] = __ldg(col + b + (uint32_t)(rand_draw(seed, (uint32_t)u) % (e - b)));
            continue;
        }
        // max of (weight, -position): the first maximum in row order
        uint64_t bw = 0;
        uint32_t bj = kNone;
        for (uint32_t j = b + lane; j < e; j += G) {
            const uint64_t x = wload(w, j);
            if (bj == kNone || x > bw) {
                bw = x;
                bj = j;
            }
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            const uint64_t ow = __shfl_xor_sync(gm, bw, o);
            const uint32_t oj = __shfl_xor_sync(gm, bj, o);
            if (oj != kNone && (bj == kNone || ow > bw || (ow == bw && oj < bj))) {
                bw = ow;
                bj = oj;
            }
        }
        if (lane == 0) hn[u] = __ldg(col + bj);
    }
}

struct MatchArgs {
    uint32_t n;
    const uint32_t *rp, *col;
    const void *w;
    int wbytes;              // 0 unit, 4, 8
    int random_level;
    uint64_t seed;
    uint32_t *hn, *vcmap;
    unsigned long long *claim;   // zero on entry
    uint8_t *act;
    uint32_t *list0, *list1;
    uint32_t *counters;      // [2] zero on entry
    uint32_t *block_tot;     // [gridDim]
    uint32_t *out;           // [0] nc, [1] rounds, [2] error
    uint32_t round_cap;
};

__device__ __forceinline__ uint64_t match_w(const MatchArgs &a, uint32_t j) {
    if (a.wbytes == 8) return __ldg((const unsigned long long *)a.w + j);
    if (a.wbytes == 4) return __ldg((const uint32_t *)a.w + j);
    return 1ull;
}

// Replacement heavy neighbour of an unmatched u (heuristics.h:1686-1716):
// among unmatched neighbours, level 1 the one of largest key, otherwise the
// last of maximum weight in row order ("<=").  One warp per vertex.
__device__ __forceinline__ uint32_t match_rehn(const MatchArgs &a, uint32_t u, unsigned lane) {
    const uint32_t b = a.rp[u], e = a.rp[u + 1];
    uint64_t bk = 0;          // level 1: key + 1; else weight
    uint32_t bj = kNone;
    for (uint32_t j = b + lane; j < e; j += 32) {
        const uint32_t v = __ldg(a.col + j);
        if (__ldcg(a.vcmap + v) != kNone) continue;
        const uint64_t k = a.random_level ? match_ord(a.seed, v) + 1 : match_w(a, j);
        if (bj == kNone || k > bk || (k == bk && j > bj)) {
            bk = k;
            bj = j;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
        const uint32_t oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
        if (oj != kNone && (bj == kNone || ok > bk || (ok == bk && oj > bj))) {
            bk = ok;
            bj = oj;
        }
    }
    return bj == kNone ? kNone : __ldg(a.col + bj);
}

// All rounds in one cooperative launch.  Round r: (A) every listed u whose
// proposal direction is open this round (ord(u) < ord(hn u) xor swap) claims
// itself and hn(u) with atomicMax of ord(u) + 1; (B) a proposal whose claim
// holds on both ends forms the pair, rooted at the proposer; (C) the claims
// are cleared and every listed u still unmatched looks for its heaviest
// unmatched neighbour, staying listed if there is one.  A proposer u loses
// only to a larger key, so the largest open proposal always succeeds and two
// rounds (both directions) assign at least one pair while any vertex is
// listed.  Unlisted unmatched vertices become singletons, then aggregates are
// numbered by ascending root.
__global__ void __launch_bounds__(512) k_match_map(MatchArgs a) {
    cg::grid_group grid = cg::this_grid();
    const uint32_t n = a.n;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = tid >> 5, nwarps = nthreads >> 5;
    uint32_t len = n, swap = 1, round = 0;
    bool err = false;
    for (;;) {
        const uint32_t *lcur = (round & 1) ? a.list1 : a.list0;
        uint32_t *lnext = (round & 1) ? a.list0 : a.list1;
        // ---- A: proposals
        for (uint64_t i = tid; i < len; i += nthreads) {
            const uint32_t u = round == 0 ? (uint32_t)i : lcur[i];
            const uint32_t v = a.hn[u];
            uint8_t act = 0;
            if (v != u) {
                const uint64_t ku = match_ord(a.seed, u), kv = match_ord(a.seed, v);
                if ((uint32_t)(ku < kv) ^ swap) {
                    act = 1;
                    atomicMax(&a.claim[u], (unsigned long long)(ku + 1));
                    atomicMax(&a.claim[v], (unsigned long long)(ku + 1));
                }
            }
            a.act[u] = act;
        }
        grid.sync();
        // ---- B: pairs
        for (uint64_t i = tid; i < len; i += nthreads) {
            const uint32_t u = round == 0 ? (uint32_t)i : lcur[i];
            if (!a.act[u]) continue;
            const uint32_t v = a.hn[u];
            const unsigned long long k = match_ord(a.seed, u) + 1;
            if (a.claim[u] == k && a.claim[v] == k) {
                a.vcmap[u] = u;
                a.vcmap[v] = u;
            }
        }
        grid.sync();
        // ---- C: clear claims, new heavy neighbours, next list
        if (blockIdx.x == 0 && threadIdx.x == 0) a.counters[(round + 1) & 1] = 0;
        for (uint64_t i = wid; i < len; i += nwarps) {
            const uint32_t u = round == 0 ? (uint32_t)i : lcur[i];
            if (lane == 0) a.claim[u] = 0;
            if (__ldcg(a.vcmap + u) != kNone) continue;   // warp-uniform
            const uint32_t h = match_rehn(a, u, lane);
            if (lane == 0 && h != kNone) {
                a.hn[u] = h;
                lnext[atomicAdd(&a.counters[round & 1], 1u)] = u;
            }
        }
        grid.sync();
        const uint32_t next = *(volatile uint32_t *)&a.counters[round & 1];
        round++;
        if (next == 0) break;
        if (round >= a.round_cap) {
            err = true;
            break;
        }
        len = next;
        swap ^= 1u;
        grid.sync();   // every block has read the counter before it is reset
    }
    if (err) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.out[1] = round;
            a.out[2] = 1;
        }
        return;   // every block takes the same branch
    }
    for (uint64_t u = tid; u < n; u += nthreads)
        if (a.vcmap[u] == kNone) a.vcmap[u] = (uint32_t)u;
    grid.sync();
    // ---- number aggregates by ascending root: tile scan over [0, n)
    __shared__ uint64_t sm[33];
    const uint32_t tile = (uint32_t)(((uint64_t)n + gridDim.x - 1) / gridDim.x);
    const uint64_t t0 = (uint64_t)blockIdx.x * tile;
    const uint64_t t1 = t0 + tile < n ? t0 + tile : n;
    uint64_t cnt = 0;
    for (uint64_t u = t0 + threadIdx.x; u < t1; u += blockDim.x) cnt += (a.vcmap[u] == (uint32_t)u);
    uint64_t tot;
    block_scan_u64(cnt, sm, &tot);
    if (threadIdx.x == 0) a.block_tot[blockIdx.x] = (uint32_t)tot;
    grid.sync();
    uint64_t base = 0;
    for (uint32_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) base += a.block_tot[b];
    {
        uint64_t all;
        block_scan_u64(base, sm, &all);
        base = all;
    }
    uint32_t *rank = a.list0;   // reused as rank[n]
    for (uint64_t c0 = t0; c0 < t1; c0 += blockDim.x) {
        const uint64_t u = c0 + threadIdx.x;
        const uint32_t f = (u < t1) && (a.vcmap[u] == (uint32_t)u);
        uint64_t t;
        const uint64_t inc = block_scan_u64(f, sm, &t);
        if (u < t1) rank[u] = (uint32_t)(base + inc - f);
        base += t;
    }
    grid.sync();
    for (uint64_t u = tid; u < n; u += nthreads) a.vcmap[u] = rank[a.vcmap[u]];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        a.out[0] = (uint32_t)base;
        a.out[1] = round;
        a.out[2] = 0;
    }
}

static int coop_grid_alt(Context &C, const void *kernel, int threads, uint32_t work, uint32_t *grid) {
    int per_sm = 0;
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
    if (per_sm < 1) {
        set_error("cooperative kernel does not fit on an SM");
        return SGP_B200_ERR_DEVICE;
    }
    const uint64_t maxg = (uint64_t)per_sm * C.num_sms;
    const uint64_t want = cdiv(work ? work : 1, (uint64_t)threads / 32);   // warp-per-vertex phase
    *grid = (uint32_t)(want < maxg ? want : maxg);
    if (*grid < 1) *grid = 1;
    return SGP_B200_OK;
}

static uint32_t rows_grid(Context &C, uint64_t items) {
    uint64_t g = (items + 255) / 256;
    const uint64_t cap = (uint64_t)C.num_sms * 16;
    if (g > cap) g = cap;
    return g ? (uint32_t)g : 1u;
}

template <typename W>
static void launch_match_hn0(Context &C, const Level &L, const W *w, int random_level, uint64_t seed, uint32_t *hn) {
    const double avg = L.n ? (double)L.m / L.n : 0;
    if (avg <= 4)
        k_match_hn0<4, W><<<rows_grid(C, (uint64_t)L.n * 4), 256, 0, C.stream>>>(L.n, L.rp, L.col, w, random_level, seed,
                                                                              hn);
    else if (avg <= 16)
        k_match_hn0<16, W><<<rows_grid(C, (uint64_t)L.n * 16), 256, 0, C.stream>>>(L.n, L.rp, L.col, w, random_level,
                                                                                seed, hn);
    else
        k_match_hn0<32, W><<<rows_grid(C, (uint64_t)L.n * 32), 256, 0, C.stream>>>(L.n, L.rp, L.col, w, random_level,
                                                                                seed, hn);
    C.kernel_launches++;
}

int match_map_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out,
                    int *rounds_out) {
    const uint32_t n = L.n;
    if (n == 0) {
        *nc_out = 0;
        *rounds_out = 0;
        return SGP_B200_OK;
    }
    MatchArgs a;
    a.n = n;
    a.rp = L.rp;
    a.col = L.col;
    a.w = L.w;
    a.wbytes = L.w ? L.wbytes : 0;
    a.random_level = random_level;
    a.seed = seed;
    a.vcmap = vcmap;
    SGPB_TRY(dalloc_t(C, &a.hn, n));
    if (L.wbytes == 8)
        launch_match_hn0<unsigned long long>(C, L, (const unsigned long long *)L.w, random_level, seed, a.hn);
    else
        launch_match_hn0<uint32_t>(C, L, (const uint32_t *)L.w, random_level, seed, a.hn);
    SGPB_TRY(dalloc_t(C, &a.claim, n));
    SGPB_TRY(dalloc_t(C, &a.act, n));
    SGPB_TRY(dalloc_t(C, &a.list0, n));
    SGPB_TRY(dalloc_t(C, &a.list1, n));
    SGPB_TRY(dalloc_t(C, &a.counters, 2));
    SGPB_TRY(dalloc_t(C, &a.out, 4));
    SGPB_TRY(dzero(C, a.claim, sizeof(unsigned long long) * n));
    SGPB_TRY(dzero(C, a.counters, sizeof(uint32_t) * 2));
    SGPB_CUDA(cudaMemsetAsync(vcmap, 0xFF, sizeof(uint32_t) * n, C.stream));
    // two rounds assign at least one pair while anything is listed
    a.round_cap = round_budget((uint64_t)n + 4);
    uint32_t grid = 1;
    SGPB_TRY(coop_grid_alt(C, (const void *)k_match_map, 512, n, &grid));
    SGPB_TRY(dalloc_t(C, &a.block_tot, grid));
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel((const void *)k_match_map, dim3(grid), dim3(512), args, 0, C.stream));
    C.kernel_launches++;
    uint32_t out[3];
    SGPB_TRY(read_u32(C, a.out, out, 3));
    if (out[2]) {
        set_error("matching exceeded %u rounds", a.round_cap);
        return SGP_B200_ERR_BUDGET;
    }
    *nc_out = out[0];
    *rounds_out = (int)out[1];
    return SGP_B200_OK;
}

// --------------------------------------------------------------- HEC_V3 --
// heuristics.h:766-834: a vertex in a mutual heavy pair points to the pair's
// smaller id; every heavy-neighbour target not in such a pair points to
// itself; every other vertex points where its heavy neighbour points.  The
// reference's compare-and-swap writes the same value from every thread, and
// the join step reads only entries set before it, so the construction is
// deterministic given the heavy neighbours.  Roots (m[u] == u) are numbered
// in ascending order (the reference's scan over the dense map).
__global__ void k_v3_pairs(uint32_t n, const uint32_t *__restrict__ hn, uint32_t *__restrict__ m) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
        const uint32_t h = hn[u];
        uint32_t x = kNone;
        if (hn[h] == (uint32_t)u) x = h < u ? h : (uint32_t)u;
        m[u] = x;
    }
}
__global__ void k_v3_targets(uint32_t n, const uint32_t *__restrict__ hn, uint32_t *__restrict__ m) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
        const uint32_t v = hn[u];
        if (m[v] == kNone) m[v] = v;   // every writer stores v
    }
}
__global__ void k_v3_join(uint32_t n, const uint32_t *__restrict__ hn, uint32_t *__restrict__ m,
                          uint32_t *__restrict__ root) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
        uint32_t x = m[u];
        if (x == kNone) x = m[hn[u]];   // set by the steps above, not written here
        root[u] = x;
    }
}
__global__ void k_v3_flags(uint32_t n, const uint32_t *__restrict__ root, uint32_t *__restrict__ f) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride)
        f[u] = root[u] == (uint32_t)u;
}
__global__ void k_v3_number(uint32_t n, const uint32_t *__restrict__ root, const uint32_t *__restrict__ rank,
                            uint32_t *__restrict__ vcmap) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) vcmap[u] = rank[root[u]];
}

int hec_v3_map_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out) {
    const uint32_t n = L.n;
    if (n == 0) {
        *nc_out = 0;
        return SGP_B200_OK;
    }
    uint32_t *hn, *m, *root, *f, *rank;
    SGPB_TRY(dalloc_t(C, &hn, n));
    SGPB_TRY(dalloc_t(C, &m, n));
    SGPB_TRY(dalloc_t(C, &root, n));
    SGPB_TRY(dalloc_t(C, &f, n));
    SGPB_TRY(dalloc_t(C, &rank, (size_t)n + 1));
    SGPB_TRY(hec_hn_level(C, L, random_level, seed, hn));
    const uint32_t g = rows_grid(C, n);
    k_v3_pairs<<<g, 256, 0, C.stream>>>(n, hn, m);
    k_v3_targets<<<g, 256, 0, C.stream>>>(n, hn, m);
    k_v3_join<<<g, 256, 0, C.stream>>>(n, hn, m, root);
    k_v3_flags<<<g, 256, 0, C.stream>>>(n, root, f);
    SGPB_TRY(scan_u32(C, f, rank, n, nullptr));
    k_v3_number<<<g, 256, 0, C.stream>>>(n, root, rank, vcmap);
    C.kernel_launches += 5;
    SGPB_CUDA(cudaGetLastError());
    return read_u32(C, rank + n, nc_out);
}

// -------------------------------------------------------------- GOSH_V2 --
// heuristics.h:444-560 with every joining pass reading a snapshot of the one
// before (the reference reads live values, so its result depends on thread
// timing).  dst[u] = src[u]; an unassigned u joins the aggregate of the
// neighbour picked among those assigned in src: mode 0 the largest edge
// weight, mode 1 the largest degree (the last in row order on a tie, the
// reference's ">="), mode 2 the first in row order.  One warp per row.
template <typename W>
__global__ void __launch_bounds__(256) k_gv2_join(uint32_t n, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ col, const W *__restrict__ w, int mode,
                                                  const uint32_t *__restrict__ src, uint32_t *__restrict__ dst) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nw) {
        const uint32_t own = src[u];
        if (own != kNone) {
            if (lane == 0) dst[u] = own;
            continue;
        }
        uint64_t bk = 0;
        uint32_t bj = kNone;
        for (uint32_t j = rp[u] + lane; j < rp[u + 1]; j += 32) {
            const uint32_t v = __ldg(col + j);
            if (src[v] == kNone) continue;
            if (mode == 2) {
                if (bj == kNone) bj = j;   // j ascends per lane
                continue;
            }
            const uint64_t k = mode == 0 ? wload(w, j) : (uint64_t)(rp[v + 1] - rp[v]);
            if (bj == kNone || k >= bk) {
                bk = k;
                bj = j;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const uint64_t ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
            const uint32_t oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
            bool take;
            if (mode == 2) take = oj < bj;   // kNone is the largest
            else take = oj != kNone && (bj == kNone || ok > bk || (ok == bk && oj > bj));
            if (take) {
                bk = ok;
                bj = oj;
            }
        }
        if (lane == 0) dst[u] = bj == kNone ? kNone : src[__ldg(col + bj)];
    }
}

__global__ void k_gv2_roots(uint32_t n, const uint32_t *__restrict__ rp, uint64_t thr, uint32_t *__restrict__ vc) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride)
        vc[u] = (uint64_t)(rp[u + 1] - rp[u]) > thr ? (uint32_t)u : kNone;
}

int gosh_v2_map_level(Context &C, const Level &L, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out, int *rounds_out) {
    const uint32_t n = L.n;
    if (n == 0) {
        *nc_out = 0;
        *rounds_out = 0;
        return SGP_B200_OK;
    }
    uint64_t thr = L.m / n;
    if (thr < 50) thr = 50;
    uint32_t *a, *hn;
    SGPB_TRY(dalloc_t(C, &a, n));
    SGPB_TRY(dalloc_t(C, &hn, n));
    k_gv2_roots<<<rows_grid(C, n), 256, 0, C.stream>>>(n, L.rp, thr, a);
    const uint32_t gw = rows_grid(C, (uint64_t)n * 32);
    // snapshots ping-pong between a and vcmap, ending in vcmap
    uint32_t *src = a, *dst = vcmap;
    for (int mode = 0; mode < 3; mode++) {
        if (L.wbytes == 8)
            k_gv2_join<unsigned long long><<<gw, 256, 0, C.stream>>>(n, L.rp, L.col, (const unsigned long long *)L.w,
                                                                     mode, src, dst);
        else
            k_gv2_join<uint32_t><<<gw, 256, 0, C.stream>>>(n, L.rp, L.col, (const uint32_t *)L.w, mode, src, dst);
        uint32_t *t = src;
        src = dst;
        dst = t;
    }
    // an odd number of passes: the last one wrote vcmap
    if (src != vcmap) SGPB_CUDA(cudaMemcpyAsync(vcmap, src, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, C.stream));
    C.kernel_launches += 4;
    SGPB_CUDA(cudaGetLastError());
    SGPB_TRY(hec_hn_level(C, L, 0, seed, hn));
    return hec_map_from_hn(C, n, hn, seed, vcmap, true, nc_out, rounds_out);
}

// ---------------------------------------------------------- MIS-2 / GOSH --
// A tuple (state, key, id) ordered lexicographically; state 1 = in the set,
// 0 = undecided, -1 = excluded.
struct Tup {
    int s;
    uint64_t k;
    uint32_t i;
};
__device__ __forceinline__ bool tup_gt(const Tup &x, const Tup &y) {
    return x.s > y.s || (x.s == y.s && (x.k > y.k || (x.k == y.k && x.i > y.i)));
}

// One hop of the maximum (heuristics.h:27-60 for MIS-2, :113-146 for GOSH):
// out[u] = max over u and its neighbours of in[].  GOSH (gosh_thr != 0)
// ignores edges whose two ends both have degree above the threshold, and
// keeps decided vertices at their own tuple.
template <int G>
__global__ void __launch_bounds__(256) k_tuple_max(uint32_t n, const uint32_t *__restrict__ rp,
                                                   const uint32_t *__restrict__ col, const int *__restrict__ st_in,
                                                   const uint64_t *__restrict__ k_in, const uint32_t *__restrict__ i_in,
                                                   const int *__restrict__ state, uint64_t gosh_thr,
                                                   int *__restrict__ st_out, uint64_t *__restrict__ k_out,
                                                   uint32_t *__restrict__ i_out) {
    const unsigned gm = group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t ng = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; u < n; u += ng) {
        Tup best{st_in[u], k_in[u], i_in[u]};
        if (gosh_thr && state[u] != 0) {   // group-uniform
            if (lane == 0) {
                st_out[u] = state[u];
                k_out[u] = rp[u + 1] - rp[u];
                i_out[u] = (uint32_t)u;
            }
            continue;
        }
        const uint32_t b = rp[u], e = rp[u + 1];
        const bool u_big = gosh_thr && (uint64_t)(e - b) > gosh_thr - 1;
        for (uint32_t j = b + lane; j < e; j += G) {
            const uint32_t v = __ldg(col + j);
            if (u_big && (uint64_t)(rp[v + 1] - rp[v]) > gosh_thr - 1) continue;
            const Tup t{st_in[v], k_in[v], i_in[v]};
            if (tup_gt(t, best)) best = t;
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            Tup t;
            t.s = __shfl_xor_sync(gm, best.s, o);
            t.k = __shfl_xor_sync(gm, best.k, o);
            t.i = __shfl_xor_sync(gm, best.i, o);
            if (tup_gt(t, best)) best = t;
        }
        if (lane == 0) {
            st_out[u] = best.s;
            k_out[u] = best.k;
            i_out[u] = best.i;
        }
    }
}

// the tuples every iteration starts from (heuristics.h:21-25, :107-111)
__global__ void k_tuple_init(uint32_t n, const uint32_t *__restrict__ rp, const int *__restrict__ state, int gosh,
                             uint64_t seed, int *__restrict__ ts, uint64_t *__restrict__ tk,
                             uint32_t *__restrict__ ti) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
        ts[u] = state[u];
        tk[u] = gosh ? (uint64_t)(rp[u + 1] - rp[u]) : prio_key(seed, (uint32_t)u);
        ti[u] = (uint32_t)u;
    }
}

// heuristics.h:63-74 / :149-162: an undecided u that is its own maximum
// joins the set; one that sees the set, or whose maximum is its own
// maximum (and so joins now), is excluded.  *left counts the undecided.
__global__ void k_set_assign(uint32_t n, int *__restrict__ state, const int *__restrict__ ts,
                             const uint32_t *__restrict__ ti, uint32_t *__restrict__ left) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u - lane < n; u += stride) {
        bool undecided = false;
        if (u < n && state[u] == 0) {
            const uint32_t m = ti[u];
            if (m == (uint32_t)u) state[u] = 1;
            else if (ts[u] == 1 || ti[m] == m) state[u] = -1;
            else undecided = true;
        }
        const unsigned c = __popc(__ballot_sync(0xFFFFFFFFu, undecided));
        if (lane == 0 && c) atomicAdd(left, c);
    }
}

// root flags for the numbering scan
__global__ void k_roots(uint32_t n, const int *__restrict__ state, uint32_t *__restrict__ f) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) f[u] = state[u] == 1;
}

// MIS-2 aggregates (heuristics.h:241-264): a root and its neighbours (the
// neighbourhoods of distance-2 independent roots are disjoint) ...
__global__ void __launch_bounds__(256) k_mis2_agg1(uint32_t n, const uint32_t *__restrict__ rp,
                                                   const uint32_t *__restrict__ col, const int *__restrict__ state,
                                                   const uint32_t *__restrict__ rank, uint32_t *__restrict__ vc) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nw) {
        if (state[u] != 1) continue;
        const uint32_t id = rank[u];
        if (lane == 0) vc[u] = id;
        for (uint32_t j = rp[u] + lane; j < rp[u + 1]; j += 32) vc[__ldg(col + j)] = id;
    }
}

// ... then every vertex still outside joins the aggregate of its first
// neighbour (row order) that is in one after the step above (the reference
// takes whichever write lands).
__global__ void __launch_bounds__(256) k_mis2_agg2(uint32_t n, const uint32_t *__restrict__ rp,
                                                   const uint32_t *__restrict__ col, const uint32_t *__restrict__ vc1,
                                                   uint32_t *__restrict__ vc, uint32_t *__restrict__ missing) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nw) {
        if (vc1[u] != kNone) continue;
        uint32_t pick = kNone;
        for (uint32_t j0 = rp[u]; j0 < rp[u + 1] && pick == kNone; j0 += 32) {
            const uint32_t j = j0 + lane;
            const uint32_t a = j < rp[u + 1] ? vc1[__ldg(col + j)] : kNone;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, a != kNone);
            if (m) pick = __shfl_sync(0xFFFFFFFFu, a, __ffs(m) - 1);
        }
        if (lane == 0) {
            vc[u] = pick;
            if (pick == kNone) atomicAdd(missing, 1u);
        }
    }
}

// GOSH aggregates (heuristics.h:325-339): every vertex outside the set joins
// its set neighbour of largest degree, the first in row order on a tie.
__global__ void __launch_bounds__(256) k_gosh_agg(uint32_t n, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ col, const int *__restrict__ state,
                                                  const uint32_t *__restrict__ rank, uint32_t *__restrict__ vc,
                                                  uint32_t *__restrict__ missing) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nw) {
        if (state[u] == 1) {
            if (lane == 0) vc[u] = rank[u];
            continue;
        }
        uint32_t bd = 0, bj = kNone;
        for (uint32_t j = rp[u] + lane; j < rp[u + 1]; j += 32) {
            const uint32_t v = __ldg(col + j);
            if (state[v] != 1) continue;
            const uint32_t d = rp[v + 1] - rp[v];
            if (d > bd) {   // j ascends per lane: the first maximum of the lane
                bd = d;
                bj = j;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const uint32_t od = __shfl_xor_sync(0xFFFFFFFFu, bd, o);
            const uint32_t oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
            if (oj != kNone && (bj == kNone || od > bd || (od == bd && oj < bj))) {
                bd = od;
                bj = oj;
            }
        }
        if (lane == 0) {
            if (bj == kNone) {
                vc[u] = kNone;
                atomicAdd(missing, 1u);
            } else {
                vc[u] = rank[__ldg(col + bj)];
            }
        }
    }
}

// The independent-set iterations of MIS-2 (hops = 2) or GOSH_clusters
// (hops = 1, degree keys, heavy-heavy edges ignored).
static int set_iterations(Context &C, const Level &L, bool gosh, uint64_t seed, int *state, int *iters_out) {
    const uint32_t n = L.n;
    int *ts[2];
    uint64_t *tk[2];
    uint32_t *ti[2], *left;
    for (int b = 0; b < 2; b++) {
        SGPB_TRY(dalloc_t(C, &ts[b], n));
        SGPB_TRY(dalloc_t(C, &tk[b], n));
        SGPB_TRY(dalloc_t(C, &ti[b], n));
    }
    SGPB_TRY(dalloc_t(C, &left, 1));
    SGPB_TRY(dzero(C, state, sizeof(int) * n));
    // heuristics.h:101: threshold = nnz / n; stored + 1 so 0 means "MIS-2"
    const uint64_t thr = gosh ? L.m / n + 1 : 0;
    const double avg = (double)L.m / n;
    const int hops = gosh ? 1 : 2;
    const uint32_t cap = round_budget(4 * (uint64_t)n + 16);
    int it = 0;
    for (;; it++) {
        if ((uint32_t)it > cap) {
            set_error("independent-set iterations exceeded %u", cap);
            return SGP_B200_ERR_BUDGET;
        }
        k_tuple_init<<<rows_grid(C, n), 256, 0, C.stream>>>(n, L.rp, state, gosh, seed, ts[0], tk[0], ti[0]);
        int cur = 0;
        for (int h = 0; h < hops; h++) {
#define SGPB_TMAX(G)                                                                                          \
    k_tuple_max<G><<<rows_grid(C, (uint64_t)n * G), 256, 0, C.stream>>>(n, L.rp, L.col, ts[cur], tk[cur], ti[cur], \
                                                                          state, thr, ts[cur ^ 1], tk[cur ^ 1],   \
                                                                          ti[cur ^ 1])
            if (avg <= 4) SGPB_TMAX(4);
            else if (avg <= 16) SGPB_TMAX(16);
            else SGPB_TMAX(32);
#undef SGPB_TMAX
            cur ^= 1;
        }
        SGPB_TRY(dzero(C, left, 4));
        k_set_assign<<<rows_grid(C, n), 256, 0, C.stream>>>(n, state, ts[cur], ti[cur], left);
        SGPB_CUDA(cudaGetLastError());
        C.kernel_launches += 2 + hops;
        uint32_t l = 0;
        SGPB_TRY(read_u32(C, left, &l));
        if (l == 0) break;
    }
    *iters_out = it + 1;
    return SGP_B200_OK;
}

// coarsener 2 (MIS2) or 3 (GOSH)
int set_map_level(Context &C, const Level &L, bool gosh, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out,
                  int *rounds_out) {
    const uint32_t n = L.n;
    if (n == 0) {
        *nc_out = 0;
        *rounds_out = 0;
        return SGP_B200_OK;
    }
    int *state;
    uint32_t *flag, *rank, *missing;
    SGPB_TRY(dalloc_t(C, &state, n));
    SGPB_TRY(set_iterations(C, L, gosh, seed, state, rounds_out));
    SGPB_TRY(dalloc_t(C, &flag, n));
    SGPB_TRY(dalloc_t(C, &rank, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &missing, 1));
    SGPB_TRY(dzero(C, missing, 4));
    k_roots<<<rows_grid(C, n), 256, 0, C.stream>>>(n, state, flag);
    SGPB_TRY(scan_u32(C, flag, rank, n, nullptr));
    SGPB_TRY(read_u32(C, rank + n, nc_out));
    const uint32_t gw = rows_grid(C, (uint64_t)n * 32);
    if (gosh) {
        k_gosh_agg<<<gw, 256, 0, C.stream>>>(n, L.rp, L.col, state, rank, vcmap, missing);
        C.kernel_launches += 2;
    } else {
        uint32_t *vc1;
        SGPB_TRY(dalloc_t(C, &vc1, n));
        SGPB_CUDA(cudaMemsetAsync(vc1, 0xFF, sizeof(uint32_t) * n, C.stream));
        k_mis2_agg1<<<gw, 256, 0, C.stream>>>(n, L.rp, L.col, state, rank, vc1);
        SGPB_CUDA(cudaMemcpyAsync(vcmap, vc1, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, C.stream));
        k_mis2_agg2<<<gw, 256, 0, C.stream>>>(n, L.rp, L.col, vc1, vcmap, missing);
        C.kernel_launches += 3;
    }
    SGPB_CUDA(cudaGetLastError());
    uint32_t miss = 0;
    SGPB_TRY(read_u32(C, missing, &miss));
    if (miss) {
        set_error("%s left %u vertices outside every aggregate", gosh ? "GOSH" : "MIS-2", miss);
        return SGP_B200_ERR_DEVICE;
    }
    return SGP_B200_OK;
}

}  // namespace sgpb
