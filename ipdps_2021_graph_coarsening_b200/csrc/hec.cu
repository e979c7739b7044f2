// hec.cu -- heavy-edge coarsening (HEC) mapping of one level.
//
// Reference: cmg/heuristics.h:930-1031 (sgp_coarsen_HEC), :614-631
// (generate_permutation), :633-693 (parallel_map_construct).  The reference is
// time-seeded and resolves conflicts with compare-and-swap races, so its
// mapping changes from run to run.  Here every random choice is a hash of
// (level seed, vertex) and every conflict is resolved by a max-key rule, so
// the mapping is a pure function of (graph, seed); the CPU oracle restates the
// same rules (oracle/sgpar_oracle.c: orc_hec_heavy, orc_hec_map).
#include "common.cuh"
#include "internal.h"

namespace sgpb {

// ----------------------------------------------------- heavy neighbour --
// Level 1 of an unweighted graph: a uniformly random neighbour (all weights
// are 1 there; heuristics.h:959-972).  One thread per vertex: reads two
// offsets and one destination.
__global__ void k_hn_random(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                            uint64_t seed, uint32_t *__restrict__ hn) {
    uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    uint32_t b = rp[u], deg = rp[u + 1] - b;
    uint64_t r = rand_draw(seed, u);
    hn[u] = deg == 0 ? (uint32_t)(r % n) : __ldg(col + b + (uint32_t)(r % deg));
}

// Levels >= 2 (and weighted inputs): argmax over the row of
// (weight, tiebreak hash, destination) -- a strict order, so the winner does
// not depend on the reduction order (the reference's MaxLoc with `>=` at
// heuristics.h:974-998 takes whichever maximum the reduction meets last).
// G lanes per row, rows grid-strided.  Rows longer than long_T entries (the
// hubs of skewed graphs, up to hundreds of thousands of entries) are left to
// k_hn_heavy_long, a block per row, and listed in long_list: one group would
// hold its SM for the whole kernel on such a row.

// entries [j0, e) in strides of `s`, four in flight: the running maximum
template <typename W>
__device__ __forceinline__ void hn_scan(const uint32_t *__restrict__ col, const W *__restrict__ w, uint64_t seed,
                                        uint32_t u, uint32_t j0, uint32_t e, uint32_t s, uint64_t &bw, uint64_t &bk,
                                        bool &have) {
    for (; j0 < e; j0 += 4 * s) {
        uint32_t v[4];
        uint64_t wt[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t j = j0 + q * s;
            v[q] = j < e ? __ldg(col + j) : 0u;
            wt[q] = j < e ? wload(w, j) : 0ull;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (j0 + q * s >= e) continue;
            const uint64_t k = ((uint64_t)tiebreak(seed, u, v[q]) << 32) | v[q];
            if (!have || wt[q] > bw || (wt[q] == bw && k > bk)) { bw = wt[q]; bk = k; have = true; }
        }
    }
}

__device__ __forceinline__ void hn_combine(uint64_t ow, uint64_t ok, int oh, uint64_t &bw, uint64_t &bk, bool &have) {
    if (oh && (!have || ow > bw || (ow == bw && ok > bk))) { bw = ow; bk = ok; have = true; }
}

template <int G, typename W>
__global__ void __launch_bounds__(256) k_hn_heavy(uint32_t n, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ col, const W *__restrict__ w,
                                                  uint64_t seed, uint32_t *__restrict__ hn, uint32_t long_T,
                                                  uint32_t *__restrict__ long_list, uint32_t *__restrict__ long_cnt) {
    const unsigned gm = group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t u64 = gid; u64 < n; u64 += ngroups) {
        uint32_t u = (uint32_t)u64;
        uint32_t b = rp[u], e = rp[u + 1];
        if (e - b > long_T) {   // group-uniform
            if (lane == 0) long_list[atomicAdd(long_cnt, 1u)] = u;
            continue;
        }
        uint64_t bw = 0, bk = 0;   // (weight, tiebreak<<32 | dest); 0 = none
        bool have = false;
        hn_scan(col, w, seed, u, b + lane, e, G, bw, bk, have);
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            uint64_t ow = __shfl_xor_sync(gm, bw, o);
            uint64_t ok = __shfl_xor_sync(gm, bk, o);
            int oh = __shfl_xor_sync(gm, (int)have, o);
            hn_combine(ow, ok, oh, bw, bk, have);
        }
        if (lane == 0) hn[u] = (e == b) ? (uint32_t)(rand_draw(seed, u) % n) : (uint32_t)(bk & 0xFFFFFFFFu);
    }
}

// the rows k_hn_heavy listed as long: a block per row, grid-strided over the list
constexpr int kHnLongThreads = 1024;
template <typename W>
__global__ void __launch_bounds__(kHnLongThreads) k_hn_heavy_long(const uint32_t *__restrict__ rp,
                                                                  const uint32_t *__restrict__ col,
                                                                  const W *__restrict__ w, uint64_t seed,
                                                                  const uint32_t *__restrict__ long_list,
                                                                  const uint32_t *__restrict__ long_cnt,
                                                                  uint32_t *__restrict__ hn) {
    __shared__ uint64_t s_w[kHnLongThreads / 32], s_k[kHnLongThreads / 32];
    __shared__ int s_h[kHnLongThreads / 32];
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t cnt = *long_cnt;
    for (uint32_t r = blockIdx.x; r < cnt; r += gridDim.x) {
        const uint32_t u = long_list[r];
        const uint32_t b = rp[u], e = rp[u + 1];
        uint64_t bw = 0, bk = 0;
        bool have = false;
        hn_scan(col, w, seed, u, b + threadIdx.x, e, blockDim.x, bw, bk, have);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            uint64_t ow = __shfl_xor_sync(0xFFFFFFFFu, bw, o);
            uint64_t ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
            int oh = __shfl_xor_sync(0xFFFFFFFFu, (int)have, o);
            hn_combine(ow, ok, oh, bw, bk, have);
        }
        if (lane == 0) { s_w[wid] = bw; s_k[wid] = bk; s_h[wid] = have; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 1; k < (int)(blockDim.x >> 5); k++) hn_combine(s_w[k], s_k[k], s_h[k], bw, bk, have);
            hn[u] = (uint32_t)(bk & 0xFFFFFFFFu);   // a long row has entries
        }
        __syncthreads();
    }
}

// ------------------------------------------------------ map construction --
constexpr int kMapThreads = 512;

struct MapArgs {
    uint32_t n;
    const uint32_t *hn;
    uint64_t seed;
    uint32_t *vcmap;
    unsigned long long *claim0, *claim1;
    uint8_t *act;
    uint32_t *list0, *list1;
    uint32_t *counters;     // [2] append counters (zeroed before launch)
    uint32_t *block_tot;    // [gridDim]
    uint32_t *out;          // [0] nc, [1] rounds, [2] error
    uint32_t round_cap;
};

// One persistent cooperative kernel for all rounds of
// parallel_map_construct (heuristics.h:633-693) plus the final numbering.
// Per round: phase A compacts the still-unassigned vertices and records
// claims (atomicMax on 64-bit keys), phase B resolves them.  Two grid barriers
// per round; the reference instead pays a host round trip per round (:687).
__global__ void __launch_bounds__(kMapThreads) k_hec_map(MapArgs a) {
    cg::grid_group grid = cg::this_grid();
    const uint64_t JOIN = ~0ull, SELF = ~0ull - 1;
    const uint32_t n = a.n;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    uint32_t len_prev = n;
    uint32_t swap = 1;
    uint32_t round = 0;
    bool err = false;
    for (;;) {
        unsigned long long *cl = (round & 1) ? a.claim1 : a.claim0;
        uint32_t *lprev = (round & 1) ? a.list0 : a.list1;
        uint32_t *lcur = (round & 1) ? a.list1 : a.list0;
        // ---- phase A
        uint64_t lim = ((uint64_t)len_prev + 31) & ~31ull;   // whole warps take part in the ballot
        for (uint64_t i = tid; i < lim; i += nthreads) {
            uint32_t u = 0;
            bool live = false;
            if (i < len_prev) {
                u = round == 0 ? (uint32_t)i : lprev[i];
                live = a.vcmap[u] == kUnassigned;
            }
            unsigned m = __ballot_sync(0xFFFFFFFFu, live);
            uint32_t base = 0;
            if (m) {
                int leader = __ffs(m) - 1;
                if (lane == leader) base = atomicAdd(&a.counters[round & 1], (uint32_t)__popc(m));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
            }
            if (!live) continue;
            lcur[base + __popc(m & ((1u << lane) - 1))] = u;
            uint32_t v = a.hn[u];
            uint8_t act;
            if (a.vcmap[v] != kUnassigned) {
                act = 1;
                atomicMax(&cl[u], JOIN);
            } else if (v == u) {
                act = 2;
                atomicMax(&cl[u], SELF);
            } else {
                uint64_t ku = prio_key(a.seed, u), kv = prio_key(a.seed, v);
                uint32_t cond = ku < kv ? 1u : 0u;
                if (cond ^ swap) {
                    act = 3;
                    atomicMax(&cl[u], (unsigned long long)(ku + 1));
                    atomicMax(&cl[v], (unsigned long long)(ku + 1));
                } else {
                    act = 0;
                }
            }
            a.act[u] = act;
        }
        grid.sync();
        const uint32_t len = *(volatile uint32_t *)&a.counters[round & 1];
        if (len == 0) break;
        if (round >= a.round_cap) { err = true; break; }
        if (blockIdx.x == 0 && threadIdx.x == 0) a.counters[(round + 1) & 1] = 0;
        // ---- phase B
        unsigned long long *other = (round & 1) ? a.claim0 : a.claim1;
        for (uint64_t i = tid; i < len; i += nthreads) {
            uint32_t u = lcur[i];
            uint32_t v = a.hn[u];
            uint8_t act = a.act[u];
            if (act == 1) {
                a.vcmap[u] = a.vcmap[v];
            } else if (act == 2) {
                a.vcmap[u] = u;
            } else if (act == 3) {
                unsigned long long k = prio_key(a.seed, u) + 1;
                if (cl[u] == k && cl[v] == k) { a.vcmap[u] = u; a.vcmap[v] = u; }
            }
            other[u] = 0;
        }
        grid.sync();
        len_prev = len;
        swap ^= 1u;
        round++;
    }
    if (err) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { a.out[1] = round; a.out[2] = 1; }
        return;   // every block takes the same branch
    }
    // ---- number aggregates by ascending root id: tile scan over [0, n)
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
        uint64_t dummy;
        // block-wide sum of base contributions (all threads take part)
        uint64_t inc = block_scan_u64(base, sm, &dummy);
        (void)inc;
        base = dummy;
    }
    uint32_t *rank = a.list0;   // reuse as rank[n]
    for (uint64_t c0 = t0; c0 < t1; c0 += blockDim.x) {
        uint64_t u = c0 + threadIdx.x;
        uint32_t f = (u < t1) && (a.vcmap[u] == (uint32_t)u);
        uint64_t t;
        uint64_t inc = block_scan_u64(f, sm, &t);
        if (u < t1) rank[u] = (uint32_t)(base + inc - f);
        base += t;
    }
    grid.sync();
    for (uint64_t u = tid; u < n; u += nthreads) a.vcmap[u] = rank[a.vcmap[u]];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        a.out[0] = (uint32_t)base;   // the last tile ends at n: base = total roots
        a.out[1] = round;
        a.out[2] = 0;
    }
}

static int coop_grid(Context &C, const void *kernel, int threads, size_t smem, uint32_t work_items,
                     uint32_t *grid_out) {
    int per_sm = 0;
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1) {
        set_error("cooperative kernel does not fit on an SM");
        return SGP_B200_ERR_DEVICE;
    }
    uint64_t maxg = (uint64_t)per_sm * C.num_sms;
    uint64_t want = cdiv(work_items ? work_items : 1, (uint64_t)threads);
    *grid_out = (uint32_t)(want < maxg ? want : maxg);
    if (*grid_out < 1) *grid_out = 1;
    return SGP_B200_OK;
}

// rows longer than this go to the block-per-row kernel
constexpr uint32_t kHnLongT = 8192;

template <typename W>
static int launch_hn_heavy(Context &C, const Level &L, const W *w, uint64_t seed, uint32_t *hn) {
    double avg = L.n ? (double)L.m / L.n : 0;
    uint32_t blocks_cap = (uint32_t)C.num_sms * 16;
    uint32_t *long_list, *long_cnt;
    SGPB_TRY(dalloc_t(C, &long_list, L.m / kHnLongT + 1));
    SGPB_TRY(dalloc_t(C, &long_cnt, 1));
    SGPB_TRY(dzero(C, long_cnt, sizeof(uint32_t)));
#define SGPB_HN(G)                                                                                      \
    {                                                                                                   \
        uint32_t blocks = cdiv((uint64_t)L.n * G, 256);                                                 \
        if (blocks > blocks_cap) blocks = blocks_cap;                                                   \
        if (blocks < 1) blocks = 1;                                                                     \
        k_hn_heavy<G, W><<<blocks, 256, 0, C.stream>>>(L.n, L.rp, L.col, w, seed, hn, kHnLongT, long_list, \
                                                       long_cnt);                                       \
    }
    if (avg <= 4) SGPB_HN(4) else if (avg <= 8) SGPB_HN(8) else if (avg <= 16) SGPB_HN(16) else SGPB_HN(32)
#undef SGPB_HN
    if (L.m > kHnLongT) {
        uint32_t gl = (uint32_t)(L.m / kHnLongT + 1);
        if (gl > (uint32_t)C.num_sms * 2) gl = C.num_sms * 2;
        k_hn_heavy_long<W><<<gl, kHnLongThreads, 0, C.stream>>>(L.rp, L.col, w, seed, long_list, long_cnt, hn);
        C.kernel_launches++;
    }
    C.kernel_launches++;
    return SGP_B200_OK;
}

// the heavy-neighbour step alone (also used by the HEC_V3 mapping)
int hec_hn_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *hn) {
    const uint32_t n = L.n;
    if (n == 0) return SGP_B200_OK;
    if (random_level) {
        k_hn_random<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, L.col, seed, hn);
        C.kernel_launches++;
    } else if (L.wbytes == 8) {
        SGPB_TRY(launch_hn_heavy<unsigned long long>(C, L, (const unsigned long long *)L.w, seed, hn));
    } else {
        SGPB_TRY(launch_hn_heavy<uint32_t>(C, L, (const uint32_t *)L.w, seed, hn));
    }
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}

int hec_map_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *vcmap,
                  uint32_t *hn_out, uint32_t *nc_out, int *rounds_out) {
    const uint32_t n = L.n;
    if (n == 0) { *nc_out = 0; *rounds_out = 0; return SGP_B200_OK; }
    uint32_t *hn = hn_out;
    if (!hn) SGPB_TRY(dalloc_t(C, &hn, n));
    SGPB_TRY(hec_hn_level(C, L, random_level, seed, hn));
    return hec_map_from_hn(C, n, hn, seed, vcmap, false, nc_out, rounds_out);
}

// The map rounds on given heavy neighbours.  prefilled: vcmap already holds
// aggregates (members hold their root vertex, roots themselves, the rest
// kUnassigned), as parallel_map_construct_prefilled (heuristics.h:378-443)
// takes them; the rounds only place the unassigned vertices.
int hec_map_from_hn(Context &C, uint32_t n, const uint32_t *hn, uint64_t seed, uint32_t *vcmap, bool prefilled,
                    uint32_t *nc_out, int *rounds_out) {
    MapArgs a;
    a.n = n; a.hn = hn; a.seed = seed; a.vcmap = vcmap;
    SGPB_TRY(dalloc_t(C, &a.claim0, n));
    SGPB_TRY(dalloc_t(C, &a.claim1, n));
    SGPB_TRY(dalloc_t(C, &a.act, n));
    SGPB_TRY(dalloc_t(C, &a.list0, n));
    SGPB_TRY(dalloc_t(C, &a.list1, n));
    SGPB_TRY(dalloc_t(C, &a.counters, 2));
    SGPB_TRY(dalloc_t(C, &a.out, 4));
    SGPB_TRY(dzero(C, a.claim0, sizeof(unsigned long long) * n));
    SGPB_TRY(dzero(C, a.claim1, sizeof(unsigned long long) * n));
    SGPB_TRY(dzero(C, a.counters, sizeof(uint32_t) * 2));
    if (!prefilled) SGPB_CUDA(cudaMemsetAsync(vcmap, 0xFF, sizeof(uint32_t) * n, C.stream));
    // Progress argument: each two rounds assign at least one vertex, so
    // 2n + 4 rounds always suffice; the cap only turns a bug into an error.
    a.round_cap = round_budget(2 * (uint64_t)n + 4);
    uint32_t grid = 1;
    SGPB_TRY(coop_grid(C, (const void *)k_hec_map, kMapThreads, 0, n, &grid));
    SGPB_TRY(dalloc_t(C, &a.block_tot, grid));
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel((const void *)k_hec_map, dim3(grid), dim3(kMapThreads), args, 0,
                                          C.stream));
    C.kernel_launches++;
    uint32_t out[3];
    SGPB_TRY(read_u32(C, a.out, out, 3));
    if (out[2]) {
        set_error("HEC map construction exceeded %u rounds", a.round_cap);
        return SGP_B200_ERR_BUDGET;
    }
    *nc_out = out[0];
    *rounds_out = (int)out[1];
    return SGP_B200_OK;
}

}  // namespace sgpb
