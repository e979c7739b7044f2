// fm.cu -- FM refinement of a bisection on the device.
//
// The reference's FM (cmg/eigensolve_kokkos.h:973-1240, fm_refine) is a
// host-serial pass over gain-bucket lists whose initial order comes from a
// parallel build, and its parallel variant (:695-971, fm_refine_par, disabled
// there) orders moves through atomics and picks the best prefix with a
// non-associative scan.  This pass keeps fm_refine_par's structure with
// deterministic rules (oracle/sgpar_oracle.c orc_fm_refine restates them):
//   1. gain(u) = neighbours across the cut minus those inside (the finest
//      level's edges all weigh 1);
//   2. each side's positive-gain vertices ordered by (gain clamped to
//      kFmBuckets - 1 descending, id ascending) -- a stable counting sort of
//      the id-ordered candidates;
//   3. the two lists interleaved by the serial FM's balance rule
//      (:1105-1140): side 0 while the balance (part-0 minus part-1 vertices)
//      is positive, side 1 while negative, at zero the head of larger gain
//      (side 0 on a tie), the other list once one runs out.  With unit
//      vertex weights this order has a closed form: ceil(|d| / 2) moves from
//      the heavy side, then pairs (fixed order at balance -+1, by gain at 0),
//      then the rest of the longer list;
//   4. sequential gains: the gain of the i-th move given that the first i
//      have moved; cut after k moves = cut - their sum;
//   5. k* = the k (0 included) of least cut whose |balance| is within the
//      serial FM's target max(|d| / 10, 20) (:1073-1076), the largest such k
//      on a tie (its "<="); the first k* moves are applied.
// Passes repeat until one applies nothing or leaves the cut unchanged.
#include <cooperative_groups.h>

#include "common.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace sgpb {

constexpr int kFmBuckets = 1024;
constexpr uint32_t kFmNone = 0xFFFFFFFFu;
constexpr int kFmTile = 1024;   // candidates per block in the counting sort

// gains, candidate flags, cut and balance.  Unit edge weights (the finest
// level): a symmetric graph with fewer than 2^32 directed entries has every
// degree below 2^31, so 32-bit sums are exact.  G lanes per row, four
// entries per lane in flight (destinations, then the part gathers).
template <int G>
__global__ void __launch_bounds__(256) k_fm_gain(uint32_t n, const uint32_t *__restrict__ rp,
                                                 const uint32_t *__restrict__ col,
                                                 const uint32_t *__restrict__ part, long long *__restrict__ gain,
                                                 uint8_t *__restrict__ f0, uint8_t *__restrict__ f1,
                                                 unsigned long long *__restrict__ sums /* [0] 2 cut, [1] bal */) {
    const unsigned gm = group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t ng = ((uint64_t)gridDim.x * blockDim.x) / G;
    unsigned long long cut2 = 0;
    long long bal = 0;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; u < n; u += ng) {
        const uint32_t pu = __ldg(part + u);
        const uint32_t b = __ldg(rp + u), e = __ldg(rp + u + 1);
        int across = 0;
        for (uint32_t j0 = b + lane; j0 < e; j0 += 4 * G) {
            uint32_t v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] = j0 + q * G < e ? __ldg(col + j0 + q * G) : 0xFFFFFFFFu;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (v[q] != 0xFFFFFFFFu) across += __ldg(part + v[q]) != pu;
        }
        across = group_sum<G>(across);
        if (lane == 0) {
            const int deg = (int)(e - b);
            const int g = 2 * across - deg;   // across minus inside
            gain[u] = g;
            f0[u] = pu == 0 && g > 0;
            f1[u] = pu != 0 && g > 0;
            cut2 += (unsigned)across;
            bal += pu == 0 ? 1 : -1;
        }
    }
    cut2 = warp_sum(cut2);
    bal = warp_sum(bal);
    if ((threadIdx.x & 31) == 0) {
        if (cut2) atomicAdd(sums, cut2);
        if (bal) atomicAdd(sums + 1, (unsigned long long)bal);
    }
}

__device__ __forceinline__ uint32_t fm_bucket(long long g) {
    return g < kFmBuckets - 1 ? (uint32_t)g : (uint32_t)(kFmBuckets - 1);
}

// counts per (descending bucket, tile): hist[(kFmBuckets - 1 - b) * ntiles + t]
__global__ void __launch_bounds__(kFmTile) k_fm_hist(uint32_t len, const uint32_t *__restrict__ idx,
                                                     const long long *__restrict__ gain, uint32_t ntiles,
                                                     uint32_t *__restrict__ hist) {
    __shared__ uint32_t cnt[kFmBuckets];
    for (int b = threadIdx.x; b < kFmBuckets; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * kFmTile + threadIdx.x;
    if (i < len) atomicAdd(&cnt[fm_bucket(gain[idx[i]])], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kFmBuckets; b += blockDim.x)
        hist[(size_t)(kFmBuckets - 1 - b) * ntiles + blockIdx.x] = cnt[b];
}

// stable placement: within a tile the warps take turns in order, and lanes
// of one bucket rank by lane
__global__ void __launch_bounds__(kFmTile) k_fm_place(uint32_t len, const uint32_t *__restrict__ idx,
                                                      const long long *__restrict__ gain, uint32_t ntiles,
                                                      const uint32_t *__restrict__ off,
                                                      uint32_t *__restrict__ sorted) {
    __shared__ uint32_t cnt[kFmBuckets];
    for (int b = threadIdx.x; b < kFmBuckets; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * kFmTile + threadIdx.x;
    const bool valid = i < len;
    const uint32_t u = valid ? idx[i] : 0u;
    const uint32_t b = valid ? fm_bucket(gain[u]) : 0u;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (unsigned turn = 0; turn < kFmTile / 32; turn++) {
        if (wid == turn) {
            const unsigned act = __ballot_sync(0xFFFFFFFFu, valid);
            if (valid) {
                const unsigned peers = __match_any_sync(act, b);
                const uint32_t r = cnt[b] + __popc(peers & ((1u << lane) - 1u));
                sorted[off[(size_t)(kFmBuckets - 1 - b) * ntiles + blockIdx.x] + r] = u;
                __syncwarp(peers);
                if ((int)lane == __ffs(peers) - 1) cnt[b] += __popc(peers);
            }
        }
        __syncthreads();
    }
}

// closed-form interleave (see the header): order[pos] = vertex, rank[v] = pos
__global__ void k_fm_interleave(uint32_t na, uint32_t nb, const uint32_t *__restrict__ A,
                                const uint32_t *__restrict__ B, const long long *__restrict__ gain, long long d,
                                uint32_t *__restrict__ order, uint32_t *__restrict__ rank,
                                uint8_t *__restrict__ side) {
    // phase 1: ceil(|d| / 2) moves from the heavier side (as many as it has)
    const bool heavy0 = d > 0;
    const uint64_t want = d > 0 ? (uint64_t)(d + 1) / 2 : (uint64_t)(-d + 1) / 2;
    const uint32_t nh = heavy0 ? na : nb;
    const uint32_t p0 = (uint32_t)(want < nh ? want : nh);
    // balance after phase 1 when the heavy side lasted: 0 or -+1
    const long long r = heavy0 ? d - 2 * (long long)p0 : d + 2 * (long long)p0;
    const uint32_t ra = heavy0 ? na - p0 : na, rb = heavy0 ? nb : nb - p0;   // left after phase 1
    const uint32_t a0 = heavy0 ? p0 : 0, b0 = heavy0 ? 0 : p0;                // first index left
    const uint32_t m = ra < rb ? ra : rb;                                     // full pairs
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint32_t tot = na > nb ? na : nb;
    for (uint64_t i = tid; i < tot; i += stride) {
        for (int s = 0; s < 2; s++) {
            const uint32_t len = s == 0 ? na : nb;
            if (i >= len) continue;
            const uint32_t u = s == 0 ? A[i] : B[i];
            uint64_t pos;
            const uint32_t first = s == 0 ? a0 : b0;
            if ((s == 0) == heavy0 && i < p0 && d != 0) {
                pos = i;                                      // phase 1
            } else if (i - first < m) {
                const uint32_t k = i - first;                 // pair k
                bool a_first;
                if (r > 0) a_first = true;                    // balance +1: side 0 then side 1
                else if (r < 0) a_first = false;
                else a_first = gain[A[a0 + k]] >= gain[B[b0 + k]];
                const bool me_first = (s == 0) == a_first;
                pos = (uint64_t)p0 + 2ull * k + (me_first ? 0 : 1);
            } else {
                pos = (uint64_t)p0 + 2ull * m + (i - first - m);   // tail of the longer list
            }
            order[pos] = u;
            rank[u] = (uint32_t)pos;
            side[pos] = (uint8_t)s;
        }
    }
}

// sequential gain of the i-th move (unit weights, 32-bit sums as above)
template <int G>
__global__ void __launch_bounds__(256) k_fm_seqgain(uint32_t k, const uint32_t *__restrict__ rp,
                                                    const uint32_t *__restrict__ col,
                                                    const uint32_t *__restrict__ part,
                                                    const uint32_t *__restrict__ order,
                                                    const uint32_t *__restrict__ rank, long long *__restrict__ gseq) {
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t ng = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; i < k; i += ng) {
        const uint32_t u = __ldg(order + i), pu = __ldg(part + u);
        const uint32_t b = __ldg(rp + u), e = __ldg(rp + u + 1);
        int plus = 0;   // neighbours counting +1: across xor moved before
        for (uint32_t j0 = b + lane; j0 < e; j0 += 4 * G) {
            uint32_t v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] = j0 + q * G < e ? __ldg(col + j0 + q * G) : 0xFFFFFFFFu;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (v[q] == 0xFFFFFFFFu) continue;
                const bool across = __ldg(part + v[q]) != pu, moved = __ldg(rank + v[q]) < (uint32_t)i;
                plus += across != moved;
            }
        }
        plus = group_sum<G>(plus);
        if (lane == 0) gseq[i] = 2 * plus - (int)(e - b);
    }
}

// best prefix: one contiguous chunk per block, chunk sums, then a scan per
// chunk evaluating every k; key = cut << 32 | ~k, minimised (least cut,
// then the largest k)
struct FmBestArgs {
    uint32_t k;
    const long long *gseq;
    const uint8_t *side;
    long long cut0, bal0, target;
    long long *chunk_g, *chunk_b;   // [gridDim]
    unsigned long long *best;
};

__global__ void __launch_bounds__(256) k_fm_best(FmBestArgs a) {
    cg::grid_group grid = cg::this_grid();
    __shared__ uint64_t sm[33];
    const uint32_t chunk = (a.k + gridDim.x - 1) / gridDim.x;
    const uint64_t c0 = (uint64_t)blockIdx.x * chunk;
    const uint64_t c1 = c0 + chunk < a.k ? c0 + chunk : a.k;
    long long sg = 0, sb = 0;
    for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
        sg += a.gseq[i];
        sb += a.side[i] == 0 ? -2 : 2;
    }
    uint64_t t1, t2;
    block_scan_u64((uint64_t)sg, sm, &t1);
    block_scan_u64((uint64_t)sb, sm, &t2);
    if (threadIdx.x == 0) {
        a.chunk_g[blockIdx.x] = (long long)t1;
        a.chunk_b[blockIdx.x] = (long long)t2;
    }
    grid.sync();
    long long base_g = 0, base_b = 0;
    for (uint32_t b = 0; b < blockIdx.x; b++) {
        base_g += a.chunk_g[b];
        base_b += a.chunk_b[b];
    }
    unsigned long long best = ~0ull;
    for (uint64_t s0 = c0; s0 < c1; s0 += blockDim.x) {
        const uint64_t i = s0 + threadIdx.x;
        const long long g = i < c1 ? a.gseq[i] : 0;
        const long long sbv = i < c1 ? (a.side[i] == 0 ? -2 : 2) : 0;
        uint64_t tg, tb;
        const long long ig = (long long)block_scan_u64((uint64_t)g, sm, &tg);
        const long long ib = (long long)block_scan_u64((uint64_t)sbv, sm, &tb);
        if (i < c1) {
            const long long cut = a.cut0 - (base_g + ig);
            long long bal = a.bal0 + base_b + ib;
            bal = bal < 0 ? -bal : bal;
            if (bal <= a.target) {
                const unsigned long long key = ((unsigned long long)cut << 32) | (0xFFFFFFFFu - (uint32_t)(i + 1));
                best = key < best ? key : best;
            }
        }
        base_g += (long long)tg;
        base_b += (long long)tb;
    }
    // block minimum, one atomic
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xFFFFFFFFu, best, o);
        best = x < best ? x : best;
    }
    if ((threadIdx.x & 31) == 0 && best != ~0ull) atomicMin(a.best, best);
}

__global__ void k_fm_apply(uint32_t k, const uint32_t *__restrict__ order, uint32_t *__restrict__ part) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += stride) part[order[i]] ^= 1u;
}

static uint32_t fm_grid(Context &C, uint64_t items) {
    uint64_t g = (items + 255) / 256;
    const uint64_t cap = (uint64_t)C.num_sms * 16;
    if (g > cap) g = cap;
    return g ? (uint32_t)g : 1u;
}

template <typename W>
static int fm_impl(Context &C, const Level &L, const W *w, uint32_t *part, uint32_t max_passes, uint64_t *cut_out,
                   uint32_t *passes_out, uint64_t *moves_out) {
    const uint32_t n = L.n;
    long long *gain, *gseq, *chunk_g, *chunk_b;
    uint8_t *f0, *f1, *side;
    uint32_t *A, *B, *sa, *sb, *order, *rank, *cnt, *hist, *off;
    unsigned long long *sums, *best;
    SGPB_TRY(dalloc_t(C, &gain, n));
    SGPB_TRY(dalloc_t(C, &gseq, n));
    SGPB_TRY(dalloc_t(C, &f0, n));
    SGPB_TRY(dalloc_t(C, &f1, n));
    SGPB_TRY(dalloc_t(C, &side, n));
    SGPB_TRY(dalloc_t(C, &A, n));
    SGPB_TRY(dalloc_t(C, &B, n));
    SGPB_TRY(dalloc_t(C, &sa, n));
    SGPB_TRY(dalloc_t(C, &sb, n));
    SGPB_TRY(dalloc_t(C, &order, n));
    SGPB_TRY(dalloc_t(C, &rank, n));
    SGPB_TRY(dalloc_t(C, &cnt, 2));
    SGPB_TRY(dalloc_t(C, &sums, 2));
    SGPB_TRY(dalloc_t(C, &best, 1));
    const uint32_t max_tiles = cdiv(n, kFmTile);
    SGPB_TRY(dalloc_t(C, &hist, (size_t)kFmBuckets * max_tiles + 1));
    SGPB_TRY(dalloc_t(C, &off, (size_t)kFmBuckets * max_tiles + 1));
    int per_sm = 0;
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fm_best, 256, 0));
    if (per_sm < 1) {
        set_error("FM best-prefix kernel does not fit on an SM");
        return SGP_B200_ERR_DEVICE;
    }
    const uint32_t bgrid_max = (uint32_t)per_sm * C.num_sms;
    SGPB_TRY(dalloc_t(C, &chunk_g, bgrid_max));
    SGPB_TRY(dalloc_t(C, &chunk_b, bgrid_max));
    const double avg = n ? (double)L.m / n : 0;
    uint64_t moves = 0;
    uint32_t pass = 0;
    for (; pass < max_passes; pass++) {
        SGPB_TRY(dzero(C, sums, 2 * sizeof(unsigned long long)));
#define SGPB_FMG(G) k_fm_gain<G><<<fm_grid(C, (uint64_t)n * G), 256, 0, C.stream>>>(n, L.rp, L.col, part, gain, f0, f1, sums)
        if (avg <= 4) SGPB_FMG(4);
        else if (avg <= 16) SGPB_FMG(16);
        else SGPB_FMG(32);
#undef SGPB_FMG
        SGPB_TRY(compact_flags(C, f0, n, A, cnt));
        SGPB_TRY(compact_flags(C, f1, n, B, cnt + 1));
        uint32_t nab[2];
        uint64_t s[2];
        SGPB_TRY(read_u32(C, cnt, nab, 2));
        SGPB_TRY(read_u64(C, (const uint64_t *)sums, s, 2));
        const long long cut0 = (long long)(s[0] / 2), bal0 = (long long)s[1];
        if (pass == 0 && cut_out) *cut_out = (uint64_t)cut0;
        const uint32_t na = nab[0], nb = nab[1], k = na + nb;
        C.kernel_launches += 1;
        if (k == 0) break;
        // stable counting sort of each list by descending clamped gain
        for (int sd = 0; sd < 2; sd++) {
            const uint32_t len = sd == 0 ? na : nb;
            if (!len) continue;
            const uint32_t *src = sd == 0 ? A : B;
            uint32_t *dst = sd == 0 ? sa : sb;
            const uint32_t nt = cdiv(len, kFmTile);
            k_fm_hist<<<nt, kFmTile, 0, C.stream>>>(len, src, gain, nt, hist);
            SGPB_TRY(scan_u32(C, hist, off, kFmBuckets * nt, nullptr));
            k_fm_place<<<nt, kFmTile, 0, C.stream>>>(len, src, gain, nt, off, dst);
            C.kernel_launches += 2;
        }
        SGPB_CUDA(cudaMemsetAsync(rank, 0xFF, sizeof(uint32_t) * n, C.stream));
        k_fm_interleave<<<fm_grid(C, na > nb ? na : nb), 256, 0, C.stream>>>(na, nb, sa, sb, gain, bal0, order, rank,
                                                                             side);
#define SGPB_FMS(G) k_fm_seqgain<G><<<fm_grid(C, (uint64_t)k * G), 256, 0, C.stream>>>(k, L.rp, L.col, part, order, rank, gseq)
        if (avg <= 4) SGPB_FMS(4);
        else if (avg <= 16) SGPB_FMS(16);
        else SGPB_FMS(32);
#undef SGPB_FMS
        FmBestArgs ba;
        ba.k = k;
        ba.gseq = gseq;
        ba.side = side;
        ba.cut0 = cut0;
        ba.bal0 = bal0;
        const long long ab = bal0 < 0 ? -bal0 : bal0;
        ba.target = ab / 10 > 20 ? ab / 10 : 20;
        ba.chunk_g = chunk_g;
        ba.chunk_b = chunk_b;
        ba.best = best;
        const unsigned long long key0 = ((unsigned long long)cut0 << 32) | 0xFFFFFFFFull;   // k = 0
        SGPB_CUDA(cudaMemcpyAsync(best, &key0, sizeof(key0), cudaMemcpyHostToDevice, C.stream));
        uint32_t bg = cdiv(k, 1024);
        if (bg > bgrid_max) bg = bgrid_max;
        if (bg < 1) bg = 1;
        void *args[] = {&ba};
        SGPB_CUDA(cudaLaunchCooperativeKernel((const void *)k_fm_best, dim3(bg), dim3(256), args, 0, C.stream));
        C.kernel_launches += 3;
        uint64_t bk = 0;
        SGPB_TRY(read_u64(C, (const uint64_t *)best, &bk));
        const uint32_t kstar = 0xFFFFFFFFu - (uint32_t)(bk & 0xFFFFFFFFu);
        const long long best_cut = (long long)(bk >> 32);
        if (kstar == 0 || best_cut == cut0) break;
        k_fm_apply<<<fm_grid(C, kstar), 256, 0, C.stream>>>(kstar, order, part);
        C.kernel_launches++;
        SGPB_CUDA(cudaGetLastError());
        moves += kstar;
        if (cut_out) *cut_out = (uint64_t)best_cut;
    }
    SGPB_CUDA(cudaGetLastError());
    if (passes_out) *passes_out = pass;
    if (moves_out) *moves_out = moves;
    return SGP_B200_OK;
}

// On the finest level, whose edges all weigh 1 in the reference (its loader
// sets every value to 1), so the cut is the edge count the split reports.
int fm_refine_level(Context &C, const Level &L, uint32_t *part, uint32_t max_passes, uint64_t *cut_out,
                    uint32_t *passes_out, uint64_t *moves_out) {
    if (L.n == 0 || max_passes == 0) {
        if (passes_out) *passes_out = 0;
        if (moves_out) *moves_out = 0;
        return SGP_B200_OK;
    }
    return fm_impl<uint32_t>(C, L, nullptr, part, max_passes, cut_out, passes_out, moves_out);
}

__global__ void k_count_zero(uint32_t n, const uint32_t *__restrict__ part, uint32_t *__restrict__ out) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t z = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) z += part[i] == 0;
    z = warp_sum(z);
    if (lane == 0 && z) atomicAdd(out, z);
}

int count_part0(Context &C, const uint32_t *part, uint32_t n, uint32_t *out) {
    uint32_t *d;
    SGPB_TRY(dalloc_t(C, &d, 1));
    SGPB_TRY(dzero(C, d, 4));
    k_count_zero<<<fm_grid(C, n), 256, 0, C.stream>>>(n, part, d);
    C.kernel_launches++;
    SGPB_CUDA(cudaGetLastError());
    return read_u32(C, d, out);
}

}  // namespace sgpb
