// build.cu -- coarse-graph construction P^T A P of one level.
//
// Reference: cmg/coarsen_kokkos.h:1061-1127 (count + map), :799-900
// (sgp_build_nonskew: scan, atomic-slot bucket scatter, dedupe, compaction),
// :750-762 + :491-509 (RADIX dedupe: per-row sort by destination, run-sum).
// Output rows are sorted by destination with duplicate weights summed and
// self loops dropped -- the RADIX build's output, independent of the order in
// which the scatter filled the buckets, so the result is deterministic.
//
// Per-row dedupe is tiered by bucket size:
//   tier 1 (<= 32 entries)   one warp, bitonic sort in registers
//   tier 1b (<= kT1 entries) a 64-thread block, radix sort in shared memory
//   tier 1c (<= kT1M)        a 128-thread block, radix sort in shared memory
//   tier 2 (<= kT2H / kT2)   a 256- / 512-thread block, radix sort in shared memory
//   tier 3 (larger)          dense accumulation over [0, nc): in one block's
//                            shared memory when nc weights and their bitmap fit
//                            (a block per row at a time), else in global memory
//                            (bitmap + weight array, L2-resident); compacted in
//                            ascending destination order
#include <type_traits>

#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kT2 = 4096;
constexpr uint32_t kSentinel = 0xFFFFFFFFu;

// Rows longer than kLongRowT entries (the hubs of skewed graphs, up to
// hundreds of thousands of entries) would hold one group for the whole of a
// rows-strided kernel: the count and key kernels list them and leave them to
// a kernel that gives each such row a block.
constexpr uint32_t kLongRowT = 8192;
// levels with at least this many entries keep their entries' coarse
// destinations from the count for the scatter (k_build_count's cvs)
constexpr uint64_t kStoreCvMin = 1ull << 20;
constexpr int kLongThreads = 1024;

__device__ __forceinline__ void list_long_row(uint32_t *long_list, uint32_t *long_cnt, uint32_t u) {
    long_list[atomicAdd(long_cnt, 1u)] = u;
}

// block-wide sum for the long-row kernels (result on thread 0)
template <typename T>
__device__ __forceinline__ T block_sum_long(T v, T *sm /* kLongThreads / 32 */) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += sm[k];
    __syncthreads();
    return t;
}

// ---------------------------------------------------------------- count --
// Per fine row u: krow[u] = entries whose coarse destination differs from
// vcmap[u]; cnt[vcmap[u]] += krow[u].  A group of G lanes per row, 4 entries
// per lane in flight (destinations, then the vcmap gathers); rows longer than
// kLongRowT are listed for k_build_count_long.
template <int G>
__global__ void __launch_bounds__(256) k_build_count(uint32_t n, const uint32_t *__restrict__ rp,
                                                     const uint32_t *__restrict__ col,
                                                     const uint32_t *__restrict__ vcmap,
                                                     uint32_t *__restrict__ cnt, uint32_t *__restrict__ krow,
                                                     uint32_t *__restrict__ long_list,
                                                     uint32_t *__restrict__ long_cnt, uint32_t *__restrict__ cvs) {
    const unsigned gm = group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t u = gid; u < n; u += ngroups) {
        const uint32_t cu = vcmap[u];
        const uint32_t b = rp[u], e = rp[u + 1];
        if (e - b > kLongRowT) {   // group-uniform
            if (lane == 0) list_long_row(long_list, long_cnt, (uint32_t)u);
            continue;
        }
        uint32_t c = 0;
        for (uint32_t j0 = b + lane; j0 < e; j0 += 4 * G) {
            uint32_t d[4];
#pragma unroll
            for (int q = 0; q < 4; q++) d[q] = j0 + q * G < e ? __ldg(col + j0 + q * G) : 0u;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (j0 + q * G < e) {
                    const uint32_t cv = __ldg(vcmap + d[q]);
                    if (cvs) cvs[j0 + q * G] = cv;
                    c += cv != cu;
                }
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) c += __shfl_xor_sync(gm, c, o);
        if (lane == 0) {
            krow[u] = c;
            if (c) atomicAdd(cnt + cu, c);
        }
    }
}

// the long rows of k_build_count, a block per row
__global__ void __launch_bounds__(kLongThreads) k_build_count_long(const uint32_t *__restrict__ rp,
                                                                 const uint32_t *__restrict__ col,
                                                                 const uint32_t *__restrict__ vcmap,
                                                                 uint32_t *__restrict__ cnt,
                                                                 uint32_t *__restrict__ krow,
                                                                 const uint32_t *__restrict__ long_list,
                                                                 const uint32_t *__restrict__ long_cnt,
                                                                 uint32_t *__restrict__ cvs) {
    __shared__ uint32_t sm[kLongThreads / 32];
    const uint32_t nl = *long_cnt;
    for (uint32_t r = blockIdx.x; r < nl; r += gridDim.x) {
        const uint32_t u = long_list[r];
        const uint32_t cu = vcmap[u];
        const uint32_t b = rp[u], e = rp[u + 1];
        uint32_t c = 0;
        for (uint32_t j0 = b + threadIdx.x; j0 < e; j0 += 4 * blockDim.x) {
            uint32_t d[4];
#pragma unroll
            for (int q = 0; q < 4; q++) d[q] = j0 + q * blockDim.x < e ? __ldg(col + j0 + q * blockDim.x) : 0u;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (j0 + q * blockDim.x < e) {
                    const uint32_t cv = __ldg(vcmap + d[q]);
                    if (cvs) cvs[j0 + q * blockDim.x] = cv;
                    c += cv != cu;
                }
        }
        c = block_sum_long(c, sm);
        if (threadIdx.x == 0) {
            krow[u] = c;
            if (c) atomicAdd(cnt + cu, c);
        }
    }
}

// -------------------------------------------------------------- scatter --
// Row u reserves krow[u] consecutive slots of bucket vcmap[u] with one atomic
// and writes its kept (coarse destination, weight) pairs there in entry
// order.  The order of the rows inside a bucket depends on the atomics; the
// dedupe sorts each bucket, so the coarse graph does not.
template <int G, typename WI>
__global__ void __launch_bounds__(256) k_build_scatter(uint32_t n, const uint32_t *__restrict__ rp,
                                                       const uint32_t *__restrict__ col, const WI *__restrict__ w,
                                                       const uint32_t *__restrict__ vcmap,
                                                       const uint32_t *__restrict__ krow,
                                                       const uint32_t *__restrict__ boff, uint32_t *__restrict__ fill,
                                                       uint32_t *__restrict__ bdst, WI *__restrict__ bw,
                                                       const uint32_t *__restrict__ cvs) {
    const unsigned gm = group_mask<G>();
    const uint32_t lane = threadIdx.x & (G - 1);
    const unsigned lane32 = threadIdx.x & 31;
    const unsigned gshift = lane32 & ~(unsigned)(G - 1);
    const unsigned gbits = 0xFFFFFFFFu >> (32 - G);
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t u = gid; u < n; u += ngroups) {
        const uint32_t k = krow[u];
        if (k == 0) continue;   // group-uniform
        const uint32_t cu = vcmap[u];
        const uint32_t b = rp[u], e = rp[u + 1];
        if (e - b > kLongRowT) continue;   // k_build_scatter_long
        uint32_t base = 0;
        if (lane == 0) base = boff[cu] + atomicAdd(fill + cu, k);
        base = __shfl_sync(gm, base, 0, G);
        for (uint32_t j0 = b; j0 < e; j0 += 4 * G) {
            uint32_t cv[4];
            WI wv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t j = j0 + q * G + lane;
                cv[q] = j < e ? __ldg((cvs ? cvs : col) + j) : 0u;
                if (w) wv[q] = j < e ? __ldg(w + j) : (WI)0;
            }
            if (!cvs)
#pragma unroll
                for (int q = 0; q < 4; q++) cv[q] = j0 + q * G + lane < e ? __ldg(vcmap + cv[q]) : cu;
            else
#pragma unroll
                for (int q = 0; q < 4; q++) cv[q] = j0 + q * G + lane < e ? cv[q] : cu;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const bool keep = cv[q] != cu;
                const unsigned bal = (__ballot_sync(gm, keep) >> gshift) & gbits;
                if (keep) {
                    const uint32_t p = base + __popc(bal & ((1u << lane) - 1u));
                    bdst[p] = cv[q];
                    if (w) bw[p] = wv[q];
                }
                base += __popc(bal);
            }
        }
    }
}

// The long rows: a block per row reserves the row's slots with one atomic
// and places its kept entries there in warp order (any order: the dedupe
// sorts each bucket, and integer weights sum the same either way).
template <typename WI>
__global__ void __launch_bounds__(kLongThreads) k_build_scatter_long(
    const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, const WI *__restrict__ w,
    const uint32_t *__restrict__ vcmap, const uint32_t *__restrict__ krow, const uint32_t *__restrict__ boff,
    uint32_t *__restrict__ fill, uint32_t *__restrict__ bdst, WI *__restrict__ bw,
    const uint32_t *__restrict__ long_list, const uint32_t *__restrict__ long_cnt, const uint32_t *__restrict__ cvs) {
    __shared__ uint32_t s_base, s_pos;
    const uint32_t nl = *long_cnt;
    const unsigned lane = threadIdx.x & 31;
    for (uint32_t r = blockIdx.x; r < nl; r += gridDim.x) {
        const uint32_t u = long_list[r];
        const uint32_t k = krow[u];
        if (k == 0) continue;   // block-uniform
        const uint32_t cu = vcmap[u];
        const uint32_t b = rp[u], e = rp[u + 1];
        if (threadIdx.x == 0) {
            s_base = boff[cu] + atomicAdd(fill + cu, k);
            s_pos = 0;
        }
        __syncthreads();
        const uint32_t base = s_base;
        // whole warps per step (the loop bound is warp-uniform)
        for (uint32_t j0 = b + (threadIdx.x & ~31u); j0 < e; j0 += blockDim.x) {
            const uint32_t j = j0 + lane;
            const uint32_t cv = j < e ? (cvs ? __ldg(cvs + j) : __ldg(vcmap + __ldg(col + j))) : cu;
            const WI wv = (w && j < e) ? __ldg(w + j) : (WI)0;
            const bool keep = cv != cu;
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
            uint32_t p0 = 0;
            if (lane == 0 && bal) p0 = atomicAdd(&s_pos, (uint32_t)__popc(bal));
            p0 = __shfl_sync(0xFFFFFFFFu, p0, 0);
            if (keep) {
                const uint32_t p = base + p0 + __popc(bal & ((1u << lane) - 1u));
                bdst[p] = cv;
                if (w) bw[p] = wv;
            }
        }
        __syncthreads();   // s_base / s_pos are rewritten for the next row
    }
}

// ------------------------------------------------------------- classify --
// Bucket sizes 1..32 -> list 0 (one warp), 33..kT1 -> list 1 (64 threads),
// ..kT1M -> list 2 (128 threads), ..kT2H -> list 3 (256 threads), ..kT2 ->
// list 4 (512 threads), ..kGiant -> list 5 (dense), larger -> list 6 (dense,
// many blocks a row); one atomic per warp and list.
constexpr uint32_t kT1 = 256;
constexpr uint32_t kT1M = 1024;
constexpr uint32_t kT2H = 2048;
constexpr int kLists = 7;

// buckets above this many entries are split over many blocks (tier 4)
constexpr uint32_t kGiant = 1u << 18;

__global__ void k_classify(uint32_t nc, const uint32_t *__restrict__ boff, uint32_t *__restrict__ dcnt,
                           uint32_t *__restrict__ lists /* kLists x nc */, uint32_t *__restrict__ tcount /* kLists */) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    int t = -1;
    if (c < nc) {
        const uint32_t sz = boff[c + 1] - boff[c];
        if (sz == 0) dcnt[c] = 0;
        else t = sz <= 32 ? 0 : sz <= kT1 ? 1 : sz <= kT1M ? 2 : sz <= kT2H ? 3 : sz <= (uint32_t)kT2 ? 4 : sz <= kGiant ? 5 : 6;
    }
#pragma unroll
    for (int q = 0; q < kLists; q++) {
        const unsigned m = __ballot_sync(0xFFFFFFFFu, t == q);
        if (!m) continue;   // warp-uniform
        const int leader = __ffs(m) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(tcount + q, (uint32_t)__popc(m));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (t == q) lists[(size_t)q * nc + base + __popc(m & ((1u << lane) - 1u))] = c;
    }
}

// --------------------------------------------------------------- tier 1 --
template <typename WI, typename WO>
__global__ void __launch_bounds__(256) k_dedupe_warp(const uint32_t *__restrict__ list, const uint32_t *__restrict__ count,
                                                     const uint32_t *__restrict__ boff, uint32_t *__restrict__ bdst,
                                                     const WI *__restrict__ bw, WO *__restrict__ tw,
                                                     uint32_t *__restrict__ dcnt) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t cntv = *count;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = wid; k < cntv; k += nw) {
        const uint32_t c = list[k];
        const uint32_t b = boff[c], sz = boff[c + 1] - b;
        uint32_t key = kSentinel;
        uint64_t wv = 0;
        if (lane < sz) {
            key = bdst[b + lane];
            wv = bw ? (uint64_t)bw[b + lane] : 1ull;
        }
        // bitonic sort of 32 (key, weight) pairs across the warp
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                uint32_t ok = __shfl_xor_sync(0xFFFFFFFFu, key, j);
                uint64_t ow = __shfl_xor_sync(0xFFFFFFFFu, wv, j);
                bool up = (lane & kk) == 0;
                bool lower = (lane & j) == 0;
                bool take = lower ? (up ? ok < key : ok > key) : (up ? ok > key : ok < key);
                if (take) { key = ok; wv = ow; }
            }
        }
        uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, key, 1);
        bool valid = key != kSentinel;
        bool head = valid && (lane == 0 || prev != key);
        unsigned hm = __ballot_sync(0xFFFFFFFFu, head);
        uint32_t seg = __popc(hm & ((2u << lane) - 1u));   // 1-based run id
        uint64_t s = wv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t t = __shfl_up_sync(0xFFFFFFFFu, s, o);
            uint32_t ts = __shfl_up_sync(0xFFFFFFFFu, seg, o);
            if (lane >= (unsigned)o && ts == seg) s += t;
        }
        uint32_t next = __shfl_down_sync(0xFFFFFFFFu, key, 1);
        bool tail = valid && (lane == 31 || next != key);
        if (tail) {
            bdst[b + seg - 1] = key;
            tw[b + seg - 1] = (WO)s;
        }
        if (lane == 0) dcnt[c] = __popc(hm);
    }
}

// ------------------------------------------------------ tiers 1b and 2 --
// Buckets of 33 .. kT2 entries: a block per bucket at a time sorts the
// (destination, weight) pairs by an LSD radix sort in shared memory, 8 bits a
// pass over the low 8 * passes bits of the destinations (all below nc), then
// merges runs of equal destinations into the bucket's head.  Item q of a
// bucket is held by warp q / (32 R), round (q / 32) mod R, lane q mod 32; a
// pass ranks each warp's rounds in order with __match_any_sync against
// per-warp digit counters, so every pass is stable and the passes compose.
// A bitonic sort of the same bucket needs O(log^2) compare-exchange stages
// with a block barrier each; the radix passes need three barriers each.
template <typename WI, int WARPS, int R>
struct RadixDedupeCfg {
    static constexpr int kThreads = WARPS * 32;
    static constexpr uint32_t kCap = (uint32_t)WARPS * 32 * R;
    typedef typename std::conditional<sizeof(WI) == 8, unsigned long long, uint32_t>::type VT;
    static constexpr size_t kSmem = (size_t)kCap * (sizeof(uint32_t) + sizeof(VT));   // dynamic part
};

template <typename WI, typename WO, int WARPS, int R>
__global__ void __launch_bounds__(WARPS * 32) k_dedupe_radix(const uint32_t *__restrict__ list,
                                                             const uint32_t *__restrict__ count,
                                                             const uint32_t *__restrict__ boff,
                                                             uint32_t *__restrict__ bdst, const WI *__restrict__ bw,
                                                             WO *__restrict__ tw, uint32_t *__restrict__ dcnt,
                                                             int passes) {
    typedef RadixDedupeCfg<WI, WARPS, R> Cfg;
    typedef typename Cfg::VT VT;
    constexpr int kThreads = Cfg::kThreads;
    constexpr uint32_t kCap = Cfg::kCap;
    constexpr int kBins = 256;
    constexpr int kDpt = kBins >= kThreads ? kBins / kThreads : 1;   // digits per thread
    __shared__ uint32_t wcnt[WARPS][kBins];
    __shared__ uint32_t dstart[kBins];
    __shared__ uint64_t scan_sm[33];
    extern __shared__ __align__(16) unsigned char rd_smem[];
    uint32_t *sk = reinterpret_cast<uint32_t *>(rd_smem);
    VT *sv = reinterpret_cast<VT *>(rd_smem + kCap * sizeof(uint32_t));
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t cntv = *count;
    for (uint32_t k = blockIdx.x; k < cntv; k += gridDim.x) {
        const uint32_t c = list[k];
        const uint32_t b = boff[c], sz = boff[c + 1] - b;
        uint32_t key[R];
        VT val[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const uint32_t q = (wid * R + r) * 32 + lane;
            const bool valid = q < sz;
            key[r] = valid ? bdst[b + q] : 0u;
            val[r] = valid ? (bw ? (VT)bw[b + q] : (VT)1) : (VT)0;
        }
        for (int pass = 0; pass < passes; pass++) {
            const int shift = 8 * pass;
            for (int d = lane; d < kBins; d += 32) wcnt[wid][d] = 0;
            __syncwarp();
            uint32_t rank[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                if ((wid * R + r) * 32 >= sz) break;   // warp-uniform: rounds past the bucket
                const uint32_t q = (wid * R + r) * 32 + lane;
                const bool valid = q < sz;
                const uint32_t d = (key[r] >> shift) & 0xFFu;
                const unsigned act = __ballot_sync(0xFFFFFFFFu, valid);
                rank[r] = 0;
                if (valid) {
                    const unsigned peers = __match_any_sync(act, d);
                    rank[r] = wcnt[wid][d] + __popc(peers & ((1u << lane) - 1u));
                    __syncwarp(act);
                    if ((int)lane == __ffs(peers) - 1) wcnt[wid][d] += __popc(peers);
                }
                __syncwarp();
            }
            __syncthreads();
            // per digit: exclusive prefixes over the warps; digit starts from
            // a block scan of the digit totals (kDpt consecutive digits a thread)
            const uint32_t d0 = threadIdx.x * kDpt;
            uint32_t tot[kDpt];
            uint64_t tsum = 0;
            if (d0 < kBins) {
#pragma unroll
                for (int j = 0; j < kDpt; j++) {
                    uint32_t t = 0;
#pragma unroll
                    for (int w = 0; w < WARPS; w++) {
                        const uint32_t cw = wcnt[w][d0 + j];
                        wcnt[w][d0 + j] = t;
                        t += cw;
                    }
                    tot[j] = t;
                    tsum += t;
                }
            }
            uint64_t all;
            uint64_t ex = block_scan_u64(d0 < kBins ? tsum : 0, scan_sm, &all) - tsum;
            if (d0 < kBins) {
#pragma unroll
                for (int j = 0; j < kDpt; j++) {
                    dstart[d0 + j] = (uint32_t)ex;
                    ex += tot[j];
                }
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R; r++) {
                const uint32_t q = (wid * R + r) * 32 + lane;
                if (q < sz) {
                    const uint32_t d = (key[r] >> shift) & 0xFFu;
                    const uint32_t slot = dstart[d] + wcnt[wid][d] + rank[r];
                    sk[slot] = key[r];
                    sv[slot] = val[r];
                }
            }
            __syncthreads();
            // the next pass works on the staged order; its first barrier
            // (after the ranking) orders these reads before its scatter, and
            // each warp clears only its own counters, which the other
            // threads last read before this pass's second barrier
            if (pass + 1 < passes) {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const uint32_t q = (wid * R + r) * 32 + lane;
                    if (q < sz) {
                        key[r] = sk[q];
                        val[r] = sv[q];
                    }
                }
            }
        }
        // runs of equal destinations: each thread owns a contiguous segment
        const uint32_t per = (sz + kThreads - 1) / kThreads;
        const uint32_t s0 = threadIdx.x * per < sz ? threadIdx.x * per : sz;
        const uint32_t s1 = s0 + per < sz ? s0 + per : sz;
        uint64_t h = 0;
        for (uint32_t i = s0; i < s1; i++)
            if (i == 0 || sk[i - 1] != sk[i]) h++;
        uint64_t tot;
        uint64_t pos = block_scan_u64(h, scan_sm, &tot) - h;
        for (uint32_t i = s0; i < s1; i++) {
            const uint32_t key0 = sk[i];
            if (i == 0 || sk[i - 1] != key0) {
                uint64_t sum = sv[i];
                for (uint32_t q = i + 1; q < sz && sk[q] == key0; q++) sum += sv[q];
                bdst[b + pos] = key0;
                tw[b + pos] = (WO)sum;
                pos++;
            }
        }
        if (threadIdx.x == 0) dcnt[c] = (uint32_t)tot;
        __syncthreads();   // the staging arrays are reloaded by the next bucket
    }
}

// --------------------------------------------------------------- tier 3 --
// scatter-add of the rows [r0, r0 + nrows) of the tier-3 list into dense
// slots; blockIdx.y = row within the batch.
template <typename WI, typename WO>
__global__ void __launch_bounds__(256) k_dense_add(const uint32_t *__restrict__ list, uint32_t r0,
                                                  const uint32_t *__restrict__ boff, const uint32_t *__restrict__ bdst,
                                                  const WI *__restrict__ bw, uint32_t nc, WO *__restrict__ acc,
                                                  uint32_t *__restrict__ bits) {
    const uint32_t c = list[r0 + blockIdx.y];
    const uint32_t b = boff[c], e = boff[c + 1];
    WO *a = acc + (size_t)blockIdx.y * nc;
    uint32_t *bm = bits + (size_t)blockIdx.y * ((nc + 31) / 32);
    for (uint32_t j = b + blockIdx.x * blockDim.x + threadIdx.x; j < e; j += gridDim.x * blockDim.x) {
        uint32_t v = bdst[j];
        WO wv = bw ? (WO)bw[j] : (WO)1;
        atomicAdd(a + v, wv);
        uint32_t bit = 1u << (v & 31);
        if (!(__ldcg(bm + (v >> 5)) & bit)) atomicOr(bm + (v >> 5), bit);
    }
}

// Tier 3 in shared memory: a block per row at a time accumulates the row's
// weights over [0, nc) with shared-memory atomics (integer sums, so the order
// does not matter), then writes the destinations with a non-zero sum (every
// weight is positive) in ascending order with their sums to the bucket's
// head.  When nc is small the block keeps R copies of the accumulator (thread
// t adds to copy t mod R, up to one per thread) so that rows of millions of
// entries over a few dozen destinations do not serialise on the same words;
// with one copy a bitmap of the touched destinations keeps the compaction
// from scanning all nc sums.
constexpr int kDenseSmemThreads = 1024;

template <typename WO>
static size_t dense_smem_bytes(uint32_t nc, uint32_t R) {
    const size_t acc = (((size_t)R * nc * sizeof(WO)) + 15) & ~(size_t)15;
    return acc + (R == 1 ? (((size_t)nc + 31) / 32) * 4 : 0);
}

template <typename WI, typename WO>
__global__ void __launch_bounds__(kDenseSmemThreads, 1)
    k_dense_smem(const uint32_t *__restrict__ list, const uint32_t *__restrict__ nrows_ptr,
                 const uint32_t *__restrict__ boff, uint32_t *__restrict__ bdst, const WI *__restrict__ bw,
                 WO *__restrict__ tw, uint32_t *__restrict__ dcnt, uint32_t nc, uint32_t R) {
    extern __shared__ __align__(16) unsigned char dyn[];
    WO *acc = reinterpret_cast<WO *>(dyn);
    uint32_t *bits = reinterpret_cast<uint32_t *>(dyn + ((((size_t)R * nc * sizeof(WO)) + 15) & ~(size_t)15));
    __shared__ uint32_t warp_tot[kDenseSmemThreads / 32];
    const bool use_bits = R == 1;
    const uint32_t words = (nc + 31) / 32;
    const uint32_t nrows = *nrows_ptr;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WO *mine = acc + (size_t)(threadIdx.x % R) * nc;
    // compaction units: bitmap words, or accumulator entries; contiguous per
    // thread so that the output order is the thread order
    const uint32_t units = use_bits ? words : nc;
    const uint32_t upt = (units + kDenseSmemThreads - 1) / kDenseSmemThreads;
    for (uint32_t r = blockIdx.x; r < nrows; r += gridDim.x) {
        const uint32_t c = list[r];
        const uint32_t b = boff[c], e = boff[c + 1];
        for (uint32_t i = threadIdx.x; i < R * nc; i += blockDim.x) acc[i] = (WO)0;
        if (use_bits)
            for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bits[i] = 0u;
        __syncthreads();
        for (uint32_t j = b + threadIdx.x; j < e; j += blockDim.x) {
            const uint32_t v = bdst[j];
            atomicAdd(&mine[v], bw ? (WO)bw[j] : (WO)1);
            if (use_bits) atomicOr(&bits[v >> 5], 1u << (v & 31));
        }
        __syncthreads();
        if (R > 1) {   // the copies' sums into copy 0
            for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) {
                WO t = acc[i];
                for (uint32_t q = 1; q < R; q++) t += acc[(size_t)q * nc + i];
                acc[i] = t;
            }
            __syncthreads();
        }
        const uint32_t u0 = threadIdx.x * upt;
        uint32_t cnt = 0;
        for (uint32_t k = 0; k < upt && u0 + k < units; k++)
            cnt += use_bits ? __popc(bits[u0 + k]) : (acc[u0 + k] != (WO)0);
        // exclusive prefix of cnt over the block
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (unsigned)o) incl += y;
        }
        if (lane == 31) warp_tot[wid] = incl;
        __syncthreads();
        uint32_t base = 0, total = 0;
        for (uint32_t k = 0; k < kDenseSmemThreads / 32; k++) {
            if (k < wid) base += warp_tot[k];
            total += warp_tot[k];
        }
        uint32_t pos = b + base + incl - cnt;
        for (uint32_t k = 0; k < upt && u0 + k < units; k++) {
            if (use_bits) {
                uint32_t word = bits[u0 + k];
                while (word) {
                    const int bit = __ffs(word) - 1;
                    word &= word - 1;
                    const uint32_t v = (u0 + k) * 32 + bit;
                    bdst[pos] = v;
                    tw[pos] = acc[v];
                    pos++;
                }
            } else if (acc[u0 + k] != (WO)0) {
                bdst[pos] = u0 + k;
                tw[pos] = acc[u0 + k];
                pos++;
            }
        }
        if (threadIdx.x == 0) dcnt[c] = total;
        __syncthreads();   // the next row clears acc, bits and warp_tot
    }
}

// Compaction of the dense slots in ascending destination order, clearing
// them for reuse.  A slot's bitmap is cut into chunks of kChunkWords words,
// one block per (chunk, slot): k_dense_count counts the bits of each chunk,
// k_dense_collect finds its chunk's output offset from the counts before it
// and writes the chunk -- every warp 32 consecutive words at a time, a lane
// per word -- so the weight loads of many chunks are in flight at once.
constexpr uint32_t kChunkWords = 8192;
constexpr int kCollectWarps = 8;                         // 256 threads
constexpr uint32_t kWarpWords = kChunkWords / kCollectWarps;   // contiguous words per warp

__global__ void __launch_bounds__(256) k_dense_count(uint32_t nc, const uint32_t *__restrict__ bits,
                                                    uint32_t *__restrict__ chunk_cnt) {
    const uint32_t nwords = (nc + 31) / 32;
    const uint32_t nchunks = gridDim.x;
    const uint32_t *bm = bits + (size_t)blockIdx.y * nwords;
    const uint32_t w0 = blockIdx.x * kChunkWords;
    uint32_t c = 0;
    for (uint32_t w = w0 + threadIdx.x; w < w0 + kChunkWords && w < nwords; w += blockDim.x) c += __popc(__ldcg(bm + w));
    c = warp_sum(c);
    __shared__ uint32_t ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += ws[i];
        chunk_cnt[(size_t)blockIdx.y * nchunks + blockIdx.x] = t;
    }
}

template <typename WO>
__global__ void __launch_bounds__(256) k_dense_collect(const uint32_t *__restrict__ list, uint32_t r0,
                                                      const uint32_t *__restrict__ boff, uint32_t nc,
                                                      WO *__restrict__ acc, uint32_t *__restrict__ bits,
                                                      const uint32_t *__restrict__ chunk_cnt,
                                                      uint32_t *__restrict__ bdst, WO *__restrict__ tw,
                                                      uint32_t *__restrict__ dcnt) {
    __shared__ uint32_t warp_tot[kCollectWarps];
    __shared__ uint32_t chunk_base;
    const uint32_t c = list[r0 + blockIdx.y];
    const uint32_t b = boff[c];
    const uint32_t nwords = (nc + 31) / 32;
    const uint32_t nchunks = gridDim.x;
    WO *a = acc + (size_t)blockIdx.y * nc;
    uint32_t *bm = bits + (size_t)blockIdx.y * nwords;
    const uint32_t *cc = chunk_cnt + (size_t)blockIdx.y * nchunks;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        uint32_t before = 0, all = 0;
        for (uint32_t k = 0; k < nchunks; k++) {
            if (k == blockIdx.x) before = all;
            all += cc[k];
        }
        chunk_base = before;
        if (blockIdx.x == 0) dcnt[c] = all;
    }
    // this warp's words and their bit count
    const uint32_t ws0 = blockIdx.x * kChunkWords + wid * kWarpWords;
    uint32_t cnt = 0;
    for (uint32_t w = ws0 + lane; w < ws0 + kWarpWords && w < nwords; w += 32) cnt += __popc(__ldcg(bm + w));
    cnt = warp_sum(cnt);
    if (lane == 0) warp_tot[wid] = cnt;
    __syncthreads();
    uint32_t pos = b + chunk_base;
    for (uint32_t k = 0; k < wid; k++) pos += warp_tot[k];
    for (uint32_t w0 = ws0; w0 < ws0 + kWarpWords && w0 < nwords; w0 += 32) {
        const uint32_t w = w0 + lane;
        uint32_t word = w < nwords ? __ldcg(bm + w) : 0u;
        const uint32_t pc = __popc(word);
        uint32_t incl = pc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (unsigned)o) incl += y;
        }
        uint32_t p = pos + incl - pc;
        if (word) bm[w] = 0;
        while (word) {
            const int bit = __ffs(word) - 1;
            word &= word - 1;
            const uint32_t v = w * 32 + bit;
            bdst[p] = v;
            tw[p] = a[v];
            a[v] = 0;
            p++;
        }
        pos += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
}

// Tier 3 when nc does not fit one block's shared memory: the destination
// range is covered in chunks of C (as many weights and their bitmap as fit);
// for each chunk the block re-reads the row's bucket (L2-resident after the
// first pass), accumulates the destinations inside the chunk in shared
// memory and appends the chunk's touched destinations in ascending order.
// The bucket is read again by later chunks, so the merged destinations go to
// the block's scratch (sdst + blockIdx.x * scap) and are copied over the
// bucket's head once the row is done; the weights go straight to tw.  No
// global accumulator slots: the global-memory form moved about 1.1 GB of DRAM
// for R-MAT scale 20's level-0 build, n_c words per row.
template <typename WI, typename WO>
__global__ void __launch_bounds__(kDenseSmemThreads, 1)
    k_dense_chunked(const uint32_t *__restrict__ list, const uint32_t *__restrict__ nrows_ptr,
                    const uint32_t *__restrict__ boff, uint32_t *__restrict__ bdst, const WI *__restrict__ bw,
                    WO *__restrict__ tw, uint32_t *__restrict__ dcnt, uint32_t nc, uint32_t C,
                    uint32_t *__restrict__ sdst, uint32_t scap) {
    extern __shared__ __align__(16) unsigned char dyn[];
    WO *acc = reinterpret_cast<WO *>(dyn);
    uint32_t *bits = reinterpret_cast<uint32_t *>(dyn + ((((size_t)C * sizeof(WO)) + 15) & ~(size_t)15));
    __shared__ uint32_t warp_tot[kDenseSmemThreads / 32];
    const uint32_t nrows = *nrows_ptr;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t *mydst = sdst + (size_t)blockIdx.x * scap;
    for (uint32_t r = blockIdx.x; r < nrows; r += gridDim.x) {
        const uint32_t c = list[r];
        const uint32_t b = boff[c], e = boff[c + 1];
        uint32_t done = 0;   // merged entries of the row so far
        for (uint32_t c0 = 0; c0 < nc; c0 += C) {
            const uint32_t clen = nc - c0 < C ? nc - c0 : C;
            const uint32_t words = (clen + 31) / 32;
            for (uint32_t i = threadIdx.x; i < clen; i += blockDim.x) acc[i] = (WO)0;
            for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bits[i] = 0u;
            __syncthreads();
            for (uint32_t j = b + threadIdx.x; j < e; j += blockDim.x) {
                const uint32_t v = bdst[j] - c0;
                if (v < clen) {
                    atomicAdd(&acc[v], bw ? (WO)bw[j] : (WO)1);
                    atomicOr(&bits[v >> 5], 1u << (v & 31));
                }
            }
            __syncthreads();
            const uint32_t upt = (words + kDenseSmemThreads - 1) / kDenseSmemThreads;
            const uint32_t u0 = threadIdx.x * upt;
            uint32_t cnt = 0;
            for (uint32_t k = 0; k < upt && u0 + k < words; k++) cnt += __popc(bits[u0 + k]);
            uint32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= (unsigned)o) incl += y;
            }
            if (lane == 31) warp_tot[wid] = incl;
            __syncthreads();
            uint32_t base = 0, total = 0;
            for (uint32_t k = 0; k < kDenseSmemThreads / 32; k++) {
                if (k < wid) base += warp_tot[k];
                total += warp_tot[k];
            }
            uint32_t pos = done + base + incl - cnt;
            for (uint32_t k = 0; k < upt && u0 + k < words; k++) {
                uint32_t word = bits[u0 + k];
                while (word) {
                    const int bit = __ffs(word) - 1;
                    word &= word - 1;
                    const uint32_t v = (u0 + k) * 32 + bit;
                    mydst[pos] = c0 + v;
                    tw[b + pos] = acc[v];
                    pos++;
                }
            }
            done += total;
            __syncthreads();   // acc, bits and warp_tot are reused by the next chunk
        }
        for (uint32_t i = threadIdx.x; i < done; i += blockDim.x) bdst[b + i] = mydst[i];
        if (threadIdx.x == 0) dcnt[c] = done;
        __syncthreads();   // the block's scratch is rewritten by its next row
    }
}

// ---------------------------------------------------------- compaction --
constexpr int kCompactU = 8;   // entries per lane in flight
// Copies the merged buckets into the coarse CSR; with 32-bit weights it also
// keeps their maximum in *wmax (when given), which decides how narrow the
// power iteration's copy of the level can store them.
template <typename WO>
__global__ void __launch_bounds__(256) k_compact_rows(uint32_t nc, const uint32_t *__restrict__ boff,
                                                     const uint32_t *__restrict__ crp,
                                                     const uint32_t *__restrict__ bdst, const WO *__restrict__ tw,
                                                     uint32_t *__restrict__ ccol, WO *__restrict__ cw,
                                                     uint32_t *__restrict__ wmax) {
    const unsigned lane = threadIdx.x & 31;
    uint32_t mx = 0;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = wid; c < nc; c += nw) {
        const uint32_t src = boff[c], dst = crp[c], len = crp[c + 1] - dst;
        // kCompactU entries per lane in flight: loads first, then stores
        for (uint32_t i0 = lane; i0 < len; i0 += 32 * kCompactU) {
            uint32_t d[kCompactU];
            WO x[kCompactU];
#pragma unroll
            for (int k = 0; k < kCompactU; k++) {
                const uint32_t i = i0 + 32 * k;
                d[k] = i < len ? __ldg(bdst + src + i) : 0u;
                x[k] = i < len ? __ldg(tw + src + i) : (WO)0;
            }
#pragma unroll
            for (int k = 0; k < kCompactU; k++) {
                const uint32_t i = i0 + 32 * k;
                if (i < len) {
                    ccol[dst + i] = d[k];
                    cw[dst + i] = x[k];
                    if constexpr (sizeof(WO) == 4) mx = (uint32_t)x[k] > mx ? (uint32_t)x[k] : mx;
                }
            }
        }
    }
    if constexpr (sizeof(WO) == 4) {
        mx = warp_max(mx);
        if (wmax && lane == 0 && mx) atomicMax(wmax, mx);
    }
}

// ---------------------------------------------------------------- dedupe --
// Sort + merge of every bucket [boff[r], boff[r+1]) of bdst (weights bw, or
// unit weights when bw is null): dcnt[r] = distinct destinations of bucket
// r, written ascending to the bucket's head with summed weights in tw.
// Empty buckets get dcnt 0.
template <typename WI, typename WO>
static int dedupe_buckets(Context &C, uint32_t nc, const uint32_t *boff, uint32_t *bdst, const WI *bw, WO *tw,
                          uint32_t *dcnt) {
    uint32_t *lists, *tcount;
    SGPB_TRY(dalloc_t(C, &lists, (size_t)kLists * nc + 4));
    SGPB_TRY(dalloc_t(C, &tcount, kLists));
    SGPB_TRY(dzero(C, tcount, sizeof(uint32_t) * kLists));
    if (nc) {
        k_classify<<<cdiv(nc, 256), 256, 0, C.stream>>>(nc, boff, dcnt, lists, tcount);
        uint32_t g1 = cdiv(nc, 8);
        if (g1 > (uint32_t)C.num_sms * 16) g1 = C.num_sms * 16;
        k_dedupe_warp<WI, WO><<<g1 ? g1 : 1, 256, 0, C.stream>>>(lists, tcount, boff, bdst, bw, tw, dcnt);
        // radix tiers, each block sized for its buckets: 33 .. kT1 entries
        // in 64 threads, .. kT1M in 128, .. kT2H in 256, .. kT2 in 512
        int bits = 0;
        while (bits < 32 && (1ull << bits) < (uint64_t)nc) bits++;
        const int passes = bits > 0 ? (bits + 7) / 8 : 1;
        typedef RadixDedupeCfg<WI, 2, 4> Cfg1;
        typedef RadixDedupeCfg<WI, 4, 8> CfgM;
        typedef RadixDedupeCfg<WI, 8, 8> CfgH;
        typedef RadixDedupeCfg<WI, 16, 8> Cfg2;
        static_assert(Cfg1::kCap == kT1 && CfgM::kCap == kT1M && CfgH::kCap == kT2H && Cfg2::kCap == (uint32_t)kT2,
                      "tier sizes");
        k_dedupe_radix<WI, WO, 2, 4><<<(uint32_t)C.num_sms * 32, Cfg1::kThreads, Cfg1::kSmem, C.stream>>>(
            lists + nc, tcount + 1, boff, bdst, bw, tw, dcnt, passes);
        k_dedupe_radix<WI, WO, 4, 8><<<(uint32_t)C.num_sms * 12, CfgM::kThreads, CfgM::kSmem, C.stream>>>(
            lists + 2 * (size_t)nc, tcount + 2, boff, bdst, bw, tw, dcnt, passes);
        k_dedupe_radix<WI, WO, 8, 8><<<(uint32_t)C.num_sms * 4, CfgH::kThreads, CfgH::kSmem, C.stream>>>(
            lists + 3 * (size_t)nc, tcount + 3, boff, bdst, bw, tw, dcnt, passes);
        SGPB_CUDA(cudaFuncSetAttribute(k_dedupe_radix<WI, WO, 16, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Cfg2::kSmem));
        k_dedupe_radix<WI, WO, 16, 8><<<(uint32_t)C.num_sms * 2, Cfg2::kThreads, Cfg2::kSmem, C.stream>>>(
            lists + 4 * (size_t)nc, tcount + 4, boff, bdst, bw, tw, dcnt, passes);
        C.kernel_launches += 6;
        SGPB_CUDA(cudaGetLastError());
        uint32_t n34[2] = {0, 0};
        SGPB_TRY(read_u32(C, tcount + 5, n34, 2));
        const uint32_t n3 = n34[0], n4 = n34[1];
        // dense accumulation in global memory (L2-resident slots) of the rows
        // of `list`, `per_row` blocks per row
        auto dense_global = [&](const uint32_t *list, uint32_t nrows, uint32_t per_row) -> int {
            const size_t words = ((size_t)nc + 31) / 32;
            const size_t slot_bytes = (size_t)nc * sizeof(WO) + words * 4;
            size_t slots = ((size_t)1 << 30) / (slot_bytes ? slot_bytes : 1);
            if (slots < 1) slots = 1;
            if (slots > nrows) slots = nrows;
            if (slots > 65535) slots = 65535;
            WO *acc;
            uint32_t *bits, *chunk_cnt;
            const uint32_t nchunks = cdiv(words, kChunkWords);
            SGPB_TRY(dalloc_t(C, &acc, slots * nc));
            SGPB_TRY(dalloc_t(C, &bits, slots * words));
            SGPB_TRY(dalloc_t(C, &chunk_cnt, slots * nchunks));
            SGPB_TRY(dzero(C, acc, slots * nc * sizeof(WO)));
            SGPB_TRY(dzero(C, bits, slots * words * 4));
            for (uint32_t r0 = 0; r0 < nrows; r0 += (uint32_t)slots) {
                uint32_t nr = nrows - r0 < slots ? nrows - r0 : (uint32_t)slots;
                dim3 ga(per_row, nr), gc(nchunks, nr);
                k_dense_add<WI, WO><<<ga, 256, 0, C.stream>>>(list, r0, boff, bdst, bw, nc, acc, bits);
                k_dense_count<<<gc, 256, 0, C.stream>>>(nc, bits, chunk_cnt);
                k_dense_collect<WO><<<gc, 256, 0, C.stream>>>(list, r0, boff, nc, acc, bits, chunk_cnt, bdst, tw, dcnt);
                C.kernel_launches += 3;
            }
            SGPB_CUDA(cudaGetLastError());
            return SGP_B200_OK;
        };
        // tier 3: one block's shared memory per row when nc fits, else global
        // memory; accumulator copies that fit in one block's shared memory
        const size_t budget = C.smem_optin - 8 * 1024;
        uint32_t R = nc ? (uint32_t)(budget / ((size_t)nc * sizeof(WO))) : 1u;
        if (R > (uint32_t)kDenseSmemThreads) R = kDenseSmemThreads;
        while (R > 1 && dense_smem_bytes<WO>(nc, R) > budget) R--;
        const size_t dsm = R ? dense_smem_bytes<WO>(nc, R) : 0;
        if (n3 && R >= 1 && dsm <= budget) {
            // the limit is a property of the function, shared by every host
            // thread (batch workers): always the same bound, never this
            // launch's size, so no thread lowers it under another's launch
            SGPB_CUDA(cudaFuncSetAttribute(k_dense_smem<WI, WO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)budget));
            const uint32_t g3 = n3 < (uint32_t)C.num_sms ? n3 : (uint32_t)C.num_sms;
            k_dense_smem<WI, WO><<<g3, kDenseSmemThreads, dsm, C.stream>>>(lists + 5 * (size_t)nc, tcount + 5, boff,
                                                                          bdst, bw, tw, dcnt, nc, R);
            C.kernel_launches++;
            SGPB_CUDA(cudaGetLastError());
        } else if (n3) {
            // chunks of the destination range: weights and their bitmap
            uint32_t Cw = (uint32_t)((budget - 64) * 8 / (8 * sizeof(WO) + 1));
            Cw &= ~1023u;
            const uint32_t g3 = n3 < (uint32_t)C.num_sms ? n3 : (uint32_t)C.num_sms;
            // a row merges to at most min(its size, nc) entries, and its size is at most kGiant
            const uint32_t scap = nc < kGiant ? nc : kGiant;
            uint32_t *sdst;
            SGPB_TRY(dalloc_t(C, &sdst, (size_t)g3 * scap));
            const size_t csm = dense_smem_bytes<WO>(Cw, 1);
            SGPB_CUDA(cudaFuncSetAttribute(k_dense_chunked<WI, WO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)budget));
            k_dense_chunked<WI, WO><<<g3, kDenseSmemThreads, csm, C.stream>>>(lists + 5 * (size_t)nc, tcount + 5,
                                                                             boff, bdst, bw, tw, dcnt, nc, Cw, sdst,
                                                                             scap);
            C.kernel_launches++;
            SGPB_CUDA(cudaGetLastError());
        }
        // tier 4: rows of more than kGiant entries (the hub aggregates of
        // skewed graphs, millions of entries each) on 64 blocks per row, so
        // that one row does not hold one SM for the whole build
        if (n4) SGPB_TRY(dense_global(lists + 6 * (size_t)nc, n4, 64));
    }
    return SGP_B200_OK;
}

// ---------------------------------------------------------------- driver --
template <typename WI, typename WO>
static int build_impl(Context &C, const Level &F, const WI *w, const uint32_t *vcmap, uint32_t nc,
                      uint32_t *crp, uint32_t **ccol_io, WO **cw_io, uint64_t *m_c, bool alloc_out,
                      uint32_t *wmax = nullptr) {
    const uint32_t n = F.n;
    uint32_t *cnt, *boff, *fill, *dcnt;
    SGPB_TRY(dalloc_t(C, &cnt, (size_t)nc + 1));
    SGPB_TRY(dalloc_t(C, &boff, (size_t)nc + 1));
    SGPB_TRY(dalloc_t(C, &fill, (size_t)nc + 1));
    SGPB_TRY(dalloc_t(C, &dcnt, (size_t)nc + 1));
    SGPB_TRY(dzero(C, cnt, sizeof(uint32_t) * ((size_t)nc + 1)));
    SGPB_TRY(dzero(C, fill, sizeof(uint32_t) * ((size_t)nc + 1)));

    const double avg = n ? (double)F.m / n : 0;
    uint32_t cap = (uint32_t)C.num_sms * 16;
#define SGPB_ROWS_LAUNCH(KERNEL, G, ...)                                                   \
    {                                                                                      \
        uint32_t blocks = cdiv((uint64_t)n * G, 256);                                      \
        if (blocks > cap) blocks = cap;                                                    \
        if (blocks < 1) blocks = 1;                                                        \
        KERNEL<<<blocks, 256, 0, C.stream>>>(__VA_ARGS__);                                 \
    }
#define SGPB_BY_G(KERNEL_T, ...)                                                           \
    if (avg <= 4) SGPB_ROWS_LAUNCH(KERNEL_T(4), 4, __VA_ARGS__)                            \
    else if (avg <= 8) SGPB_ROWS_LAUNCH(KERNEL_T(8), 8, __VA_ARGS__)                       \
    else if (avg <= 16) SGPB_ROWS_LAUNCH(KERNEL_T(16), 16, __VA_ARGS__)                    \
    else SGPB_ROWS_LAUNCH(KERNEL_T(32), 32, __VA_ARGS__)

    uint32_t *krow, *long_list, *long_cnt;
    SGPB_TRY(dalloc_t(C, &krow, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &long_list, F.m / kLongRowT + 1));
    SGPB_TRY(dalloc_t(C, &long_cnt, 1));
    SGPB_TRY(dzero(C, long_cnt, sizeof(uint32_t)));
    uint32_t glong = (uint32_t)(F.m / kLongRowT + 1);
    if (glong > (uint32_t)C.num_sms * 2) glong = C.num_sms * 2;
    // large levels: the count keeps each entry's coarse destination, so the
    // scatter streams it instead of gathering vcmap a second time (the
    // random gathers, not the bytes, bound both passes)
    uint32_t *cvs = nullptr;
    if (F.m >= kStoreCvMin) SGPB_TRY(dalloc_t(C, &cvs, (size_t)F.m + 1));
#define K_COUNT(G) k_build_count<G>
    SGPB_BY_G(K_COUNT, n, F.rp, F.col, vcmap, cnt, krow, long_list, long_cnt, cvs)
    if (F.m > kLongRowT) {
        k_build_count_long<<<glong, kLongThreads, 0, C.stream>>>(F.rp, F.col, vcmap, cnt, krow, long_list, long_cnt,
                                                                 cvs);
        C.kernel_launches++;
    }
    SGPB_TRY(scan_u32(C, cnt, boff, nc, nullptr));
    uint32_t kept = 0;
    SGPB_TRY(read_u32(C, boff + nc, &kept));
    uint32_t *bdst;
    WI *bw = nullptr;
    WO *tw;
    SGPB_TRY(dalloc_t(C, &bdst, (size_t)kept + 1));
    if (w) SGPB_TRY(dalloc_t(C, &bw, (size_t)kept + 1));
    SGPB_TRY(dalloc_t(C, &tw, (size_t)kept + 1));
#define K_SCATTER(G) k_build_scatter<G, WI>
    SGPB_BY_G(K_SCATTER, n, F.rp, F.col, w, vcmap, krow, boff, fill, bdst, bw, cvs)
    if (F.m > kLongRowT) {
        k_build_scatter_long<WI><<<glong, kLongThreads, 0, C.stream>>>(F.rp, F.col, w, vcmap, krow, boff, fill, bdst,
                                                                      bw, long_list, long_cnt, cvs);
        C.kernel_launches++;
    }
#undef K_COUNT
#undef K_SCATTER
#undef SGPB_BY_G
#undef SGPB_ROWS_LAUNCH
    C.kernel_launches += 2;
    SGPB_TRY((dedupe_buckets<WI, WO>(C, nc, boff, bdst, bw, tw, dcnt)));
    SGPB_TRY(scan_u32(C, dcnt, crp, nc, nullptr));
    uint32_t mc = 0;
    SGPB_TRY(read_u32(C, crp + nc, &mc));
    *m_c = mc;
    if (alloc_out) {
        SGPB_TRY(dalloc_t(C, ccol_io, (size_t)mc + 1));
        SGPB_TRY(dalloc_t(C, cw_io, (size_t)mc + 1));
    }
    if (nc) {
        uint32_t g = cdiv(nc, 8);
        if (g > (uint32_t)C.num_sms * 16) g = C.num_sms * 16;
        k_compact_rows<WO><<<g ? g : 1, 256, 0, C.stream>>>(nc, boff, crp, bdst, tw, *ccol_io, *cw_io, wmax);
        C.kernel_launches++;
    }
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}

// -------------------------------------------------------- sorted build --
// Unit-weight fine levels with many entries.  Every entry becomes the key
// (vcmap[u] << b | vcmap[v]) -- all ones for an entry inside an aggregate --
// and one stable LSD radix sort (csrc/sort.cu) orders the keys by coarse row
// and destination.  Each run of equal keys is one coarse entry whose weight is
// the run length: the RADIX build's output (rows sorted by destination,
// duplicates summed, self loops dropped) with no per-row sorts.
constexpr uint64_t kNoKey = ~0ull;

template <int G>
__global__ void __launch_bounds__(256) k_sb_keys(uint32_t n, const uint32_t *__restrict__ rp,
                                                 const uint32_t *__restrict__ col,
                                                 const uint32_t *__restrict__ vcmap, int b,
                                                 unsigned long long *__restrict__ keys,
                                                 unsigned long long *__restrict__ kept,
                                                 uint32_t *__restrict__ long_list, uint32_t *__restrict__ long_cnt) {
    __shared__ unsigned long long wsum[8];
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    unsigned long long c = 0;
    for (uint64_t u = gid; u < n; u += ngroups) {
        const unsigned long long cu = vcmap[u];
        const uint32_t e = rp[u + 1];
        if (e - rp[u] > kLongRowT) {   // group-uniform: k_sb_keys_long
            if (lane == 0) list_long_row(long_list, long_cnt, (uint32_t)u);
            continue;
        }
        // four entries per lane in flight: destinations, then their vcmap gathers
        for (uint32_t j0 = rp[u] + lane; j0 < e; j0 += 4 * G) {
            uint32_t d[4];
#pragma unroll
            for (int q = 0; q < 4; q++) d[q] = j0 + q * G < e ? __ldg(col + j0 + q * G) : 0u;
            uint32_t cv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) cv[q] = j0 + q * G < e ? __ldg(vcmap + d[q]) : 0u;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (j0 + q * G < e) {
                    const bool keep = cv[q] != cu;
                    keys[j0 + q * G] = keep ? (cu << b | cv[q]) : kNoKey;
                    c += keep;
                }
            }
        }
    }
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += wsum[k];
        if (t) atomicAdd(kept, t);
    }
}

// the long rows of k_sb_keys, a block per row
__global__ void __launch_bounds__(kLongThreads) k_sb_keys_long(const uint32_t *__restrict__ rp,
                                                             const uint32_t *__restrict__ col,
                                                             const uint32_t *__restrict__ vcmap, int b,
                                                             unsigned long long *__restrict__ keys,
                                                             unsigned long long *__restrict__ kept,
                                                             const uint32_t *__restrict__ long_list,
                                                             const uint32_t *__restrict__ long_cnt) {
    __shared__ unsigned long long sm[kLongThreads / 32];
    const uint32_t nl = *long_cnt;
    for (uint32_t r = blockIdx.x; r < nl; r += gridDim.x) {
        const uint32_t u = long_list[r];
        const unsigned long long cu = vcmap[u];
        const uint32_t e = rp[u + 1];
        unsigned long long c = 0;
        for (uint32_t j0 = rp[u] + threadIdx.x; j0 < e; j0 += 4 * blockDim.x) {
            uint32_t d[4], cv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) d[q] = j0 + q * blockDim.x < e ? __ldg(col + j0 + q * blockDim.x) : 0u;
#pragma unroll
            for (int q = 0; q < 4; q++) cv[q] = j0 + q * blockDim.x < e ? __ldg(vcmap + d[q]) : 0u;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (j0 + q * blockDim.x < e) {
                    const bool keep = cv[q] != cu;
                    keys[j0 + q * blockDim.x] = keep ? (cu << b | cv[q]) : kNoKey;
                    c += keep;
                }
            }
        }
        c = block_sum_long(c, sm);
        if (threadIdx.x == 0 && c) atomicAdd(kept, c);
    }
}

// flag[i] = 1 where a run of equal (valid) keys starts
__global__ void __launch_bounds__(256) k_sb_heads(uint64_t m, const unsigned long long *__restrict__ s,
                                                  uint32_t *__restrict__ flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = s[i];
        flag[i] = (k != kNoKey && (i == 0 || s[i - 1] != k)) ? 1u : 0u;
    }
}

// heads: destination, run start and the coarse row's entry count (rows are
// sorted, so a warp's heads mostly share rows: one atomic per row per warp)
__global__ void __launch_bounds__(256) k_sb_emit(uint64_t m, const unsigned long long *__restrict__ s,
                                                 const uint32_t *__restrict__ pos, int b,
                                                 uint32_t *__restrict__ ccol, uint32_t *__restrict__ start,
                                                 uint32_t *__restrict__ rcnt) {
    const unsigned long long mask = (1ull << b) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < m; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool head = i < m && pos[i + 1] != pos[i];
        uint32_t row = 0xFFFFFFFFu;
        if (head) {
            const unsigned long long k = s[i];
            const uint32_t p = pos[i];
            ccol[p] = (uint32_t)(k & mask);
            start[p] = (uint32_t)i;
            row = (uint32_t)(k >> b);
        }
        const unsigned act = __ballot_sync(0xFFFFFFFFu, head);
        if (head) {
            const unsigned peers = __match_any_sync(act, row);
            if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(rcnt + row, (uint32_t)__popc(peers));
        }
    }
}

template <typename WO>
__global__ void __launch_bounds__(256) k_sb_weights(uint32_t mc, const uint32_t *__restrict__ start, uint64_t nvalid,
                                                    WO *__restrict__ cw) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < mc; p += gridDim.x * blockDim.x) {
        const uint64_t e = p + 1 < mc ? (uint64_t)start[p + 1] : nvalid;
        cw[p] = (WO)(e - start[p]);
    }
}

// The sorted build runs only when SGPB_BUILD_SORTED=1 asks for it (every
// unit-weight level then takes it): with the radix-sorted bucket tiers the
// tiered build is as fast or faster on every family measured (R-MAT 22's
// coarsening 16.7 ms sorted against 15.9 ms tiered; random geometric, grid,
// Erdos-Renyi and Chung-Lu graphs of 4M vertices the same or better).
static bool sorted_build_wanted(const Level &F) {
    if (F.w || F.m == 0) return false;
    const char *e = getenv("SGPB_BUILD_SORTED");
    return e && *e && atoi(e) != 0;
}

template <typename WO>
static int build_sorted_unit(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, uint32_t *crp,
                             uint32_t **ccol_io, WO **cw_io, uint64_t *m_c, bool alloc_out) {
    const uint32_t n = F.n;
    const uint64_t m = F.m;
    // 2^b > nc: a valid key's low 2b bits are never all ones, so the
    // sentinels sort after every valid key
    int b = 1;
    while (b < 32 && (1ull << b) <= (uint64_t)nc) b++;
    unsigned long long *keys, *tmp, *kept;
    uint32_t *flag, *pos, *rcnt;
    SGPB_TRY(dalloc_t(C, &keys, m));
    SGPB_TRY(dalloc_t(C, &tmp, m));
    SGPB_TRY(dalloc_t(C, &kept, 1));
    SGPB_TRY(dalloc_t(C, &flag, m + 1));
    SGPB_TRY(dalloc_t(C, &pos, m + 1));
    SGPB_TRY(dalloc_t(C, &rcnt, (size_t)nc + 1));
    SGPB_TRY(dzero(C, kept, 8));
    SGPB_TRY(dzero(C, rcnt, sizeof(uint32_t) * ((size_t)nc + 1)));
    const double avg = n ? (double)m / n : 0;
    const uint32_t cap = (uint32_t)C.num_sms * 16;
    auto rows_grid = [&](int G) {
        uint32_t g = cdiv((uint64_t)n * G, 256);
        return g > cap ? cap : (g ? g : 1u);
    };
    uint32_t *long_list, *long_cnt;
    SGPB_TRY(dalloc_t(C, &long_list, F.m / kLongRowT + 1));
    SGPB_TRY(dalloc_t(C, &long_cnt, 1));
    SGPB_TRY(dzero(C, long_cnt, sizeof(uint32_t)));
    if (avg <= 4)
        k_sb_keys<4><<<rows_grid(4), 256, 0, C.stream>>>(n, F.rp, F.col, vcmap, b, keys, kept, long_list, long_cnt);
    else if (avg <= 16)
        k_sb_keys<16><<<rows_grid(16), 256, 0, C.stream>>>(n, F.rp, F.col, vcmap, b, keys, kept, long_list, long_cnt);
    else
        k_sb_keys<32><<<rows_grid(32), 256, 0, C.stream>>>(n, F.rp, F.col, vcmap, b, keys, kept, long_list, long_cnt);
    C.kernel_launches++;
    if (F.m > kLongRowT) {
        uint32_t gl = (uint32_t)(F.m / kLongRowT + 1);
        if (gl > (uint32_t)C.num_sms * 2) gl = C.num_sms * 2;
        k_sb_keys_long<<<gl, kLongThreads, 0, C.stream>>>(F.rp, F.col, vcmap, b, keys, kept, long_list, long_cnt);
        C.kernel_launches++;
    }
    bool in_tmp = false;
    SGPB_TRY(radix_sort_keys(C, keys, m, 2 * b, tmp, &in_tmp));
    const unsigned long long *sk = in_tmp ? tmp : keys;
    const uint32_t eg = (uint32_t)(cdiv(m, 256) > cap ? cap : cdiv(m, 256));
    k_sb_heads<<<eg, 256, 0, C.stream>>>(m, sk, flag);
    C.kernel_launches++;
    SGPB_TRY(scan_u32(C, flag, pos, (uint32_t)m, nullptr));
    uint32_t mc = 0;
    uint64_t nvalid = 0;
    SGPB_TRY(read_u32(C, pos + m, &mc));
    SGPB_TRY(read_u64(C, (const uint64_t *)kept, &nvalid));
    *m_c = mc;
    if (alloc_out) {
        SGPB_TRY(dalloc_t(C, ccol_io, (size_t)mc + 1));
        SGPB_TRY(dalloc_t(C, cw_io, (size_t)mc + 1));
    }
    uint32_t *start;
    SGPB_TRY(dalloc_t(C, &start, (size_t)mc + 1));
    k_sb_emit<<<eg, 256, 0, C.stream>>>(m, sk, pos, b, *ccol_io, start, rcnt);
    C.kernel_launches++;
    SGPB_TRY(scan_u32(C, rcnt, crp, nc, nullptr));
    if (mc) {
        const uint32_t wg = (uint32_t)(cdiv(mc, 256) > cap ? cap : cdiv(mc, 256));
        k_sb_weights<WO><<<wg, 256, 0, C.stream>>>(mc, start, nvalid, *cw_io);
        C.kernel_launches++;
    }
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}

// Builds level `out` (allocating its arrays from the context) from F + vcmap.
// c_vtx_w[vcmap[u]] += vtx_w[u] over the fine vertices u (unit weights when
// fw is null); integer atomics, so the sums do not depend on their order
__global__ void k_vertex_weights(uint32_t n, const uint32_t *__restrict__ vcmap, const uint32_t *__restrict__ fw,
                                 uint32_t *cw) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&cw[vcmap[i]], fw ? fw[i] : 1u);
}

int coarse_vertex_weights(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, uint32_t **out) {
    uint32_t *cw;
    SGPB_TRY(dalloc_t(C, &cw, (size_t)nc + 1));
    SGPB_TRY(dzero(C, cw, sizeof(uint32_t) * ((size_t)nc + 1)));
    uint32_t blocks = cdiv(F.n, 256);
    if (blocks > (uint32_t)C.num_sms * 8) blocks = C.num_sms * 8;
    if (F.n) k_vertex_weights<<<blocks, 256, 0, C.stream>>>(F.n, vcmap, F.vtx_w, cw);
    C.kernel_launches++;
    SGPB_CUDA(cudaGetLastError());
    *out = cw;
    return SGP_B200_OK;
}

int build_coarse_level(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, int out_wbytes,
                       Level *out) {
    uint32_t *crp;
    SGPB_TRY(dalloc_t(C, &crp, (size_t)nc + 1));
    uint32_t *ccol = nullptr;
    uint64_t mc = 0;
    out->n = nc;
    out->rp = crp;
    out->wbytes = out_wbytes;
    out->sorted = 1;
    if (F.wbytes == 8 && out_wbytes != 8) {
        set_error("coarse weights must be at least as wide as fine weights");
        return SGP_B200_ERR_INVALID;
    }
    if (sorted_build_wanted(F)) {
        if (out_wbytes == 8) {
            unsigned long long *cw = nullptr;
            SGPB_TRY((build_sorted_unit<unsigned long long>(C, F, vcmap, nc, crp, &ccol, &cw, &mc, true)));
            out->w = cw;
        } else {
            uint32_t *cw = nullptr;
            SGPB_TRY((build_sorted_unit<uint32_t>(C, F, vcmap, nc, crp, &ccol, &cw, &mc, true)));
            out->w = cw;
        }
        out->col = ccol;
        out->m = mc;
        return SGP_B200_OK;
    }
    if (out_wbytes == 8) {
        unsigned long long *cw = nullptr;
        if (F.wbytes == 8)
            SGPB_TRY((build_impl<unsigned long long, unsigned long long>(C, F, (const unsigned long long *)F.w, vcmap, nc,
                                                                         crp, &ccol, &cw, &mc, true)));
        else
            SGPB_TRY((build_impl<uint32_t, unsigned long long>(C, F, (const uint32_t *)F.w, vcmap, nc, crp, &ccol, &cw,
                                                               &mc, true)));
        out->w = cw;
    } else {
        uint32_t *cw = nullptr, *wmax = nullptr;
        SGPB_TRY(dalloc_t(C, &wmax, 1));
        SGPB_TRY(dzero(C, wmax, sizeof(uint32_t)));
        SGPB_TRY((build_impl<uint32_t, uint32_t>(C, F, (const uint32_t *)F.w, vcmap, nc, crp, &ccol, &cw, &mc, true,
                                                 wmax)));
        out->w = cw;
        out->wmax = wmax;
    }
    out->col = ccol;
    out->m = mc;
    return SGP_B200_OK;
}

// Variant writing into caller buffers (the C-ABI test entry point).
int build_coarse_into(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, int out_wbytes,
                      uint32_t *crp, uint32_t *ccol, void *cw, uint64_t *m_c) {
    if (F.wbytes == 8 && out_wbytes != 8) {
        set_error("coarse weights must be at least as wide as fine weights");
        return SGP_B200_ERR_INVALID;
    }
    if (sorted_build_wanted(F)) {
        if (out_wbytes == 8) {
            unsigned long long *w8 = (unsigned long long *)cw;
            return build_sorted_unit<unsigned long long>(C, F, vcmap, nc, crp, &ccol, &w8, m_c, false);
        }
        uint32_t *w4 = (uint32_t *)cw;
        return build_sorted_unit<uint32_t>(C, F, vcmap, nc, crp, &ccol, &w4, m_c, false);
    }
    if (out_wbytes == 8) {
        unsigned long long *w8 = (unsigned long long *)cw;
        if (F.wbytes == 8)
            return build_impl<unsigned long long, unsigned long long>(C, F, (const unsigned long long *)F.w, vcmap, nc,
                                                                      crp, &ccol, &w8, m_c, false);
        return build_impl<uint32_t, unsigned long long>(C, F, (const uint32_t *)F.w, vcmap, nc, crp, &ccol, &w8, m_c,
                                                        false);
    }
    uint32_t *w4 = (uint32_t *)cw;
    return build_impl<uint32_t, uint32_t>(C, F, (const uint32_t *)F.w, vcmap, nc, crp, &ccol, &w4, m_c, false);
}

}  // namespace sgpb
