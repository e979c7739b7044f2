// sort.cu -- stable LSD radix sort of 64-bit keys with an optional payload.
//
// Used where a whole edge list must be grouped by row and ordered by column:
// the keys are (row << b | column) packed into the fewest bits, so a sort by
// the low 2b bits puts every row's entries together in column order.
//
// Each 8-bit pass is two kernels and a scan:
//   k_rs_hist     per tile of kRsTile keys, the digit counts, written
//                 digit-major (hist[d * ntiles + t]) so one exclusive scan
//                 gives every (digit, tile) its output offset;
//   k_rs_scatter  the same tile again: each warp ranks its 32-key rounds in
//                 order with __match_any_sync against per-warp digit counters
//                 in shared memory, a block prefix over the warps turns that
//                 into the rank inside the tile, the tile is staged in digit
//                 order in shared memory, and consecutive threads then write
//                 consecutive keys of a digit to its (digit, tile) range, so
//                 the stores coalesce.  Keys keep their input order within a
//                 digit, so the sort is stable and LSD passes compose.
#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kRsWarps = 16;
constexpr int kRsThreads = kRsWarps * 32;
constexpr int kRsRounds = 8;                              // 32-key rounds per warp
constexpr uint32_t kRsTile = kRsWarps * 32 * kRsRounds;   // 4096 keys per block
constexpr int kRsBins = 256;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned long long *__restrict__ keys, uint64_t n,
                                                        int shift, uint32_t ntiles, uint32_t *__restrict__ hist) {
    __shared__ uint32_t cnt[kRsBins];
    for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * kRsTile;
    for (uint32_t k = threadIdx.x; k < kRsTile; k += blockDim.x) {
        const uint64_t i = t0 + k;
        if (i < n) atomicAdd(&cnt[(uint32_t)(__ldg(keys + i) >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kRsBins; b += blockDim.x) hist[(size_t)b * ntiles + blockIdx.x] = cnt[b];
}

// three blocks per SM (40 registers, a few spilled): more warps in flight for
// the per-warp ranking chains beat spill-free code at two blocks (rows phase of
// the converter 11.9 -> 10.3 ms on R-MAT 22)
template <typename V>
__global__ void __launch_bounds__(kRsThreads, 3) k_rs_scatter(const unsigned long long *__restrict__ keys,
                                                           const V *__restrict__ vals, uint64_t n, int shift,
                                                           uint32_t ntiles, const uint32_t *__restrict__ off,
                                                           unsigned long long *__restrict__ keys_out,
                                                           V *__restrict__ vals_out) {
    // per-warp digit counts, then exclusive prefixes over the warps
    __shared__ uint32_t wcnt[kRsWarps][kRsBins];
    __shared__ uint32_t dstart[kRsBins];   // first slot of each digit in the tile
    __shared__ uint32_t doff[kRsBins];     // the digit's output offset for this tile
    __shared__ uint64_t scan_sm[33];
    extern __shared__ __align__(16) unsigned char rs_smem[];
    unsigned long long *sk = reinterpret_cast<unsigned long long *>(rs_smem);   // kRsTile keys in digit order
    V *sv = reinterpret_cast<V *>(rs_smem + kRsTile * sizeof(unsigned long long));
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int b = lane; b < kRsBins; b += 32) wcnt[wid][b] = 0;
    if (threadIdx.x < kRsBins) doff[threadIdx.x] = off[(size_t)threadIdx.x * ntiles + blockIdx.x];
    __syncwarp();
    const uint64_t tile0 = (uint64_t)blockIdx.x * kRsTile;
    const uint64_t base = tile0 + (uint64_t)wid * 32 * kRsRounds;
    unsigned long long k[kRsRounds];
    uint32_t rank[kRsRounds];
    V v[kRsRounds];
#pragma unroll
    for (int r = 0; r < kRsRounds; r++) {
        const uint64_t i = base + (uint64_t)r * 32 + lane;
        const bool valid = i < n;
        k[r] = valid ? __ldg(keys + i) : 0ull;
        if (vals) v[r] = valid ? __ldg(vals + i) : (V)0;
        const uint32_t d = (uint32_t)(k[r] >> shift) & 0xFF;
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
    // per digit: prefixes over the warps and the digit's total in the tile
    uint32_t total = 0;
    if (threadIdx.x < kRsBins) {
        const int d = threadIdx.x;
#pragma unroll
        for (int w = 0; w < kRsWarps; w++) {
            const uint32_t c = wcnt[w][d];
            wcnt[w][d] = total;
            total += c;
        }
    }
    // digit starts inside the tile: an exclusive scan of the totals
    uint64_t all;
    const uint64_t incl = block_scan_u64(threadIdx.x < kRsBins ? total : 0, scan_sm, &all);
    if (threadIdx.x < kRsBins) dstart[threadIdx.x] = (uint32_t)(incl - total);
    __syncthreads();
    // stage the tile in digit order
#pragma unroll
    for (int r = 0; r < kRsRounds; r++) {
        const uint64_t i = base + (uint64_t)r * 32 + lane;
        if (i >= n) continue;
        const uint32_t d = (uint32_t)(k[r] >> shift) & 0xFF;
        const uint32_t slot = dstart[d] + wcnt[wid][d] + rank[r];
        sk[slot] = k[r];
        if (vals) sv[slot] = v[r];
    }
    __syncthreads();
    // stream it out: consecutive slots of one digit go to consecutive addresses
    const uint32_t len = n - tile0 < kRsTile ? (uint32_t)(n - tile0) : kRsTile;
    for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) {
        const unsigned long long key = sk[j];
        const uint32_t d = (uint32_t)(key >> shift) & 0xFF;
        const uint64_t pos = (uint64_t)doff[d] + (j - dstart[d]);
        keys_out[pos] = key;
        if (vals) vals_out[pos] = sv[j];
    }
}

// Sorts keys[0, n) (and vals alongside, when given) by their low `bits`
// bits.  tmp buffers of n entries are used alternately; *in_tmp reports
// whether the sorted data ended in the tmp buffers.  n < 2^32.
template <typename V>
static int radix_sort_impl(Context &C, unsigned long long *keys, V *vals, uint64_t n, int bits,
                           unsigned long long *keys_tmp, V *vals_tmp, bool *in_tmp) {
    *in_tmp = false;
    if (n <= 1 || bits <= 0) return SGP_B200_OK;
    if (n >= 0xFFFFFFFFull) {
        set_error("radix sort of %llu keys: more than 2^32 - 1", (unsigned long long)n);
        return SGP_B200_ERR_TOO_LARGE;
    }
    const uint32_t ntiles = cdiv(n, kRsTile);
    uint32_t *hist, *off;
    SGPB_TRY(dalloc_t(C, &hist, (size_t)kRsBins * ntiles + 1));
    SGPB_TRY(dalloc_t(C, &off, (size_t)kRsBins * ntiles + 1));
    // the staged tile: keys, then payloads; the limit is the same bound for
    // every launch (host threads share the function attribute)
    const size_t smem = (size_t)kRsTile * (sizeof(unsigned long long) + sizeof(unsigned long long));
    SGPB_CUDA(cudaFuncSetAttribute(k_rs_scatter<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    unsigned long long *ks = keys, *kd = keys_tmp;
    V *vs = vals, *vd = vals_tmp;
    for (int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<ntiles, kRsThreads, 0, C.stream>>>(ks, n, shift, ntiles, hist);
        SGPB_TRY(scan_u32(C, hist, off, kRsBins * ntiles, nullptr));
        k_rs_scatter<V><<<ntiles, kRsThreads, vals ? smem : (size_t)kRsTile * sizeof(unsigned long long),
                          C.stream>>>(ks, vs, n, shift, ntiles, off, kd, vd);
        C.kernel_launches += 2;
        std::swap(ks, kd);
        std::swap(vs, vd);
        *in_tmp = !*in_tmp;
    }
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}

int radix_sort_keys(Context &C, unsigned long long *keys, uint64_t n, int bits, unsigned long long *keys_tmp,
                    bool *in_tmp) {
    return radix_sort_impl<uint32_t>(C, keys, nullptr, n, bits, keys_tmp, nullptr, in_tmp);
}
int radix_sort_pairs_u32(Context &C, unsigned long long *keys, uint32_t *vals, uint64_t n, int bits,
                         unsigned long long *keys_tmp, uint32_t *vals_tmp, bool *in_tmp) {
    return radix_sort_impl<uint32_t>(C, keys, vals, n, bits, keys_tmp, vals_tmp, in_tmp);
}
int radix_sort_pairs_u64(Context &C, unsigned long long *keys, unsigned long long *vals, uint64_t n, int bits,
                         unsigned long long *keys_tmp, unsigned long long *vals_tmp, bool *in_tmp) {
    return radix_sort_impl<unsigned long long>(C, keys, vals, n, bits, keys_tmp, vals_tmp, in_tmp);
}

}  // namespace sgpb
