// common.cuh -- shared device helpers for the sm_100a spectral-bisection path.
#pragma once
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <stdint.h>

namespace cg = cooperative_groups;

namespace sgpb {

constexpr uint32_t kUnassigned = 0xFFFFFFFFu;
constexpr int kWarp = 32;

// ------------------------------------------------------------- hashing --
// Counter-based hashes of (level seed, vertex).  They replace the reference's
// time-seeded XorShift pool (cmg/heuristics.h:614-631, :947) so that the HEC
// mapping is reproducible; the CPU oracle uses the same three formulas.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// 63-bit priority key: 31 hash bits above the vertex id (a strict total order)
__host__ __device__ __forceinline__ uint64_t prio_key(uint64_t seed, uint32_t u) {
    uint64_t h = mix64(seed ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)u + 1)));
    return ((h >> 33) << 32) | (uint64_t)u;
}
__host__ __device__ __forceinline__ uint64_t rand_draw(uint64_t seed, uint32_t u) {
    return mix64(seed ^ 0x632BE59BD9B4E019ULL ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)u + 1)));
}
__host__ __device__ __forceinline__ uint32_t tiebreak(uint64_t seed, uint32_t u, uint32_t v) {
    return (uint32_t)(mix64(seed ^ 0xD1B54A32D192ED03ULL ^ (((uint64_t)u << 32) | v)) >> 32);
}

// ----------------------------------------------------------- reductions --
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { T x = __shfl_xor_sync(0xFFFFFFFFu, v, o); v = x > v ? x : v; }
    return v;
}
// mask of this lane's aligned group of G lanes (G power of two <= 32): the
// lanes that a group-level shuffle may name, so groups of one warp can leave
// a row loop after different numbers of rows
template <int G>
__device__ __forceinline__ unsigned group_mask() {
    if constexpr (G == 32) {
        return 0xFFFFFFFFu;
    } else {
        const unsigned lane = threadIdx.x & 31;
        return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
    }
}
// sum over aligned groups of G lanes; result in all lanes of the group
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
    const unsigned gm = group_mask<G>();
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o);
    return v;
}

// Deterministic block-wide sum of NV doubles: fixed shuffle tree per warp, then
// warp 0 combines the warp totals in index order.  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum_d(double (&v)[NV], double *smem /* >= NV*32 */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) smem[k * 32 + wid] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = lane < nw ? smem[k * 32 + lane] : 0.0;
            v[k] = warp_sum(x);
        }
    }
    __syncthreads();
}

// Inclusive prefix sum within a block of uint64 values (one per thread).
// Returns the inclusive prefix; *total receives the block total.
__device__ __forceinline__ uint64_t block_scan_u64(uint64_t x, uint64_t *smem /* >= 33 */, uint64_t *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    uint64_t s = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
        if (lane >= o) s += y;
    }
    __syncthreads();
    if (lane == 31) smem[wid] = s;
    __syncthreads();
    if (wid == 0) {
        uint64_t t = lane < nw ? smem[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) smem[lane] = t;
    }
    __syncthreads();
    uint64_t base = wid > 0 ? smem[wid - 1] : 0;
    *total = smem[nw - 1];
    __syncthreads();
    return s + base;
}

// weight load: a null pointer means unit weights
template <typename W>
__device__ __forceinline__ uint64_t wload(const W *w, uint32_t e) {
    return w ? (uint64_t)__ldg(w + e) : 1ull;
}

}  // namespace sgpb
