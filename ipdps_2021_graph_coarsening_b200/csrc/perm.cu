// perm.cu -- hub-first relabelled copy of a level for the power iteration.
//
// Column references of power-law levels concentrate on few vertices (on the
// first coarse level of an R-MAT scale-20 graph the 16k most referenced
// vertices carry ~3/4 of all entries, ~1/2 at scale 22).  The power iteration
// of such a level runs on a copy P A P^T whose vertices are ordered by
// descending floor(log2(degree)), stable in the original order, so the most
// gathered iterate entries form a dense prefix: the kernel gathers it with L1
// evict-last priority and every other entry without L1 allocation, and L1
// keeps the hub lines.  Each row keeps its entries in their original order.
// The hierarchy itself is not
// relabelled; only the eigen-solve sees the copy, and it maps its start
// vector in and its result out through the permutation.
#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kBuckets = 33;       // floor(log2(deg)) + 1 for deg >= 1, 0 for deg == 0
constexpr int kPermTile = 1024;    // rows per block of the stable scatter

__device__ __forceinline__ uint32_t deg_key(uint32_t deg) {
    // key 0 = highest degree class; ascending key = descending degree
    const uint32_t b = deg ? 32u - __clz(deg) : 0u;   // 1..32, 0 for empty
    return (uint32_t)(kBuckets - 1) - b;
}

__global__ void k_bucket_count(uint32_t n, const uint32_t *rp, uint32_t nb, uint32_t *cnt) {
    __shared__ uint32_t c[kBuckets];
    for (int k = threadIdx.x; k < kBuckets; k += blockDim.x) c[k] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * kPermTile;
    for (uint64_t i = t0 + threadIdx.x; i < t0 + kPermTile && i < n; i += blockDim.x)
        atomicAdd(&c[deg_key(rp[i + 1] - rp[i])], 1u);
    __syncthreads();
    for (int k = threadIdx.x; k < kBuckets; k += blockDim.x) cnt[(size_t)k * nb + blockIdx.x] = c[k];
}

// A block per tile of kPermTile rows, 256 rows at a time: each warp ranks its
// rows within their degree class with __match_any_sync, a prefix over the
// warps per class (and the class's running position in the tile) gives the
// new ids.  Rows keep their order inside a class: stable, deterministic.
constexpr int kPermThreads = 256;

__global__ void __launch_bounds__(kPermThreads) k_bucket_scatter(uint32_t n, const uint32_t *rp, uint32_t nb,
                                                                 const uint32_t *off, uint32_t *perm, uint32_t *inv) {
    constexpr int kWarps = kPermThreads / 32;
    __shared__ uint32_t pos[kBuckets];
    __shared__ uint32_t wc[kWarps][kBuckets];
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x < kBuckets) pos[threadIdx.x] = off[(size_t)threadIdx.x * nb + blockIdx.x];
    const uint64_t t0 = (uint64_t)blockIdx.x * kPermTile;
    for (uint32_t c0 = 0; c0 < (uint32_t)kPermTile; c0 += kPermThreads) {
        for (int k = threadIdx.x; k < kWarps * kBuckets; k += kPermThreads) (&wc[0][0])[k] = 0;
        __syncthreads();
        const uint64_t i = t0 + c0 + threadIdx.x;
        const bool valid = i < n;
        const uint32_t k = valid ? deg_key(rp[i + 1] - rp[i]) : 0u;
        const unsigned act = __ballot_sync(0xFFFFFFFFu, valid);
        uint32_t rank = 0;
        if (valid) {
            const unsigned peers = __match_any_sync(act, k);
            rank = __popc(peers & ((1u << lane) - 1u));
            if ((int)lane == __ffs(peers) - 1) wc[wid][k] = __popc(peers);
        }
        __syncthreads();
        if (threadIdx.x < kBuckets) {
            uint32_t t = pos[threadIdx.x];
            for (int w = 0; w < kWarps; w++) {
                const uint32_t c = wc[w][threadIdx.x];
                wc[w][threadIdx.x] = t;
                t += c;
            }
            pos[threadIdx.x] = t;
        }
        __syncthreads();
        if (valid) {
            const uint32_t p = wc[wid][k] + rank;
            perm[i] = p;
            inv[p] = (uint32_t)i;
        }
        __syncthreads();
    }
}

__global__ void k_perm_degrees(uint32_t n, const uint32_t *rp, const uint32_t *inv, uint32_t *deg) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint32_t o = inv[i];
        deg[i] = rp[o + 1] - rp[o];
    }
}

template <typename WI, typename WO>
__global__ void __launch_bounds__(256) k_perm_fill(uint32_t n, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ col, const WI *__restrict__ w,
                                                  const uint32_t *__restrict__ perm, const uint32_t *__restrict__ inv,
                                                  const uint32_t *__restrict__ nrp, uint32_t *__restrict__ ncol,
                                                  WO *__restrict__ nw) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = wid; i < n; i += nwarps) {
        const uint32_t o = inv[i];
        const uint32_t b = rp[o], e = rp[o + 1], d = nrp[i];
        // eight entries per lane in flight: destinations, their new ids, stores
        for (uint32_t j0 = b + lane; j0 < e; j0 += 256) {
            uint32_t c[8];
            WI x[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t j = j0 + 32 * k;
                c[k] = j < e ? col[j] : 0u;
                if (w) x[k] = j < e ? w[j] : (WI)0;
            }
#pragma unroll
            for (int k = 0; k < 8; k++) c[k] = j0 + 32 * k < e ? perm[c[k]] : 0u;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t j = j0 + 32 * k;
                if (j < e) {
                    ncol[d + (j - b)] = c[k];
                    if (w) nw[d + (j - b)] = (WO)x[k];
                }
            }
        }
    }
}

// the copy's weights are WO (as wide as the input, or narrower when every
// weight fits); the padding lets vector loads run past the last entry
template <typename WI, typename WO>
static int fill_impl(Context &C, const Level &L, const uint32_t *perm, const uint32_t *inv, Level *out) {
    WO *nw = nullptr;
    if (L.w) SGPB_TRY(dalloc_t(C, &nw, (size_t)L.m + kStagePad));
    uint32_t blocks = cdiv((uint64_t)L.n * 32, 256);
    if (blocks > (uint32_t)C.num_sms * 16) blocks = C.num_sms * 16;
    k_perm_fill<WI, WO><<<blocks ? blocks : 1, 256, 0, C.stream>>>(L.n, L.rp, L.col, (const WI *)L.w, perm, inv,
                                                                  out->rp, out->col, nw);
    C.kernel_launches++;
    out->w = nw;
    out->wbytes = L.w ? (int)sizeof(WO) : 0;
    return SGP_B200_OK;
}

__global__ void k_max_u32(uint64_t m, const uint32_t *w, uint32_t *out) {
    uint32_t mx = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        mx = w[i] > mx ? w[i] : mx;
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(out, mx);
}

int hub_first_copy(Context &C, const Level &L, uint32_t **perm_out, uint32_t **inv_out, Level *out) {
    const uint32_t n = L.n;
    const uint32_t nb = cdiv(n, kPermTile);
    uint32_t *cnt, *off, *perm, *inv, *deg;
    SGPB_TRY(dalloc_t(C, &cnt, (size_t)nb * kBuckets + 1));
    SGPB_TRY(dalloc_t(C, &off, (size_t)nb * kBuckets + 1));
    SGPB_TRY(dalloc_t(C, &perm, n));
    SGPB_TRY(dalloc_t(C, &inv, n));
    SGPB_TRY(dalloc_t(C, &deg, (size_t)n + 1));
    k_bucket_count<<<nb, 256, 0, C.stream>>>(n, L.rp, nb, cnt);
    SGPB_TRY(scan_u32(C, cnt, off, nb * kBuckets, nullptr));
    k_bucket_scatter<<<nb, kPermThreads, 0, C.stream>>>(n, L.rp, nb, off, perm, inv);
    k_perm_degrees<<<cdiv(n, 256), 256, 0, C.stream>>>(n, L.rp, inv, deg);
    C.kernel_launches += 3;
    *out = L;
    out->vcmap = nullptr;
    SGPB_TRY(dalloc_t(C, &out->rp, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &out->col, (size_t)L.m + kStagePad));
    SGPB_TRY(scan_u32(C, deg, out->rp, n, nullptr));
    if (L.wbytes == 8) {
        SGPB_TRY((fill_impl<unsigned long long, unsigned long long>(C, L, perm, inv, out)));
    } else if (L.w) {
        // 32-bit weights that all fit 8 or 16 bits are stored narrow: the
        // power iteration streams them every iteration
        // (the tiered build records the maximum; other levels are scanned)
        uint32_t *mx = L.wmax, hmx = 0;
        if (!mx) {
            SGPB_TRY(dalloc_t(C, &mx, 1));
            SGPB_TRY(dzero(C, mx, 4));
            uint32_t g = (uint32_t)cdiv(L.m, 256);
            if (g > (uint32_t)C.num_sms * 8) g = C.num_sms * 8;
            k_max_u32<<<g ? g : 1, 256, 0, C.stream>>>(L.m, (const uint32_t *)L.w, mx);
            C.kernel_launches++;
        }
        SGPB_TRY(read_u32(C, mx, &hmx));
        if (hmx <= 0xFFu) SGPB_TRY((fill_impl<uint32_t, uint8_t>(C, L, perm, inv, out)));
        else if (hmx <= 0xFFFFu) SGPB_TRY((fill_impl<uint32_t, uint16_t>(C, L, perm, inv, out)));
        else SGPB_TRY((fill_impl<uint32_t, uint32_t>(C, L, perm, inv, out)));
    } else {
        SGPB_TRY((fill_impl<uint32_t, uint32_t>(C, L, perm, inv, out)));
    }
    SGPB_CUDA(cudaGetLastError());
    *perm_out = perm;
    *inv_out = inv;
    return SGP_B200_OK;
}

}  // namespace sgpb
