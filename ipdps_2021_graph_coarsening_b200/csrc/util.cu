// util.cu -- context, stream-ordered allocation, device scan and compaction.
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include "common.cuh"
#include "internal.h"

struct sgp_b200_ctx {
    sgpb::Context c;
};

namespace sgpb {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char *last_error() { return g_err; }

Context *ctx_get(sgp_b200_ctx_t *c) { return c ? &c->c : nullptr; }

int dalloc(Context &C, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(p, bytes, C.stream);
    if (e != cudaSuccess) {
        set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return SGP_B200_ERR_DEVICE;
    }
    C.owned.push_back(*p);
    return SGP_B200_OK;
}

uint32_t round_budget(uint64_t natural) {
    uint64_t cap = natural < 0xFFFFFFF0ull ? natural : 0xFFFFFFF0ull;
    if (const char *e = getenv("SGPB_ROUND_CAP")) {
        const unsigned long long t = strtoull(e, nullptr, 10);
        if (t > 0 && t < cap) cap = t;
    }
    return (uint32_t)cap;
}

int dzero(Context &C, void *p, size_t bytes) {
    SGPB_CUDA(cudaMemsetAsync(p, 0, bytes, C.stream));
    return SGP_B200_OK;
}

void release_all(Context &C) {
    for (void *p : C.owned) cudaFreeAsync(p, C.stream);
    C.owned.clear();
}

int read_u32(Context &C, const uint32_t *d, uint32_t *h, int count) {
    SGPB_CUDA(cudaMemcpyAsync(C.h_pinned, d, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    memcpy(h, C.h_pinned, sizeof(uint32_t) * count);
    return SGP_B200_OK;
}
int read_u64(Context &C, const uint64_t *d, uint64_t *h, int count) {
    SGPB_CUDA(cudaMemcpyAsync(C.h_pinned, d, sizeof(uint64_t) * count, cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    memcpy(h, C.h_pinned, sizeof(uint64_t) * count);
    return SGP_B200_OK;
}

// ------------------------------------------------------------------ scan --
// Three-kernel exclusive scan: tile sums, one-block scan of the tile sums,
// tile scan with the tile base added.  Tiles are kScanThreads * kScanItems.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const uint32_t *in, uint32_t n, uint64_t *tile_sum) {
    __shared__ uint64_t sm[33];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        uint64_t i = base + (uint64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint64_t tot;
    block_scan_u64(s, sm, &tot);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

// single block: exclusive scan of tile sums in place; writes total
__global__ void __launch_bounds__(1024) k_scan_tiles(uint64_t *tile_sum, uint32_t ntiles, uint32_t *out_total,
                                                     uint32_t *overflow) {
    __shared__ uint64_t sm[33];
    uint64_t carry = 0;
    for (uint32_t b = 0; b < ntiles; b += blockDim.x) {
        uint32_t i = b + threadIdx.x;
        uint64_t x = i < ntiles ? tile_sum[i] : 0;
        uint64_t tot;
        uint64_t inc = block_scan_u64(x, sm, &tot);
        if (i < ntiles) tile_sum[i] = carry + inc - x;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        if (carry > 0xFFFFFFFFull) {
            if (overflow) *overflow = 1;
            *out_total = 0xFFFFFFFFu;
        } else {
            *out_total = (uint32_t)carry;
        }
    }
}

__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const uint32_t *in, uint32_t n, const uint64_t *tile_base,
                                                            uint32_t *out) {
    __shared__ uint64_t sm[33];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    // each thread owns kScanItems consecutive items
    uint32_t v[kScanItems];
    uint64_t s = 0;
    uint64_t i0 = base + (uint64_t)threadIdx.x * kScanItems;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        uint64_t i = i0 + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    uint64_t tot;
    uint64_t inc = block_scan_u64(s, sm, &tot);
    uint64_t run = tile_base[blockIdx.x] + inc - s;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        uint64_t i = i0 + k;
        if (i < n) out[i] = (uint32_t)run;
        run += v[k];
    }
}

int scan_u32(Context &C, const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *d_overflow) {
    uint32_t ntiles = n ? cdiv(n, kScanTile) : 1;
    uint64_t *tile = nullptr;
    SGPB_TRY(dalloc_t(C, &tile, ntiles));
    if (n == 0) {
        SGPB_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), C.stream));
        return SGP_B200_OK;
    }
    k_tile_sums<<<ntiles, kScanThreads, 0, C.stream>>>(in, n, tile);
    k_scan_tiles<<<1, 1024, 0, C.stream>>>(tile, ntiles, out + n, d_overflow);
    k_tile_scan<<<ntiles, kScanThreads, 0, C.stream>>>(in, n, tile, out);
    C.kernel_launches += 3;
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}

// --------------------------------------------------------- compaction --
__global__ void k_flags_to_u32(const uint8_t *f, uint32_t n, uint32_t *o) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = f[i] ? 1u : 0u;
}
__global__ void k_scatter_flags(const uint8_t *f, uint32_t n, const uint32_t *pos, uint32_t *out_idx) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && f[i]) out_idx[pos[i]] = i;
}

int compact_flags(Context &C, const uint8_t *flags, uint32_t n, uint32_t *out_idx, uint32_t *d_count) {
    uint32_t *f32 = nullptr, *pos = nullptr;
    SGPB_TRY(dalloc_t(C, &f32, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &pos, (size_t)n + 1));
    if (n) k_flags_to_u32<<<cdiv(n, 256), 256, 0, C.stream>>>(flags, n, f32);
    SGPB_TRY(scan_u32(C, f32, pos, n, nullptr));
    if (n) k_scatter_flags<<<cdiv(n, 256), 256, 0, C.stream>>>(flags, n, pos, out_idx);
    SGPB_CUDA(cudaMemcpyAsync(d_count, pos + n, sizeof(uint32_t), cudaMemcpyDeviceToDevice, C.stream));
    C.kernel_launches += 2;
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}

}  // namespace sgpb

using namespace sgpb;

extern "C" {

sgp_b200_ctx_t *sgp_b200_create(int device) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error("no CUDA device available (%s)", e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
        return nullptr;
    }
    if (device < 0 || device >= ndev) {
        set_error("device %d out of range (0..%d)", device, ndev - 1);
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        set_error("cudaSetDevice(%d) failed", device);
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        set_error("cudaGetDeviceProperties failed");
        return nullptr;
    }
    if (prop.major < 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return nullptr;
    }
    sgp_b200_ctx_t *x = new sgp_b200_ctx_t();
    Context &C = x->c;
    C.device = device;
    C.num_sms = prop.multiProcessorCount;
    C.smem_optin = prop.sharedMemPerBlockOptin;
    {
        char key[160];
        snprintf(key, sizeof(key), "%s|sm%d%d|%dSMs", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
        for (char *c = key; *c; c++)
            if (*c == ' ') *c = '_';
        C.dev_key = key;
    }
    if (cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void **)&C.h_pinned, 4096) != cudaSuccess) {
        set_error("stream / pinned buffer creation failed");
        delete x;
        return nullptr;
    }
    // keep freed pool memory cached across calls
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    return x;
}

void sgp_b200_destroy(sgp_b200_ctx_t *x) {
    if (!x) return;
    Context &C = x->c;
    for (sgp_b200_ctx_t *w : C.workers) sgp_b200_destroy(w);
    C.workers.clear();
    cudaSetDevice(C.device);
    release_all(C);
    if (C.stream) {
        cudaStreamSynchronize(C.stream);
        cudaStreamDestroy(C.stream);
    }
    if (C.h_pinned) cudaFreeHost(C.h_pinned);
    if (C.h_stage) cudaFreeHost(C.h_stage);
    for (cudaEvent_t e : C.stage_ev)
        if (e) cudaEventDestroy(e);
    delete x;
}

const char *sgp_b200_last_error(void) { return last_error(); }

void *sgp_b200_stream(sgp_b200_ctx_t *x) { return x ? (void *)x->c.stream : nullptr; }

}  // extern "C"
