// split.cu -- median split of the Fiedler vector and its edge cut.
//
// Reference: cmg/sgpar.h:1969-2071 (sgp_compute_partition, local search off):
// sort (ev, u) ascending, ties by u; the first n - imbr vertices form part 0,
// the rest part 1; vertices at sorted positions [imbl, imbr) move to part 0
// while that does not raise the cut; edge cut = directed cross entries / 2.
//
// The reference sorts all n pairs on the host.  Only the order statistic at
// position imbl matters for the split, so this is a radix *select*: twelve
// 8-bit digit passes (64 key bits of the order-preserving image of the double,
// then 32 index bits) inside one cooperative kernel, each pass a histogram
// and a grid barrier.  part[i] = ((key_i, i) < threshold) ? 0 : 1, then one
// pass over the CSR counts the cut and the single sweep vertex of an odd n
// (perc_imbalance_allowed = 0, the value the reference's driver passes,
// sgpar.cpp:55) is decided on the device.
#include <mutex>

#include <cooperative_groups.h>

#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kSplitThreads = 512;

struct SplitArgs {
    uint32_t n;
    const uint32_t *rp;
    const uint32_t *col;
    const double *evec;
    uint32_t k;            // imbl: sorted position of the threshold element
    uint32_t sweep;        // 1 when position k is also the sweep vertex (imbr - imbl == 1)
    unsigned long long *keys;
    uint32_t *hist;        // [3][256], all zero at launch
    uint32_t *part;
    unsigned long long *cut_part;   // [gridDim]
    unsigned long long *out;        // [0] edgecut [1] part0 size [2] threshold index
};

__device__ __forceinline__ unsigned long long order_key(double x) {
    if (x == 0.0) x = 0.0;   // -0.0 == +0.0 in the reference's comparator
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void __launch_bounds__(kSplitThreads) k_split(SplitArgs a) {
    cg::grid_group grid = cg::this_grid();
    __shared__ uint32_t sh[256];
    __shared__ uint64_t sm[64];
    const uint32_t n = a.n;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < n; i += nth) a.keys[i] = order_key(a.evec[i]);
    // select: prefix over (key:64, index:32) = 96 bits, 12 digits MSB first
    unsigned long long kpre = 0;   // selected key bits so far
    uint32_t ipre = 0;             // selected index bits so far
    uint32_t rank = a.k;           // rank among candidates matching the prefix
    for (int pass = 0; pass < 12; pass++) {
        uint32_t *h = a.hist + (pass % 3) * 256;
        // Clear the buffer of the next pass.  It was last read after the barrier
        // of pass - 2, which every block has passed; it is next written after the
        // barrier of this pass.
        if (blockIdx.x == 0)
            for (int t = threadIdx.x; t < 256; t += blockDim.x) a.hist[((pass + 1) % 3) * 256 + t] = 0;
        for (int t = threadIdx.x; t < 256; t += blockDim.x) sh[t] = 0;
        __syncthreads();
        for (uint64_t i = tid; i < n; i += nth) {
            unsigned long long key = a.keys[i];
            uint32_t digit;
            if (pass < 8) {
                int shift = 56 - 8 * pass;
                // candidates: key bits above the current digit equal the prefix
                unsigned long long hi = pass == 0 ? 0 : (key >> (shift + 8));
                unsigned long long phi = pass == 0 ? 0 : (kpre >> (shift + 8));
                if (hi != phi) continue;
                digit = (uint32_t)((key >> shift) & 0xFF);
            } else {
                if (key != kpre) continue;
                int shift = 24 - 8 * (pass - 8);
                uint32_t idx = (uint32_t)i;
                uint32_t hi = pass == 8 ? 0 : (idx >> (shift + 8));
                uint32_t phi = pass == 8 ? 0 : (ipre >> (shift + 8));
                if (hi != phi) continue;
                digit = (idx >> shift) & 0xFF;
            }
            atomicAdd(&sh[digit], 1u);
        }
        __syncthreads();
        for (int t = threadIdx.x; t < 256; t += blockDim.x)
            if (sh[t]) atomicAdd(&h[t], sh[t]);
        grid.sync();
        // every block picks the same digit from the global histogram
        if (threadIdx.x == 0) {
            uint32_t acc = 0, d = 0;
            for (d = 0; d < 256; d++) {
                uint32_t c = h[d];
                if (rank < acc + c) break;
                acc += c;
            }
            sh[0] = d;
            sh[1] = rank - acc;
        }
        __syncthreads();
        const uint32_t d = sh[0];
        rank = sh[1];
        if (pass < 8) kpre |= (unsigned long long)d << (56 - 8 * pass);
        else ipre |= d << (24 - 8 * (pass - 8));
        __syncthreads();
    }
    // assign parts
    uint64_t c0 = 0;
    for (uint64_t i = tid; i < n; i += nth) {
        unsigned long long key = a.keys[i];
        bool less = key < kpre || (key == kpre && (uint32_t)i < ipre);
        a.part[i] = less ? 0u : 1u;
        c0 += less;
    }
    grid.sync();
    // directed cross entries, one warp per row
    uint64_t cut = 0;
    {
        const unsigned lane = threadIdx.x & 31;
        const uint64_t wid = tid >> 5, nw = nth >> 5;
        for (uint64_t i = wid; i < n; i += nw) {
            const uint32_t pi = a.part[i];
            uint32_t c = 0;
            for (uint32_t j = a.rp[i] + lane; j < a.rp[i + 1]; j += 32) c += (a.part[a.col[j]] != pi);
            cut += c;
        }
    }
    {
        uint64_t t1, t2;
        block_scan_u64(cut, sm, &t1);
        block_scan_u64(c0, sm, &t2);
        if (threadIdx.x == 0) {
            a.cut_part[2 * blockIdx.x] = t1;
            a.cut_part[2 * blockIdx.x + 1] = t2;
        }
    }
    grid.sync();
    if (blockIdx.x == 0) {
        uint64_t s = 0, s0 = 0;
        for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            s += a.cut_part[2 * b];
            s0 += a.cut_part[2 * b + 1];
        }
        uint64_t tot, tot0;
        block_scan_u64(s, sm, &tot);
        block_scan_u64(s0, sm, &tot0);
        // sweep of the vertex at position k (sgpar.h:2046-2071)
        long long upd = 0;
        if (a.sweep) {
            const uint32_t u = ipre;
            long long c = 0;
            for (uint32_t j = a.rp[u] + threadIdx.x; j < a.rp[u + 1]; j += blockDim.x)
                c += (a.part[a.col[j]] == 1) ? 1 : -1;
            uint64_t uc = (uint64_t)(c + (1ll << 40));   // bias to keep the scan unsigned
            uint64_t tt;
            block_scan_u64(uc, sm, &tt);
            upd = (long long)tt - (long long)blockDim.x * (1ll << 40);
        }
        if (threadIdx.x == 0) {
            long long cur = (long long)tot, best = (long long)tot;
            uint64_t p0 = tot0;
            if (a.sweep) {
                cur = cur + 2 * upd;
                if (cur <= best) {
                    a.part[ipre] = 0;
                    best = cur;
                    p0++;
                }
            }
            a.out[0] = (unsigned long long)(best / 2);
            a.out[1] = p0;
            a.out[2] = ipre;
        }
    }
}

int split_level(Context &C, const Level &L, const double *evec, int perc_imbalance, uint32_t *part,
                uint64_t *edgecut, uint32_t *n_part0) {
    const uint32_t n = L.n;
    if (n == 0) { *edgecut = 0; if (n_part0) *n_part0 = 0; return SGP_B200_OK; }
    if (perc_imbalance != 0) {
        set_error("perc_imbalance_allowed must be 0 (the value sgpar.cpp passes); got %d", perc_imbalance);
        return SGP_B200_ERR_INVALID;
    }
    // sgpar.h:2009-2012
    long long max_part_size = (long long)ceil(n / 2.0);
    uint32_t imbr = (uint32_t)floor(max_part_size * (1.0 + perc_imbalance / 100.0));
    uint32_t imbl = n - imbr;
    SplitArgs a;
    a.n = n; a.rp = L.rp; a.col = L.col; a.evec = evec; a.part = part;
    // With imbl == n there is no threshold element (cannot happen for p = 0).
    a.k = imbl < n ? imbl : n - 1;
    a.sweep = (imbr > imbl) ? 1u : 0u;
    SGPB_TRY(dalloc_t(C, &a.keys, n));
    SGPB_TRY(dalloc_t(C, &a.hist, 768));
    SGPB_TRY(dzero(C, a.hist, 768 * sizeof(uint32_t)));
    SGPB_TRY(dalloc_t(C, &a.out, 4));
    int per_sm = 0;
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_split, kSplitThreads, 0));
    if (per_sm < 1) { set_error("split kernel does not fit"); return SGP_B200_ERR_DEVICE; }
    if (per_sm > 2) per_sm = 2;
    uint64_t maxg = (uint64_t)per_sm * C.num_sms;
    uint64_t want = cdiv(n, kSplitThreads * 8ull);
    uint32_t grid = (uint32_t)(want < maxg ? want : maxg);
    if (grid < 1) grid = 1;
    SGPB_TRY(dalloc_t(C, &a.cut_part, 2 * (size_t)grid));
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel((const void *)k_split, dim3(grid), dim3(kSplitThreads), args, 0, C.stream));
    C.kernel_launches++;
    uint64_t out[3];
    SGPB_TRY(read_u64(C, (const uint64_t *)a.out, out, 3));
    *edgecut = out[0];
    if (n_part0) *n_part0 = (uint32_t)out[1];
    return SGP_B200_OK;
}

// --------------------------------------------------- split, no allocation --
// Scratch of sgp_b200_split_noalloc: sort keys for SGP_B200_NOALLOC_MAX_N
// vertices, the three digit histograms, per-block cut partials for up to
// kNoAllocMaxBlocks blocks and the result words.  It is a file-scope device
// array, so every GPU that loads this library holds it (about 8 MiB) until the
// process exits, and every call on a device shares it.
constexpr uint32_t kNoAllocMaxBlocks = 1024;
constexpr size_t kNoAllocKeysBytes = (size_t)SGP_B200_NOALLOC_MAX_N * sizeof(unsigned long long);
constexpr size_t kNoAllocHistOff = kNoAllocKeysBytes;
constexpr size_t kNoAllocCutOff = kNoAllocHistOff + 768 * sizeof(uint32_t);
constexpr size_t kNoAllocOutOff = kNoAllocCutOff + 2 * (size_t)kNoAllocMaxBlocks * sizeof(unsigned long long);
constexpr size_t kNoAllocBytes = kNoAllocOutOff + 4 * sizeof(unsigned long long);
static __device__ __align__(256) unsigned char g_split_scratch[kNoAllocBytes];

// Per-device set-up, done by the first call on that device: the host
// address of g_split_scratch is only a stand-in, so the device address comes
// from cudaGetSymbolAddress with the device current.  The address belongs to
// the context that loaded the module: after cudaDeviceReset (or any new
// context on the device) the cached one is stale, so the set-up is keyed by
// the current context's id and redone when that id changes.
struct NoAllocDevice {
    unsigned char *scratch = nullptr;
    int num_sms = 0;
    int per_sm = 0;
    unsigned long long ctx_id = 0;
    bool ready = false;
};
static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc_dev[64];

// Unique id of the calling thread's current context (cuCtxGetCurrent and
// cuCtxGetId through the runtime's driver entry points, so the library does
// not link the driver library itself).  Every context ever created in the
// process gets a distinct id.
typedef int (*CtxGetCurrentFn)(void **ctx);
typedef int (*CtxGetIdFn)(void *ctx, unsigned long long *id);
static int current_ctx_id(int device, unsigned long long *id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)f;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f;
    });
    if (!get_current || !get_id) {
        set_error("the CUDA driver does not provide cuCtxGetCurrent / cuCtxGetId");
        return SGP_B200_ERR_DEVICE;
    }
    // makes the device's primary context current if no context is yet
    SGPB_CUDA(cudaSetDevice(device));
    void *ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) {
        set_error("no current CUDA context on device %d", device);
        return SGP_B200_ERR_DEVICE;
    }
    return SGP_B200_OK;
}

static int noalloc_setup(int device, NoAllocDevice **out) {
    if (device < 0 || device >= 64) {
        set_error("device %d out of range for the no-allocation entry point", device);
        return SGP_B200_ERR_INVALID;
    }
    unsigned long long id = 0;
    SGPB_TRY(current_ctx_id(device, &id));
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice &d = g_noalloc_dev[device];
    if (!d.ready || d.ctx_id != id) {
        d.ready = false;
        void *p = nullptr;
        SGPB_CUDA(cudaGetSymbolAddress(&p, g_split_scratch));
        SGPB_CUDA(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, device));
        SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.per_sm, (const void *)k_split, kSplitThreads, 0));
        if (d.per_sm < 1) {
            set_error("split kernel does not fit on an SM");
            return SGP_B200_ERR_DEVICE;
        }
        d.scratch = (unsigned char *)p;
        d.ctx_id = id;
        d.ready = true;
    }
    *out = &d;
    return SGP_B200_OK;
}

// ------------------------------------------------------------- edge cut --
__global__ void k_cut(uint32_t n, const uint32_t *rp, const uint32_t *col, const uint32_t *part,
                      unsigned long long *out) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint32_t c = 0;
    for (uint64_t i = wid; i < n; i += nw) {
        const uint32_t pi = part[i];
        for (uint32_t j = rp[i] + lane; j < rp[i + 1]; j += 32) c += (part[col[j]] != pi);
    }
    c = warp_sum(c);
    if (lane == 0 && c) atomicAdd(out, (unsigned long long)c);
}

int edge_cut_device(Context &C, const Level &L, const uint32_t *part, uint64_t *edgecut) {
    unsigned long long *o;
    SGPB_TRY(dalloc_t(C, &o, 1));
    SGPB_TRY(dzero(C, o, 8));
    if (L.n) {
        uint32_t g = cdiv(L.n, 8);
        if (g > (uint32_t)C.num_sms * 8) g = C.num_sms * 8;
        k_cut<<<g, 256, 0, C.stream>>>(L.n, L.rp, L.col, part, o);
        C.kernel_launches++;
    }
    uint64_t h;
    SGPB_TRY(read_u64(C, (const uint64_t *)o, &h));
    *edgecut = h / 2;
    return SGP_B200_OK;
}

// --------------------------------------------------------- local search --
// sgpar.h:2080-2170: after the split, alternately flip the vertex of largest
// positive gain (cross minus same-side neighbours; first id on a tie) among
// ids [mid - n/3, mid) and then among [mid, mid + n/3), mid being the part-0
// size the split left; a missing second move undoes the first and ends the
// search, as does a missing first move or n/3 completed pairs.  The
// reference recomputes every candidate's gain per move (O(n m) in all); here
// the gains are kept incrementally -- a flip negates the vertex's own gain
// and moves each neighbour's by 2 -- and each half-step is a grid-wide
// argmax plus one row update in a single cooperative launch.
//
// Ordering: a flip of part[v] is deferred to the next phase (after a grid
// barrier), so no thread reads part[v] while it is written; the argmax
// phase reads gains only.  Four argmax slots rotate; the slot two
// half-steps ahead is cleared while the current one is read.  Gains and
// parts change between barriers on other SMs, so after the first phase
// they are read with ld.global.cg (L2), never from a possibly stale L1 line.
constexpr int kLSThreads = 512;

struct LSArgs {
    uint32_t n;
    const uint32_t *rp, *col;
    uint32_t *part;
    int *gain;
    uint32_t lo, mid, hi, max_swaps;
    unsigned long long *key;   // [4], zero on entry
    uint32_t *out;             // [0] swaps
};

namespace cgls = cooperative_groups;

__global__ void __launch_bounds__(kLSThreads) k_local_search(LSArgs a) {
    cgls::grid_group grid = cgls::this_grid();
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    __shared__ unsigned long long wmax[kLSThreads / 32];
    // gains, a warp per row
    for (uint64_t u = tid >> 5; u < a.n; u += nthreads >> 5) {
        const uint32_t pu = a.part[u];
        int x = 0;
        for (uint32_t j = a.rp[u] + lane; j < a.rp[u + 1]; j += 32) x += a.part[__ldg(a.col + j)] != pu ? 1 : -1;
        x = warp_sum(x);
        if (lane == 0) a.gain[u] = x;
    }
    grid.sync();
    uint32_t pending = 0xFFFFFFFFu, first = 0xFFFFFFFFu, swaps = 0, slot = 0;
    for (int half = 0;; half ^= 1) {
        if (half == 0 && swaps >= a.max_swaps) break;
        // ---- argmax of (gain, -id) over this half's range, gains > 0 only
        if (leader && pending != 0xFFFFFFFFu) a.part[pending] = __ldcg(a.part + pending) ^ 1u;
        pending = 0xFFFFFFFFu;
        const uint32_t b = half == 0 ? a.lo : a.mid, e = half == 0 ? a.mid : a.hi;
        unsigned long long best = 0;
        for (uint64_t i = b + tid; i < e; i += nthreads) {
            const int g = __ldcg(a.gain + i);
            if (g > 0) {
                const unsigned long long k = ((unsigned long long)(uint32_t)g << 32) | (0xFFFFFFFFu - (uint32_t)i);
                best = k > best ? k : best;
            }
        }
        best = warp_max(best);
        if (lane == 0) wmax[wid] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long m = 0;
            for (int w = 0; w < kLSThreads / 32; w++) m = wmax[w] > m ? wmax[w] : m;
            if (m) atomicMax(a.key + slot, m);
        }
        grid.sync();
        // ---- apply: flip the winner (deferred) and move its neighbours' gains
        const unsigned long long k = *(volatile unsigned long long *)(a.key + slot);
        if (leader) a.key[(slot + 2) & 3] = 0;
        slot = (slot + 1) & 3;
        uint32_t v;
        if (k == 0) {
            if (half == 0) break;   // no first move: done
            v = first;              // no second move: undo the first, then done
        } else {
            v = 0xFFFFFFFFu - (uint32_t)(k & 0xFFFFFFFFu);
        }
        const uint32_t old = __ldcg(a.part + v);
        for (uint64_t j = a.rp[v] + tid; j < a.rp[v + 1]; j += nthreads) {
            const uint32_t u = __ldg(a.col + j);
            // rows hold u once: no other writer of gain[u] in this phase
            a.gain[u] = __ldcg(a.gain + u) + (__ldcg(a.part + u) != old ? -2 : 2);
        }
        if (leader) a.gain[v] = -__ldcg(a.gain + v);
        pending = v;
        grid.sync();
        if (k == 0) break;          // the undo above ends the search
        if (half == 0) first = v;
        else swaps++;
    }
    grid.sync();
    if (leader) {
        if (pending != 0xFFFFFFFFu) a.part[pending] = __ldcg(a.part + pending) ^ 1u;
        a.out[0] = swaps;
    }
    grid.sync();
    // part-0 size after the search (the moves need not balance)
    uint32_t z = 0;
    for (uint64_t i = tid; i < a.n; i += nthreads) z += __ldcg(a.part + i) == 0;
    z = warp_sum(z);
    if (lane == 0 && z) atomicAdd(a.out + 1, z);
}

int local_search_level(Context &C, const Level &L, uint32_t *part, uint32_t mid, uint32_t *swaps_out,
                       uint32_t *part0_out) {
    const uint32_t n = L.n;
    if (n < 3) {
        if (swaps_out) *swaps_out = 0;
        if (part0_out) *part0_out = mid;
        return SGP_B200_OK;
    }
    LSArgs a;
    a.n = n;
    a.rp = L.rp;
    a.col = L.col;
    a.part = part;
    a.mid = mid;
    a.lo = mid > n / 3 ? mid - n / 3 : 0;
    a.hi = (uint64_t)mid + n / 3 < n ? mid + n / 3 : n;
    a.max_swaps = n / 3;
    SGPB_TRY(dalloc_t(C, &a.gain, n));
    SGPB_TRY(dalloc_t(C, &a.key, 4));
    SGPB_TRY(dalloc_t(C, &a.out, 2));
    SGPB_TRY(dzero(C, a.out, 2 * sizeof(uint32_t)));
    SGPB_TRY(dzero(C, a.key, 4 * sizeof(unsigned long long)));
    int per_sm = 0;
    SGPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_local_search, kLSThreads, 0));
    if (per_sm < 1) {
        set_error("local-search kernel does not fit on an SM");
        return SGP_B200_ERR_DEVICE;
    }
    // one block per SM at most: the per-move barriers cost less with fewer
    // blocks, and a range of n/3 gains is a light scan
    uint32_t grid = cdiv((uint64_t)n, 4096);
    if (grid > (uint32_t)C.num_sms) grid = C.num_sms;
    if (grid < 1) grid = 1;
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel((const void *)k_local_search, dim3(grid), dim3(kLSThreads), args, 0,
                                          C.stream));
    C.kernel_launches++;
    uint32_t o[2] = {0, 0};
    SGPB_TRY(read_u32(C, a.out, o, 2));
    if (swaps_out) *swaps_out = o[0];
    if (part0_out) *part0_out = o[1];
    return SGP_B200_OK;
}

// ------------------------------------------------- induced sub-graphs --
// sgpar.h:2666-2752: vertices of each part relabelled in ascending order,
// edges inside each part kept in row order.
__global__ void k_same_part_counts(uint32_t n, const uint32_t *rp, const uint32_t *col, const uint32_t *part,
                                   uint32_t *cnt0, uint32_t *cnt1, uint32_t *is0, uint32_t *is1) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = wid; i < n; i += nw) {
        const uint32_t pi = part[i];
        uint32_t c = 0;
        for (uint32_t j = rp[i] + lane; j < rp[i + 1]; j += 32) c += (part[col[j]] == pi);
        c = warp_sum(c);
        if (lane == 0) {
            cnt0[i] = pi == 0 ? c : 0;
            cnt1[i] = pi == 0 ? 0 : c;
            is0[i] = pi == 0;
            is1[i] = pi != 0;
        }
    }
}

__global__ void k_fill_sub(uint32_t n, const uint32_t *rp, const uint32_t *col, const uint32_t *part,
                           const uint32_t *map0, const uint32_t *map1, const uint32_t *off0, const uint32_t *off1,
                           uint32_t *rp1, uint32_t *col1, uint32_t *rp2, uint32_t *col2) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = wid; i < n; i += nw) {
        const uint32_t pi = part[i];
        uint32_t o = pi == 0 ? off0[i] : off1[i];
        uint32_t *dst = pi == 0 ? col1 : col2;
        if (lane == 0) {
            if (pi == 0) rp1[map0[i]] = o; else rp2[map1[i]] = o;
        }
        const uint32_t b = rp[i], e = rp[i + 1];
        for (uint32_t j0 = b; j0 < e; j0 += 32) {
            uint32_t j = j0 + lane;
            bool keep = false;
            uint32_t v = 0;
            if (j < e) { v = col[j]; keep = part[v] == pi; }
            unsigned m = __ballot_sync(0xFFFFFFFFu, keep);
            if (keep) dst[o + __popc(m & ((1u << lane) - 1u))] = pi == 0 ? map0[v] : map1[v];
            o += __popc(m);
        }
    }
}

int induced_subgraphs(Context &C, const Level &L, const uint32_t *part, Level *g1, Level *g2, uint32_t **map0_out,
                      uint32_t **map1_out) {
    const uint32_t n = L.n;
    uint32_t *cnt0, *cnt1, *is0, *is1, *off0, *off1, *map0, *map1;
    SGPB_TRY(dalloc_t(C, &cnt0, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &cnt1, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &is0, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &is1, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &off0, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &off1, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &map0, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &map1, (size_t)n + 1));
    uint32_t g = n ? cdiv(n, 8) : 1;
    if (g > (uint32_t)C.num_sms * 8) g = C.num_sms * 8;
    if (n) k_same_part_counts<<<g, 256, 0, C.stream>>>(n, L.rp, L.col, part, cnt0, cnt1, is0, is1);
    SGPB_TRY(scan_u32(C, cnt0, off0, n, nullptr));
    SGPB_TRY(scan_u32(C, cnt1, off1, n, nullptr));
    SGPB_TRY(scan_u32(C, is0, map0, n, nullptr));
    SGPB_TRY(scan_u32(C, is1, map1, n, nullptr));
    uint32_t tots[2], nn[2];
    SGPB_TRY(read_u32(C, off0 + n, &tots[0]));
    SGPB_TRY(read_u32(C, off1 + n, &tots[1]));
    SGPB_TRY(read_u32(C, map0 + n, &nn[0]));
    SGPB_TRY(read_u32(C, map1 + n, &nn[1]));
    g1->n = nn[0]; g1->m = tots[0]; g1->wbytes = 0; g1->w = nullptr;
    g2->n = nn[1]; g2->m = tots[1]; g2->wbytes = 0; g2->w = nullptr;
    SGPB_TRY(dalloc_t(C, &g1->rp, (size_t)nn[0] + 1));
    SGPB_TRY(dalloc_t(C, &g2->rp, (size_t)nn[1] + 1));
    SGPB_TRY(dalloc_t(C, &g1->col, (size_t)tots[0] + 1));
    SGPB_TRY(dalloc_t(C, &g2->col, (size_t)tots[1] + 1));
    if (n)
        k_fill_sub<<<g, 256, 0, C.stream>>>(n, L.rp, L.col, part, map0, map1, off0, off1, g1->rp, g1->col, g2->rp,
                                            g2->col);
    SGPB_CUDA(cudaMemcpyAsync(g1->rp + nn[0], off0 + n, 4, cudaMemcpyDeviceToDevice, C.stream));
    SGPB_CUDA(cudaMemcpyAsync(g2->rp + nn[1], off1 + n, 4, cudaMemcpyDeviceToDevice, C.stream));
    C.kernel_launches += 2;
    SGPB_CUDA(cudaGetLastError());
    if (map0_out) *map0_out = map0;
    if (map1_out) *map1_out = map1;
    return SGP_B200_OK;
}

}  // namespace sgpb

using namespace sgpb;

// Median split + edge cut of a device eigenvector without any allocation: the
// scratch is g_split_scratch above.  Meant for callers that cannot allocate
// device memory at that point: a host application that owns every device
// allocation through its own pool, code running inside an out-of-memory
// handler, or a plug-in whose allocation calls are forbidden by its host.
// The first call on a device (and the first after the device's context
// changed, e.g. after cudaDeviceReset) fetches the scratch address (see
// noalloc_setup); make that first call before any stream capture.  The stream
// must belong to the current device.  Calls that overlap on the GPU
// (different streams, or graphs replayed concurrently) share the scratch and
// race; serialise them.
extern "C" int sgp_b200_split_noalloc(void *stream, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                                      const double *evec, uint32_t *part, uint64_t *result) {
    // col may be NULL for a graph without edges, as for sgp_b200_split
    if (!row_ptr || !evec || !part || !result) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    if (n == 0 || n > SGP_B200_NOALLOC_MAX_N) {
        set_error("sgp_b200_split_noalloc handles 1 .. %u vertices (its fixed scratch size); got %u",
                  (unsigned)SGP_B200_NOALLOC_MAX_N, n);
        return SGP_B200_ERR_TOO_LARGE;
    }
    int device = 0;
    SGPB_CUDA(cudaGetDevice(&device));
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        int sdev = -1;
        SGPB_CUDA(cudaStreamGetDevice(s, &sdev));
        if (sdev != device) {
            set_error("sgp_b200_split_noalloc: the stream belongs to device %d but device %d is current; "
                      "make the stream's device current",
                      sdev, device);
            return SGP_B200_ERR_INVALID;
        }
    }
    NoAllocDevice *d = nullptr;
    SGPB_TRY(noalloc_setup(device, &d));
    SplitArgs a;
    a.n = n;
    a.rp = row_ptr;
    a.col = col;
    a.evec = evec;
    a.part = part;
    // sgpar.h:2009-2012 with perc_imbalance_allowed = 0
    const uint32_t imbr = (uint32_t)ceil(n / 2.0);
    const uint32_t imbl = n - imbr;
    a.k = imbl < n ? imbl : n - 1;
    a.sweep = imbr > imbl ? 1u : 0u;
    a.keys = reinterpret_cast<unsigned long long *>(d->scratch);
    a.hist = reinterpret_cast<uint32_t *>(d->scratch + kNoAllocHistOff);
    a.cut_part = reinterpret_cast<unsigned long long *>(d->scratch + kNoAllocCutOff);
    a.out = reinterpret_cast<unsigned long long *>(d->scratch + kNoAllocOutOff);
    // the scratch keeps the previous call's contents: the histograms must
    // start at zero; keys, partials and results are written before use
    SGPB_CUDA(cudaMemsetAsync(a.hist, 0, 768 * sizeof(uint32_t), s));
    const int per_sm = d->per_sm > 2 ? 2 : d->per_sm;
    uint64_t grid = (uint64_t)per_sm * d->num_sms;
    const uint64_t want = cdiv(n, kSplitThreads * 8ull);
    if (want < grid) grid = want;
    if (grid > kNoAllocMaxBlocks) grid = kNoAllocMaxBlocks;
    if (grid < 1) grid = 1;
    void *args[] = {&a};
    SGPB_CUDA(cudaLaunchCooperativeKernel((const void *)k_split, dim3((unsigned)grid), dim3(kSplitThreads), args, 0, s));
    // result[0] = edge cut, result[1] = size of part 0 (device array)
    SGPB_CUDA(cudaMemcpyAsync(result, a.out, 2 * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    SGPB_CUDA(cudaGetLastError());
    return SGP_B200_OK;
}
