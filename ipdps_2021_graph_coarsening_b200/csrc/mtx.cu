// mtx.cu -- MatrixMarket coordinate text to the CSR graph of its largest
// connected component, on the device.
//
// Reference: cmg/mtx2csr.cpp:13-303 (cmg/mtx2csr_large.cpp: the same steps
// with 64-bit words in the output file).  The rules are the reference's:
//   * a banner line ("%%...") must contain "coordinate"; "general" marks a
//     non-symmetric pattern (:51-80); other lines starting with '%' are
//     comments;
//   * the first other line is the size line "rows cols entries"; a general
//     square matrix is read as A + A^T, a general rectangular one as the
//     bipartite graph whose vertices 0..cols-1 are the columns and
//     cols..cols+rows-1 the rows (:87-104);
//   * every entry line "i j [value]" adds both directions; self loops are
//     dropped unless bipartite; values are ignored (:105-128);
//   * rows sorted ascending with duplicates removed (:132-157);
//   * the largest connected component is kept (the first in vertex order
//     among equally large ones), its vertices renumbered in ascending order
//     (:166-264);
//   * file: six 64-bit words N, M (directed entries), 1, 0, 1, 0, then
//     offsets[N+1] and destinations[M] as 32-bit words (64-bit for the
//     large variant) (:266-289).
// Where the reference's behaviour is undefined (an id of 0 or beyond the
// size line, an entry line that is not "i j ...", a symmetric banner on a
// non-square size line, a later banner that switches the format) this path
// fails naming the line; blank lines are skipped.
//
// Device pipeline:
//   1. the file is copied to HBM through a pinned ring, so reading the file
//      overlaps the copy; the buffer is zero padded past its end;
//   2. line starts are counted per 8 KiB tile (one 32-byte vector load per
//      thread, '\n' found with a SIMD byte compare) and the tile counts
//      scanned;
//   3. one pass parses every line -- line index = tile base + block prefix --
//      into the two packed keys (u << b | v) and (v << b | u) of its entry;
//   4. one stable radix sort of all keys (sort.cu) groups every row's
//      entries in column order; the first key of each run of equal keys is
//      a distinct entry, and the heads, numbered by a scan, are the CSR
//      columns in order;
//   5. a lock-free union-find labels components by their smallest vertex: a
//      union hooks the larger of two roots under the smaller with a CAS,
//      finds halve paths, and parent[x] <= x always holds, so every walk
//      terminates.  Edges are joined in the sampling order of Afforest
//      (Sutton, Ben-Nun, Barak, IPDPS 2018): every vertex with its first two
//      neighbours, then the root holding most of 1024 probed vertices is the
//      giant component and only vertices outside it join their remaining
//      neighbours;
//   6. component sizes by warp-aggregated atomics, the largest (ties: the
//      smallest label, i.e. the first the reference's BFS finds) by a 64-bit
//      max over (size << 32 | ~label);
//   7. the component is extracted with its rows whole (every neighbour of a
//      component vertex is in it) and columns renumbered through a scan of
//      the keep flags, so rows stay sorted.
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>

#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace sgpb {

constexpr int kMtxThreads = 256;
constexpr int kMtxBytes = 32;                                   // bytes per thread
constexpr uint64_t kMtxTile = (uint64_t)kMtxThreads * kMtxBytes;  // bytes per block
constexpr uint32_t kNoEdge = 0xFFFFFFFFu;
constexpr unsigned long long kNoKey = ~0ull;   // sorts after every entry key
constexpr int kMaxBanners = 16;
constexpr int kStageSlots = 4;
constexpr size_t kStageSlotBytes = (size_t)32 << 20;

enum : uint32_t { kLineSyntax = 1, kLineZero = 2, kLineRange = 3 };

// Line starts: position p + 1 starts a line when p == lo (the size line's
// terminator) or text[p] == '\n', for p in [lo, len - 1).
struct MtxScan {
    const uint8_t *text;   // file bytes, zero padded by at least one tile
    uint64_t len;
    uint64_t lo;
    uint64_t t0;           // first tile: tile t covers [t * kMtxTile, (t + 1) * kMtxTile)
};

// bit b set: position base + b precedes a line start
__device__ __forceinline__ uint32_t start_mask(const MtxScan &s, uint64_t base) {
    const uint64_t end = s.len - 1;
    if (base + kMtxBytes <= s.lo || base >= end) return 0u;
    const uint4 *p = reinterpret_cast<const uint4 *>(s.text + base);
    const uint4 a = __ldg(p), b = __ldg(p + 1);
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t eq = __vcmpeq4(w[k], 0x0A0A0A0Au);   // 0xFF in every byte equal to '\n'
        const uint32_t nib = ((eq >> 7) & 1u) | ((eq >> 14) & 2u) | ((eq >> 21) & 4u) | ((eq >> 28) & 8u);
        m |= nib << (4 * k);
    }
    if (base <= s.lo) {
        const uint32_t i = (uint32_t)(s.lo - base);
        m = ((m >> i) << i) | (1u << i);
    }
    if (base + kMtxBytes > end) m &= (1u << (uint32_t)(end - base)) - 1u;
    return m;
}

__global__ void __launch_bounds__(kMtxThreads) k_mtx_count(MtxScan s, uint32_t *__restrict__ tile_cnt) {
    __shared__ uint32_t ws[kMtxThreads / 32];
    const uint64_t base = (s.t0 + blockIdx.x) * kMtxTile + (uint64_t)threadIdx.x * kMtxBytes;
    uint32_t c = warp_sum((uint32_t)__popc(start_mask(s, base)));
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int i = 0; i < kMtxThreads / 32; i++) t += ws[i];
        tile_cnt[blockIdx.x] = t;
    }
}

struct MtxParse {
    MtxScan s;
    const uint32_t *tile_base;   // exclusive scan of the tile counts
    uint32_t rows, cols;         // bounds of the two ids
    uint32_t shift;              // bipartite: row id i is vertex cols + i - 1; else 0
    int drop_loops;
    unsigned long long *keys;    // per line two keys, (u << b | v) and (v << b | u), kNoKey when it adds nothing
    int b;                       // bits per id in a key
    uint32_t *valid;             // lines that add an entry
    unsigned long long *err;     // min over failing lines of (line << 8 | reason)
    unsigned long long *banner;  // [0] count, [1..kMaxBanners] offsets of banner lines
};

__device__ __forceinline__ bool is_blank(uint32_t c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
}

// The unsigned decimal at text[i..] as scanf's %u reads it after its
// whitespace skip: optional '+', then digits.  Saturates far above any id.
__device__ __forceinline__ bool parse_id(const uint8_t *__restrict__ t, uint64_t &i, uint64_t &v) {
    uint32_t c = __ldg(t + i);
    while (is_blank(c)) c = __ldg(t + ++i);
    if (c == '+') c = __ldg(t + ++i);
    if (c < '0' || c > '9') return false;
    v = 0;
    do {
        v = v * 10 + (c - '0');
        if (v > (1ull << 40)) v = 1ull << 40;
        c = __ldg(t + ++i);
    } while (c >= '0' && c <= '9');
    return true;
}

__device__ __forceinline__ void line_fail(const MtxParse &a, uint32_t k, uint32_t why) {
    atomicMin(a.err, ((unsigned long long)k << 8) | why);
}

// The line starting at byte s (line k after the size line).
__device__ __forceinline__ void parse_line(const MtxParse &a, uint64_t s, uint32_t k, uint32_t &u, uint32_t &v) {
    const uint8_t *__restrict__ t = a.s.text;
    uint32_t c = __ldg(t + s);
    if (c == '%') {
        if (__ldg(t + s + 1) == '%') {
            const unsigned long long slot = atomicAdd(a.banner, 1ull);
            if (slot < kMaxBanners) a.banner[1 + slot] = s;
        }
        return;
    }
    uint64_t i = s;
    while (is_blank(c)) c = __ldg(t + ++i);
    if (c == '\n' || c == 0) return;
    uint64_t x = 0, y = 0;
    if (!parse_id(t, i, x) || !parse_id(t, i, y)) return line_fail(a, k, kLineSyntax);
    if (x == 0 || y == 0) return line_fail(a, k, kLineZero);
    if (x > a.rows || y > a.cols) return line_fail(a, k, kLineRange);
    const uint32_t uu = (uint32_t)(x - 1) + a.shift, vv = (uint32_t)(y - 1);
    if (a.drop_loops && uu == vv) return;
    u = uu;
    v = vv;
}

// cnt[x] += 1 for every lane with x != kNoEdge, one atomic per distinct x in
// the warp.  All 32 lanes must call it.
__device__ __forceinline__ void add_one(uint32_t *cnt, uint32_t x) {
    const unsigned act = __ballot_sync(0xFFFFFFFFu, x != kNoEdge);
    if (x != kNoEdge) {
        const unsigned peers = __match_any_sync(act, x);
        if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(cnt + x, (uint32_t)__popc(peers));
    }
}

__global__ void __launch_bounds__(kMtxThreads) k_mtx_parse(MtxParse a) {
    __shared__ uint64_t sm[33];
    const uint64_t base = (a.s.t0 + blockIdx.x) * kMtxTile + (uint64_t)threadIdx.x * kMtxBytes;
    uint32_t m = start_mask(a.s, base);
    const uint32_t mine = __popc(m);
    uint64_t tot;
    uint32_t k = a.tile_base[blockIdx.x] + (uint32_t)(block_scan_u64(mine, sm, &tot) - mine);
    uint32_t valid = 0;
    while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        uint32_t u = kNoEdge, v = kNoEdge;
        parse_line(a, base + b + 1, k, u, v);
        unsigned long long k0 = kNoKey, k1 = kNoKey;
        if (u != kNoEdge) {
            k0 = ((unsigned long long)u << a.b) | v;
            k1 = ((unsigned long long)v << a.b) | u;
            valid++;
        }
        reinterpret_cast<ulonglong2 *>(a.keys)[k] = make_ulonglong2(k0, k1);
        k++;
    }
    valid = warp_sum(valid);
    if ((threadIdx.x & 31) == 0 && valid) atomicAdd(a.valid, valid);
}

// Sorted keys -> CSR: a key that differs from its predecessor starts a run
// (duplicates merged); heads are numbered by a scan, and since the keys are
// sorted by (row, column) the heads are the CSR entries in order.
__global__ void __launch_bounds__(256) k_mtx_heads(uint64_t cnt, const unsigned long long *__restrict__ keys,
                                                   uint32_t *__restrict__ head) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += stride)
        head[i] = i == 0 || __ldg(keys + i) != __ldg(keys + i - 1);
}

// col[pos] = the head's column; rows[row] counts heads (one atomic per run of
// equal rows within a warp: the keys are sorted)
__global__ void __launch_bounds__(256) k_mtx_emit(uint64_t cnt, const unsigned long long *__restrict__ keys,
                                                  const uint32_t *__restrict__ head, const uint32_t *__restrict__ pos,
                                                  int b, uint32_t *__restrict__ col, uint32_t *__restrict__ rows) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned long long mask = (1ull << b) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i - lane < cnt; i += stride) {
        uint32_t r = kNoEdge;
        if (i < cnt && head[i]) {
            const unsigned long long k = __ldg(keys + i);
            col[pos[i]] = (uint32_t)(k & mask);
            r = (uint32_t)(k >> b);
        }
        add_one(rows, r);
    }
}

// ------------------------------------------------------------ components --
// parent[x] <= x for every x at all times; x is a root iff parent[x] == x.
// Loads and stores of parent bypass L1 (other SMs change it).
__device__ __forceinline__ uint32_t cc_find(uint32_t *parent, uint32_t x) {
    uint32_t p = __ldcg(parent + x);
    while (p != x) {
        const uint32_t g = __ldcg(parent + p);
        if (g == p) return p;
        __stcg(parent + x, g);   // halve: x now hangs under its grandparent
        x = g;
        p = __ldcg(parent + x);
    }
    return x;
}

// Every failed CAS means another thread linked `hi`, which happens once per
// vertex, so a union retries at most n times; `cap` = n + 1 only guards a bug.
__device__ __forceinline__ void cc_union(uint32_t *parent, uint32_t a, uint32_t b, uint32_t cap, uint32_t *err) {
    a = cc_find(parent, a);
    b = cc_find(parent, b);
    for (uint32_t tries = 0; a != b; tries++) {
        if (tries > cap) {
            atomicOr(err, 1u);
            return;
        }
        const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
        const uint32_t old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) return;
        a = cc_find(parent, old);
        b = cc_find(parent, lo);
    }
}

__global__ void __launch_bounds__(256) k_cc_init(uint32_t n, uint32_t *__restrict__ parent) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) parent[i] = (uint32_t)i;
}

// sampling round r: every vertex joins its r-th neighbour
__global__ void __launch_bounds__(256) k_cc_sample(uint32_t n, const uint32_t *__restrict__ rp,
                                                   const uint32_t *__restrict__ col, uint32_t *parent, uint32_t r,
                                                   uint32_t *err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
        const uint32_t j = rp[u] + r;
        if (j < rp[u + 1]) cc_union(parent, (uint32_t)u, __ldg(col + j), n + 1, err);
    }
}

// parent[x] = root of x
__global__ void __launch_bounds__(256) k_cc_compress(uint32_t n, uint32_t *parent) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        __stcg(parent + i, cc_find(parent, (uint32_t)i));
}

__global__ void k_cc_probe(uint32_t n, uint32_t count, const uint32_t *__restrict__ parent, uint32_t *out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] = parent[(uint64_t)k * n / count];
}

// The entries from r0 on of every vertex not hanging directly under `skip`
// (the root of the component that the sampling made largest), G lanes per
// row.  An edge (u, v) skipped from u's side is joined from v's unless v
// hangs under `skip` too, in which case both ends are already connected.
template <int G>
__global__ void __launch_bounds__(256) k_cc_rest(uint32_t n, const uint32_t *__restrict__ rp,
                                                 const uint32_t *__restrict__ col, uint32_t *parent, uint32_t skip,
                                                 uint32_t r0, uint32_t *err) {
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t ng = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; u < n; u += ng) {
        // each lane reads this on its own, so lanes of a row may differ when
        // u is hooked meanwhile; skipping any subset of u's entries is safe
        if (__ldcg(parent + u) == skip) continue;
        const uint32_t e = rp[u + 1];
        for (uint32_t j = rp[u] + r0 + lane; j < e; j += G) cc_union(parent, (uint32_t)u, __ldg(col + j), n + 1, err);
    }
}

// parent[x] = root of x; size[root] += 1
__global__ void __launch_bounds__(256) k_cc_flatten(uint32_t n, uint32_t *parent, uint32_t *size) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i - lane < n; i += stride) {
        uint32_t r = kNoEdge;
        if (i < n) {
            r = cc_find(parent, (uint32_t)i);
            __stcg(parent + i, r);
        }
        add_one(size, r);
    }
}

// best = max over roots of (size << 32 | ~root); ncomp = number of roots
__global__ void __launch_bounds__(256) k_cc_best(uint32_t n, const uint32_t *__restrict__ parent,
                                                 const uint32_t *__restrict__ size,
                                                 unsigned long long *best, uint32_t *ncomp) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i - lane < n; i += stride) {
        const bool root = i < n && parent[i] == (uint32_t)i;
        unsigned long long key = root ? ((unsigned long long)size[i] << 32) | (0xFFFFFFFFu - (uint32_t)i) : 0ull;
        key = warp_max(key);
        const unsigned roots = __popc(__ballot_sync(0xFFFFFFFFu, root));
        if (lane == 0 && roots) {
            atomicMax(best, key);
            atomicAdd(ncomp, roots);
        }
    }
}

// ------------------------------------------------------------ extraction --
__global__ void __launch_bounds__(256) k_lcc_mark(uint32_t n, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ parent, uint32_t root,
                                                  uint32_t *__restrict__ keep, uint32_t *__restrict__ len) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const bool k = parent[i] == root;
        keep[i] = k;
        len[i] = k ? rp[i + 1] - rp[i] : 0u;
    }
}

__global__ void __launch_bounds__(256) k_lcc_fill(uint32_t n, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ col,
                                                  const uint32_t *__restrict__ parent, uint32_t root,
                                                  const uint32_t *__restrict__ map, const uint32_t *__restrict__ off,
                                                  uint32_t *__restrict__ orp, uint32_t *__restrict__ ocol) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        if (parent[r] != root) continue;   // warp-uniform
        const uint32_t b = rp[r], len = rp[r + 1] - b, o = off[r];
        if (lane == 0) orp[map[r]] = o;
        for (uint32_t i = lane; i < len; i += 32) ocol[o + i] = __ldg(map + __ldg(col + b + i));
    }
}

// ----------------------------------------------------------------- host --
struct MtxHead {
    int general = 0;
    int have_size = 0;
    uint64_t rows = 0, cols = 0, nnz = 0;
    uint64_t body = 0;    // first byte after the size line
    uint64_t lines = 0;   // lines up to and including the size line
};

// only blanks before the end of the line or a NUL (where the C string that
// sscanf reads ends)
static bool blank_line(const char *t, uint64_t n) {
    for (uint64_t i = 0; i < n && t[i] != 0; i++)
        if (!(t[i] == ' ' || t[i] == '\t' || t[i] == '\r' || t[i] == '\v' || t[i] == '\f')) return false;
    return true;
}

// banner rules of mtx2csr.cpp:53-79 for one line starting with "%%"
// (line_no 0: a banner after the size line, whose number is not tracked)
static int check_banner(const char *t, uint64_t n, uint64_t line_no, int *general) {
    const std::string line(t, n);
    if (line.find("coordinate") == std::string::npos) {
        if (line_no)
            set_error("line %llu: the banner does not say \"coordinate\"; only coordinate files are read",
                      (unsigned long long)line_no);
        else
            set_error("a banner after the size line does not say \"coordinate\": %s", line.c_str());
        return SGP_B200_ERR_INVALID;
    }
    if (line.find("general") != std::string::npos) *general = 1;
    return SGP_B200_OK;
}

// Banners, comments and the size line at the head of `t` (the first `avail`
// bytes; `whole`: they are the entire file).  Returns 1 when more bytes are
// needed to reach the end of the size line.
static int parse_head(const char *t, uint64_t avail, bool whole, MtxHead *h) {
    *h = MtxHead();
    uint64_t i = 0;
    while (i < avail) {
        const char *nl = (const char *)memchr(t + i, '\n', avail - i);
        if (!nl && !whole) return 1;
        const uint64_t e = nl ? (uint64_t)(nl - t) : avail;
        h->lines++;
        if (t[i] == '%') {
            if (e - i > 1 && t[i + 1] == '%') SGPB_TRY(check_banner(t + i, e - i, h->lines, &h->general));
        } else if (!blank_line(t + i, e - i)) {
            const std::string line(t + i, e - i);
            long long v[3] = {0, 0, 0};
            int got = sscanf(line.c_str(), "%lld %lld %lld", &v[0], &v[1], &v[2]);
            if (got < 2 || v[0] < 0 || v[1] < 0) {
                set_error("line %llu: the size line must start with two non-negative integers (rows cols)",
                          (unsigned long long)h->lines);
                return SGP_B200_ERR_INVALID;
            }
            h->rows = (uint64_t)v[0];
            h->cols = (uint64_t)v[1];
            h->nnz = got > 2 && v[2] > 0 ? (uint64_t)v[2] : 0;
            h->have_size = 1;
            h->body = nl ? e + 1 : e;
            return SGP_B200_OK;
        }
        i = nl ? e + 1 : avail;
    }
    if (!whole) return 1;
    h->body = avail;
    return SGP_B200_OK;
}

// The text source of one call: a host buffer, a device buffer or a file.
struct MtxSource {
    const char *host = nullptr;
    const char *dev = nullptr;
    FILE *f = nullptr;
    uint64_t len = 0;
    std::string prefix;   // head bytes fetched from a file or the device
};

static int fetch_prefix(Context &C, MtxSource &src, uint64_t want, const char **out) {
    if (want > src.len) want = src.len;
    if (src.host) {
        *out = src.host;
        return SGP_B200_OK;
    }
    src.prefix.resize(want);
    if (src.f) {
        if (fseek(src.f, 0, SEEK_SET) != 0 || fread(&src.prefix[0], 1, want, src.f) != want) {
            set_error("short read of the file head");
            return SGP_B200_ERR_INVALID;
        }
    } else if (want) {
        SGPB_CUDA(cudaMemcpyAsync(&src.prefix[0], src.dev, want, cudaMemcpyDeviceToHost, C.stream));
        SGPB_CUDA(cudaStreamSynchronize(C.stream));
    }
    *out = src.prefix.data();
    return SGP_B200_OK;
}

static int read_head(Context &C, MtxSource &src, MtxHead *h) {
    for (uint64_t want = (uint64_t)1 << 16;; want *= 4) {
        const char *t = nullptr;
        const uint64_t avail = want < src.len ? want : src.len;
        SGPB_TRY(fetch_prefix(C, src, avail, &t));
        const int rc = parse_head(t, avail, avail == src.len, h);
        if (rc != 1) return rc;
    }
}

// A process-wide pool of host threads for the staging copies: one core's
// memcpy or pread (5-10 GB/s) is far below the host<->device copy rate, so
// the pinned ring is filled and drained by several.  Jobs run one at a time.
class HostPool {
  public:
    static HostPool &get() {
        // never destroyed: idle workers end with the process.  A forked
        // child has none of the parent's workers, so it builds its own pool
        // (the parent's object is left untouched).
        static std::mutex mu;
        static HostPool *p = nullptr;
        static pid_t owner = 0;
        std::lock_guard<std::mutex> lk(mu);
        if (!p || owner != getpid()) {
            p = new HostPool();
            owner = getpid();
        }
        return *p;
    }
    int width() const { return (int)th_.size() + 1; }
    // fn(k) for every k in [0, parts), on the workers and the calling thread
    void run(int parts, const std::function<void(int)> &fn) {
        std::lock_guard<std::mutex> one(run_mu_);
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &fn;
            parts_ = parts;
            next_.store(0);
            busy_ = (int)th_.size();
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return busy_ == 0; });
        job_ = nullptr;
    }

  private:
    HostPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        const int w = hw > 8 ? 8 : (hw ? (int)hw : 1);
        for (int i = 1; i < w; i++) th_.emplace_back([this] { loop(); });
    }
    void work() {
        for (;;) {
            const int k = next_.fetch_add(1);
            if (k >= parts_) return;
            (*job_)(k);
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> lk(mu_);
            if (--busy_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)> *job_ = nullptr;
    int parts_ = 0, busy_ = 0;
    std::atomic<int> next_{0};
    uint64_t gen_ = 0;
};

// dst[0, n) = src[0, n) in pool-sized pieces of at least 1 MiB
static void par_copy(void *dst, const void *src, size_t n) {
    HostPool &P = HostPool::get();
    const size_t min_piece = (size_t)1 << 20;
    int parts = (int)((n + min_piece - 1) / min_piece);
    if (parts > P.width()) parts = P.width();
    if (parts <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const size_t piece = (n + parts - 1) / parts;
    P.run(parts, [&](int k) {
        const size_t o = (size_t)k * piece;
        if (o < n) memcpy((char *)dst + o, (const char *)src + o, n - o < piece ? n - o : piece);
    });
}

// buf[0, n) = bytes [off, off + n) of file descriptor fd, in parallel pieces
static bool par_pread(int fd, uint8_t *buf, size_t n, uint64_t off) {
    HostPool &P = HostPool::get();
    const size_t min_piece = (size_t)1 << 20;
    int parts = (int)((n + min_piece - 1) / min_piece);
    if (parts > P.width()) parts = P.width();
    if (parts < 1) parts = 1;
    const size_t piece = (n + parts - 1) / parts;
    std::atomic<bool> ok{true};
    P.run(parts, [&](int k) {
        size_t o = (size_t)k * piece;
        const size_t e = o + piece < n ? o + piece : n;
        while (o < e) {
            const ssize_t r = pread(fd, buf + o, e - o, (off_t)(off + o));
            if (r <= 0) {
                ok.store(false);
                return;
            }
            o += (size_t)r;
        }
    });
    return ok.load();
}

static int ensure_stage(Context &C) {
    if (C.h_stage) return SGP_B200_OK;
    SGPB_CUDA(cudaMallocHost((void **)&C.h_stage, kStageSlots * kStageSlotBytes));
    C.h_stage_slot = kStageSlotBytes;
    for (int i = 0; i < kStageSlots; i++) SGPB_CUDA(cudaEventCreateWithFlags(&C.stage_ev[i], cudaEventDisableTiming));
    return SGP_B200_OK;
}

static bool is_pinned(const void *p) {
    cudaPointerAttributes at;
    const bool pinned = cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return pinned;
}

// The whole text into `dtext` (capacity >= len): pinned host memory and device
// memory in one copy; pageable memory and files through the pinned ring, the
// fill of one slot (by the host pool) overlapping the copies of the others.
static int upload_text(Context &C, MtxSource &src, uint8_t *dtext) {
    if (src.dev) {
        SGPB_CUDA(cudaMemcpyAsync(dtext, src.dev, src.len, cudaMemcpyDeviceToDevice, C.stream));
        return SGP_B200_OK;
    }
    if (src.host && is_pinned(src.host)) {
        SGPB_CUDA(cudaMemcpyAsync(dtext, src.host, src.len, cudaMemcpyHostToDevice, C.stream));
        return SGP_B200_OK;
    }
    SGPB_TRY(ensure_stage(C));
    int slot = 0;
    for (uint64_t off = 0; off < src.len; off += C.h_stage_slot, slot = (slot + 1) % kStageSlots) {
        const size_t n = (size_t)(src.len - off < C.h_stage_slot ? src.len - off : C.h_stage_slot);
        uint8_t *buf = C.h_stage + (size_t)slot * C.h_stage_slot;
        SGPB_CUDA(cudaEventSynchronize(C.stage_ev[slot]));
        if (src.f) {
            if (!par_pread(fileno(src.f), buf, n, off)) {
                set_error("short read at byte %llu", (unsigned long long)off);
                return SGP_B200_ERR_INVALID;
            }
        } else {
            par_copy(buf, src.host + off, n);
        }
        SGPB_CUDA(cudaMemcpyAsync(dtext + off, buf, n, cudaMemcpyHostToDevice, C.stream));
        SGPB_CUDA(cudaEventRecord(C.stage_ev[slot], C.stream));
    }
    return SGP_B200_OK;
}

// Device -> pageable host through the pinned ring: the copy of one slot out
// (by the host pool) overlaps the transfers into the others.
struct CopySeg {
    void *dst;
    const void *src;
    size_t bytes;
};
static int download_staged(Context &C, const CopySeg *segs, int nseg) {
    SGPB_TRY(ensure_stage(C));
    struct Chunk {
        char *dst;
        const char *src;
        size_t n;
    };
    std::vector<Chunk> ch;
    for (int i = 0; i < nseg; i++)
        for (size_t o = 0; o < segs[i].bytes; o += C.h_stage_slot)
            ch.push_back({(char *)segs[i].dst + o, (const char *)segs[i].src + o,
                          segs[i].bytes - o < C.h_stage_slot ? segs[i].bytes - o : C.h_stage_slot});
    const int K = (int)ch.size();
    auto issue = [&](int k) -> int {
        const int slot = k % kStageSlots;
        SGPB_CUDA(cudaMemcpyAsync(C.h_stage + (size_t)slot * C.h_stage_slot, ch[k].src, ch[k].n,
                                  cudaMemcpyDeviceToHost, C.stream));
        SGPB_CUDA(cudaEventRecord(C.stage_ev[slot], C.stream));
        return SGP_B200_OK;
    };
    for (int k = 0; k < K && k < kStageSlots; k++) SGPB_TRY(issue(k));
    for (int k = 0; k < K; k++) {
        const int slot = k % kStageSlots;
        SGPB_CUDA(cudaEventSynchronize(C.stage_ev[slot]));
        par_copy(ch[k].dst, C.h_stage + (size_t)slot * C.h_stage_slot, ch[k].n);
        if (k + kStageSlots < K) SGPB_TRY(issue(k + kStageSlots));
    }
    return SGP_B200_OK;
}

// One text line at byte `off` (for messages about later banner lines).
static int fetch_line(Context &C, MtxSource &src, const uint8_t *dtext, uint64_t off, std::string *line) {
    uint64_t n = src.len - off < 4096 ? src.len - off : 4096;
    line->assign(n, '\0');
    if (src.host) {
        memcpy(&(*line)[0], src.host + off, n);
    } else if (n) {
        SGPB_CUDA(cudaMemcpyAsync(&(*line)[0], dtext + off, n, cudaMemcpyDeviceToHost, C.stream));
        SGPB_CUDA(cudaStreamSynchronize(C.stream));
    }
    const size_t e = line->find('\n');
    if (e != std::string::npos) line->resize(e);
    return SGP_B200_OK;
}

// Host arrays the caller frees with free(): large ones 2 MiB aligned and
// advised for transparent huge pages, so that the first touch by the copy-out
// faults once per 2 MiB instead of once per 4 KiB page.
static void *host_alloc_large(size_t bytes) {
    const size_t huge = (size_t)2 << 20;
    if (bytes < 4 * huge) return malloc(bytes);
    const size_t rounded = (bytes + huge - 1) / huge * huge;
    void *p = aligned_alloc(huge, rounded);
    if (p) madvise(p, rounded, MADV_HUGEPAGE);   // advisory: ignored where huge pages are off
    return p;
}

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static uint32_t grid_for(Context &C, uint64_t items, uint32_t per_block) {
    uint64_t g = (items + per_block - 1) / per_block;
    const uint64_t cap = (uint64_t)C.num_sms * 16;
    if (g > cap) g = cap;
    return g ? (uint32_t)g : 1u;
}

static int copy_out(Context &C, uint32_t n, uint64_t m, const uint32_t *rp, const uint32_t *col, int out_mem,
                    sgp_b200_graph_t *out) {
    uint32_t *orp = nullptr, *ocol = nullptr;
    const size_t brp = sizeof(uint32_t) * ((size_t)n + 1), bcol = sizeof(uint32_t) * (m ? m : 1);
    if (out_mem == SGP_B200_DEVICE) {
        // from the device's stream-ordered pool, which keeps freed memory
        // mapped (sgp_b200_create): a repeated conversion does not map and
        // unmap half a gigabyte per call.  cudaFree in sgp_b200_graph_free
        // returns it to the pool.
        cudaError_t e1 = cudaMallocAsync((void **)&orp, brp, C.stream);
        cudaError_t e2 = cudaMallocAsync((void **)&ocol, bcol, C.stream);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            if (orp) cudaFreeAsync(orp, C.stream);
            if (ocol) cudaFreeAsync(ocol, C.stream);
            set_error("device allocation of the output graph failed");
            return SGP_B200_ERR_DEVICE;
        }
    } else {
        orp = (uint32_t *)host_alloc_large(brp);
        ocol = (uint32_t *)host_alloc_large(bcol);
        if (!orp || !ocol) {
            free(orp);
            free(ocol);
            set_error("host allocation of the output graph failed");
            return SGP_B200_ERR_INVALID;
        }
    }
    int rc = SGP_B200_OK;
    if (out_mem == SGP_B200_DEVICE) {
        cudaError_t e = cudaMemcpyAsync(orp, rp, brp, cudaMemcpyDeviceToDevice, C.stream);
        if (e == cudaSuccess && m) e = cudaMemcpyAsync(ocol, col, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, C.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(C.stream);
        if (e != cudaSuccess) {
            set_error("CUDA error copying the output graph: %s", cudaGetErrorString(e));
            rc = SGP_B200_ERR_DEVICE;
        }
    } else {
        const CopySeg segs[2] = {{orp, rp, brp}, {ocol, col, sizeof(uint32_t) * m}};
        rc = download_staged(C, segs, m ? 2 : 1);
    }
    if (rc != SGP_B200_OK) {
        if (out_mem == SGP_B200_DEVICE) {
            cudaFreeAsync(orp, C.stream);
            cudaFreeAsync(ocol, C.stream);
            cudaStreamSynchronize(C.stream);
        } else {
            free(orp);
            free(ocol);
        }
        return rc;
    }
    out->n = n;
    out->m = m;
    out->row_ptr = orp;
    out->col = ocol;
    out->w = nullptr;
    out->mem = out_mem;
    return SGP_B200_OK;
}

static int mtx_impl(Context &C, MtxSource &src, int out_mem, sgp_b200_graph_t *out, sgp_b200_mtx_info_t *info) {
    const double t_start = now_ms();
    const uint32_t launches0 = C.kernel_launches;
    sgp_b200_mtx_info_t I;
    memset(&I, 0, sizeof(I));
    MtxHead h;
    SGPB_TRY(read_head(C, src, &h));
    uint64_t nv = 0, shift = 0;
    int drop_loops = 1;
    if (h.have_size) {
        if (!h.general && h.rows != h.cols) {
            set_error("line %llu: a symmetric matrix needs rows == cols (got %llu x %llu)",
                      (unsigned long long)h.lines, (unsigned long long)h.rows, (unsigned long long)h.cols);
            return SGP_B200_ERR_INVALID;
        }
        if (h.rows == h.cols) {
            nv = h.rows;
        } else {
            nv = h.rows + h.cols;
            shift = h.cols;
            drop_loops = 0;
            I.bipartite = 1;
        }
    }
    if (nv >= 0xFFFFFFFFull || h.rows >= 0xFFFFFFFFull || h.cols >= 0xFFFFFFFFull) {
        set_error("%llu vertices do not fit 32-bit ids", (unsigned long long)nv);
        return SGP_B200_ERR_TOO_LARGE;
    }
    const uint32_t n = (uint32_t)nv;
    I.rows = h.rows;
    I.cols = h.cols;
    I.entries_declared = h.nnz;
    I.n_all = n;

    // 1. text to the device
    const uint64_t len = src.len;
    const bool any_lines = h.have_size && h.body < len;
    const uint64_t lo = h.body ? h.body - 1 : 0;
    uint64_t t0 = 0, ntiles = 0;
    if (any_lines) {
        t0 = lo / kMtxTile;
        ntiles = (len - 2) / kMtxTile - t0 + 1;   // tiles holding positions lo .. len-2
        if (ntiles >= 0x7FFFFFFFull) {
            set_error("file too large (%llu bytes)", (unsigned long long)len);
            return SGP_B200_ERR_TOO_LARGE;
        }
    }
    const uint64_t cap = (len / kMtxTile + 2) * kMtxTile;   // whole tiles plus one tile of zeros
    uint8_t *dtext;
    SGPB_TRY(dalloc_t(C, &dtext, cap));
    SGPB_TRY(dzero(C, dtext + len, cap - len));
    SGPB_TRY(upload_text(C, src, dtext));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    const double t_read = now_ms();
    I.ms_read = (float)(t_read - t_start);

    cudaEvent_t ev[5];
    for (auto &e : ev) SGPB_CUDA(cudaEventCreate(&e));
    struct EvGuard {
        cudaEvent_t *e;
        ~EvGuard() {
            for (int i = 0; i < 5; i++) cudaEventDestroy(e[i]);
        }
    } guard{ev};
    SGPB_CUDA(cudaEventRecord(ev[0], C.stream));

    // 2-3. line starts, parse, degrees
    // key layout: b = bit length of n, so every id (< n <= 2^b - 1) and every
    // key stays below kNoKey in the sorted 2b bits
    int kb = 1;
    while (kb < 32 && ((uint64_t)1 << kb) <= (uint64_t)n) kb++;
    unsigned long long *keys = nullptr;
    uint32_t *valid;
    SGPB_TRY(dalloc_t(C, &valid, 1));
    SGPB_TRY(dzero(C, valid, 4));
    unsigned long long *flags;   // [0] err, [1] banner count, [2..] banner offsets
    SGPB_TRY(dalloc_t(C, &flags, 2 + kMaxBanners));
    SGPB_TRY(dzero(C, flags, sizeof(unsigned long long) * (2 + kMaxBanners)));
    SGPB_CUDA(cudaMemsetAsync(flags, 0xFF, sizeof(unsigned long long), C.stream));
    uint32_t nl = 0;
    if (any_lines) {
        MtxScan s{dtext, len, lo, t0};
        uint32_t *tcnt, *tbase, *ovf;
        SGPB_TRY(dalloc_t(C, &tcnt, ntiles + 1));
        SGPB_TRY(dalloc_t(C, &tbase, ntiles + 1));
        SGPB_TRY(dalloc_t(C, &ovf, 1));
        SGPB_TRY(dzero(C, ovf, 4));
        k_mtx_count<<<(uint32_t)ntiles, kMtxThreads, 0, C.stream>>>(s, tcnt);
        SGPB_CUDA(cudaGetLastError());
        SGPB_TRY(scan_u32(C, tcnt, tbase, (uint32_t)ntiles, ovf));
        uint32_t r[1];
        SGPB_TRY(read_u32(C, ovf, r));
        if (r[0]) {
            set_error("more than 2^32 - 1 lines");
            return SGP_B200_ERR_TOO_LARGE;
        }
        SGPB_TRY(read_u32(C, tbase + ntiles, &nl));
        if ((uint64_t)nl * 2 >= 0xFFFFFFFFull) {
            set_error("more than 2^32 - 1 directed entries");
            return SGP_B200_ERR_TOO_LARGE;
        }
        SGPB_TRY(dalloc_t(C, &keys, (size_t)2 * nl + 2));
        MtxParse a;
        a.s = s;
        a.tile_base = tbase;
        a.rows = (uint32_t)h.rows;
        a.cols = (uint32_t)h.cols;
        a.shift = (uint32_t)shift;
        a.drop_loops = drop_loops;
        a.keys = keys;
        a.b = kb;
        a.valid = valid;
        a.err = flags;
        a.banner = flags + 1;
        k_mtx_parse<<<(uint32_t)ntiles, kMtxThreads, 0, C.stream>>>(a);
        SGPB_CUDA(cudaGetLastError());
        C.kernel_launches += 2;
        uint64_t fl[2 + kMaxBanners];
        SGPB_TRY(read_u64(C, (const uint64_t *)flags, (uint64_t *)fl, 2 + kMaxBanners));
        if (fl[0] != ~0ull) {
            static const char *why[] = {"", "is not \"i j ...\" with unsigned ids", "has an id of 0",
                                        "has an id beyond the size line"};
            const uint32_t code = (uint32_t)(fl[0] & 0xFF);
            set_error("line %llu %s", (unsigned long long)(h.lines + (fl[0] >> 8) + 1), why[code < 4 ? code : 0]);
            return SGP_B200_ERR_INVALID;
        }
        if (fl[1] > (uint64_t)kMaxBanners) {
            set_error("%llu banner lines after the size line", (unsigned long long)fl[1]);
            return SGP_B200_ERR_INVALID;
        }
        for (uint64_t b = 0; b < fl[1]; b++) {
            std::string line;
            SGPB_TRY(fetch_line(C, src, dtext, fl[2 + b], &line));
            int general = 0;
            SGPB_TRY(check_banner(line.data(), line.size(), 0, &general));
            if (general && !I.bipartite) {
                set_error("a banner after the size line switches to \"general\": %s", line.c_str());
                return SGP_B200_ERR_INVALID;
            }
        }
    }
    I.lines = nl;
    SGPB_CUDA(cudaEventRecord(ev[1], C.stream));

    // 4. rows: one radix sort of all keys (the kNoKey of skipped lines sort
    // last and are cut off), then run heads
    uint32_t nvalid = 0;
    SGPB_TRY(read_u32(C, valid, &nvalid));
    const uint64_t cnt = 2ull * nvalid;
    uint32_t *rp, *col, *rows;
    SGPB_TRY(dalloc_t(C, &rp, (size_t)n + 1));
    SGPB_TRY(dalloc_t(C, &rows, (size_t)n + 1));
    SGPB_TRY(dzero(C, rows, sizeof(uint32_t) * ((size_t)n + 1)));
    uint32_t m_all = 0;
    if (cnt) {
        unsigned long long *tmp;
        SGPB_TRY(dalloc_t(C, &tmp, (size_t)2 * nl + 2));
        bool in_tmp = false;
        SGPB_TRY(radix_sort_keys(C, keys, 2ull * nl, 2 * kb, tmp, &in_tmp));
        const unsigned long long *sk = in_tmp ? tmp : keys;
        uint32_t *head, *pos;
        SGPB_TRY(dalloc_t(C, &head, (size_t)cnt + 1));
        SGPB_TRY(dalloc_t(C, &pos, (size_t)cnt + 1));
        k_mtx_heads<<<grid_for(C, cnt, 256), 256, 0, C.stream>>>(cnt, sk, head);
        SGPB_TRY(scan_u32(C, head, pos, (uint32_t)cnt, nullptr));
        SGPB_TRY(read_u32(C, pos + cnt, &m_all));
        SGPB_TRY(dalloc_t(C, &col, (size_t)m_all + 1));
        k_mtx_emit<<<grid_for(C, cnt, 256), 256, 0, C.stream>>>(cnt, sk, head, pos, kb, col, rows);
        SGPB_CUDA(cudaGetLastError());
        C.kernel_launches += 2;
    } else {
        SGPB_TRY(dalloc_t(C, &col, 1));
    }
    SGPB_TRY(scan_u32(C, rows, rp, n, nullptr));
    I.m_all = m_all;
    SGPB_CUDA(cudaEventRecord(ev[2], C.stream));

    // 5-6. components
    uint32_t lcc_root = 0, lcc_n = n;
    if (n) {
        uint32_t *parent, *size, *cc;   // cc: [0] error, [1] components
        unsigned long long *best;
        SGPB_TRY(dalloc_t(C, &parent, (size_t)n + 1));
        SGPB_TRY(dalloc_t(C, &size, (size_t)n + 1));
        SGPB_TRY(dalloc_t(C, &cc, 2));
        SGPB_TRY(dalloc_t(C, &best, 1));
        SGPB_TRY(dzero(C, size, sizeof(uint32_t) * ((size_t)n + 1)));
        SGPB_TRY(dzero(C, cc, 8));
        SGPB_TRY(dzero(C, best, 8));
        // sampling (two neighbour rounds), the largest sampled component,
        // then the remaining entries of the vertices outside it
        constexpr uint32_t kRounds = 2, kProbe = 1024;
        k_cc_init<<<grid_for(C, n, 256), 256, 0, C.stream>>>(n, parent);
        for (uint32_t r = 0; r < kRounds; r++)
            k_cc_sample<<<grid_for(C, n, 256), 256, 0, C.stream>>>(n, rp, col, parent, r, cc);
        k_cc_compress<<<grid_for(C, n, 256), 256, 0, C.stream>>>(n, parent);
        const uint32_t probes = n < kProbe ? n : kProbe;
        k_cc_probe<<<cdiv(probes, 256), 256, 0, C.stream>>>(n, probes, parent, size);
        SGPB_CUDA(cudaGetLastError());
        std::vector<uint32_t> lab(probes);
        SGPB_TRY(read_u32(C, size, lab.data(), (int)probes));
        std::sort(lab.begin(), lab.end());
        uint32_t skip = lab[0], run = 0, best_run = 0;
        for (uint32_t i = 0; i < probes; i++) {
            run = (i > 0 && lab[i] == lab[i - 1]) ? run + 1 : 1;
            if (run > best_run) {
                best_run = run;
                skip = lab[i];
            }
        }
        SGPB_TRY(dzero(C, size, sizeof(uint32_t) * ((size_t)n + 1)));
        const double avg = (double)m_all / n;
        if (avg <= 4)
            k_cc_rest<4><<<grid_for(C, (uint64_t)n * 4, 256), 256, 0, C.stream>>>(n, rp, col, parent, skip, kRounds, cc);
        else if (avg <= 16)
            k_cc_rest<16><<<grid_for(C, (uint64_t)n * 16, 256), 256, 0, C.stream>>>(n, rp, col, parent, skip, kRounds,
                                                                                   cc);
        else
            k_cc_rest<32><<<grid_for(C, (uint64_t)n * 32, 256), 256, 0, C.stream>>>(n, rp, col, parent, skip, kRounds,
                                                                                   cc);
        C.kernel_launches += 4 + kRounds;   // init, samples, compress, probe, rest
        k_cc_flatten<<<grid_for(C, n, 256), 256, 0, C.stream>>>(n, parent, size);
        k_cc_best<<<grid_for(C, n, 256), 256, 0, C.stream>>>(n, parent, size, best, cc + 1);
        SGPB_CUDA(cudaGetLastError());
        C.kernel_launches += 2;
        uint32_t ccv[2];
        uint64_t bk = 0;
        SGPB_TRY(read_u32(C, cc, ccv, 2));
        SGPB_TRY(read_u64(C, (const uint64_t *)best, &bk));
        if (ccv[0]) {
            set_error("union-find retry guard exceeded");
            return SGP_B200_ERR_DEVICE;
        }
        I.components = ccv[1];
        lcc_n = (uint32_t)(bk >> 32);
        lcc_root = 0xFFFFFFFFu - (uint32_t)(bk & 0xFFFFFFFFu);
        SGPB_CUDA(cudaEventRecord(ev[3], C.stream));

        // 7. extraction
        if (lcc_n < n) {
            uint32_t *keep, *len_, *map, *off, *orp, *ocol;
            SGPB_TRY(dalloc_t(C, &keep, (size_t)n + 1));
            SGPB_TRY(dalloc_t(C, &len_, (size_t)n + 1));
            SGPB_TRY(dalloc_t(C, &map, (size_t)n + 1));
            SGPB_TRY(dalloc_t(C, &off, (size_t)n + 1));
            k_lcc_mark<<<grid_for(C, n, 256), 256, 0, C.stream>>>(n, rp, parent, lcc_root, keep, len_);
            SGPB_TRY(scan_u32(C, keep, map, n, nullptr));
            SGPB_TRY(scan_u32(C, len_, off, n, nullptr));
            uint32_t mm = 0;
            SGPB_TRY(read_u32(C, off + n, &mm));
            SGPB_TRY(dalloc_t(C, &orp, (size_t)lcc_n + 1));
            SGPB_TRY(dalloc_t(C, &ocol, (size_t)mm + 1));
            k_lcc_fill<<<grid_for(C, (uint64_t)n * 32, 256), 256, 0, C.stream>>>(n, rp, col, parent, lcc_root, map, off,
                                                                               orp, ocol);
            SGPB_CUDA(cudaMemcpyAsync(orp + lcc_n, off + n, 4, cudaMemcpyDeviceToDevice, C.stream));
            SGPB_CUDA(cudaGetLastError());
            C.kernel_launches += 2;
            rp = orp;
            col = ocol;
            I.m = mm;
        } else {
            I.m = m_all;
        }
    } else {
        I.m = 0;
        SGPB_CUDA(cudaEventRecord(ev[3], C.stream));
    }
    I.n = lcc_n;
    SGPB_CUDA(cudaEventRecord(ev[4], C.stream));
    SGPB_CUDA(cudaEventSynchronize(ev[4]));
    cudaEventElapsedTime(&I.ms_parse, ev[0], ev[1]);
    cudaEventElapsedTime(&I.ms_rows, ev[1], ev[2]);
    cudaEventElapsedTime(&I.ms_components, ev[2], ev[3]);
    cudaEventElapsedTime(&I.ms_extract, ev[3], ev[4]);

    const double t_out = now_ms();
    SGPB_TRY(copy_out(C, lcc_n, I.m, rp, col, out_mem, out));
    const double t_end = now_ms();
    I.ms_out = (float)(t_end - t_out);
    I.ms_total = (float)(t_end - t_start);
    I.kernel_launches = C.kernel_launches - launches0;
    if (info) *info = I;
    return SGP_B200_OK;
}

static int mtx_entry(sgp_b200_ctx_t *x, MtxSource &src, int out_mem, sgp_b200_graph_t *out,
                     sgp_b200_mtx_info_t *info) {
    Context *C = ctx_get(x);
    if (!C || !out) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    if (out_mem != SGP_B200_HOST && out_mem != SGP_B200_DEVICE) {
        set_error("out_mem must be SGP_B200_HOST or SGP_B200_DEVICE");
        return SGP_B200_ERR_INVALID;
    }
    memset(out, 0, sizeof(*out));
    cudaSetDevice(C->device);
    int rc = mtx_impl(*C, src, out_mem, out, info);
    release_all(*C);
    return rc;
}

}  // namespace sgpb

using namespace sgpb;

extern "C" {

int sgp_b200_mtx_parse(sgp_b200_ctx_t *x, const char *text, uint64_t len, int text_mem, int out_mem,
                       sgp_b200_graph_t *out, sgp_b200_mtx_info_t *info) {
    if (!text && len) {
        set_error("null text");
        return SGP_B200_ERR_INVALID;
    }
    if (text_mem != SGP_B200_HOST && text_mem != SGP_B200_DEVICE) {
        set_error("text_mem must be SGP_B200_HOST or SGP_B200_DEVICE");
        return SGP_B200_ERR_INVALID;
    }
    MtxSource src;
    static const char empty[1] = {0};
    if (text_mem == SGP_B200_DEVICE && len) src.dev = text;
    else src.host = len ? text : empty;
    src.len = len;
    return mtx_entry(x, src, out_mem, out, info);
}

int sgp_b200_mtx_read(sgp_b200_ctx_t *x, const char *path, int out_mem, sgp_b200_graph_t *out,
                      sgp_b200_mtx_info_t *info) {
    if (!path) {
        set_error("null path");
        return SGP_B200_ERR_INVALID;
    }
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error("could not open input file %s", path);
        return SGP_B200_ERR_INVALID;
    }
    struct stat st;
    if (fstat(fileno(f), &st) != 0 || st.st_size < 0) {
        fclose(f);
        set_error("could not stat %s", path);
        return SGP_B200_ERR_INVALID;
    }
    MtxSource src;
    src.f = f;
    src.len = (uint64_t)st.st_size;
    int rc = mtx_entry(x, src, out_mem, out, info);
    fclose(f);
    return rc;
}

void sgp_b200_graph_free(sgp_b200_graph_t *g) {
    if (!g) return;
    if (g->mem == SGP_B200_DEVICE) {
        cudaFree((void *)g->row_ptr);
        cudaFree((void *)g->col);
        cudaFree((void *)g->w);
    } else {
        free((void *)g->row_ptr);
        free((void *)g->col);
        free((void *)g->w);
    }
    g->row_ptr = g->col = g->w = nullptr;
    g->n = 0;
    g->m = 0;
}

int sgp_b200_csr_write(const char *path, const sgp_b200_graph_t *g, int id_bytes) {
    if (!path || !g || (g->n && !g->row_ptr) || (g->m && !g->col)) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    if (g->mem != SGP_B200_HOST || (id_bytes != 4 && id_bytes != 8)) {
        set_error("sgp_b200_csr_write takes a host graph and id_bytes 4 or 8");
        return SGP_B200_ERR_INVALID;
    }
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error("could not open output CSR file %s", path);
        return SGP_B200_ERR_INVALID;
    }
    const int64_t hdr[6] = {(int64_t)g->n, (int64_t)g->m, 1, 0, 1, 0};
    bool ok = fwrite(hdr, sizeof(int64_t), 6, f) == 6;
    const uint32_t zero = 0;
    const uint32_t *rp = g->n || g->row_ptr ? g->row_ptr : &zero;
    if (id_bytes == 4) {
        ok = ok && fwrite(rp, 4, (size_t)g->n + 1, f) == (size_t)g->n + 1;
        ok = ok && (g->m == 0 || fwrite(g->col, 4, g->m, f) == g->m);
    } else {
        // widen through a bounded buffer
        const size_t chunk = (size_t)1 << 20;
        uint64_t *buf = (uint64_t *)malloc(chunk * sizeof(uint64_t));
        ok = ok && buf;
        for (int part = 0; part < 2 && ok; part++) {
            const uint32_t *a = part == 0 ? rp : g->col;
            const uint64_t cnt = part == 0 ? (uint64_t)g->n + 1 : g->m;
            for (uint64_t o = 0; o < cnt && ok; o += chunk) {
                const size_t k = (size_t)(cnt - o < chunk ? cnt - o : chunk);
                for (size_t i = 0; i < k; i++) buf[i] = a[o + i];
                ok = fwrite(buf, 8, k, f) == k;
            }
        }
        free(buf);
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) {
        set_error("write to %s failed", path);
        return SGP_B200_ERR_INVALID;
    }
    return SGP_B200_OK;
}

int sgp_b200_mtx2csr(sgp_b200_ctx_t *x, const char *mtx_path, const char *csr_path, int id_bytes,
                     sgp_b200_mtx_info_t *info) {
    if (!csr_path || (id_bytes != 4 && id_bytes != 8)) {
        set_error("csr_path required and id_bytes 4 or 8");
        return SGP_B200_ERR_INVALID;
    }
    sgp_b200_graph_t g;
    SGPB_TRY(sgp_b200_mtx_read(x, mtx_path, SGP_B200_HOST, &g, info));
    int rc = sgp_b200_csr_write(csr_path, &g, id_bytes);
    sgp_b200_graph_free(&g);
    return rc;
}

}  // extern "C"
