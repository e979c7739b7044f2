// internal.h -- host-side plumbing shared by the .cu files of libsgpar_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>

#include "../../include/sgpar_b200.h"

namespace sgpb {

// Error status carried out of the C ABI (sgp_b200_last_error()).
void set_error(const char *fmt, ...);
const char *last_error();

struct Status {
    int code = SGP_B200_OK;
    bool ok() const { return code == SGP_B200_OK; }
};

#define SGPB_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ::sgpb::set_error("CUDA error %s at %s:%d: %s", cudaGetErrorName(e_), __FILE__,     \
                              __LINE__, cudaGetErrorString(e_));                               \
            return SGP_B200_ERR_DEVICE;                                                        \
        }                                                                                      \
    } while (0)

#define SGPB_TRY(call)                                                                         \
    do {                                                                                       \
        int s_ = (call);                                                                       \
        if (s_ != SGP_B200_OK) return s_;                                                      \
    } while (0)

// Stream-ordered device allocations from the device's memory pool; the pool
// keeps freed memory cached so repeated partitions reuse it.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    size_t smem_optin = 0;
    uint64_t *h_pinned = nullptr;   // small pinned staging area for scalar read-backs
    uint8_t *h_stage = nullptr;     // pinned ring for streaming host bytes to the device (mtx.cu)
    size_t h_stage_slot = 0;        // bytes per ring slot
    cudaEvent_t stage_ev[4] = {};   // copy of each slot done
    std::vector<void *> owned;      // allocations released at the end of a call
    std::vector<sgp_b200_ctx_t *> workers;   // contexts of the batch workers (same device), kept across calls
    // timing of the last partition (ms, CUDA events)
    float t_total = 0, t_coarsen = 0, t_eigen = 0, t_split = 0, t_h2d = 0, t_d2h = 0;
    float t_map = 0, t_build = 0;   // coarsening of the last partition: HEC mapping / coarse builds
    uint32_t kernel_launches = 0;
    std::string dev_key;            // device name, SM count and compute capability (autotuner cache key)
    uint32_t grid_cap = 0;          // > 0: at most this many blocks per power-iteration launch
};

Context *ctx_get(sgp_b200_ctx_t *c);

int dalloc(Context &C, void **p, size_t bytes);          // tracked, freed by release_all
template <typename T>
int dalloc_t(Context &C, T **p, size_t count) { return dalloc(C, (void **)p, count * sizeof(T)); }
int dzero(Context &C, void *p, size_t bytes);
void release_all(Context &C);

// device-wide exclusive scan of n uint32 counts into uint32 offsets[n+1]
// (out[n] = total).  Returns SGP_B200_ERR_TOO_LARGE when the total does not
// fit in 32 bits (flag checked on read-back by the caller).
int scan_u32(Context &C, const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *d_overflow);
// stable compaction of indices i in [0, n) with flag(i) != 0 (flags as uint8).
int compact_flags(Context &C, const uint8_t *flags, uint32_t n, uint32_t *out_idx, uint32_t *d_count);

// read a few device scalars (synchronises the stream)
int read_u32(Context &C, const uint32_t *d, uint32_t *h, int count = 1);
int read_u64(Context &C, const uint64_t *d, uint64_t *h, int count = 1);
// Round or iteration budget of a coarsening construction whose natural bound
// (a progress argument) is `natural`: that bound, clamped to 32 bits, or the
// smaller positive value of the environment variable SGPB_ROUND_CAP -- a test
// hook that makes the give-up path (SGP_B200_ERR_BUDGET) reachable; it never
// raises a bound.
uint32_t round_budget(uint64_t natural);

inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// --------------------------------------------------------------- levels --
// One level of the hierarchy on the device.  wbytes: 0 = unit weights,
// 4 = uint32, 8 = uint64; 1 = uint8 and 2 = uint16 only in the relabelled
// copy a power iteration makes of a level.
struct Level {
    uint32_t n = 0;
    uint64_t m = 0;              // directed entries
    uint32_t *rp = nullptr;
    uint32_t *col = nullptr;
    void *w = nullptr;
    int wbytes = 0;
    int sorted = 0;              // 1: every row ascending by destination (coarse levels)
    uint32_t *vcmap = nullptr;   // this level -> next coarser level
    uint32_t *vtx_w = nullptr;   // vertex weights; null: every vertex weighs 1 (the input level)
    uint32_t *wmax = nullptr;    // device word: the largest 32-bit weight (tiered builds), null: unknown
    uint32_t max_deg = 0;
    uint32_t seed_hi = 0, seed_lo = 0;
    int hec_rounds = 0;
    uint64_t pi_iters = 0;
    float pi_ms = 0;
    int pi_capped = 0;
    double pi_dot = 0, pi_lambda = 0;
};

// kernels (implemented in hec.cu / build.cu / eigen.cu / split.cu)
int hec_map_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *vcmap,
                  uint32_t *hn_out, uint32_t *nc_out, int *rounds_out);
int build_coarse_level(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, int out_wbytes,
                       Level *out);
// Vertex weights of the coarse level of F under vcmap: the sum of the fine
// vertex weights of each aggregate (coarsen_kokkos.h:1098), into *out (nc
// entries, allocated here).
int coarse_vertex_weights(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, uint32_t **out);
// the alternative coarseners (coarsen_alt.cu): heavy-edge matching, and the
// MIS-2 (gosh false) / GOSH (gosh true) aggregations
int match_map_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out,
                    int *rounds_out);
// heavy neighbours of a level (hec.cu) and the HEC_V3 mapping built on them
int hec_hn_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *hn);
int hec_v3_map_level(Context &C, const Level &L, int random_level, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out);
int hec_map_from_hn(Context &C, uint32_t n, const uint32_t *hn, uint64_t seed, uint32_t *vcmap, bool prefilled,
                    uint32_t *nc_out, int *rounds_out);
int gosh_v2_map_level(Context &C, const Level &L, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out, int *rounds_out);
int set_map_level(Context &C, const Level &L, bool gosh, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out,
                  int *rounds_out);
// Work split of one level's power iteration, chosen per level shape by the
// autotuner (tune.cpp): the SpMV variant (0 CSR streaming, 5 pipelined warp
// rows), the divisor of a warp's cost share above which a row is cut into
// block-shared segments, and the cost units per thread that size the grid.
struct PITune {
    int mode = 5;
    uint32_t heavy_div = 16;
    uint32_t units = 16;
};
// The tuned split cached for level-shape key `key` on the context's device;
// false when none is cached.  Thread-safe; the cache lives for the process
// and in the file SGPB_TUNE_CACHE names (default
// $HOME/.cache/sgpar_b200/pi_tune.txt; an empty value keeps it in memory).
bool tune_lookup(const Context &C, const std::string &key, PITune *t);
void tune_store(const Context &C, const std::string &key, const PITune &t, double ms_best, double ms_rule);
// serialises the tuning of a level shape across host threads (batch workers)
void tune_lock();
void tune_unlock();
// SGPB_AUTOTUNE=0 turns the autotuner off (the built-in rules then decide)
bool autotune_enabled();

// Entries of padding behind the destination and weight arrays of a
// relabelled power-iteration copy: its staged SpMV copies whole chunks of this
// many entries (16-byte aligned), so the last chunk stays in bounds.
constexpr uint32_t kStagePad = 256;

struct PowerIterOpts {
    double tol = 1e-10;
    uint64_t iter_cap = 0;   // 0: the reference's 1e14 / n only
    int mixed = 0;           // 1: FP32 edge-difference SpMV arithmetic, FP64 iterate and reductions
    int allow_relabel = 1;   // skewed levels may iterate on a hub-first relabelled copy
    int normlap = 0;         // refine_alg 1: normalized-Laplacian (lazy random walk) iteration
    uint64_t mid_limit = 0;  // largest cost (m + 8n) of a level on the cluster kernel; 0 = 2^17
    int mid_blocks = 0;       // blocks per cluster of the cluster kernel (2 or 8); 0 = 8
};
struct PowerIterResult {
    uint64_t niter = 0;
    int capped = 0;
    double dot = 0, gb = 0, lambda = 0, resid = 0;
    float kernel_ms = 0;     // cooperative-kernel time (CUDA events)
};
// x_in: coarse vector (prolongated through vcmap when vcmap != null) or the
// initial vector; x_out: n doubles (may alias nothing).
int power_iter_level(Context &C, const Level &L, const double *x_in, const uint32_t *vcmap,
                     double *x_out, const PowerIterOpts &o, PowerIterResult *res, int want_residual);
// |L x - lambda x| / (bound on the spectrum) of a level's result into res->resid
int level_residual(Context &C, const Level &L, const double *x, int normlap, PowerIterResult *res);
// Small levels (one block, the level in shared memory).  A chain is the
// consecutive small levels of one hierarchy, coarsest first: the first reads
// x0 (through its vcmap when set), each later one the previous result through
// its own vcmap.  power_iter_chains runs any number of chains in one launch,
// a block per chain at a time, and fills each level's result.
bool power_iter_small_ok(const Level &L, const PowerIterOpts &o);
struct PIChainLevel {
    const Level *L = nullptr;
    const uint32_t *vcmap = nullptr;   // this level's vertex -> vertex of the vector it starts from
    double *x_out = nullptr;           // L->n doubles
    PowerIterResult res;
};
struct PIChain {
    const double *x0 = nullptr;
    std::vector<PIChainLevel> lev;
};
int power_iter_chains(Context &C, const std::vector<PIChain *> &chains, const PowerIterOpts &o);
// Mid-size levels (a cluster of blocks, the iterate in global memory, one
// cluster barrier per iteration): chains of consecutive such levels, coarsest
// first, one cluster per chain at a time, in one launch.
bool power_iter_mid_ok(const Level &L, const PowerIterOpts &o);
int power_iter_mid_chains(Context &C, const std::vector<PIChain *> &chains, const PowerIterOpts &o);
int split_level(Context &C, const Level &L, const double *evec, int perc_imbalance, uint32_t *part,
                uint64_t *edgecut, uint32_t *n_part0);
int edge_cut_device(Context &C, const Level &L, const uint32_t *part, uint64_t *edgecut);
// the reference's local search after the split (sgpar.h:2080-2170); mid =
// the part-0 size the split left
int local_search_level(Context &C, const Level &L, uint32_t *part, uint32_t mid, uint32_t *swaps_out,
                       uint32_t *part0_out);
// FM passes on a bisection of the finest level (fm.cu); *cut_out = its cut
int fm_refine_level(Context &C, const Level &L, uint32_t *part, uint32_t max_passes, uint64_t *cut_out,
                    uint32_t *passes_out, uint64_t *moves_out);
int count_part0(Context &C, const uint32_t *part, uint32_t n, uint32_t *out);
// map0 / map1 (optional): vertex i of L -> its id in g1 (part 0) / g2
int induced_subgraphs(Context &C, const Level &L, const uint32_t *part, Level *g1, Level *g2,
                      uint32_t **map0 = nullptr, uint32_t **map1 = nullptr);
// stable LSD radix sort by the low `bits` bits of 64-bit keys, 8 bits per
// pass, optional payload; tmp buffers hold n entries; *in_tmp: the result is
// in the tmp buffers (sort.cu)
int radix_sort_keys(Context &C, unsigned long long *keys, uint64_t n, int bits, unsigned long long *keys_tmp,
                    bool *in_tmp);
int radix_sort_pairs_u32(Context &C, unsigned long long *keys, uint32_t *vals, uint64_t n, int bits,
                         unsigned long long *keys_tmp, uint32_t *vals_tmp, bool *in_tmp);
int radix_sort_pairs_u64(Context &C, unsigned long long *keys, unsigned long long *vals, uint64_t n, int bits,
                         unsigned long long *keys_tmp, unsigned long long *vals_tmp, bool *in_tmp);

}  // namespace sgpb
