// driver.cu -- the multilevel path behind the C ABI.
//
// Reference call structure (cmg/sgpar.h:2363-2430, Kokkos branch):
//   sgp_generate_coarse_graphs (coarsen_kokkos.h:1165-1234)
//   sgp_eigensolve            (eigensolve_kokkos.h:1493-1595)
//   sgp_compute_partition     (sgpar.h:1969)
// All three run on the device here; the host only sequences kernels and reads
// back a few scalars per level (coarse vertex / edge counts).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "internal.h"

struct sgp_b200_hierarchy {
    sgpb::Context *C = nullptr;
    std::vector<sgpb::Level> levels;
    std::vector<void *> owned;
};

namespace sgpb {

int build_coarse_into(Context &C, const Level &F, const uint32_t *vcmap, uint32_t nc, int out_wbytes,
                      uint32_t *crp, uint32_t *ccol, void *cw, uint64_t *m_c);

static uint32_t pcg32(uint64_t *state, uint64_t inc) {
    uint64_t old = *state;
    *state = old * 6364136223846793005ULL + (inc | 1);
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}

__global__ void k_sum_u32(const uint32_t *w, uint64_t m, unsigned long long *out) {
    uint64_t s = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        s += w[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, (unsigned long long)s);
}

__global__ void k_check_csr(uint32_t n, uint64_t m, const uint32_t *rp, const uint32_t *col, uint32_t *bad) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && rp[i + 1] < rp[i]) atomicOr(bad, 1u);
    if (i == 0 && (rp[0] != 0 || rp[n] != m)) atomicOr(bad, 2u);
    for (uint64_t j = i; j < m; j += (uint64_t)gridDim.x * blockDim.x)
        if (col[j] >= n) { atomicOr(bad, 4u); break; }
}

// Copy (or adopt) the input graph as level 0 and validate it on the device.
static int stage_input(Context &C, const sgp_b200_graph_t *g, Level *L0) {
    if (!g || g->n == 0) {
        set_error("empty graph");
        return SGP_B200_ERR_INVALID;
    }
    if (g->m > 0xFFFFFFFFull) {
        set_error("graph has %llu directed entries; 32-bit offsets hold at most 4294967295",
                  (unsigned long long)g->m);
        return SGP_B200_ERR_TOO_LARGE;
    }
    if (!g->row_ptr || (g->m && !g->col)) {
        set_error("null CSR arrays");
        return SGP_B200_ERR_INVALID;
    }
    L0->n = g->n;
    L0->m = g->m;
    L0->wbytes = g->w ? 4 : 0;
    if (g->mem == SGP_B200_DEVICE) {
        L0->rp = (uint32_t *)g->row_ptr;
        L0->col = (uint32_t *)g->col;
        L0->w = (void *)g->w;
    } else {
        SGPB_TRY(dalloc_t(C, &L0->rp, (size_t)g->n + 1));
        SGPB_TRY(dalloc_t(C, &L0->col, (size_t)g->m + 1));
        SGPB_CUDA(cudaMemcpyAsync(L0->rp, g->row_ptr, sizeof(uint32_t) * ((size_t)g->n + 1), cudaMemcpyHostToDevice,
                                  C.stream));
        SGPB_CUDA(cudaMemcpyAsync(L0->col, g->col, sizeof(uint32_t) * g->m, cudaMemcpyHostToDevice, C.stream));
        if (g->w) {
            uint32_t *w;
            SGPB_TRY(dalloc_t(C, &w, (size_t)g->m + 1));
            SGPB_CUDA(cudaMemcpyAsync(w, g->w, sizeof(uint32_t) * g->m, cudaMemcpyHostToDevice, C.stream));
            L0->w = w;
        }
    }
    uint32_t *bad;
    SGPB_TRY(dalloc_t(C, &bad, 1));
    SGPB_TRY(dzero(C, bad, 4));
    uint32_t blocks = cdiv(g->n + 1, 256);
    if (blocks > (uint32_t)C.num_sms * 8) blocks = C.num_sms * 8;
    k_check_csr<<<blocks, 256, 0, C.stream>>>(g->n, g->m, L0->rp, L0->col, bad);
    C.kernel_launches++;
    uint32_t hb = 0;
    SGPB_TRY(read_u32(C, bad, &hb));
    if (hb) {
        set_error("malformed CSR (code %u: 1 = decreasing offsets, 2 = row_ptr[0] != 0 or row_ptr[n] != m, "
                  "4 = destination >= n)", hb);
        return SGP_B200_ERR_INVALID;
    }
    return SGP_B200_OK;
}

static int weight_width(Context &C, const Level &L0, int *wbytes) {
    if (!L0.w) { *wbytes = 4; return SGP_B200_OK; }   // unit weights: total = m < 2^32
    unsigned long long *s;
    SGPB_TRY(dalloc_t(C, &s, 1));
    SGPB_TRY(dzero(C, s, 8));
    uint32_t blocks = (uint32_t)C.num_sms * 8;
    k_sum_u32<<<blocks, 256, 0, C.stream>>>((const uint32_t *)L0.w, L0.m, s);
    C.kernel_launches++;
    uint64_t tot;
    SGPB_TRY(read_u64(C, (const uint64_t *)s, &tot));
    // every coarse weight and weighted degree is a partial sum of the total
    *wbytes = tot <= 0xFFFFFFFFull ? 4 : 8;
    return SGP_B200_OK;
}

// coarsen_kokkos.h:1196-1232: levels while n > cutoff, at most 200; a
// coarsest level below 10 vertices is dropped.
static int generate(Context &C, const Level &L0, uint32_t cutoff, uint64_t *rng_state, uint64_t rng_inc,
                    std::vector<Level> &levels, int coarsener = SGP_B200_COARSEN_HEC) {
    const int kind = coarsener & 15;
    if (kind > SGP_B200_COARSEN_GOSH_V2 || (coarsener & ~(15 | SGP_B200_COARSEN_NONE | SGP_B200_COARSEN_RATIO_STOP))) {
        set_error("coarsener %d: HEC 0, MATCH 1, MIS2 2, GOSH 3, HEC_V3 4 or GOSH_V2 5, optionally | NONE (16) | "
                  "RATIO_STOP (32)", coarsener);
        return SGP_B200_ERR_INVALID;
    }
    levels.clear();
    levels.push_back(L0);
    int out_wbytes = 4;
    SGPB_TRY(weight_width(C, L0, &out_wbytes));
    cudaEvent_t ev[3];
    for (auto &e : ev) SGPB_CUDA(cudaEventCreate(&e));
    struct EvFree {
        cudaEvent_t *e;
        ~EvFree() { for (int i = 0; i < 3; i++) cudaEventDestroy(e[i]); }
    } evfree{ev};
    C.t_map = C.t_build = 0;
    while (!(coarsener & SGP_B200_COARSEN_NONE) && levels.back().n > cutoff) {
        Level &F = levels.back();
        uint32_t hi = pcg32(rng_state, rng_inc);
        uint32_t lo = pcg32(rng_state, rng_inc);
        uint64_t seed = ((uint64_t)hi << 32) | lo;
        F.seed_hi = hi;
        F.seed_lo = lo;
        uint32_t *vcmap;
        SGPB_TRY(dalloc_t(C, &vcmap, F.n));
        uint32_t nc = 0;
        int rounds = 0;
        const int random_level = (levels.size() == 1) && (L0.w == nullptr);
        SGPB_CUDA(cudaEventRecord(ev[0], C.stream));
        if (kind == SGP_B200_COARSEN_HEC)
            SGPB_TRY(hec_map_level(C, F, random_level, seed, vcmap, nullptr, &nc, &rounds));
        else if (kind == SGP_B200_COARSEN_MATCH)
            SGPB_TRY(match_map_level(C, F, random_level, seed, vcmap, &nc, &rounds));
        else if (kind == SGP_B200_COARSEN_HEC_V3)
            SGPB_TRY(hec_v3_map_level(C, F, random_level, seed, vcmap, &nc));
        else if (kind == SGP_B200_COARSEN_GOSH_V2)
            SGPB_TRY(gosh_v2_map_level(C, F, seed, vcmap, &nc, &rounds));
        else
            SGPB_TRY(set_map_level(C, F, kind == SGP_B200_COARSEN_GOSH, seed, vcmap, &nc, &rounds));
        F.vcmap = vcmap;
        F.hec_rounds = rounds;
        SGPB_CUDA(cudaEventRecord(ev[1], C.stream));
        Level Cl;
        SGPB_TRY(build_coarse_level(C, F, vcmap, nc, out_wbytes, &Cl));
        SGPB_TRY(coarse_vertex_weights(C, F, vcmap, nc, &Cl.vtx_w));
        SGPB_CUDA(cudaEventRecord(ev[2], C.stream));
        SGPB_CUDA(cudaEventSynchronize(ev[2]));
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        C.t_map += a;
        C.t_build += b;
        const uint32_t fine_n = F.n;   // F is invalidated by the push
        levels.push_back(Cl);
        if (levels.size() > 200) break;
        if ((coarsener & SGP_B200_COARSEN_RATIO_STOP) && (double)nc / (double)fine_n > 0.9) break;
    }
    if (levels.size() > 1 && levels.back().n < 10) {
        levels.pop_back();
        levels.back().vcmap = nullptr;
    }
    return SGP_B200_OK;
}

__global__ void k_normalize_guess(double *x, uint32_t n) {
    // single block: x /= |x| (eigensolve_kokkos.h:1505)
    __shared__ double sm[64];
    double s[1] = {0};
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s[0] += x[i] * x[i];
    block_sum_d<1>(s, sm);
    if (threadIdx.x == 0) sm[40] = 1.0 / sqrt(s[0]);
    __syncthreads();
    double inv = sm[40];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) x[i] *= inv;
}

// eigensolve_kokkos.h:1493-1595 without FM, in two parts so that a batch can
// run the small and mid-size levels of all its hierarchies in two launches.
// eigen_begin draws and normalises the coarsest guess and plans the chain of
// small levels from the coarsest one up, then the chain of mid-size levels
// above it (the levels stay in `levels`, which must not be resized
// afterwards); the chains run through power_iter_chains and
// power_iter_mid_chains (run_chains); eigen_finish records their results and
// iterates the remaining levels, prolongating down.
struct EigenState {
    double *x0 = nullptr;
    PIChain chain;   // small levels
    PIChain mid;     // mid-size levels, starting from the small chain's result
};

static int eigen_begin(Context &C, std::vector<Level> &levels, uint64_t *rng_state, uint64_t rng_inc,
                       const PowerIterOpts &o, EigenState *E) {
    const int L = (int)levels.size();
    const uint32_t gn = levels[L - 1].n;
    std::vector<double> guess(gn);
    for (uint32_t i = 0; i < gn; i++) guess[i] = ((double)pcg32(rng_state, rng_inc)) / 4294967295.0;
    double *x;
    SGPB_TRY(dalloc_t(C, &x, gn));
    SGPB_CUDA(cudaMemcpyAsync(x, guess.data(), sizeof(double) * gn, cudaMemcpyHostToDevice, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));   // guess lives on the host stack
    k_normalize_guess<<<1, 256, 0, C.stream>>>(x, gn);
    C.kernel_launches++;
    E->x0 = x;
    E->chain.x0 = x;
    E->chain.lev.clear();
    int l = L - 1;
    for (; l >= 0 && power_iter_small_ok(levels[l], o); l--) {
        PIChainLevel cl;
        cl.L = &levels[l];
        cl.vcmap = (l == L - 1) ? nullptr : levels[l].vcmap;
        SGPB_TRY(dalloc_t(C, &cl.x_out, levels[l].n));
        E->chain.lev.push_back(cl);
    }
    E->mid.x0 = E->chain.lev.empty() ? x : E->chain.lev.back().x_out;
    E->mid.lev.clear();
    for (; l >= 0 && power_iter_mid_ok(levels[l], o); l--) {
        PIChainLevel cl;
        cl.L = &levels[l];
        cl.vcmap = (l == L - 1) ? nullptr : levels[l].vcmap;
        SGPB_TRY(dalloc_t(C, &cl.x_out, levels[l].n));
        E->mid.lev.push_back(cl);
    }
    return SGP_B200_OK;
}

// the small-level chains of every hierarchy in one launch, then their
// mid-size chains in another
static int run_chains(Context &C, const std::vector<EigenState *> &es, const PowerIterOpts &o) {
    std::vector<PIChain *> small, mid;
    for (EigenState *e : es) {
        small.push_back(&e->chain);
        mid.push_back(&e->mid);
    }
    SGPB_TRY(power_iter_chains(C, small, o));
    return power_iter_mid_chains(C, mid, o);
}

static int eigen_finish(Context &C, std::vector<Level> &levels, const PowerIterOpts &o, const EigenState &E,
                        double **evec_out, PowerIterResult *finest) {
    const int L = (int)levels.size();
    std::vector<const PIChainLevel *> done;   // chain levels from the coarsest one down
    for (const PIChainLevel &cl : E.chain.lev) done.push_back(&cl);
    for (const PIChainLevel &cl : E.mid.lev) done.push_back(&cl);
    const int nc = (int)done.size();
    for (int k = 0; k < nc; k++) {
        Level &lv = levels[L - 1 - k];
        const PowerIterResult &r = done[k]->res;
        lv.pi_iters = r.niter;
        lv.pi_ms = r.kernel_ms;
        lv.pi_capped = r.capped;
        lv.pi_dot = r.dot;
        lv.pi_lambda = r.lambda;
        if (L - 1 - k == 0) {
            *finest = r;
            SGPB_TRY(level_residual(C, lv, done[k]->x_out, o.normlap, finest));
        }
    }
    const double *xin = nc ? done[nc - 1]->x_out : E.x0;
    for (int l = L - 1 - nc; l >= 0; l--) {
        Level &lv = levels[l];
        double *xo;
        SGPB_TRY(dalloc_t(C, &xo, lv.n));
        PowerIterResult r;
        const uint32_t *vc = (l == L - 1) ? nullptr : lv.vcmap;
        // the finest level runs few iterations from the prolonged vector: a
        // relabelled copy of it would not pay for itself
        PowerIterOpts ol = o;
        ol.allow_relabel = o.allow_relabel && l > 0;
        SGPB_TRY(power_iter_level(C, lv, xin, vc, xo, ol, &r, l == 0));
        lv.pi_iters = r.niter;
        lv.pi_ms = r.kernel_ms;
        lv.pi_capped = r.capped;
        lv.pi_dot = r.dot;
        lv.pi_lambda = r.lambda;
        if (l == 0) *finest = r;
        xin = xo;
    }
    *evec_out = (double *)xin;
    return SGP_B200_OK;
}

static int eigensolve(Context &C, std::vector<Level> &levels, uint64_t *rng_state, uint64_t rng_inc,
                      const PowerIterOpts &o, double **evec_out, PowerIterResult *finest) {
    EigenState E;
    SGPB_TRY(eigen_begin(C, levels, rng_state, rng_inc, o, &E));
    SGPB_TRY(run_chains(C, {&E}, o));
    return eigen_finish(C, levels, o, E, evec_out, finest);
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// One graph between the phases of a partition: its hierarchy, rng state and
// eigensolve plan.
struct Staged {
    std::vector<Level> levels;
    uint64_t st = 0;
    PowerIterOpts po;
    EigenState es;
};

// The path on a staged level 0, in two halves around the run of the small
// levels (partition_staged below for one graph, sgp_b200_partition_batch for
// many).  partition_begin builds the hierarchy and plans the eigensolve;
// partition_end finishes it and splits.  part_d is a device array of L0.n
// entries; the caller copies it out.  ev[0] was recorded before staging (the
// H2D window), ev[1..4] are recorded here.
static int partition_begin(Context &C, const Level &L0, const sgp_b200_options_t *opt, cudaEvent_t *ev, Staged *S,
                           bool batch = false) {
    if (opt->refine_alg != 0 && opt->refine_alg != 1) {
        set_error("refine_alg %d: 0 (shifted combinatorial Laplacian) or 1 (normalized Laplacian)", opt->refine_alg);
        return SGP_B200_ERR_INVALID;
    }
    SGPB_CUDA(cudaEventRecord(ev[1], C.stream));
    S->st = opt->rng_state;
    SGPB_TRY(generate(C, L0, opt->cutoff, &S->st, opt->rng_inc, S->levels, opt->coarsener));
    SGPB_CUDA(cudaEventRecord(ev[2], C.stream));
    S->po.tol = opt->tol;
    S->po.iter_cap = opt->iter_cap;
    S->po.mixed = opt->mixed;
    S->po.normlap = opt->refine_alg == 1;
    // the cluster kernel's share of the levels: up to 2^17 cost units for a
    // single partition (latency), 2^23 in a batch (many levels at once)
    const uint32_t lg = opt->cluster_max_log2 ? (opt->cluster_max_log2 < 40 ? opt->cluster_max_log2 : 40u)
                                              : (batch ? 23u : 17u);
    S->po.mid_limit = 1ull << lg;
    // blocks per cluster: 8 for a single partition, 2 in a batch
    if (opt->cluster_blocks != 0 && opt->cluster_blocks != 2 && opt->cluster_blocks != 8) {
        set_error("options.cluster_blocks must be 0, 2 or 8 (got %u)", opt->cluster_blocks);
        return SGP_B200_ERR_INVALID;
    }
    S->po.mid_blocks = opt->cluster_blocks ? (int)opt->cluster_blocks : (batch ? 2 : 8);
    SGPB_TRY(eigen_begin(C, S->levels, &S->st, opt->rng_inc, S->po, &S->es));
    return SGP_B200_OK;
}

static int partition_end(Context &C, const sgp_b200_options_t *opt, sgp_b200_result_t *res, uint32_t *part_d,
                         cudaEvent_t *ev, Staged &S) {
    std::vector<Level> &levels = S.levels;
    double *evec = nullptr;
    PowerIterResult fin;
    SGPB_TRY(eigen_finish(C, levels, S.po, S.es, &evec, &fin));
    SGPB_CUDA(cudaEventRecord(ev[3], C.stream));
    uint64_t cut = 0;
    uint32_t p0 = 0;
    SGPB_TRY(split_level(C, levels[0], evec, opt->perc_imbalance, part_d, &cut, &p0));
    res->ls_swaps = 0;
    if (opt->local_search_alg) {
        // the part-0 size is the reference's curr_split when the split's
        // sweep range holds at most one vertex (perc_imbalance_allowed 0)
        if (opt->perc_imbalance != 0) {
            set_error("the local search takes perc_imbalance_allowed 0");
            return SGP_B200_ERR_INVALID;
        }
        SGPB_TRY(local_search_level(C, levels[0], part_d, p0, &res->ls_swaps, &p0));
        SGPB_TRY(edge_cut_device(C, levels[0], part_d, &cut));
    }
    res->fm_passes_run = 0;
    res->fm_moves = 0;
    if (opt->fm_passes) {
        SGPB_TRY(fm_refine_level(C, levels[0], part_d, opt->fm_passes, &cut, &res->fm_passes_run, &res->fm_moves));
        SGPB_TRY(count_part0(C, part_d, levels[0].n, &p0));
    }
    SGPB_CUDA(cudaEventRecord(ev[4], C.stream));
    res->edgecut = cut;
    res->part0_size = p0;
    res->lambda = fin.lambda;
    res->residual = fin.resid;
    res->levels = (int)levels.size();
    res->iter_max_reached = 0;
    for (size_t l = 0; l < levels.size() && l < SGP_B200_MAX_LEVELS; l++) {
        res->level_n[l] = levels[l].n;
        res->level_m[l] = levels[l].m;
        res->level_iters[l] = levels[l].pi_iters;
        res->level_hec_rounds[l] = levels[l].hec_rounds;
        res->level_pi_ms[l] = levels[l].pi_ms;
        res->iter_max_reached |= levels[l].pi_capped;
    }
    res->rng_state = S.st;
    return SGP_B200_OK;
}

static int partition_staged(Context &C, const Level &L0, const sgp_b200_options_t *opt, sgp_b200_result_t *res,
                            uint32_t *part_d, cudaEvent_t *ev) {
    Staged S;
    SGPB_TRY(partition_begin(C, L0, opt, ev, &S));
    SGPB_TRY(run_chains(C, {&S.es}, S.po));
    return partition_end(C, opt, res, part_d, ev, S);
}

struct Events {
    cudaEvent_t e[6] = {};
    int create() {
        for (auto &x : e) SGPB_CUDA(cudaEventCreate(&x));
        return SGP_B200_OK;
    }
    ~Events() {
        for (auto &x : e)
            if (x) cudaEventDestroy(x);
    }
};

static void fill_times(Context &C, const Events &E, sgp_b200_result_t *res) {
    res->ms_h2d = ev_ms(E.e[0], E.e[1]);
    res->ms_coarsen = ev_ms(E.e[1], E.e[2]);
    res->ms_eigen = ev_ms(E.e[2], E.e[3]);
    res->ms_split = ev_ms(E.e[3], E.e[4]);
    res->ms_d2h = ev_ms(E.e[4], E.e[5]);
    res->ms_total = ev_ms(E.e[0], E.e[5]);
    res->kernel_launches = C.kernel_launches;
    res->ms_map = C.t_map;
    res->ms_build = C.t_build;
    C.t_total = res->ms_total; C.t_coarsen = res->ms_coarsen; C.t_eigen = res->ms_eigen; C.t_split = res->ms_split;
}

static int partition_impl(Context &C, const sgp_b200_graph_t *g, const sgp_b200_options_t *opt,
                          sgp_b200_result_t *res) {
    Events E;
    SGPB_TRY(E.create());
    C.kernel_launches = 0;
    SGPB_CUDA(cudaEventRecord(E.e[0], C.stream));
    Level L0;
    SGPB_TRY(stage_input(C, g, &L0));
    uint32_t *part_d = (opt->part_mem == SGP_B200_DEVICE) ? res->part : nullptr;
    if (!part_d) SGPB_TRY(dalloc_t(C, &part_d, g->n));
    SGPB_TRY(partition_staged(C, L0, opt, res, part_d, E.e));
    if (opt->part_mem != SGP_B200_DEVICE)
        SGPB_CUDA(cudaMemcpyAsync(res->part, part_d, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaEventRecord(E.e[5], C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    fill_times(C, E, res);
    return SGP_B200_OK;
}

// part4[i] = 2 part[i] + the sub-bisection's label of i in its induced subgraph
__global__ void k_combine4(uint32_t n, const uint32_t *part, const uint32_t *map0, const uint32_t *map1,
                           const uint32_t *pa, const uint32_t *pb, uint32_t *part4) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = part[i];
    const uint32_t s = p == 0 ? (pa ? pa[map0[i]] : 0u) : (pb ? pb[map1[i]] : 0u);
    part4[i] = 2 * p + s;
}

// sgpar.cpp:62-89: bisection, induced subgraphs (sgpar.h:2666-2752), one
// bisection of each with the rng carried along, cut4 = cut + ec1 + ec2.
static int partition4_impl(Context &C, const sgp_b200_graph_t *g, const sgp_b200_options_t *opt, uint32_t *part4,
                           uint64_t out[3]) {
    Events E;
    SGPB_TRY(E.create());
    C.kernel_launches = 0;
    SGPB_CUDA(cudaEventRecord(E.e[0], C.stream));
    Level L0;
    SGPB_TRY(stage_input(C, g, &L0));
    const uint32_t n = g->n;
    sgp_b200_options_t o = *opt;
    o.part_mem = SGP_B200_DEVICE;
    std::vector<sgp_b200_result_t> r(3);
    uint32_t *p;
    SGPB_TRY(dalloc_t(C, &p, n));
    SGPB_TRY(partition_staged(C, L0, &o, &r[0], p, E.e));
    o.rng_state = r[0].rng_state;
    Level sub[2];
    uint32_t *maps[2] = {nullptr, nullptr};
    SGPB_TRY(induced_subgraphs(C, L0, p, &sub[0], &sub[1], &maps[0], &maps[1]));
    uint32_t *sp[2] = {nullptr, nullptr};
    uint64_t ec[2] = {0, 0};
    for (int k = 0; k < 2; k++) {
        if (sub[k].n < 2) continue;   // nothing to bisect
        SGPB_TRY(dalloc_t(C, &sp[k], sub[k].n));
        SGPB_TRY(partition_staged(C, sub[k], &o, &r[k + 1], sp[k], E.e));
        o.rng_state = r[k + 1].rng_state;
        ec[k] = r[k + 1].edgecut;
    }
    uint32_t *p4 = opt->part_mem == SGP_B200_DEVICE ? part4 : nullptr;
    if (!p4) SGPB_TRY(dalloc_t(C, &p4, n));
    k_combine4<<<cdiv(n, 256), 256, 0, C.stream>>>(n, p, maps[0], maps[1], sp[0], sp[1], p4);
    C.kernel_launches++;
    SGPB_CUDA(cudaGetLastError());
    if (opt->part_mem != SGP_B200_DEVICE)
        SGPB_CUDA(cudaMemcpyAsync(part4, p4, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, C.stream));
    SGPB_CUDA(cudaStreamSynchronize(C.stream));
    out[0] = r[0].edgecut;
    out[1] = r[0].edgecut + ec[0] + ec[1];
    out[2] = o.rng_state;
    return SGP_B200_OK;
}

// thread-local default context for the part-1 (sgpar.h) entry points
static thread_local sgp_b200_ctx_t *g_default = nullptr;
static Context *default_ctx() {
    if (!g_default) {
        int dev = 0;
        cudaGetDevice(&dev);
        g_default = sgp_b200_create(dev);
    }
    return g_default ? ctx_get(g_default) : nullptr;
}

static sgp_real_t g_tol = 1e-10;   // sgpar.h:139 SGPAR_POWERITER_TOL

}  // namespace sgpb

using namespace sgpb;

extern "C" {

int change_tol(sgp_real_t new_tol) {
    g_tol = new_tol;
    return 0;
}

void sgp_b200_default_options(sgp_b200_options_t *o) {
    memset(o, 0, sizeof(*o));
    o->cutoff = 50;
    o->tol = g_tol;
    o->mixed = 0;
    o->perc_imbalance = 0;
    o->iter_cap = 0;
    o->rng_state = 0x853c49e6748fea9bULL;
    o->rng_inc = 1;
    o->part_mem = SGP_B200_HOST;
    o->refine_alg = 0;
    o->coarsener = SGP_B200_COARSEN_HEC;
    o->local_search_alg = 0;
    o->fm_passes = 0;
}

int sgp_b200_partition(sgp_b200_ctx_t *x, const sgp_b200_graph_t *g, const sgp_b200_options_t *opt,
                       sgp_b200_result_t *res) {
    Context *C = ctx_get(x);
    if (!C || !g || !opt || !res || !res->part) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    cudaSetDevice(C->device);
    int rc = partition_impl(*C, g, opt, res);
    release_all(*C);
    return rc;
}

int sgp_b200_partition_4way(sgp_b200_ctx_t *x, const sgp_b200_graph_t *g, const sgp_b200_options_t *opt,
                            uint32_t *part4, uint64_t *result4) {
    Context *C = ctx_get(x);
    if (!C || !g || !opt || !part4 || !result4) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    cudaSetDevice(C->device);
    int rc = partition4_impl(*C, g, opt, part4, result4);
    release_all(*C);
    return rc;
}

int sgp_b200_partition_batch(sgp_b200_ctx_t *x, const sgp_b200_graph_t *graphs, int count,
                             const sgp_b200_options_t *opt, sgp_b200_result_t *results, int workers) {
    Context *C = ctx_get(x);
    if (!C || (count > 0 && (!graphs || !results)) || !opt || count < 0) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    for (int i = 0; i < count; i++)
        if (!results[i].part) {
            set_error("results[%d].part is null", i);
            return SGP_B200_ERR_INVALID;
        }
    if (count == 0) return SGP_B200_OK;
    if (workers < 1) workers = 1;
    if (workers > count) workers = count;
    cudaSetDevice(C->device);
    while ((int)C->workers.size() < workers) {
        sgp_b200_ctx_t *w = sgp_b200_create(C->device);
        if (!w) return SGP_B200_ERR_DEVICE;
        C->workers.push_back(w);
    }
    {
        const char *gc = getenv("SGPB_BATCH_GRID");
        for (sgp_b200_ctx_t *w : C->workers) ctx_get(w)->grid_cap = gc ? (uint32_t)atoi(gc) : 0u;
    }
    // largest graphs first (LPT): the workers take the next index of this order
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return graphs[a].m > graphs[b].m; });
    std::atomic<int> first_rc(SGP_B200_OK);
    std::mutex err_mu;
    std::string err;
    auto fail = [&](int i, int rc) {
        int expect = SGP_B200_OK;
        if (first_rc.compare_exchange_strong(expect, rc)) {
            std::lock_guard<std::mutex> lk(err_mu);
            err = std::string("graph ") + std::to_string(i) + ": " + last_error();
        }
    };
    // Waves of up to kWave graphs, three phases each: the workers stage and
    // coarsen every graph of the wave (keeping the hierarchies), one launch
    // iterates the small levels of all of them (a block per hierarchy at a
    // time), then the workers iterate the remaining levels and split.  A
    // graph's results are identical to a single call's: every level runs the
    // same kernels with the same inputs.
    constexpr int kWave = 1024;
    struct Item {
        Events E;
        Level L0;
        Staged S;
        uint32_t *part_d = nullptr;
        uint32_t launches = 0;
        float t_map = 0, t_build = 0;
    };
    int rc_all = SGP_B200_OK;
    // wall time of each phase, summed over the waves (the phases are
    // separated by host synchronisation)
    double ph[3] = {0, 0, 0};
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto ms_since = [](std::chrono::steady_clock::time_point t0) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    for (int w0 = 0; w0 < count && first_rc.load() == SGP_B200_OK; w0 += kWave) {
        const int w1 = count - w0 < kWave ? count : w0 + kWave;
        std::unique_ptr<Item[]> items(new Item[w1 - w0]);
        auto run_phase = [&](auto &&body) {
            std::atomic<int> next(w0);
            auto work = [&](sgp_b200_ctx_t *wx) {
                Context &W = *ctx_get(wx);
                cudaSetDevice(W.device);
                while (first_rc.load() == SGP_B200_OK) {
                    const int k = next.fetch_add(1);
                    if (k >= w1) break;
                    const int i = order[k];
                    const int rc = body(W, items[k - w0], i);
                    if (rc != SGP_B200_OK) fail(i, rc);
                }
                cudaStreamSynchronize(W.stream);
            };
            std::vector<std::thread> th;
            for (int t = 1; t < workers; t++) th.emplace_back(work, C->workers[t]);
            work(C->workers[0]);
            for (auto &t : th) t.join();
        };
        // phase 1: stage, coarsen, draw the coarsest guess
        auto t0 = now();
        run_phase([&](Context &W, Item &it, int i) -> int {
            SGPB_TRY(it.E.create());
            W.kernel_launches = 0;
            SGPB_CUDA(cudaEventRecord(it.E.e[0], W.stream));
            SGPB_TRY(stage_input(W, &graphs[i], &it.L0));
            it.part_d = (opt->part_mem == SGP_B200_DEVICE) ? results[i].part : nullptr;
            if (!it.part_d) SGPB_TRY(dalloc_t(W, &it.part_d, graphs[i].n));
            SGPB_TRY(partition_begin(W, it.L0, opt, it.E.e, &it.S, true));
            it.launches = W.kernel_launches + 2;   // and the shared launches of phase 2
            it.t_map = W.t_map;
            it.t_build = W.t_build;
            return SGP_B200_OK;
        });
        ph[0] += ms_since(t0);
        // phase 2: the small levels of every hierarchy in one launch, then
        // their mid-size levels in another
        t0 = now();
        if (first_rc.load() == SGP_B200_OK) {
            std::vector<EigenState *> es;
            for (int k = 0; k < w1 - w0; k++) es.push_back(&items[k].S.es);
            const int rc = run_chains(*C, es, items[0].S.po);
            if (rc != SGP_B200_OK) fail(order[w0], rc);
        }
        ph[1] += ms_since(t0);
        // phase 3: the remaining levels, the split, the copy-out
        t0 = now();
        if (first_rc.load() == SGP_B200_OK)
            run_phase([&](Context &W, Item &it, int i) -> int {
                sgp_b200_result_t *res = &results[i];
                W.kernel_launches = it.launches;
                SGPB_TRY(partition_end(W, opt, res, it.part_d, it.E.e, it.S));
                if (opt->part_mem != SGP_B200_DEVICE)
                    SGPB_CUDA(cudaMemcpyAsync(res->part, it.part_d, sizeof(uint32_t) * graphs[i].n,
                                              cudaMemcpyDeviceToHost, W.stream));
                SGPB_CUDA(cudaEventRecord(it.E.e[5], W.stream));
                SGPB_CUDA(cudaStreamSynchronize(W.stream));
                W.t_map = it.t_map;
                W.t_build = it.t_build;
                fill_times(W, it.E, res);
                return SGP_B200_OK;
            });
        ph[2] += ms_since(t0);
        for (int t = 0; t < workers; t++) release_all(*ctx_get(C->workers[t]));
        release_all(*C);
    }
    C->t_coarsen = (float)ph[0];
    C->t_eigen = (float)ph[1];
    C->t_split = (float)ph[2];
    C->t_total = (float)(ph[0] + ph[1] + ph[2]);
    if (first_rc.load() != SGP_B200_OK) {
        set_error("%s", err.c_str());
        rc_all = first_rc.load();
    }
    return rc_all;
}

int sgp_b200_last_timing(sgp_b200_ctx_t *x, float *t, float *c, float *e, float *s) {
    Context *C = ctx_get(x);
    if (!C) return SGP_B200_ERR_INVALID;
    if (t) *t = C->t_total;
    if (c) *c = C->t_coarsen;
    if (e) *e = C->t_eigen;
    if (s) *s = C->t_split;
    return 0;
}

// ---------------------------------------------------------- hierarchy --
int sgp_b200_generate_coarse_graphs(sgp_b200_ctx_t *x, const sgp_b200_graph_t *g, uint32_t cutoff,
                                    sgp_pcg32_random_t *rng, sgp_b200_hierarchy_t **out) {
    Context *C = ctx_get(x);
    if (!C || !g || !rng || !out) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    cudaSetDevice(C->device);
    Level L0;
    int rc = stage_input(*C, g, &L0);
    std::vector<Level> levels;
    if (rc == SGP_B200_OK) rc = generate(*C, L0, cutoff, &rng->state, rng->inc, levels);
    if (rc != SGP_B200_OK) {
        release_all(*C);
        return rc;
    }
    cudaStreamSynchronize(C->stream);
    sgp_b200_hierarchy_t *h = new sgp_b200_hierarchy_t();
    h->C = C;
    h->levels = levels;
    h->owned.swap(C->owned);
    *out = h;
    return SGP_B200_OK;
}

int sgp_b200_hierarchy_levels(const sgp_b200_hierarchy_t *h) { return h ? (int)h->levels.size() : 0; }

int sgp_b200_hierarchy_level(const sgp_b200_hierarchy_t *h, int l, uint32_t *n, uint64_t *m, const uint32_t **rp,
                             const uint32_t **col, const void **w, int *wbytes, const uint32_t **vcmap) {
    if (!h || l < 0 || l >= (int)h->levels.size()) {
        set_error("level index out of range");
        return SGP_B200_ERR_INVALID;
    }
    const Level &L = h->levels[l];
    if (n) *n = L.n;
    if (m) *m = L.m;
    if (rp) *rp = L.rp;
    if (col) *col = L.col;
    if (w) *w = L.w;
    if (wbytes) *wbytes = L.wbytes;
    if (vcmap) *vcmap = L.vcmap;
    return SGP_B200_OK;
}

int sgp_b200_hierarchy_vertex_weights(const sgp_b200_hierarchy_t *h, int l, const uint32_t **vtx_w) {
    if (!h || !vtx_w || l < 0 || l >= (int)h->levels.size()) {
        set_error("level index out of range");
        return SGP_B200_ERR_INVALID;
    }
    *vtx_w = h->levels[l].vtx_w;
    return SGP_B200_OK;
}

int sgp_b200_eigensolve(sgp_b200_ctx_t *x, sgp_b200_hierarchy_t *h, sgp_pcg32_random_t *rng, double tol, int mixed,
                        uint64_t iter_cap, double *eigenvec, int mem, sgp_b200_result_t *stats) {
    Context *C = ctx_get(x);
    if (!C || !h || !rng || !eigenvec) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    cudaSetDevice(C->device);
    PowerIterOpts o;
    o.tol = tol;
    o.mixed = mixed;
    o.iter_cap = iter_cap;
    double *ev = nullptr;
    PowerIterResult fin;
    int rc = eigensolve(*C, h->levels, &rng->state, rng->inc, o, &ev, &fin);
    if (rc == SGP_B200_OK) {
        cudaError_t e = cudaMemcpyAsync(eigenvec, ev, sizeof(double) * h->levels[0].n,
                                        mem == SGP_B200_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                        C->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(C->stream);
        if (e != cudaSuccess) {
            set_error("eigenvector copy failed: %s", cudaGetErrorString(e));
            rc = SGP_B200_ERR_DEVICE;
        }
    }
    if (rc == SGP_B200_OK && stats) {
        stats->lambda = fin.lambda;
        stats->residual = fin.resid;
        stats->levels = (int)h->levels.size();
        for (size_t l = 0; l < h->levels.size() && l < SGP_B200_MAX_LEVELS; l++) {
            stats->level_n[l] = h->levels[l].n;
            stats->level_m[l] = h->levels[l].m;
            stats->level_iters[l] = h->levels[l].pi_iters;
            stats->level_pi_ms[l] = h->levels[l].pi_ms;
        }
    }
    release_all(*C);
    return rc;
}

void sgp_b200_hierarchy_free(sgp_b200_hierarchy_t *h) {
    if (!h) return;
    cudaSetDevice(h->C->device);
    for (void *p : h->owned) cudaFreeAsync(p, h->C->stream);
    cudaStreamSynchronize(h->C->stream);
    delete h;
}

// ------------------------------------------------------ kernel entries --
int sgp_b200_hec(sgp_b200_ctx_t *x, uint32_t n, const uint32_t *rp, const uint32_t *col, const void *w, int wbytes,
                 int random_level, uint64_t seed, uint32_t *hn, uint32_t *vcmap, uint32_t *nc, int *rounds) {
    Context *C = ctx_get(x);
    if (!C || !rp || !vcmap || !nc) { set_error("null argument"); return SGP_B200_ERR_INVALID; }
    if (wbytes != 0 && wbytes != 4 && wbytes != 8) { set_error("wbytes must be 0, 4 or 8"); return SGP_B200_ERR_INVALID; }
    cudaSetDevice(C->device);
    Level L;
    L.n = n; L.rp = (uint32_t *)rp; L.col = (uint32_t *)col; L.w = (void *)(wbytes ? w : nullptr);
    L.wbytes = wbytes ? wbytes : 0;
    uint32_t mm = 0;
    int rc = n ? read_u32(*C, rp + n, &mm) : 0;
    L.m = mm;
    int r = 0;
    if (rc == SGP_B200_OK) rc = hec_map_level(*C, L, random_level, seed, vcmap, hn, nc, &r);
    if (rounds) *rounds = r;
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc;
}

int sgp_b200_coarsen_map(sgp_b200_ctx_t *x, uint32_t n, const uint32_t *rp, const uint32_t *col, const void *w,
                         int wbytes, int coarsener, int random_level, uint64_t seed, uint32_t *vcmap, uint32_t *nc,
                         int *rounds) {
    Context *C = ctx_get(x);
    if (!C || !rp || !vcmap || !nc) { set_error("null argument"); return SGP_B200_ERR_INVALID; }
    if (wbytes != 0 && wbytes != 4 && wbytes != 8) { set_error("wbytes must be 0, 4 or 8"); return SGP_B200_ERR_INVALID; }
    if (coarsener < SGP_B200_COARSEN_MATCH || coarsener > SGP_B200_COARSEN_GOSH_V2) {
        set_error("sgp_b200_coarsen_map takes MATCH (1), MIS2 (2), GOSH (3), HEC_V3 (4) or GOSH_V2 (5); HEC is "
                  "sgp_b200_hec");
        return SGP_B200_ERR_INVALID;
    }
    cudaSetDevice(C->device);
    Level L;
    L.n = n; L.rp = (uint32_t *)rp; L.col = (uint32_t *)col; L.w = (void *)(wbytes ? w : nullptr);
    L.wbytes = wbytes ? wbytes : 0;
    uint32_t mm = 0;
    int rc = n ? read_u32(*C, rp + n, &mm) : 0;
    L.m = mm;
    int r = 0;
    if (rc == SGP_B200_OK) {
        if (coarsener == SGP_B200_COARSEN_MATCH) rc = match_map_level(*C, L, random_level, seed, vcmap, nc, &r);
        else if (coarsener == SGP_B200_COARSEN_HEC_V3) rc = hec_v3_map_level(*C, L, random_level, seed, vcmap, nc);
        else if (coarsener == SGP_B200_COARSEN_GOSH_V2) rc = gosh_v2_map_level(*C, L, seed, vcmap, nc, &r);
        else rc = set_map_level(*C, L, coarsener == SGP_B200_COARSEN_GOSH, seed, vcmap, nc, &r);
    }
    if (rounds) *rounds = r;
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc;
}

int sgp_b200_fm_refine(sgp_b200_ctx_t *x, uint32_t n, const uint32_t *rp, const uint32_t *col, uint32_t *part,
                       uint32_t max_passes, uint64_t *cut, uint32_t *passes, uint64_t *moves) {
    Context *C = ctx_get(x);
    if (!C || !rp || !col || !part) { set_error("null argument"); return SGP_B200_ERR_INVALID; }
    cudaSetDevice(C->device);
    Level L;
    L.n = n; L.rp = (uint32_t *)rp; L.col = (uint32_t *)col; L.w = nullptr; L.wbytes = 0;
    uint32_t mm = 0;
    int rc = n ? read_u32(*C, rp + n, &mm) : 0;
    L.m = mm;
    uint64_t c = 0;
    if (rc == SGP_B200_OK) rc = edge_cut_device(*C, L, part, &c);
    if (rc == SGP_B200_OK) rc = fm_refine_level(*C, L, part, max_passes, &c, passes, moves);
    if (rc == SGP_B200_OK && cut) *cut = c;
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc;
}

int sgp_b200_build_coarse(sgp_b200_ctx_t *x, uint32_t n, const uint32_t *rp, const uint32_t *col, const void *w,
                          int wbytes, const uint32_t *vcmap, uint32_t nc, int out_wbytes, uint32_t *crp,
                          uint32_t *ccol, void *cw, uint64_t *m_c) {
    Context *C = ctx_get(x);
    if (!C || !rp || !vcmap || !crp || !ccol || !cw || !m_c) { set_error("null argument"); return SGP_B200_ERR_INVALID; }
    if ((wbytes != 0 && wbytes != 4 && wbytes != 8) || (out_wbytes != 4 && out_wbytes != 8)) {
        set_error("weight widths must be 0/4/8 in and 4/8 out");
        return SGP_B200_ERR_INVALID;
    }
    cudaSetDevice(C->device);
    Level L;
    L.n = n; L.rp = (uint32_t *)rp; L.col = (uint32_t *)col; L.w = (void *)(wbytes ? w : nullptr); L.wbytes = wbytes;
    uint32_t mm = 0;
    int rc = n ? read_u32(*C, rp + n, &mm) : 0;
    L.m = mm;
    if (rc == SGP_B200_OK) rc = build_coarse_into(*C, L, vcmap, nc, out_wbytes, crp, ccol, cw, m_c);
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc;
}

int sgp_b200_power_iter(sgp_b200_ctx_t *x, uint32_t n, const uint32_t *rp, const uint32_t *col, const void *w,
                        int wbytes, const double *x_in, const uint32_t *vcmap, double *x_out, double tol,
                        uint64_t iter_cap, int mixed, uint64_t *niter, double *lambda, double *residual) {
    Context *C = ctx_get(x);
    if (!C || !rp || !x_in || !x_out) { set_error("null argument"); return SGP_B200_ERR_INVALID; }
    if (wbytes != 0 && wbytes != 4 && wbytes != 8) { set_error("wbytes must be 0, 4 or 8"); return SGP_B200_ERR_INVALID; }
    cudaSetDevice(C->device);
    Level L;
    L.n = n; L.rp = (uint32_t *)rp; L.col = (uint32_t *)col; L.w = (void *)(wbytes ? w : nullptr); L.wbytes = wbytes;
    uint32_t mm = 0;
    int rc = n ? read_u32(*C, rp + n, &mm) : 0;
    L.m = mm;
    PowerIterOpts o;
    o.tol = tol;
    o.iter_cap = iter_cap;
    o.mixed = mixed;
    PowerIterResult r;
    if (rc == SGP_B200_OK) rc = power_iter_level(*C, L, x_in, vcmap, x_out, o, &r, residual != nullptr);
    if (rc == SGP_B200_OK) {
        if (niter) *niter = r.niter;
        if (lambda) *lambda = r.lambda;
        if (residual) *residual = r.resid;
    }
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc;
}

int sgp_b200_split(sgp_b200_ctx_t *x, uint32_t n, const uint32_t *rp, const uint32_t *col, const double *evec,
                   int perc_imbalance, uint32_t *part, uint64_t *edgecut) {
    Context *C = ctx_get(x);
    if (!C || !rp || !evec || !part || !edgecut) { set_error("null argument"); return SGP_B200_ERR_INVALID; }
    cudaSetDevice(C->device);
    Level L;
    L.n = n; L.rp = (uint32_t *)rp; L.col = (uint32_t *)col;
    int rc = split_level(*C, L, evec, perc_imbalance, part, edgecut, nullptr);
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc;
}

int sgp_b200_config_options(const config_t *config, int perc_imbalance_allowed, const sgp_pcg32_random_t *rng,
                            sgp_b200_options_t *o) {
    if (!config || !rng || !o) {
        set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    if (config->refine_alg != 0 && config->refine_alg != 1) {
        set_error("refine_alg must be 0 (shifted combinatorial Laplacian) or 1 (normalized Laplacian)");
        return SGP_B200_ERR_INVALID;
    }
    sgp_b200_default_options(o);
    o->tol = config->tol > 0 ? config->tol : g_tol;
    o->refine_alg = config->refine_alg;
    // sgpar.h:2457-2475: bit 4 skips coarsening, bit 0 picks heavy-edge
    // matching with the 0.9 coarsening-ratio stop (bits 1-2 choose a dedupe
    // method, which does not change the coarse graph)
    o->coarsener = (config->coarsening_alg & 16) ? SGP_B200_COARSEN_NONE
                   : (config->coarsening_alg & 1) ? (SGP_B200_COARSEN_MATCH | SGP_B200_COARSEN_RATIO_STOP)
                                                  : SGP_B200_COARSEN_HEC;
    o->perc_imbalance = perc_imbalance_allowed;
    o->local_search_alg = config->local_search_alg;
    o->rng_state = rng->state;
    o->rng_inc = rng->inc;
    return SGP_B200_OK;
}

// ------------------------------------------------------ sgpar.h API --
int sgp_partition_graph(sgp_vid_t *part, sgp_eid_t *edge_cut, config_t *config, const int perc_imbalance_allowed,
                        const sgp_graph_t g, sgp_pcg32_random_t *rng) {
    if (!part || !edge_cut || !config || !rng) {
        set_error("null argument");
        return 1;
    }
    if (config->refine_alg != 0 && config->refine_alg != 1) {
        set_error("refine_alg must be 0 (shifted combinatorial Laplacian) or 1 (normalized Laplacian)");
        return 1;
    }
    Context *C = default_ctx();
    if (!C) return 1;
    sgp_b200_graph_t dg;
    dg.n = g.nvertices;
    dg.m = g.source_offsets ? g.source_offsets[g.nvertices] : 0;
    dg.row_ptr = g.source_offsets;
    dg.col = g.destination_indices;
    dg.w = g.eweights;
    dg.mem = SGP_B200_HOST;
    sgp_b200_options_t o;
    if (sgp_b200_config_options(config, perc_imbalance_allowed, rng, &o) != SGP_B200_OK) return 1;
    sgp_b200_result_t *r = (sgp_b200_result_t *)calloc(1, sizeof(sgp_b200_result_t));
    if (!r) return 1;
    r->part = part;
    int rc = sgp_b200_partition(g_default, &dg, &o, r);
    if (rc == SGP_B200_OK) {
        *edge_cut = (sgp_eid_t)r->edgecut;
        rng->state = r->rng_state;
    }
    free(r);
    return rc == SGP_B200_OK ? 0 : 1;
}

int sgp_compute_partition(sgp_vid_t *part, sgp_vid_t num_partitions, sgp_eid_t *edgecut, int perc_imbalance_allowed,
                          int local_search_alg, sgp_real_t *evec, sgp_graph_t g) {
    if (num_partitions != 2 && num_partitions != 4) { set_error("num_partitions must be 2 or 4"); return 1; }
    if (local_search_alg != 0 && perc_imbalance_allowed != 0) {
        set_error("the local search takes perc_imbalance_allowed 0");
        return 1;
    }
    Context *C = default_ctx();
    if (!C || !part || !edgecut || !evec) return 1;
    cudaSetDevice(C->device);
    sgp_b200_graph_t dg;
    dg.n = g.nvertices;
    dg.m = g.source_offsets[g.nvertices];
    dg.row_ptr = g.source_offsets;
    dg.col = g.destination_indices;
    dg.w = nullptr;
    dg.mem = SGP_B200_HOST;
    Level L0;
    int rc = stage_input(*C, &dg, &L0);
    double *ev = nullptr;
    uint32_t *pd = nullptr;
    if (rc == SGP_B200_OK) rc = dalloc_t(*C, &ev, g.nvertices);
    if (rc == SGP_B200_OK) rc = dalloc_t(*C, &pd, g.nvertices);
    if (rc == SGP_B200_OK &&
        cudaMemcpyAsync(ev, evec, sizeof(double) * g.nvertices, cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
        rc = SGP_B200_ERR_DEVICE;
    uint64_t cut = 0;
    uint32_t p0 = 0;
    if (rc == SGP_B200_OK) rc = split_level(*C, L0, ev, perc_imbalance_allowed, pd, &cut, &p0);
    if (rc == SGP_B200_OK && local_search_alg) {   // sgpar.h:2080-2170
        rc = local_search_level(*C, L0, pd, p0, nullptr, nullptr);
        if (rc == SGP_B200_OK) rc = edge_cut_device(*C, L0, pd, &cut);
    }
    if (rc == SGP_B200_OK &&
        cudaMemcpyAsync(part, pd, sizeof(uint32_t) * g.nvertices, cudaMemcpyDeviceToHost, C->stream) != cudaSuccess)
        rc = SGP_B200_ERR_DEVICE;
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    if (rc == SGP_B200_OK) *edgecut = (sgp_eid_t)cut;
    return rc == SGP_B200_OK ? 0 : 1;
}

int sgp_use_partition(sgp_vid_t *part, const sgp_graph_t g, sgp_graph_t *g1, sgp_graph_t *g2) {
    Context *C = default_ctx();
    if (!C || !part || !g1 || !g2) return 1;
    cudaSetDevice(C->device);
    sgp_b200_graph_t dg;
    dg.n = g.nvertices;
    dg.m = g.source_offsets[g.nvertices];
    dg.row_ptr = g.source_offsets;
    dg.col = g.destination_indices;
    dg.w = nullptr;
    dg.mem = SGP_B200_HOST;
    Level L0, a, b;
    uint32_t *pd = nullptr;
    int rc = stage_input(*C, &dg, &L0);
    if (rc == SGP_B200_OK) rc = dalloc_t(*C, &pd, g.nvertices);
    if (rc == SGP_B200_OK &&
        cudaMemcpyAsync(pd, part, sizeof(uint32_t) * g.nvertices, cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
        rc = SGP_B200_ERR_DEVICE;
    if (rc == SGP_B200_OK) rc = induced_subgraphs(*C, L0, pd, &a, &b);
    sgp_graph_t *outs[2] = {g1, g2};
    Level *ls[2] = {&a, &b};
    for (int k = 0; k < 2 && rc == SGP_B200_OK; k++) {
        sgp_graph_t *o = outs[k];
        memset(o, 0, sizeof(*o));
        o->nvertices = ls[k]->n;
        o->nedges = (sgp_eid_t)ls[k]->m;   // the reference stores the directed count here (sgpar.h:2735)
        o->source_offsets = (sgp_eid_t *)malloc(sizeof(sgp_eid_t) * ((size_t)ls[k]->n + 1));
        o->destination_indices = (sgp_vid_t *)malloc(sizeof(sgp_vid_t) * (ls[k]->m ? ls[k]->m : 1));
        if (!o->source_offsets || !o->destination_indices) { rc = 1; break; }
        if (cudaMemcpyAsync(o->source_offsets, ls[k]->rp, sizeof(uint32_t) * ((size_t)ls[k]->n + 1),
                            cudaMemcpyDeviceToHost, C->stream) != cudaSuccess ||
            cudaMemcpyAsync(o->destination_indices, ls[k]->col, sizeof(uint32_t) * ls[k]->m, cudaMemcpyDeviceToHost,
                            C->stream) != cudaSuccess)
            rc = SGP_B200_ERR_DEVICE;
    }
    cudaStreamSynchronize(C->stream);
    release_all(*C);
    return rc == SGP_B200_OK ? 0 : 1;
}

}  // extern "C"
