/*
 * ref_harness.cpp -- C-ABI shim over the reference's own serial/OpenMP
 * implementation (cmg/sgpar.h, compiled from its sources where they lie; see
 * oracle/Makefile).  TEST AND CPU-REFERENCE INFRASTRUCTURE ONLY: used by tests/ to
 * pin the oracle restatement and by bench.py's reference arm as the CPU
 * baseline.  Nothing here is shipped.
 *
 * Built twice: without -fopenmp (the deterministic serial path of sgpar.h) and
 * with -fopenmp -DUSE_GNU_PARALLELMODE (the flags of cmg/Makefile's `sgpar`
 * target), each for the cutoffs 50 (reference default) and 32.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define SGPAR_IMPLEMENTATION
#include "sgpar.h"

using namespace sgpar;

static sgp_graph_t make_graph(uint32_t n, const uint32_t *row_ptr, const uint32_t *col) {
    sgp_graph_t g;
    g.nvertices = n;
    g.nedges = row_ptr[n] / 2;
    g.source_offsets = (sgp_eid_t *)row_ptr;
    g.destination_indices = (sgp_vid_t *)col;
    g.edges_per_source = NULL;
    g.weighted_degree = NULL;
    g.eweights = NULL;
    return g;
}

/* silence the reference's per-level printf chatter around a call */
struct Quiet {
    int saved;
    explicit Quiet(int on) : saved(-1) {
        if (!on) return;
        fflush(stdout);
        saved = dup(1);
        FILE *nul = fopen("/dev/null", "w");
        if (nul) { dup2(fileno(nul), 1); fclose(nul); }
    }
    ~Quiet() {
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

extern "C" {

int ref_cutoff(void) { return SGPAR_COARSENING_VTX_CUTOFF; }
int ref_is_openmp(void) {
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

/* sgpar.h:1790 (serial) / :1513 (OpenMP) sgp_power_iter, normLap = 0.
 * w == NULL with final = 1 is the finest level; otherwise the weighted form
 * with edges_per_source = full rows. */
int ref_power_iter(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                   const uint32_t *w, int final_level, double *u, double tol, int quiet) {
    Quiet q(quiet);
    change_tol(tol);
    sgp_graph_t g = make_graph(n, row_ptr, col);
    uint32_t *eps = NULL, *wd = NULL, *ones = NULL;
    if (!final_level) {
        eps = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        wd = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        if (!w) {
            ones = (uint32_t *)malloc((size_t)row_ptr[n] * sizeof(uint32_t) + 4);
            for (uint32_t j = 0; j < row_ptr[n]; j++) ones[j] = 1;
        }
        const uint32_t *ww = w ? w : ones;
        for (uint32_t i = 0; i < n; i++) {
            eps[i] = row_ptr[i + 1] - row_ptr[i];
            uint32_t s = 0;
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) s += ww[j];
            wd[i] = s;
        }
        g.edges_per_source = eps;
        g.weighted_degree = wd;
        g.eweights = (sgp_wgt_t *)ww;
    }
    int rc = sgp_power_iter(u, g, 0, final_level);
    free(eps); free(wd); free(ones);
    return rc;
}

/* sgp_power_iter with normLap = 1 (refine_alg 1) on a coarse level
 * (final = 0: weighted degrees and weights set, as the serial driver has
 * them for every level but the finest). */
int ref_power_iter_nl(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                      const uint32_t *w, double *u, double tol, int quiet) {
    Quiet q(quiet);
    change_tol(tol);
    sgp_graph_t g = make_graph(n, row_ptr, col);
    uint32_t *eps = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    uint32_t *wd = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    uint32_t *ones = NULL;
    if (!w) {
        ones = (uint32_t *)malloc((size_t)row_ptr[n] * sizeof(uint32_t) + 4);
        for (uint32_t j = 0; j < row_ptr[n]; j++) ones[j] = 1;
    }
    const uint32_t *ww = w ? w : ones;
    for (uint32_t i = 0; i < n; i++) {
        eps[i] = row_ptr[i + 1] - row_ptr[i];
        uint32_t s = 0;
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) s += ww[j];
        wd[i] = s;
    }
    g.edges_per_source = eps;
    g.weighted_degree = wd;
    g.eweights = (sgp_wgt_t *)ww;
    int rc = sgp_power_iter(u, g, 1, 0);
    free(eps); free(wd); free(ones);
    return rc;
}

/* sgpar.h:1969 sgp_compute_partition with 2 parts, local search off. */
int ref_compute_partition(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                          double *evec, int perc_imbalance_allowed,
                          uint32_t *part, uint64_t *edgecut, int quiet) {
    Quiet q(quiet);
    sgp_graph_t g = make_graph(n, row_ptr, col);
    sgp_eid_t ec = 0;
    int rc = sgp_compute_partition(part, 2, &ec, perc_imbalance_allowed, 0, evec, g);
    *edgecut = ec;
    return rc;
}

/* sgpar.h:1969-2170 with a local search: the split followed by the
 * reference's greedy swap search over vertex-id ranges (local_search_alg != 0). */
int ref_compute_partition_ls(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                             double *evec, int perc_imbalance_allowed, int local_search_alg,
                             uint32_t *part, uint64_t *edgecut, int quiet) {
    Quiet q(quiet);
    sgp_graph_t g = make_graph(n, row_ptr, col);
    sgp_eid_t ec = 0;
    int rc = sgp_compute_partition(part, 2, &ec, perc_imbalance_allowed, local_search_alg, evec, g);
    *edgecut = ec;
    return rc;
}

/* sgpar.h:1223 sgp_build_coarse_graph_msd on a given mapping.  Output is the
 * reference's bucketed layout: offsets[nc+1] (bucket starts), counts[nc]
 * (deduplicated row lengths), cols / wgts sized offsets[nc] <= row_ptr[n]. */
int ref_build_coarse_msd(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                         const uint32_t *w, int coarsening_level, int coarsening_alg,
                         uint32_t *vcmap, uint32_t nc,
                         uint32_t *out_offsets, uint32_t *out_counts,
                         uint32_t *out_cols, uint32_t *out_wgts, uint64_t *out_nedges) {
    sgp_graph_t g = make_graph(n, row_ptr, col);
    uint32_t *eps = NULL;
    if (coarsening_level != 1) {
        /* level >= 2 graphs carry weights and per-row counts */
        eps = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        for (uint32_t i = 0; i < n; i++) eps[i] = row_ptr[i + 1] - row_ptr[i];
        g.edges_per_source = eps;
        g.eweights = (sgp_wgt_t *)w;
    }
    sgp_graph_t gc;
    memset(&gc, 0, sizeof(gc));
    gc.nvertices = nc;
    double tp[6] = {0, 0, 0, 0, 0, 0};
    int rc = sgp_build_coarse_graph_msd(&gc, vcmap, g, coarsening_level, tp, coarsening_alg);
    if (rc == 0) {
        memcpy(out_offsets, gc.source_offsets, ((size_t)nc + 1) * sizeof(uint32_t));
        memcpy(out_counts, gc.edges_per_source, (size_t)nc * sizeof(uint32_t));
        uint32_t tot = gc.source_offsets[nc];
        memcpy(out_cols, gc.destination_indices, (size_t)tot * sizeof(uint32_t));
        memcpy(out_wgts, gc.eweights, (size_t)tot * sizeof(uint32_t));
        *out_nedges = gc.nedges;
    }
    free(eps);
    sgp_free_graph(&gc);
    return rc;
}

/* sgpar.h:601-703 (serial) / 454-599 (OpenMP) sgp_coarsen_HEC. */
int ref_coarsen_hec(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                    const uint32_t *w, int coarsening_level,
                    uint64_t *rng_state, uint64_t rng_inc, uint32_t *vcmap, uint32_t *nc) {
    sgp_graph_t g = make_graph(n, row_ptr, col);
    uint32_t *eps = NULL;
    if (coarsening_level != 1) {
        eps = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        for (uint32_t i = 0; i < n; i++) eps[i] = row_ptr[i + 1] - row_ptr[i];
        g.edges_per_source = eps;
        g.eweights = (sgp_wgt_t *)w;
    }
    sgp_pcg32_random_t rng;
    rng.state = *rng_state; rng.inc = rng_inc;
    sgp_vid_t ncv = 0;
    int rc = sgp_coarsen_HEC(vcmap, &ncv, g, coarsening_level, &rng);
    *rng_state = rng.state;
    *nc = ncv;
    free(eps);
    return rc;
}

/* sgpar.h:2363 sgp_partition_graph (non-Kokkos branch :2432-2661). */
int ref_partition_graph(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                        int coarsening_alg, int refine_alg, int local_search_alg,
                        int num_partitions, double tol, int perc_imbalance_allowed,
                        uint64_t *rng_state, uint64_t rng_inc,
                        uint32_t *part, uint64_t *edgecut, int quiet) {
    Quiet q(quiet);
    config_t cfg;
    cfg.coarsening_alg = coarsening_alg;
    cfg.refine_alg = refine_alg;
    cfg.local_search_alg = local_search_alg;
    cfg.num_partitions = num_partitions;
    cfg.num_iter = 1;
    cfg.tol = tol;
    change_tol(tol);
    sgp_graph_t g = make_graph(n, row_ptr, col);
    sgp_pcg32_random_t rng;
    rng.state = *rng_state; rng.inc = rng_inc;
    sgp_eid_t ec = 0;
    int rc = sgp_partition_graph(part, &ec, &cfg, perc_imbalance_allowed, g, &rng);
    *rng_state = rng.state;
    *edgecut = ec;
    return rc;
}

/* sgpar.h:2666 sgp_use_partition; caller frees with ref_free. */
int ref_use_partition(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t *part,
                      uint32_t *n1, uint32_t **rp1, uint32_t **col1,
                      uint32_t *n2, uint32_t **rp2, uint32_t **col2) {
    sgp_graph_t g = make_graph(n, row_ptr, col), g1, g2;
    int rc = sgp_use_partition(part, g, &g1, &g2);
    *n1 = g1.nvertices; *rp1 = g1.source_offsets; *col1 = g1.destination_indices;
    *n2 = g2.nvertices; *rp2 = g2.source_offsets; *col2 = g2.destination_indices;
    return rc;
}
void ref_free(void *p) { free(p); }

/* The two known-answer dedupe routines pinned by cmg/tests.cpp:7-107. */
int ref_heap_deduplicate(uint32_t *offsets2, uint32_t *dests, uint32_t *wgts,
                         uint32_t *eps, uint64_t *total) {
    sgp_eid_t t = 0;
    heap_deduplicate(offsets2, dests, wgts, eps, &t);
    *total = t;
    return 0;
}
int ref_hashmap_deduplicate(uint32_t *offsets2, uint32_t *dests, uint32_t *wgts,
                            uint32_t *eps, uint64_t *total) {
    sgp_eid_t t = 0;
    hashmap_deduplicate(offsets2, dests, wgts, eps, &t);
    *total = t;
    return 0;
}

} /* extern "C" */
