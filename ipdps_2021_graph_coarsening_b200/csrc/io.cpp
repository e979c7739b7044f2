// io.cpp -- host-side file loaders and small helpers of the sgpar.h API.
//
// Formats and semantics follow cmg/sgpar.h:
//   sgp_load_graph           :2262-2289  binary CSR (6 x int64 header, uint32 offsets, uint32 destinations)
//   sgp_free_graph           :2291-2319
//   sgp_load_partition       :2321-2341
//   compute_partition_edit_distance :2343-2361
//   sgp_load_config          :2754-2787  six whitespace-separated fields
//   sgp_pcg32_random_r       :84-92
// Failures return EXIT_FAILURE with a message instead of asserting.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/sgpar_b200.h"

namespace sgpb {
void set_error(const char *fmt, ...);
}

extern "C" {

uint32_t sgp_pcg32_random_r(sgp_pcg32_random_t *rng) {
    uint64_t old = rng->state;
    rng->state = old * 6364136223846793005ULL + (rng->inc | 1);
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}

int sgp_load_graph(sgp_graph_t *g, char *csr_filename) {
    if (!g || !csr_filename) return EXIT_FAILURE;
    FILE *f = fopen(csr_filename, "rb");
    if (!f) {
        sgpb::set_error("could not open input file %s", csr_filename);
        return EXIT_FAILURE;
    }
    int64_t hdr[6];
    if (fread(hdr, sizeof(int64_t), 6, f) != 6 || hdr[0] < 0 || hdr[1] < 0 || hdr[0] >= 0xFFFFFFFFll ||
        hdr[1] > 0xFFFFFFFFll) {
        sgpb::set_error("bad CSR header in %s", csr_filename);
        fclose(f);
        return EXIT_FAILURE;
    }
    uint64_t n = (uint64_t)hdr[0], m = (uint64_t)hdr[1];
    g->nvertices = (sgp_vid_t)n;
    g->nedges = (sgp_eid_t)(m / 2);
    g->source_offsets = (sgp_eid_t *)malloc(sizeof(sgp_eid_t) * (n + 1));
    g->destination_indices = (sgp_vid_t *)malloc(sizeof(sgp_vid_t) * (2 * (uint64_t)g->nedges + 1));
    g->eweights = NULL;
    g->weighted_degree = NULL;
    g->edges_per_source = NULL;
    int ok = g->source_offsets && g->destination_indices;
    ok = ok && fread(g->source_offsets, sizeof(sgp_eid_t), n + 1, f) == n + 1;
    ok = ok && fread(g->destination_indices, sizeof(sgp_vid_t), 2 * (uint64_t)g->nedges, f) == 2 * (uint64_t)g->nedges;
    fclose(f);
    if (!ok) {
        sgpb::set_error("short read in %s", csr_filename);
        free(g->source_offsets);
        free(g->destination_indices);
        g->source_offsets = NULL;
        g->destination_indices = NULL;
        return EXIT_FAILURE;
    }
    return EXIT_SUCCESS;
}

int sgp_free_graph(sgp_graph_t *g) {
    if (!g) return EXIT_FAILURE;
    free(g->source_offsets); g->source_offsets = NULL;
    free(g->destination_indices); g->destination_indices = NULL;
    free(g->eweights); g->eweights = NULL;
    free(g->weighted_degree); g->weighted_degree = NULL;
    free(g->edges_per_source); g->edges_per_source = NULL;
    return EXIT_SUCCESS;
}

int sgp_load_partition(sgp_vid_t *part, sgp_vid_t size, char *part_filename) {
    FILE *f = fopen(part_filename, "r");
    if (!f) {
        sgpb::set_error("could not open partition file %s", part_filename);
        return EXIT_FAILURE;
    }
    for (sgp_vid_t i = 0; i < size; i++) {
        unsigned int v;
        if (fscanf(f, "%u", &v) != 1) {
            fclose(f);
            return EXIT_FAILURE;
        }
        part[i] = v;
    }
    fclose(f);
    return EXIT_SUCCESS;
}

int compute_partition_edit_distance(const sgp_vid_t *part1, const sgp_vid_t *part2, sgp_vid_t size,
                                    sgp_vid_t *diff) {
    sgp_vid_t d = 0, d2 = 0;
    for (sgp_vid_t i = 0; i < size; i++) {
        if (part1[i] != part2[i]) d++;
        else d2++;
    }
    *diff = (d < d2 ? d : d2) / 2;
    return EXIT_SUCCESS;
}

int sgp_load_config(const char *config_f, config_t *c) {
    FILE *f = fopen(config_f, "r");
    if (!f) {
        sgpb::set_error("could not open config file %s", config_f);
        return EXIT_FAILURE;
    }
    int ok = fscanf(f, "%i", &c->coarsening_alg) == 1 && fscanf(f, "%i", &c->refine_alg) == 1 &&
             fscanf(f, "%i", &c->local_search_alg) == 1 && fscanf(f, "%i", &c->num_partitions) == 1 &&
             fscanf(f, "%i", &c->num_iter) == 1 && fscanf(f, "%lf", &c->tol) == 1;
    fclose(f);
    if (!ok) {
        sgpb::set_error("malformed config file %s", config_f);
        return EXIT_FAILURE;
    }
    change_tol(c->tol);
    return EXIT_SUCCESS;
}

// ExperimentLoggerUtil.cpp:145-192 (record layout), :57-63 (coarse level),
// sgpar.h:2405-2409 (timing window, finest cut), eigensolve_kokkos.h:190-198
// (one coarse-level entry per power iteration, coarsest first).
int sgp_b200_write_metrics(const char *path, const sgp_b200_result_t *r, uint64_t edge_cut_4way,
                           uint64_t partition_diff, int first, int last) {
    if (!path || !r) {
        sgpb::set_error("null argument");
        return SGP_B200_ERR_INVALID;
    }
    if (r->levels < 1 || r->levels > SGP_B200_MAX_LEVELS) {
        sgpb::set_error("result holds %d levels", r->levels);
        return SGP_B200_ERR_INVALID;
    }
    FILE *f = fopen(path, "a");
    if (!f) {
        sgpb::set_error("could not open %s", path);
        return EXIT_FAILURE;
    }
    static const char *names[] = {"coarsen-map", "coarsen-build", "coarsen-count", "coarsen-prefix-sum",
                                  "coarsen-bucket", "coarsen-dedupe", "coarsen-radix-sort", "coarsen-radix-dedupe",
                                  "coarsen-write-graph", "coarsen-permute", "coarsen-map-construct", "fm-refine",
                                  "fm-recoarsen", "heavy"};
    const double s_h2d = r->ms_h2d / 1e3, s_coarsen = r->ms_coarsen / 1e3, s_eigen = r->ms_eigen / 1e3;
    const double meas[14] = {r->ms_map / 1e3, r->ms_build / 1e3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (first) fputc('[', f);
    fprintf(f, "{\"edge-cut\":%llu,\"edge-cut-four-way\":%llu,\"partition-diff\":%llu,",
            (unsigned long long)r->edgecut, (unsigned long long)edge_cut_4way, (unsigned long long)partition_diff);
    fprintf(f, "\"total-duration-seconds\":%.9g,\"coarsen-duration-seconds\":%.9g,\"refine-duration-seconds\":%.9g,",
            s_h2d + s_coarsen + s_eigen, s_h2d + s_coarsen, s_eigen);
    fprintf(f, "\"number-coarse-levels\":%d,", r->levels);
    fprintf(f, "\"level-1-first-two-passes-assign-rate\":0,\"level-1-total-passes\":%d,",
            r->levels > 1 ? r->level_hec_rounds[0] : 0);
    fprintf(f, "\"level-2-first-two-passes-assign-rate\":0,\"level-2-total-passes\":%d,",
            r->levels > 2 ? r->level_hec_rounds[1] : 0);
    for (int i = 0; i < 14; i++) fprintf(f, "\"%s-duration-seconds\":%.9g,", names[i], meas[i]);
    fputs("\"coarse-levels\":[", f);
    for (int l = r->levels - 1; l >= 0; l--) {
        // the per-level cap without an iteration budget: 1e14 / n (eigensolve_kokkos.h:153), at most 5e6
        uint64_t cap = r->level_n[l] ? 100000000000000ULL / r->level_n[l] : 0;
        if (cap > 5000000ULL) cap = 5000000ULL;
        fprintf(f, "%s{\"refine-iterations\":%llu,\"iteration-max-reached\":%d,\"number-vertices\":%u,"
                   "\"unrefined-edge-cut\":%llu}",
                l == r->levels - 1 ? "" : ",", (unsigned long long)r->level_iters[l],
                r->level_iters[l] >= cap ? 1 : 0, r->level_n[l], (unsigned long long)(l == 0 ? r->edgecut : 0));
    }
    fputs("]}", f);
    fputc(last ? ']' : ',', f);
    fclose(f);
    return SGP_B200_OK;
}

}  // extern "C"
