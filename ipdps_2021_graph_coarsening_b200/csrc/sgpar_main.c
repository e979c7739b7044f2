/*
 * sgpar_main.c -- the config-file driver:
 *
 *     sgpar_b200 <csr_filename> <metrics_filename> <config_file> [best_partition_file]
 *
 * The command the reference's experiment scripts run (cmg/sgpar.cpp:11-106,
 * built as hec_spec and friends; cmg/jsonExperimentRunner.py:155 calls it
 * with base_config.txt), on the C ABI of include/sgpar_b200.h:
 *
 *   - the config (six fields: coarsening_alg refine_alg local_search_alg
 *     num_partitions num_iter tol, e.g. cmg/base_config.txt or
 *     cmg/fourpart_config.txt) and the binary CSR graph are read;
 *   - num_iter partitions run one after another with one PCG32 rng carried
 *     through all of them (state from the clock, inc 1, as sgpar.cpp:45-46;
 *     the environment variable SGPB_RNG_STATE fixes the state instead, for
 *     reproducible runs);
 *   - with a best-partition file, each bisection's edit distance to it
 *     (compute_partition_edit_distance) is recorded;
 *   - with num_partitions == 4, the two induced sub-graphs of the bisection
 *     (sgp_use_partition) are bisected with the same rng, and the 4-way cut
 *     is the sum of the three cuts (sgpar.cpp:62-89);
 *   - one record per partition is appended to the metrics file in the
 *     layout of ExperimentLoggerUtil::log (first record opens the JSON list,
 *     the last closes it), so the reference's runner aggregates it unchanged;
 *   - the smallest bisection cut is printed at the end.
 *
 * Every bisection runs on the GPU (CUDA device 0, or the device named by
 * SGPB_DEVICE); there is no CPU path.  Exit status: EXIT_SUCCESS, or
 * EXIT_FAILURE with the library's message on stderr (the reference's
 * CHECK_SGPAR returns EXIT_FAILURE from main the same way).
 */
#include <inttypes.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/sgpar_b200.h"

#define CHECK(call, what)                                                                  \
    do {                                                                                   \
        int rc_ = (call);                                                                  \
        if (rc_ != 0) {                                                                    \
            fprintf(stderr, "sgpar_b200: %s failed (%d): %s\n", what, rc_, sgp_b200_last_error()); \
            return EXIT_FAILURE;                                                           \
        }                                                                                  \
    } while (0)

/* host view of an sgp_graph_t for the context interface */
static sgp_b200_graph_t view(const sgp_graph_t *g) {
    sgp_b200_graph_t v;
    memset(&v, 0, sizeof(v));
    v.n = g->nvertices;
    v.m = g->source_offsets ? g->source_offsets[g->nvertices] : 0;
    v.row_ptr = g->source_offsets;
    v.col = g->destination_indices;
    v.w = g->eweights;
    v.mem = SGP_B200_HOST;
    return v;
}

/* One bisection of g as sgp_partition_graph runs it (perc_imbalance_allowed
 * 0, as sgpar.cpp:55 passes), with the statistics the metrics record needs;
 * the rng is advanced. */
static int bisect(sgp_b200_ctx_t *ctx, const sgp_graph_t *g, const config_t *config, sgp_pcg32_random_t *rng,
                  sgp_vid_t *part, sgp_b200_result_t *res) {
    sgp_b200_options_t o;
    int rc = sgp_b200_config_options(config, 0, rng, &o);
    if (rc != SGP_B200_OK) return rc;
    const sgp_b200_graph_t v = view(g);
    memset(res, 0, sizeof(*res));
    res->part = part;
    rc = sgp_b200_partition(ctx, &v, &o, res);
    if (rc == SGP_B200_OK) rng->state = res->rng_state;
    return rc;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        printf("You input %d args\n", argc);
        fprintf(stderr, "Usage: %s csr_filename metrics_filename config_file [best_partition_file]\n", argv[0]);
        return EXIT_FAILURE;
    }
    char *filename = argv[1];
    const char *metrics = argv[2];

    config_t config;
    CHECK(sgp_load_config(argv[3], &config), "reading the config");
    if (config.num_iter < 1) {
        fprintf(stderr, "sgpar_b200: num_iter must be at least 1 (config %s)\n", argv[3]);
        return EXIT_FAILURE;
    }
    sgp_graph_t g;
    CHECK(sgp_load_graph(&g, filename), "reading the graph");
    printf("n: %ld, m: %ld\n", (long)g.nvertices, (long)g.nedges);
    printf("coarsening_alg: %d, refine_alg: %d, local_alg %d, num_iter %d\n", config.coarsening_alg,
           config.refine_alg, config.local_search_alg, config.num_iter);

    sgp_vid_t *part = (sgp_vid_t *)malloc(((size_t)g.nvertices + 1) * sizeof(sgp_vid_t));
    sgp_b200_result_t *res = (sgp_b200_result_t *)malloc(sizeof(sgp_b200_result_t));
    sgp_b200_result_t *sub = (sgp_b200_result_t *)malloc(sizeof(sgp_b200_result_t));
    if (!part || !res || !sub) {
        fprintf(stderr, "sgpar_b200: out of host memory\n");
        return EXIT_FAILURE;
    }
    sgp_vid_t *best_part = NULL;
    if (argc > 4) {
        best_part = (sgp_vid_t *)malloc(((size_t)g.nvertices + 1) * sizeof(sgp_vid_t));
        if (!best_part) return EXIT_FAILURE;
        CHECK(sgp_load_partition(best_part, g.nvertices, argv[4]), "reading the best partition");
    }

    const char *dev_s = getenv("SGPB_DEVICE");
    sgp_b200_ctx_t *ctx = sgp_b200_create(dev_s ? atoi(dev_s) : 0);
    if (!ctx) {
        fprintf(stderr, "sgpar_b200: no CUDA device: %s\n", sgp_b200_last_error());
        return EXIT_FAILURE;
    }

    long edgecut_min = 1L << 30;
    sgp_pcg32_random_t rng;
    const char *seed_s = getenv("SGPB_RNG_STATE");
    rng.state = seed_s ? strtoull(seed_s, NULL, 0) : (uint64_t)time(NULL);
    rng.inc = 1;
    for (int i = 0; i < config.num_iter; i++) {
        CHECK(bisect(ctx, &g, &config, &rng, part, res), "partitioning the graph");
        const uint64_t edgecut = res->edgecut;

        sgp_vid_t part_diff = 0;
        if (best_part) CHECK(compute_partition_edit_distance(part, best_part, g.nvertices, &part_diff),
                             "comparing with the best partition");

        uint64_t cut4 = 0;
        if (config.num_partitions == 4) {
            sgp_graph_t g1, g2;
            CHECK(sgp_use_partition(part, g, &g1, &g2), "taking the induced sub-graphs");
            sgp_vid_t *part1 = (sgp_vid_t *)malloc(((size_t)g1.nvertices + 1) * sizeof(sgp_vid_t));
            sgp_vid_t *part2 = (sgp_vid_t *)malloc(((size_t)g2.nvertices + 1) * sizeof(sgp_vid_t));
            if (!part1 || !part2) return EXIT_FAILURE;
            CHECK(bisect(ctx, &g1, &config, &rng, part1, sub), "partitioning the first sub-graph");
            const uint64_t ec1 = sub->edgecut;
            CHECK(bisect(ctx, &g2, &config, &rng, part2, sub), "partitioning the second sub-graph");
            const uint64_t ec2 = sub->edgecut;
            cut4 = edgecut + ec1 + ec2;
            sgp_free_graph(&g1);
            sgp_free_graph(&g2);
            free(part1);
            free(part2);
        }

        if ((long)edgecut < edgecut_min) edgecut_min = (long)edgecut;
        CHECK(sgp_b200_write_metrics(metrics, res, cut4, part_diff, i == 0, i + 1 == config.num_iter),
              "writing the metrics");
    }
    printf("graph %s, min edgecut found is %ld\n", filename, edgecut_min);

    sgp_b200_destroy(ctx);
    CHECK(sgp_free_graph(&g), "freeing the graph");
    free(part);
    free(res);
    free(sub);
    free(best_part);
    return EXIT_SUCCESS;
}
