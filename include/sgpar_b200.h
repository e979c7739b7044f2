/*
 * sgpar_b200.h -- C ABI of the B200-native multilevel spectral bisection path.
 *
 * Part 1 keeps the partition API of the reference's cmg/sgpar.h (the block at
 * sgpar.h:2230-2244) with its struct layouts for the default build (32-bit
 * vertex ids, offsets and weights), exported with C linkage so that a C, C++,
 * cgo, JNI or ctypes caller binds it directly.  Behind these entry points the
 * hot path -- HEC mapping, coarse-graph construction, Fiedler power iteration
 * with prolongation and the median split -- runs as hand-written sm_100a
 * kernels; there is no CPU fallback.
 *
 * Part 2 is the explicit-context interface (device, stream, memory reuse,
 * mixed precision, device-resident inputs/outputs, per-level statistics) and
 * the lower boundary the reference exposes between its layers
 * (coarsen_kokkos.h:1165 sgp_generate_coarse_graphs, eigensolve_kokkos.h:1493
 * sgp_eigensolve) plus per-kernel entry points used by the parity tests.
 *
 * Return codes: 0 = success (EXIT_SUCCESS), 1 = failure (EXIT_FAILURE), and
 * the more specific SGP_B200_ERR_* values of part 2; sgp_b200_last_error()
 * returns the message of the last failure on the calling thread.
 */
#ifndef SGPAR_B200_H_
#define SGPAR_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ *
 * Part 1: the sgpar.h partition API                                         *
 * ------------------------------------------------------------------------ */

typedef uint32_t sgp_vid_t;   /* sgpar.h:109-111 (default build) */
typedef uint32_t sgp_eid_t;
typedef double sgp_real_t;
typedef uint32_t sgp_wgt_t;   /* sgpar.h:117-121: sgp_vid_t outside the Kokkos build */

/* sgpar.h:82 */
typedef struct { uint64_t state; uint64_t inc; } sgp_pcg32_random_t;

/* sgpar.h:145-153 */
typedef struct {
    sgp_vid_t nvertices;
    sgp_eid_t nedges;              /* undirected edges = source_offsets[n] / 2 */
    sgp_eid_t *source_offsets;
    sgp_vid_t *edges_per_source;
    sgp_vid_t *destination_indices;
    sgp_wgt_t *weighted_degree;
    sgp_wgt_t *eweights;           /* NULL: unit weights (as the reference loader leaves it) */
} sgp_graph_t;

/* sgpar.h:186-193 */
typedef struct configuration {
    int coarsening_alg;
    int refine_alg;
    int local_search_alg;
    int num_iter;
    double tol;
    int num_partitions;
} config_t;

/* sgpar.h:84 -- PCG32 (XSH-RR) step. */
uint32_t sgp_pcg32_random_r(sgp_pcg32_random_t *rng);

/* sgpar.h:195 -- process-wide default tolerance used when config->tol <= 0. */
int change_tol(sgp_real_t new_tol);

/* sgpar.h:2262 -- read the reference's binary CSR file (6 x int64 header,
 * uint32 offsets[n+1], uint32 destinations[m]).  Arrays are malloc'd. */
int sgp_load_graph(sgp_graph_t *g, char *csr_filename);

/* sgpar.h:2291 -- free and NULL the arrays of g. */
int sgp_free_graph(sgp_graph_t *g);

/* sgpar.h:2321 -- read `size` whitespace-separated part ids. */
int sgp_load_partition(sgp_vid_t *part, sgp_vid_t size, char *part_filename);

/* sgpar.h:2754 -- six whitespace-separated fields: coarsening_alg refine_alg
 * local_search_alg num_partitions num_iter tol (a trailing token is ignored). */
int sgp_load_config(const char *config_f, config_t *config);

/* sgpar.h:2343 -- label-swap-invariant difference of two bisections / 2. */
int compute_partition_edit_distance(const sgp_vid_t *part1, const sgp_vid_t *part2,
                                    sgp_vid_t size, sgp_vid_t *diff);

/* sgpar.h:2363 -- multilevel spectral bisection of g on the current CUDA
 * device: coarsening until at most 50 vertices remain (HEC; heavy-edge
 * matching when config->coarsening_alg & 1, stopping after a level that keeps
 * more than 0.9 of the vertices; none when config->coarsening_alg & 16, as
 * sgpar.h:2457-2475 reads those bits), Fiedler power
 * iteration (tolerance config->tol, FP64) up the hierarchy, median split.
 * part[n] is caller-allocated host memory; *edge_cut receives the cut of the
 * bisection.  rng seeds the mapping hashes and the coarsest guess and is
 * advanced.  config->refine_alg 0 (shifted combinatorial Laplacian) or 1
 * (normalized Laplacian); config->local_search_alg != 0 runs the reference's
 * local search after the split (sgpar.h:2080-2170); other refine_alg values
 * return EXIT_FAILURE.  With
 * config->num_partitions == 4 the call still bisects (the 4-way recursion is
 * the caller's, sgpar.cpp:62-89, via sgp_use_partition). */
int sgp_partition_graph(sgp_vid_t *part, sgp_eid_t *edge_cut, config_t *config,
                        const int perc_imbalance_allowed, const sgp_graph_t g,
                        sgp_pcg32_random_t *rng);

/* sgpar.h:1969 -- median split of an eigenvector and its edge cut (run on the
 * device; evec and part are host arrays of g.nvertices entries).
 * num_partitions must be 2 or 4 (4 splits in two as in the reference). */
int sgp_compute_partition(sgp_vid_t *part, sgp_vid_t num_partitions, sgp_eid_t *edgecut,
                          int perc_imbalance_allowed, int local_search_alg,
                          sgp_real_t *evec, sgp_graph_t g);

/* sgpar.h:2666 -- the two induced sub-graphs of a bisection, vertices of each
 * part relabelled in ascending order; g1/g2 arrays are malloc'd (free with
 * sgp_free_graph).  Built on the device. */
int sgp_use_partition(sgp_vid_t *part, const sgp_graph_t g, sgp_graph_t *g1, sgp_graph_t *g2);

/* ------------------------------------------------------------------------ *
 * Part 2: explicit-context interface                                        *
 * ------------------------------------------------------------------------ */

#define SGP_B200_OK 0
#define SGP_B200_FAIL 1
#define SGP_B200_ERR_INVALID 2      /* bad argument or malformed graph */
#define SGP_B200_ERR_DEVICE 3       /* CUDA error */
#define SGP_B200_ERR_TOO_LARGE 4    /* a count exceeds the 32-bit index space */
#define SGP_B200_ERR_BUDGET 5       /* an iteration / round budget ran out */

typedef struct sgp_b200_ctx sgp_b200_ctx_t;

/* Create a context on CUDA device `device` with its own stream. */
sgp_b200_ctx_t *sgp_b200_create(int device);
void sgp_b200_destroy(sgp_b200_ctx_t *ctx);
const char *sgp_b200_last_error(void);
/* The stream all work of ctx is issued on (a cudaStream_t). */
void *sgp_b200_stream(sgp_b200_ctx_t *ctx);

/* memory kind of the pointers in a graph / result */
#define SGP_B200_HOST 0
#define SGP_B200_DEVICE 1

typedef struct {
    uint32_t n;
    uint64_t m;                 /* directed entries = row_ptr[n] */
    const uint32_t *row_ptr;    /* n + 1 */
    const uint32_t *col;        /* m */
    const uint32_t *w;          /* m or NULL (unit weights) */
    int mem;                    /* SGP_B200_HOST or SGP_B200_DEVICE */
} sgp_b200_graph_t;

typedef struct {
    uint32_t cutoff;            /* coarsen while n > cutoff (reference: 50) */
    double tol;                 /* power-iteration tolerance (reference: 1e-10) */
    int mixed;                  /* 0: FP64 SpMV; 1: mixed precision -- on levels of
                                   >= 4096 vertices the Laplacian is applied as
                                   sum_j w_ij (x_i - x_j) with FP32 differences,
                                   products and row sums; the iterate, shift,
                                   deflation, normalisation, dot product and
                                   stopping test stay FP64 */
    int perc_imbalance;         /* sgp_compute_partition's perc_imbalance_allowed */
    uint64_t iter_cap;          /* extra cap on power iterations per level, 0 = none */
    uint64_t rng_state, rng_inc;/* PCG32 seeding (advanced copy returned in result) */
    int part_mem;               /* memory kind of result->part */
    int refine_alg;             /* 0: shifted combinatorial Laplacian (reference default);
                                   1: normalized Laplacian, lazy random walk (I + D^-1 A) / 2
                                   without deflation in the loop, as eigensolve_kokkos.h:103-206 */
    int local_search_alg;       /* != 0: the reference's local search after the split
                                   (sgpar.h:2080-2170), as config_t.local_search_alg */
    uint32_t fm_passes;         /* > 0: up to this many FM passes on the final bisection
                                   (sgp_b200_fm_refine); 0 = none (the reference's spectral path) */
    int coarsener;              /* SGP_B200_COARSEN_*: the reference's compile-time coarsener
                                   choice (coarsen_kokkos.h:1138-1150); | SGP_B200_COARSEN_NONE
                                   skips coarsening, | SGP_B200_COARSEN_RATIO_STOP stops after a
                                   level keeping more than 0.9 of the vertices (sgpar.h:2466-2475) */
    uint32_t cluster_max_log2;  /* power-iteration levels above one block's shared memory and of at
                                   most 2^k cost units (entries + 8 per vertex) run on a cluster of
                                   blocks (one cluster barrier per iteration, several levels at
                                   once); larger ones on the whole GPU.  0 = the default: 17 for
                                   single partitions, 23 for sgp_b200_partition_batch, whose levels
                                   of many graphs then share the GPU.  Equal values give equal bits. */
    uint32_t cluster_blocks;    /* blocks per cluster of that kernel: 8 or 2.  0 = the default: 8 for
                                   single partitions (each level's latency), 2 for
                                   sgp_b200_partition_batch (twice as many hierarchies iterate at
                                   once; 2,048 graphs of 10^3..2.5*10^5 vertices: 10.6 -> 8.6 s).
                                   Equal values (with equal cluster_max_log2) give equal bits. */
} sgp_b200_options_t;

#define SGP_B200_COARSEN_HEC 0      /* heavy-edge coarsening, heuristics.h:930-1031 (default) */
#define SGP_B200_COARSEN_MATCH 1    /* heavy-edge matching, heuristics.h:1584-1740 (PUREMATCH) */
#define SGP_B200_COARSEN_MIS2 2     /* distance-2 independent-set aggregation, heuristics.h:8-80, :218-310 */
#define SGP_B200_COARSEN_GOSH 3     /* degree-keyed cluster aggregation, heuristics.h:81-216, :312-365 */
#define SGP_B200_COARSEN_HEC_V3 4   /* HEC with the pointer-jumping map construction, heuristics.h:766-834 */
#define SGP_B200_COARSEN_GOSH_V2 5  /* high-degree roots + joins + prefilled HEC rounds, heuristics.h:444-560 */
#define SGP_B200_COARSEN_NONE 16
#define SGP_B200_COARSEN_RATIO_STOP 32

#define SGP_B200_MAX_LEVELS 202

typedef struct {
    uint32_t *part;             /* n entries, caller-allocated (kind part_mem) */
    uint64_t edgecut;
    uint32_t part0_size;
    double lambda;              /* Rayleigh quotient of the finest vector */
    double residual;            /* ||L x - lambda x||_2 / (2 max_i d_i), x unit */
    int levels;
    uint32_t level_n[SGP_B200_MAX_LEVELS];
    uint64_t level_m[SGP_B200_MAX_LEVELS];
    uint64_t level_iters[SGP_B200_MAX_LEVELS];
    int level_hec_rounds[SGP_B200_MAX_LEVELS];
    float level_pi_ms[SGP_B200_MAX_LEVELS];   /* power-iteration kernel time per level (CUDA events) */
    int iter_max_reached;
    uint64_t rng_state;         /* rng after the call */
    float ms_total, ms_h2d, ms_coarsen, ms_eigen, ms_split, ms_d2h;
    uint32_t kernel_launches;
    float ms_map, ms_build;     /* coarsening split into HEC mapping and coarse builds */
    uint32_t ls_swaps;          /* local-search move pairs (local_search_alg != 0) */
    uint32_t fm_passes_run;     /* FM passes run (fm_passes > 0) */
    uint64_t fm_moves;          /* FM moves applied */
} sgp_b200_result_t;

void sgp_b200_default_options(sgp_b200_options_t *opt);

/* The options sgp_partition_graph (sgpar.h:2363) runs with for a config_t:
 * tolerance (the change_tol default when config->tol <= 0), refine_alg,
 * local_search_alg, the coarsener coarsening_alg's bits select (bit 4: none;
 * bit 0: heavy-edge matching with the 0.9 ratio stop; else HEC,
 * sgpar.h:2457-2475), perc_imbalance_allowed and the rng's state.
 * SGP_B200_ERR_INVALID for a refine_alg other than 0 or 1. */
int sgp_b200_config_options(const config_t *config, int perc_imbalance_allowed, const sgp_pcg32_random_t *rng,
                            sgp_b200_options_t *opt);

/* The whole path on one graph (the body of sgp_partition_graph). */
int sgp_b200_partition(sgp_b200_ctx_t *ctx, const sgp_b200_graph_t *g,
                       const sgp_b200_options_t *opt, sgp_b200_result_t *res);

/* The reference driver's 4-way mode (sgpar.cpp:62-89, num_partitions = 4):
 * bisect g, take the two induced subgraphs (sgp_use_partition,
 * sgpar.h:2666-2752), bisect each with the rng carried on from the previous
 * call.  All on the device.  part4 (n entries, kind opt->part_mem) gets
 * 2 * (bisection part) + (part inside its subgraph).  result4[0] = cut of the
 * bisection, result4[1] = cut4 = result4[0] + both subgraph cuts,
 * result4[2] = rng state after the three bisections.  Subgraph weights are
 * dropped, as sgp_use_partition drops them. */
int sgp_b200_partition_4way(sgp_b200_ctx_t *ctx, const sgp_b200_graph_t *g,
                            const sgp_b200_options_t *opt, uint32_t *part4, uint64_t *result4);

/* No counterpart in the reference (its experiment runner starts one process
 * per graph).  Partitions graphs[0..count) independently, each with opt as
 * given (the same rng seeding for every graph), into results[i] (whose part
 * the caller sets, kind opt->part_mem).  In waves of up to 1024 graphs:
 * `workers` host threads, each on its own stream of the context's device,
 * coarsen the graphs (largest first) and keep the hierarchies; one launch
 * then iterates the small coarse levels of every hierarchy (a block per
 * hierarchy at a time); the workers finish the larger levels and the splits.
 * The worker contexts are kept by ctx for later calls.  Results equal single
 * calls' and do not depend on `workers`; the per-graph phase times include
 * waiting for the shared launch.  On failure the first error is returned
 * and the message names the graph. */
int sgp_b200_partition_batch(sgp_b200_ctx_t *ctx, const sgp_b200_graph_t *graphs, int count,
                             const sgp_b200_options_t *opt, sgp_b200_result_t *results,
                             int workers);

/* ---- lower boundary: hierarchy handle (coarsen_kokkos.h:1165,
 *      eigensolve_kokkos.h:1493) ---- */
typedef struct sgp_b200_hierarchy sgp_b200_hierarchy_t;

/* Copy g to the device (when host) and coarsen it level by level.
 * rng is advanced by two PCG32 draws per level. */
int sgp_b200_generate_coarse_graphs(sgp_b200_ctx_t *ctx, const sgp_b200_graph_t *g,
                                    uint32_t cutoff, sgp_pcg32_random_t *rng,
                                    sgp_b200_hierarchy_t **out);
int sgp_b200_hierarchy_levels(const sgp_b200_hierarchy_t *h);
/* Device pointers of level l (0 = input graph); vcmap is NULL on the last
 * level; wbytes is 0 (unit), 4 or 8. */
int sgp_b200_hierarchy_level(const sgp_b200_hierarchy_t *h, int l, uint32_t *n, uint64_t *m,
                             const uint32_t **row_ptr, const uint32_t **col, const void **w,
                             int *wbytes, const uint32_t **vcmap);
/* Vertex weights of level l (device array of n entries): the number of
 * input vertices each vertex stands for, i.e. the fine weights summed over
 * each aggregate (coarsen_kokkos.h:1098 c_vtx_w); NULL for level 0, whose
 * vertices weigh 1. */
int sgp_b200_hierarchy_vertex_weights(const sgp_b200_hierarchy_t *h, int l, const uint32_t **vtx_w);
/* Fiedler vector of the finest level: coarsest guess from rng, power
 * iteration per level, prolongation; eigenvec has n_0 entries of kind mem. */
int sgp_b200_eigensolve(sgp_b200_ctx_t *ctx, sgp_b200_hierarchy_t *h, sgp_pcg32_random_t *rng,
                        double tol, int mixed, uint64_t iter_cap, double *eigenvec, int mem,
                        sgp_b200_result_t *stats);
void sgp_b200_hierarchy_free(sgp_b200_hierarchy_t *h);

/* ---- per-kernel entry points (device pointers, stream of ctx) ---- */

/* HEC mapping of one level (heuristics.h:930-1031): heavy neighbour hn[n]
 * and coarse map vcmap[n] onto [0, *nc).  random_level = 1 selects the
 * level-1 random neighbour of an unweighted graph.  wbytes: 0, 4 or 8. */
int sgp_b200_hec(sgp_b200_ctx_t *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                 const void *w, int wbytes, int random_level, uint64_t seed,
                 uint32_t *hn, uint32_t *vcmap, uint32_t *nc, int *rounds);

/* Coarse graph of one level (coarsen_kokkos.h:1061-1127): rows sorted by
 * destination, duplicate weights summed, self loops dropped.  c_row_ptr has
 * nc + 1 entries; c_col / c_w have capacity row_ptr[n] entries; out_wbytes is
 * 4 or 8 (weights of c_w).  *m_c receives the coarse entry count. */
int sgp_b200_build_coarse(sgp_b200_ctx_t *ctx, uint32_t n, const uint32_t *row_ptr,
                          const uint32_t *col, const void *w, int wbytes, const uint32_t *vcmap,
                          uint32_t nc, int out_wbytes, uint32_t *c_row_ptr, uint32_t *c_col,
                          void *c_w, uint64_t *m_c);

/* Power iteration of one level (eigensolve_kokkos.h:102-206): x_in is the
 * start vector (n entries) or, with vcmap != NULL, the coarse vector that
 * is prolongated (x_in[vcmap[i]], eigensolve_kokkos.h:1556-1559).  x_out
 * receives the normalised, deflated iterate of the start of the last
 * iteration (what the reference returns). */
int sgp_b200_power_iter(sgp_b200_ctx_t *ctx, uint32_t n, const uint32_t *row_ptr,
                        const uint32_t *col, const void *w, int wbytes, const double *x_in,
                        const uint32_t *vcmap, double *x_out, double tol, uint64_t iter_cap,
                        int mixed, uint64_t *niter, double *lambda, double *residual);

/* Median split + edge cut (sgpar.h:1969-2071) of a device eigenvector;
 * part is a device array of n entries. */
/* FM refinement of a bisection (device arrays; part[n] in {0, 1}, updated in
 * place): passes of gain-ordered moves in the structure of the reference's
 * parallel FM (eigensolve_kokkos.h:695-971) with the serial FM's balance
 * rule and imbalance target (:1073-1140), made deterministic -- each side's
 * positive-gain vertices by (gain clamped to 1023 descending, id), the sides
 * interleaved for balance, sequential gains, the best prefix within
 * max(|balance| / 10, 20) applied -- until a pass does not lower the cut or
 * max_passes.  Edges count 1 (the finest level).  *cut receives the cut. */
int sgp_b200_fm_refine(sgp_b200_ctx_t *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                       uint32_t *part, uint32_t max_passes, uint64_t *cut, uint32_t *passes, uint64_t *moves);

/* One level's mapping by an alternative coarsener (coarsener MATCH, MIS2,
 * GOSH, HEC_V3 or GOSH_V2; the HEC mapping is sgp_b200_hec) on device arrays: vcmap[n] receives
 * the coarse vertex of each vertex, *nc the coarse count, *rounds the
 * matching rounds or independent-set iterations. */
int sgp_b200_coarsen_map(sgp_b200_ctx_t *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                         const void *w, int wbytes, int coarsener, int random_level, uint64_t seed,
                         uint32_t *vcmap, uint32_t *nc, int *rounds);
int sgp_b200_split(sgp_b200_ctx_t *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                   const double *evec, int perc_imbalance, uint32_t *part, uint64_t *edgecut);

/* Largest vertex count of sgp_b200_split_noalloc (its fixed scratch). */
#define SGP_B200_NOALLOC_MAX_N (1u << 20)

/* No counterpart in the reference.  The same median split and edge cut as
 * sgp_b200_split, for callers that cannot allocate device memory at the time
 * of the call (a host application that owns every device allocation through
 * its own pool, code running in an out-of-memory handler, a plug-in whose
 * host forbids allocation): it allocates nothing and uses a fixed scratch
 * array inside the library (about 8 MiB per GPU, held until the process
 * exits).  At most SGP_B200_NOALLOC_MAX_N vertices; larger graphs return
 * SGP_B200_ERR_TOO_LARGE.  Asynchronous on `stream` (a cudaStream_t, NULL =
 * default stream): part (n entries) and result (device array: result[0] =
 * edge cut, result[1] = size of part 0) are valid once the stream has
 * reached the call (col may be NULL when the graph has no edges).  `stream`
 * must belong to the current device
 * (SGP_B200_ERR_INVALID otherwise).  The first call on a device looks up the
 * scratch address and should come before any stream capture; the look-up is
 * repeated when the device's context has changed (after cudaDeviceReset).
 * All calls on a device share the scratch: calls that overlap on the GPU
 * race and must be serialised. */
int sgp_b200_split_noalloc(void *stream, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                           const double *evec, uint32_t *part, uint64_t *result);

/* Appends the record of one partition to the JSON metrics file `path` in the
 * layout of the reference's ExperimentLoggerUtil::log
 * (ExperimentLoggerUtil.cpp:145-192): "[" before the first record (first
 * != 0), "," after every record but the last, "]" after the last (last != 0),
 * so the reference's experiment runner aggregates it unchanged.  Times follow
 * the reference's window (sgpar.h:2379-2407): total = upload + coarsening +
 * eigensolve (not the split), coarsen = upload + coarsening, refine =
 * eigensolve; coarsen-map / coarsen-build are the HEC and coarse-build shares;
 * the per-kernel timers this path does not have are 0.  coarse-levels lists
 * the levels coarsest first with their power iterations; the finest carries
 * the cut. */
int sgp_b200_write_metrics(const char *path, const sgp_b200_result_t *res, uint64_t edge_cut_4way,
                           uint64_t partition_diff, int first, int last);

/* ------------------------------------------------------------------------ *
 * Part 3: MatrixMarket input (replaces the cmg/mtx2csr.cpp command)          *
 * ------------------------------------------------------------------------ */

typedef struct {
    uint64_t rows, cols, entries_declared;  /* the size line */
    uint64_t lines;             /* lines after the size line (entries, comments, blank) */
    int bipartite;              /* 1: "general" rectangular matrix read as a bipartite graph */
    uint32_t n_all;             /* vertices before the component filter */
    uint64_t m_all;             /* directed entries after dedupe and self-loop removal */
    uint32_t components;        /* connected components, isolated vertices included */
    uint32_t n;                 /* vertices of the largest component (the output) */
    uint64_t m;                 /* its directed entries */
    float ms_total;             /* whole call (host clock) */
    float ms_read;              /* file read + copy of the text to the device (host clock) */
    float ms_parse, ms_rows, ms_components, ms_extract;   /* device phases (CUDA events) */
    float ms_out;               /* result copy-out (host clock) */
    uint32_t kernel_launches;   /* kernels this call launched */
} sgp_b200_mtx_info_t;

/* MatrixMarket coordinate text -> symmetric CSR of its largest connected
 * component, computed on the device.  Same rules and output as
 * cmg/mtx2csr.cpp:13-264: banner lines must say "coordinate"; "general"
 * reads a square matrix as A + A^T and a rectangular one as a bipartite graph
 * (columns are vertices 0..cols-1, rows cols..cols+rows-1); every entry adds
 * both directions, self loops dropped unless bipartite, values ignored; rows
 * sorted with duplicates removed; the largest component kept (the first in
 * vertex order among equally large ones), renumbered in ascending order.
 * Where the reference's behaviour is undefined (an id of 0 or beyond the size
 * line, an entry line that is not "i j ...", a "symmetric" banner on a
 * non-square size line, a later banner that switches to "general") the call
 * fails with SGP_B200_ERR_INVALID naming the line; blank lines are skipped.
 *
 * `out` receives library-allocated arrays (out->w NULL) of kind out_mem
 * (SGP_B200_HOST: malloc; SGP_B200_DEVICE: cudaMalloc on the context's device);
 * release them with sgp_b200_graph_free.  `info` may be NULL. */
int sgp_b200_mtx_read(sgp_b200_ctx_t *ctx, const char *mtx_path, int out_mem, sgp_b200_graph_t *out,
                      sgp_b200_mtx_info_t *info);
/* The same from `len` bytes of file text at `text` (kind text_mem). */
int sgp_b200_mtx_parse(sgp_b200_ctx_t *ctx, const char *text, uint64_t len, int text_mem, int out_mem,
                       sgp_b200_graph_t *out, sgp_b200_mtx_info_t *info);
void sgp_b200_graph_free(sgp_b200_graph_t *g);
/* Writes a host graph as the reference's binary CSR file (mtx2csr.cpp:266-289):
 * six 64-bit words n, m (directed entries), 1, 0, 1, 0, then row offsets[n+1]
 * and destinations[m] as 32-bit words (id_bytes 4) or 64-bit words (id_bytes
 * 8, the layout of cmg/mtx2csr_large.cpp). */
int sgp_b200_csr_write(const char *csr_path, const sgp_b200_graph_t *g, int id_bytes);
/* The command `mtx2csr <MM file> <binary CSR file>`: read + write. */
int sgp_b200_mtx2csr(sgp_b200_ctx_t *ctx, const char *mtx_path, const char *csr_path, int id_bytes,
                     sgp_b200_mtx_info_t *info);

/* The power iteration's autotuner (no counterpart in the reference, whose
 * SpMV launch shape follows fixed rules, kokkos-kernels
 * KokkosSparse_spmv_impl.hpp:222-258).  The first time a level of a given
 * shape (weight width, relabelled or not, precision, octave of the vertex
 * count, half octave of the mean degree) and at least 2^18 cost units is
 * iterated on a kind of device, candidate work splits -- SpMV variant, long-row
 * threshold, grid size -- run ten trial iterations each into scratch memory
 * and the fastest is kept for every later level of that shape, in memory and
 * in the file the environment variable SGPB_TUNE_CACHE names (default
 * $HOME/.cache/sgpar_b200/pi_tune.txt; empty: memory only).  Results then depend
 * on the kept split only through the order of floating-point sums, and are
 * reproducible while it stays.  SGPB_AUTOTUNE=0 uses the built-in rules.
 * sgp_b200_autotune_clear forgets this process's splits (they are read from
 * the file, or tuned, again). */
void sgp_b200_autotune_clear(void);

/* Milliseconds of the phases of the last sgp_b200_partition / eigensolve
 * (CUDA events).  After sgp_b200_partition_batch: host wall time of its
 * phases summed over the waves -- coarsening (ms_coarsen), the shared launch
 * of the small levels (ms_eigen), the remaining levels and the splits
 * (ms_split), and their sum (ms_total). */
int sgp_b200_last_timing(sgp_b200_ctx_t *ctx, float *ms_total, float *ms_coarsen,
                         float *ms_eigen, float *ms_split);

#ifdef __cplusplus
}
#endif
#endif /* SGPAR_B200_H_ */
