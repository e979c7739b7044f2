/*
 * sgpar_oracle.c -- CPU restatement of cmg's multilevel spectral bisection path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The shipped library never links or calls it.
 *
 * What it restates (reference files under cmg/ of IPDPS_2021_Graph_Coarsening):
 *   - PCG32 (sgpar.h:82-92)
 *   - heavy-neighbour choice of HEC (heuristics.h:959-998; serial form
 *     sgpar.h:647-695), with the deterministic tie-break this project defines
 *   - HEC map construction rounds (heuristics.h:633-693), made deterministic:
 *     claims are resolved by a max-key rule instead of compare-and-swap races
 *   - coarse-graph construction P^T A P minus self loops with integer weight
 *     sums and rows sorted by destination (coarsen_kokkos.h:1061-1127,
 *     799-900 and the RADIX dedupe 750-762 / 491-509)
 *   - shifted-Laplacian power iteration deflated against the constant vector,
 *     in the serial reference's exact floating-point operation order
 *     (sgpar.h:1790-1948, vector kernels sgpar.h:1687-1730)
 *   - median split + one-vertex sweep + edge cut (sgpar.h:1969-2071) and the
 *     local search after it (sgpar.h:2080-2170)
 *   - a deterministic parallel-form FM pass (structure of fm_refine_par,
 *     eigensolve_kokkos.h:695-971, acceptance target of fm_refine :1073)
 *   - induced sub-graphs for 4-way recursion (sgpar.h:2666-2752)
 *   - the level loop of sgp_generate_coarse_graphs (coarsen_kokkos.h:1165-1234)
 *     and sgp_eigensolve (eigensolve_kokkos.h:1493-1595)
 *   - the alternative coarseners MATCH, MIS-2 and GOSH (heuristics.h:8-365,
 *     :1584-1740) with this project's deterministic rules
 *
 * Parity pins: the power iteration, the split and the coarse build are checked
 * against the reference's own serial build compiled from its sources
 * (oracle/ref_harness.cpp); the dedupe is checked against the reference's
 * known-answer test (tests.cpp:7-56).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_UNASSIGNED 0xFFFFFFFFu

/* ---------------------------------------------------------------- PCG32 -- */
/* sgpar.h:84-92: 64-bit LCG state, XSH-RR output permutation. */
uint32_t orc_pcg32(uint64_t *state, uint64_t inc) {
    uint64_t old = *state;
    *state = old * 6364136223846793005ULL + (inc | 1);
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}

/* ------------------------------------------------------- seeded hashes -- */
/* The reference draws vertex priorities from a time-seeded XorShift pool
 * (heuristics.h:614-631, :947).  This project replaces that by counter-based
 * hashes of (level seed, vertex) so that the mapping is reproducible.  The same
 * three formulas are used by the CUDA kernels. */
static inline uint64_t orc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
/* 63-bit priority key: 31 hash bits above the 32-bit vertex id (unique). */
static inline uint64_t orc_prio_key(uint64_t seed, uint32_t u) {
    uint64_t h = orc_mix64(seed ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)u + 1)));
    return ((h >> 33) << 32) | (uint64_t)u;
}
/* random draw for the level-1 random neighbour and isolated vertices */
static inline uint64_t orc_rand_draw(uint64_t seed, uint32_t u) {
    return orc_mix64(seed ^ 0x632BE59BD9B4E019ULL ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)u + 1)));
}
/* tie-break among equally heavy edges (u -> v) */
static inline uint32_t orc_tiebreak(uint64_t seed, uint32_t u, uint32_t v) {
    return (uint32_t)(orc_mix64(seed ^ 0xD1B54A32D192ED03ULL ^ (((uint64_t)u << 32) | v)) >> 32);
}

uint64_t orc_hash_prio_key(uint64_t seed, uint32_t u) { return orc_prio_key(seed, u); }
uint64_t orc_hash_rand_draw(uint64_t seed, uint32_t u) { return orc_rand_draw(seed, u); }
uint32_t orc_hash_tiebreak(uint64_t seed, uint32_t u, uint32_t v) { return orc_tiebreak(seed, u, v); }

/* ------------------------------------------------------ heavy neighbour -- */
/* heuristics.h:959-998.  Level 1 of an unweighted input picks a random
 * neighbour (all weights are 1 there, heuristics.h:959-972); otherwise the
 * neighbour of maximum weight, ties broken by (tiebreak hash, destination).
 * A vertex with no edges is paired with a random vertex (urand % n, :967-970).
 * w64 == NULL means unit weights. */
void orc_hec_heavy(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                   const uint64_t *w64, int random_level, uint64_t seed,
                   uint32_t *hn) {
    for (uint32_t u = 0; u < n; u++) {
        uint32_t b = row_ptr[u], e = row_ptr[u + 1];
        uint32_t deg = e - b;
        if (deg == 0) {
            hn[u] = (uint32_t)(orc_rand_draw(seed, u) % n);
            continue;
        }
        if (random_level) {
            hn[u] = col[b + (uint32_t)(orc_rand_draw(seed, u) % deg)];
            continue;
        }
        uint64_t bw = 0; uint32_t bt = 0, bv = 0; int have = 0;
        for (uint32_t j = b; j < e; j++) {
            uint64_t w = w64 ? w64[j] : 1;
            uint32_t v = col[j];
            uint32_t t = orc_tiebreak(seed, u, v);
            if (!have || w > bw || (w == bw && (t > bt || (t == bt && v > bv)))) {
                bw = w; bt = t; bv = v; have = 1;
            }
        }
        hn[u] = bv;
    }
}

/* ----------------------------------------------------- map construction -- */
/* heuristics.h:633-693 (parallel_map_construct), restated deterministically.
 *
 * Each round looks at the still-unassigned vertices u with v = hn[u]:
 *   - v already assigned in an earlier round: u joins v's aggregate
 *     (heuristics.h:664-666) and shields its own slot from claims;
 *   - v == u: u becomes a singleton aggregate (the u == v case at :656);
 *   - (prio(u) < prio(v)) xor swap (the ordering condition of :653-654):
 *     u claims both slots u and v with key(u)+1 (atomic max on the GPU);
 *     u wins when it holds both slots, and u, v form a new aggregate
 *     (the double compare-and-swap of :655-661).
 * swap flips every round (:684).  Aggregates are labelled by their root vertex
 * during the rounds and numbered by ascending root id at the end, so the
 * coarse numbering does not depend on thread timing (the reference uses an
 * atomic counter, :657).
 * Returns the number of rounds; nc receives the coarse vertex count. */
/* prefilled: vcmap already holds aggregates (members point to their root
 * vertex, roots to themselves, the rest ORC_UNASSIGNED), as in
 * parallel_map_construct_prefilled (heuristics.h:378-443) */
int orc_hec_map_pre(uint32_t n, const uint32_t *hn, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out,
                    int prefilled) {
    const uint64_t JOIN_KEY = ~0ULL, SELF_KEY = ~0ULL - 1;
    uint64_t *claim[2];
    claim[0] = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    claim[1] = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    uint8_t *act = (uint8_t *)malloc(n ? n : 1);
    uint32_t *list = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t *next = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    for (uint32_t u = 0; u < n; u++) {
        if (!prefilled) vcmap[u] = ORC_UNASSIGNED;
        list[u] = u;
    }
    uint32_t len = n;
    int swap = 1, round = 0;
    while (1) {
        uint64_t *cl = claim[round & 1], *other = claim[(round + 1) & 1];
        /* phase A: compact the survivors, classify, claim */
        uint32_t nlen = 0;
        for (uint32_t i = 0; i < len; i++) {
            uint32_t u = list[i];
            if (vcmap[u] != ORC_UNASSIGNED) continue;
            next[nlen++] = u;
            uint32_t v = hn[u];
            if (vcmap[v] != ORC_UNASSIGNED) {
                act[u] = 1; if (cl[u] < JOIN_KEY) cl[u] = JOIN_KEY;
            } else if (v == u) {
                act[u] = 2; if (cl[u] < SELF_KEY) cl[u] = SELF_KEY;
            } else {
                uint64_t ku = orc_prio_key(seed, u), kv = orc_prio_key(seed, v);
                int cond = ku < kv;
                if (cond ^ swap) {
                    act[u] = 3;
                    uint64_t k = ku + 1;
                    if (cl[u] < k) cl[u] = k;
                    if (cl[v] < k) cl[v] = k;
                } else {
                    act[u] = 0;
                }
            }
        }
        if (nlen == 0) break;
        /* phase B: resolve (reads the phase-A state only: joins read vcmap of
         * vertices assigned in earlier rounds, winners write slots they own) */
        for (uint32_t i = 0; i < nlen; i++) {
            uint32_t u = next[i];
            uint32_t v = hn[u];
            if (act[u] == 1) {
                vcmap[u] = vcmap[v];
            } else if (act[u] == 2) {
                vcmap[u] = u;
            } else if (act[u] == 3) {
                uint64_t k = orc_prio_key(seed, u) + 1;
                if (cl[u] == k && cl[v] == k) { vcmap[u] = u; vcmap[v] = u; }
            }
            other[u] = 0;
        }
        /* note: a join in phase B reads vcmap[v] for v assigned before this
         * round; winners only write vertices unassigned before this round, so
         * the sequential order of phase B is irrelevant. */
        uint32_t *t = list; list = next; next = t; len = nlen;
        swap ^= 1; round++;
    }
    /* number aggregates by ascending root id (roots have vcmap[r] == r) */
    uint32_t *rank = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t nc = 0;
    for (uint32_t u = 0; u < n; u++) { rank[u] = nc; if (vcmap[u] == u) nc++; }
    for (uint32_t u = 0; u < n; u++) vcmap[u] = rank[vcmap[u]];
    *nc_out = nc;
    free(rank); free(claim[0]); free(claim[1]); free(act); free(list); free(next);
    return round;
}

int orc_hec_map(uint32_t n, const uint32_t *hn, uint64_t seed, uint32_t *vcmap, uint32_t *nc_out) {
    return orc_hec_map_pre(n, hn, seed, vcmap, nc_out, 0);
}

/* HEC validity (invariant of the serial form, sgpar.h:686-695):
 * vcmap maps onto [0, nc); every u shares its aggregate with hn[u] or with
 * some w with hn[w] == u.  Returns 0 when valid, else 1 + failing vertex kind. */
int orc_hec_check(uint32_t n, const uint32_t *hn, const uint32_t *vcmap, uint32_t nc) {
    uint8_t *seen = (uint8_t *)calloc(nc ? nc : 1, 1);
    uint8_t *ok = (uint8_t *)calloc(n ? n : 1, 1);
    int rc = 0;
    for (uint32_t u = 0; u < n && !rc; u++) {
        if (vcmap[u] >= nc) { rc = 1; break; }
        seen[vcmap[u]] = 1;
        if (hn[u] >= n) { rc = 2; break; }
        if (vcmap[u] == vcmap[hn[u]]) ok[u] = 1;
    }
    for (uint32_t w = 0; w < n && !rc; w++)
        if (vcmap[w] == vcmap[hn[w]]) ok[hn[w]] = 1;
    for (uint32_t u = 0; u < n && !rc; u++) if (!ok[u]) rc = 3;
    for (uint32_t c = 0; c < nc && !rc; c++) if (!seen[c]) rc = 4;
    free(seen); free(ok);
    return rc;
}

/* ---------------------------------------------------- coarse-graph build -- */
static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}
typedef struct { uint32_t v; uint64_t w; } orc_vw_t;
static int cmp_vw(const void *a, const void *b) {
    uint32_t x = ((const orc_vw_t *)a)->v, y = ((const orc_vw_t *)b)->v;
    return x < y ? -1 : x > y;
}

/* coarsen_kokkos.h:1061-1127 + 799-900 + 750-762: map every fine entry
 * (u, v, w) to (vcmap[u], vcmap[v], w), drop self loops, bucket by coarse
 * source, sort by destination and sum duplicate weights (64-bit sums).
 * Coarse vertex weights: c_vw[vcmap[u]] += f_vw[u] (coarsen_kokkos.h:1098).
 * c_col / c_w must hold at least row_ptr[n] entries.  Returns m_c. */
uint64_t orc_build_coarse(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                          const uint64_t *w64, const uint32_t *vcmap, uint32_t nc,
                          const uint64_t *f_vw, uint64_t *c_vw,
                          uint32_t *c_row_ptr, uint32_t *c_col, uint64_t *c_w) {
    uint32_t *cnt = (uint32_t *)calloc((size_t)nc + 1, sizeof(uint32_t));
    for (uint32_t u = 0; u < n; u++) {
        uint32_t cu = vcmap[u];
        for (uint32_t j = row_ptr[u]; j < row_ptr[u + 1]; j++)
            if (vcmap[col[j]] != cu) cnt[cu]++;
    }
    uint32_t *bo = (uint32_t *)malloc(((size_t)nc + 1) * sizeof(uint32_t));
    bo[0] = 0;
    for (uint32_t c = 0; c < nc; c++) bo[c + 1] = bo[c] + cnt[c];
    orc_vw_t *bucket = (orc_vw_t *)malloc(((size_t)bo[nc] + 1) * sizeof(orc_vw_t));
    memset(cnt, 0, ((size_t)nc + 1) * sizeof(uint32_t));
    for (uint32_t u = 0; u < n; u++) {
        uint32_t cu = vcmap[u];
        for (uint32_t j = row_ptr[u]; j < row_ptr[u + 1]; j++) {
            uint32_t cv = vcmap[col[j]];
            if (cv == cu) continue;
            orc_vw_t *e = &bucket[bo[cu] + cnt[cu]++];
            e->v = cv; e->w = w64 ? w64[j] : 1;
        }
    }
    if (c_vw) {
        for (uint32_t c = 0; c < nc; c++) c_vw[c] = 0;
        for (uint32_t u = 0; u < n; u++) c_vw[vcmap[u]] += f_vw ? f_vw[u] : 1;
    }
    uint64_t m = 0;
    c_row_ptr[0] = 0;
    for (uint32_t c = 0; c < nc; c++) {
        orc_vw_t *r = bucket + bo[c];
        uint32_t len = bo[c + 1] - bo[c];
        qsort(r, len, sizeof(orc_vw_t), cmp_vw);   /* weights are summed below, so stability is irrelevant */
        for (uint32_t i = 0; i < len; i++) {
            if (i > 0 && r[i].v == r[i - 1].v) { c_w[m - 1] += r[i].w; continue; }
            c_col[m] = r[i].v; c_w[m] = r[i].w; m++;
        }
        c_row_ptr[c + 1] = (uint32_t)m;
    }
    free(cnt); free(bo); free(bucket);
    (void)cmp_u32;
    return m;
}

/* Per-row dedupe of a bucketed row (the contract the reference's tests.cpp
 * pins for heap_deduplicate / hashmap_deduplicate): returns the distinct
 * count, rows written sorted by destination with summed weights. */
uint32_t orc_dedupe_row(uint32_t len, uint32_t *dst, uint64_t *w) {
    orc_vw_t *r = (orc_vw_t *)malloc((len ? len : 1) * sizeof(orc_vw_t));
    for (uint32_t i = 0; i < len; i++) { r[i].v = dst[i]; r[i].w = w[i]; }
    qsort(r, len, sizeof(orc_vw_t), cmp_vw);
    uint32_t m = 0;
    for (uint32_t i = 0; i < len; i++) {
        if (m > 0 && r[i].v == dst[m - 1]) { w[m - 1] += r[i].w; continue; }
        dst[m] = r[i].v; w[m] = r[i].w; m++;
    }
    free(r);
    return m;
}

/* ------------------------------------------------------ power iteration -- */
/* sgpar.h:1790-1948 (serial sgp_power_iter, normLap = 0) with the serial
 * vector kernels sgpar.h:1687-1730, in the same operation order so that the
 * result is bit-identical to the reference serial build on the same CSR.
 * gb = max_i 2 d_i, floored at 2 as in eigensolve_kokkos.h:126-135.
 * On return u holds the iterate from the start of the last iteration (the
 * reference returns u, not v).  Returns the iteration count. */
uint64_t orc_power_iter(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                        const uint64_t *w64, double *u, double tol, uint64_t iter_cap,
                        double *lambda_out) {
    double *vec1 = (double *)malloc((size_t)n * sizeof(double));
    double *v = (double *)malloc((size_t)n * sizeof(double));
    uint64_t *d = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    uint64_t gb = 2;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t s = 0;
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) s += w64 ? w64[j] : 1;
        d[i] = s;
        if (gb < 2 * s) gb = 2 * s;
    }
    uint64_t iter_max = 100000000000000ULL / (uint64_t)n;
    if (iter_cap && iter_max > iter_cap) iter_max = iter_cap;
    /* vec1 = 1, normalise (sgpar.h:1687-1703) */
    double ss = 0;
    for (uint32_t i = 0; i < n; i++) { vec1[i] = 1.0; }
    for (uint32_t i = 0; i < n; i++) ss += vec1[i] * vec1[i];
    double inv = 1 / sqrt(ss);
    for (uint32_t i = 0; i < n; i++) vec1[i] = vec1[i] * inv;
    /* orthogonalise u against vec1 (sgpar.h:1721-1730), normalise */
    double mult = 0;
    for (uint32_t i = 0; i < n; i++) mult += u[i] * vec1[i];
    for (uint32_t i = 0; i < n; i++) u[i] -= mult * vec1[i];
    ss = 0;
    for (uint32_t i = 0; i < n; i++) ss += u[i] * u[i];
    inv = 1 / sqrt(ss);
    for (uint32_t i = 0; i < n; i++) u[i] = u[i] * inv;
    for (uint32_t i = 0; i < n; i++) v[i] = u[i];
    double dot = 0, last = 1;
    uint64_t niter = 0;
    while (fabs(dot - last) > tol && niter < iter_max) {
        for (uint32_t i = 0; i < n; i++) u[i] = v[i];
        for (uint32_t i = 0; i < n; i++) {
            double vi = (double)(gb - d[i]) * u[i];
            double mv = 0;
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) {
                if (w64) mv += u[col[j]] * (double)w64[j];
                else mv += u[col[j]];
            }
            vi += mv;
            v[i] = vi;
        }
        mult = 0;
        for (uint32_t i = 0; i < n; i++) mult += v[i] * vec1[i];
        for (uint32_t i = 0; i < n; i++) v[i] -= mult * vec1[i];
        ss = 0;
        for (uint32_t i = 0; i < n; i++) ss += v[i] * v[i];
        inv = 1 / sqrt(ss);
        for (uint32_t i = 0; i < n; i++) v[i] = v[i] * inv;
        last = dot;
        dot = 0;
        for (uint32_t i = 0; i < n; i++) dot += u[i] * v[i];
        niter++;
    }
    if (lambda_out) {
        /* Rayleigh quotient of the returned vector: u.Lu / u.u */
        double num = 0, den = 0;
        for (uint32_t i = 0; i < n; i++) {
            double lu = (double)d[i] * u[i];
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++)
                lu -= (w64 ? (double)w64[j] : 1.0) * u[col[j]];
            num += u[i] * lu; den += u[i] * u[i];
        }
        *lambda_out = num / den;
    }
    free(vec1); free(v); free(d);
    return niter;
}

/* sgpar.h:1790-1948 with normLap = 1 (refine_alg 1; eigensolve_kokkos.h
 * :103-206 is the same recurrence), non-final form: d = weighted degrees.
 * The start vector is D-orthogonalised against the normalised constant
 * vector (sgpar.h:1732-1757: u -= (u.D1 / 1.D1) 1 with 1 normalised) and
 * normalised; each iteration v_i = 0.5 u_i + 0.5 (A u)_i / d_i, v normalised
 * (no deflation inside the loop), dot = u.v.  Same operation order as the
 * reference serial build.  *lambda_out: eigenvalue of the random-walk
 * Laplacian from the Rayleigh quotient of the lazy walk, 2 (1 - u.Mu / u.u).
 * A vertex of degree 0 contributes 0.5 u_i (the reference divides by 0). */
uint64_t orc_power_iter_nl(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                           const uint64_t *w64, double *u, double tol, uint64_t iter_cap,
                           double *lambda_out) {
    double *vec1 = (double *)malloc((size_t)n * sizeof(double));
    double *v = (double *)malloc((size_t)n * sizeof(double));
    uint64_t *d = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    for (uint32_t i = 0; i < n; i++) {
        uint64_t s = 0;
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) s += w64 ? w64[j] : 1;
        d[i] = s;
    }
    uint64_t iter_max = 100000000000000ULL / (uint64_t)n;
    if (iter_cap && iter_max > iter_cap) iter_max = iter_cap;
    double ss = 0;
    for (uint32_t i = 0; i < n; i++) vec1[i] = 1.0;
    for (uint32_t i = 0; i < n; i++) ss += vec1[i] * vec1[i];
    double inv = 1 / sqrt(ss);
    for (uint32_t i = 0; i < n; i++) vec1[i] = vec1[i] * inv;
    /* D-orthogonalise u against vec1 (sgpar.h:1732-1757) */
    double numer = 0, denom = 0;
    for (uint32_t i = 0; i < n; i++) {
        numer += u[i] * (double)d[i] * vec1[i];
        denom += vec1[i] * (double)d[i] * vec1[i];
    }
    for (uint32_t i = 0; i < n; i++) u[i] -= numer * vec1[i] / denom;
    ss = 0;
    for (uint32_t i = 0; i < n; i++) ss += u[i] * u[i];
    inv = 1 / sqrt(ss);
    for (uint32_t i = 0; i < n; i++) u[i] = u[i] * inv;
    for (uint32_t i = 0; i < n; i++) v[i] = u[i];
    double dot = 0, last = 1;
    uint64_t niter = 0;
    while (fabs(dot - last) > tol && niter < iter_max) {
        for (uint32_t i = 0; i < n; i++) u[i] = v[i];
        for (uint32_t i = 0; i < n; i++) {
            const double dinv = 1.0 / (double)d[i];
            double vi = 0.5 * u[i];
            double mv = 0;
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) {
                if (w64) mv += u[col[j]] * (double)w64[j];
                else mv += u[col[j]];
            }
            if (d[i]) vi += 0.5 * mv * dinv;
            v[i] = vi;
        }
        ss = 0;
        for (uint32_t i = 0; i < n; i++) ss += v[i] * v[i];
        inv = 1 / sqrt(ss);
        for (uint32_t i = 0; i < n; i++) v[i] = v[i] * inv;
        last = dot;
        dot = 0;
        for (uint32_t i = 0; i < n; i++) dot += u[i] * v[i];
        niter++;
    }
    if (lambda_out) {
        double num = 0, den = 0;
        for (uint32_t i = 0; i < n; i++) {
            double mv = 0;
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) mv += (w64 ? (double)w64[j] : 1.0) * u[col[j]];
            const double mu = 0.5 * u[i] + (d[i] ? 0.5 * mv / (double)d[i] : 0.0);
            num += u[i] * mu; den += u[i] * u[i];
        }
        *lambda_out = 2.0 * (1.0 - num / den);
    }
    free(vec1); free(v); free(d);
    return niter;
}

/* ------------------------------------------------------------ the split -- */
typedef struct { double ev; uint32_t u; } orc_vu_t;
static int cmp_vu(const void *a, const void *b) {
    const orc_vu_t *x = (const orc_vu_t *)a, *y = (const orc_vu_t *)b;
    if (x->ev < y->ev) return -1;
    if (x->ev > y->ev) return 1;
    return x->u < y->u ? -1 : x->u > y->u;
}

/* sgpar.h:1969-2071 with local_search_alg = 0: sort (ev, u) ascending, the
 * first n - imbr vertices go to part 0, the rest to part 1, then vertices at
 * positions [imbl, imbr) are moved to part 0 while that does not raise the
 * cut (the running cut is not reverted after a rejected move, as in the
 * reference).  Edge cut counts directed cross entries / 2. */
int orc_compute_partition(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                          const double *evec, int perc_imbalance_allowed,
                          uint32_t *part, uint64_t *edgecut) {
    orc_vu_t *vu = (orc_vu_t *)malloc((size_t)(n ? n : 1) * sizeof(orc_vu_t));
    for (uint32_t i = 0; i < n; i++) { vu[i].ev = evec[i]; vu[i].u = i; }
    qsort(vu, n, sizeof(orc_vu_t), cmp_vu);
    long max_part_size = (long)ceil(n / 2.0);
    uint32_t imbr = (uint32_t)floor(max_part_size * (1.0 + perc_imbalance_allowed / 100.0));
    uint32_t imbl = n - imbr;
    for (uint32_t i = 0; i < imbl; i++) part[vu[i].u] = 0;
    for (uint32_t i = imbl; i < n; i++) part[vu[i].u] = 1;
    long cur = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++)
            if (part[col[j]] != part[i]) cur++;
    long best = cur;
    for (uint32_t i = imbl; i < imbr; i++) {
        uint32_t u = vu[i].u;
        long upd = 0;
        for (uint32_t j = row_ptr[u]; j < row_ptr[u + 1]; j++)
            upd += (part[col[j]] == 1) ? 1 : -1;
        cur = cur + 2 * upd;
        if (cur <= best) { part[u] = 0; best = cur; }
    }
    *edgecut = (uint64_t)(best / 2);
    free(vu);
    return 0;
}

/* sgpar.h:2080-2170: the local search after the split.  With curr_split the
 * part-0 size left by the split, it alternates: among vertex ids
 * [curr_split - n/3, curr_split) the first id of largest positive gain
 * (cross minus same-side neighbours) is flipped, then among
 * [curr_split, curr_split + n/3) likewise; a missing second move undoes the
 * first and ends the search, as does a missing first move or n/3 completed
 * pairs.  Gains are kept incrementally here (the reference recomputes them
 * per candidate); the values are the same integers.  Returns the swaps. */
uint32_t orc_local_search(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint32_t *part,
                          uint32_t curr_split) {
    int64_t *g = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
    for (uint32_t i = 0; i < n; i++) {
        int64_t x = 0;
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) x += part[col[j]] != part[i] ? 1 : -1;
        g[i] = x;
    }
    int64_t lo = (int64_t)curr_split - n / 3, hi = (int64_t)curr_split + n / 3;
    if (lo < 0) lo = 0;
    if (hi > (int64_t)n) hi = n;
    uint32_t swaps = 0, max_swaps = n / 3;
    while (swaps < max_swaps) {
        uint32_t pick[2];
        int side;
        for (side = 0; side < 2; side++) {
            int64_t a = side == 0 ? lo : curr_split, b = side == 0 ? (int64_t)curr_split : hi;
            int64_t best = 0;
            pick[side] = ORC_UNASSIGNED;
            for (int64_t i = a; i < b; i++)
                if (g[i] > best) { best = g[i]; pick[side] = (uint32_t)i; }
            if (pick[side] == ORC_UNASSIGNED) break;
            uint32_t v = pick[side], old = part[v];
            part[v] = 1 - old;
            g[v] = -g[v];
            for (uint32_t j = row_ptr[v]; j < row_ptr[v + 1]; j++) g[col[j]] += part[col[j]] != old ? -2 : 2;
        }
        if (side == 0) break;
        if (side == 1) {   /* roll the first move back */
            uint32_t v = pick[0], old = part[v];
            part[v] = 1 - old;
            g[v] = -g[v];
            for (uint32_t j = row_ptr[v]; j < row_ptr[v + 1]; j++) g[col[j]] += part[col[j]] != old ? -2 : 2;
            break;
        }
        swaps++;
    }
    free(g);
    return swaps;
}

/* The split of orc_compute_partition followed by the local search; the
 * part-0 size after the split is the reference's curr_split when
 * perc_imbalance_allowed is 0 (the sweep range holds at most one vertex). */
int orc_compute_partition_ls(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const double *evec,
                             int local_search_alg, uint32_t *part, uint64_t *edgecut, uint32_t *swaps_out) {
    orc_compute_partition(n, row_ptr, col, evec, 0, part, edgecut);
    uint32_t swaps = 0;
    if (local_search_alg) {
        uint32_t p0 = 0;
        for (uint32_t i = 0; i < n; i++) p0 += part[i] == 0;
        swaps = orc_local_search(n, row_ptr, col, part, p0);
        uint64_t c = 0;
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) c += part[col[j]] != part[i];
        *edgecut = c / 2;
    }
    if (swaps_out) *swaps_out = swaps;
    return 0;
}

/* ------------------------------------------------------ FM refinement -- */
/* A deterministic, parallel-form FM pass after the split, following the
 * structure of the reference's parallel FM (eigensolve_kokkos.h:695-971,
 * fm_refine_par) and the acceptance target of its serial FM
 * (:1073-1076: target imbalance max(|balance| / 10, 20)):
 *   1. gain(u) = sum over neighbours of w * (+1 across the cut, -1 inside);
 *   2. the vertices of positive gain of each side, ordered by (gain clamped
 *      to ORC_FM_BUCKETS - 1, descending; id ascending);
 *   3. the two lists interleaved by the serial FM's balance rule
 *      (:1105-1140): take from side 0 while the balance (part-0 minus part-1
 *      vertices) is positive, from side 1 while negative, at zero the head of
 *      larger gain (side 0 on a tie), the other list once one runs out;
 *   4. sequential gains: gain of u given that every vertex before it in the
 *      order has moved; cut after k moves = cut - sum of the first k;
 *   5. k* = the k (0 included) of least cut among those whose |balance| is
 *      within the target, the largest such k on a tie (the serial FM's
 *      "<="); the first k* moves are applied.
 * Passes repeat until one applies no move or leaves the cut unchanged, at
 * most max_passes.  Vertex weights are 1 (the finest level).  Returns the
 * passes run; *moves_out the moves applied in all. */
#define ORC_FM_BUCKETS 1024
typedef struct { int64_t g; uint32_t u; } orc_fmc_t;
static int orc_fm_cmp(const void *a, const void *b) {
    const orc_fmc_t *x = (const orc_fmc_t *)a, *y = (const orc_fmc_t *)b;
    int64_t gx = x->g < ORC_FM_BUCKETS - 1 ? x->g : ORC_FM_BUCKETS - 1;
    int64_t gy = y->g < ORC_FM_BUCKETS - 1 ? y->g : ORC_FM_BUCKETS - 1;
    if (gx != gy) return gx > gy ? -1 : 1;
    return x->u < y->u ? -1 : (x->u > y->u);
}

uint32_t orc_fm_refine(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const uint64_t *w,
                       uint32_t *part, uint32_t max_passes, uint64_t *cut_io, uint64_t *moves_out) {
    int64_t *gain = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
    uint32_t *rank = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t *seq = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    int64_t *gseq = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
    orc_fmc_t *A = (orc_fmc_t *)malloc(((size_t)n + 1) * sizeof(orc_fmc_t));
    orc_fmc_t *B = (orc_fmc_t *)malloc(((size_t)n + 1) * sizeof(orc_fmc_t));
    uint64_t moves = 0;
    uint32_t pass = 0;
    for (; pass < max_passes; pass++) {
        int64_t cut = 0, bal = 0;
        uint32_t na = 0, nb = 0;
        for (uint32_t u = 0; u < n; u++) {
            int64_t g = 0;
            for (uint32_t j = row_ptr[u]; j < row_ptr[u + 1]; j++) {
                int64_t x = (int64_t)(w ? w[j] : 1);
                if (part[col[j]] != part[u]) { g += x; cut += x; } else g -= x;
            }
            gain[u] = g;
            bal += part[u] == 0 ? 1 : -1;
            rank[u] = ORC_UNASSIGNED;
            if (g > 0) {
                if (part[u] == 0) { A[na].g = g; A[na].u = u; na++; }
                else { B[nb].g = g; B[nb].u = u; nb++; }
            }
        }
        cut /= 2;
        qsort(A, na, sizeof(orc_fmc_t), orc_fm_cmp);
        qsort(B, nb, sizeof(orc_fmc_t), orc_fm_cmp);
        /* interleave (serial FM balance rule) */
        uint32_t ia = 0, ib = 0, k = 0;
        int64_t b = bal;
        while (ia < na || ib < nb) {
            int take_a;
            if (ia == na) take_a = 0;
            else if (ib == nb) take_a = 1;
            else if (b > 0) take_a = 1;
            else if (b < 0) take_a = 0;
            else take_a = A[ia].g >= B[ib].g;
            uint32_t u = take_a ? A[ia++].u : B[ib++].u;
            b += take_a ? -2 : 2;
            rank[u] = k;
            seq[k++] = u;
        }
        /* sequential gains, prefix cut and balance, best prefix */
        const int64_t abs0 = bal < 0 ? -bal : bal;
        const int64_t target = abs0 / 10 > 20 ? abs0 / 10 : 20;
        int64_t best_cut = cut, run = cut, rb = bal;
        uint32_t best_k = 0;
        for (uint32_t i = 0; i < k; i++) {
            uint32_t u = seq[i];
            int64_t g = 0;
            for (uint32_t j = row_ptr[u]; j < row_ptr[u + 1]; j++) {
                uint32_t v = col[j];
                int64_t x = (int64_t)(w ? w[j] : 1);
                int across = part[v] != part[u];
                int moved = rank[v] < i;
                g += (across ^ moved) ? x : -x;
            }
            gseq[i] = g;
            run -= g;
            rb += part[u] == 0 ? -2 : 2;
            int64_t ab = rb < 0 ? -rb : rb;
            if (ab <= target && run <= best_cut) { best_cut = run; best_k = i + 1; }
        }
        if (best_k == 0 || best_cut == cut) break;
        for (uint32_t i = 0; i < best_k; i++) part[seq[i]] ^= 1u;
        moves += best_k;
        *cut_io = (uint64_t)best_cut;
    }
    if (moves_out) *moves_out = moves;
    free(gain); free(rank); free(seq); free(gseq); free(A); free(B);
    return pass;
}

/* Edge cut of an arbitrary 2-way partition (directed cross entries / 2). */
uint64_t orc_edge_cut(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const uint32_t *part) {
    uint64_t c = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++)
            if (part[col[j]] != part[i]) c++;
    return c / 2;
}

/* sgpar.h:2666-2752: relabel part-0 and part-1 vertices in ascending order and
 * keep the edges inside each part.  Output arrays sized by the caller
 * (row ptrs n+1, cols row_ptr[n]).  Returns 0. */
int orc_use_partition(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                      const uint32_t *part,
                      uint32_t *n1, uint32_t *rp1, uint32_t *col1,
                      uint32_t *n2, uint32_t *rp2, uint32_t *col2) {
    uint32_t *map = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t c1 = 0, c2 = 0;
    for (uint32_t i = 0; i < n; i++) map[i] = part[i] == 0 ? c1++ : c2++;
    uint32_t e1 = 0, e2 = 0, a = 0, b = 0;
    rp1[0] = 0; rp2[0] = 0;
    for (uint32_t i = 0; i < n; i++) {
        for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) {
            uint32_t d = col[j];
            if (part[i] != part[d]) continue;
            if (part[i] == 0) col1[e1++] = map[d]; else col2[e2++] = map[d];
        }
        if (part[i] == 0) rp1[++a] = e1; else rp2[++b] = e2;
    }
    *n1 = c1; *n2 = c2;
    free(map);
    return 0;
}

/* ---------------------------------------------- alternative coarseners -- */
/* The reference's other coarseners with this project's deterministic rules
 * (the CUDA path, coarsen_alt.cu, follows the same rules):
 *   MATCH  heuristics.h:1584-1740 (PUREMATCH): proposal rounds along the
 *          heavy edge, retries along the heaviest unmatched edge, singletons
 *   MIS2   heuristics.h:8-80 + :218-310: distance-2 maximal independent set,
 *          roots take their neighbours, the rest join the first aggregated
 *          neighbour in row order
 *   GOSH   heuristics.h:81-216 + :312-365: degree-keyed independent set
 *          ignoring edges between two vertices above the mean degree, the
 *          rest join their set neighbour of largest degree (first on a tie)
 * Random keys are orc_prio_key(seed, u); aggregates are numbered by
 * ascending root vertex. */
static uint64_t orc_wt(const uint64_t *w, uint32_t j) { return w ? w[j] : 1; }

/* number aggregates by ascending root (vcmap[u] == u marks a root) */
static uint32_t orc_number_roots(uint32_t n, uint32_t *vcmap) {
    uint32_t *rank = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t nc = 0;
    for (uint32_t u = 0; u < n; u++) rank[u] = vcmap[u] == u ? nc++ : 0;
    for (uint32_t u = 0; u < n; u++) vcmap[u] = rank[vcmap[u]];
    free(rank);
    return nc;
}

int orc_match_map(uint32_t n, const uint32_t *rp, const uint32_t *col, const uint64_t *w, int random_level,
                  uint64_t seed, uint32_t *vcmap, uint32_t *nc_out, uint32_t *rounds_out) {
    uint32_t *hn = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t *list = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t *next = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint64_t *claim = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint8_t *act = (uint8_t *)calloc((size_t)n + 1, 1);
    /* initial heavy neighbour (heuristics.h:1616-1640) */
    for (uint32_t u = 0; u < n; u++) {
        uint32_t b = rp[u], e = rp[u + 1];
        vcmap[u] = ORC_UNASSIGNED;
        list[u] = u;
        if (b == e) { hn[u] = u; continue; }
        if (random_level) { hn[u] = col[b + (uint32_t)(orc_rand_draw(seed, u) % (e - b))]; continue; }
        uint64_t bw = orc_wt(w, b);
        uint32_t bj = b;
        for (uint32_t j = b + 1; j < e; j++)
            if (orc_wt(w, j) > bw) { bw = orc_wt(w, j); bj = j; }
        hn[u] = col[bj];
    }
    uint32_t len = n, swap = 1, rounds = 0;
    for (;;) {
        for (uint32_t i = 0; i < len; i++) {
            uint32_t u = list[i], v = hn[u];
            act[u] = 0;
            if (v == u) continue;
            uint64_t ku = orc_prio_key(seed, u), kv = orc_prio_key(seed, v);
            if ((uint32_t)(ku < kv) ^ swap) {
                act[u] = 1;
                if (claim[u] < ku + 1) claim[u] = ku + 1;
                if (claim[v] < ku + 1) claim[v] = ku + 1;
            }
        }
        for (uint32_t i = 0; i < len; i++) {
            uint32_t u = list[i];
            if (!act[u]) continue;
            uint32_t v = hn[u];
            uint64_t k = orc_prio_key(seed, u) + 1;
            if (claim[u] == k && claim[v] == k) { vcmap[u] = u; vcmap[v] = u; }
        }
        uint32_t nn = 0;
        for (uint32_t i = 0; i < len; i++) {
            uint32_t u = list[i];
            claim[u] = 0;
            if (vcmap[u] != ORC_UNASSIGNED) continue;
            /* heaviest unmatched neighbour, the last maximum in row order
             * (heuristics.h:1686-1716, "<="); level 1 orders by key */
            uint64_t bk = 0;
            uint32_t bj = ORC_UNASSIGNED;
            for (uint32_t j = rp[u]; j < rp[u + 1]; j++) {
                uint32_t v = col[j];
                if (vcmap[v] != ORC_UNASSIGNED) continue;
                uint64_t k = random_level ? orc_prio_key(seed, v) + 1 : orc_wt(w, j);
                if (bj == ORC_UNASSIGNED || k >= bk) { bk = k; bj = j; }
            }
            if (bj != ORC_UNASSIGNED) { hn[u] = col[bj]; next[nn++] = u; }
        }
        rounds++;
        if (nn == 0) break;
        uint32_t *t = list; list = next; next = t;
        len = nn;
        swap ^= 1u;
    }
    for (uint32_t u = 0; u < n; u++)
        if (vcmap[u] == ORC_UNASSIGNED) vcmap[u] = u;
    *nc_out = orc_number_roots(n, vcmap);
    *rounds_out = rounds;
    free(hn); free(list); free(next); free(claim); free(act);
    return 0;
}

/* heuristics.h:766-834 (parallel_map_construct_v3) on given heavy
 * neighbours: mutual heavy pairs point to their smaller id, other heavy
 * targets to themselves, the rest where their heavy neighbour points; roots
 * numbered in ascending order. */
int orc_hec_v3_map(uint32_t n, const uint32_t *hn, uint32_t *vcmap, uint32_t *nc_out) {
    uint32_t *m = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    for (uint32_t u = 0; u < n; u++) {
        m[u] = ORC_UNASSIGNED;
        if (hn[hn[u]] == u) m[u] = hn[u] < u ? hn[u] : u;
    }
    for (uint32_t u = 0; u < n; u++)
        if (m[hn[u]] == ORC_UNASSIGNED) m[hn[u]] = hn[u];
    for (uint32_t u = 0; u < n; u++) vcmap[u] = m[u] != ORC_UNASSIGNED ? m[u] : m[hn[u]];
    *nc_out = orc_number_roots(n, vcmap);
    free(m);
    return 0;
}

/* heuristics.h:444-560 (sgp_coarsen_GOSH_v2) with every step reading a
 * snapshot of the one before (the reference reads live values, so its
 * result depends on thread timing): vertices of degree above max(nnz/n, 50)
 * are roots; the others join their root neighbour of largest edge weight
 * (the last in row order on a tie, ">="); the rest their aggregated
 * neighbour of largest degree (last on a tie); the rest their first
 * aggregated neighbour in row order; what remains goes through the HEC map
 * rounds with those aggregates prefilled, heavy neighbours by (weight,
 * tie-break hash) over all neighbours. */
int orc_gosh_v2_map(uint32_t n, const uint32_t *rp, const uint32_t *col, const uint64_t *w, uint64_t seed,
                    uint32_t *vcmap, uint32_t *nc_out) {
    uint64_t thr = n ? (uint64_t)rp[n] / n : 0;
    if (thr < 50) thr = 50;
    uint32_t *a = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    for (uint32_t u = 0; u < n; u++) a[u] = (uint64_t)(rp[u + 1] - rp[u]) > thr ? u : ORC_UNASSIGNED;
    for (int mode = 0; mode < 3; mode++) {
        for (uint32_t u = 0; u < n; u++) {
            vcmap[u] = a[u];
            if (a[u] != ORC_UNASSIGNED) continue;
            uint64_t bk = 0;
            uint32_t bj = ORC_UNASSIGNED;
            for (uint32_t j = rp[u]; j < rp[u + 1]; j++) {
                uint32_t v = col[j];
                if (a[v] == ORC_UNASSIGNED) continue;
                if (mode == 2) { bj = j; break; }
                uint64_t k = mode == 0 ? (w ? w[j] : 1) : (uint64_t)(rp[v + 1] - rp[v]);
                if (bj == ORC_UNASSIGNED || k >= bk) { bk = k; bj = j; }
            }
            if (bj != ORC_UNASSIGNED) vcmap[u] = a[col[bj]];
        }
        memcpy(a, vcmap, (size_t)n * sizeof(uint32_t));
    }
    free(a);
    uint32_t *hn = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    orc_hec_heavy(n, rp, col, w, 0, seed, hn);
    orc_hec_map_pre(n, hn, seed, vcmap, nc_out, 1);
    free(hn);
    return 0;
}

typedef struct { int s; uint64_t k; uint32_t i; } orc_tup_t;
static int orc_tup_gt(orc_tup_t x, orc_tup_t y) {
    return x.s > y.s || (x.s == y.s && (x.k > y.k || (x.k == y.k && x.i > y.i)));
}

/* gosh = 0: MIS-2 (two hops of the maximum per iteration, random keys);
 * gosh = 1: GOSH_clusters (one hop, degree keys, decided vertices keep their
 * own tuple, edges between two vertices of degree > nnz / n ignored). */
int orc_set_map(uint32_t n, const uint32_t *rp, const uint32_t *col, int gosh, uint64_t seed, uint32_t *vcmap,
                uint32_t *nc_out, uint32_t *iters_out) {
    int *state = (int *)calloc((size_t)n + 1, sizeof(int));
    orc_tup_t *a = (orc_tup_t *)malloc(((size_t)n + 1) * sizeof(orc_tup_t));
    orc_tup_t *b = (orc_tup_t *)malloc(((size_t)n + 1) * sizeof(orc_tup_t));
    const uint64_t thr = n ? (uint64_t)rp[n] / n : 0;
    int it = 0;
    for (;; it++) {
        for (uint32_t u = 0; u < n; u++) {
            a[u].s = state[u];
            a[u].k = gosh ? (uint64_t)(rp[u + 1] - rp[u]) : orc_prio_key(seed, u);
            a[u].i = u;
        }
        for (int h = 0; h < (gosh ? 1 : 2); h++) {
            for (uint32_t u = 0; u < n; u++) {
                if (gosh && state[u] != 0) {
                    b[u].s = state[u]; b[u].k = rp[u + 1] - rp[u]; b[u].i = u;
                    continue;
                }
                orc_tup_t best = a[u];
                int u_big = gosh && (uint64_t)(rp[u + 1] - rp[u]) > thr;
                for (uint32_t j = rp[u]; j < rp[u + 1]; j++) {
                    uint32_t v = col[j];
                    if (u_big && (uint64_t)(rp[v + 1] - rp[v]) > thr) continue;
                    if (orc_tup_gt(a[v], best)) best = a[v];
                }
                b[u] = best;
            }
            orc_tup_t *t = a; a = b; b = t;
        }
        uint32_t left = 0;
        for (uint32_t u = 0; u < n; u++) {
            if (state[u] != 0) continue;
            uint32_t m = a[u].i;
            if (m == u) state[u] = 1;
            else if (a[u].s == 1 || a[m].i == m) state[u] = -1;
            else left++;
        }
        if (left == 0) break;
    }
    *iters_out = (uint32_t)(it + 1);
    uint32_t *rank = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t nc = 0;
    for (uint32_t u = 0; u < n; u++) rank[u] = state[u] == 1 ? nc++ : ORC_UNASSIGNED;
    int rc = 0;
    if (!gosh) {
        uint32_t *vc1 = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
        for (uint32_t u = 0; u < n; u++) vc1[u] = ORC_UNASSIGNED;
        for (uint32_t u = 0; u < n; u++) {
            if (state[u] != 1) continue;
            vc1[u] = rank[u];
            for (uint32_t j = rp[u]; j < rp[u + 1]; j++) vc1[col[j]] = rank[u];
        }
        for (uint32_t u = 0; u < n; u++) {
            vcmap[u] = vc1[u];
            if (vc1[u] != ORC_UNASSIGNED) continue;
            for (uint32_t j = rp[u]; j < rp[u + 1]; j++)
                if (vc1[col[j]] != ORC_UNASSIGNED) { vcmap[u] = vc1[col[j]]; break; }
            if (vcmap[u] == ORC_UNASSIGNED) rc = 1;
        }
        free(vc1);
    } else {
        for (uint32_t u = 0; u < n; u++) {
            if (state[u] == 1) { vcmap[u] = rank[u]; continue; }
            uint32_t bd = 0, bv = ORC_UNASSIGNED;
            for (uint32_t j = rp[u]; j < rp[u + 1]; j++) {
                uint32_t v = col[j], d = rp[v + 1] - rp[v];
                if (state[v] == 1 && d > bd) { bd = d; bv = v; }
            }
            vcmap[u] = bv == ORC_UNASSIGNED ? ORC_UNASSIGNED : rank[bv];
            if (bv == ORC_UNASSIGNED) rc = 1;
        }
    }
    *nc_out = nc;
    free(state); free(a); free(b); free(rank);
    return rc;
}

/* ------------------------------------------------------ multilevel path -- */
/* The whole path with this project's seeding convention: every coarsening
 * level draws two PCG32 outputs (high word first) for its hash seed; the
 * coarsest guess then draws one output per coarse vertex divided by
 * UINT32_MAX (eigensolve_kokkos.h:1500-1505).  Levels are generated while
 * n > cutoff, at most 200 (coarsen_kokkos.h:1200-1218); a coarsest level below
 * 10 vertices is dropped (:1226-1231).  w64 may be NULL (unit weights); with
 * unit input weights level 1 uses the random neighbour.
 * stats (optional, >= 3 + 2*201 doubles): [levels, lambda, finest niter,
 * then per level (fine to coarse) n and niter]. */
typedef struct { uint32_t n; uint32_t *rp; uint32_t *col; uint64_t *w; uint32_t *vcmap; } orc_level_t;

int orc_partition_graph(uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                        const uint64_t *w64, uint32_t cutoff, double tol,
                        uint64_t *rng_state, uint64_t rng_inc,
                        int perc_imbalance_allowed, int normlap, int coarsener, int local_search_alg,
                        uint32_t *part, uint64_t *edgecut, double *evec_out, double *stats) {
    orc_level_t L[202];
    int nl = 1;
    const int kind = coarsener & 15;
    L[0].n = n; L[0].rp = (uint32_t *)row_ptr; L[0].col = (uint32_t *)col;
    L[0].w = (uint64_t *)w64; L[0].vcmap = NULL;
    /* coarsener: 0 HEC, 1 MATCH, 2 MIS2, 3 GOSH, 4 HEC_V3, 5 GOSH_V2; | 16 no coarsening, | 32 stop
     * after a level keeping more than 0.9 of the vertices (sgpar.h:2466-2475) */
    while (!(coarsener & 16) && L[nl - 1].n > cutoff) {
        orc_level_t *f = &L[nl - 1];
        uint64_t seed = ((uint64_t)orc_pcg32(rng_state, rng_inc) << 32);
        seed |= orc_pcg32(rng_state, rng_inc);
        f->vcmap = (uint32_t *)malloc((size_t)f->n * sizeof(uint32_t));
        int random_level = (nl == 1) && (w64 == NULL);
        uint32_t nc = 0, rounds = 0;
        if (kind == 0) {
            uint32_t *hn = (uint32_t *)malloc((size_t)f->n * sizeof(uint32_t));
            orc_hec_heavy(f->n, f->rp, f->col, f->w, random_level, seed, hn);
            orc_hec_map(f->n, hn, seed, f->vcmap, &nc);
            free(hn);
        } else if (kind == 1) {
            orc_match_map(f->n, f->rp, f->col, f->w, random_level, seed, f->vcmap, &nc, &rounds);
        } else if (kind == 5) {
            orc_gosh_v2_map(f->n, f->rp, f->col, f->w, seed, f->vcmap, &nc);
        } else if (kind == 4) {
            uint32_t *hn = (uint32_t *)malloc((size_t)f->n * sizeof(uint32_t));
            orc_hec_heavy(f->n, f->rp, f->col, f->w, random_level, seed, hn);
            orc_hec_v3_map(f->n, hn, f->vcmap, &nc);
            free(hn);
        } else {
            if (orc_set_map(f->n, f->rp, f->col, kind == 3, seed, f->vcmap, &nc, &rounds)) return 1;
        }
        orc_level_t *c = &L[nl];
        uint32_t mf = f->rp[f->n];
        c->n = nc;
        c->rp = (uint32_t *)malloc(((size_t)nc + 1) * sizeof(uint32_t));
        c->col = (uint32_t *)malloc(((size_t)mf + 1) * sizeof(uint32_t));
        c->w = (uint64_t *)malloc(((size_t)mf + 1) * sizeof(uint64_t));
        c->vcmap = NULL;
        orc_build_coarse(f->n, f->rp, f->col, f->w, f->vcmap, nc, NULL, NULL, c->rp, c->col, c->w);
        nl++;
        if (nl > 200) break;
        if ((coarsener & 32) && (double)nc / (double)f->n > 0.9) break;
    }
    if (nl > 1 && L[nl - 1].n < 10) {
        nl--;
        free(L[nl].rp); free(L[nl].col); free(L[nl].w);
    }
    if (stats) stats[0] = nl;
    /* coarsest guess */
    uint32_t gn = L[nl - 1].n;
    double *vec = (double *)malloc((size_t)gn * sizeof(double));
    for (uint32_t i = 0; i < gn; i++) vec[i] = ((double)orc_pcg32(rng_state, rng_inc)) / 4294967295.0;
    double ss = 0;
    for (uint32_t i = 0; i < gn; i++) ss += vec[i] * vec[i];
    double inv = 1 / sqrt(ss);
    for (uint32_t i = 0; i < gn; i++) vec[i] *= inv;
    double lambda = 0;
    for (int l = nl - 1; l >= 0; l--) {
        orc_level_t *lv = &L[l];
        uint64_t it = normlap ? orc_power_iter_nl(lv->n, lv->rp, lv->col, lv->w, vec, tol, 0, l == 0 ? &lambda : NULL)
                              : orc_power_iter(lv->n, lv->rp, lv->col, lv->w, vec, tol, 0, l == 0 ? &lambda : NULL);
        if (stats) { stats[3 + 2 * l] = lv->n; stats[4 + 2 * l] = (double)it; }
        if (l == 0) { if (stats) stats[2] = (double)it; break; }
        /* prolongation fine[i] = coarse[vcmap[i]] (eigensolve_kokkos.h:1556-1559) */
        orc_level_t *fl = &L[l - 1];
        double *fine = (double *)malloc((size_t)fl->n * sizeof(double));
        for (uint32_t i = 0; i < fl->n; i++) fine[i] = vec[fl->vcmap[i]];
        free(vec);
        vec = fine;
    }
    if (stats) stats[1] = lambda;
    if (local_search_alg)
        orc_compute_partition_ls(n, row_ptr, col, vec, local_search_alg, part, edgecut, NULL);
    else
        orc_compute_partition(n, row_ptr, col, vec, perc_imbalance_allowed, part, edgecut);
    if (evec_out) memcpy(evec_out, vec, (size_t)n * sizeof(double));
    free(vec);
    for (int l = 0; l < nl; l++) {
        free(L[l].vcmap);
        if (l > 0) { free(L[l].rp); free(L[l].col); free(L[l].w); }
    }
    return 0;
}
