// graphgen.cpp -- seeded synthetic graphs with the shapes of the benchmark
// configurations, written as symmetric CSR with sorted rows, no self loops and
// no duplicate entries (the invariants cmg/mtx2csr.cpp:132-264 establishes
// for the reference's inputs), restricted to the largest connected component.
//
//   grid2d        nx x ny 5-point grid
//   grid2d_holes  grid with a fraction of vertices removed uniformly
//   rmat          R-MAT (a, b, c, d) with edge factor, labels scrambled
//   rgg3d         random geometric graph in the unit cube (cell list)
//   er            Erdos-Renyi G(n, m) with a given mean degree
//   chunglu       Chung-Lu with Pareto expected degrees and integer weights
//
// Also the reference's binary CSR file format (mtx2csr.cpp:276-288 writes it,
// sgpar.h:2262-2289 reads it): 6 x int64 header (n, m_directed, 1, 0, 1, 0),
// uint32 offsets[n+1], uint32 destinations[m_directed].
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <vector>
#include <algorithm>
#include <numeric>
#include <atomic>
#include <omp.h>
#include <string>

extern "C" {
typedef struct {
    uint32_t n;
    uint64_t m;          // directed entries = row_ptr[n]
    uint32_t *row_ptr;   // n + 1
    uint32_t *col;       // m
    uint32_t *w;         // m, or NULL for unit weights
} sgpgen_csr_t;
}

namespace {

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
struct Rng {  // splitmix64 stream
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    inline uint64_t next() { s += 0x9E3779B97F4A7C15ULL; return mix64(s); }
    inline double unit() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Edges { std::vector<uint32_t> u, v; };

// symmetric CSR from an undirected edge list: drops self loops, merges
// duplicates, sorts rows.  Weight per undirected edge from wfun(min, max).
template <class WF>
void edges_to_csr(uint32_t n, const Edges &E, bool weighted, WF wfun, std::vector<uint32_t> &rp,
                  std::vector<uint32_t> &col, std::vector<uint32_t> &w) {
    size_t m = E.u.size();
    std::vector<std::atomic<uint32_t>> deg(n);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) deg[i].store(0, std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        uint32_t a = E.u[e], b = E.v[e];
        if (a == b) continue;
        deg[a].fetch_add(1, std::memory_order_relaxed);
        deg[b].fetch_add(1, std::memory_order_relaxed);
    }
    std::vector<uint64_t> off(n + 1, 0);
    for (uint32_t i = 0; i < n; i++) off[i + 1] = off[i] + deg[i].load(std::memory_order_relaxed);
    std::vector<uint32_t> tmp(off[n]);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) deg[i].store(0, std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        uint32_t a = E.u[e], b = E.v[e];
        if (a == b) continue;
        tmp[off[a] + deg[a].fetch_add(1, std::memory_order_relaxed)] = b;
        tmp[off[b] + deg[b].fetch_add(1, std::memory_order_relaxed)] = a;
    }
    std::vector<uint32_t> len(n);
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint32_t *b = tmp.data() + off[i], *e = tmp.data() + off[i + 1];
        std::sort(b, e);
        len[i] = (uint32_t)(std::unique(b, e) - b);
    }
    rp.assign(n + 1, 0);
    for (uint32_t i = 0; i < n; i++) rp[i + 1] = rp[i] + len[i];
    col.resize(rp[n]);
    if (weighted) w.resize(rp[n]);
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        memcpy(col.data() + rp[i], tmp.data() + off[i], (size_t)len[i] * 4);
        if (weighted)
            for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
                uint32_t a = (uint32_t)i, b = col[j];
                w[j] = wfun(std::min(a, b), std::max(a, b));
            }
    }
}

// keep the largest connected component, relabelled in ascending order
void keep_lcc(uint32_t &n, std::vector<uint32_t> &rp, std::vector<uint32_t> &col, std::vector<uint32_t> &w) {
    std::vector<uint32_t> comp(n, UINT32_MAX), queue(n);
    uint32_t best = 0, best_size = 0, ncomp = 0;
    for (uint32_t s = 0; s < n; s++) {
        if (comp[s] != UINT32_MAX) continue;
        uint32_t h = 0, t = 0;
        queue[t++] = s; comp[s] = ncomp;
        while (h < t) {
            uint32_t x = queue[h++];
            for (uint32_t j = rp[x]; j < rp[x + 1]; j++) {
                uint32_t y = col[j];
                if (comp[y] == UINT32_MAX) { comp[y] = ncomp; queue[t++] = y; }
            }
        }
        if (t > best_size) { best_size = t; best = ncomp; }
        ncomp++;
    }
    if (ncomp <= 1) return;
    std::vector<uint32_t> map(n, UINT32_MAX);
    uint32_t nn = 0;
    for (uint32_t i = 0; i < n; i++) if (comp[i] == best) map[i] = nn++;
    std::vector<uint32_t> nrp(nn + 1, 0), ncol, nw;
    for (uint32_t i = 0; i < n; i++) if (map[i] != UINT32_MAX) nrp[map[i] + 1] = rp[i + 1] - rp[i];
    for (uint32_t i = 0; i < nn; i++) nrp[i + 1] += nrp[i];
    ncol.resize(nrp[nn]);
    if (!w.empty()) nw.resize(nrp[nn]);
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        if (map[i] == UINT32_MAX) continue;
        uint32_t o = nrp[map[i]];
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
            ncol[o] = map[col[j]];   // monotone relabel keeps rows sorted
            if (!w.empty()) nw[o] = w[j];
            o++;
        }
    }
    n = nn; rp.swap(nrp); col.swap(ncol); w.swap(nw);
}

int finish(uint32_t n, std::vector<uint32_t> &rp, std::vector<uint32_t> &col, std::vector<uint32_t> &w,
           bool lcc, sgpgen_csr_t *out) {
    if (lcc) keep_lcc(n, rp, col, w);
    out->n = n;
    out->m = rp[n];
    out->row_ptr = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    out->col = (uint32_t *)malloc(sizeof(uint32_t) * (out->m ? out->m : 1));
    out->w = NULL;
    if (!out->row_ptr || !out->col) return 1;
    memcpy(out->row_ptr, rp.data(), sizeof(uint32_t) * ((size_t)n + 1));
    memcpy(out->col, col.data(), sizeof(uint32_t) * out->m);
    if (!w.empty()) {
        out->w = (uint32_t *)malloc(sizeof(uint32_t) * (out->m ? out->m : 1));
        if (!out->w) return 1;
        memcpy(out->w, w.data(), sizeof(uint32_t) * out->m);
    }
    return 0;
}

auto no_w = [](uint32_t, uint32_t) { return 1u; };

}  // namespace

extern "C" {

void sgpgen_free(sgpgen_csr_t *g) {
    if (!g) return;
    free(g->row_ptr); free(g->col); free(g->w);
    g->row_ptr = NULL; g->col = NULL; g->w = NULL;
}

int sgpgen_grid2d(uint32_t nx, uint32_t ny, sgpgen_csr_t *out) {
    uint64_t n64 = (uint64_t)nx * ny;
    if (n64 == 0 || n64 >= 0xFFFFFFFFull) return 1;
    uint32_t n = (uint32_t)n64;
    std::vector<uint32_t> rp(n + 1), col, w;
    for (uint32_t r = 0; r < ny; r++)
        for (uint32_t c = 0; c < nx; c++) {
            uint32_t i = r * nx + c;
            rp[i + 1] = (r > 0) + (c > 0) + (c + 1 < nx) + (r + 1 < ny);
        }
    for (uint32_t i = 0; i < n; i++) rp[i + 1] += rp[i];
    col.resize(rp[n]);
    #pragma omp parallel for schedule(static)
    for (int64_t rr = 0; rr < (int64_t)ny; rr++) {
        uint32_t r = (uint32_t)rr;
        for (uint32_t c = 0; c < nx; c++) {
            uint32_t i = r * nx + c, o = rp[i];
            if (r > 0) col[o++] = i - nx;
            if (c > 0) col[o++] = i - 1;
            if (c + 1 < nx) col[o++] = i + 1;
            if (r + 1 < ny) col[o++] = i + nx;
        }
    }
    return finish(n, rp, col, w, false, out);
}

int sgpgen_grid2d_holes(uint32_t nx, uint32_t ny, double frac_removed, uint64_t seed, sgpgen_csr_t *out) {
    uint64_t n64 = (uint64_t)nx * ny;
    if (n64 == 0 || n64 >= 0xFFFFFFFFull) return 1;
    uint32_t N = (uint32_t)n64;
    std::vector<uint8_t> keep(N, 1);
    uint64_t thr = (uint64_t)(frac_removed * 18446744073709551615.0);
    for (uint32_t i = 0; i < N; i++) if (mix64(seed ^ (0xA24BAED4963EE407ULL * (i + 1ull))) < thr) keep[i] = 0;
    std::vector<uint32_t> id(N, UINT32_MAX);
    uint32_t n = 0;
    for (uint32_t i = 0; i < N; i++) if (keep[i]) id[i] = n++;
    Edges E;
    for (uint32_t r = 0; r < ny; r++)
        for (uint32_t c = 0; c < nx; c++) {
            uint32_t i = r * nx + c;
            if (!keep[i]) continue;
            if (c + 1 < nx && keep[i + 1]) { E.u.push_back(id[i]); E.v.push_back(id[i + 1]); }
            if (r + 1 < ny && keep[i + nx]) { E.u.push_back(id[i]); E.v.push_back(id[i + nx]); }
        }
    std::vector<uint32_t> rp, col, w;
    edges_to_csr(n, E, false, no_w, rp, col, w);
    return finish(n, rp, col, w, true, out);
}

int sgpgen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                int scramble, sgpgen_csr_t *out) {
    if (scale < 1 || scale > 31) return 1;
    uint32_t n = 1u << scale;
    uint64_t m = (uint64_t)edge_factor << scale;
    Edges E;
    E.u.resize(m); E.v.resize(m);
    const double ab = a + b, abc = a + b + c;
    const uint64_t ta = (uint64_t)(a * 4294967296.0), tab = (uint64_t)(ab * 4294967296.0),
                   tabc = (uint64_t)(abc * 4294967296.0);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        uint64_t s = mix64(seed ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)e + 1)));
        uint32_t u = 0, v = 0;
        uint64_t bits = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 1) == 0) { s += 0x9E3779B97F4A7C15ULL; bits = mix64(s); }
            uint64_t r = (l & 1) ? (bits >> 32) : (bits & 0xFFFFFFFFull);
            uint32_t ub, vb;
            if (r < ta) { ub = 0; vb = 0; }
            else if (r < tab) { ub = 0; vb = 1; }
            else if (r < tabc) { ub = 1; vb = 0; }
            else { ub = 1; vb = 1; }
            u = (u << 1) | ub; v = (v << 1) | vb;
        }
        E.u[e] = u; E.v[e] = v;
    }
    if (scramble) {  // seeded label permutation (Fisher-Yates)
        std::vector<uint32_t> perm(n);
        std::iota(perm.begin(), perm.end(), 0u);
        Rng r(seed ^ 0x5851F42D4C957F2DULL);
        for (uint32_t i = n - 1; i > 0; i--) std::swap(perm[i], perm[r.next() % (i + 1)]);
        #pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < (int64_t)m; e++) { E.u[e] = perm[E.u[e]]; E.v[e] = perm[E.v[e]]; }
    }
    std::vector<uint32_t> rp, col, w;
    edges_to_csr(n, E, false, no_w, rp, col, w);
    Edges().u.swap(E.u);
    return finish(n, rp, col, w, true, out);
}

int sgpgen_er(uint32_t n, double mean_degree, uint64_t seed, sgpgen_csr_t *out) {
    if (n < 2) return 1;
    uint64_t m = (uint64_t)(mean_degree * n / 2.0 + 0.5);
    Edges E;
    E.u.resize(m); E.v.resize(m);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        uint64_t x = mix64(seed ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)e + 1)));
        uint64_t y = mix64(x ^ 0xD6E8FEB86659FD93ULL);
        E.u[e] = (uint32_t)(x % n); E.v[e] = (uint32_t)(y % n);
    }
    std::vector<uint32_t> rp, col, w;
    edges_to_csr(n, E, false, no_w, rp, col, w);
    return finish(n, rp, col, w, true, out);
}

int sgpgen_rgg3d(uint32_t n, double radius, uint64_t seed, sgpgen_csr_t *out) {
    if (n < 2 || radius <= 0 || radius >= 1) return 1;
    uint32_t G = (uint32_t)floor(1.0 / radius);
    if (G < 1) G = 1;
    if ((uint64_t)G * G * G > 0x7FFFFFFFull) G = 1290;
    uint64_t ncell = (uint64_t)G * G * G;
    std::vector<float> px(n), py(n), pz(n);
    std::vector<uint32_t> cell(n);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        Rng r(mix64(seed ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)i + 1))));
        double x = r.unit(), y = r.unit(), z = r.unit();
        px[i] = (float)x; py[i] = (float)y; pz[i] = (float)z;
        uint32_t cx = std::min<uint32_t>((uint32_t)(px[i] * G), G - 1);
        uint32_t cy = std::min<uint32_t>((uint32_t)(py[i] * G), G - 1);
        uint32_t cz = std::min<uint32_t>((uint32_t)(pz[i] * G), G - 1);
        cell[i] = (uint32_t)(((uint64_t)cz * G + cy) * G + cx);
    }
    // counting sort of points by cell; vertex ids follow cell order
    std::vector<uint32_t> cstart(ncell + 1, 0);
    for (uint32_t i = 0; i < n; i++) cstart[cell[i] + 1]++;
    for (uint64_t c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
    std::vector<uint32_t> order(n), fill(cstart.begin(), cstart.end() - 1);
    for (uint32_t i = 0; i < n; i++) order[fill[cell[i]]++] = i;
    std::vector<float> sx(n), sy(n), sz(n);
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)n; k++) { uint32_t i = order[k]; sx[k] = px[i]; sy[k] = py[i]; sz[k] = pz[i]; }
    std::vector<float>().swap(px); std::vector<float>().swap(py); std::vector<float>().swap(pz);
    const float r2 = (float)(radius * radius);
    std::vector<uint32_t> deg(n);
    auto scan_nb = [&](uint32_t k, auto emit) {
        uint32_t cx = std::min<uint32_t>((uint32_t)(sx[k] * G), G - 1);
        uint32_t cy = std::min<uint32_t>((uint32_t)(sy[k] * G), G - 1);
        uint32_t cz = std::min<uint32_t>((uint32_t)(sz[k] * G), G - 1);
        for (int dz = -1; dz <= 1; dz++) {
            int64_t zz = (int64_t)cz + dz; if (zz < 0 || zz >= G) continue;
            for (int dy = -1; dy <= 1; dy++) {
                int64_t yy = (int64_t)cy + dy; if (yy < 0 || yy >= G) continue;
                for (int dx = -1; dx <= 1; dx++) {
                    int64_t xx = (int64_t)cx + dx; if (xx < 0 || xx >= G) continue;
                    uint64_t c = ((uint64_t)zz * G + yy) * G + xx;
                    for (uint32_t q = cstart[c]; q < cstart[c + 1]; q++) {
                        if (q == k) continue;
                        float ddx = sx[q] - sx[k], ddy = sy[q] - sy[k], ddz = sz[q] - sz[k];
                        if (ddx * ddx + ddy * ddy + ddz * ddz <= r2) emit(q);
                    }
                }
            }
        }
    };
    #pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t k = 0; k < (int64_t)n; k++) {
        uint32_t d = 0;
        scan_nb((uint32_t)k, [&](uint32_t) { d++; });
        deg[k] = d;
    }
    std::vector<uint32_t> rp(n + 1, 0), col, w;
    for (uint32_t k = 0; k < n; k++) rp[k + 1] = rp[k] + deg[k];
    col.resize(rp[n]);
    #pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t k = 0; k < (int64_t)n; k++) {
        uint32_t o = rp[k];
        scan_nb((uint32_t)k, [&](uint32_t q) { col[o++] = q; });
        std::sort(col.begin() + rp[k], col.begin() + rp[k + 1]);
    }
    return finish(n, rp, col, w, true, out);
}

int sgpgen_chunglu(uint32_t n, double alpha, double dmin, double dmax, uint32_t wmax,
                   uint64_t seed, sgpgen_csr_t *out) {
    if (n < 2 || alpha <= 1.0 || dmin <= 0 || dmax < dmin) return 1;
    // expected degrees: Pareto with shape alpha and scale dmin (P(D > d) =
    // (dmin / d)^alpha, mean alpha dmin / (alpha - 1)) capped at dmax
    std::vector<double> wdeg(n);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        Rng r(mix64(seed ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)i + 1))));
        double uu = 1.0 - r.unit();
        double d = dmin * pow(uu, -1.0 / alpha);
        wdeg[i] = d > dmax ? dmax : d;
    }
    std::vector<double> cdf(n + 1, 0.0);
    for (uint32_t i = 0; i < n; i++) cdf[i + 1] = cdf[i] + wdeg[i];
    double W = cdf[n];
    uint64_t m = (uint64_t)(W / 2.0);
    Edges E;
    E.u.resize(m); E.v.resize(m);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        Rng r(mix64(seed ^ 0x2545F4914F6CDD1DULL ^ (0x9E3779B97F4A7C15ULL * ((uint64_t)e + 1))));
        double x = r.unit() * W, y = r.unit() * W;
        E.u[e] = (uint32_t)std::min<size_t>(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin() - 1, n - 1);
        E.v[e] = (uint32_t)std::min<size_t>(std::upper_bound(cdf.begin(), cdf.end(), y) - cdf.begin() - 1, n - 1);
    }
    std::vector<uint32_t> rp, col, w;
    uint64_t wseed = seed ^ 0x94D049BB133111EBULL;
    auto wf = [wseed, wmax](uint32_t lo, uint32_t hi) {
        return (uint32_t)(mix64(wseed ^ (((uint64_t)lo << 32) | hi)) % wmax) + 1u;
    };
    edges_to_csr(n, E, wmax > 0, wf, rp, col, w);
    return finish(n, rp, col, w, true, out);
}

// reference binary CSR format (writer of mtx2csr.cpp:276-288)
int sgpgen_write_csr(const char *path, const sgpgen_csr_t *g) {
    FILE *f = fopen(path, "wb");
    if (!f) return 1;
    int64_t hdr[6] = {(int64_t)g->n, (int64_t)g->m, 1, 0, 1, 0};
    int ok = fwrite(hdr, sizeof(int64_t), 6, f) == 6;
    ok = ok && fwrite(g->row_ptr, 4, (size_t)g->n + 1, f) == (size_t)g->n + 1;
    ok = ok && fwrite(g->col, 4, g->m, f) == g->m;
    ok = (fclose(f) == 0) && ok;
    return ok ? 0 : 1;
}

int sgpgen_num_threads(void) { return omp_get_max_threads(); }

// MatrixMarket entry lines "u+1 v+1[ value]\n" (or "\r\n") for m pairs,
// formatted in parallel chunks: the input text of the MatrixMarket converter
// at benchmark sizes.  value_kind 0: none, 1: real values, 2: integer values
// (cycling through a few spellings, so parsers must skip them).  Returns the
// bytes written to out, or 0 when cap is too small.
uint64_t sgpgen_mtx_lines(const uint32_t *u, const uint32_t *v, uint64_t m, int value_kind, int crlf, char *out,
                          uint64_t cap) {
    static const char *reals[4] = {" 1", " -2.5", " 3.75e-1", " 0.125"};
    static const char *ints[3] = {" 1", " 7", " -3"};
    const int T = omp_get_max_threads();
    const uint64_t per = (m + T - 1) / (T ? T : 1);
    std::vector<std::string> part(T);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const uint64_t b = (uint64_t)t * per, e = std::min<uint64_t>(m, b + per);
        std::string &s = part[t];
        if (b < e) s.reserve((e - b) * 24);
        char buf[64];
        for (uint64_t i = b; i < e; i++) {
            int k = snprintf(buf, sizeof(buf), "%u %u", u[i] + 1u, v[i] + 1u);
            s.append(buf, k);
            if (value_kind == 1) s.append(reals[i & 3]);
            else if (value_kind == 2) s.append(ints[i % 3]);
            if (crlf) s.push_back('\r');
            s.push_back('\n');
        }
    }
    uint64_t total = 0;
    for (auto &p : part) total += p.size();
    if (total > cap) return 0;
    uint64_t off = 0;
    std::vector<uint64_t> offs(T);
    for (int t = 0; t < T; t++) {
        offs[t] = off;
        off += part[t].size();
    }
#pragma omp parallel for num_threads(T)
    for (int t = 0; t < T; t++) memcpy(out + offs[t], part[t].data(), part[t].size());
    return total;
}

}  // extern "C"
