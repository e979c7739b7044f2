// tune.cpp -- the per-device cache of the power iteration's autotuner.
//
// The reference picks its SpMV launch shape from fixed rules on the matrix's
// mean row length (kokkos-kernels/src/sparse/impl/KokkosSparse_spmv_impl.hpp:222-258,
// spmv_launch_parameters).  Here eigen.cu times candidate work splits of a
// level (SpMV variant, long-row threshold, grid size) for a few iterations the
// first time a level of its shape is met on a device, and keeps the fastest;
// this file holds the results: a map from (device, level shape) to the split,
// mirrored in a text file so later processes on the same kind of device skip
// the trials.  Lines: "<device key> <shape key> <mode> <heavy_div> <units>
// <ms best> <ms of the built-in rule>".
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <map>
#include <mutex>
#include <string>

#include "internal.h"

namespace sgpb {

namespace {
std::mutex g_mu;        // guards the map and the file
std::mutex g_tune_mu;   // held while a level shape is being tuned
bool g_loaded = false;
std::map<std::string, PITune> g_map;   // "<device key> <shape key>" -> split

std::string cache_path() {
    if (const char *p = getenv("SGPB_TUNE_CACHE")) return p;   // "" = memory only
    const char *home = getenv("HOME");
    if (!home || !*home) return "";
    return std::string(home) + "/.cache/sgpar_b200/pi_tune.txt";
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const std::string path = cache_path();
    if (path.empty()) return;
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return;
    char dev[200], shape[200];
    int mode;
    unsigned div, units;
    double a, b;
    while (fscanf(f, "%199s %199s %d %u %u %lf %lf", dev, shape, &mode, &div, &units, &a, &b) == 7) {
        if ((mode != 0 && mode != 5) || div == 0 || units == 0) continue;   // not a split this build runs
        PITune t;
        t.mode = mode;
        t.heavy_div = div;
        t.units = units;
        g_map[std::string(dev) + " " + shape] = t;
    }
    fclose(f);
}

void mkdirs(const std::string &path) {
    for (size_t i = 1; i < path.size(); i++)
        if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
}
}  // namespace

bool autotune_enabled() {
    const char *e = getenv("SGPB_AUTOTUNE");
    return !(e && atoi(e) == 0);
}

bool tune_lookup(const Context &C, const std::string &key, PITune *t) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    auto it = g_map.find(C.dev_key + " " + key);
    if (it == g_map.end()) return false;
    *t = it->second;
    return true;
}

void tune_store(const Context &C, const std::string &key, const PITune &t, double ms_best, double ms_rule) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    g_map[C.dev_key + " " + key] = t;
    const std::string path = cache_path();
    if (path.empty()) return;
    mkdirs(path);
    if (FILE *f = fopen(path.c_str(), "a")) {   // best effort: the map is authoritative for this process
        fprintf(f, "%s %s %d %u %u %.6f %.6f\n", C.dev_key.c_str(), key.c_str(), t.mode, t.heavy_div, t.units,
                ms_best, ms_rule);
        fclose(f);
    }
}

void tune_lock() { g_tune_mu.lock(); }
void tune_unlock() { g_tune_mu.unlock(); }

}  // namespace sgpb

extern "C" void sgp_b200_autotune_clear(void) {
    std::lock_guard<std::mutex> tl(sgpb::g_tune_mu);
    std::lock_guard<std::mutex> lock(sgpb::g_mu);
    sgpb::g_map.clear();
    sgpb::g_loaded = false;
}
