// Autotuning table of the tensor-core parse: the fastest (partner-tile width, row-block
// order) per shape class, process-wide behind a mutex, persisted as JSON.
//
// A shape class is what the host sees of a parse without reading device memory: population
// count, haplotype or genotype path, padded sample bytes (the K extent of the Gram
// products), bin count, the cutoff's decade and log2 of the mean window size (together the
// band class: how many partners an anchor has).  pg_gpu sizes its pair chunks from free
// memory instead (ld_pipeline.py:16-49); here the work is a fixed tile schedule and the
// table picks among its variants.
//
// File format (written by ldk_autotune_save, read by ldk_autotune_load; one object per line
// inside "entries" so that the reader stays a few lines):
//   {"format": "ldk-autotune", "version": 1, "entries": [
//    {"pops": 3, "genotypes": 0, "k_bytes": 512, "bins": 16, "cutoff_decade": 6, "window_log2": 11,
//     "tile_variant": 0, "tile_partners": 32, "order": 0, "ms": 49.1},
//    ...]}
// "order": 0 = row blocks of the largest windows first, 1 = window order.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "ldk_internal.h"

namespace ldk {
namespace {

std::mutex g_mu;
std::map<TuneKey, TuneChoice> g_table;
int g_tunings = 0;         // tuning runs this process performed
bool g_env_loaded = false;

const char* env_path() {
    const char* p = getenv("LDK_AUTOTUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

// "key": number inside one line of the entries list; false if absent.
bool field(const std::string& line, const char* key, double* v) {
    const std::string k = std::string("\"") + key + "\"";
    const size_t at = line.find(k);
    if (at == std::string::npos) return false;
    const size_t colon = line.find(':', at + k.size());
    if (colon == std::string::npos) return false;
    char* end = nullptr;
    *v = strtod(line.c_str() + colon + 1, &end);
    return end != line.c_str() + colon + 1;
}

int load_locked(const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return -1;
    int n = 0;
    char buf[1024];
    bool ok_format = false;
    while (fgets(buf, sizeof(buf), f)) {
        const std::string line(buf);
        if (line.find("\"ldk-autotune\"") != std::string::npos) ok_format = true;
        if (!ok_format || line.find("\"tile_variant\"") == std::string::npos) continue;
        double P, g, k, b, c, w, v, o, ms = 0.0;
        if (!field(line, "pops", &P) || !field(line, "genotypes", &g) || !field(line, "k_bytes", &k) ||
            !field(line, "bins", &b) || !field(line, "cutoff_decade", &c) || !field(line, "window_log2", &w) ||
            !field(line, "tile_variant", &v) || !field(line, "order", &o))
            continue;
        field(line, "ms", &ms);
        const TuneKey key{(int)P, (int)g, (int)k, (int)b, (int)c, (int)w};
        TuneChoice ch;
        ch.variant = (int)v;
        ch.order = (int)o;
        ch.ms = (float)ms;
        if (ch.variant < 0 || ch.variant > 1 || ch.order < 0 || ch.order > 1) continue;
        g_table[key] = ch;
        ++n;
    }
    fclose(f);
    return ok_format ? n : -1;
}

int save_locked(const char* path) {
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) return -1;
    fprintf(f, "{\"format\": \"ldk-autotune\", \"version\": 1, \"entries\": [\n");
    int n = 0;
    for (const auto& kv : g_table) {
        const TuneKey& k = kv.first;
        const TuneChoice& c = kv.second;
        ParseShape sh{};
        sh.P = k.P;
        sh.genotypes = k.genotypes;
        fprintf(f,
                "%s {\"pops\": %d, \"genotypes\": %d, \"k_bytes\": %d, \"bins\": %d, \"cutoff_decade\": %d, "
                "\"window_log2\": %d, \"tile_variant\": %d, \"tile_partners\": %d, \"order\": %d, \"ms\": %.4f}\n",
                n ? "," : "", k.P, k.genotypes, k.ktot, k.n_bins, k.cutoff_decade, k.window_log2, c.variant,
                tc_tile_width(sh, c.variant), c.order, (double)c.ms);
        ++n;
    }
    fprintf(f, "]}\n");
    const bool ok = fclose(f) == 0;
    if (!ok || rename(tmp.c_str(), path) != 0) return -1;
    return n;
}

void load_env_once_locked() {
    if (g_env_loaded) return;
    g_env_loaded = true;
    if (const char* p = env_path()) load_locked(p);
}

}  // namespace

TuneKey tune_key_of(const ldk_parse_t* d, const ParseShape& sh) {
    const int nw = d->window_offsets ? d->n_windows : 1;
    const double mean_window = (double)d->n_var / (nw > 0 ? nw : 1);
    TuneKey k;
    k.P = sh.P;
    k.genotypes = sh.genotypes;
    k.ktot = sh.ktot;
    k.n_bins = d->n_bins;
    k.cutoff_decade = d->max_dist >= 1.0 ? (int)std::floor(std::log10(d->max_dist)) : -1;
    k.window_log2 = mean_window >= 1.0 ? (int)std::floor(std::log2(mean_window)) : 0;
    return k;
}

bool tune_lookup(const TuneKey& k, TuneChoice* c) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_env_once_locked();
    auto it = g_table.find(k);
    if (it == g_table.end()) return false;
    *c = it->second;
    return true;
}

void tune_store(const TuneKey& k, const TuneChoice& c) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_env_once_locked();
    g_table[k] = c;
    ++g_tunings;
    if (const char* p = env_path()) save_locked(p);
}

}  // namespace ldk

extern "C" {

int ldk_autotune_load(const char* path) {
    if (!path) { ldk::set_error("null path"); return LDK_ERR_ARG; }
    std::lock_guard<std::mutex> lock(ldk::g_mu);
    const int n = ldk::load_locked(path);
    if (n < 0) { ldk::set_error("cannot read an autotune table from %s", path); return LDK_ERR_ARG; }
    return n;
}

int ldk_autotune_save(const char* path) {
    if (!path) { ldk::set_error("null path"); return LDK_ERR_ARG; }
    std::lock_guard<std::mutex> lock(ldk::g_mu);
    const int n = ldk::save_locked(path);
    if (n < 0) { ldk::set_error("cannot write the autotune table to %s", path); return LDK_ERR_ARG; }
    return n;
}

int ldk_autotune_count(int* tunings) {
    std::lock_guard<std::mutex> lock(ldk::g_mu);
    if (tunings) *tunings = ldk::g_tunings;
    return (int)ldk::g_table.size();
}

int ldk_autotune_clear(void) {
    std::lock_guard<std::mutex> lock(ldk::g_mu);
    ldk::g_table.clear();
    ldk::g_env_loaded = true;  // a cleared table stays empty until loaded again
    return LDK_OK;
}

}  // extern "C"
