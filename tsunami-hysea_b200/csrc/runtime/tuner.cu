// Autotuner of the stepping kernels' warp tilings: search state per key,
// environment overrides and the optional cache file (tuner.h).
#include "tuner.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>

namespace thy {

namespace {

constexpr int kRounds = 2;          // samples of each candidate per dimension
constexpr double kMargin = 0.01;    // an alternative must be this much faster
constexpr int kDims = 3;            // search order: deep phase 2, deep phase 1, general

int &field(Tiling &t, int dim) { return dim == 0 ? t.deep2 : dim == 1 ? t.deep1 : t.general; }

struct Entry {
    Tiling inc;                     // incumbent (best so far)
    int dim = 0;                    // dimension being searched
    int pos = 0;                    // samples taken in it (candidate pos % 3)
    double best[3] = {1e300, 1e300, 1e300};
    bool done = false;
};

// candidate j of the current dimension: j = 0 the incumbent, 1 and 2 the
// other two variants in ascending order
Tiling candidate(const Entry &e, int j)
{
    Tiling t = e.inc;
    if (j == 0) return t;
    const int cur = field(t, e.dim);
    int v = -1;
    for (int k = 0, seen = 0; k < kTilingVariants; k++)
        if (k != cur && ++seen == j) v = k;
    field(t, e.dim) = v;
    return t;
}

struct State {
    std::mutex mu;
    std::map<std::tuple<int, int, int>, Entry> keys;
    bool env_read = false;
    bool forced = false;
    bool off = false;
    Tiling force;
    std::string cache_path;
    std::map<int, bool> cache_loaded;   // per device
};

State &state()
{
    static State s;
    return s;
}

bool parse_tiling(const char *txt, Tiling *t)
{
    int a, b, c;
    if (!txt || std::sscanf(txt, "%d,%d,%d", &a, &b, &c) != 3) return false;
    if (a < 0 || b < 0 || c < 0 || a >= kTilingVariants || b >= kTilingVariants || c >= kTilingVariants) return false;
    t->deep1 = a;
    t->deep2 = b;
    t->general = c;
    return true;
}

void read_env(State &s)
{
    if (s.env_read) return;
    s.env_read = true;
    Tiling t;
    if (parse_tiling(std::getenv("THY_TILING"), &t)) {
        s.forced = true;
        s.force = t;
    }
    const char *off = std::getenv("THY_TUNE");
    if (off && std::strcmp(off, "0") == 0) s.off = true;
    const char *path = std::getenv("THY_TUNE_CACHE");
    if (path && *path) s.cache_path = path;
}

// device identity written to the cache file: name (blanks replaced) and SM count
std::string device_id(int device)
{
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown 0";
    std::string n = p.name;
    for (auto &ch : n)
        if (ch == ' ' || ch == '\t') ch = '_';
    return n + " " + std::to_string(p.multiProcessorCount);
}

void load_cache(State &s, int device)
{
    if (s.cache_path.empty() || s.cache_loaded[device]) return;
    s.cache_loaded[device] = true;
    FILE *f = std::fopen(s.cache_path.c_str(), "r");
    if (!f) return;
    const std::string id = device_id(device);
    char name[256];
    int sms, bd, bg, a, b, c;
    while (std::fscanf(f, "%255s %d %d %d %d %d %d", name, &sms, &bd, &bg, &a, &b, &c) == 7) {
        if (std::string(name) + " " + std::to_string(sms) != id) continue;
        if (a < 0 || b < 0 || c < 0 || a >= kTilingVariants || b >= kTilingVariants || c >= kTilingVariants) continue;
        Entry &e = s.keys[std::make_tuple(device, bd, bg)];
        e.inc.deep1 = a;
        e.inc.deep2 = b;
        e.inc.general = c;
        e.done = true;
    }
    std::fclose(f);
}

void store_cache(const State &s, const TuneKey &k, const Tiling &t)
{
    if (s.cache_path.empty()) return;
    FILE *f = std::fopen(s.cache_path.c_str(), "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d %d %d\n", device_id(k.device).c_str(), k.deep, k.general, t.deep1, t.deep2, t.general);
    std::fclose(f);
}

Entry &entry(State &s, const TuneKey &k)
{
    read_env(s);
    load_cache(s, k.device);
    return s.keys[std::make_tuple(k.device, k.deep, k.general)];
}

}  // namespace

int tune_bucket(double units)
{
    int b = 0;
    while (b < 62 && (double)(1ll << b) < units) b++;
    return b;
}

// Steps of at most kSmallWork units (deep + general, from the buckets' upper
// bounds) are not tuned: the kernels then have fewer units than the GPU has
// resident CTAs, each runs at the latency of one unit, and the graph
// captures a search costs would outweigh what it could find.  They run the
// tiling with the shortest per-warp row chains in the phase-2 kernels (deep
// phase 2 and the general kernel in their most row groups), which the search
// picked at 512 x 512 (13.9 against 17.7 ms of device time for 259 steps
// with the default tiling).
constexpr long long kSmallWork = 512;
bool small_work(const TuneKey &k)
{
    return k.deep < 40 && k.general < 40 && (1ll << k.deep) + (1ll << k.general) <= kSmallWork;
}
Tiling small_tiling()
{
    Tiling t;
    t.deep1 = 0;
    t.deep2 = 2;
    t.general = 2;
    return t;
}

Tiling tuner_pick(const TuneKey &k, bool *sampling)
{
    State &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    Entry &e = entry(s, k);
    *sampling = false;
    if (s.forced) return s.force;
    if (s.off) return Tiling();
    if (small_work(k)) return small_tiling();
    if (e.done) return e.inc;
    *sampling = true;
    return candidate(e, e.pos % 3);
}

void tuner_sample(const TuneKey &k, const Tiling &t, double v)
{
    State &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    Entry &e = entry(s, k);
    if (s.forced || s.off || e.done || small_work(k)) return;
    const int j = e.pos % 3;
    if (t != candidate(e, j) || !(v > 0.0)) return;   // a stale tiling (another batch switched first)
    if (v < e.best[j]) e.best[j] = v;
    if (++e.pos < 3 * kRounds) return;
    int win = 0;
    for (int c = 1; c < 3; c++)
        if (e.best[c] < e.best[win]) win = c;
    if (win != 0 && e.best[win] < e.best[0] * (1.0 - kMargin)) e.inc = candidate(e, win);
    e.pos = 0;
    for (double &b : e.best) b = 1e300;
    if (++e.dim == kDims) {
        e.done = true;
        store_cache(s, k, e.inc);
    }
}

bool tuner_decided(const TuneKey &k, Tiling *best)
{
    State &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    Entry &e = entry(s, k);
    if (s.forced) {
        if (best) *best = s.force;
        return true;
    }
    if (s.off) {
        if (best) *best = Tiling();
        return true;
    }
    if (small_work(k)) {
        if (best) *best = small_tiling();
        return true;
    }
    if (best) *best = e.inc;
    return e.done;
}

void tuner_force(const Tiling *t)
{
    State &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    read_env(s);
    s.forced = t != nullptr;
    if (t) s.force = *t;
}

void tuner_clear()
{
    State &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    s.keys.clear();
    s.cache_loaded.clear();
}

}  // namespace thy
