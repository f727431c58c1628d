// Drives the tiling autotuner (runtime/tuner.cu) with synthetic chunk times
// on the host: a cost per tiling, samples fed the way Batch::run_chunk feeds
// them, the decision printed.  Used by tests/test_tuner.py; no GPU needed.
//
//   tuner_driver <scenario>
//   descent  costs with a known coordinate-descent answer
//   margin   an alternative less than 1 % faster is not taken
//   stale    samples of a tiling other than the expected one are ignored
//   noisy    each candidate's minimum over its samples counts
//   keys     buckets are independent
//   cache    THY_TUNE_CACHE written on a decision, read by a fresh search
#include "runtime/tuner.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

using namespace thy;

// cost model: per-kernel contributions, one per variant
struct Costs {
    double d1[3], d2[3], g[3];
    double of(const Tiling &t) const { return d1[t.deep1] + d2[t.deep2] + g[t.general]; }
};

static int run_to_decision(const TuneKey &k, const Costs &c, double noise_amp, int *chunks)
{
    int n = 0;
    Tiling best;
    while (!tuner_decided(k, &best) && n < 1000) {
        bool sampling = false;
        const Tiling t = tuner_pick(k, &sampling);
        if (!sampling) break;
        // deterministic noise: every other sample of a tiling is slower
        const double v = c.of(t) * (1.0 + ((n & 1) ? noise_amp : 0.0));
        tuner_sample(k, t, v);
        n++;
    }
    *chunks = n;
    return 0;
}

static void print(const char *tag, const TuneKey &k, int chunks)
{
    Tiling t;
    const bool done = tuner_decided(k, &t);
    std::printf("%s done=%d tiling=%d,%d,%d chunks=%d\n", tag, done ? 1 : 0, t.deep1, t.deep2, t.general, chunks);
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    const char *sc = argv[1];
    const TuneKey k{0, 13, 10};
    int chunks = 0;
    if (!std::strcmp(sc, "descent")) {
        // deep phase 2 best at variant 1, deep phase 1 at 2, general at 0
        Costs c{{1.0, 0.9, 0.8}, {1.0, 0.7, 1.2}, {0.5, 0.6, 0.55}};
        run_to_decision(k, c, 0.0, &chunks);
        print("descent", k, chunks);
    } else if (!std::strcmp(sc, "margin")) {
        // alternatives 0.5 % faster everywhere: the default stays
        Costs c{{1.0, 0.995, 0.996}, {1.0, 0.995, 0.999}, {1.0, 0.996, 0.995}};
        run_to_decision(k, c, 0.0, &chunks);
        print("margin", k, chunks);
    } else if (!std::strcmp(sc, "stale")) {
        Costs c{{1.0, 0.9, 1.1}, {1.0, 1.1, 1.2}, {1.0, 1.1, 1.2}};
        // a sample of a tiling that is not the current candidate changes nothing
        Tiling wrong;
        wrong.deep2 = 2;
        wrong.deep1 = 2;
        for (int i = 0; i < 50; i++) tuner_sample(k, wrong, 1e-9);
        bool s = false;
        const Tiling t = tuner_pick(k, &s);
        std::printf("stale first=%d,%d,%d sampling=%d\n", t.deep1, t.deep2, t.general, s ? 1 : 0);
        run_to_decision(k, c, 0.0, &chunks);
        print("stale", k, chunks);
    } else if (!std::strcmp(sc, "noisy")) {
        // every other sample 30 % slow: minima decide, as without noise
        Costs c{{1.0, 0.9, 0.8}, {1.0, 0.7, 1.2}, {0.5, 0.6, 0.55}};
        run_to_decision(k, c, 0.3, &chunks);
        print("noisy", k, chunks);
    } else if (!std::strcmp(sc, "keys")) {
        Costs a{{1.0, 0.5, 1.0}, {1.0, 1.0, 1.0}, {1.0, 1.0, 1.0}};
        Costs b{{1.0, 1.0, 1.0}, {1.0, 1.0, 1.0}, {1.0, 1.0, 0.5}};
        const TuneKey k2{0, 10, 3};
        run_to_decision(k, a, 0.0, &chunks);
        print("keys-a", k, chunks);
        run_to_decision(k2, b, 0.0, &chunks);
        print("keys-b", k2, chunks);
        std::printf("bucket 1=%d 2=%d 3=%d 1024=%d 1025=%d\n", tune_bucket(1), tune_bucket(2), tune_bucket(3),
                    tune_bucket(1024), tune_bucket(1025));
    } else if (!std::strcmp(sc, "small")) {
        // a step of at most 512 units: the short-chain tiling, decided, no sample wanted
        const TuneKey ks{0, 7, 8};
        bool s = true;
        const Tiling t = tuner_pick(ks, &s);
        Tiling best;
        best.deep1 = 9;
        const bool done = tuner_decided(ks, &best);
        std::printf("small pick=%d,%d,%d sampling=%d done=%d best=%d,%d,%d\n", t.deep1, t.deep2, t.general, s ? 1 : 0,
                    done ? 1 : 0, best.deep1, best.deep2, best.general);
        const TuneKey kb{0, 9, 1};   // 514 units: tuned
        const Tiling u = tuner_pick(kb, &s);
        std::printf("larger pick=%d,%d,%d sampling=%d\n", u.deep1, u.deep2, u.general, s ? 1 : 0);
    } else if (!std::strcmp(sc, "cache")) {
        // first process: decide and write; then forget and read back
        Costs c{{1.0, 0.5, 1.0}, {1.0, 1.0, 0.5}, {1.0, 1.0, 1.0}};
        run_to_decision(k, c, 0.0, &chunks);
        print("cache-write", k, chunks);
        tuner_clear();
        print("cache-read", k, 0);
    } else if (!std::strcmp(sc, "force")) {
        Tiling f;
        f.deep1 = 2;
        f.deep2 = 1;
        f.general = 2;
        tuner_force(&f);
        bool s = true;
        const Tiling t = tuner_pick(k, &s);
        std::printf("force pick=%d,%d,%d sampling=%d\n", t.deep1, t.deep2, t.general, s ? 1 : 0);
        tuner_force(nullptr);
        const Tiling u = tuner_pick(k, &s);
        std::printf("unforced pick=%d,%d,%d sampling=%d\n", u.deep1, u.deep2, u.general, s ? 1 : 0);
    } else {
        return 2;
    }
    return 0;
}
