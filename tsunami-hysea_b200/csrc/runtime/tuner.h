// Autotuner of the stepping kernels' warp tilings (kernels.h: Tiling).
//
// A tiling does not change any cell's arithmetic, only how the warps of a CTA
// share a work unit and how many CTAs an SM keeps, so the tuner times real
// chunks of real runs: every full chunk a batch steps is one sample of the
// tiling it ran with (device time per stepped unit).  Samples are kept per key
// (below), process-wide, so that every batch and every run with that work
// shares one search.  The search is coordinate descent over the three
// kernels (deep phase 2, deep phase 1, general), each dimension timing the
// incumbent and its two alternatives round robin, kRounds samples each, the
// minimum of each kept; an alternative replaces the incumbent when it is more
// than 1 % faster.  A decided key runs its best tiling from then on.
//
// Steps of at most 512 work units are not tuned: they run the tiling with
// the most row groups in the phase-2 kernels (deep 1 default, deep 2 and
// general variant 2).
//
// Environment: THY_TILING="d1,d2,g" forces a tiling (variant indices);
// THY_TUNE=0 keeps the default tiling; THY_TUNE_CACHE=<file> keeps decided
// keys across processes (one line per key: device name, SM count, deep and
// general buckets, tiling).
#pragma once
#include "../kernels/kernels.h"

namespace thy {

// Key: the device and the work of a step, as ceil log2 buckets of its deep
// units and of its general units (the best tiling of each kernel depends on
// how many units it has to spread over the SMs).
struct TuneKey {
    int device;
    int deep;      // tune_bucket(deep units per step)
    int general;   // tune_bucket(general units per step)
};

int tune_bucket(double units);                       // ceil log2, 0 for units <= 1
// tiling for the next chunk of a batch with this key; *sampling: the chunk's
// time is wanted
Tiling tuner_pick(const TuneKey &k, bool *sampling);
// one sample: the tiling a full chunk ran with, device ms per stepped unit
void tuner_sample(const TuneKey &k, const Tiling &t, double ms_per_unit_step);
bool tuner_decided(const TuneKey &k, Tiling *best);
void tuner_force(const Tiling *t);                   // nullptr: tune again
void tuner_clear();                                  // forget every key (not the cache file)

}  // namespace thy
