// Launch tuning per frame profile (0 = 2K, 1 = 4K): the knobs whose best value depends on the
// workload and the GPU, set by the autotuner (libgail_b200/autotune.py) through
// gb_set_tuning and read by every launch of that profile.
#pragma once
#include <cstdint>

namespace gb {

struct Tuning {
    uint32_t soloDecisions = 16384;  // MQ: blocks with at least this many decisions coded alone in a warp
    int cmCtasPerSm = 16;            // context modelling grid cap
    int mqCtasPerSm = 16;            // MQ grid cap
    int decCtasPerSm = 32;           // Tier-1 decode grid cap
    int t1Persistent = 0;            // Tier-1 encode as one persistent launch (1) or four (0)
    int decHeavyPct = 150;           // Tier-1 decode: blocks above this % of the mean codeword bytes per
                                     // warp run on SMs of their own (0: none)
    int dwtTile1 = 0;                // front-end tile at level 1: 0 = 64 x 64, 1 = 128 x 64, 2 = 64 x 128
    int dwtTileN = 0;                // the same for levels 2..
};

Tuning defaultTuning();
Tuning tuningFor(int profile);
// Validates and stores (soloDecisions rounded down to a power of two, caps clamped to the
// hardware's resident limits); throws std::logic_error on a value out of range.
void setTuning(int profile, const Tuning& t);
void resetTuning(int profile);

}  // namespace gb
