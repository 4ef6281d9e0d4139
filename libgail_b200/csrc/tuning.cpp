// Launch tuning per frame profile (see tuning.h).
#include "tuning.h"

#include <mutex>
#include <stdexcept>

namespace gb {

namespace {
std::mutex g_m;
Tuning g_t[2];
}  // namespace

Tuning defaultTuning() { return Tuning{}; }

Tuning tuningFor(int profile) {
    std::lock_guard<std::mutex> lock(g_m);
    return g_t[profile == 1 ? 1 : 0];
}

void setTuning(int profile, const Tuning& t) {
    if (profile != 0 && profile != 1) throw std::logic_error("tuning profile must be 0 (2K) or 1 (4K)");
    if (t.soloDecisions < 256) throw std::logic_error("solo threshold below 256 decisions");
    if (t.cmCtasPerSm < 1 || t.cmCtasPerSm > 64 || t.mqCtasPerSm < 1 || t.mqCtasPerSm > 64 || t.decCtasPerSm < 1 ||
        t.decCtasPerSm > 64)
        throw std::logic_error("grid caps must be 1..64 CTAs per SM");
    if (t.t1Persistent != 0 && t.t1Persistent != 1) throw std::logic_error("t1Persistent must be 0 or 1");
    if (t.decHeavyPct < 0 || t.decHeavyPct > 100000) throw std::logic_error("decHeavyPct must be 0..100000");
    if (t.dwtTile1 < 0 || t.dwtTile1 > 2 || t.dwtTileN < 0 || t.dwtTileN > 2)
        throw std::logic_error("tile shapes must be 0 (64 x 64), 1 (128 x 64) or 2 (64 x 128)");
    Tuning v = t;
    uint32_t p = 1;
    while (p * 2 <= v.soloDecisions && p < (1u << 30)) p *= 2;
    v.soloDecisions = p;  // a boundary of the largest-first order
    std::lock_guard<std::mutex> lock(g_m);
    g_t[profile] = v;
}

void resetTuning(int profile) {
    std::lock_guard<std::mutex> lock(g_m);
    g_t[profile == 1 ? 1 : 0] = Tuning{};
}

}  // namespace gb
