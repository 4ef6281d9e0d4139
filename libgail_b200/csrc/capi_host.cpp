// C-ABI entry points over the host-side pieces that callers without libgail need to
// drive the plugin: the frame layout and the colour tables.
#include <cstring>
#include <stdexcept>

#include "capi_util.h"
#include "color.h"
#include "gail_b200.h"
#include "layout.h"
#include "tuning.h"

using namespace gb;

extern "C" {

GB_API int gb_make_layout(int width, int height, int fourk, double baseStep, GbSubband* bands, int maxBands,
                          int* numBands, int* numCblks) {
    return gbGuard([&] {
        const Layout L = makeLayout(width, height, fourk ? 1 : 0, baseStep);
        if ((int)L.bands.size() > maxBands) throw std::logic_error("band array too small");
        std::memcpy(bands, L.bands.data(), L.bands.size() * sizeof(GbSubband));
        *numBands = (int)L.bands.size();
        *numCblks = L.numCblks();
    });
}

GB_API int gb_color_tables(const GailCudaColor* color, float* eotf65536, float* matrix9, float* thresholds4096) {
    return gbGuard([&] {
        const ColorTables t = buildColorTables(*color);
        if (eotf65536) std::memcpy(eotf65536, t.eotf.data(), 65536 * 4);
        if (matrix9) std::memcpy(matrix9, t.m, 36);
        if (thresholds4096) std::memcpy(thresholds4096, t.thr.data(), 4096 * 4);
    });
}

GB_API int gb_set_tuning(int profile, const GbTuning* t) {
    return gbGuard([&] {
        if (!t) {
            if (profile != 0 && profile != 1) throw std::logic_error("tuning profile must be 0 (2K) or 1 (4K)");
            resetTuning(profile);
            return;
        }
        Tuning v;
        v.soloDecisions = t->soloDecisions;
        v.cmCtasPerSm = t->cmCtasPerSm;
        v.mqCtasPerSm = t->mqCtasPerSm;
        v.decCtasPerSm = t->decCtasPerSm;
        v.t1Persistent = t->t1Persistent;
        v.decHeavyPct = t->decHeavyPct;
        setTuning(profile, v);
    });
}

GB_API int gb_get_tuning(int profile, GbTuning* t) {
    return gbGuard([&] {
        if (!t) throw std::logic_error("null argument");
        if (profile != 0 && profile != 1) throw std::logic_error("tuning profile must be 0 (2K) or 1 (4K)");
        const Tuning v = tuningFor(profile);
        *t = {v.soloDecisions, v.cmCtasPerSm, v.mqCtasPerSm, v.decCtasPerSm, v.t1Persistent, v.decHeavyPct};
    });
}

}  // extern "C"
