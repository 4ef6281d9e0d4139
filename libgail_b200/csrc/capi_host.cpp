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

GB_API int gb_color_route(const GailCudaColor* color, float* params48, int32_t* route, int32_t* lutN) {
    return gbGuard([&] {
        if (!color || !params48) throw std::logic_error("null argument");
        const ColorTables t = buildColorTables(*color);
        const ToneParams& p = t.tone;
        // the reference's parameter-block positions (kernels/color_params.h)
        float* o = params48;
        std::memset(o, 0, 48 * 4);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) o[4 * r + c] = t.m[3 * r + c];
        o[12] = (float)p.tone;
        o[13] = p.srcRef;
        o[14] = p.gain;
        o[15] = p.knee;
        o[16] = p.shoulderT;
        o[17] = p.peak;
        o[18] = (float)p.gamut;
        o[19] = p.gamutThresh;
        std::memcpy(o + 20, p.toTarget, 36);
        std::memcpy(o + 29, p.fromTarget, 36);
        o[38] = (float)t.lutN;
        o[39] = p.pqSrcMax;
        o[40] = p.pqMaxLum;
        o[41] = p.pqKs;
        o[42] = (float)p.norm;
        if (route) *route = t.route;
        if (lutN) *lutN = t.lutN;
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
        v.dwtTile1 = t->dwtTile1;
        v.dwtTileN = t->dwtTileN;
        setTuning(profile, v);
    });
}

GB_API int gb_get_tuning(int profile, GbTuning* t) {
    return gbGuard([&] {
        if (!t) throw std::logic_error("null argument");
        if (profile != 0 && profile != 1) throw std::logic_error("tuning profile must be 0 (2K) or 1 (4K)");
        const Tuning v = tuningFor(profile);
        *t = {v.soloDecisions, v.cmCtasPerSm, v.mqCtasPerSm, v.decCtasPerSm, v.t1Persistent, v.decHeavyPct,
              v.dwtTile1, v.dwtTileN};
    });
}

}  // extern "C"
