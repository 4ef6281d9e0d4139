// C-ABI of the batched, served encode engine (engine.h).
#include <memory>

#include "capi_util.h"
#include "engine.h"
#include "gail_b200.h"

struct GbEngine {
    std::unique_ptr<gb::EncodeEngine> e;
};

using namespace gb;

extern "C" {

GB_API int gb_engine_create(int device, uint64_t hbmBudget, int maxBatch, GbEngine** out) {
    return gbGuard([&] {
        if (!out) throw std::logic_error("null argument");
        auto g = std::make_unique<GbEngine>();
        g->e = std::make_unique<EncodeEngine>(device, hbmBudget, maxBatch);
        *out = g.release();
    });
}

GB_API void gb_engine_destroy(GbEngine* e) { delete e; }

GB_API int gb_engine_add_encoder(GbEngine* e, const GailCudaLayout* layout, const GailCudaEncodeSettings* settings,
                                 int* classId, uint64_t* frameBytes) {
    return gbGuard([&] {
        if (!e || !layout || !settings || !classId) throw std::logic_error("null argument");
        *classId = e->e->addClass(*layout, *settings, frameBytes);
    });
}

GB_API int gb_engine_submit(GbEngine* e, int classId, const void* frame, int onDevice, double slope, int64_t* id) {
    return gbGuard([&] {
        if (!e || !id) throw std::logic_error("null argument");
        *id = e->e->submit(classId, frame, onDevice != 0, slope);
    });
}

GB_API int gb_engine_wait(GbEngine* e, int timeoutMs, int64_t* id, GailCudaTier1* out, double* latencyMs, int* frameStatus) {
    return gbGuard([&] {
        if (!e || !id || !out || !latencyMs || !frameStatus) throw std::logic_error("null argument");
        if (!e->e->wait(timeoutMs, id, out, latencyMs, frameStatus)) *id = -1;
    });
}

GB_API int gb_engine_release(GbEngine* e, int64_t id) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("null argument");
        e->e->release(id);
    });
}

GB_API int gb_engine_set_codestream(GbEngine* e, double fps, double maxMbps, double compMbps, const char* label,
                                    const char* tag, int threads, int check, int flags) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("null argument");
        if (flags & ~(GB_CS_HOST | GB_CS_TIER1)) throw std::logic_error("unknown codestream flags");
        EncodeEngine::CodestreamConfig c;
        c.onDevice = !(flags & GB_CS_HOST);
        c.tier1 = (flags & GB_CS_TIER1) != 0;
        c.fps = fps;
        c.maxMbps = maxMbps;
        c.compMbps = compMbps;
        c.label = label ? label : "";
        c.tag = tag ? tag : "";
        c.threads = threads;
        c.check = check != 0;
        e->e->setCodestream(c);
    });
}

GB_API int gb_engine_codestream(GbEngine* e, int64_t id, const uint8_t** data, uint64_t* size, int* dciOk) {
    return gbGuard([&] {
        if (!e || !data || !size || !dciOk) throw std::logic_error("null argument");
        if (!e->e->codestream(id, data, size, dciOk)) throw std::logic_error("codestreams are off");
    });
}

GB_API int gb_engine_add_decoder(GbEngine* e, const GailCudaLayout* layout, const GailCudaDecodeSettings* settings,
                                 int* classId, uint64_t* frameBytes) {
    return gbGuard([&] {
        if (!e || !layout || !settings || !classId) throw std::logic_error("null argument");
        *classId = e->e->addDecodeClass(*layout, *settings, frameBytes);
    });
}

GB_API int gb_engine_submit_decode(GbEngine* e, int classId, const uint8_t* data, uint64_t size, int64_t* id) {
    return gbGuard([&] {
        if (!e || !id) throw std::logic_error("null argument");
        *id = e->e->submitDecode(classId, data, size);
    });
}

GB_API int gb_engine_picture(GbEngine* e, int64_t id, const uint16_t** pix, int* width, int* height) {
    return gbGuard([&] {
        if (!e || !pix || !width || !height) throw std::logic_error("null argument");
        if (!e->e->picture(id, pix, width, height)) throw std::logic_error("not a decode request");
    });
}

GB_API int gb_engine_hull(GbEngine* e, int64_t id, const uint8_t** passes, const double** slope) {
    return gbGuard([&] {
        if (!e || !passes || !slope) throw std::logic_error("null argument");
        if (!e->e->hull(id, passes, slope)) throw std::logic_error("not an encode request");
    });
}

GB_API int gb_engine_set_slope_factor(GbEngine* e, double factor) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("null argument");
        e->e->setSlopeFactor(factor);
    });
}

GB_API int gb_engine_frame_info(GbEngine* e, int64_t id, double* threshold, int* recoded) {
    return gbGuard([&] {
        if (!e || !threshold || !recoded) throw std::logic_error("null argument");
        if (!e->e->frameInfo(id, threshold, recoded)) throw std::logic_error("not an encode request");
    });
}

GB_API int gb_engine_set_policy(GbEngine* e, int maxBatch, int minBatchPct, double maxWaitMs) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("null argument");
        e->e->setPolicy(maxBatch, minBatchPct, maxWaitMs);
    });
}

GB_API int gb_engine_counters(GbEngine* e, uint64_t* h2d, uint64_t* d2h, uint64_t* launches) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("null argument");
        const EncodeEngine::Stats s = e->e->stats();
        if (h2d) *h2d = s.h2dBytes;
        if (d2h) *d2h = s.d2hBytes;
        if (launches) *launches = s.launches;
    });
}

GB_API int gb_engine_stage_timing(GbEngine* e, int on) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("null argument");
        e->e->setStageTiming(on != 0);
    });
}

GB_API int gb_engine_stage_times(GbEngine* e, int reset, double* ms6, uint64_t* counts4) {
    return gbGuard([&] {
        if (!e || !ms6 || !counts4) throw std::logic_error("null argument");
        const EncodeEngine::StageTimes t = e->e->stageTimes(reset != 0);
        const double ms[6] = {t.frontMs, t.cmMs, t.orderMs, t.mqMs, t.packMs, t.rcMs};
        const uint64_t n[4] = {t.frontFrames, t.batches, t.batchFrames, t.rcFrames};
        for (int i = 0; i < 6; ++i) ms6[i] = ms[i];
        for (int i = 0; i < 4; ++i) counts4[i] = n[i];
    });
}

GB_API int gb_engine_stats(GbEngine* e, uint64_t* out5) {
    return gbGuard([&] {
        if (!e || !out5) throw std::logic_error("null argument");
        const EncodeEngine::Stats s = e->e->stats();
        out5[0] = s.frames;
        out5[1] = s.batches;
        out5[2] = s.batchFrames;
        out5[3] = s.slots;
        out5[4] = s.slotBytes;
    });
}

}  // extern "C"
