// C-ABI of the batched, served encode engine (engine.h).
#include <atomic>
#include <chrono>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

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

GB_API int gb_engine_reserve(GbEngine* e, int classId, int slots, int* have) {
    return gbGuard([&] {
        if (!e || slots < 0) throw std::logic_error("bad argument");
        const int h = e->e->reserve(classId, slots);
        if (have) *have = h;
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

GB_API int gb_engine_open_loop(GbEngine* e, uint32_t n, const int* classId, const int* kind, const void* const* item,
                               const uint64_t* size, const int* onDevice, const double* arrivalSec, double* latencyMs,
                               int* status, double* elapsedSec) {
    return gbGuard([&] {
        if (!e || (n && (!classId || !kind || !item || !arrivalSec || !latencyMs || !status)) || !elapsedSec)
            throw std::logic_error("null argument");
        for (uint32_t i = 0; i < n; ++i) {
            if (kind[i] != 0 && kind[i] != 1) throw std::logic_error("request kind is 0 (encode) or 1 (decode)");
            if (kind[i] == 1 && !size) throw std::logic_error("decode requests need their sizes");
            if (i && arrivalSec[i] < arrivalSec[i - 1]) throw std::logic_error("arrival times must not decrease");
        }
        using Clock = std::chrono::steady_clock;
        EncodeEngine& eng = *e->e;
        // the collector: every finished request's latency and status by id, released at once
        struct Done {
            double ms;
            int st;
        };
        std::unordered_map<int64_t, Done> done;
        done.reserve(n);
        std::string failure;
        std::atomic<bool> abort{false};
        Clock::time_point last;
        const auto t0 = Clock::now();
        std::thread collector([&] {
            try {
                for (uint32_t k = 0; k < n && !abort.load(); ++k) {
                    int64_t id = -1;
                    GailCudaTier1 t1{};
                    double ms = 0;
                    int st = 0;
                    while (!eng.wait(1000, &id, &t1, &ms, &st))
                        if (abort.load()) return;
                    done[id] = {ms, st};
                    eng.release(id);
                }
                last = Clock::now();
            } catch (const std::exception& ex) {
                failure = ex.what();
                abort = true;
            }
        });
        std::vector<int64_t> ids(n, -1);
        try {
            for (uint32_t i = 0; i < n && !abort.load(); ++i) {
                std::this_thread::sleep_until(t0 + std::chrono::duration_cast<Clock::duration>(
                                                       std::chrono::duration<double>(arrivalSec[i])));
                ids[i] = kind[i] == 0 ? eng.submit(classId[i], item[i], onDevice && onDevice[i], 0.0)
                                      : eng.submitDecode(classId[i], static_cast<const uint8_t*>(item[i]), size[i]);
            }
        } catch (...) {
            abort = true;
            collector.join();
            throw;
        }
        collector.join();
        if (!failure.empty()) throw std::runtime_error(failure);
        for (uint32_t i = 0; i < n; ++i) {
            const auto it = done.find(ids[i]);
            if (it == done.end()) throw std::runtime_error("a request did not come back");
            latencyMs[i] = it->second.ms;
            status[i] = it->second.st;
        }
        *elapsedSec = n ? std::chrono::duration<double>(last - t0).count() : 0.0;
    });
}

GB_API int gb_engine_decode_times(GbEngine* e, int reset, double* ms3, uint64_t* counts2) {
    return gbGuard([&] {
        if (!e || !ms3 || !counts2) throw std::logic_error("null argument");
        const EncodeEngine::DecodeTimes t = e->e->decodeTimes(reset != 0);
        ms3[0] = t.waitMs;
        ms3[1] = t.parseMs;
        ms3[2] = t.runMs;
        counts2[0] = t.decodes;
        counts2[1] = t.slotsMadeLater;
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
