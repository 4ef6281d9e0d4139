// C-ABI entry points of the host codec: rate control and codestream assembly over a
// Tier-1 frame the plugin returned, the DCI check, and the reading of a codestream into
// per-block code for decoder_decode.
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>

#include "capi_util.h"
#include "codestream.h"
#include "gail_b200.h"
#include "layout.h"
#include "rate_gpu.h"

using namespace gb;

namespace {

Tier1View viewOf(const GailCudaTier1& t) {
    Tier1View v;
    v.info = reinterpret_cast<const GbCblkInfo*>(t.info);
    v.passLen = t.passLen;
    v.passDist = t.passDist;
    v.data = t.data;
    v.numInfo = t.numInfo;
    v.numPasses = t.numPasses;
    v.numData = t.numData;
    return v;
}

// A writer per (calling thread, layout, label): the packet order is flattened once.
CodestreamWriter& writerFor(const GailCudaLayout& abi, const char* label) {
    thread_local std::unique_ptr<CodestreamWriter> w;
    thread_local std::vector<GbSubband> bands;
    thread_local GailCudaLayout key{};
    const std::string lab = label ? label : "";
    const bool same = w && key.profile == abi.profile && key.width == abi.width && key.height == abi.height &&
                      key.levels == abi.levels && key.guardBits == abi.guardBits && key.numBands == abi.numBands &&
                      key.baseStep == abi.baseStep && w->label() == lab &&
                      std::memcmp(bands.data(), abi.bands, sizeof(GbSubband) * (size_t)abi.numBands) == 0;
    if (!same) {
        Layout L;
        layoutFromAbi(abi, L);
        w = std::make_unique<CodestreamWriter>(L, lab);
        key = abi;
        bands.assign(abi.bands, abi.bands + abi.numBands);
    }
    return *w;
}

void checkTier1(const GailCudaLayout& abi, const GailCudaTier1& t) {
    if ((int)t.numInfo != abi.numCblks) throw std::logic_error("Tier-1 frame and layout have different code-block counts");
    if (t.numInfo && !t.info) throw std::logic_error("Tier-1 frame without block records");
    const GbCblkInfo* info = reinterpret_cast<const GbCblkInfo*>(t.info);
    for (uint32_t i = 0; i < t.numInfo; ++i) {
        const GbCblkInfo& c = info[i];
        if (c.numPasses > 164 || (uint64_t)c.passBase + c.numPasses > t.numPasses ||
            (uint64_t)c.dataOffset + c.dataLen > t.numData)
            throw std::logic_error("Tier-1 block record " + std::to_string(i) + " points outside its tables");
        for (uint32_t k = 0; k < c.numPasses; ++k)
            if (t.passLen[c.passBase + k] > c.dataLen) throw std::logic_error("pass length beyond its codeword");
    }
}

}  // namespace

extern "C" {

GB_API int gb_dci_limits(double fps, double maxMbps, double compMbps, uint64_t* total, uint64_t* comp) {
    return gbGuard([&] {
        const RateLimits l = dciLimits(fps, maxMbps, compMbps);
        if (total) *total = l.maxTotal;
        if (comp) *comp = l.maxComp;
    });
}

GB_API int gb_empty_codestream_bytes(const GailCudaLayout* layout, const char* label, uint64_t* bytes) {
    return gbGuard([&] {
        if (!layout || !bytes) throw std::logic_error("null argument");
        *bytes = writerFor(*layout, label).emptyBytes();
    });
}

GB_API int gb_build_codestream(const GailCudaLayout* layout, const GailCudaTier1* t1, const uint8_t* passes,
                               const char* label, const char* tag, uint8_t* out, uint64_t cap, uint64_t* size) {
    return gbGuard([&] {
        if (!layout || !t1 || !passes || !size) throw std::logic_error("null argument");
        checkTier1(*layout, *t1);
        const Tier1View v = viewOf(*t1);
        for (uint32_t i = 0; i < v.numInfo; ++i)
            if (passes[i] > v.info[i].numPasses) throw std::logic_error("more passes than the block has");
        thread_local std::vector<uint8_t> cs;
        writerFor(*layout, label).build(v, passes, &cs, tag ? tag : "");
        *size = cs.size();
        if (out) {
            if (cs.size() > cap) throw std::logic_error("codestream buffer too small");
            std::memcpy(out, cs.data(), cs.size());
        }
    });
}

GB_API int gb_rate_and_build_hull(const GailCudaLayout* layout, const GailCudaTier1* t1, const uint8_t* hullPasses,
                                  const double* hullSlope, double fps, double maxMbps, double compMbps,
                                  const char* label, const char* tag, uint8_t* passesOut, uint8_t* out, uint64_t cap,
                                  uint64_t* size, double* lambda) {
    return gbGuard([&] {
        if (!layout || !t1 || !size) throw std::logic_error("null argument");
        if (!hullPasses != !hullSlope) throw std::logic_error("hull passes and slopes go together");
        checkTier1(*layout, *t1);
        const Tier1View v = viewOf(*t1);
        CodestreamWriter& w = writerFor(*layout, label);
        const RateLimits lim = dciLimits(fps, maxMbps, compMbps);
        if (w.emptyBytes() > lim.maxTotal) throw std::logic_error("the frame budget is below the smallest codestream");
        const HullView hv{hullPasses, hullSlope};
        const RateResult rr = allocateRate(w, v, lim, hullPasses ? &hv : nullptr);
        thread_local std::vector<uint8_t> cs;
        w.build(v, rr.passes.data(), &cs, tag ? tag : "");
        *size = cs.size();
        if (lambda) *lambda = rr.lambda;
        if (passesOut) std::memcpy(passesOut, rr.passes.data(), rr.passes.size());
        if (out) {
            if (cs.size() > cap) throw std::logic_error("codestream buffer too small");
            std::memcpy(out, cs.data(), cs.size());
        }
    });
}

GB_API int gb_rate_and_build(const GailCudaLayout* layout, const GailCudaTier1* t1, double fps, double maxMbps,
                             double compMbps, const char* label, const char* tag, uint8_t* passesOut, uint8_t* out,
                             uint64_t cap, uint64_t* size, double* lambda) {
    return gb_rate_and_build_hull(layout, t1, nullptr, nullptr, fps, maxMbps, compMbps, label, tag, passesOut, out,
                                  cap, size, lambda);
}

GB_API int gb_device_rate_and_build(int device, const GailCudaLayout* layout, const GailCudaTier1* t1, double fps,
                                    double maxMbps, double compMbps, const char* label, const char* tag,
                                    uint8_t* passesOut, uint8_t* out, uint64_t cap, uint64_t* size, double* lambda) {
    return gbGuard([&] {
        if (!layout || !t1 || !size) throw std::logic_error("null argument");
        checkTier1(*layout, *t1);
        int count = 0;
        GB_CHECK(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) throw std::logic_error("no such device");
        GB_CHECK(cudaSetDevice(device));
        ensureDevice();
        // a device rate control per (calling thread, device, layout, label), on its own stream
        struct Cached {
            int device = -1;
            GailCudaLayout key{};
            std::vector<GbSubband> bands;
            std::string label;
            std::unique_ptr<DeviceRateControl> rc;
            cudaStream_t st = nullptr;
            ~Cached() {
                rc.reset();
                if (st) cudaStreamDestroy(st);
            }
        };
        thread_local Cached c;
        const std::string lab = label ? label : "";
        const bool same = c.rc && c.device == device && c.key.profile == layout->profile &&
                          c.key.width == layout->width && c.key.height == layout->height &&
                          c.key.levels == layout->levels && c.key.guardBits == layout->guardBits &&
                          c.key.numBands == layout->numBands && c.key.baseStep == layout->baseStep && c.label == lab &&
                          std::memcmp(c.bands.data(), layout->bands, sizeof(GbSubband) * (size_t)layout->numBands) == 0;
        if (!same) {
            c.rc.reset();
            if (c.st && c.device != device) {
                cudaStreamDestroy(c.st);
                c.st = nullptr;
            }
            Layout L;
            layoutFromAbi(*layout, L);
            c.rc = std::make_unique<DeviceRateControl>(device, L, lab);
            if (!c.st) GB_CHECK(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
            c.device = device;
            c.key = *layout;
            c.bands.assign(layout->bands, layout->bands + layout->numBands);
            c.label = lab;
        }
        const RateLimits lim = dciLimits(fps, maxMbps, compMbps);
        if (c.rc->emptyBytes() > lim.maxTotal) throw std::logic_error("the frame budget is below the smallest codestream");
        thread_local std::vector<uint8_t> cs;
        const RateResult rr = c.rc->runHost(viewOf(*t1), lim, tag ? tag : "", cs, c.st);
        *size = cs.size();
        if (lambda) *lambda = rr.lambda;
        if (passesOut) std::memcpy(passesOut, rr.passes.data(), rr.passes.size());
        if (out) {
            if (cs.size() > cap) throw std::logic_error("codestream buffer too small");
            std::memcpy(out, cs.data(), cs.size());
        }
    });
}

GB_API int gb_tier1_hull(const GailCudaLayout* layout, const GailCudaTier1* t1, uint8_t* passes, double* slope) {
    return gbGuard([&] {
        if (!layout || !t1 || !passes || !slope) throw std::logic_error("null argument");
        checkTier1(*layout, *t1);
        Layout L;
        layoutFromAbi(*layout, L);
        computeHull(L, viewOf(*t1), passes, slope);
    });
}

GB_API int gb_check_dci(const uint8_t* data, uint64_t size, double fps, char* msg, uint64_t msgCap, int* ok) {
    return gbGuard([&] {
        if (!data || !ok) throw std::logic_error("null argument");
        const DciReport r = checkDci(data, size, fps);
        *ok = r.ok ? 1 : 0;
        if (msg && msgCap) {
            const std::string m = r.ok ? r.comment : r.errors.front();
            std::snprintf(msg, msgCap, "%s", m.c_str());
        }
    });
}

GB_API int gb_parse_codestream(const uint8_t* data, uint64_t size, GbSubband* bands, int maxBands, int* numBands,
                               GbCblkCode* blocks, uint64_t maxBlocks, uint64_t* numBlocks, int* width, int* height,
                               int* profile) {
    return gbGuard([&] {
        if (!data || !numBands || !numBlocks) throw std::logic_error("null argument");
        Layout L;
        std::vector<GbCblkCode> b;
        parseCodestream(data, size, L, b);
        *numBands = (int)L.bands.size();
        *numBlocks = b.size();
        if (width) *width = L.width;
        if (height) *height = L.height;
        if (profile) *profile = L.profile;
        if (bands) {
            if ((int)L.bands.size() > maxBands) throw std::logic_error("band array too small");
            std::memcpy(bands, L.bands.data(), L.bands.size() * sizeof(GbSubband));
        }
        if (blocks) {
            if (b.size() > maxBlocks) throw std::logic_error("block array too small");
            std::memcpy(blocks, b.data(), b.size() * sizeof(GbCblkCode));
        }
    });
}

}  // extern "C"
