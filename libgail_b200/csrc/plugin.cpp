// The GAIL CUDA plugin table (gail_cuda_plugin_abi.h): what libgail calls. It turns the
// interface's plain data into this library's objects, runs them, and turns exceptions
// into status codes (the role of the reference's src/cuda/cuda_plugin.cpp:49-245).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "capi_util.h"
#include "decoder.h"
#include "encoder.h"
#include "gail_b200.h"
#include "gail_cuda_plugin_abi.h"
#include "layout.h"

using namespace gb;

struct GailCudaDevice {
    int index = 0;
    std::string name;
    GailCudaLog log = nullptr;
    void* user = nullptr;
};

struct GailCudaEncoder {
    std::unique_ptr<EncoderSlot> slot;
};

struct GailCudaDecoder {
    std::unique_ptr<DecoderSlot> slot;
    Layout frame;
};

namespace {

struct DeviceEntry {
    int index, major, minor;
    uint64_t memory;
    std::string name, uuid, pci;
};

// The devices of the first successful enumeration (the runtime's numbering does not
// change while the process lives).
const std::vector<DeviceEntry>& devices() {
    static const std::vector<DeviceEntry> list = [] {
        int n = 0;
        const cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error(cudaGetErrorString(e));
        }
        std::vector<DeviceEntry> out;
        for (int i = 0; i < n; ++i) {
            cudaDeviceProp p;
            if (cudaGetDeviceProperties(&p, i) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            char uuid[48], pci[32];
            const unsigned char* b = reinterpret_cast<const unsigned char*>(p.uuid.bytes);
            std::snprintf(uuid, sizeof uuid, "GPU-%02x%02x%02x%02x-%02x%02x-%02x%02x-%02x%02x-%02x%02x%02x%02x%02x%02x", b[0],
                          b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8], b[9], b[10], b[11], b[12], b[13], b[14], b[15]);
            std::snprintf(pci, sizeof pci, "%04x:%02x:%02x.0", p.pciDomainID, p.pciBusID, p.pciDeviceID);
            out.push_back({i, p.major, p.minor, (uint64_t)p.totalGlobalMem, p.name, uuid, pci});
        }
        return out;
    }();
    return list;
}

const char* pLastError() { return lastError(); }

int pDeviceCount() {
    int n = -1;
    if (gbGuard([&] { n = (int)devices().size(); }) != kOk) return -1;
    return n;
}

int pDeviceDesc(int index, GailCudaDeviceDesc* out) {
    return gbGuard([&] {
        const DeviceEntry& d = devices().at((size_t)index);
        std::memset(out, 0, sizeof *out);
        out->index = d.index;
        out->smMajor = d.major;
        out->smMinor = d.minor;
        out->memoryBytes = d.memory;
        std::snprintf(out->name, sizeof out->name, "%s", d.name.c_str());
        std::snprintf(out->uuid, sizeof out->uuid, "%s", d.uuid.c_str());
        std::snprintf(out->pciBusId, sizeof out->pciBusId, "%s", d.pci.c_str());
    });
}

int pDeviceUsable(int index) {
    std::string why;
    bool noCode = false;
    const int r = gbGuard([&] {
        const DeviceEntry& d = devices().at((size_t)index);
        cudaError_t e = cudaSetDevice(d.index);
        if (e == cudaSuccess) e = kernelsLoadable();
        if (e == cudaSuccess) return;
        cudaGetLastError();
        noCode = e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction;
        why = noCode ? "not built for this architecture (sm_100a only)" : cudaGetErrorString(e);
    });
    if (r != kOk) return r;
    if (why.empty()) return kOk;
    setLastError(why);
    return noCode ? kNoCode : kError;
}

int pDeviceCreate(int index, GailCudaLog log, void* user, GailCudaDevice** out) {
    return gbGuard([&] {
        const DeviceEntry& d = devices().at((size_t)index);
        GB_CHECK(cudaSetDevice(d.index));
        // slot threads sleep in stream synchronisation rather than spin: a frame takes
        // milliseconds, and the host cores are wanted for rate control
        if (cudaSetDeviceFlags(cudaDeviceScheduleBlockingSync | cudaDeviceMapHost) != cudaSuccess) cudaGetLastError();
        ensureDevice();
        auto dev = std::make_unique<GailCudaDevice>();
        dev->index = d.index;
        dev->name = d.name + " (CUDA)";
        dev->log = log;
        dev->user = user;
        if (log) {
            char buf[512];
            std::snprintf(buf, sizeof buf, "cuda: device %d %s (sm_%d%d, %.1f GB), gail_b200 sm_100a kernels", d.index,
                          d.name.c_str(), d.major, d.minor, d.memory / 1e9);
            log(user, 2, buf);
        }
        *out = dev.release();
    });
}

void pDeviceDestroy(GailCudaDevice* d) { delete d; }
const char* pDeviceName(GailCudaDevice* d) { return d->name.c_str(); }

int pDeviceMemory(GailCudaDevice* d, GailCudaMemory* out) {
    return gbGuard([&] {
        GB_CHECK(cudaSetDevice(d->index));
        size_t f = 0, t = 0;
        GB_CHECK(cudaMemGetInfo(&f, &t));
        *out = {(uint64_t)t, (uint64_t)f, 1};
    });
}

uint64_t pEncoderBytes(GailCudaDevice*, const GailCudaLayout* layout, const GailCudaEncodeSettings* s) {
    uint64_t bytes = 0;
    gbGuard([&] {
        Layout L;
        layoutFromAbi(*layout, L);
        bytes = slotSizes(L, s->input).deviceBytes();
        // an application 3D LUT lives on the device too
        const GailCudaColor& c = s->color;
        uint64_t lut = c.lut3dData ? c.lut3dCount : 0;
        if (!lut && c.lut3d && c.lut3d[0]) {
            int32_t n = 0;
            lut = readCube(c.lut3d, n).size();
        }
        bytes += (lut * 4 + 255) / 256 * 256;
    });
    return bytes;
}

int pEncoderCreate(GailCudaDevice* d, const GailCudaLayout* layout, const GailCudaEncodeSettings* s, GailCudaEncoder** out) {
    return gbGuard([&] {
        GB_CHECK(cudaSetDevice(d->index));
        ensureDevice();
        Layout L;
        layoutFromAbi(*layout, L);
        auto e = std::make_unique<GailCudaEncoder>();
        e->slot = std::make_unique<EncoderSlot>(d->index, L, *s);
        *out = e.release();
    });
}

void pEncoderDestroy(GailCudaEncoder* e) { delete e; }
void* pEncoderInput(GailCudaEncoder* e) { return e->slot->inputBuffer(); }
void pEncoderSetSlope(GailCudaEncoder* e, double t) { e->slot->setSlope(t); }

int pEncoderEncode(GailCudaEncoder* e, const void* frame, GailCudaTier1* out, GbFrameTimings* tm, GailCudaDebug* dbg) {
    return gbGuard([&] { e->slot->encode(frame, out, tm, dbg); });
}

uint64_t pDecoderBytes(GailCudaDevice*, const GailCudaLayout* layout, const GailCudaDecodeSettings* s) {
    uint64_t bytes = 0;
    gbGuard([&] {
        Layout L;
        layoutFromAbi(*layout, L);
        bytes = decoderSlotBytes(L, *s);
    });
    return bytes;
}

int pDecoderCreate(GailCudaDevice* d, const GailCudaLayout* layout, const GailCudaDecodeSettings* s, GailCudaDecoder** out) {
    return gbGuard([&] {
        GB_CHECK(cudaSetDevice(d->index));
        ensureDevice();
        Layout L;
        layoutFromAbi(*layout, L);
        auto dec = std::make_unique<GailCudaDecoder>();
        dec->frame = L;
        dec->slot = std::make_unique<DecoderSlot>(d->index, L, *s);
        *out = dec.release();
    });
}

void pDecoderDestroy(GailCudaDecoder* d) { delete d; }

int pDecoderDecode(GailCudaDecoder* d, const GailCudaLayout* frame, const uint8_t* data, size_t size, const GbCblkCode* blocks,
                   size_t numBlocks, void* dst, ptrdiff_t strideBytes, GailCudaDecodeTimings* tm) {
    return gbGuard([&] {
        layoutFromAbi(*frame, d->frame);
        d->slot->decode(d->frame, data, size, blocks, numBlocks, dst, strideBytes, tm);
    });
}

// FNV-1a over the sizes of the structures that cross the boundary, as libgail computes
// it (cudaPluginLayout, src/cuda/cuda_plugin.h:208-217); evaluated at compile time, so the
// table below is a constant and nothing runs when the library loads.
constexpr uint64_t layoutHash() {
    constexpr uint64_t sizes[] = {sizeof(GbSubband),          sizeof(GbCblkInfo),         sizeof(GbCblkCode),
                                  sizeof(GbFrameFormat),      sizeof(GbFrameTimings),     sizeof(GailCudaDeviceDesc),
                                  sizeof(GailCudaLayout),     sizeof(GailCudaEncodeSettings), sizeof(GailCudaTier1),
                                  sizeof(GailCudaDebug),      sizeof(GailCudaDecodeTimings), sizeof(GailCudaPlugin)};
    uint64_t h = 1469598103934665603ull;
    for (uint64_t v : sizes) h = (h ^ v) * 1099511628211ull;
    return h;
}

// The toolkit that compiled this file: nvcc's own version macros.
#define GB_STR2(x) #x
#define GB_STR(x) GB_STR2(x)
#define GB_TOOLKIT_VERSION GB_STR(__CUDACC_VER_MAJOR__) "." GB_STR(__CUDACC_VER_MINOR__) "." GB_STR(__CUDACC_VER_BUILD__)

constexpr GailCudaPlugin kPlugin = {
    GAIL_CUDA_PLUGIN_ABI,
    (uint32_t)sizeof(GailCudaPlugin),
    layoutHash(),
    "gail_cuda13",
    GB_TOOLKIT_VERSION,
    "100a",
    pLastError,
    pDeviceCount,
    pDeviceDesc,
    pDeviceUsable,
    pDeviceCreate,
    pDeviceDestroy,
    pDeviceName,
    pDeviceMemory,
    pEncoderBytes,
    pEncoderCreate,
    pEncoderDestroy,
    pEncoderInput,
    pEncoderSetSlope,
    pEncoderEncode,
    pDecoderBytes,
    pDecoderCreate,
    pDecoderDestroy,
    pDecoderDecode,
};

}  // namespace

extern "C" const GailCudaPlugin* gail_cuda_plugin_get(uint32_t abi) { return abi == GAIL_CUDA_PLUGIN_ABI ? &kPlugin : nullptr; }

extern "C" GB_API uint64_t gb_plugin_layout_hash(void) { return layoutHash(); }

// ---- device-resident frames (gail_b200.h) -------------------------------------------
extern "C" GB_API void* gb_encoder_stream(GailCudaEncoder* e) { return e ? (void*)e->slot->stream() : nullptr; }

extern "C" GB_API int gb_encoder_enqueue_device(GailCudaEncoder* e, const void* dFrame) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("no encoder");
        e->slot->enqueue(dFrame);
    });
}

extern "C" GB_API int gb_encoder_finish(GailCudaEncoder* e) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("no encoder");
        e->slot->finish();
    });
}

extern "C" GB_API int gb_encoder_stage_timing(GailCudaEncoder* e, int on) {
    return gbGuard([&] {
        if (!e) throw std::logic_error("no encoder");
        e->slot->setTiming(on != 0);
    });
}

extern "C" GB_API int gb_encoder_stage_times(GailCudaEncoder* e, double* ms5, int* count) {
    return gbGuard([&] {
        if (!e || !ms5 || !count) throw std::logic_error("null argument");
        *count = e->slot->stageTimes(ms5);
    });
}
