// Test harness: drives the reference's public C API (include/gail/gail.h), as an
// application does, over oracle/_ref/libgail.so: the reference library built from its own
// sources (src/api, src/core and the CUDA plugin loader src/cuda/cuda_host.cpp) with no
// CUDA plugin of its own. Placed next to a libgail_cuda13.so, that library loads it through
// CudaHost (dlopen, gail_cuda_plugin_get, the ABI / size / layout checks) and runs its CUDA
// backend on it. TEST INFRASTRUCTURE ONLY: the drop-in test loads this; the product never
// does.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "gail/gail.h"

namespace {
thread_local std::string g_err;

void copyOut(const char* s, char* buf, size_t cap) {
    if (!buf || !cap) return;
    std::strncpy(buf, s ? s : "", cap - 1);
    buf[cap - 1] = 0;
}

struct EncodeArgs {
    int backend;    // gail_backend
    int profile;    // gail_profile
    int container;  // gail_container
    int format;     // gail_pixel_format
    int matrix;     // gail_matrix (Y'CbCr input)
    int preset;     // gail_preset (R'G'B' / Y'CbCr input), -1: the defaults
    double fps, maxMbps;
    int framesInFlight;
};

bool configure(const EncodeArgs& a, gail_config& c) {
    gail_config_defaults(&c);
    c.profile = (gail_profile)a.profile;
    c.container = (gail_container)a.container;
    c.fps = a.fps;
    c.max_mbps = a.maxMbps;
    c.backend = (gail_backend)a.backend;
    c.input.format = (gail_pixel_format)a.format;
    c.input.matrix = (gail_matrix)a.matrix;
    if (a.preset >= 0) gail_color_preset((gail_preset)a.preset, &c.color);
    c.frames_in_flight = a.framesInFlight;
    c.check = 1;
    return true;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* probe_last_error() { return g_err.c_str(); }

__attribute__((visibility("default"))) const char* probe_version() { return gail_version_string(); }

__attribute__((visibility("default"))) int probe_list_devices(int backend, char* buf, size_t cap) {
    return gail_list_devices((gail_backend)backend, buf, cap);
}

// Encodes `count` frames (each three plane pointers; R'G'B' / X'Y'Z' use plane 0) on one
// encoder through gail_encoder_send / gail_encoder_receive, in send order. Codestream i goes
// to out + i * cap; sizes[i] and compliant[i] are set. Returns GAIL_OK or a status
// (probe_last_error() then says why).
static int encodeStream(int backend, int profile, int container, int format, int matrix, int preset, double fps,
                        double maxMbps, int framesInFlight, const void* const* planes, int count, uint8_t* out,
                        size_t cap, uint64_t* sizes, int* compliant, char* devices, size_t devCap, double* seconds);

__attribute__((visibility("default"))) int probe_encode(int backend, int profile, int container, int format,
                                                        int matrix, int preset, double fps, double maxMbps,
                                                        int framesInFlight, const void* const* planes, int count,
                                                        uint8_t* out, size_t cap, uint64_t* sizes, int* compliant,
                                                        char* devices, size_t devCap) {
    return encodeStream(backend, profile, container, format, matrix, preset, fps, maxMbps, framesInFlight, planes,
                        count, out, cap, sizes, compliant, devices, devCap, nullptr);
}

// probe_encode with the seconds from the first gail_encoder_send to the last codestream
// received (the encoder's set-up before it and its tear-down after it excluded), as a
// throughput benchmark of the library times a stream.
__attribute__((visibility("default"))) int probe_encode_timed(int backend, int profile, int container, int format,
                                                              int matrix, int preset, double fps, double maxMbps,
                                                              int framesInFlight, const void* const* planes, int count,
                                                              uint8_t* out, size_t cap, uint64_t* sizes,
                                                              int* compliant, char* devices, size_t devCap,
                                                              double* seconds) {
    return encodeStream(backend, profile, container, format, matrix, preset, fps, maxMbps, framesInFlight, planes,
                        count, out, cap, sizes, compliant, devices, devCap, seconds);
}

static int encodeStream(int backend, int profile, int container, int format, int matrix, int preset, double fps,
                        double maxMbps, int framesInFlight, const void* const* planes, int count, uint8_t* out,
                        size_t cap, uint64_t* sizes, int* compliant, char* devices, size_t devCap, double* seconds) {
    const EncodeArgs a{backend, profile, container, format, matrix, preset, fps, maxMbps, framesInFlight};
    gail_config c;
    configure(a, c);
    gail_encoder* e = nullptr;
    int st = gail_encoder_create(&c, &e);
    if (st != GAIL_OK) {
        g_err = gail_last_error();
        return st;
    }
    copyOut(gail_encoder_devices(e), devices, devCap);
    int received = 0;
    const auto t0 = std::chrono::steady_clock::now();
    auto take = [&](int wait) -> int {
        gail_packet pkt;
        std::memset(&pkt, 0, sizeof pkt);
        const int r = gail_encoder_receive(e, &pkt, wait);
        if (r != GAIL_OK) return r;
        const int64_t i = pkt.index;
        if (i < 0 || i >= count || pkt.size > cap) {
            gail_packet_free(&pkt);
            g_err = "packet out of range";
            return GAIL_ERROR_FAILED;
        }
        std::memcpy(out + (size_t)i * cap, pkt.data, pkt.size);
        sizes[i] = pkt.size;
        compliant[i] = pkt.compliant;
        gail_packet_free(&pkt);
        ++received;
        return GAIL_OK;
    };
    for (int i = 0; i < count && st == GAIL_OK; ++i) {
        gail_frame f;
        std::memset(&f, 0, sizeof f);
        for (int k = 0; k < 3; ++k) f.data[k] = planes[3 * i + k];
        st = gail_encoder_send(e, &f);
        while (st == GAIL_OK) {  // collect what is ready, so send never waits on a full queue
            const int r = take(0);
            if (r == GAIL_EAGAIN) break;
            if (r != GAIL_OK) st = r;
        }
    }
    if (st == GAIL_OK) st = gail_encoder_send(e, nullptr);
    while (st == GAIL_OK && received < count) {
        const int r = take(1);
        if (r == GAIL_EOF) break;
        if (r != GAIL_OK) st = r;
    }
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st != GAIL_OK) g_err = gail_encoder_error(e) ? gail_encoder_error(e) : gail_last_error();
    else if (received != count) {
        g_err = "not every frame came back";
        st = GAIL_ERROR_FAILED;
    }
    gail_encoder_destroy(e);
    return st;
}

// One frame on a fresh encoder through gail_encoder_encode. Returns the codestream size, or
// a negative status.
__attribute__((visibility("default"))) long long probe_encode_one(int backend, int profile, int container, int format,
                                                                  int matrix, int preset, double fps, double maxMbps,
                                                                  const void* p0, const void* p1, const void* p2,
                                                                  uint8_t* out, size_t cap, int* compliant,
                                                                  char* devices, size_t devCap) {
    const EncodeArgs a{backend, profile, container, format, matrix, preset, fps, maxMbps, 0};
    gail_config c;
    configure(a, c);
    gail_encoder* e = nullptr;
    int st = gail_encoder_create(&c, &e);
    if (st != GAIL_OK) {
        g_err = gail_last_error();
        return st;
    }
    copyOut(gail_encoder_devices(e), devices, devCap);
    gail_frame f;
    std::memset(&f, 0, sizeof f);
    f.data[0] = p0;
    f.data[1] = p1;
    f.data[2] = p2;
    gail_packet pkt;
    std::memset(&pkt, 0, sizeof pkt);
    st = gail_encoder_encode(e, &f, &pkt);
    long long size = st;
    if (st == GAIL_OK) {
        if (pkt.size > cap) {
            g_err = "codestream larger than the buffer";
            size = GAIL_ERROR_FAILED;
        } else {
            std::memcpy(out, pkt.data, pkt.size);
            size = (long long)pkt.size;
            *compliant = pkt.compliant;
        }
        gail_packet_free(&pkt);
    } else {
        g_err = gail_encoder_error(e) ? gail_encoder_error(e) : gail_last_error();
    }
    gail_encoder_destroy(e);
    return size;
}

// Decodes one codestream with gail_decoder_decode into out (12-bit codes in the low bits,
// rows of stride bytes). Returns GAIL_OK or a status.
__attribute__((visibility("default"))) int probe_decode(int backend, const uint8_t* data, size_t size, int reduce,
                                                        uint16_t* out, long long stride, char* devices,
                                                        size_t devCap) {
    gail_decoder_config c;
    gail_decoder_config_defaults(&c);
    c.backend = (gail_backend)backend;
    c.output = GAIL_PIX_XYZ12;
    c.reduce = reduce;
    gail_decoder* d = nullptr;
    int st = gail_decoder_create(&c, &d);
    if (st != GAIL_OK) {
        g_err = gail_last_error();
        return st;
    }
    copyOut(gail_decoder_devices(d), devices, devCap);
    gail_packet pkt;
    std::memset(&pkt, 0, sizeof pkt);
    pkt.data = const_cast<uint8_t*>(data);
    pkt.size = size;
    gail_image img;
    std::memset(&img, 0, sizeof img);
    img.data[0] = out;
    img.stride[0] = (ptrdiff_t)stride;
    st = gail_decoder_decode(d, &pkt, &img);
    if (st != GAIL_OK) g_err = gail_decoder_error(d) ? gail_decoder_error(d) : gail_last_error();
    gail_decoder_destroy(d);
    return st;
}

}  // extern "C"
