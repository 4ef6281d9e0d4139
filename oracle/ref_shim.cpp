// Test harness: a C-ABI over the reference CPU path, compiled together with the
// reference's own sources (Josephur/libgail src/core) by oracle/Makefile into
// oracle/_ref/libgailref.so. TEST INFRASTRUCTURE ONLY: it validates the C restatement in
// oracle/gail_oracle.c, pins the golden fixtures, checks the product's host codec
// (rate control, Tier-2, DCI checker, packet parser) and serves as the reference CPU
// baseline. The product never loads it.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "core/backend.h"
#include "core/build_version.h"
#include "core/codestream_check.h"
#include "core/codestream_parse.h"
#include "core/color.h"
#include "core/decode_backend.h"
#include "core/dwt_cpu.h"
#include "core/layout.h"
#include "core/quant.h"
#include "core/rate_control.h"
#include "core/t1_dec.h"
#include "core/t1_ref.h"
#include "core/t2.h"
#include "core/t2_parse.h"
#include "core/thread_pool.h"
#include "cuda/cuda_plugin.h"

// The reference's rate control, compiled here rather than as its own object so that
// ref_hull below can call its file-local buildHull.
#include "core/rate_control.cpp"

using namespace gail;

// build_version.cpp needs a header the reference's CMake generates; a build from this
// source tree outside its own git repository is stamped with the plain release number
// (cmake/BuildVersion.cmake: "no git, or not GAIL's own repository 1.1.0").
namespace gail {
const char* buildVersion() { return "1.1.0"; }
}  // namespace gail

namespace {
thread_local std::string g_err;

FrameLayout layoutOf(int width, int height, int fourk, double baseStep) {
    return makeLayout(width, height, fourk ? Profile::Cinema4K : Profile::Cinema2K, baseStep);
}

struct RefFrame {
    FrameLayout L;
    Tier1Frame t1;
};
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// ---- Tier-1 -------------------------------------------------------------------------
struct RefT1 {
    int32_t nbps, numPasses;
    uint32_t dataLen, numSymbols;
    uint32_t passLen[64];
    int32_t passDist[64];
};

int ref_t1_encode(const uint32_t* coeffs, int w, int h, int orient, int maxPasses, float slopeThresh, float distScale,
                  uint8_t* buf, size_t cap, RefT1* out) {
    try {
        T1Result r;
        T1Trace tr;
        T1EarlyStop stop{slopeThresh, distScale};
        t1EncodeRef(coeffs, w, h, orient, r, &tr, maxPasses, &stop);
        if (r.data.size() > cap) return -2;
        std::memset(out, 0, sizeof *out);
        out->nbps = r.nbps;
        out->numPasses = r.numPasses;
        out->dataLen = (uint32_t)r.data.size();
        out->numSymbols = (uint32_t)tr.symbols.size();
        for (int k = 0; k < r.numPasses; ++k) {
            out->passLen[k] = r.passLen[k];
            out->passDist[k] = r.passDist[k];
        }
        if (!r.data.empty()) std::memcpy(buf, r.data.data(), r.data.size());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

uint32_t ref_quantize(float v, float invDelta, uint32_t maxMag) { return quantizeCoeff(v, invDelta, maxMag); }

void ref_t1_decode(const uint8_t* data, uint32_t len, int w, int h, int orient, int nbps, int passes, uint32_t* out) {
    t1DecodeBlock(data, len, w, h, orient, nbps, passes, out);
}

// The reference quantiser over a whole frame: three Mallat planes -> the code-block-major
// words of every code-block (quantizeFrame, src/core/quant.cpp:23-26).
int ref_quantize_frame(int width, int height, int fourk, double baseStep, const float* p0, const float* p1,
                       const float* p2, uint32_t* out) {
    try {
        FrameLayout L = layoutOf(width, height, fourk, baseStep);
        const float* planes[3] = {p0, p1, p2};
        quantizeFrame(L, planes, out);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// ---- wavelet ------------------------------------------------------------------------
void ref_fdwt97_2d(float* plane, int width, int height, int levels) { fdwt97_2d(plane, width, height, levels); }

void ref_idwt97_2d(float* plane, int width, int height, int levels, int skip) {
    float* p[1] = {plane};
    idwt97_2d(p, 1, width, height, levels, skip, nullptr);
}

// ---- layout -------------------------------------------------------------------------
struct RefBand {
    int32_t comp, res, level, orient, px0, py0, w, h, ncbx, ncby, cblkBase, eps, mu, mb;
    float delta;
    double weight;
};

int ref_layout_counts(int width, int height, int fourk, int* numBands, int* numCblks) {
    try {
        FrameLayout L = layoutOf(width, height, fourk, 1.0);
        *numBands = (int)L.bands.size();
        *numCblks = L.numCblks();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int ref_make_layout(int width, int height, int fourk, double baseStep, RefBand* bands, int32_t* cblks5) {
    try {
        FrameLayout L = layoutOf(width, height, fourk, baseStep);
        for (size_t i = 0; i < L.bands.size(); ++i) {
            const Subband& b = L.bands[i];
            bands[i] = {b.comp, b.res, b.level, b.orient, b.px0, b.py0, b.w, b.h, b.ncbx, b.ncby, b.cblkBase,
                        b.eps, b.mu, b.Mb, b.delta, b.weight};
        }
        for (int i = 0; i < L.numCblks(); ++i) {
            const CodeBlock& c = L.cblks[i];
            int32_t* o = cblks5 + 5 * i;
            o[0] = c.band;
            o[1] = c.x0;
            o[2] = c.y0;
            o[3] = c.w;
            o[4] = c.h;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

double ref_synthesis_norm(int level, int orient) { return synthesisNorm(level, orient); }

// ---- colour -------------------------------------------------------------------------
static ColorParams colorParams(int transfer, int primaries, double sdrWhite) {
    ColorParams c;
    c.transfer = (Transfer)transfer;
    c.primaries = (Primaries)primaries;
    c.sdrWhite = sdrWhite;
    return c;
}

int ref_color_tables(int transfer, int primaries, double sdrWhite, float* eotf65536, float* params48) {
    try {
        ColorConverter cc(colorParams(transfer, primaries, sdrWhite));
        std::memcpy(eotf65536, cc.lut().data(), 65536 * 4);
        std::memcpy(params48, cc.params().data(), cc.params().size() * 4);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void ref_color_frame(int transfer, int primaries, double sdrWhite, const uint16_t* rgb, int npix, float* p0, float* p1,
                     float* p2, uint16_t* xyz12) {
    ColorConverter cc(colorParams(transfer, primaries, sdrWhite));
    float* planes[3] = {p0, p1, p2};
    cc.convertFrame(rgb, npix, 1, planes, xyz12);
}

// Every colour setting (ColorParams, core/color.h:84-100; the enums' numbering): tone
// map, norm, target gamut, a 3D LUT in memory or by .cube path.
struct RefColor {
    int32_t transfer, primaries, toneMap, toneNorm, gamut, lutSize;
    double sdrWhite, hdrPeak, cinemaPeak, hdrRefWhite, cinemaRefWhite, knee, gamutThreshold;
    const float* lutData;
    uint64_t lutCount;
    const char* lutPath;
};

static ColorParams colorOf(const RefColor& r) {
    ColorParams c;
    c.transfer = (Transfer)r.transfer;
    c.primaries = (Primaries)r.primaries;
    c.toneMap = (ToneMap)r.toneMap;
    c.toneNorm = (ToneNorm)r.toneNorm;
    c.gamut = (TargetGamut)r.gamut;
    c.sdrWhite = r.sdrWhite;
    c.hdrPeak = r.hdrPeak;
    c.cinemaPeak = r.cinemaPeak;
    c.hdrRefWhite = r.hdrRefWhite;
    c.cinemaRefWhite = r.cinemaRefWhite;
    c.knee = r.knee;
    c.gamutThreshold = r.gamutThreshold;
    if (r.lutData && r.lutCount) c.lut3dData.assign(r.lutData, r.lutData + r.lutCount);
    c.lut3dSize = r.lutSize;
    c.lut3d = r.lutPath ? r.lutPath : "";
    return c;
}

// The converter's parameter block (CP_COUNT floats, kernels/color_params.h) and its LUT size.
int ref_color_params(const RefColor* c, float* params48, int* lutN) {
    try {
        ColorConverter cc(colorOf(*c));
        std::memcpy(params48, cc.params().data(), cc.params().size() * 4);
        *lutN = cc.lut3dSize();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int ref_color_frame_full(const RefColor* c, const uint16_t* rgb, int npix, float* p0, float* p1, float* p2,
                         uint16_t* xyz12) {
    try {
        ColorConverter cc(colorOf(*c));
        float* planes[3] = {p0, p1, p2};
        cc.convertFrame(rgb, npix, 1, planes, xyz12);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// readCubeLut (core/color.cpp:245-282): the LUT's size and up to cap floats of it.
int ref_read_cube(const char* path, int* n, float* out, uint64_t cap) {
    try {
        int size = 0;
        const std::vector<float> v = readCubeLut(path, size);
        *n = size;
        std::memcpy(out, v.data(), std::min<uint64_t>(cap, v.size()) * 4);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

struct RefPlanar {
    int32_t width, height, activeW, activeH, ox, oy, sx, sy, rgb, bits, fullRange, chroma;
    double kr, kb;
};

static FrameFormat formatOf(const RefPlanar& p) {
    FrameFormat f;
    f.kind = FrameFormat::Kind::Planar;
    f.chroma = (FrameFormat::Chroma)p.chroma;
    f.width = p.width;
    f.height = p.height;
    f.activeW = p.activeW;
    f.activeH = p.activeH;
    f.ox = p.ox;
    f.oy = p.oy;
    f.sx = p.sx;
    f.sy = p.sy;
    f.rgb = p.rgb != 0;
    f.bits = p.bits;
    f.fullRange = p.fullRange != 0;
    f.kr = p.kr;
    f.kb = p.kb;
    return f;
}

void ref_planar_to_rgb48(const RefPlanar* p, const void* src, uint16_t* rgb) { planarToRgb48(formatOf(*p), src, rgb); }

// ---- whole-frame CPU encoder (CpuSlot) ----------------------------------------------
// input: RGB48 interleaved (planar == NULL) or a planar frame described by planar.
struct EncView {
    FrameLayout L;
    std::unique_ptr<Device> dev;
    std::unique_ptr<EncoderSlot> slot;
    Tier1Frame t1;
    FrameDebug dbg;
};

static void* encoderCreate(int width, int height, int fourk, double baseStep, const ColorParams& color,
                           const RefPlanar* planar, int threads);

void* ref_encoder_create(int width, int height, int fourk, double baseStep, int transfer, int primaries, double sdrWhite,
                         const RefPlanar* planar, int threads) {
    return encoderCreate(width, height, fourk, baseStep, colorParams(transfer, primaries, sdrWhite), planar, threads);
}

void* ref_encoder_create_color(int width, int height, int fourk, double baseStep, const RefColor* color,
                               const RefPlanar* planar, int threads) {
    try {
        return encoderCreate(width, height, fourk, baseStep, colorOf(*color), planar, threads);
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return nullptr;
    }
}

static void* encoderCreate(int width, int height, int fourk, double baseStep, const ColorParams& color,
                           const RefPlanar* planar, int threads) {
    try {
        auto e = std::make_unique<EncView>();
        e->L = layoutOf(width, height, fourk, baseStep);
        EncodeSettings s;
        s.profile = fourk ? Profile::Cinema4K : Profile::Cinema2K;
        s.width = width;
        s.height = height;
        s.baseStep = baseStep;
        s.color = color;
        if (planar) {
            s.input = formatOf(*planar);
        } else {
            s.input.kind = FrameFormat::Kind::RGB48;
            s.input.width = width;
            s.input.height = height;
        }
        e->dev = createCpuDevice(threads);
        e->slot = e->dev->createSlot(e->L, s);
        return e.release();
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return nullptr;
    }
}

struct RefEncOut {
    const CblkInfo* info;
    const uint32_t* passLen;
    const int32_t* passDist;
    const uint8_t* data;
    uint64_t numInfo, numPasses, numData;
    const uint16_t* xyz12;
    const uint32_t* coeffs;
    double ms;
};

int ref_encoder_encode(void* h, const void* frame, double slopeThresh, int debug, RefEncOut* out) {
    try {
        auto* e = static_cast<EncView*>(h);
        e->slot->setSlopeThreshold(slopeThresh);
        FrameTimings tm;
        const auto t0 = std::chrono::steady_clock::now();
        e->slot->encode(frame, e->t1, &tm, debug ? &e->dbg : nullptr);
        const auto t1 = std::chrono::steady_clock::now();
        out->info = e->t1.info.data();
        out->passLen = e->t1.passLen.data();
        out->passDist = e->t1.passDist.data();
        out->data = e->t1.data.data();
        out->numInfo = e->t1.info.size();
        out->numPasses = e->t1.passLen.size();
        out->numData = e->t1.data.size();
        out->xyz12 = debug ? e->dbg.xyz12.data() : nullptr;
        out->coeffs = debug ? e->dbg.coeffs.data() : nullptr;
        out->ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

void ref_encoder_destroy(void* h) { delete static_cast<EncView*>(h); }

// ---- rate control, Tier-2, checker --------------------------------------------------
// A Tier-1 frame given as plain arrays (CblkInfo = 5 words per block).
static Tier1Frame tier1Of(const uint32_t* info5, uint64_t n, const uint32_t* passLen, const int32_t* passDist,
                          uint64_t numPasses, const uint8_t* data, uint64_t numData) {
    Tier1Frame t;
    t.info.resize(n);
    std::memcpy(t.info.data(), info5, n * sizeof(CblkInfo));
    t.passLen.assign(passLen, passLen + numPasses);
    t.passDist.assign(passDist, passDist + numPasses);
    t.data.assign(data, data + numData);
    return t;
}

// Runs allocateRate and buildCodestream. passesOut: one byte per block. csOut receives up
// to csCap bytes; returns the codestream size, or -1.
long long ref_rate_and_build(int width, int height, int fourk, double baseStep, const uint32_t* info5, uint64_t n,
                             const uint32_t* passLen, const int32_t* passDist, uint64_t numPasses, const uint8_t* data,
                             uint64_t numData, double fps, double maxMbps, const char* tag, uint8_t* passesOut,
                             uint8_t* csOut, uint64_t csCap, double* lambdaOut, double* msOut) {
    try {
        FrameLayout L = layoutOf(width, height, fourk, baseStep);
        Tier1Frame t = tier1Of(info5, n, passLen, passDist, numPasses, data, numData);
        const auto t0 = std::chrono::steady_clock::now();
        RateResult rr = allocateRate(L, t, dciLimits(fps, maxMbps));
        std::vector<uint8_t> cs;
        buildCodestream(L, t, rr.passes.data(), &cs, nullptr, tag ? std::string(tag) : std::string());
        const auto t1 = std::chrono::steady_clock::now();
        if (msOut) *msOut = std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (lambdaOut) *lambdaOut = rr.lambda;
        std::memcpy(passesOut, rr.passes.data(), rr.passes.size());
        if (cs.size() > csCap) return -1;
        std::memcpy(csOut, cs.data(), cs.size());
        return (long long)cs.size();
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// The reference's PCRD hull points (buildHull), laid out per pass slot of the Tier-1 frame:
// block i's points from its passBase on, the entries after them passes 0, slope 0.
// Returns 0, or -1.
int ref_hull(int width, int height, int fourk, double baseStep, const uint32_t* info5, uint64_t n,
             const uint32_t* passLen, const int32_t* passDist, uint64_t numPasses, uint8_t* passesOut,
             double* slopeOut) {
    try {
        FrameLayout L = layoutOf(width, height, fourk, baseStep);
        Tier1Frame t = tier1Of(info5, n, passLen, passDist, numPasses, nullptr, 0);
        const Hull H = buildHull(L, t);
        std::memset(passesOut, 0, numPasses);
        std::memset(slopeOut, 0, numPasses * sizeof(double));
        for (uint64_t i = 0; i < n; ++i) {
            const uint32_t base = t.info[i].passBase;
            for (uint32_t h = H.start[i]; h < H.start[i + 1]; ++h) {
                passesOut[base + h - H.start[i]] = H.passes[h];
                slopeOut[base + h - H.start[i]] = H.slope[h];
            }
        }
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// buildCodestream with given passes. Returns the size.
long long ref_build(int width, int height, int fourk, double baseStep, const uint32_t* info5, uint64_t n,
                    const uint32_t* passLen, const int32_t* passDist, uint64_t numPasses, const uint8_t* data,
                    uint64_t numData, const uint8_t* passes, const char* tag, uint8_t* csOut, uint64_t csCap) {
    try {
        FrameLayout L = layoutOf(width, height, fourk, baseStep);
        Tier1Frame t = tier1Of(info5, n, passLen, passDist, numPasses, data, numData);
        std::vector<uint8_t> cs;
        buildCodestream(L, t, passes, &cs, nullptr, tag ? std::string(tag) : std::string());
        if (cs.size() > csCap) return -1;
        std::memcpy(csOut, cs.data(), cs.size());
        return (long long)cs.size();
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

long long ref_empty_codestream_bytes(int width, int height, int fourk) {
    return (long long)emptyCodestreamBytes(layoutOf(width, height, fourk, 1.0));
}

void ref_dci_limits(double fps, double maxMbps, double compMbps, uint64_t* total, uint64_t* comp) {
    RateLimits l = dciLimits(fps, maxMbps, compMbps);
    *total = l.maxTotal;
    *comp = l.maxComp;
}

// Returns 1 when compliant, 0 when not (first error in msg), writes the COM text.
int ref_check_dci(const uint8_t* data, uint64_t size, double fps, char* msg, uint64_t msgCap) {
    CheckReport r = checkDciCodestream(data, size, fps);
    std::string m = r.ok ? r.comment : (r.errors.empty() ? std::string("?") : r.errors[0]);
    if (msg && msgCap) std::snprintf(msg, msgCap, "%s", m.c_str());
    return r.ok ? 1 : 0;
}

// ---- decoding -----------------------------------------------------------------------
// parseCodestream + parsePackets; blocks8: per block {offset, len, passes, nbps} as
// uint32 offset, uint32 len, uint8 passes, uint8 nbps (the CblkCode layout).
int ref_parse(const uint8_t* data, uint64_t size, int reduce, void* blocksOut, uint64_t maxBlocks, int* numBlocks,
              int* width, int* height, int* levels) {
    try {
        StreamHeader h;
        std::string err;
        if (!parseCodestream(data, size, false, h, err)) {
            g_err = err;
            return -1;
        }
        FrameLayout L = layoutFor(h);
        std::vector<CblkCode> blocks;
        if (!parsePackets(data, h, L, L.levels - reduce, blocks, err)) {
            g_err = err;
            return -1;
        }
        *numBlocks = (int)blocks.size();
        *width = L.width;
        *height = L.height;
        *levels = L.levels;
        if (blocks.size() > maxBlocks) return -2;
        std::memcpy(blocksOut, blocks.data(), blocks.size() * sizeof(CblkCode));
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// Full CPU decode of a codestream into dst (interleaved 16-bit, rows strideBytes apart).
// wavelet: optional 3 * width * height floats receiving the dequantised planes.
int ref_decode(const uint8_t* data, uint64_t size, int reduce, int highBits, int threads, void* dst, long long strideBytes,
               float* wavelet, double* msOut) {
    try {
        StreamHeader h;
        std::string err;
        if (!parseCodestream(data, size, false, h, err)) {
            g_err = err;
            return -1;
        }
        const auto t0 = std::chrono::steady_clock::now();
        FrameLayout L = layoutFor(h);
        std::vector<CblkCode> blocks;
        if (!parsePackets(data, h, L, L.levels - reduce, blocks, err)) {
            g_err = err;
            return -1;
        }
        auto pool = std::make_shared<ThreadPool>(threads > 0 ? threads : usableCpuCount(), false);
        DecodeSettings s;
        s.reduce = reduce;
        s.highBits = highBits != 0;
        auto slot = createCpuDecoderSlot(L, s, pool);
        std::vector<float> wv[3];
        DecodeTimings tm;
        if (wavelet) tm.wavelet = wv;
        slot->decode(L, data, size, blocks, dst, (ptrdiff_t)strideBytes, &tm);
        const auto t1 = std::chrono::steady_clock::now();
        if (msOut) *msOut = std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (wavelet) {
            const size_t npix = (size_t)L.width * L.height;
            for (int c = 0; c < 3; ++c) std::memcpy(wavelet + c * npix, wv[c].data(), npix * 4);
        }
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// ---- the reference tests' random code-block suites -----------------------------------
// suite 0: the blocks of testT1Truncation / testT1Decode (tests/test_main.cpp:340-357,
// std::mt19937 seed 42, 400 trials); suite 1: testT1PassLimit (:652-663, seed 9, 300
// trials, with the pass limit each trial codes). Same generator calls in the same order,
// so the blocks are the reference's own. meta: w, h, orient, pass limit (64 = none).
int ref_suite_blocks(int suite, int ntrials, uint32_t* coeffs, int32_t* meta) {
    if (suite == 0) {
        std::mt19937 rng(42);
        for (int trial = 0; trial < ntrials; ++trial) {
            const int w = trial % 7 == 0 ? 1 + rng() % 32 : 32;
            const int h = trial % 5 == 0 ? 1 + rng() % 32 : 32;
            uint32_t* c = coeffs + (size_t)trial * kCblkArea;
            std::fill(c, c + kCblkArea, 0u);
            const int mode = trial % 3;
            std::normal_distribution<double> g(0, mode == 0 ? 20 : (mode == 1 ? 300 : 3000));
            std::uniform_real_distribution<double> sp(0, 1);
            for (int y = 0; y < h; ++y)
                for (int x = 0; x < w; ++x) {
                    double v = g(rng);
                    if (mode == 1 && sp(rng) < 0.7) v *= 0.05;
                    c[y * 32 + x] = quantizeCoeff((float)v, 1.0f, (1u << 26) - 1);
                }
            meta[4 * trial] = w;
            meta[4 * trial + 1] = h;
            meta[4 * trial + 2] = trial % 4;
            meta[4 * trial + 3] = kMaxPasses;
        }
        return 0;
    }
    if (suite == 1) {
        std::mt19937 rng(9);
        for (int trial = 0; trial < ntrials; ++trial) {
            const int w = 32, h = trial % 3 == 0 ? 17 : 32, orient = trial % 4;
            uint32_t* c = coeffs + (size_t)trial * kCblkArea;
            std::fill(c, c + kCblkArea, 0u);
            std::normal_distribution<double> g(0, 500);
            for (int y = 0; y < h; ++y)
                for (int x = 0; x < w; ++x) c[y * 32 + x] = quantizeCoeff((float)g(rng), 1.0f, (1u << 26) - 1);
            T1Result full;
            t1EncodeRef(c, w, h, orient, full);
            meta[4 * trial] = w;
            meta[4 * trial + 1] = h;
            meta[4 * trial + 2] = orient;
            meta[4 * trial + 3] = 1 + trial % std::max(1, full.numPasses - 1);
        }
        return 0;
    }
    return -1;
}

// ---- plugin ABI facts ---------------------------------------------------------------
uint64_t ref_plugin_layout_hash() { return cudaPluginLayout(); }

void ref_plugin_sizes(uint64_t* out12) {
    const uint64_t v[12] = {sizeof(Subband),        sizeof(CblkInfo),       sizeof(CblkCode),
                            sizeof(FrameFormat),    sizeof(FrameTimings),   sizeof(GailCudaDeviceDesc),
                            sizeof(GailCudaLayout), sizeof(GailCudaEncodeSettings), sizeof(GailCudaTier1),
                            sizeof(GailCudaDebug),  sizeof(GailCudaDecodeTimings), sizeof(GailCudaPlugin)};
    std::memcpy(out12, v, sizeof v);
}

int ref_usable_cpus() { return usableCpuCount(); }

}  // extern "C"
