// Colour tables (host side): EOTF, primaries matrix, 12-bit encoding thresholds, the
// managed route's tone-map and gamut constants, application 3D LUTs.
#include "color.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

namespace gb {

namespace {

constexpr double kDciNorm = 52.37;  // SMPTE ST 428-1 normalising constant

// SMPTE ST 2084 (PQ) EOTF.
double pqEotf(double e) {
    const double m1 = 2610.0 / 16384.0, m2 = 2523.0 / 4096.0 * 128.0, c1 = 3424.0 / 4096.0, c2 = 2413.0 / 4096.0 * 32.0,
                 c3 = 2392.0 / 4096.0 * 32.0;
    e = std::clamp(e, 0.0, 1.0);
    const double p = std::pow(e, 1.0 / m2);
    return 10000.0 * std::pow(std::max(p - c1, 0.0) / (c2 - c3 * p), 1.0 / m1);
}

// Its inverse: cd/m^2 -> PQ signal in [0, 1].
double pqInverseEotf(double nits) {
    const double m1 = 2610.0 / 16384.0, m2 = 2523.0 / 4096.0 * 128.0, c1 = 3424.0 / 4096.0, c2 = 2413.0 / 4096.0 * 32.0,
                 c3 = 2392.0 / 4096.0 * 32.0;
    const double y = std::pow(std::clamp(nits / 10000.0, 0.0, 1.0), m1);
    return std::pow((c1 + c2 * y) / (1.0 + c3 * y), m2);
}

// ITU-R BT.2100 HLG inverse OETF.
double hlgInverseOetf(double e) {
    const double a = 0.17883277, b = 1.0 - 4.0 * a, c = 0.5 - a * std::log(4.0 * a);
    return e <= 0.5 ? e * e / 3.0 : (std::exp((e - c) / a) + b) / 12.0;
}

void invert3(const double m[9], double r[9]) {
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    r[0] = (m[4] * m[8] - m[5] * m[7]) / det;
    r[1] = (m[2] * m[7] - m[1] * m[8]) / det;
    r[2] = (m[1] * m[5] - m[2] * m[4]) / det;
    r[3] = (m[5] * m[6] - m[3] * m[8]) / det;
    r[4] = (m[0] * m[8] - m[2] * m[6]) / det;
    r[5] = (m[2] * m[3] - m[0] * m[5]) / det;
    r[6] = (m[3] * m[7] - m[4] * m[6]) / det;
    r[7] = (m[1] * m[6] - m[0] * m[7]) / det;
    r[8] = (m[0] * m[4] - m[1] * m[3]) / det;
}

// Linear RGB (white Y = 1) -> CIE XYZ from chromaticities: BT.709, BT.2020, P3-D65, DCI-P3.
void rgbToXyz(int primaries, double M[9]) {
    static const double xy[4][4][2] = {
        {{0.640, 0.330}, {0.300, 0.600}, {0.150, 0.060}, {0.3127, 0.3290}},
        {{0.708, 0.292}, {0.170, 0.797}, {0.131, 0.046}, {0.3127, 0.3290}},
        {{0.680, 0.320}, {0.265, 0.690}, {0.150, 0.060}, {0.3127, 0.3290}},
        {{0.680, 0.320}, {0.265, 0.690}, {0.150, 0.060}, {0.314, 0.351}},
    };
    if (primaries == 4) {
        for (int i = 0; i < 9; ++i) M[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    if (primaries < 0 || primaries > 4) throw std::logic_error("unknown primaries");
    const double(*c)[2] = xy[primaries];
    double P[9], Pi[9], S[3];
    for (int i = 0; i < 3; ++i) {
        P[0 + i] = c[i][0] / c[i][1];
        P[3 + i] = 1.0;
        P[6 + i] = (1.0 - c[i][0] - c[i][1]) / c[i][1];
    }
    const double W[3] = {c[3][0] / c[3][1], 1.0, (1.0 - c[3][0] - c[3][1]) / c[3][1]};
    invert3(P, Pi);
    for (int i = 0; i < 3; ++i) S[i] = Pi[3 * i] * W[0] + Pi[3 * i + 1] * W[1] + Pi[3 * i + 2] * W[2];
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) M[3 * r + k] = P[3 * r + k] * S[k];
}

}  // namespace

int dciCode(float n) { return (int)std::floor(4095.0f * std::pow(n, 1.0f / 2.6f) + 0.5f); }

namespace {

// Parses up to `want` numbers from the start of s (spaces between, anything after the last
// ignored); returns how many it read.
int leadingFloats(const char* s, float* out, int want) {
    int got = 0;
    while (got < want) {
        while (*s == ' ' || *s == '\t') ++s;
        if (!(std::isdigit((unsigned char)*s) || *s == '-' || *s == '+' || *s == '.')) break;
        char* end = nullptr;
        const float v = std::strtof(s, &end);
        if (end == s) break;
        out[got++] = v;
        s = end;
    }
    return got;
}

}  // namespace

std::vector<float> readCube(const char* path, int32_t& n) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("cannot open LUT ") + path);
    std::string text;
    char buf[1 << 16];
    for (size_t got; (got = std::fread(buf, 1, sizeof buf, f)) > 0;) text.append(buf, got);
    std::fclose(f);
    std::vector<float> nodes;
    n = 0;
    size_t at = 0;
    while (at < text.size()) {
        size_t eol = text.find('\n', at);
        if (eol == std::string::npos) eol = text.size();
        const std::string line = text.substr(at, eol - at);
        at = eol + 1;
        if (line.empty() || line[0] == '#') continue;
        const size_t k0 = line.find_first_not_of(" \t\r");
        if (k0 == std::string::npos) continue;
        const size_t k1 = std::min(line.find_first_of(" \t\r", k0), line.size());
        const std::string key = line.substr(k0, k1 - k0);
        const char* rest = line.c_str() + k1;
        if (key == "LUT_3D_SIZE") {
            n = (int32_t)std::strtol(rest, nullptr, 10);
        } else if (key == "LUT_1D_SIZE") {
            throw std::runtime_error(std::string("1D .cube LUTs are not supported: ") + path);
        } else if (key == "DOMAIN_MIN" || key == "DOMAIN_MAX") {
            float d[3];
            const float want = key == "DOMAIN_MIN" ? 0.f : 1.f;
            if (leadingFloats(rest, d, 3) != 3 || d[0] != want || d[1] != want || d[2] != want)
                throw std::runtime_error(std::string("LUT domain must be 0..1: ") + path);
        } else if (key != "TITLE") {
            float v[3];
            if (leadingFloats(line.c_str(), v, 3) == 3) nodes.insert(nodes.end(), v, v + 3);
        }
    }
    if (n < 2 || nodes.size() != (size_t)n * n * n * 3)
        throw std::runtime_error(std::string("malformed 3D LUT (size / entry count) in ") + path);
    return nodes;
}

ColorTables buildColorTables(const GailCudaColor& c) {
    const bool hdr = c.transfer == 2 || c.transfer == 3;
    const bool passthrough = c.primaries == 4;
    ColorTables t;
    t.eotf.resize(65536);
    for (int i = 0; i < 65536; ++i) {
        const double e = i / 65535.0;
        double nits = 0;
        switch (c.transfer) {
        case 0: nits = std::pow(e, 2.4) * c.sdrWhite; break;
        case 1: nits = (e <= 0.04045 ? e / 12.92 : std::pow((e + 0.055) / 1.055, 2.4)) * c.sdrWhite; break;
        case 4: nits = e * c.sdrWhite; break;
        case 5: nits = std::pow(e, 2.6) * kDciNorm; break;
        case 2: nits = c.toneMap == 0 ? std::pow(e, 2.4) * c.sdrWhite : pqEotf(e); break;
        case 3: nits = c.toneMap == 0 ? std::pow(e, 2.4) * c.sdrWhite : 1000.0 * std::pow(hlgInverseOetf(e), 1.2); break;
        default: throw std::logic_error("unknown transfer function");
        }
        t.eotf[i] = (float)nits;
    }
    double M[9];
    rgbToXyz(c.primaries, M);
    for (int i = 0; i < 9; ++i) t.m[i] = (float)M[i];
    // the managed route's constants (ColorConverter's parameter block, core/color.cpp:344-388)
    ToneParams& tp = t.tone;
    tp.peak = (float)c.cinemaPeak;
    if (hdr && !passthrough && c.toneMap == 1) {
        const double gain = c.cinemaRefWhite / c.cinemaPeak;
        const double vmax = gain * c.hdrPeak / c.hdrRefWhite;  // the source peak on the output scale
        const double knee = vmax <= 1.0 ? 1.0 : std::clamp(c.knee, 0.05, 0.99);
        tp.tone = 1;
        tp.srcRef = (float)c.hdrRefWhite;
        tp.gain = (float)gain;
        tp.knee = (float)knee;
        tp.shoulderT = (float)std::max(1e-3, (vmax - knee) / (1.0 - knee));
    } else if (hdr && !passthrough && c.toneMap == 2 && c.hdrPeak > c.cinemaPeak) {
        tp.tone = 2;
        tp.pqSrcMax = (float)pqInverseEotf(c.hdrPeak);
        tp.pqMaxLum = (float)(pqInverseEotf(c.cinemaPeak) / pqInverseEotf(c.hdrPeak));
        tp.pqKs = std::max(0.f, 1.5f * tp.pqMaxLum - 0.5f);
    }
    tp.norm = c.toneNorm == 0 ? 2 : c.toneNorm == 1 ? 1 : 0;
    if (!passthrough) {
        double T[9], Ti[9];
        rgbToXyz(c.gamut == 1 ? 3 : 2, T);  // DCI-P3 or P3-D65 projector primaries
        invert3(T, Ti);
        for (int i = 0; i < 9; ++i) {
            tp.toTarget[i] = (float)(Ti[i] / c.cinemaPeak);
            tp.fromTarget[i] = (float)(T[i] * c.cinemaPeak);
        }
        if (c.gamut != 2) {
            tp.gamut = 1;
            tp.gamutThresh = (float)std::clamp(c.gamutThreshold, 0.0, 0.99);
        }
    }
    if (tp.tone != 0 || tp.gamut != 0) t.route = kRouteManaged;
    // an application LUT replaces everything above: in memory, else from a .cube file
    if (c.lut3dData && c.lut3dCount > 0) {
        if (c.lut3dSize < 2 || c.lut3dCount != (uint64_t)c.lut3dSize * c.lut3dSize * c.lut3dSize * 3)
            throw std::runtime_error("3D LUT data does not match its size");
        t.lut3.assign(c.lut3dData, c.lut3dData + c.lut3dCount);
        t.lutN = c.lut3dSize;
    } else if (c.lut3d && c.lut3d[0]) {
        t.lut3 = readCube(c.lut3d, t.lutN);
    }
    if (t.lutN > 1) t.route = kRouteLut;
    // thresholds by bisection on the float bit patterns of [0, 1] (the code is
    // non-decreasing in n; the tests check every threshold against its neighbours)
    t.thr.assign(4096, 0.f);
    for (int k = 1; k < 4096; ++k) {
        uint32_t lo = 0, hi = 0x3F800000u;  // code(1.0) = 4095 >= k
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            float f;
            std::memcpy(&f, &mid, 4);
            if (dciCode(f) >= k) hi = mid;
            else lo = mid + 1;
        }
        std::memcpy(&t.thr[k], &lo, 4);
    }
    return t;
}

PlanarParams planarParams(const GbFrameFormat& f) {
    PlanarParams p{};
    p.width = f.width;
    p.height = f.height;
    p.aw = f.activeW;
    p.ah = f.activeH;
    p.ox = f.ox;
    p.oy = f.oy;
    p.sx = f.sx;
    p.sy = f.sy;
    p.cw = (f.activeW + f.sx) >> f.sx;
    p.ch = (f.activeH + f.sy) >> f.sy;
    p.bits = f.bits;
    p.fullRange = f.fullRange ? 1 : 0;
    p.rgb = f.rgb ? 1 : 0;
    p.chroma = f.chroma;
    p.maxv = (float)((1 << f.bits) - 1);
    p.scale = (float)(1 << (f.bits - 8));
    const double kg = 1.0 - f.kr - f.kb;
    p.crR = (float)(2 * (1 - f.kr));
    p.cbB = (float)(2 * (1 - f.kb));
    p.cbG = (float)(2 * f.kb * (1 - f.kb) / kg);
    p.crG = (float)(2 * f.kr * (1 - f.kr) / kg);
    return p;
}

uint64_t frameBytes(const GbFrameFormat& f) {
    if (f.kind == GB_FRAME_RGB48) return (uint64_t)f.width * f.height * 6;
    const uint64_t bps = f.bits > 8 ? 2 : 1;
    const uint64_t cw = (uint64_t)((f.activeW + f.sx) >> f.sx), ch = (uint64_t)((f.activeH + f.sy) >> f.sy);
    return ((uint64_t)f.activeW * f.activeH + 2 * cw * ch) * bps;
}

}  // namespace gb
