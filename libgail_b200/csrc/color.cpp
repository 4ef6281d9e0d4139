// Colour tables (host side): EOTF, primaries matrix, 12-bit encoding thresholds.
#include "color.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

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

ColorTables buildColorTables(const GailCudaColor& c) {
    if (c.lut3dSize > 0 || (c.lut3d && c.lut3d[0]) || c.lut3dData)
        throw std::logic_error("3D LUT colour conversion is not implemented on this backend");
    const bool hdr = c.transfer == 2 || c.transfer == 3;
    const bool passthrough = c.primaries == 4;
    if (hdr && !passthrough && (c.toneMap == 1 || c.toneMap == 2))
        throw std::logic_error("the shoulder and BT.2390 tone maps are not implemented on this backend");
    if (!passthrough && c.gamut != 2) throw std::logic_error("gamut compression is not implemented on this backend");
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
