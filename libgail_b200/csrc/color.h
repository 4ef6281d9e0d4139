// Colour tables for the encoder front end: source R'G'B' code values to 12-bit DCI
// X'Y'Z' (SMPTE ST 428-1). Built on the host in the reference's arithmetic
// (Josephur/libgail core/color.cpp:296-372, kernels/color_math.h:109-179) so that the
// device path, which only looks them up, gives the reference's codes.
#pragma once
#include <cstdint>
#include <vector>

#include "gail_cuda_plugin_abi.h"

namespace gb {

// How a pixel's R'G'B' becomes X'Y'Z' codes.
enum ColorRoute : int32_t {
    kRouteDirect = 0,   // EOTF, 3x3 to XYZ, 12-bit encoding
    kRouteManaged = 1,  // the same with a tone map and / or gamut compression between
    kRouteLut = 2,      // an application 3D LUT straight to X'Y'Z'
};

// The managed route's constants, as floats rounded from the host's doubles the way the
// reference's parameter block is (core/color.cpp:344-388).
struct ToneParams {
    int32_t tone;       // 0 none, 1 shoulder (scene-relative), 2 BT.2390 EETF (absolute, PQ domain)
    int32_t norm;       // what the curve is applied to: 0 luminance, 1 max(R,G,B), 2 each target channel
    int32_t gamut;      // 1: compress into the target gamut
    float peak;         // target peak white, cd/m^2
    float srcRef, gain, knee, shoulderT;  // shoulder
    float pqSrcMax, pqMaxLum, pqKs;       // BT.2390
    float gamutThresh;
    float toTarget[9];  // XYZ (cd/m^2) -> target RGB, 1 = peak white
    float fromTarget[9];
};

struct ColorTables {
    std::vector<float> eotf;  // 65536 entries: 16-bit code -> cd/m^2
    float m[9];               // linear RGB -> XYZ, row-major
    // thresholds of the 12-bit encoding X' = floor(4095 (X / 52.37)^(1/2.6) + 0.5):
    // thr[k] is the smallest n = X / 52.37 in [0, 1] whose code is at least k (thr[0] = 0)
    std::vector<float> thr;
    int32_t route = kRouteDirect;
    ToneParams tone{};
    std::vector<float> lut3;  // route 2: lutN^3 nodes of three floats, red fastest
    int32_t lutN = 0;
};

// Builds the tables of a colour setting (a 3D LUT given by path is read here). Throws
// std::runtime_error for a LUT that cannot be read or does not match its size.
ColorTables buildColorTables(const GailCudaColor& c);

// Reads a .cube 3D LUT: LUT_3D_SIZE n and n^3 lines "r g b" (red fastest); comment lines,
// TITLE and a 0..1 DOMAIN_MIN / DOMAIN_MAX are accepted; a 1D LUT, another domain or a
// wrong entry count throw std::runtime_error.
std::vector<float> readCube(const char* path, int32_t& n);

// The 12-bit code of a normalised value n in [0, 1] by the host's own arithmetic (used to
// build and to check the thresholds).
int dciCode(float n);

// Planar input parameters as the device kernel takes them (FrameFormat::matrix and
// planarRowImpl constants, core/color.h:64-72, core/color.cpp:145-150).
struct PlanarParams {
    int32_t width, height, aw, ah, ox, oy, cw, ch, sx, sy, bits, fullRange, rgb, chroma;
    float maxv, scale, crR, cbG, crG, cbB;
};
PlanarParams planarParams(const GbFrameFormat& f);
// Bytes of one input frame of this format (FrameFormat::bytes, core/color.h:56-60).
uint64_t frameBytes(const GbFrameFormat& f);

}  // namespace gb
