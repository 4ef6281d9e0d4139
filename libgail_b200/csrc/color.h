// Colour tables for the encoder front end: source R'G'B' code values to 12-bit DCI
// X'Y'Z' (SMPTE ST 428-1). Built on the host in the reference's arithmetic
// (Josephur/libgail core/color.cpp:296-372, kernels/color_math.h:109-179) so that the
// device path, which only looks them up, gives the reference's codes.
#pragma once
#include <cstdint>
#include <vector>

#include "gail_cuda_plugin_abi.h"

namespace gb {

struct ColorTables {
    std::vector<float> eotf;  // 65536 entries: 16-bit code -> cd/m^2
    float m[9];               // linear RGB -> XYZ, row-major
    // thresholds of the 12-bit encoding X' = floor(4095 (X / 52.37)^(1/2.6) + 0.5):
    // thr[k] is the smallest n = X / 52.37 in [0, 1] whose code is at least k (thr[0] = 0)
    std::vector<float> thr;
};

// Builds the tables of a colour setting. Throws std::logic_error for the routes the
// device path does not implement (tone maps other than "signal" on HDR input, gamut
// compression, 3D LUTs).
ColorTables buildColorTables(const GailCudaColor& c);

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
