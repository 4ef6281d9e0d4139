// Encoder front end on sm_100a: colour conversion, the 9/7 wavelet and dead-zone
// quantisation, fused level by level.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "color.h"

namespace gb {

// One subband a level writes, for one component.
struct BandOut {
    uint32_t cblkBase;  // global index of the band's first code-block
    int32_t ncbx, ncby;
    int32_t w, h;       // band size
    int32_t px0, py0;   // position in the Mallat plane (for the float tap)
    float invDelta;     // 1 / step (the reference's float division)
    uint32_t maxMag;    // ((1 << Mb) << 6) - 1
};

struct LevelArgs {
    int32_t w, h;            // the level's input region
    const float* src;        // previous level's LL planes (level > 1)
    int32_t srcStride;
    uint64_t srcComp;        // floats between components
    float* ll;               // this level's LL output for the next level (NULL at the last)
    int32_t llStride;
    uint64_t llComp;
    uint32_t* coeffs;        // code-block-major quantised words
    BandOut band[3][4];      // [component][orient], orient 0 = LL
    int32_t last;            // the last level: LL is quantised too
    float* tap;              // Mallat float planes (debug), or NULL
    int32_t tapStride;
    uint64_t tapComp;
};

struct ColorArgs {
    int32_t kind;            // 0 interleaved R'G'B' 16-bit, 1 planar
    const void* src;         // the frame in device memory
    PlanarParams pp;
    const float* eotf;       // 65536 entries
    const float* thr;        // 4096 thresholds
    float m[9];
    uint16_t* xyz;           // debug tap: interleaved 12-bit codes, or NULL
    int32_t route;           // ColorRoute
    ToneParams tone;         // route 1
    const float* lut3;       // route 2: lutN^3 nodes of three floats, red fastest
    int32_t lutN;
};

// Level 1 with the colour conversion folded into its tile loads; shape: the tile, 0 = 64 x
// 64, 1 = 128 x 64, 2 = 64 x 128 (the tone-map and LUT routes always take 64 x 64).
void launchLevel1(const ColorArgs& c, const LevelArgs& a, int shape, cudaStream_t st);
// Levels 2.. from the previous level's LL planes, with tile shape `shape`.
void launchLevel(const LevelArgs& a, int shape, cudaStream_t st);
// Per-device set-up (shared-memory opt-in).
void frontendInit();

}  // namespace gb
