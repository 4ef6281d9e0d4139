// Packing of Tier-1 results into the Tier1Frame layout.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "t1_encode.cuh"

namespace gb {

struct CompactArgs {
    uint32_t n;
    const uint32_t* info;      // 4 words per block (nbps, passes, decisions, bytes)
    const uint32_t* passLen;   // 64 per block
    const int32_t* passDist;   // 64 per block
    const T1Job* jobs;         // each block's codeword region
    uint32_t* outInfo;         // 5 words per block: CblkInfo
    uint32_t* outPassLen;
    int32_t* outPassDist;      // may be null: no distortions
    uint8_t* outData;
    uint32_t* tot;             // [0] data bytes, [1] passes, [2] set when outData was too small
    uint64_t dataCap;          // bytes outData holds
    uint32_t* scratch;         // device, 2 words per 1024 blocks; free once MQ coding ended
                               // on this stream, so the Tier-1 launch's perm table will do
    uint2* offsets;            // device, per block: codeword byte offset, pass offset
    int hostOut;               // the out* buffers are mapped host memory: fewer copying CTAs
    // PCRD hull points (optional: none when scale is null). Per block, the points of the
    // lower convex hull of its (rate, weighted distortion reduction) curve, computed with the
    // host rate control's double arithmetic, so the host can take them in place of its own.
    const double* scale;       // device, per block: its band's step^2 x weight
    uint8_t* hullPasses;       // device, kMaxPasses per block: coding passes at each point
    double* hullSlope;         // device, kMaxPasses per block: slope from the previous point
    uint8_t* outHullPasses;    // packed at the pass offsets like outPassLen; a block's points
    double* outHullSlope;      // end at its pass count or at the first 0 in outHullPasses
};

// The out* pointers and tot may be mapped host memory: the kernels only write them, with
// whole contiguous words, and read nothing back from them.

void compactTier1(const CompactArgs& a, cudaStream_t st);

}  // namespace gb
