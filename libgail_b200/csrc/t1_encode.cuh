// EBCOT Tier-1 encoder on sm_100a: context modelling, MQ coding, exact truncation
// lengths and per-pass distortions, bit-exact with the reference CPU coder
// (Josephur/libgail core/t1_ref.cpp). Host-side view of the device work.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace gb {

// One code-block to code, wherever its frame's buffers are: a launch can take the blocks of
// any number of frames. 48 bytes, read once per block by each kernel.
struct T1Job {
    const uint32_t* coeffs;  // its 1024 sign-magnitude words (32 x 32, zero outside w x h)
    uint8_t* sym;            // its decision region (16-aligned)
    uint8_t* cw;             // its codeword region (16-aligned)
    uint32_t cap;            // bytes in either region
    uint32_t geom;           // (w-1) | (h-1) << 5 | orient << 10 | maxPasses << 12
    float dscale;            // band delta^2 * weight: distortion units of the early-termination rule
    uint32_t slope;          // index of its frame's early-termination threshold
    uint32_t pad[2];
};

inline uint32_t t1Geom(int w, int h, int orient, int maxPasses) {
    return (uint32_t)(w - 1) | ((uint32_t)(h - 1) << 5) | ((uint32_t)orient << 10) | ((uint32_t)maxPasses << 12);
}

// Worst-case MQ decisions of a block: each sample is coded once per bit-plane with at most
// a significance and a sign decision, plus run-length decisions (3 per stripe column of 4
// samples, which then skip one significance decision): 2.5 per sample and plane.
inline uint32_t t1SymbolBound(int w, int h, int planes) {
    const uint32_t perPlane = (uint32_t)((5 * w * h + 1) / 2);
    return ((perPlane * (uint32_t)planes + 64u) + 15u) & ~15u;
}

// Device pointers of one Tier-1 launch (any number of frames: the jobs say where). The
// per-job tables are indexed by the job's position in `jobs`.
struct T1Launch {
    const T1Job* jobs;
    uint32_t n;
    uint32_t* info;      // 4 words per job: nbps, passes, symbols, codeword bytes
    uint32_t* passEnd;   // 64 per job: decisions coded by the end of each pass
    uint32_t* passLen;   // 64 per job: truncation length after each pass
    int32_t* passDist;   // 64 per job: distortion reduction of each pass (x4096, plane units)
    uint4* snaps;        // 64 per job: MQ state at the end of each pass
    uint32_t* perm;      // n: jobs in MQ order (most decisions first)
    uint32_t* ctl;       // [0] MQ queue head, [1] status bits, [2] total decisions
    const float* slope;  // early-termination thresholds, indexed by T1Job::slope (NULL: every pass)
    // launch tuning (0: the defaults): blocks of at least soloDecisions decisions are
    // MQ-coded alone in a warp (a power of two); grids of at most so many CTAs per SM
    uint32_t soloDecisions;
    uint16_t cmCtasPerSm, mqCtasPerSm;
    // one persistent launch instead of four (when work is given): work holds
    // t1WorkWords(n) words of its queues, zeroed by t1Encode
    uint16_t persistent;
    uint32_t* work;
};

// Words of a persistent launch's work area: control words and the order's buckets, then
// one list entry per block.
constexpr uint32_t kT1WorkHead = 16 + 128;
inline size_t t1WorkWords(uint32_t n) { return kT1WorkHead + (size_t)n; }

// Enqueues the whole Tier-1 stage on st: context modelling, ordering, MQ coding and
// truncation lengths, as four launches or (persistent and work set) as one.
// ctl must be zeroed by the caller (it is part of the launch so that graphs can hold it).
// marks (optional): two events recorded after context modelling and after ordering (both
// after the launch when it is one).
void t1Encode(const T1Launch& L, cudaStream_t st, cudaEvent_t* marks = nullptr);

// Uploads the context tables (once per device, before the first launch).
void t1Init();

}  // namespace gb
