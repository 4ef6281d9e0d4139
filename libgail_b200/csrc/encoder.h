// One frame in flight on the device: the plain per-frame encode path behind the
// plugin's encoder_* entry points (the role of the reference's CudaSlot,
// Josephur/libgail src/cuda/cuda_backend.cu:778-1008): upload, front end, Tier-1,
// compaction, download.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "color.h"
#include "compact.cuh"
#include "frontend.cuh"
#include "gail_cuda_plugin_abi.h"
#include "layout.h"
#include "t1_encode.cuh"

namespace gb {

// Device memory of one slot, in allocation order (also what encoder_bytes reports).
struct SlotSizes {
    // outCap: the packed codewords' bound, 6 bytes per sample (beyond any 12-bit content;
    // a frame past it fails with a status, not an overrun)
    uint64_t npix = 0, n = 0, inBytes = 0, arena = 0, llFloats = 0, outCap = 0;
    uint64_t deviceBytes() const;
};
SlotSizes slotSizes(const Layout& L, const GbFrameFormat& in);

// Appends the Tier-1 jobs of one frame: per block its coefficient words (coeffs + 1024 i),
// its decision and codeword regions (sym / cw + offset, sized for the band's Mb
// bit-planes), geometry and slope index. Returns the arena size one frame needs; with
// NULL buffers it only counts.
uint64_t buildJobs(const Layout& L, const uint32_t* coeffs, uint8_t* sym, uint8_t* cw, uint32_t slope,
                   std::vector<T1Job>& jobs);
// The same with each block's decision and codeword regions as offsets from the start of the
// frame's arena (stored in the pointer fields), for arenas placed when the frame is coded.
uint64_t buildJobOffsets(const Layout& L, const uint32_t* coeffs, uint32_t slope, std::vector<T1Job>& jobs);

// Per block, the weight of its Tier-1 distortions in the PCRD hull: its band's
// step^2 x weight, in double (as the host rate control forms it).
std::vector<double> blockScales(const Layout& L);

// Enqueues the front end of one frame on st: colour + level 1 from c.src, then the deeper
// levels through the LL ping-pong buffers (3 x llFloats each), quantised words into coeffs
// (code-block-major), float planes into tap when not NULL.
void launchFrontEnd(const Layout& L, const ColorArgs& c, float* ll0, float* ll1, uint64_t llFloats, uint32_t* coeffs,
                    float* tap, cudaStream_t st);

class EncoderSlot {
public:
    EncoderSlot(int device, const Layout& L, const GailCudaEncodeSettings& s);
    ~EncoderSlot();
    EncoderSlot(const EncoderSlot&) = delete;
    EncoderSlot& operator=(const EncoderSlot&) = delete;

    void* inputBuffer() { return hIn_; }
    void setSlope(double t) { slope_ = (float)t; }
    // The plain path: frame (host memory) in, Tier-1 frame (this slot's pinned memory) out.
    void encode(const void* frame, GailCudaTier1* out, GbFrameTimings* tm, GailCudaDebug* dbg);

    // The same work split up for callers whose frames are already in device memory:
    // enqueue() puts the front end, Tier-1 and compaction of the frame at dFrame (device
    // memory of frameBytes(); NULL: this slot's own input buffer) on the slot's stream and
    // returns without waiting; the packed results stay on the device. finish() waits for
    // them and checks the kernels' status.
    void enqueue(const void* dFrame);
    void finish();
    cudaStream_t stream() const { return st_; }
    uint64_t inputBytes() const { return z_.inBytes; }

    // Stage timing of enqueue(): when on, every enqueue records CUDA events between its
    // stages (front end, context modelling, ordering, MQ, packing) on the slot's stream.
    // stageTimes() (after finish()) sums their durations in ms over the enqueues since the
    // last call, at most kTimingRing of them, and returns how many it summed.
    static constexpr int kTimingRing = 512;
    void setTiming(bool on) { timing_ = on; }
    int stageTimes(double ms[5]);

    const Layout& layout() const { return L_; }

private:
    void release();
    void uploadStatic();
    void enqueueStages(const void* dFrame, bool taps, bool fullTaps);

    int dev_;
    Layout L_;
    GailCudaEncodeSettings s_;
    SlotSizes z_;
    float slope_ = 0.f;
    cudaStream_t st_ = nullptr;
    cudaEvent_t ev_[5] = {};
    bool timing_ = false;
    std::vector<cudaEvent_t> ring_;  // kTimingRing x 6 events
    int ringNext_ = 0, ringCount_ = 0;
    std::vector<void*> dev_allocs_;
    std::vector<T1Job> jobs_;

    // device
    void* dIn_ = nullptr;
    float *dEotf_ = nullptr, *dThr_ = nullptr, *dLut_ = nullptr, *dLL_[2] = {nullptr, nullptr}, *dSlope_ = nullptr, *dTap_ = nullptr;
    uint32_t *dCoeffs_ = nullptr, *dInfo_ = nullptr, *dEnd_ = nullptr, *dLen_ = nullptr, *dPerm_ = nullptr,
             *dCtl_ = nullptr, *dOutInfo_ = nullptr, *dOutLen_ = nullptr, *dWork_ = nullptr;
    int32_t *dDist_ = nullptr, *dOutDist_ = nullptr;
    uint4* dSnaps_ = nullptr;
    uint2* dOffsets_ = nullptr;
    uint8_t *dSym_ = nullptr, *dCw_ = nullptr, *dOutData_ = nullptr;
    uint16_t* dXyz_ = nullptr;
    T1Job* dJobs_ = nullptr;
    ColorTables color_;
    float m_[9];
    // host (pinned)
    void* hIn_ = nullptr;
    uint32_t *hInfo_ = nullptr, *hLen_ = nullptr, *hSmall_ = nullptr;
    int32_t* hDist_ = nullptr;
    uint8_t* hData_ = nullptr;
    uint64_t hDataCap_ = 0;
    float* hSlope_ = nullptr;
    // debug taps
    std::vector<uint16_t> xyz_;
    std::vector<uint32_t> coeffs_;
    std::vector<float> wavelet_;
};

}  // namespace gb
