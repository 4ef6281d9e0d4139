// One decode in flight on the device: the plugin's decoder_* entry points (the role of
// the reference's CudaDecoderSlot, Josephur/libgail src/cuda/cuda_decode.cu:181-376).
// The host has parsed the headers and packets; this runs Tier-1 decoding with
// dequantisation, the inverse wavelet and the inverse ICT on the device.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <vector>

#include "gail_cuda_plugin_abi.h"
#include "layout.h"

namespace gb {

// A code-block as the decoder kernels see it (static per layout).
struct DecBlock {
    uint32_t dst;     // index of its top-left sample in the component planes (comp * npix + y * W + x)
    uint16_t w, h;
    uint8_t orient, band;
    uint8_t wanted;   // its resolution is decoded
    uint8_t pad;
};

uint64_t decoderSlotBytes(const Layout& L, const GailCudaDecodeSettings& s);
// Per-device set-up of the decoder kernels (tables, shared-memory opt-in).
void decoderInit();

class DecoderSlot {
public:
    // heavySms: decode the heaviest code-blocks on SMs of their own (the tuning's decHeavyPct),
    // for a decode that has the GPU to itself; slots of which several decode at once (the
    // served engine's) leave it off, as their launches would all reserve the same SMs.
    DecoderSlot(int device, const Layout& L, const GailCudaDecodeSettings& s, bool heavySms = true);
    ~DecoderSlot();
    DecoderSlot(const DecoderSlot&) = delete;
    DecoderSlot& operator=(const DecoderSlot&) = delete;

    // frame: this frame's layout (the slot's geometry, the stream's step sizes).
    void decode(const Layout& frame, const uint8_t* data, size_t size, const GbCblkCode* blocks, size_t numBlocks, void* dst,
                ptrdiff_t strideBytes, GailCudaDecodeTimings* tm);
    // The same in two halves: enqueue() copies the codestream and the blocks into the
    // slot's pinned buffers and starts every stage on the slot's stream; finish() waits,
    // checks the kernels' status and returns the picture in pinned host memory (outH rows
    // of outW x 3 codes), valid until the next enqueue. With pinnedDst the picture goes from
    // the device straight into those rows (page-locked host memory, dstStride bytes apart)
    // instead; with bands > 1 it comes back in that many row bands, each recording
    // bandDone(k) when it has arrived.
    void enqueue(const Layout& frame, const uint8_t* data, size_t size, const GbCblkCode* blocks, size_t numBlocks,
                 bool wantWavelet, void* pinnedDst = nullptr, ptrdiff_t dstStride = 0, int bands = 1);
    const uint16_t* finish(GailCudaDecodeTimings* tm);
    int outW() const { return outW_; }
    int outH() const { return outH_; }

private:
    void release();
    int dev_;
    Layout L_;
    GailCudaDecodeSettings s_;
    int outW_ = 0, outH_ = 0;
    bool heavySms_ = true;
    cudaStream_t st_ = nullptr;
    cudaEvent_t ev_[4] = {};
    static constexpr int kBands = 8;
    cudaEvent_t bandEv_[kBands] = {};  // a band of the picture has arrived in host memory
    std::vector<void*> allocs_;
    uint64_t capBytes_ = 0;
    float *dPlanes_ = nullptr, *dLL_[2] = {nullptr, nullptr}, *dHalf_ = nullptr;
    uint8_t* dBytes_ = nullptr;
    GbCblkCode* dCodes_ = nullptr;
    DecBlock* dBlocks_ = nullptr;
    uint32_t *dPerm_ = nullptr, *dCtl_ = nullptr;
    uint16_t* dOut_ = nullptr;
    uint8_t* hBytes_ = nullptr;
    GbCblkCode* hCodes_ = nullptr;
    uint16_t* hOut_ = nullptr;
    float* hHalf_ = nullptr;
    uint32_t* hCtl_ = nullptr;
    std::vector<float> wavelet_[3];
    bool wantWavelet_ = false;
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace gb
