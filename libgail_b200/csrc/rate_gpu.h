// PCRD rate control and Tier-2 on the device: the slope range and slope histogram of the
// hull points, every exact size measurement of the threshold search (a warp per packet
// codes its header: tag trees, pass counts, lengths), and the final packets, written
// into the codestream body on the device. The host runs only the threshold search
// itself (rate_search.h, the same code as the host rate control) on a few numbers per
// measurement, and wraps the body in the main header and tile-part markers. Codeword
// bytes never leave the device unless they are in the codestream.
//
// Results are those of allocateRate + CodestreamWriter::build (and so of the reference's
// allocateRate + buildCodestream, Josephur/libgail src/core/rate_control.cpp:161-279,
// src/core/t2.cpp:38-254): the same bins (a hull point whose log2 slope lies within
// 1e-7 of a bin edge is binned on the host with the host's log2), the same sizes, the
// same thresholds, the same bytes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "codestream.h"
#include "layout.h"

namespace gb {

// A packed Tier-1 frame in device memory (the Tier1Frame layout: CblkInfo records, pass
// lengths at each block's passBase, codewords at each block's dataOffset) and its PCRD
// hull points in the HullView layout, also in device memory.
struct DeviceTier1 {
    const GbCblkInfo* info = nullptr;
    const uint32_t* passLen = nullptr;
    const uint8_t* data = nullptr;
    const uint8_t* hullPasses = nullptr;
    const double* hullSlope = nullptr;
};

// One layout's device rate control. Not thread-safe: one per worker thread. The calls
// run on the given stream and wait for it.
class DeviceRateControl {
public:
    // bodyHint: codestream bytes the buffers are first sized for (they grow when a frame
    // needs more, which waits for the device)
    DeviceRateControl(int device, const Layout& L, const std::string& label, size_t bodyHint = 4u << 20);
    ~DeviceRateControl();
    DeviceRateControl(const DeviceRateControl&) = delete;
    DeviceRateControl& operator=(const DeviceRateControl&) = delete;

    // Rate control to lim and the codestream (COM: label + " " + tag) of a frame on the
    // device; res.passes: the passes per block in it; res.distortion is not estimated.
    RateResult run(const DeviceTier1& f, const RateLimits& lim, const std::string& tag, std::vector<uint8_t>& out,
                   cudaStream_t st);
    // The same for a Tier-1 frame in host memory: uploaded, its hull computed on the
    // device, then run().
    RateResult runHost(const Tier1View& t1, const RateLimits& lim, const std::string& tag, std::vector<uint8_t>& out,
                       cudaStream_t st);

    const Layout& layout() const;
    size_t emptyBytes();

private:
    struct Impl;
    std::unique_ptr<Impl> p_;
};

}  // namespace gb
