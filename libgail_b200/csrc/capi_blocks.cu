// C-ABI entry points over single stages, for callers that hold code-blocks rather than
// frames (and for the parity tests): a batch of quantised code-blocks through the
// Tier-1 encoder, and a batch of codewords through the Tier-1 decoder.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "capi_util.h"
#include "gail_b200.h"
#include "common.cuh"
#include "t1_encode.cuh"

using namespace gb;

namespace {

template <class T>
struct DevBuf {
    T* p = nullptr;
    explicit DevBuf(size_t n) { GB_CHECK(cudaMalloc((void**)&p, (n ? n : 1) * sizeof(T))); }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

}  // namespace

extern "C" {

GB_API int gb_t1_encode_blocks(const uint32_t* coeffs, const int32_t* geom4, uint32_t n, float slope, const float* distScale,
                        uint32_t* info4, uint32_t* passLen, int32_t* passDist, uint8_t* data, uint32_t dataStride) {
    return gbGuard([&] {
        if (!coeffs || !geom4 || !info4 || !passLen || !passDist || !data) throw std::logic_error("null argument");
        if (n == 0) return;
        ensureDevice();
        std::vector<T1Job> jobs(n);
        std::vector<uint64_t> offset(n);
        uint64_t region = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const int w = geom4[4 * i], h = geom4[4 * i + 1], orient = geom4[4 * i + 2], mp = geom4[4 * i + 3];
            if (w < 1 || w > 32 || h < 1 || h > 32 || orient < 0 || orient > 3 || mp < 0 || mp > 64)
                throw std::logic_error("code-block geometry out of range");
            offset[i] = region;
            region += t1SymbolBound(w, h, kMaxPlanes);
        }
        DevBuf<uint32_t> dCoeffs((size_t)n * kCblkArea), dInfo(4 * (size_t)n), dEnd((size_t)n * kMaxPasses),
            dLen((size_t)n * kMaxPasses), dPerm(n), dCtl(4);
        DevBuf<int32_t> dDist((size_t)n * kMaxPasses);
        DevBuf<uint4> dSnaps((size_t)n * kMaxPasses);
        DevBuf<uint8_t> dSym(region), dCw(region);
        DevBuf<T1Job> dJobs(n);
        DevBuf<float> dSlope(1);
        for (uint32_t i = 0; i < n; ++i) {
            const int w = geom4[4 * i], h = geom4[4 * i + 1], orient = geom4[4 * i + 2], mp = geom4[4 * i + 3];
            jobs[i] = {dCoeffs.p + (size_t)i * kCblkArea, dSym.p + offset[i], dCw.p + offset[i],
                       t1SymbolBound(w, h, kMaxPlanes), t1Geom(w, h, orient, mp), distScale ? distScale[i] : 1.f, 0, {0, 0}};
        }
        GB_CHECK(cudaMemcpy(dCoeffs.p, coeffs, (size_t)n * kCblkArea * 4, cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemcpy(dJobs.p, jobs.data(), n * sizeof(T1Job), cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemcpy(dSlope.p, &slope, 4, cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemset(dCtl.p, 0, 16));
        T1Launch L{dJobs.p, n, dInfo.p, dEnd.p, dLen.p, dDist.p, dSnaps.p, dPerm.p, dCtl.p, dSlope.p};
        t1Encode(L, 0);
        GB_CHECK(cudaDeviceSynchronize());
        uint32_t ctl[4];
        GB_CHECK(cudaMemcpy(ctl, dCtl.p, 16, cudaMemcpyDeviceToHost));
        if (ctl[1]) throw std::runtime_error("Tier-1 encoder status " + std::to_string(ctl[1]));
        GB_CHECK(cudaMemcpy(info4, dInfo.p, 16 * (size_t)n, cudaMemcpyDeviceToHost));
        GB_CHECK(cudaMemcpy(passLen, dLen.p, (size_t)n * kMaxPasses * 4, cudaMemcpyDeviceToHost));
        GB_CHECK(cudaMemcpy(passDist, dDist.p, (size_t)n * kMaxPasses * 4, cudaMemcpyDeviceToHost));
        std::vector<uint8_t> cw(region);
        GB_CHECK(cudaMemcpy(cw.data(), dCw.p, region, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t len = info4[4 * i + 3];
            if (len > dataStride) throw std::logic_error("dataStride too small for a codeword");
            std::memcpy(data + (size_t)i * dataStride, cw.data() + offset[i], len);
        }
    });
}

GB_API int gb_t1_wait_selftest(uint32_t limitMs, uint32_t* status, float* elapsedMs) {
    return gbGuard([&] {
        if (!status) throw std::logic_error("null argument");
        if (limitMs < 1 || limitMs > 2000) throw std::logic_error("limitMs must be 1..2000");
        ensureDevice();
        *status = t1WaitSelftest(limitMs, elapsedMs);
    });
}

}  // extern "C"
