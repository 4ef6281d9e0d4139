// Tier-1 output compaction: per-block results from the fixed-stride device tables into
// the packed Tier1Frame form the host codec consumes (Josephur/libgail
// core/tier1_types.h:12-28): CblkInfo per block, pass lengths and distortions back to
// back, codewords back to back on 4-byte boundaries.
#include <cuda_runtime.h>

#include "common.cuh"
#include "compact.cuh"

namespace gb {

namespace {

constexpr int SCAN_THREADS = 1024;

__device__ __forceinline__ uint32_t warpInclusive(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// One CTA: exclusive scans of (codeword bytes rounded to 4) and pass counts, and the
// CblkInfo records. Totals go to tot[0] (bytes) and tot[1] (passes).
__global__ void __launch_bounds__(SCAN_THREADS) scanKernel(CompactArgs a) {
    __shared__ uint32_t sBytes[32], sPasses[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t per = divUp(a.n, SCAN_THREADS);
    const uint32_t b = min(a.n, tid * per), e = min(a.n, b + per);
    uint32_t bytes = 0, passes = 0;
    for (uint32_t i = b; i < e; ++i) {
        bytes += (a.info[4 * (size_t)i + 3] + 3u) & ~3u;
        passes += a.info[4 * (size_t)i + 1];
    }
    const uint32_t ib = warpInclusive(bytes, lane), ip = warpInclusive(passes, lane);
    if (lane == 31) {
        sBytes[wid] = ib;
        sPasses[wid] = ip;
    }
    __syncthreads();
    if (wid == 0) {
        const uint32_t vb = sBytes[lane], vp = sPasses[lane];
        const uint32_t xb = warpInclusive(vb, lane), xp = warpInclusive(vp, lane);
        sBytes[lane] = xb - vb;
        sPasses[lane] = xp - vp;
        if (lane == 31) {
            a.tot[0] = xb;
            a.tot[1] = xp;
        }
    }
    __syncthreads();
    uint32_t ob = sBytes[wid] + ib - bytes, op = sPasses[wid] + ip - passes;
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t* in = a.info + 4 * (size_t)i;
        const uint32_t np = in[1], len = in[3];
        uint32_t* o = a.outInfo + 5 * (size_t)i;
        o[0] = in[0];
        o[1] = np;
        o[2] = ob;
        o[3] = len;
        o[4] = op;
        ob += (len + 3u) & ~3u;
        op += np;
    }
}

// One warp per block: its pass tables and codeword to their packed places.
__global__ void __launch_bounds__(256) packKernel(CompactArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < a.n; i += warps) {
        const uint32_t* o = a.outInfo + 5 * (size_t)i;
        const uint32_t np = o[1], dOff = o[2], len = o[3], pOff = o[4];
        if (lane < (int)np) {
            a.outPassLen[pOff + lane] = a.passLen[(size_t)i * kMaxPasses + lane];
            a.outPassDist[pOff + lane] = a.passDist[(size_t)i * kMaxPasses + lane];
        }
        if (lane + 32 < (int)np) {
            a.outPassLen[pOff + lane + 32] = a.passLen[(size_t)i * kMaxPasses + lane + 32];
            a.outPassDist[pOff + lane + 32] = a.passDist[(size_t)i * kMaxPasses + lane + 32];
        }
        const uint32_t words = (len + 3u) >> 2;
        if ((uint64_t)dOff + words * 4ull > a.dataCap) {
            if (lane == 0) a.tot[2] = 1u;
            continue;
        }
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.jobs[i].cw);
        uint32_t* dst = reinterpret_cast<uint32_t*>(a.outData + dOff);
        // whole words; the bytes past the codeword in its last word are zeroed so that the
        // packed frame does not depend on what the region held before
        const uint32_t tailMask = (len & 3u) ? (1u << (8 * (len & 3u))) - 1u : 0xFFFFFFFFu;
        for (uint32_t k = lane; k < words; k += 32) dst[k] = k == words - 1 ? src[k] & tailMask : src[k];
    }
}

}  // namespace

void compactTier1(const CompactArgs& a, cudaStream_t st) {
    if (a.n == 0) return;
    scanKernel<<<1, SCAN_THREADS, 0, st>>>(a);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    packKernel<<<min(divUp(a.n, 8), (uint32_t)sms * 8), 256, 0, st>>>(a);
    GB_CHECK(cudaGetLastError());
}

}  // namespace gb
