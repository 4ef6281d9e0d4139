// Tier-1 encoding without any allocation: gb_t1_encode_blocks_noalloc.
//
// Who this is for: callers that must not allocate device memory on their own. Examples
// are a real-time frame thread, where cudaMalloc can wait for the whole device to go idle
// and so turns into a latency spike, and a host process whose device memory is budgeted
// up front (a serving loop that admits work against a fixed HBM budget, or an
// application that hands this library a fixed share of a GPU it partitions among
// tenants), where memory taken outside that budget is not allowed. gb_t1_encode_blocks
// allocates its device buffers on every call; this entry point uses one static device
// array instead.
//
// The array (kNoAllocBytes, 7.6 MB) is a file-scope __device__ variable: it is reserved
// on every GPU that loads this library, from the load until the process exits, whether or
// not the entry point is ever called. It holds at most kNoAllocMaxBlocks code-blocks per
// call; a larger call is refused with GAIL_CUDA_MISUSE.
//
// Every call uses the same array and leaves its contents behind. The call clears the
// control words the kernels count with before it starts; everything else is written
// before it is read. Two calls whose device work overlaps (from different host threads,
// or on different streams) race on the array and corrupt each other's results: callers
// must serialise their calls.
//
// The work runs on a non-blocking stream that the library makes once per device, together
// with the array's address, and the call waits on that stream alone: other streams' work
// on the device is neither waited for nor held up. The address and the stream are kept
// for the life of the process, so cudaDeviceReset on a device after the first call there
// is not supported (the kept address and stream would belong to the destroyed context).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "capi_util.h"
#include "common.cuh"
#include "gail_b200.h"
#include "t1_encode.cuh"

namespace gb {

namespace {

constexpr uint32_t kNoAllocMaxBlocks = 64;
// Every block gets the region of a block with the most bit-planes a band can signal.
constexpr uint32_t kRegion = ((2560u * kMaxPlanes + 64u) + 15u) & ~15u;  // = t1SymbolBound(32, 32, 22)
// Layout of the array, per call of up to kNoAllocMaxBlocks blocks (offsets in bytes):
constexpr size_t kOffCtl = 0;                                                   // 16 words
constexpr size_t kOffSlope = 64;                                                // 1 float
constexpr size_t kOffJobs = 256;                                                // T1Job per block
constexpr size_t kOffCoeffs = kOffJobs + kNoAllocMaxBlocks * sizeof(T1Job);     // 1024 words per block
constexpr size_t kOffInfo = kOffCoeffs + (size_t)kNoAllocMaxBlocks * kCblkArea * 4;
constexpr size_t kOffEnd = kOffInfo + kNoAllocMaxBlocks * 16;
constexpr size_t kOffLen = kOffEnd + (size_t)kNoAllocMaxBlocks * kMaxPasses * 4;
constexpr size_t kOffDist = kOffLen + (size_t)kNoAllocMaxBlocks * kMaxPasses * 4;
constexpr size_t kOffSnaps = kOffDist + (size_t)kNoAllocMaxBlocks * kMaxPasses * 4;
constexpr size_t kOffPerm = kOffSnaps + (size_t)kNoAllocMaxBlocks * kMaxPasses * 16;
constexpr size_t kOffSym = (kOffPerm + kNoAllocMaxBlocks * 4 + 255) & ~(size_t)255;
constexpr size_t kOffCw = kOffSym + (size_t)kNoAllocMaxBlocks * kRegion;
constexpr size_t kNoAllocBytes = kOffCw + (size_t)kNoAllocMaxBlocks * kRegion;

static __device__ __align__(256) unsigned char g_scratch[kNoAllocBytes];

// Per device: the array's device address (in host code the name g_scratch is only a
// stand-in for the symbol, not an address a kernel may use) and the stream the calls run
// on, both made by the first call on that device.
constexpr int kMaxDevices = 64;
struct DeviceScratch {
    unsigned char* address = nullptr;
    cudaStream_t stream = nullptr;
};
std::mutex g_mutex;
DeviceScratch g_device[kMaxDevices];

DeviceScratch scratchForCurrentDevice() {
    int dev = 0;
    GB_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device index out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceScratch& d = g_device[dev];
    if (!d.address) {
        ensureDevice();
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error(std::string("no device address for the Tier-1 scratch array: ") +
                                     cudaGetErrorString(e));
        }
        cudaStream_t st = nullptr;
        GB_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        d.stream = st;
        d.address = static_cast<unsigned char*>(p);
    }
    return d;
}

}  // namespace

}  // namespace gb

using namespace gb;

extern "C" GB_API int gb_t1_encode_blocks_noalloc(const uint32_t* coeffs, const int32_t* geom4, uint32_t n, float slope,
                                                  const float* distScale, uint32_t* info4, uint32_t* passLen,
                                                  int32_t* passDist, uint8_t* data, uint32_t dataStride) {
    return gbGuard([&] {
        if (!coeffs || !geom4 || !info4 || !passLen || !passDist || !data) throw std::logic_error("null argument");
        if (n > kNoAllocMaxBlocks)
            throw std::logic_error("gb_t1_encode_blocks_noalloc takes at most " + std::to_string(kNoAllocMaxBlocks) +
                                   " code-blocks per call (" + std::to_string(n) + " given)");
        if (n == 0) return;
        const DeviceScratch dev = scratchForCurrentDevice();
        unsigned char* base = dev.address;
        const cudaStream_t st = dev.stream;
        T1Job jobs[kNoAllocMaxBlocks];
        for (uint32_t i = 0; i < n; ++i) {
            const int w = geom4[4 * i], h = geom4[4 * i + 1], orient = geom4[4 * i + 2], mp = geom4[4 * i + 3];
            if (w < 1 || w > 32 || h < 1 || h > 32 || orient < 0 || orient > 3 || mp < 0 || mp > 64)
                throw std::logic_error("code-block geometry out of range");
            jobs[i] = {reinterpret_cast<const uint32_t*>(base + kOffCoeffs) + (size_t)i * kCblkArea,
                       base + kOffSym + (size_t)i * kRegion,
                       base + kOffCw + (size_t)i * kRegion,
                       kRegion,
                       t1Geom(w, h, orient, mp),
                       distScale ? distScale[i] : 1.f,
                       0,
                       {0, 0}};
        }
        T1Launch L{reinterpret_cast<const T1Job*>(base + kOffJobs),
                   n,
                   reinterpret_cast<uint32_t*>(base + kOffInfo),
                   reinterpret_cast<uint32_t*>(base + kOffEnd),
                   reinterpret_cast<uint32_t*>(base + kOffLen),
                   reinterpret_cast<int32_t*>(base + kOffDist),
                   reinterpret_cast<uint4*>(base + kOffSnaps),
                   reinterpret_cast<uint32_t*>(base + kOffPerm),
                   reinterpret_cast<uint32_t*>(base + kOffCtl),
                   reinterpret_cast<const float*>(base + kOffSlope)};
        // inputs in, the previous call's control words cleared
        GB_CHECK(cudaMemcpyAsync(base + kOffCoeffs, coeffs, (size_t)n * kCblkArea * 4, cudaMemcpyHostToDevice, st));
        GB_CHECK(cudaMemcpyAsync(base + kOffJobs, jobs, n * sizeof(T1Job), cudaMemcpyHostToDevice, st));
        GB_CHECK(cudaMemcpyAsync(base + kOffSlope, &slope, 4, cudaMemcpyHostToDevice, st));
        GB_CHECK(cudaMemsetAsync(base + kOffCtl, 0, 64, st));
        t1Encode(L, st);
        uint32_t ctl[4];
        GB_CHECK(cudaMemcpyAsync(ctl, base + kOffCtl, 16, cudaMemcpyDeviceToHost, st));
        GB_CHECK(cudaStreamSynchronize(st));
        if (ctl[1]) throw std::runtime_error("Tier-1 encoder status " + std::to_string(ctl[1]));
        GB_CHECK(cudaMemcpyAsync(info4, base + kOffInfo, 16 * (size_t)n, cudaMemcpyDeviceToHost, st));
        GB_CHECK(cudaMemcpyAsync(passLen, base + kOffLen, (size_t)n * kMaxPasses * 4, cudaMemcpyDeviceToHost, st));
        GB_CHECK(cudaMemcpyAsync(passDist, base + kOffDist, (size_t)n * kMaxPasses * 4, cudaMemcpyDeviceToHost, st));
        GB_CHECK(cudaStreamSynchronize(st));
        for (uint32_t i = 0; i < n; ++i)
            if (info4[4 * i + 3] > dataStride) throw std::logic_error("dataStride too small for a codeword");
        // each codeword, exactly its length, into the caller's row; the row's bytes after
        // it are left as the caller had them
        for (uint32_t i = 0; i < n; ++i)
            if (const uint32_t len = info4[4 * i + 3])
                GB_CHECK(cudaMemcpyAsync(data + (size_t)i * dataStride, base + kOffCw + (size_t)i * kRegion, len,
                                         cudaMemcpyDeviceToHost, st));
        GB_CHECK(cudaStreamSynchronize(st));
    });
}
