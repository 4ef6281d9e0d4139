// Shared helpers for the sm_100a kernels and their host launchers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace gb {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kCblk = 32;            // code-blocks are 32 x 32 (DCI: xcb = ycb = 5)
constexpr int kCblkArea = 1024;
constexpr int kMaxPasses = 64;       // per code-block pass table capacity (3 * 22 - 2 fits)
constexpr int kMaxPlanes = 22;       // magnitude bit-planes a band may signal (Mb <= 22)
constexpr int kFracBits = 6;         // fractional magnitude bits carried with each coefficient

// Device status word bits (a kernel reports, the host turns them into an error).
enum : uint32_t {
    kErrTooManyPlanes = 1u,   // a block with more bit-planes than the pass table holds
    kErrSymbolSpace = 2u,     // a block's symbol region was too small (cannot happen for valid input)
    kErrCodewordSpace = 4u,   // a codeword outgrew its region
    kErrDecodeInput = 8u,     // a decode descriptor pointed outside its buffers
    kErrQueueWait = 16u,      // a persistent launch's wait for other warps' work gave up
};

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Out of device memory while the device stays usable (GAIL_CUDA_DEVICE_MEMORY).
struct DeviceMemoryError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) throw DeviceMemoryError(std::string(what) + ": " + cudaGetErrorString(e));
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

#define GB_CHECK(x) ::gb::check((x), #x)

__host__ __device__ inline uint32_t divUp(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace gb
