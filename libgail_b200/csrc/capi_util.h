// Status handling shared by every C-ABI entry point: no exception crosses the boundary;
// a failure returns a status and leaves its message for the calling thread.
#pragma once
#include <cuda_runtime.h>

#include <new>
#include <stdexcept>
#include <string>

#include "common.cuh"

namespace gb {

// GailCudaStatus values (the plugin ABI's status codes).
enum : int { kOk = 0, kError = 1, kDeviceMemory = 2, kHostMemory = 3, kMisuse = 4, kNoCode = 5 };

void setLastError(const std::string& msg);
const char* lastError();

template <class F>
int gbGuard(F&& fn) noexcept {
    try {
        fn();
        return kOk;
    } catch (const DeviceMemoryError& e) {
        setLastError(e.what());
        return kDeviceMemory;
    } catch (const std::bad_alloc&) {
        setLastError("out of host memory");
        return kHostMemory;
    } catch (const std::logic_error& e) {
        setLastError(e.what());
        return kMisuse;
    } catch (const std::exception& e) {
        setLastError(e.what());
        return kError;
    } catch (...) {
        setLastError("unknown error");
        return kError;
    }
}

// Makes sure the calling thread has a current device with this library's tables loaded.
void ensureDevice();
// Whether this library's kernels load on the current device (cudaSuccess when they do).
cudaError_t kernelsLoadable();
// One warp of the persistent Tier-1 launch's wait, on a flag nothing sets, given up after
// limitMs: returns the status bits it left (kErrQueueWait) and the launch's duration.
uint32_t t1WaitSelftest(uint32_t limitMs, float* elapsedMs);

}  // namespace gb
