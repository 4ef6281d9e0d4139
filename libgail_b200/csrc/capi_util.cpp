// Thread-local error text and per-device set-up for the C-ABI.
#include "capi_util.h"
#include "gail_b200.h"

#include <cuda_runtime.h>

#include <mutex>
#include <set>

#include "decoder.h"
#include "frontend.cuh"
#include "t1_encode.cuh"

namespace gb {

namespace {
thread_local std::string g_error = "no error";
std::mutex g_initMutex;
std::set<int> g_ready;
}  // namespace

void setLastError(const std::string& msg) { g_error = msg; }
const char* lastError() { return g_error.c_str(); }

void ensureDevice() {
    int dev = 0;
    GB_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_initMutex);
    if (g_ready.count(dev)) return;
    t1Init();
    frontendInit();
    decoderInit();
    g_ready.insert(dev);
}

}  // namespace gb

extern "C" GB_API const char* gb_last_error(void) { return gb::lastError(); }
