// A small persistent thread pool for the host codec's per-frame work (rate control phases,
// packet measurement and writing). The calling thread always runs a share itself, so a call
// completes even when every pool thread is busy with other callers' work.
#pragma once
#include <functional>

namespace gb {

// Runs fn(i) for i in [0, n) on the pool and the calling thread; returns when all are done.
// Exceptions thrown by fn are rethrown here (the first one).
void parallelFor(int n, const std::function<void(int)>& fn);
// Threads the pool uses besides the caller (0: none, all work on the caller).
void setPoolThreads(int n);
int poolThreads();

}  // namespace gb
