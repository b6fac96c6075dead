// device_once.h -- per-device, thread-safe memo for host-side kernel setup.
//
// cudaFuncSetAttribute (and occupancy answers derived from it) hold for the device that is
// current when they are made, so one process driving several GPUs must repeat them per
// device; handles on different threads may reach the same launcher at once.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

namespace ops_solver
{
constexpr int ONCE_MAX_DEVICES = 64;

// Runs set() until it succeeds once on the current device (devices past the table run it
// every time).  Two threads may both run it the first time; the attribute calls it makes
// are idempotent.
template <typename Set>
cudaError_t once_per_device(std::atomic<unsigned long long> &done, Set set)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= ONCE_MAX_DEVICES) return set();
    const unsigned long long bit = 1ull << dev;
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = set();
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// A value computed once per device by get() (a non-negative int), cached as value + 1.
template <typename Get>
int value_per_device(std::atomic<int> (&cache)[ONCE_MAX_DEVICES], Get get)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= ONCE_MAX_DEVICES) return get();
    const int v = cache[dev].load(std::memory_order_acquire);
    if (v > 0) return v - 1;
    const int g = get();
    cache[dev].store(g + 1, std::memory_order_release);
    return g;
}
}  // namespace ops_solver
