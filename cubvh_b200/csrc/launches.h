// Count of the kernels this library has launched in the process, for
// measurement (cubvh_kernel_launches in the C ABI).  Every launch site calls
// count_launch() after its launch; replays of a captured CUDA graph are not
// launches of this library and are not counted.
#pragma once
#include <atomic>
#include <cstdint>

namespace cubvh {
extern std::atomic<uint64_t> g_kernel_launches;
inline void count_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace cubvh
