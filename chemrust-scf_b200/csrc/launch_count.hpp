// Process-wide count of kernel launches issued by this library (reported by
// chfsi_launch_count; used to state how many device kernels a step runs).
#pragma once

#include <atomic>

namespace chfsi {
extern std::atomic<long long> g_launch_count;
inline void count_launch(int n = 1) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }
}  // namespace chfsi
