// Process-wide count of the kernels this library has launched (reported by
// dgmr_launch_count(); benchmarks use it to state how many kernels ran).
#pragma once

#include <atomic>
#include <cstdint>

namespace dgmr {

inline std::atomic<uint64_t>& launch_counter()
{
    static std::atomic<uint64_t> counter { 0 };
    return counter;
}

inline void note_launch(uint64_t n = 1) { launch_counter().fetch_add(n, std::memory_order_relaxed); }

} // namespace dgmr
