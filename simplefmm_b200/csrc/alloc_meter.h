// Device-allocation meters (pure C++; memory.cu implements them, the
// serving loop uses them).
#pragma once

#include <atomic>
#include <cstdint>

namespace sfmm {

// While a thread has meters set, every device allocation and release it
// makes adds / subtracts the block's bytes to their `live` count and raises
// their `peak`.  The serving loop meters each request (its own peak) and the
// whole server (the sum over the requests running at once).
struct AllocMeter {
    std::atomic<int64_t> live{0}, peak{0};
    void add(int64_t b)
    {
        const int64_t v = live.fetch_add(b) + b;
        int64_t pk = peak.load();
        while (v > pk && !peak.compare_exchange_weak(pk, v)) {
        }
    }
    void sub(int64_t b) { live.fetch_sub(b); }
};

void set_thread_alloc_meters(AllocMeter* request, AllocMeter* server) noexcept;
// The calling thread's meters and cache setting (a helper thread that works
// for a request takes them over).
void get_thread_alloc_meters(AllocMeter** request, AllocMeter** server) noexcept;
bool thread_block_cache() noexcept;

// While off for a thread, the device blocks it releases go straight back to
// the memory pool instead of the block cache, so a server holds no device
// memory beyond what its running requests use.
void set_thread_block_cache(bool on) noexcept;

}  // namespace sfmm
