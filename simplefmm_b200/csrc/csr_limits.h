// Size limit of the device CSR lists (pure C++, shared with a CPU test).
//
// Row pointers and entry indices of the interaction list and of the
// near-field ranges are int32.  Their totals are summed in 64 bits on the
// device (exclusive_scan_i32's total64) and checked here before the lists
// are allocated, so a tree whose lists would pass 2^31 - 1 entries is
// refused instead of wrapping the row pointers.
#pragma once

#include <cstdint>
#include <string>

namespace sfmm {

constexpr int64_t kMaxCsrEntries = 2147483647;     // INT32_MAX

inline bool csr_total_fits(int64_t total) { return total >= 0 && total <= kMaxCsrEntries; }

inline std::string csr_overflow_message(const char* what, int64_t total)
{
    return std::string(what) + " would hold " + std::to_string(total) +
           " entries, more than the 2147483647 its int32 row pointers can index; use a larger leaf size or fewer points";
}

}  // namespace sfmm
