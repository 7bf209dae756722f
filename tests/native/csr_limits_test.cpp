// CPU test of the CSR size guard (simplefmm_b200/csrc/csr_limits.h): totals
// are summed in 64 bits, and a total past INT32_MAX is refused rather than
// wrapped into the int32 row pointers.
#include <cstdint>
#include <cstdio>

#include "csr_limits.h"

static int fails = 0;
#define EXPECT(c)                                                      \
    do {                                                               \
        if (!(c)) {                                                    \
            std::printf("FAILED: %s (line %d)\n", #c, __LINE__);       \
            ++fails;                                                   \
        }                                                              \
    } while (0)

int main()
{
    using namespace sfmm;
    EXPECT(csr_total_fits(0));
    EXPECT(csr_total_fits(2147483647LL));
    EXPECT(!csr_total_fits(2147483648LL));
    EXPECT(!csr_total_fits(-1));
    // a full interaction list: 189 entries per node (partition.hpp:149);
    // the node count at which the int32 sum would wrap
    const int64_t per_node = 189;
    const int64_t nodes_ok = kMaxCsrEntries / per_node, nodes_bad = nodes_ok + 1;
    // the 64-bit total of nodes_bad full rows does not fit; an int32 running
    // sum would have wrapped to a negative value (computed in unsigned here)
    const int64_t sum64 = nodes_bad * per_node;
    const int32_t sum32 = static_cast<int32_t>(static_cast<uint32_t>(sum64));
    EXPECT(!csr_total_fits(sum64));
    EXPECT(sum32 < 0);
    EXPECT(csr_total_fits(nodes_ok * per_node));
    EXPECT(csr_overflow_message("the interaction list", sum64).find("2147483647") != std::string::npos);
    if (!fails) std::printf("csr limits ok\n");
    return fails ? 1 : 0;
}
