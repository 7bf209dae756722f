// CPU test of the work split of a sharded solve (simplefmm_b200/csrc/shard_ranges.h).
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "shard_ranges.h"

int main()
{
    using namespace sfmm;
    std::mt19937_64 rng(7);
    int fails = 0;
    for (int trial = 0; trial < 2000; ++trial) {
        const int64_t nl = rng() % 300;
        std::vector<int64_t> prefix(nl + 1, 0);
        int64_t maxleaf = 0;
        for (int64_t i = 0; i < nl; ++i) {
            const int64_t c = 1 + int64_t(rng() % 200);      // a leaf holds at least one point
            prefix[i + 1] = prefix[i] + c;
            maxleaf = c > maxleaf ? c : maxleaf;
        }
        const int count = 1 + int(rng() % 9);
        int64_t prev = 0;
        for (int r = 0; r < count; ++r) {
            const auto rg = balanced_leaf_range(prefix.data(), nl, count, r);
            if (rg.first != prev || rg.second < rg.first) ++fails;             // consecutive, ordered
            prev = rg.second;
            // the cut is the first leaf whose prefix reaches the share's start
            const int64_t lo = shard_begin(prefix[nl], count, r);
            if (rg.first > 0 && prefix[rg.first - 1] >= lo && rg.first != 0) ++fails;
            if (rg.first < nl && prefix[rg.first] < lo) ++fails;
            const int64_t pts = prefix[rg.second] - prefix[rg.first];
            const int64_t share = shard_end(prefix[nl], count, r) - lo;
            if (pts > share + maxleaf || pts + maxleaf < share) ++fails;       // balanced within a leaf
        }
        if (prev != nl) ++fails;                                                 // covers every leaf
    }
    // node ranges: contiguous and covering
    for (int64_t n : {0, 1, 7, 1000}) {
        int64_t prev = 0;
        for (int c = 1; c <= 8; ++c) {
            prev = 0;
            for (int r = 0; r < c; ++r) {
                if (shard_begin(n, c, r) != prev) ++fails;
                prev = shard_end(n, c, r);
            }
            if (prev != n) ++fails;
        }
    }
    if (!fails) std::printf("shard ranges ok\n");
    else std::printf("%d failures\n", fails);
    return fails ? 1 : 0;
}
