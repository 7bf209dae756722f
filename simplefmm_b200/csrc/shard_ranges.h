// Work split of one solve over `count` shards (pure C++: the library's
// sharded evaluation and the oracle's restatement of it share this code).
//
// It follows the reference's split over MPI ranks:
//   * contiguous ranges [n r / count, n (r+1) / count)   (distributed.hpp:14-25)
//   * a level's leaves cut where the running point count reaches the same
//     fractions of the level's points (balanced_leaf_range, fmm.hpp:503-522)
// applied per level to
//   * leaves (P2M, L2P and the near field of their points), balanced by points;
//   * parents of the level's M2L targets (a sibling group is never split:
//     the M2L kernels own the children of a parent), contiguous ranges.
// The shards' partial moments and locals are summed between stages
// (fmm.hpp:832-859 does the same with MPI_Allreduce per level).
#pragma once

#include <cstdint>
#include <utility>

namespace sfmm {

inline int64_t shard_begin(int64_t n, int count, int index) { return n * index / count; }
inline int64_t shard_end(int64_t n, int count, int index) { return n * (index + 1) / count; }

// Leaves [first, last) of one level whose points prefix[] (n_leaf + 1 running
// point counts, prefix[0] = 0) are this shard's: the cut of a target count
// is the first leaf whose prefix reaches it.
inline std::pair<int64_t, int64_t> balanced_leaf_range(const int64_t* prefix, int64_t n_leaf, int count, int index)
{
    const int64_t total = prefix[n_leaf];
    auto cut = [&](int64_t target) {
        int64_t lo = 0, hi = n_leaf;
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (prefix[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    return {cut(shard_begin(total, count, index)), cut(shard_end(total, count, index))};
}

}  // namespace sfmm
