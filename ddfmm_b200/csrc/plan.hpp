// Host-only pieces of a session's launch plan, apart from the device uploads
// so that they can be built and checked without a GPU.
#pragma once
#include <vector>

#include "tree.hpp"

namespace ddfmm {

// One source of a V-list group (kernels.cuh, VlistGroups; the same 8 bytes as
// the kernels' int2): its spectrum row, and (tbase << 8) | mask, tbase the
// pair's tensor index for child position 0 and bit c of mask set when the
// child at position c lists the source.
struct VgEntry {
    int row, tbase_mask;
};
static_assert(sizeof(VgEntry) == 8, "a V-list entry is one int2");

// Translation-tensor index of child position c (= 4a + 2b + c') relative to
// child position 0: a + 7b + 49c'.
inline int vlist_child_voff(int c) { return ((c >> 2) & 1) + 7 * ((c >> 1) & 1) + 49 * (c & 1); }

struct VlistGroupPlan {
    std::vector<int> trg;         // low-frequency id of each target, in summed-spectrum row order
    std::vector<int> gptr;        // groups + 1: the entries of each group
    std::vector<VgEntry> gsrc;    // the entries
    std::vector<int> gtrg;        // 8 per group: row of each child position; -1 where none
    std::vector<int> src;         // low-frequency ids of the level's V-list sources, ascending
    long long pairs = 0;          // (target, source) pairs
};

// The V-list sum groups of one level (src/wave3d_eval.cpp:602-661 computes
// the same pairs target by target): the target boxes among `ids`
// (low-frequency ids; tree box lfbox[id], lfidx the inverse map) grouped by
// parent, in the parents' Morton order.  Throws if a V-list source lies
// outside the parent's 6^3 neighbourhood of child positions.
VlistGroupPlan vlist_groups(const Tree& T, const std::vector<int>& lfbox, const std::vector<int>& lfidx,
                            const std::vector<int>& ids);

}  // namespace ddfmm
