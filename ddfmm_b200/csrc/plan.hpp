// Host-only pieces of a session's launch plan, apart from the device uploads
// so that they can be built and checked without a GPU.
#pragma once
#include <vector>

#include "tree.hpp"

namespace ddfmm {

// One source position of a V-list group (kernels.cuh, VlistGroups; the same
// 16 bytes as the kernels' int4): the spectrum rows of parent A's and parent
// B's source there (-1 where none), the pair's tensor index for child
// position 0, and mask A | mask B << 8 of the children that list the source.
struct VgEntry {
    int row_a, row_b, tbase, masks;
};
static_assert(sizeof(VgEntry) == 16, "a V-list entry is one int4");

// Translation-tensor index of child position c (= 4a + 2b + c') relative to
// child position 0: a + 7b + 49c'.
inline int vlist_child_voff(int c) { return ((c >> 2) & 1) + 7 * ((c >> 1) & 1) + 49 * (c & 1); }

struct VlistGroupPlan {
    std::vector<int> trg;         // low-frequency id of each target, in summed-spectrum row order
    std::vector<int> gptr;        // groups + 1: the entries of each group
    std::vector<VgEntry> gsrc;    // the entries
    std::vector<int> gtrg;        // 16 per group: row of each child position of parent A, then B; -1 where none
    std::vector<int> src;         // low-frequency ids of the level's V-list sources, ascending
    long long pairs = 0;          // (target, source) pairs
};

// The V-list sum groups of one level (src/wave3d_eval.cpp:602-661 computes
// the same pairs target by target): the target boxes among `ids`
// (low-frequency ids; tree box lfbox[id], lfidx the inverse map) grouped by
// parent in the parents' Morton order, a parent paired with its +x neighbour
// when that one has targets too.  Throws if a V-list source lies outside the
// parent's 6^3 neighbourhood of child positions.
VlistGroupPlan vlist_groups(const Tree& T, const std::vector<int>& lfbox, const std::vector<int>& lfidx,
                            const std::vector<int>& ids);

}  // namespace ddfmm
