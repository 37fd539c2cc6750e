// Host-only pieces of a session's launch plan, apart from the device uploads
// so that they can be built and checked without a GPU.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <map>
#include <utility>
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

// f(i) for i in [0, n) on the host's cores (DDFMM_HOST_THREADS, when set,
// caps them); the first exception is rethrown after every thread joined.
void host_parallel_for(size_t n, const std::function<void(size_t)>& f);

// A (box, wedge) node of the high-frequency passes: its canonical wedge
// (index into the session's canonical operators), its vector's offset
// (outgoing equivalent densities / incoming check values), its offset in the
// level's temporary, and the dense id of its (width, wedge).
struct HfNode {
    int box;
    Idx3 dir;
    int canon;
    long long off, toff;
    int did;
};
// The nodes of one direction (outgoing or incoming), level by level; a box's
// nodes are contiguous and in its (sorted) wedge order.
struct HfNodes {
    std::vector<HfNode> v;
    std::vector<int> first, cnt;              // per tree box
    std::map<int, std::pair<int, int> > range;  // level -> [begin, end)
    int find(int box, const Idx3& dir) const;  // binary search in the box's nodes; -1 if absent
};

// The M2L far pairs (src/wave3d_eval.cpp:876-928) of incoming nodes
// [i0, i1) of one level, grouped by (canonical wedge, canonical offset) --
// the offset c_t - c_s mapped by the wedge's canonical permutation and signs,
// so M(dir, offset) = M(canon, canonical offset) -- in first-seen order, each
// with its columns: the source's outgoing vector and the target's incoming.
struct M2LChunk {
    int level, i0, i1;
    std::vector<uint64_t> keys;  // canon << 33 | (offset + 1024) packed 11 bits a component
    std::vector<int> kcanon;
    std::vector<std::array<int, 3> > koc;  // canonical offsets
    std::vector<std::vector<long long> > X, Y;
    long long pairs = 0;
};
// Every incoming node's far pairs, in chunks of `chunk` nodes (never across
// levels) listed on all host cores; in chunk order the keys' first
// appearances and the columns are those of one pass over the nodes in order.
std::vector<M2LChunk> m2l_pairs(const Tree& T, const HfNodes& up, const HfNodes& dn, int chunk = 2048);

// Problems in first-seen order (keyed by (wedge id, child position) or by
// canonical wedge) with their input and output columns.
struct ColLists {
    std::vector<int> key;
    std::vector<std::vector<long long> > x, y;
    void add(std::vector<int>& tab, int k, long long xv, long long yv);
};
// The column lists of every level's M2M, E2, E2^T and L2L launches, one job per
// level and pass on all host cores (src/wave3d_eval.cpp:796-849 upward,
// 938-991 downward).  kids: the children with points of every box (8 per box,
// -1 where none); lf_off: the low-frequency vector offset of a box (children
// of width-1 boxes); ndirs, ncanon: the ranges of HfNode::did and ::canon.
struct HfColumns {
    std::map<int, ColLists> m2m, e2, e2t, l2l;  // by level
};
HfColumns hf_columns(const Tree& T, const HfNodes& up, const HfNodes& dn, const std::vector<int>& kids,
                     const std::vector<long long>& lf_off, size_t ndirs, size_t ncanon);

}  // namespace ddfmm
