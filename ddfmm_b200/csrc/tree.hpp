// Octree and interaction lists of the directional FMM, host side.
//
// Rebuilds, with this project's own data structures, exactly the tree and
// lists the reference's Wave3d::setup produces for one rank:
//   * setup_tree            src/wave3d_setup.cpp:100-299
//   * setup_tree_callowlist src/wave3d_setup.cpp:302-390  (U/V/W/X lists)
//   * setup_tree_calhghlist src/wave3d_setup.cpp:393-443  (near / far-by-wedge)
//   * setup_tree_find       src/wave3d_setup.cpp:446-460
//   * setup_tree_adjacent   src/wave3d_setup.cpp:463-477
//   * direction geometry    src/wave3d.cpp:43-142 (nml2dir, ParentDir,
//                           ChildDir, Dir2Width, BoxCenter)
//   * canonical wedges      src/mlib3d.cpp:283-357 (predir, HighFetchShuffle,
//                           HighFetchIndex3Sort)
// Boxes live in one vector; an open-addressing hash table from the packed key
// (level, i, j, k) finds them, and "key order" (the order of the reference's
// std::map<BoxKey>) is level first, then i, j, k lexicographically.
#pragma once
#include <array>
#include <cstdint>
#include <map>
#include <set>
#include <string>
#include <vector>

namespace ddfmm {

typedef std::array<int, 3> Idx3;     // Index3 (lexicographic order)
typedef std::array<double, 3> Pt3;   // Point3

enum { TAG_PTS = 1, TAG_TERMINAL = 2 };

struct Box {
    int level = 0;
    Idx3 idx{{0, 0, 0}};
    int tag = 0;
    int kid0 = -1;                             // a split box's 8 children are boxes kid0 .. kid0 + 7
    std::vector<int> pts;                      // point ids of a terminal box
    std::vector<int> ulist, vlist, wlist, xlist;  // LF lists, key order
    std::vector<int> nearlist;                 // HF near boxes (endeidxvec)
    std::map<Idx3, std::vector<int> > far;     // HF far boxes by wedge (fndeidxvec)
    std::set<Idx3> outdirs, incdirs;           // HF outgoing / incoming wedges
    bool has_pts() const { return tag & TAG_PTS; }
    bool terminal() const { return tag & TAG_TERMINAL; }
};

struct TreeParams {
    double K = 64;       // root-box width in wavelengths (-wave3d_K)
    Pt3 ctr{{0, 0, 0}};  // root-box centre (-wave3d_ctr)
    int ptsmax = 100;    // -wave3d_ptsmax
    int maxlevel = 12;   // -wave3d_maxlevel
    int npq = 4;         // wedges per quadrant (-wave3d_NPQ)
    int ncell = 8;       // cells per edge of the partition tensor (geomprtn.m())
};

class Tree {
public:
    TreeParams prm;
    const double* pos = nullptr;  // 3*N, point-major
    int npts = 0;
    std::vector<Box> boxes;
    std::vector<int> order;       // box indices in key order

    // Build the tree and all lists; throws std::runtime_error on the
    // conditions where the reference throws (CHECK_TRUE).
    void build(const double* pos3n, int n, const TreeParams& p);

    int unitlevel() const;
    int cell_level() const;
    double width(int level) const;       // BoxWidth
    Pt3 center(const Box& b) const;      // BoxCenter
    int find(int level, const Idx3& idx) const;  // -1 if absent
    int child(int b, int ind) const;             // child ind (0..7), -1 if absent

    Idx3 nml2dir(const Pt3& n, double W) const;
    static Idx3 parent_dir(const Idx3& d);
    static std::vector<Idx3> child_dirs(const Idx3& d);
    double dir_width(const Idx3& d) const;

private:
    // packed key -> box index: linear probing in a power-of-two table kept at
    // most half full (keys are never ~0, the empty mark)
    struct BoxIndex {
        std::vector<uint64_t> keys;
        std::vector<int> vals;
        size_t used = 0;
        void clear();
        bool insert(uint64_t k, int v);  // false if k is present
        int find(uint64_t k) const;      // -1 if absent
    };
    BoxIndex index_;
    // nml2dir's bin edges tan(t (pi/2) / C), t = 1-C/2 .. C/2-1, by C (filled by
    // build() for the widths of the tree before the parallel list passes)
    std::vector<std::vector<double> > edges_;
    static uint64_t pack(int level, const Idx3& idx);
    bool adjacent(const Box& a, const Box& b) const;
    int find_or_ancestor(int level, Idx3 idx) const;
    void lowlist(int b);
    void highlist(int b);
};

// Canonical wedge of a direction (src/mlib3d.cpp:328-357): srt = sorted
// |dir|, sgn = signs, prm = where each sorted component came from.
void index3_sort(Idx3 val, Idx3& srt, Idx3& sgn, Idx3& prm);
// ParentDir / predir (identical maps, src/wave3d.cpp:74-95, mlib3d.cpp:283-303)
inline Idx3 predir(const Idx3& d) { return Tree::parent_dir(d); }

}  // namespace ddfmm
