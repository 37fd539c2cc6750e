// Order-sensitive hash of every box and list of the host tree
// (ddfmm_b200/csrc/tree.hpp): box keys and tags, point ids, the U/V/W/X and
// near lists, the far lists by wedge, the outgoing and incoming wedges, each
// in the order the tree holds them.  A change to how the lists are computed
// must leave the hash unchanged.
//   tree_hash <points.bin (3n doubles)> <n> <K> <ncell> <maxlevel> <ptsmax>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tree.hpp"

using namespace ddfmm;

static unsigned long long H = 1469598103934665603ull;  // FNV-1a over 64-bit words
static void mix(long long v) {
    H ^= (unsigned long long)v;
    H *= 1099511628211ull;
}

int main(int argc, char** argv) {
    if (argc < 7) return 2;
    const int n = std::atoi(argv[2]);
    std::vector<double> pos(3 * (size_t)n);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(pos.data(), sizeof(double), pos.size(), f) != pos.size()) return 2;
    std::fclose(f);
    TreeParams p;
    p.K = std::atof(argv[3]);
    p.ncell = std::atoi(argv[4]);
    p.maxlevel = std::atoi(argv[5]);
    p.ptsmax = std::atoi(argv[6]);
    Tree T;
    T.build(pos.data(), n, p);
    long long entries = 0;
    auto list = [&](const std::vector<int>& v) {
        mix((long long)v.size());
        for (int x : v) {
            const Box& o = T.boxes[x];
            mix(o.level);
            for (int d = 0; d < 3; ++d) mix(o.idx[d]);
            ++entries;
        }
    };
    for (int b : T.order) {
        const Box& B = T.boxes[b];
        mix(B.level);
        for (int d = 0; d < 3; ++d) mix(B.idx[d]);
        mix(B.tag);
        mix(0);
        for (int x : B.pts) mix(x);
        list(B.ulist);
        list(B.vlist);
        list(B.wlist);
        list(B.xlist);
        list(B.nearlist);
        mix((long long)B.far.size());
        for (auto& kv : B.far) {
            for (int d = 0; d < 3; ++d) mix(kv.first[d]);
            list(kv.second);
        }
        for (auto& d : B.outdirs)
            for (int e = 0; e < 3; ++e) mix(d[e]);
        mix(-7);
        for (auto& d : B.incdirs)
            for (int e = 0; e < 3; ++e) mix(d[e]);
    }
    std::printf("boxes %zu entries %lld hash %016llx\n", T.boxes.size(), entries, H);
    return 0;
}
