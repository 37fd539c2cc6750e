// Host-only check of the V-list sum groups (ddfmm_b200/csrc/plan.hpp) on a
// tree built from points read from a file: every (target, source) pair of
// every target's V list (src/wave3d_setup.cpp:302-390 builds those lists) is
// covered exactly once, by an entry whose tensor index is the pair's offset
// index, and nothing else is covered.
//   plan_test <points.bin (3n doubles)> <n> <K> <ncell> <maxlevel> <ptsmax>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <vector>

#include "plan.hpp"
#include "tree.hpp"

using namespace ddfmm;

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
    // low-frequency boxes with points, in key order (as the session numbers them)
    std::vector<int> lfbox, lfidx(T.boxes.size(), -1);
    for (int b : T.order)
        if (T.boxes[b].has_pts() && T.width(T.boxes[b].level) < 1 - 1e-12) {
            lfidx[b] = (int)lfbox.size();
            lfbox.push_back(b);
        }
    std::map<int, std::vector<int> > levels;
    for (int l = 0; l < (int)lfbox.size(); ++l) levels[T.boxes[lfbox[l]].level].push_back(l);
    long long pairs = 0, groups = 0;
    for (auto& kv : levels) {
        const VlistGroupPlan g = vlist_groups(T, lfbox, lfidx, kv.second);
        std::set<std::pair<int, int> > want, got;  // (target lf id, source lf id)
        for (int l : kv.second)
            for (int s : T.boxes[lfbox[l]].vlist) want.insert(std::make_pair(l, lfidx[s]));
        std::set<int> rows;
        for (size_t k = 0; k + 1 < g.gptr.size(); ++k) {
            groups++;
            for (int e = g.gptr[k]; e < g.gptr[k + 1]; ++e) {
                const VgEntry& E = g.gsrc[e];
                const int mask = E.tbase_mask & 255, tbase = E.tbase_mask >> 8;
                for (int c = 0; c < 8; ++c) {
                    if (!(mask & (1 << c))) continue;
                    const int tr = g.gtrg[8 * k + c];
                    if (tr < 0) { std::printf("pair for a missing child\n"); return 1; }
                    const int t = g.trg[tr];
                    const Box& TB = T.boxes[lfbox[t]];
                    const Box& SB = T.boxes[lfbox[E.row]];
                    int o[3];
                    for (int d = 0; d < 3; ++d) o[d] = TB.idx[d] - SB.idx[d];
                    const int voff = (o[0] + 3) + 7 * ((o[1] + 3) + 7 * (o[2] + 3));
                    if (tbase + vlist_child_voff(c) != voff) { std::printf("tensor index\n"); return 1; }
                    if ((TB.idx[0] & 1) * 4 + (TB.idx[1] & 1) * 2 + (TB.idx[2] & 1) != c) {
                        std::printf("child position\n");
                        return 1;
                    }
                    if (!got.insert(std::make_pair(t, E.row)).second) { std::printf("pair twice\n"); return 1; }
                }
            }
            for (int c = 0; c < 8; ++c)
                if (g.gtrg[8 * k + c] >= 0 && !rows.insert(g.gtrg[8 * k + c]).second) {
                    std::printf("row twice\n");
                    return 1;
                }
        }
        if (got != want) { std::printf("pairs differ: %zu against %zu\n", got.size(), want.size()); return 1; }
        if ((long long)got.size() != g.pairs) { std::printf("pair count\n"); return 1; }
        if (rows.size() != g.trg.size()) { std::printf("rows\n"); return 1; }
        pairs += g.pairs;
    }
    std::printf("ok pairs %lld groups %lld\n", pairs, groups);
    return 0;
}
