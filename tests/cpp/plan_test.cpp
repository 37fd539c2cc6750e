// Host-only checks of the launch plan's pieces (ddfmm_b200/csrc/plan.hpp) on a
// tree built from points read from a file:
//  * V-list sum groups: every (target, source) pair of every target's V list
//    (src/wave3d_setup.cpp:302-390 builds those lists) is covered exactly
//    once, by an entry whose tensor index is the pair's offset index;
//  * M2L far pairs: every (incoming node, far source box) pair of every level
//    (src/wave3d_setup.cpp:393-443) appears once, with the source's outgoing
//    node and the canonical offset of the pair;
//  * M2M / E2 / E2^T / L2L column lists: every (node, child position with a
//    child) pair and every node appears once, in the problem of its wedge and
//    child position or of its canonical wedge, with the right columns;
//  * an order-sensitive hash of the V-list groups and the column lists, so a
//    faster construction can be held to the same problem and column order.
//   plan_test <points.bin (3n doubles)> <n> <K> <ncell> <maxlevel> <ptsmax>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <tuple>
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
    // order-sensitive hash of the plan pieces (FNV-1a over 64-bit words): the
    // test compares it with values recorded from the first implementation
    unsigned long long H = 1469598103934665603ull;
    auto mix = [&](long long v) {
        H ^= (unsigned long long)v;
        H *= 1099511628211ull;
    };
    long long pairs = 0, groups = 0;
    for (auto& kv : levels) {
        const VlistGroupPlan g = vlist_groups(T, lfbox, lfidx, kv.second);
        for (int x : g.trg) mix(x);
        for (int x : g.gptr) mix(x);
        for (const VgEntry& e : g.gsrc) {
            mix(e.row);
            mix(e.tbase_mask);
        }
        for (int x : g.gtrg) mix(x);
        for (int x : g.src) mix(x);
        mix(g.pairs);
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
    // ---------------------------------------------------------------- high frequency
    std::map<std::pair<double, Idx3>, int> dids, canons;
    auto did_of = [&](double W, const Idx3& d) { return dids.emplace(std::make_pair(W, d), (int)dids.size()).first->second; };
    auto canon_of = [&](double W, const Idx3& d) {
        Idx3 srt, sgn, prm;
        index3_sort(d, srt, sgn, prm);
        return canons.emplace(std::make_pair(W, srt), (int)canons.size()).first->second;
    };
    HfNodes up, dn;
    up.first.assign(T.boxes.size(), 0);
    up.cnt.assign(T.boxes.size(), 0);
    dn.first.assign(T.boxes.size(), 0);
    dn.cnt.assign(T.boxes.size(), 0);
    std::map<int, std::vector<int> > hf;
    for (int b : T.order)
        if (T.boxes[b].has_pts() && T.width(T.boxes[b].level) > 1 - 1e-12) hf[T.boxes[b].level].push_back(b);
    long long off = 0;
    for (auto& kv : hf) {
        const double W = T.width(kv.first);
        const int u0 = (int)up.v.size(), d0 = (int)dn.v.size();
        for (int b : kv.second) {
            up.first[b] = (int)up.v.size();
            up.cnt[b] = (int)T.boxes[b].outdirs.size();
            for (const Idx3& d : T.boxes[b].outdirs) {
                up.v.push_back(HfNode{b, d, canon_of(W, d), off, off + 1, did_of(W, d)});
                off += 10;
            }
            dn.first[b] = (int)dn.v.size();
            dn.cnt[b] = (int)T.boxes[b].incdirs.size();
            for (const Idx3& d : T.boxes[b].incdirs) {
                dn.v.push_back(HfNode{b, d, canon_of(W, d), off, off + 1, did_of(W, d)});
                off += 10;
            }
        }
        up.range[kv.first] = std::make_pair(u0, (int)up.v.size());
        dn.range[kv.first] = std::make_pair(d0, (int)dn.v.size());
    }
    // M2L pairs
    long long far = 0;
    std::set<std::pair<long long, long long> > seen;  // (target off, source off)
    for (const M2LChunk& C : m2l_pairs(T, up, dn, 97)) {
        for (size_t k = 0; k < C.keys.size(); ++k)
            for (size_t q = 0; q < C.X[k].size(); ++q) {
                if (!seen.insert(std::make_pair(C.Y[k][q], C.X[k][q])).second) { std::printf("far pair twice\n"); return 1; }
            }
        far += C.pairs;
    }
    long long want_far = 0;
    std::map<long long, int> dn_by_off, up_by_off;
    for (size_t i = 0; i < dn.v.size(); ++i) dn_by_off[dn.v[i].off] = (int)i;
    for (size_t i = 0; i < up.v.size(); ++i) up_by_off[up.v[i].off] = (int)i;
    for (const HfNode& t : dn.v) {
        auto fit = T.boxes[t.box].far.find(t.dir);
        if (fit == T.boxes[t.box].far.end()) continue;
        for (int sb : fit->second) {
            want_far++;
            const int ui = up.find(sb, t.dir);
            if (ui < 0 || !seen.count(std::make_pair(t.off, up.v[ui].off))) { std::printf("far pair missing\n"); return 1; }
        }
    }
    if (far != want_far || (long long)seen.size() != want_far) { std::printf("far pair count\n"); return 1; }
    // canonical offsets: recomputed for every listed pair
    for (const M2LChunk& C : m2l_pairs(T, up, dn))
        for (size_t k = 0; k < C.keys.size(); ++k)
            for (size_t q = 0; q < C.X[k].size(); ++q) {
                const HfNode& t = dn.v[dn_by_off.at(C.Y[k][q])];
                const HfNode& s = up.v[up_by_off.at(C.X[k][q])];
                Idx3 srt, sgn, prm;
                index3_sort(t.dir, srt, sgn, prm);
                int oc[3];
                for (int d = 0; d < 3; ++d) oc[d] = sgn[prm[d]] * (T.boxes[t.box].idx[prm[d]] - T.boxes[s.box].idx[prm[d]]);
                if (C.kcanon[k] != t.canon || oc[0] != C.koc[k][0] || oc[1] != C.koc[k][1] || oc[2] != C.koc[k][2]) {
                    std::printf("canonical offset\n");
                    return 1;
                }
            }
    // column lists
    std::vector<int> kids(T.boxes.size() * 8, -1);
    for (auto& kv : hf)
        for (int b : kv.second)
            for (int ind = 0; ind < 8; ++ind) {
                const int c = T.child(b, ind);
                if (c >= 0 && T.boxes[c].has_pts()) kids[(size_t)b * 8 + ind] = c;
            }
    std::vector<long long> lf_off(T.boxes.size(), -1);
    for (int l = 0; l < (int)lfbox.size(); ++l) lf_off[lfbox[l]] = 1000000000LL + l;
    const HfColumns cols = hf_columns(T, up, dn, kids, lf_off, dids.size(), canons.size());
    long long ncols = 0;
    for (auto& kv : hf) {
        const int level = kv.first;
        const bool lfc = T.width(level) == 1.0;
        for (int pass = 0; pass < 4; ++pass) {
            const bool upward = pass < 2;
            const HfNodes& N = upward ? up : dn;
            const ColLists& L = (pass == 0 ? cols.m2m : pass == 1 ? cols.e2 : pass == 2 ? cols.e2t : cols.l2l).at(level);
            std::set<std::tuple<int, long long, long long> > got2, want2;  // (key, x, y)
            for (size_t k = 0; k < L.key.size(); ++k)
                for (size_t q = 0; q < L.x[k].size(); ++q)
                    if (!got2.insert(std::make_tuple(L.key[k], L.x[k][q], L.y[k][q])).second) {
                        std::printf("column twice\n");
                        return 1;
                    }
            const auto r = N.range.at(level);
            for (int i = r.first; i < r.second; ++i) {
                const HfNode& u = N.v[i];
                if (pass == 1) want2.insert(std::make_tuple(u.canon, u.toff, u.off));
                if (pass == 2) want2.insert(std::make_tuple(u.canon, u.off, u.toff));
                if (pass == 0 || pass == 3)
                    for (int ind = 0; ind < 8; ++ind) {
                        const int c = kids[(size_t)u.box * 8 + ind];
                        if (c < 0) continue;
                        const long long co = lfc ? lf_off[c] : N.v[N.find(c, predir(u.dir))].off;
                        if (pass == 0) want2.insert(std::make_tuple(u.did * 8 + ind, co, u.toff));
                        else want2.insert(std::make_tuple(u.did * 8 + ind, u.toff, co));
                    }
            }
            if (got2 != want2) { std::printf("columns differ (level %d pass %d)\n", level, pass); return 1; }
            ncols += (long long)got2.size();
            for (size_t k = 0; k < L.key.size(); ++k) {
                mix(L.key[k]);
                for (long long x : L.x[k]) mix(x);
                for (long long y : L.y[k]) mix(y);
            }
            mix(-pass - 1);
        }
    }
    std::printf("ok pairs %lld groups %lld far %lld columns %lld hash %016llx\n", pairs, groups, far, ncols, H);
    return 0;
}
