// Host-only pieces of a session's launch plan (plan.hpp).
#include "plan.hpp"

#include <algorithm>
#include <cstdint>
#include <map>
#include <stdexcept>

namespace ddfmm {

VlistGroupPlan vlist_groups(const Tree& T, const std::vector<int>& lfbox, const std::vector<int>& lfidx,
                            const std::vector<int>& ids) {
    auto morton = [](const Idx3& x) {
        uint64_t m = 0;
        for (int bit = 0; bit < 21; ++bit)
            for (int d = 0; d < 3; ++d) m |= (uint64_t)((x[d] >> bit) & 1) << (3 * bit + d);
        return m;
    };
    VlistGroupPlan out;
    // (parent Morton key, child position, lf id) of every target
    std::vector<std::pair<uint64_t, std::pair<int, int> > > tlist;
    for (int l : ids) {
        const Box& B = T.boxes[lfbox[l]];
        if (B.vlist.empty()) continue;
        const Idx3 par{{B.idx[0] >> 1, B.idx[1] >> 1, B.idx[2] >> 1}};
        const int ct = 4 * (B.idx[0] & 1) + 2 * (B.idx[1] & 1) + (B.idx[2] & 1);
        tlist.push_back(std::make_pair(morton(par), std::make_pair(ct, l)));
    }
    std::sort(tlist.begin(), tlist.end());
    // per target parent: its children's rows and, by local source position (the
    // tensor index of the pair for child 0, tbase), the source and the mask of the
    // children that list it
    struct Parent {
        Idx3 idx;
        int trow[8];
        std::map<int, std::pair<int, int> > by_tbase;  // tbase -> (source lf id, child mask)
    };
    std::vector<Parent> parents;
    std::map<Idx3, int> parent_at;
    std::vector<char> is_src(lfidx.empty() ? 0 : *std::max_element(lfidx.begin(), lfidx.end()) + 1, 0);
    for (size_t i = 0; i < tlist.size();) {
        size_t j = i;
        while (j < tlist.size() && tlist[j].first == tlist[i].first) ++j;  // one parent: [i, j)
        Parent pa;
        for (int c = 0; c < 8; ++c) pa.trow[c] = -1;
        for (size_t k = i; k < j; ++k) {
            const int ct = tlist[k].second.first, l = tlist[k].second.second;
            const Box& B = T.boxes[lfbox[l]];
            pa.idx = Idx3{{B.idx[0] >> 1, B.idx[1] >> 1, B.idx[2] >> 1}};
            pa.trow[ct] = (int)out.trg.size();
            out.trg.push_back(l);
            for (int s : B.vlist) {
                const Box& SB = T.boxes[s];
                int rel[3], o[3];
                for (int d = 0; d < 3; ++d) {
                    rel[d] = SB.idx[d] - 2 * (B.idx[d] >> 1);
                    o[d] = B.idx[d] - SB.idx[d];
                    if (SB.level != B.level || rel[d] < -2 || rel[d] > 3)
                        throw std::runtime_error("V-list source outside the parent's neighbourhood");
                }
                const int tbase = (3 - rel[0]) + 7 * ((3 - rel[1]) + 7 * (3 - rel[2]));
                // the kernel's offset index for this pair: tbase + a + 7b + 49c
                const int voff = (o[0] + 3) + 7 * ((o[1] + 3) + 7 * (o[2] + 3));
                if (tbase + vlist_child_voff(ct) != voff) throw std::logic_error("V-list offset bookkeeping");
                auto& e = pa.by_tbase[tbase];
                if (e.second == 0) e.first = lfidx[s];
                if (e.first != lfidx[s]) throw std::logic_error("V-list source position bookkeeping");
                e.second |= 1 << ct;
                is_src[lfidx[s]] = 1;
                out.pairs++;
            }
        }
        parent_at[pa.idx] = (int)parents.size();
        parents.push_back(std::move(pa));
        i = j;
    }
    // groups: a parent with its +x neighbour when that one has targets too (each
    // source position's tensor values then serve both), else alone; in the
    // parents' Morton order
    out.gptr.assign(1, 0);
    std::vector<char> taken(parents.size(), 0);
    for (size_t pi = 0; pi < parents.size(); ++pi) {
        if (taken[pi]) continue;
        taken[pi] = 1;
        const Parent& A = parents[pi];
        const Parent* B = nullptr;
        auto it = parent_at.find(Idx3{{A.idx[0] + 1, A.idx[1], A.idx[2]}});
        if (it != parent_at.end() && !taken[it->second]) {
            taken[it->second] = 1;
            B = &parents[it->second];
        }
        for (int c = 0; c < 8; ++c) out.gtrg.push_back(A.trow[c]);
        for (int c = 0; c < 8; ++c) out.gtrg.push_back(B ? B->trow[c] : -1);
        std::map<int, VgEntry> ents;  // by tbase
        for (auto& kv : A.by_tbase) ents[kv.first] = VgEntry{kv.second.first, -1, kv.first, kv.second.second};
        if (B)
            for (auto& kv : B->by_tbase) {
                auto e = ents.find(kv.first);
                if (e == ents.end()) {
                    ents[kv.first] = VgEntry{-1, kv.second.first, kv.first, kv.second.second << 8};
                } else {
                    e->second.row_b = kv.second.first;
                    e->second.masks |= kv.second.second << 8;
                }
            }
        for (auto& kv : ents) out.gsrc.push_back(kv.second);
        out.gptr.push_back((int)out.gsrc.size());
    }
    for (size_t l = 0; l < is_src.size(); ++l)
        if (is_src[l]) out.src.push_back((int)l);
    return out;
}

}  // namespace ddfmm
