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
    // one group per target parent: its children's rows and the union of their
    // sources, each with the mask of the children that list it
    std::vector<char> is_src(lfidx.empty() ? 0 : *std::max_element(lfidx.begin(), lfidx.end()) + 1, 0);
    out.gptr.assign(1, 0);
    for (size_t i = 0; i < tlist.size();) {
        size_t j = i;
        while (j < tlist.size() && tlist[j].first == tlist[i].first) ++j;  // one parent: [i, j)
        const size_t g0 = out.gtrg.size();
        out.gtrg.resize(g0 + 8, -1);
        std::map<int, int> srcs;  // source lf id -> (tbase << 8) | mask
        for (size_t k = i; k < j; ++k) {
            const int ct = tlist[k].second.first, l = tlist[k].second.second;
            const Box& B = T.boxes[lfbox[l]];
            out.gtrg[g0 + ct] = (int)out.trg.size();
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
                int& e = srcs[lfidx[s]];
                e = (tbase << 8) | (e & 255) | (1 << ct);
                is_src[lfidx[s]] = 1;
                out.pairs++;
            }
        }
        for (auto& kv : srcs) out.gsrc.push_back(VgEntry{kv.first, kv.second});
        out.gptr.push_back((int)out.gsrc.size());
        i = j;
    }
    for (size_t l = 0; l < is_src.size(); ++l)
        if (is_src[l]) out.src.push_back((int)l);
    return out;
}

}  // namespace ddfmm
