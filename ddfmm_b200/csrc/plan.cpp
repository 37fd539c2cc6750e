// Host-only pieces of a session's launch plan (plan.hpp).
#include "plan.hpp"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <exception>
#include <map>
#include <stdexcept>
#include <thread>
#include <unordered_map>

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
    // sources, each with the mask of the children that list it, in source-id
    // order; groups are built on all host cores, then concatenated in order
    std::vector<std::pair<size_t, size_t> > grp;  // [i, j) of tlist
    for (size_t i = 0; i < tlist.size();) {
        size_t j = i;
        while (j < tlist.size() && tlist[j].first == tlist[i].first) ++j;
        grp.push_back(std::make_pair(i, j));
        i = j;
    }
    const size_t ng = grp.size();
    out.trg.resize(tlist.size());
    out.gtrg.assign(ng * 8, -1);
    std::vector<std::vector<VgEntry> > ent(ng);
    std::vector<long long> gpairs(ng, 0);
    host_parallel_for(ng, [&](size_t g) {
        std::vector<std::pair<int, int> > e;  // (source lf id, (tbase << 8) | child bit)
        for (size_t k = grp[g].first; k < grp[g].second; ++k) {
            const int ct = tlist[k].second.first, l = tlist[k].second.second;
            const Box& B = T.boxes[lfbox[l]];
            out.gtrg[8 * g + ct] = (int)k;  // targets are numbered in tlist order
            out.trg[k] = l;
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
                e.push_back(std::make_pair(lfidx[s], (tbase << 8) | (1 << ct)));
            }
        }
        gpairs[g] = (long long)e.size();
        std::sort(e.begin(), e.end());
        std::vector<VgEntry>& v = ent[g];
        for (size_t k = 0; k < e.size();) {  // a source's pairs share tbase (one parent): OR the bits
            int m = 0;
            size_t q = k;
            for (; q < e.size() && e[q].first == e[k].first; ++q) m |= e[q].second & 255;
            v.push_back(VgEntry{e[k].first, (e[k].second & ~255) | m});
            k = q;
        }
    });
    out.gptr.assign(1, 0);
    std::vector<char> is_src(lfidx.empty() ? 0 : *std::max_element(lfidx.begin(), lfidx.end()) + 1, 0);
    for (size_t g = 0; g < ng; ++g) {
        out.gsrc.insert(out.gsrc.end(), ent[g].begin(), ent[g].end());
        out.gptr.push_back((int)out.gsrc.size());
        out.pairs += gpairs[g];
        for (const VgEntry& v : ent[g]) is_src[v.row] = 1;
    }
    for (size_t l = 0; l < is_src.size(); ++l)
        if (is_src[l]) out.src.push_back((int)l);
    return out;
}

void host_parallel_for(size_t n, const std::function<void(size_t)>& f) {
    const char* e = std::getenv("DDFMM_HOST_THREADS");
    const int v = e ? std::atoi(e) : 0;
    const size_t hw = v > 0 ? (size_t)v : std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(std::min<size_t>(hw, 64), n);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::exception_ptr> err(nt);
    std::vector<std::thread> th;
    for (size_t t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            try {
                for (size_t i = t; i < n; i += nt) f(i);
            } catch (...) {
                err[t] = std::current_exception();
            }
        });
    for (auto& x : th) x.join();
    for (auto& x : err)
        if (x) std::rethrow_exception(x);
}

int HfNodes::find(int box, const Idx3& dir) const {
    const int f = first[box], c = cnt[box];
    int lo = f, hi = f + c;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v[mid].dir < dir)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < f + c && v[lo].dir == dir) ? lo : -1;
}

std::vector<M2LChunk> m2l_pairs(const Tree& T, const HfNodes& up, const HfNodes& dn, int chunk) {
    std::vector<M2LChunk> chunks;
    for (auto& kv : dn.range)
        for (int i0 = kv.second.first; i0 < kv.second.second; i0 += chunk) {
            M2LChunk c;
            c.level = kv.first;
            c.i0 = i0;
            c.i1 = std::min(kv.second.second, i0 + chunk);
            chunks.push_back(std::move(c));
        }
    host_parallel_for(chunks.size(), [&](size_t ci) {
        M2LChunk& C = chunks[ci];
        std::unordered_map<uint64_t, int> loc;
        for (int i = C.i0; i < C.i1; ++i) {
            const HfNode& t = dn.v[i];
            const Box& tb = T.boxes[t.box];
            auto fit = tb.far.find(t.dir);
            if (fit == tb.far.end()) continue;
            Idx3 sgn, pv, srt;
            index3_sort(t.dir, srt, sgn, pv);
            for (int sb_i : fit->second) {
                const int uit = up.find(sb_i, t.dir);
                if (uit < 0) throw std::runtime_error("M2L source has no outgoing equivalent density");
                const Box& sb = T.boxes[sb_i];
                int o[3];
                std::array<int, 3> oc;
                for (int d = 0; d < 3; ++d) o[d] = tb.idx[d] - sb.idx[d];
                for (int d = 0; d < 3; ++d) oc[d] = sgn[pv[d]] * o[pv[d]];
                const uint64_t key = ((uint64_t)t.canon << 33) | ((uint64_t)(oc[0] + 1024) << 22) |
                                     ((uint64_t)(oc[1] + 1024) << 11) | (uint64_t)(oc[2] + 1024);
                auto it = loc.find(key);
                int li;
                if (it == loc.end()) {
                    li = (int)C.keys.size();
                    loc.emplace(key, li);
                    C.keys.push_back(key);
                    C.kcanon.push_back(t.canon);
                    C.koc.push_back(oc);
                    C.X.emplace_back();
                    C.Y.emplace_back();
                } else {
                    li = it->second;
                }
                C.X[li].push_back(up.v[uit].off);
                C.Y[li].push_back(t.off);
                C.pairs++;
            }
        }
    });
    return chunks;
}

void ColLists::add(std::vector<int>& tab, int k, long long xv, long long yv) {
    int p = tab[k];
    if (p < 0) {
        p = tab[k] = (int)key.size();
        key.push_back(k);
        x.emplace_back();
        y.emplace_back();
    }
    x[p].push_back(xv);
    y[p].push_back(yv);
}

HfColumns hf_columns(const Tree& T, const HfNodes& up, const HfNodes& dn, const std::vector<int>& kids,
                     const std::vector<long long>& lf_off, size_t ndirs, size_t ncanon) {
    HfColumns out;
    // jobs (level, pass, child position): an M2M / L2L pass splits by child
    // position, whose keys (wedge id * 8 + position) are disjoint, and the
    // positions' lists are concatenated in position order afterwards -- the
    // first-seen order of one loop over positions, then nodes
    struct Job {
        int level, pass, ind;
    };
    std::vector<Job> jobs;
    for (auto& kv : up.range)
        for (int pass = 0; pass < 4; ++pass) {
            (pass == 0 ? out.m2m : pass == 1 ? out.e2 : pass == 2 ? out.e2t : out.l2l)[kv.first];
            if (pass == 0 || pass == 3)
                for (int ind = 0; ind < 8; ++ind) jobs.push_back(Job{kv.first, pass, ind});
            else
                jobs.push_back(Job{kv.first, pass, -1});
        }
    std::vector<ColLists> part(jobs.size());
    host_parallel_for(jobs.size(), [&](size_t j) {
        const int level = jobs[j].level, pass = jobs[j].pass, ind = jobs[j].ind;
        const bool upward = pass == 0 || pass == 1;
        const HfNodes& N = upward ? up : dn;
        const auto r = N.range.at(level);
        ColLists& L = part[j];
        if (pass == 0 || pass == 3) {
            // M2M: child w -> parent sum; L2L: parent t -> child u (a problem per (wedge, child position))
            const bool lf_children = T.width(level) == 1.0;
            std::vector<int> tab(ndirs * 8, -1);
            for (int i = r.first; i < r.second; ++i) {
                const HfNode& u = N.v[i];
                const int c = kids[(size_t)u.box * 8 + ind];
                if (c < 0) continue;
                long long coff;
                if (lf_children) {
                    coff = lf_off[c];
                } else {
                    const int ci = N.find(c, predir(u.dir));
                    if (ci < 0)
                        throw std::runtime_error(upward ? "child has no directional equivalent density"
                                                        : "child has no directional check value");
                    coff = N.v[ci].off;
                }
                if (upward)
                    L.add(tab, u.did * 8 + ind, coff, u.toff);
                else
                    L.add(tab, u.did * 8 + ind, u.toff, coff);
            }
        } else {
            // E2 (upward: temporary -> outgoing vector) and E2^T (downward: incoming -> temporary)
            std::vector<int> tab(ncanon, -1);
            for (int i = r.first; i < r.second; ++i) {
                const HfNode& u = N.v[i];
                if (upward)
                    L.add(tab, u.canon, u.toff, u.off);
                else
                    L.add(tab, u.canon, u.off, u.toff);
            }
        }
    });
    for (size_t j = 0; j < jobs.size(); ++j) {  // jobs of one (level, pass) are adjacent, positions ascending
        const int pass = jobs[j].pass;
        ColLists& L = (pass == 0 ? out.m2m : pass == 1 ? out.e2 : pass == 2 ? out.e2t : out.l2l).at(jobs[j].level);
        ColLists& P = part[j];
        for (size_t k = 0; k < P.key.size(); ++k) {
            L.key.push_back(P.key[k]);
            L.x.push_back(std::move(P.x[k]));
            L.y.push_back(std::move(P.y[k]));
        }
    }
    return out;
}

}  // namespace ddfmm
