// Octree and interaction lists (see tree.hpp for the reference map).
#include "tree.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <exception>
#include <stdexcept>
#include <thread>

namespace ddfmm {

static void check(bool ok, const char* what) {
    if (!ok) throw std::runtime_error(what);
}

uint64_t Tree::pack(int level, const Idx3& idx) {
    return ((uint64_t)level << 57) | ((uint64_t)idx[0] << 38) | ((uint64_t)idx[1] << 19) |
           (uint64_t)idx[2];
}

int Tree::unitlevel() const { return (int)std::round(std::log(prm.K) / std::log(2.0)); }
int Tree::cell_level() const { return (int)std::round(std::log((double)prm.ncell) / std::log(2.0)); }
double Tree::width(int level) const { return prm.K / (double)(1 << level); }

// BoxCenter, src/wave3d.cpp:131-142 (same operation order)
Pt3 Tree::center(const Box& b) const {
    int tmp = 1 << b.level;
    Pt3 t;
    for (int d = 0; d < 3; ++d) t[d] = prm.ctr[d] - prm.K / 2 + (b.idx[d] + 0.5) / tmp * prm.K;
    return t;
}

static inline uint64_t mix64(uint64_t k) {  // a 64-bit finalizer: every key bit reaches the slot bits
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

void Tree::BoxIndex::clear() {
    keys.assign(1024, ~0ull);
    vals.assign(1024, -1);
    used = 0;
}

bool Tree::BoxIndex::insert(uint64_t k, int v) {
    if (2 * (used + 1) > keys.size()) {  // grow to keep the table at most half full
        std::vector<uint64_t> ok;
        std::vector<int> ov;
        ok.swap(keys);
        ov.swap(vals);
        keys.assign(2 * ok.size(), ~0ull);
        vals.assign(2 * ok.size(), -1);
        used = 0;
        for (size_t i = 0; i < ok.size(); ++i)
            if (ok[i] != ~0ull) insert(ok[i], ov[i]);
    }
    const size_t mask = keys.size() - 1;
    for (size_t s = mix64(k) & mask;; s = (s + 1) & mask) {
        if (keys[s] == k) return false;
        if (keys[s] == ~0ull) {
            keys[s] = k;
            vals[s] = v;
            ++used;
            return true;
        }
    }
}

int Tree::BoxIndex::find(uint64_t k) const {
    const size_t mask = keys.size() - 1;
    for (size_t s = mix64(k) & mask;; s = (s + 1) & mask) {
        if (keys[s] == k) return vals[s];
        if (keys[s] == ~0ull) return -1;
    }
}

int Tree::find(int level, const Idx3& idx) const { return index_.find(pack(level, idx)); }

// a box has all 8 children (some without points) or none
int Tree::child(int b, int ind) const { return boxes[b].kid0 >= 0 ? boxes[b].kid0 + ind : -1; }

// nml2dir, src/wave3d.cpp:43-71
// Component d: t = floor(atan(n[d] / mval) / Ang) clamped to [-B, B-1], and
// 2t + 1; the largest component becomes C round(atan(+-1)) = +-C.  Where the
// tree holds the bin edges for C, t is found among them, and the arithmetic
// above runs only for a ratio within 1e-9 of an edge (so t is the same as the
// arithmetic's: away from an edge, rounding in atan and the division cannot
// move the quotient across an integer).
Idx3 Tree::nml2dir(const Pt3& n, double W) const {
    int C = prm.npq * (int)std::round(W);
    int B = C / 2;
    int midx = 0;
    double mval = std::fabs(n[0]);
    for (int d = 1; d < 3; ++d)
        if (mval < std::fabs(n[d])) {
            midx = d;
            mval = std::fabs(n[d]);
        }
    const double Ang = (M_PI / 2) / C;
    const std::vector<double>* E = C < (int)edges_.size() && !edges_[C].empty() ? &edges_[C] : nullptr;
    Idx3 res;
    for (int d = 0; d < 3; ++d) {
        if (d == midx) continue;
        const double x = n[d] / mval;
        int t = 0;
        bool exact = true;
        if (E) {
            // edges <= x: t = -B below every edge, edge j is tan((j + 1 - B) Ang)
            const size_t i = std::upper_bound(E->begin(), E->end(), x) - E->begin();
            const double lo = i > 0 ? (*E)[i - 1] : -2.0, hi = i < E->size() ? (*E)[i] : 2.0;
            if (x - lo > 1e-9 && hi - x > 1e-9) {
                t = (int)i - B;
                exact = false;
            }
        }
        if (exact) t = (int)std::floor(std::atan(x) / Ang);
        t = std::min(std::max(t, -B), B - 1);
        res[d] = 2 * t + 1;
    }
    // n[midx] / mval is exactly +-1, and round(atan(+-1)) = +-1
    res[midx] = n[midx] > 0 ? C : -C;
    return res;
}

static int linfty(const Idx3& d) {
    return std::max(std::abs(d[0]), std::max(std::abs(d[1]), std::abs(d[2])));
}

// ParentDir, src/wave3d.cpp:74-95 (== Mlib3d::predir, src/mlib3d.cpp:283-303)
Idx3 Tree::parent_dir(const Idx3& dir) {
    int C = linfty(dir);
    int B = C / 2;
    int midx = -1;
    for (int d = 0; d < 3; ++d)
        if (std::abs(dir[d]) == C) midx = d;
    check(midx != -1, "parent_dir: no main axis");
    Idx3 res;
    for (int d = 0; d < 3; ++d) {
        res[d] = (dir[d] + C - 1) / 2;
        res[d] = 2 * (res[d] / 2) + 1 - B;
    }
    res[midx] = dir[midx] / 2;
    return res;
}

// ChildDir, src/wave3d.cpp:98-119
std::vector<Idx3> Tree::child_dirs(const Idx3& dir) {
    int C = linfty(dir);
    int oidx[2], no = 0;
    for (int d = 0; d < 3; ++d)
        if (std::abs(dir[d]) != C && no < 2) oidx[no++] = d;
    check(no == 2, "child_dirs: not a wedge");
    std::vector<Idx3> res;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            Idx3 t{{2 * dir[0], 2 * dir[1], 2 * dir[2]}};
            t[oidx[0]] += 2 * a - 1;
            t[oidx[1]] += 2 * b - 1;
            res.push_back(t);
        }
    return res;
}

double Tree::dir_width(const Idx3& d) const { return (double)(linfty(d) / prm.npq); }

// setup_tree_adjacent, src/wave3d_setup.cpp:463-477
bool Tree::adjacent(const Box& me, const Box& yo) const {
    int md = std::max(me.level, yo.level);
    int sm = 1 << (md - me.level), sy = 1 << (md - yo.level);
    int rad = sm + sy, dmax = 0;
    for (int d = 0; d < 3; ++d) {
        int dif = std::abs((2 * me.idx[d] + 1) * sm - (2 * yo.idx[d] + 1) * sy);
        if (dif > rad) return false;
        dmax = std::max(dmax, dif);
    }
    return dmax == rad;
}

// setup_tree_find, src/wave3d_setup.cpp:446-460: the box itself, else its
// nearest existing ancestor, stopping at the cell level.
int Tree::find_or_ancestor(int level, Idx3 idx) const {
    int cl = cell_level();
    while (level != cl) {
        int b = find(level, idx);
        if (b >= 0) return b;
        level -= 1;
        for (int d = 0; d < 3; ++d) idx[d] /= 2;
    }
    return find(level, idx);
}

static Pt3 sub(const Pt3& a, const Pt3& b) { return Pt3{{a[0] - b[0], a[1] - b[1], a[2] - b[2]}}; }
static double l2(const Pt3& a) {
    double s = 0;
    for (int d = 0; d < 3; ++d) s = s + a[d] * a[d];
    return std::sqrt(s);
}

// setup_tree_callowlist, src/wave3d_setup.cpp:302-390
void Tree::lowlist(int bi) {
    Box& cur = boxes[bi];
    check(cur.level != cell_level(), "low-frequency box at the cell level");
    // key sets as vectors, sorted and deduplicated at the end (key order, as the
    // reference's std::set<BoxKey>)
    std::vector<uint64_t> U, V, Wl, X;
    Idx3 par{{cur.idx[0] / 2, cur.idx[1] / 2, cur.idx[2] / 2}};
    int L = 1 << cur.level;
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = std::max(2 * par[d] - 2, 0);
        hi[d] = std::min(2 * par[d] + 4, L);
    }
    // find_or_ancestor(cur.level, tp) for the 6^3 block: tp's parent-level box
    // tp / 2 is one of the parent's 27 neighbours; the box at tp exists exactly
    // when that neighbour exists and is split (then it is child tp & 1),
    // otherwise the answer is the neighbour's own nearest existing ancestor
    int nb[27];
    for (int a = 0; a < 27; ++a) {
        const Idx3 q{{par[0] + a / 9 - 1, par[1] + (a / 3) % 3 - 1, par[2] + a % 3 - 1}};
        const int half = L / 2;
        nb[a] = (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= half || q[1] >= half || q[2] >= half)
                    ? -1
                    : find_or_ancestor(cur.level - 1, q);
    }
    for (int i = lo[0]; i < hi[0]; ++i)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int k = lo[2]; k < hi[2]; ++k) {
                Idx3 tp{{i, j, k}};
                if (tp == cur.idx) continue;
                const int q = nb[(i / 2 - par[0] + 1) * 9 + (j / 2 - par[1] + 1) * 3 + (k / 2 - par[2] + 1)];
                int ri = q;
                if (q >= 0 && boxes[q].level == cur.level - 1 && boxes[q].kid0 >= 0)
                    ri = boxes[q].kid0 + (i & 1) * 4 + (j & 1) * 2 + (k & 1);
                if (ri < 0) continue;
                const Box& res = boxes[ri];
                bool adj = adjacent(res, cur);
                if (res.level < cur.level && res.has_pts()) {
                    if (!adj)
                        X.push_back(pack(res.level, res.idx));
                    else if (cur.terminal())
                        U.push_back(pack(res.level, res.idx));
                }
                if (res.level == cur.level) {
                    if (!adj) {
                        Idx3 bb{{res.idx[0] - cur.idx[0], res.idx[1] - cur.idx[1], res.idx[2] - cur.idx[2]}};
                        check(linfty(bb) <= 3, "V-list offset beyond 3");
                        if (res.has_pts()) V.push_back(pack(res.level, res.idx));
                    } else if (cur.terminal()) {
                        std::vector<int> rest(1, ri);  // boxes still to visit (any order: the lists are sets)
                        while (!rest.empty()) {
                            int fi = rest.back();
                            rest.pop_back();
                            const Box& fnt = boxes[fi];
                            bool a2 = adjacent(fnt, cur);
                            if (!a2 && fnt.has_pts()) Wl.push_back(pack(fnt.level, fnt.idx));
                            if (a2 && fnt.terminal() && fnt.has_pts()) U.push_back(pack(fnt.level, fnt.idx));
                            if (a2 && !fnt.terminal())
                                for (int ind = 0; ind < 8; ++ind) {
                                    int c = child(fi, ind);
                                    check(c >= 0, "missing child of a split box");
                                    rest.push_back(c);
                                }
                        }
                    }
                }
            }
    if (cur.terminal() && cur.has_pts()) U.push_back(pack(cur.level, cur.idx));
    auto out = [&](std::vector<uint64_t>& s, std::vector<int>& v) {
        std::sort(s.begin(), s.end());
        s.erase(std::unique(s.begin(), s.end()), s.end());
        v.clear();
        v.reserve(s.size());
        for (uint64_t key : s) {
            const int b = index_.find(key);
            check(b >= 0, "listed box missing");
            v.push_back(b);
        }
    };
    out(U, cur.ulist);
    out(V, cur.vlist);
    out(Wl, cur.wlist);
    out(X, cur.xlist);
}

// setup_tree_calhghlist, src/wave3d_setup.cpp:393-443
void Tree::highlist(int bi) {
    Box& cur = boxes[bi];
    Pt3 cc = center(cur);
    double W = width(cur.level);
    double D = W * W + W;
    double threshold = D - 1e-12;
    // far boxes grouped by wedge in visiting order: a small open-addressing table
    // from wedge to group (a box has tens of wedges), the groups moved into the
    // map in wedge order at the end
    std::vector<std::pair<Idx3, std::vector<int> > > groups;
    std::vector<int> slot(256, -1);  // kept at most half full
    auto hash = [](const Idx3& d) {
        return (unsigned)(d[0] * 73856093) ^ (unsigned)(d[1] * 19349663) ^ (unsigned)(d[2] * 83492791);
    };
    auto group_of = [&](const Idx3& d) -> std::vector<int>& {
        unsigned mask = (unsigned)slot.size() - 1;
        unsigned s = hash(d) & mask;
        for (; slot[s] >= 0; s = (s + 1) & mask)
            if (groups[slot[s]].first == d) return groups[slot[s]].second;
        groups.emplace_back(d, std::vector<int>());
        if (2 * groups.size() <= slot.size()) {
            slot[s] = (int)groups.size() - 1;
        } else {  // grow, and place every group again
            slot.assign(2 * slot.size(), -1);
            mask = (unsigned)slot.size() - 1;
            for (int g = 0; g < (int)groups.size(); ++g) {
                unsigned t = hash(groups[g].first) & mask;
                while (slot[t] >= 0) t = (t + 1) & mask;
                slot[t] = g;
            }
        }
        return groups.back().second;
    };
    auto classify = [&](int oi) {
        const Box& oth = boxes[oi];
        if (!oth.has_pts()) return;
        Pt3 diff = sub(cc, center(oth));
        double n = l2(diff);
        if (n >= threshold) {
            Pt3 u{{diff[0] / n, diff[1] / n, diff[2] / n}};
            group_of(nml2dir(u, W)).push_back(oi);
        } else {
            cur.nearlist.push_back(oi);
        }
    };
    if (cur.level == cell_level()) {
        for (int oi : order) {
            if (boxes[oi].level != cell_level()) break;
            classify(oi);
        }
    } else {
        int pi = find(cur.level - 1, Idx3{{cur.idx[0] / 2, cur.idx[1] / 2, cur.idx[2] / 2}});
        check(pi >= 0, "missing parent of a high-frequency box");
        std::vector<int> pnear = boxes[pi].nearlist;
        for (int t : pnear)
            for (int ind = 0; ind < 8; ++ind) {
                int oi = child(t, ind);
                check(oi >= 0, "missing child of a near box");
                classify(oi);
            }
    }
    std::sort(groups.begin(), groups.end(),
              [](const std::pair<Idx3, std::vector<int> >& a, const std::pair<Idx3, std::vector<int> >& b) {
                  return a.first < b.first;
              });
    for (auto& g : groups) cur.far.emplace_hint(cur.far.end(), g.first, std::move(g.second));
}

// Host threads for list construction: DDFMM_HOST_THREADS when set (> 0), else
// every hardware thread.
static size_t host_threads() {
    const char* e = std::getenv("DDFMM_HOST_THREADS");
    const int v = e ? std::atoi(e) : 0;
    return v > 0 ? (size_t)v : std::max(1u, std::thread::hardware_concurrency());
}

// f(i) for i in [0, n) on the host's cores; each i is independent.  The first
// exception thrown by any call is rethrown here after every thread has joined.
template <class F>
static void parallel_for(size_t n, F f) {
    const size_t hw = host_threads();
    const size_t nt = std::min<size_t>(std::min<size_t>(hw, 64), (n + 255) / 256);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::exception_ptr> err(nt);
    std::vector<std::thread> th;
    for (size_t t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            try {
                for (size_t i = t; i < n; i += nt) f(i);  // interleaved: boxes of a level differ in cost
            } catch (...) {
                err[t] = std::current_exception();
            }
        });
    for (auto& x : th) x.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// setup_tree, src/wave3d_setup.cpp:100-299
void Tree::build(const double* p3n, int n, const TreeParams& p) {
    prm = p;
    pos = p3n;
    npts = n;
    boxes.clear();
    order.clear();
    index_.clear();
    edges_.clear();
    check(prm.ncell >= 1 && (prm.ncell & (prm.ncell - 1)) == 0, "ncell must be a power of two");
    const bool trace = std::getenv("DDFMM_SETUP_TRACE") != nullptr;
    auto tmark = std::chrono::steady_clock::now();
    auto phase = [&](const char* what) {
        if (!trace) return;
        const auto t = std::chrono::steady_clock::now();
        std::fprintf(stderr, "ddfmm tree  %-16s %8.3f s\n", what, std::chrono::duration<double>(t - tmark).count());
        tmark = t;
    };
    const int numC = prm.ncell, lvlC = cell_level();
    const double K = prm.K;
    // cells (all of them, empty or not), points in id order
    std::vector<std::vector<int> > cellpts((size_t)numC * numC * numC);
    for (int id = 0; id < n; ++id) {
        int ix[3];
        for (int d = 0; d < 3; ++d) {
            ix[d] = (int)std::floor(numC * ((p3n[3 * id + d] - prm.ctr[d] + K / 2) / K));
            check(ix[d] >= 0 && ix[d] < numC, "point outside the root box");
        }
        cellpts[((size_t)ix[0] * numC + ix[1]) * numC + ix[2]].push_back(id);
    }
    std::deque<int> q;
    auto add = [&](int level, const Idx3& idx, std::vector<int>&& pts) {
        Box b;
        b.level = level;
        b.idx = idx;
        b.pts = std::move(pts);
        boxes.push_back(std::move(b));
        int bi = (int)boxes.size() - 1;
        check(index_.insert(pack(level, idx), bi), "duplicate box");
        q.push_back(bi);
    };
    for (int a = 0; a < numC; ++a)
        for (int b = 0; b < numC; ++b)
            for (int c = 0; c < numC; ++c)
                add(lvlC, Idx3{{a, b, c}}, std::move(cellpts[((size_t)a * numC + b) * numC + c]));
    const int ul = unitlevel();
    while (!q.empty()) {
        int bi = q.front();
        q.pop_front();
        int level = boxes[bi].level;
        size_t np = boxes[bi].pts.size();
        if (np > 0) boxes[bi].tag |= TAG_PTS;
        bool split = (level <= ul && np > 0) || ((int)np > prm.ptsmax && level < prm.maxlevel - 1);
        if (split) {
            Pt3 cc = center(boxes[bi]);
            std::vector<int> cp[8];
            for (int id : boxes[bi].pts) {
                int a = p3n[3 * id + 0] >= cc[0], b = p3n[3 * id + 1] >= cc[1], c = p3n[3 * id + 2] >= cc[2];
                cp[a * 4 + b * 2 + c].push_back(id);
            }
            Idx3 base = boxes[bi].idx;
            boxes[bi].pts.clear();
            boxes[bi].kid0 = (int)boxes.size();  // add() appends the children in ind order
            for (int ind = 0; ind < 8; ++ind)
                add(level + 1, Idx3{{2 * base[0] + ((ind & 4) >> 2), 2 * base[1] + ((ind & 2) >> 1), 2 * base[2] + (ind & 1)}},
                    std::move(cp[ind]));
        } else {
            boxes[bi].tag |= TAG_TERMINAL;
        }
    }
    phase("partition");
    order.resize(boxes.size());
    for (size_t i = 0; i < boxes.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return pack(boxes[x].level, boxes[x].idx) < pack(boxes[y].level, boxes[y].idx);
    });
    // lists for every box with points (src/wave3d_setup.cpp:206-220), then the
    // directional sets (:255-296).  A box's low-frequency lists read only the tree;
    // its high-frequency lists and directional sets read its parent's, so both run
    // level by level (levels are contiguous in key order), the boxes of a level in
    // parallel.  Every box's lists come from the same sequential code, so the result
    // does not depend on the thread count.
    phase("sort");
    const double eps = 1e-12;
    // nml2dir's bin edges for every high-frequency width of the tree
    for (size_t i = 0; i < order.size(); ++i) {
        if (i > 0 && boxes[order[i]].level == boxes[order[i - 1]].level) continue;
        const double W = width(boxes[order[i]].level);
        if (W < 1 - eps) continue;
        const int C = prm.npq * (int)std::round(W), B = C / 2;
        if (C <= 0 || C > (1 << 16)) continue;
        if ((int)edges_.size() <= C) edges_.resize(C + 1);
        if (!edges_[C].empty()) continue;
        const double Ang = (M_PI / 2) / C;
        for (int t = 1 - B; t <= B - 1; ++t) edges_[C].push_back(std::tan(t * Ang));
    }
    std::vector<size_t> lv(1, 0);
    for (size_t i = 1; i < order.size(); ++i)
        if (boxes[order[i]].level != boxes[order[i - 1]].level) lv.push_back(i);
    lv.push_back(order.size());
    for (size_t l = 0; l + 1 < lv.size(); ++l)
        parallel_for(lv[l + 1] - lv[l], [&](size_t i) {
            const int bi = order[lv[l] + i];
            if (!boxes[bi].has_pts()) return;
            if (width(boxes[bi].level) < 1 - eps)
                lowlist(bi);
            else
                highlist(bi);
        });
    phase("lists");
    for (size_t l = 0; l + 1 < lv.size(); ++l)
        parallel_for(lv[l + 1] - lv[l], [&](size_t i) {
            Box& cur = boxes[order[lv[l] + i]];
            double W = width(cur.level);
            if (!(W > 1 - eps && cur.has_pts())) return;
            // the sets as sorted, deduplicated vectors first (most insertions repeat)
            std::vector<Idx3> out, inc;
            if (cur.level != lvlC) {
                int pi = find(cur.level - 1, Idx3{{cur.idx[0] / 2, cur.idx[1] / 2, cur.idx[2] / 2}});
                check(pi >= 0, "missing parent");
                for (const Idx3& d : boxes[pi].outdirs) out.push_back(parent_dir(d));
                for (const Idx3& d : boxes[pi].incdirs) inc.push_back(parent_dir(d));
            }
            Pt3 cc = center(cur);
            for (auto& kv : cur.far) {
                // the incoming direction of every far box is its key: highlist classified
                // (cc - oc) / |cc - oc| with the same arithmetic
                inc.push_back(kv.first);
                for (int oi : kv.second) {
                    Pt3 t = sub(center(boxes[oi]), cc);
                    double nt = l2(t);
                    for (int d = 0; d < 3; ++d) t[d] /= nt;
                    const Idx3 dir = nml2dir(t, W);
                    if (out.empty() || out.back() != dir) out.push_back(dir);  // runs repeat a wedge
                }
            }
            for (std::vector<Idx3>* v : {&out, &inc}) {
                std::sort(v->begin(), v->end());
                v->erase(std::unique(v->begin(), v->end()), v->end());
            }
            cur.outdirs.insert(out.begin(), out.end());
            cur.incdirs.insert(inc.begin(), inc.end());
        });
    phase("directions");
}

// HighFetchIndex3Sort, src/mlib3d.cpp:328-357
void index3_sort(Idx3 val, Idx3& srt, Idx3& sgn, Idx3& prm) {
    for (int d = 0; d < 3; ++d) {
        sgn[d] = val[d] < 0 ? -1 : 1;
        val[d] = std::abs(val[d]);
    }
    int upp = linfty(val) + 1;
    for (int d = 0; d < 3; ++d) {
        int minidx = d, minval = val[d];
        for (int e = 0; e < 3; ++e)
            if (val[e] < minval) {
                minval = val[e];
                minidx = e;
            }
        srt[d] = minval;
        prm[d] = minidx;
        val[minidx] = upp;
    }
}

}  // namespace ddfmm
