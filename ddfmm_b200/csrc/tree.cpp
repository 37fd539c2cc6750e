// Octree and interaction lists (see tree.hpp for the reference map).
#include "tree.hpp"

#include <algorithm>
#include <cmath>
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

int Tree::find(int level, const Idx3& idx) const {
    auto it = index_.find(pack(level, idx));
    return it == index_.end() ? -1 : it->second;
}

int Tree::child(int b, int ind) const {
    const Box& p = boxes[b];
    Idx3 c{{2 * p.idx[0] + ((ind & 4) >> 2), 2 * p.idx[1] + ((ind & 2) >> 1), 2 * p.idx[2] + (ind & 1)}};
    return find(p.level + 1, c);
}

// nml2dir, src/wave3d.cpp:43-71
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
    double val[3];
    for (int d = 0; d < 3; ++d) val[d] = std::atan(n[d] / mval);
    double Ang = (M_PI / 2) / C;
    Idx3 res;
    for (int d = 0; d < 3; ++d) {
        int t = (int)std::floor(val[d] / Ang);
        t = std::min(std::max(t, -B), B - 1);
        res[d] = 2 * t + 1;
    }
    res[midx] = C * (int)std::round(val[midx]);
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
    std::set<uint64_t> U, V, Wl, X;
    Idx3 par{{cur.idx[0] / 2, cur.idx[1] / 2, cur.idx[2] / 2}};
    int L = 1 << cur.level;
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = std::max(2 * par[d] - 2, 0);
        hi[d] = std::min(2 * par[d] + 4, L);
    }
    for (int i = lo[0]; i < hi[0]; ++i)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int k = lo[2]; k < hi[2]; ++k) {
                Idx3 tp{{i, j, k}};
                if (tp == cur.idx) continue;
                int ri = find_or_ancestor(cur.level, tp);
                if (ri < 0) continue;
                const Box& res = boxes[ri];
                bool adj = adjacent(res, cur);
                if (res.level < cur.level && res.has_pts()) {
                    if (!adj)
                        X.insert(pack(res.level, res.idx));
                    else if (cur.terminal())
                        U.insert(pack(res.level, res.idx));
                }
                if (res.level == cur.level) {
                    if (!adj) {
                        Idx3 bb{{res.idx[0] - cur.idx[0], res.idx[1] - cur.idx[1], res.idx[2] - cur.idx[2]}};
                        check(linfty(bb) <= 3, "V-list offset beyond 3");
                        if (res.has_pts()) V.insert(pack(res.level, res.idx));
                    } else if (cur.terminal()) {
                        std::deque<int> rest(1, ri);
                        while (!rest.empty()) {
                            int fi = rest.front();
                            rest.pop_front();
                            const Box& fnt = boxes[fi];
                            bool a2 = adjacent(fnt, cur);
                            if (!a2 && fnt.has_pts()) Wl.insert(pack(fnt.level, fnt.idx));
                            if (a2 && fnt.terminal() && fnt.has_pts()) U.insert(pack(fnt.level, fnt.idx));
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
    if (cur.terminal() && cur.has_pts()) U.insert(pack(cur.level, cur.idx));
    auto out = [&](const std::set<uint64_t>& s, std::vector<int>& v) {
        v.clear();
        for (uint64_t key : s) v.push_back(index_.at(key));
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
    auto classify = [&](int oi) {
        const Box& oth = boxes[oi];
        if (!oth.has_pts()) return;
        Pt3 diff = sub(cc, center(oth));
        double n = l2(diff);
        if (n >= threshold) {
            Pt3 u{{diff[0] / n, diff[1] / n, diff[2] / n}};
            cur.far[nml2dir(u, W)].push_back(oi);
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
    check(prm.ncell >= 1 && (prm.ncell & (prm.ncell - 1)) == 0, "ncell must be a power of two");
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
        check(index_.emplace(pack(level, idx), bi).second, "duplicate box");
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
            for (int ind = 0; ind < 8; ++ind)
                add(level + 1, Idx3{{2 * base[0] + ((ind & 4) >> 2), 2 * base[1] + ((ind & 2) >> 1), 2 * base[2] + (ind & 1)}},
                    std::move(cp[ind]));
        } else {
            boxes[bi].tag |= TAG_TERMINAL;
        }
    }
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
    const double eps = 1e-12;
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
    for (size_t l = 0; l + 1 < lv.size(); ++l)
        parallel_for(lv[l + 1] - lv[l], [&](size_t i) {
            Box& cur = boxes[order[lv[l] + i]];
            double W = width(cur.level);
            if (!(W > 1 - eps && cur.has_pts())) return;
            if (cur.level != lvlC) {
                int pi = find(cur.level - 1, Idx3{{cur.idx[0] / 2, cur.idx[1] / 2, cur.idx[2] / 2}});
                check(pi >= 0, "missing parent");
                for (const Idx3& d : boxes[pi].outdirs) cur.outdirs.insert(parent_dir(d));
                for (const Idx3& d : boxes[pi].incdirs) cur.incdirs.insert(parent_dir(d));
            }
            Pt3 cc = center(cur);
            for (auto& kv : cur.far) {
                // the incoming direction of every far box is its key: highlist classified
                // (cc - oc) / |cc - oc| with the same arithmetic
                cur.incdirs.insert(kv.first);
                for (int oi : kv.second) {
                    Pt3 t = sub(center(boxes[oi]), cc);
                    double nt = l2(t);
                    for (int d = 0; d < 3; ++d) t[d] /= nt;
                    cur.outdirs.insert(nml2dir(t, W));
                }
            }
        });
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
