// FP64 translation-operator precompute (precompute.hpp).
#include "precompute.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <mutex>
#include <numeric>
#include <set>
#include <stdexcept>
#include <thread>

#include "dense.hpp"
#include "hull.hpp"

namespace ddfmm {
namespace precompute {

namespace {
constexpr double kTwoPi = 6.283185307179586;  // TPK = 2*pi (aug3d_lowdata.m:20)

// ---------------------------------------------------------------- random numbers
inline uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// xoshiro256** (Blackman and Vigna), doubles in [0, 1) from the top 53 bits
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        for (auto& w : s) w = splitmix64(seed);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// MATLAB sort(ceil(rand(1,n)*(total-n))) + [1:n], as 0-based indices
// (aug3d_hghdata.m:189,206,225,232): n distinct sorted indices in [0, total)
std::vector<int> sample_sorted(Rng& rng, int n, int total) {
    std::vector<long long> r(n);
    for (int k = 0; k < n; ++k) r[k] = (long long)std::ceil(rng.uniform() * (double)(total - n));
    std::sort(r.begin(), r.end());
    std::vector<int> out(n);
    for (int k = 0; k < n; ++k) out[k] = (int)(r[k] + k);
    return out;
}

std::vector<int> sorted_union(std::initializer_list<const std::vector<int>*> parts) {
    std::vector<int> u;
    for (const auto* p : parts) u.insert(u.end(), p->begin(), p->end());
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    return u;
}

// ---------------------------------------------------------------- point sets
inline double px(const PMat& p, int k, int d) { return p.x[3 * (size_t)k + d]; }

PMat make_pmat(int n) {
    PMat p;
    p.n = n;
    p.x.assign(3 * (size_t)n, 0.0);
    return p;
}

PMat cols(const PMat& p, const std::vector<int>& idx) {
    PMat q = make_pmat((int)idx.size());
    for (size_t k = 0; k < idx.size(); ++k)
        for (int d = 0; d < 3; ++d) q.x[3 * k + d] = px(p, idx[k], d);
    return q;
}

PMat concat(const std::vector<const PMat*>& parts) {
    PMat q;
    for (const PMat* p : parts) {
        q.x.insert(q.x.end(), p->x.begin(), p->x.end());
        q.n += p->n;
    }
    return q;
}

PMat shifted(const PMat& p, double sx, double sy, double sz) {
    PMat q = p;
    for (int k = 0; k < p.n; ++k) {
        q.x[3 * (size_t)k] = px(p, k, 0) + sx;
        q.x[3 * (size_t)k + 1] = px(p, k, 1) + sy;
        q.x[3 * (size_t)k + 2] = px(p, k, 2) + sz;
    }
    return q;
}

PMat negated(const PMat& p) {
    PMat q = p;
    for (double& v : q.x) v = -v;
    return q;
}

// MATLAB unique(pts', 'rows')': distinct points sorted by x, then y, then z
PMat unique_rows(const PMat& p) {
    std::vector<int> o(p.n);
    std::iota(o.begin(), o.end(), 0);
    auto less = [&](int a, int b) {
        for (int d = 0; d < 3; ++d) {
            if (px(p, a, d) < px(p, b, d)) return true;
            if (px(p, b, d) < px(p, a, d)) return false;
        }
        return false;
    };
    std::sort(o.begin(), o.end(), less);
    std::vector<int> keep;
    for (size_t i = 0; i < o.size(); ++i)
        if (i == 0 || less(o[i - 1], o[i])) keep.push_back(o[i]);
    return cols(p, keep);
}

// ndgrid([-h h]) offsets, x fastest (aug3d_hghdata.m:94-96,120)
void corner_offset(int t, double h, double out[3]) {
    out[0] = (t & 1) ? h : -h;
    out[1] = (t & 2) ? h : -h;
    out[2] = (t & 4) ? h : -h;
}

// wedge coordinates of unit vectors (aug3d_hghdata_dir.m)
void wedge_coords(const double u[3], int C, double out[3]) {
    const double t = std::max(std::abs(u[0]), std::max(std::abs(u[1]), std::abs(u[2])));
    for (int d = 0; d < 3; ++d) out[d] = std::atan(u[d] / t) / (M_PI / 4) * C;
}

// 3-D DFT (forward, e^{-2 pi i jk/G}, unnormalised) of a G^3 tensor, x fastest
void fft3(std::vector<cpx>& a, int G) {
    std::vector<cpx> w(G), line(G), outl(G);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < G; ++m) {
        const long double ang = -twopi * (long double)m / (long double)G;
        w[m] = cpx((double)cosl(ang), (double)sinl(ang));
    }
    const size_t stride[3] = {1, (size_t)G, (size_t)G * G};
    for (int ax = 0; ax < 3; ++ax) {
        const size_t st = stride[ax];
        for (size_t base = 0; base < (size_t)G * G * G; ++base) {
            if ((base / st) % G != 0) continue;  // start of a line along this axis
            for (int j = 0; j < G; ++j) line[j] = a[base + j * st];
            for (int k = 0; k < G; ++k) {
                cpx s(0, 0);
                for (int j = 0; j < G; ++j) s += line[j] * w[(size_t)j * k % G];
                outl[k] = s;
            }
            for (int k = 0; k < G; ++k) a[base + k * st] = outl[k];
        }
    }
}

struct HfParams {
    double eps;
    int rr, rt, nt;
};
// aug3d_hghdata.m:47-54
HfParams hf_params(int accu) {
    switch (accu) {
        case 1: return HfParams{1e-4, 70, 4, 2400};
        case 2: return HfParams{1e-6, 120, 5, 2400};
        case 3: return HfParams{1e-8, 160, 6, 4800};
    }
    throw std::invalid_argument("ACCU must be 1, 2 or 3");
}

// Run job(i) for i in [0, n) on up to `threads` host threads; rethrows the first failure.
void parallel_for(int n, int threads, const std::function<void(int)>& job) {
    const int nt = std::max(1, std::min(threads, n));
    std::atomic<int> next(0);
    std::exception_ptr err;
    std::mutex mu;
    auto worker = [&] {
        for (;;) {
            const int i = next++;
            if (i >= n) return;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (err) return;
            }
            try {
                job(i);
            } catch (...) {
                std::lock_guard<std::mutex> lk(mu);
                if (!err) err = std::current_exception();
            }
        }
    };
    if (nt == 1) {
        worker();
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(worker);
        for (auto& x : th) x.join();
    }
    if (err) std::rethrow_exception(err);
}

int host_threads(int threads) {
    if (threads > 0) return threads;
    const unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}
}  // namespace

int accu_to_p(int accu) {
    switch (accu) {
        case 1: return 4;
        case 2: return 6;
        case 3: return 8;
    }
    throw std::invalid_argument("ACCU must be 1, 2 or 3");
}

CMat kernel_matrix(const PMat& trg, const PMat& src, int kind) {
    if (kind != 0 && kind != 1) throw std::invalid_argument("unknown kernel type");
    CMat M = dense::zeros(trg.n, src.n);
    for (int j = 0; j < src.n; ++j) {
        const double sx = px(src, j, 0), sy = px(src, j, 1), sz = px(src, j, 2);
        cpx* col = &M(0, j);
        for (int i = 0; i < trg.n; ++i) {
            const double x = px(trg, i, 0) - sx, y = px(trg, i, 1) - sy, z = px(trg, i, 2) - sz;
            const double r = std::sqrt(x * x + y * y + z * z);
            double sn, cs;
            sincos(kTwoPi * r, &sn, &cs);
            col[i] = kind == 0 ? cpx(cs / r, sn / r) : cpx(cs, sn);
        }
    }
    return M;
}

PMat surface_grid(double L, int P) {
    std::vector<double> v(P);
    const double step = L / (P - 1);
    for (int i = 0; i < P; ++i) v[i] = (double)i * step + (-L / 2);
    v[0] = -L / 2;
    v[P - 1] = L / 2;
    PMat p;
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) {
                const double q[3] = {v[i], v[j], v[k]};
                const double mx = std::max(std::abs(q[0]), std::max(std::abs(q[1]), std::abs(q[2])));
                if (mx == L / 2) {
                    p.x.insert(p.x.end(), q, q + 3);
                    p.n++;
                }
            }
    return p;
}

LowFreqOp low_entry(int accu, double W, int kind) {
    const int P = accu_to_p(accu), G = 2 * P;
    LowFreqOp op;
    op.W = W;
    op.uep = surface_grid(W, P);
    op.ucp = surface_grid(3 * W, P);
    // pseudo-inverse of the check-to-equivalent map (aug3d_lowdata.m:55-61)
    const CMat M = kernel_matrix(op.ucp, op.uep, kind);
    CMat U, V;
    std::vector<double> s;
    dense::svd(M, U, s, V);
    int r = 0;
    while (r < (int)s.size() && s[r] > 1e-16 * s[0]) ++r;
    const int nE = op.uep.n;
    op.v = dense::zeros(nE, r);
    op.is = dense::zeros(r, 1);
    op.up = dense::zeros(r, nE);
    for (int k = 0; k < r; ++k) {
        op.is(k, 0) = cpx(1.0 / s[k], 0.0);
        for (int i = 0; i < nE; ++i) {
            op.v(i, k) = V(i, k);
            op.up(k, i) = std::conj(U(i, k));
        }
    }
    // FFT'd translation tensors of the 316 well-separated offsets (aug3d_lowdata.m:81-105)
    const double step = W / (P - 1);
    std::vector<double> t(G);
    for (int i = 0; i < G; ++i) t[i] = (double)(i < P ? i : i - G) * step;
    op.ue2dc.assign(343, std::vector<cpx>());
    op.tdim = G;
    for (int c = 0; c < 7; ++c)
        for (int b = 0; b < 7; ++b)
            for (int a = 0; a < 7; ++a) {
                const int sa = a - 3, sb = b - 3, sc = c - 3;
                if (std::abs(sa) <= 1 && std::abs(sb) <= 1 && std::abs(sc) <= 1) continue;
                std::vector<cpx> tns((size_t)G * G * G);
                for (int z = 0; z < G; ++z)
                    for (int y = 0; y < G; ++y)
                        for (int x = 0; x < G; ++x) {
                            const double X = t[x] + sa * W, Y = t[y] + sb * W, Z = t[z] + sc * W;
                            const double rr = std::sqrt(X * X + Y * Y + Z * Z);
                            double sn, cs;
                            sincos(kTwoPi * rr, &sn, &cs);
                            tns[x + (size_t)G * (y + (size_t)G * z)] = kind == 0 ? cpx(cs / rr, sn / rr) : cpx(cs, sn);
                        }
                fft3(tns, G);
                op.ue2dc[a + 7 * b + 49 * c] = std::move(tns);
            }
    return op;
}

Idx3 predir(const Idx3& n) {
    const int C = std::max(std::abs(n[0]), std::max(std::abs(n[1]), std::abs(n[2])));
    auto fdiv = [](int a, int b) {  // floor(a / b), b > 0
        return a >= 0 ? a / b : -((-a + b - 1) / b);
    };
    Idx3 r;
    for (int d = 0; d < 3; ++d) {
        const int q = fdiv(n[d] + C - 1, 2);
        r[d] = 2 * fdiv(q, 2) + 1 - C / 2;
    }
    r[2] = n[2] / 2;
    return r;
}

uint64_t wedge_seed(int kind, int accu, double W, const Idx3& n) {
    uint64_t bits;
    std::memcpy(&bits, &W, 8);
    uint64_t h = 0x6464666d6d2d6866ull;  // a fixed start
    uint64_t x = h ^ (uint64_t)kind;
    h = splitmix64(x);
    x = h ^ (uint64_t)accu;
    h = splitmix64(x);
    x = h ^ bits;
    h = splitmix64(x);
    for (int d = 0; d < 3; ++d) {
        x = h ^ (uint64_t)(uint32_t)n[d];
        h = splitmix64(x);
    }
    return h;
}

HighFreqOp high_wedge(int accu, double W, int kind, const Idx3& n, const PMat& pspre, const PMat& ptpre,
                      uint64_t seed) {
    const HfParams hp = hf_params(accu);
    Rng rng(seed);
    const double D = W * W + W, DP = (2 * W) * (2 * W) + 2 * W;
    const int C = (int)std::lround(4 * W);
    // far-field box centres in the positive octant with D <= |c| <= 5D (aug3d_hghdata.m:27-33)
    const int nt = (int)std::floor(5 * D / W + 1e-9) + 1;
    std::vector<double> tmp(nt);
    for (int i = 0; i < nt; ++i) tmp[i] = (double)i * W;
    PMat sfts;
    for (int k = 0; k < nt; ++k)
        for (int j = 0; j < nt; ++j)
            for (int i = 0; i < nt; ++i) {
                const double q[3] = {tmp[i], tmp[j], tmp[k]};
                const double sr = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                if (sr >= D - 1e-8 && sr <= 5 * D) {
                    sfts.x.insert(sfts.x.end(), q, q + 3);
                    sfts.n++;
                }
            }
    // the children's source and target collections (aug3d_hghdata.m:94-108)
    std::vector<PMat> parts_s, parts_t;
    for (int t = 0; t < 8; ++t) {
        double o[3];
        corner_offset(t, W / 4, o);
        parts_s.push_back(shifted(pspre, o[0], o[1], o[2]));
        parts_t.push_back(shifted(ptpre, o[0], o[1], o[2]));
    }
    std::vector<const PMat*> ps_parts, pt_parts;
    for (int t = 0; t < 8; ++t) {
        ps_parts.push_back(&parts_s[t]);
        pt_parts.push_back(&parts_t[t]);
    }
    const PMat ps = unique_rows(concat(ps_parts));
    const PMat ptcol = unique_rows(concat(pt_parts));
    const std::vector<int> salw = hull_vertices(ps.x);  // (:112-113)
    // far-field centres in this wedge and the boxes around them (:116-127)
    const double tol = 1.0 + 1e-8;
    std::vector<int> good;
    for (int k = 0; k < sfts.n; ++k) {
        const double r = std::sqrt(px(sfts, k, 0) * px(sfts, k, 0) + px(sfts, k, 1) * px(sfts, k, 1) +
                                   px(sfts, k, 2) * px(sfts, k, 2));
        const double u[3] = {px(sfts, k, 0) / r, px(sfts, k, 1) / r, px(sfts, k, 2) / r};
        double w[3];
        wedge_coords(u, C, w);
        if (std::abs(w[0] - n[0]) <= tol && std::abs(w[1] - n[1]) <= tol && std::abs(w[2] - n[2]) <= 1e-8)
            good.push_back(k);
    }
    if (good.empty()) throw std::runtime_error("wedge has no far-field centres");
    const PMat sss = cols(sfts, good);
    PMat play;
    std::vector<double> dis(sss.n);
    for (int k = 0; k < sss.n; ++k) {
        const double c[3] = {px(sss, k, 0), px(sss, k, 1), px(sss, k, 2)};
        dis[k] = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        const double f = dis[k] < DP - 1e-8 ? 1.0 : 3.0;
        for (int t = 0; t < 8; ++t) {
            double o[3];
            corner_offset(t, W / 2, o);
            for (int d = 0; d < 3; ++d) play.x.push_back(f * o[d] + c[d]);
            play.n++;
        }
    }
    // targets: the hull of those boxes, the nearest children, random points in the cone (:128-175)
    const PMat pt0 = cols(play, hull_vertices(play.x));
    const double mindis = *std::min_element(dis.begin(), dis.end());
    std::vector<PMat> near;
    for (int k = 0; k < sss.n; ++k)
        if (dis[k] < mindis + 1e-8) near.push_back(shifted(ptcol, px(sss, k, 0), px(sss, k, 1), px(sss, k, 2)));
    std::vector<const PMat*> near_p;
    for (const PMat& q : near) near_p.push_back(&q);
    const PMat pt1 = unique_rows(concat(near_p));
    double tlo = 1e300, thi = -1e300, plo = 1e300, phi_hi = -1e300;
    for (int k = 0; k < play.n; ++k) {
        const double x = px(play, k, 0), y = px(play, k, 1), z = px(play, k, 2);
        const double r = std::sqrt(x * x + y * y + z * z);
        const double th = std::atan2(x / r, z / r), ph = std::atan2(y / r, z / r);
        tlo = std::min(tlo, th);
        thi = std::max(thi, th);
        plo = std::min(plo, ph);
        phi_hi = std::max(phi_hi, ph);
    }
    const double a = n[0], b = n[1];
    if (tlo > (a - 1) / C * M_PI / 4 || thi < (a + 1) / C * M_PI / 4 || plo > (b - 1) / C * M_PI / 4 ||
        phi_hi < (b + 1) / C * M_PI / 4)
        throw std::runtime_error("wedge sample cone does not cover the wedge");
    const double rlo = mindis - W / 2, rhi = 6 * D;
    std::vector<double> the(hp.nt), phi(hp.nt), rho(hp.nt);
    for (double& v : the) v = rng.uniform() * (thi - tlo) + tlo;
    for (double& v : phi) v = rng.uniform() * (phi_hi - plo) + plo;
    for (double& v : rho) v = rng.uniform() * (rhi - rlo) + rlo;
    PMat pt2 = make_pmat(hp.nt);
    for (int k = 0; k < hp.nt; ++k) {
        const double ta = std::tan(the[k]), tb = std::tan(phi[k]);
        const double t = std::sqrt(ta * ta + tb * tb + 1);
        pt2.x[3 * (size_t)k] = ta / t * rho[k];
        pt2.x[3 * (size_t)k + 1] = tb / t * rho[k];
        pt2.x[3 * (size_t)k + 2] = 1 / t * rho[k];
    }
    const PMat talw2 = cols(pt2, hull_vertices(pt2.x));
    const PMat pt = unique_rows(concat({&pt0, &pt1, &pt2}));
    const PMat talw_pts = unique_rows(concat({&pt0, &pt1, &talw2}));
    // indices of talw_pts inside pt (MATLAB intersect(..., 'rows')): both are sorted
    std::vector<int> talw;
    {
        auto cmp = [](const PMat& p, int i, const PMat& q, int j) {
            for (int d = 0; d < 3; ++d) {
                if (px(p, i, d) < px(q, j, d)) return -1;
                if (px(q, j, d) < px(p, i, d)) return 1;
            }
            return 0;
        };
        int i = 0, j = 0;
        while (i < pt.n && j < talw_pts.n) {
            const int c = cmp(pt, i, talw_pts, j);
            if (c == 0) {
                talw.push_back(i);
                ++i;
                ++j;
            } else if (c < 0) {
                ++i;
            } else {
                ++j;
            }
        }
    }
    // randomised pivoted-QR skeletons (aug3d_hghdata.m:179-218)
    const int M = pt.n, N = ps.n;
    const int sz1 = hp.rr * hp.rt, sz2 = hp.rr * hp.rt * hp.rt;
    std::vector<int> all_m(M), all_n(N);
    std::iota(all_m.begin(), all_m.end(), 0);
    std::iota(all_n.begin(), all_n.end(), 0);
    const int nr1 = (int)std::lround(sz1 * std::sqrt((double)M / N));
    std::vector<int> rs = nr1 > M ? all_m : sample_sorted(rng, nr1, M);
    rs = sorted_union({&rs, &talw});
    std::vector<int> idx1;
    {
        const CMat M1 = kernel_matrix(cols(pt, rs), ps, kind);
        idx1 = dense::qr_pivoted(M1, hp.eps);
    }
    const PMat psidx = cols(ps, idx1);
    CMat Q1, R1;
    dense::qr(kernel_matrix(pt, psidx, kind), Q1, R1);
    std::vector<int> cs = sz1 > N ? all_n : sample_sorted(rng, sz1, N);
    cs = sorted_union({&cs, &salw, &idx1});
    std::vector<int> idx2;
    {
        CMat M2h;
        {
            const CMat M2 = kernel_matrix(pt, cols(ps, cs), kind);
            M2h = dense::conj_transpose(M2);
        }
        idx2 = dense::qr_pivoted(std::move(M2h), hp.eps);
    }
    const PMat ptidx = cols(pt, idx2);
    CMat Q2, R2;
    dense::qr(dense::conj_transpose(kernel_matrix(ptidx, ps, kind)), Q2, R2);
    // middle factor G = pinv(Q1(rs,:)) M3 pinv(Q2(cs,:)') (aug3d_hghdata.m:220-238)
    std::vector<int> cs3 = sz2 > N ? all_n : sample_sorted(rng, sz2, N);
    cs3 = sorted_union({&idx1, &cs3});
    std::vector<int> rs3 = sz2 > M ? all_m : sample_sorted(rng, sz2, M);
    rs3 = sorted_union({&idx2, &rs3});
    const CMat B1 = dense::pinv(dense::take_rows(Q1, rs3));                              // r1 x |rs3|
    const CMat C2 = dense::pinv(dense::conj_transpose(dense::take_rows(Q2, cs3)));      // |cs3| x r2
    const int r1 = (int)idx1.size(), r2 = (int)idx2.size();
    if (r1 > 400 || r2 > 400) throw std::runtime_error("skeleton rank exceeds DVMAX=400 (src/wave3d_eval.cpp:25)");
    const PMat prs = cols(pt, rs3);
    CMat X = dense::zeros(r1, (int)cs3.size());  // B1 M3, M3 generated a column block at a time
    constexpr int CB = 128;
    for (int c0 = 0; c0 < (int)cs3.size(); c0 += CB) {
        const int c1 = std::min((int)cs3.size(), c0 + CB);
        std::vector<int> blk(cs3.begin() + c0, cs3.begin() + c1);
        const CMat M3 = kernel_matrix(prs, cols(ps, blk), kind);
        const CMat Xb = dense::gemm(B1, false, M3, false);
        std::memcpy(&X(0, c0), Xb.a.data(), sizeof(cpx) * Xb.a.size());
    }
    HighFreqOp op;
    op.uep = psidx;
    op.ucp = ptidx;
    op.E1 = dense::inv_triangular(R1);
    op.E2 = dense::gemm(X, false, C2, false);
    op.E3 = dense::inv_triangular(dense::conj_transpose(R2), true);
    return op;
}

std::map<double, LowFreqOp> low_levels(int accu, int kind, int threads) {
    std::vector<LowFreqOp> out(7);
    parallel_for(7, host_threads(threads), [&](int i) { out[i] = low_entry(accu, std::ldexp(1.0, i - 7), kind); });
    std::map<double, LowFreqOp> ld;
    for (auto& e : out) ld[e.W] = std::move(e);
    return ld;
}

std::map<double, std::map<Idx3, HighFreqOp> > high_levels(int accu, int kind, int wmax, int threads,
                                                         const std::function<void(double, int, int)>& progress) {
    if (wmax < 1) throw std::invalid_argument("wmax must be >= 1");
    const int P = accu_to_p(accu);
    std::map<double, std::map<Idx3, HighFreqOp> > hd;
    const std::map<Idx3, HighFreqOp>* prev = nullptr;
    for (int Wi = 1; Wi <= wmax; Wi *= 2) {
        const double W = Wi;
        const int C = 4 * Wi;  // NPQ = 4 wedges per quadrant (aug3d_script.m:55)
        std::set<Idx3> uns;    // (aug3d_hghdata.m:42-45)
        for (int x = 1; x < C; x += 2)
            for (int y = 1; y < C; y += 2) {
                Idx3 t{{x, y, C}};
                std::sort(t.begin(), t.end());
                uns.insert(t);
            }
        const std::vector<Idx3> wedges(uns.begin(), uns.end());
        std::vector<HighFreqOp> res(wedges.size());
        const PMat pg = surface_grid(W / 2, P);  // W = 1: the low-frequency surface of the children (:63-78)
        std::atomic<int> done(0);
        std::mutex pmu;
        parallel_for((int)wedges.size(), host_threads(threads), [&](int i) {
            const Idx3& n = wedges[i];
            if (Wi == 1) {
                res[i] = high_wedge(accu, W, kind, n, pg, pg, wedge_seed(kind, accu, W, n));
            } else {
                auto it = prev->find(predir(n));  // (:80-90)
                if (it == prev->end()) throw std::logic_error("parent wedge missing from the previous width");
                res[i] = high_wedge(accu, W, kind, n, it->second.uep, negated(it->second.uep),
                                    wedge_seed(kind, accu, W, n));
            }
            const int d = ++done;
            if (progress) {
                std::lock_guard<std::mutex> lk(pmu);
                progress(W, d, (int)wedges.size());
            }
        });
        auto& lvl = hd[W];
        for (size_t i = 0; i < wedges.size(); ++i) lvl[wedges[i]] = std::move(res[i]);
        prev = &lvl;
    }
    return hd;
}

// ---------------------------------------------------------------- writers
namespace {
struct Out {
    std::ofstream f;
    std::string path;
    explicit Out(const std::string& p) : f(p, std::ios::binary), path(p) {
        if (!f) throw std::runtime_error("cannot write " + p);
    }
    void i32(int v) { f.write(reinterpret_cast<const char*>(&v), 4); }
    void f64(double v) { f.write(reinterpret_cast<const char*>(&v), 8); }
    void pmat(const PMat& p) {
        i32(3);
        i32(p.n);
        f.write(reinterpret_cast<const char*>(p.x.data()), 8 * p.x.size());
    }
    void cmat(const CMat& c) {
        i32(c.m);
        i32(c.n);
        f.write(reinterpret_cast<const char*>(c.a.data()), 16 * c.a.size());
    }
    void ctns(const std::vector<cpx>& t, int edge) {
        const int e = t.empty() ? 0 : edge;
        i32(e);
        i32(e);
        i32(e);
        f.write(reinterpret_cast<const char*>(t.data()), 16 * t.size());
    }
    void close() {
        f.close();
        if (!f) throw std::runtime_error("write failed: " + path);
    }
};
}  // namespace

// map<double, {DblNumMat uep, DblNumMat ucp, NumVec<CpxNumMat> uc2ue, NumTns<CpxNumTns> ue2dc}>
// (aug3d_script.m:35-50, read by src/mlib3d.cpp:361-379)
void write_ld(const std::string& path, const std::map<double, LowFreqOp>& ld) {
    Out o(path);
    o.i32((int)ld.size());
    for (const auto& kv : ld) {
        const LowFreqOp& e = kv.second;
        o.f64(kv.first);
        o.pmat(e.uep);
        o.pmat(e.ucp);
        o.i32(3);
        o.cmat(e.v);
        o.cmat(e.is);
        o.cmat(e.up);
        o.i32(7);
        o.i32(7);
        o.i32(7);
        for (int i = 0; i < 343; ++i) o.ctns(e.ue2dc[i], e.tdim);
    }
    o.close();
}

// map<double, map<Index3, {DblNumMat uep, DblNumMat ucp, NumVec<CpxNumMat> uc2ue}>>
// (aug3d_script.m:70-85, read by src/mlib3d.cpp:382-405)
void write_hd(const std::string& path, const std::map<double, std::map<Idx3, HighFreqOp> >& hd) {
    Out o(path);
    o.i32((int)hd.size());
    for (const auto& kv : hd) {
        o.f64(kv.first);
        o.i32((int)kv.second.size());
        for (const auto& dk : kv.second) {
            for (int d = 0; d < 3; ++d) o.i32(dk.first[d]);
            o.pmat(dk.second.uep);
            o.pmat(dk.second.ucp);
            o.i32(3);
            o.cmat(dk.second.E1);
            o.cmat(dk.second.E2);
            o.cmat(dk.second.E3);
        }
    }
    o.close();
}

}  // namespace precompute
}  // namespace ddfmm
