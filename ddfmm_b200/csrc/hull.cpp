// Extreme points of a 3-D point set (hull.hpp).
#include "hull.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <stdexcept>
#include <unordered_map>

namespace ddfmm {

namespace {
struct V3 {
    double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

struct Face {
    int v[3];
    V3 n;      // outward unit normal
    double d;  // plane n.x = d
    bool alive;
};

inline uint64_t edge_key(int a, int b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }
}  // namespace

std::vector<int> hull_vertices(const std::vector<double>& pts) {
    const int n = (int)(pts.size() / 3);
    if (n < 4) throw std::invalid_argument("convex hull needs at least 4 points");
    auto P = [&](int i) { return V3{pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2]}; };
    V3 lo = P(0), hi = P(0);
    for (int i = 1; i < n; ++i) {
        const V3 p = P(i);
        lo = V3{std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
        hi = V3{std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
    }
    const double scale = norm(sub(hi, lo));
    if (!(scale > 0)) throw std::invalid_argument("convex hull of coincident points");
    const double eps = 1e-11 * scale;

    // initial tetrahedron: min-x point, the point farthest from it, the point
    // farthest from their line, the point farthest from their plane
    int i0 = 0;
    for (int i = 1; i < n; ++i)
        if (P(i).x < P(i0).x) i0 = i;
    int i1 = -1;
    double best = -1;
    for (int i = 0; i < n; ++i) {
        const double d = norm(sub(P(i), P(i0)));
        if (d > best) best = d, i1 = i;
    }
    const V3 e01 = sub(P(i1), P(i0));
    int i2 = -1;
    best = -1;
    for (int i = 0; i < n; ++i) {
        const double d = norm(cross(e01, sub(P(i), P(i0))));
        if (d > best) best = d, i2 = i;
    }
    if (best <= eps * norm(e01)) throw std::invalid_argument("convex hull of collinear points");
    const V3 n012 = cross(e01, sub(P(i2), P(i0)));
    int i3 = -1;
    best = -1;
    for (int i = 0; i < n; ++i) {
        const double d = std::abs(dot(n012, sub(P(i), P(i0))));
        if (d > best) best = d, i3 = i;
    }
    if (best <= eps * norm(n012)) throw std::invalid_argument("convex hull of coplanar points");
    const V3 c0 = P(i0), c1 = P(i1), c2 = P(i2), c3 = P(i3);
    const V3 inside{(c0.x + c1.x + c2.x + c3.x) / 4, (c0.y + c1.y + c2.y + c3.y) / 4, (c0.z + c1.z + c2.z + c3.z) / 4};

    std::vector<Face> faces;
    std::unordered_map<uint64_t, int> edge;  // directed edge -> face holding it
    auto make_face = [&](int a, int b, int c) {
        Face f;
        f.v[0] = a;
        f.v[1] = b;
        f.v[2] = c;
        V3 nn = cross(sub(P(b), P(a)), sub(P(c), P(a)));
        const double len = norm(nn);
        nn = V3{nn.x / len, nn.y / len, nn.z / len};
        f.n = nn;
        f.d = dot(nn, P(a));
        f.alive = true;
        const int id = (int)faces.size();
        faces.push_back(f);
        edge[edge_key(a, b)] = id;
        edge[edge_key(b, c)] = id;
        edge[edge_key(c, a)] = id;
        return id;
    };
    {
        // orient the four faces outward
        const int t[4][3] = {{i0, i1, i2}, {i0, i3, i1}, {i1, i3, i2}, {i2, i3, i0}};
        const bool flip = dot(cross(sub(c1, c0), sub(c2, c0)), sub(c3, c0)) > 0;
        for (auto& f : t) {
            if (flip)
                make_face(f[0], f[2], f[1]);
            else
                make_face(f[0], f[1], f[2]);
        }
    }
    // the rest, farthest from the interior point first (fewer points on faces
    // or edges become provisional vertices)
    std::vector<int> order;
    order.reserve(n);
    for (int i = 0; i < n; ++i)
        if (i != i0 && i != i1 && i != i2 && i != i3) order.push_back(i);
    std::vector<double> dist(n);
    for (int i = 0; i < n; ++i) dist[i] = norm(sub(P(i), inside));
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dist[a] > dist[b]; });

    std::vector<int> visible;
    std::vector<std::pair<int, int> > horizon;
    int nalive = 4;
    for (int p : order) {
        const V3 x = P(p);
        visible.clear();
        for (int f = 0; f < (int)faces.size(); ++f)
            if (faces[f].alive && dot(faces[f].n, x) - faces[f].d > eps) visible.push_back(f);
        if (visible.empty()) continue;
        for (int f : visible) faces[f].alive = false;
        horizon.clear();
        for (int f : visible)
            for (int k = 0; k < 3; ++k) {
                const int a = faces[f].v[k], b = faces[f].v[(k + 1) % 3];
                auto it = edge.find(edge_key(b, a));
                if (it == edge.end()) throw std::logic_error("convex hull: open surface");
                if (faces[it->second].alive) horizon.push_back(std::make_pair(a, b));
            }
        for (int f : visible)
            for (int k = 0; k < 3; ++k) {
                auto it = edge.find(edge_key(faces[f].v[k], faces[f].v[(k + 1) % 3]));
                if (it != edge.end() && it->second == f) edge.erase(it);
            }
        nalive -= (int)visible.size();
        for (auto& h : horizon) make_face(h.first, h.second, p);
        nalive += (int)horizon.size();
        if ((int)faces.size() > 4 * nalive + 64) {  // drop dead faces
            std::vector<Face> keep;
            keep.reserve(nalive);
            edge.clear();
            for (const Face& f : faces)
                if (f.alive) {
                    const int id = (int)keep.size();
                    keep.push_back(f);
                    edge[edge_key(f.v[0], f.v[1])] = id;
                    edge[edge_key(f.v[1], f.v[2])] = id;
                    edge[edge_key(f.v[2], f.v[0])] = id;
                }
            faces.swap(keep);
        }
    }
    // extreme points: hull vertices whose incident normals span three dimensions
    std::vector<std::vector<int> > inc(n);
    for (int f = 0; f < (int)faces.size(); ++f)
        if (faces[f].alive)
            for (int k = 0; k < 3; ++k) inc[faces[f].v[k]].push_back(f);
    const double ang = 1e-9;
    std::vector<int> out;
    for (int i = 0; i < n; ++i) {
        const auto& fs = inc[i];
        if (fs.size() < 3) continue;
        const V3 a = faces[fs[0]].n;
        V3 ab{0, 0, 0};
        bool two = false, three = false;
        for (size_t k = 1; k < fs.size() && !two; ++k) {
            ab = cross(a, faces[fs[k]].n);
            two = norm(ab) > ang;
        }
        if (!two) continue;
        for (size_t k = 1; k < fs.size() && !three; ++k) three = std::abs(dot(ab, faces[fs[k]].n)) > ang * norm(ab);
        if (three) out.push_back(i);
    }
    return out;
}

}  // namespace ddfmm
