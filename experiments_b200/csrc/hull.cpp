// Convex-hull polyhedral features for registration (host side).
//
// Behaviour follows btConvexUtility::initializePolyhedralFeatures and
// ::initialize (P1/btConvexUtility.cpp:31-270, 339-513) over the hull that
// bullet2's btConvexHullComputer returns for the same points:
//   * the points are quantised to btConvexHullComputer's integer grid
//     (btConvexHullInternal::compute, bullet2/LinearMath/
//     btConvexHullComputer.cpp:1940-2030: per-axis extent / 10216, axes
//     ordered medium, largest, smallest, coordinates truncated toward zero)
//     and the hull is computed exactly on the grid points; its vertices are
//     the grid points mapped back (getCoordinates, :2075-2082: point *
//     scaling + center, in float), so they sit where the reference's do;
//   * faces are the hull's maximal planar polygons, wound counter-clockwise
//     seen from outside; each face's plane is computed from its first two
//     normalised edges and its lowest vertex in float, as btConvexUtility
//     does (:56-108);
//   * faces whose normals agree to dot > 0.999 (in float) are welded into
//     one polygon (2D hull of their points, plane of the group's reference
//     face), unless a dropped point is used by a face outside the group;
//   * unique edge directions: normalised (v[smaller] - v[larger]) deduped
//     by +/- within 1e-6 per component;
//   * local centre = average of the hull vertices
//     (CLPhysicsDemo::registerConvexPolyhedron, P2/CLPhysicsDemo.cpp:360-366).
// The hull itself is this file's own incremental construction with exact
// 64-bit integer predicates on the grid (O(points x faces)); vertices are
// listed in the order of their first input point, faces by their vertex
// indices (the reference lists both in its hull traversal order).
#include "hull.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <numeric>
#include <unordered_map>

namespace b3hull {

namespace {

struct V3 {
    double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double len(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 norm(V3 a) {
    double l = len(a);
    return l > 0 ? mul(a, 1.0 / l) : a;
}

// float vector arithmetic in btVector3's operation order
struct F3 {
    float x, y, z;
};
inline F3 fsub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 fcross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline F3 fnormalized(F3 a) {
    // btVector3::normalize: *this /= length(), the division as a multiply
    // by the reciprocal
    const float r = 1.f / std::sqrt(fdot(a, a));
    return {a.x * r, a.y * r, a.z * r};
}

// ---------------------------------------------------------------------------
// btConvexHullComputer's integer grid
// ---------------------------------------------------------------------------
struct Grid {
    int medAxis = 0, maxAxis = 0, minAxis = 0;
    float scaling[3] = {0, 0, 0}, center[3] = {0, 0, 0}, inv[3] = {0, 0, 0};
};

Grid make_grid(const float* p, int n) {
    Grid g;
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            const float v = p[3 * i + k];
            if (v < mn[k]) mn[k] = v;   // btSetMin
            if (mx[k] < v) mx[k] = v;   // btSetMax
        }
    float s[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    // btVector3::maxAxis / minAxis (bullet2/LinearMath/btVector3.h:453-463)
    g.maxAxis = s[0] < s[1] ? (s[1] < s[2] ? 2 : 1) : (s[0] < s[2] ? 2 : 0);
    g.minAxis = s[0] < s[1] ? (s[0] < s[2] ? 0 : 2) : (s[1] < s[2] ? 1 : 2);
    if (g.minAxis == g.maxAxis) g.minAxis = (g.maxAxis + 1) % 3;
    g.medAxis = 3 - g.maxAxis - g.minAxis;
    const volatile float div = 10216.f;
    const float r = 1.f / div;  // s /= 10216: a multiply by the reciprocal
    for (int k = 0; k < 3; ++k) s[k] *= r;
    if (((g.medAxis + 1) % 3) != g.maxAxis)
        for (int k = 0; k < 3; ++k) s[k] *= -1.f;
    for (int k = 0; k < 3; ++k) {
        g.scaling[k] = s[k];
        g.inv[k] = s[k] != 0.f ? 1.f / s[k] : s[k];
        g.center[k] = (mn[k] + mx[k]) * 0.5f;
    }
    return g;
}

struct IV {
    int64_t x, y, z;
    bool operator==(const IV& o) const { return x == o.x && y == o.y && z == o.z; }
};
inline IV isub(IV a, IV b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline IV icross(IV a, IV b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline int64_t idot(IV a, IV b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// grid coordinates of one point: x along the medium axis, y the largest,
// z the smallest, truncated toward zero
IV quantize(const Grid& g, const float* p) {
    float q[3];
    for (int k = 0; k < 3; ++k) q[k] = (p[k] - g.center[k]) * g.inv[k];
    return {(int64_t)(int32_t)q[g.medAxis], (int64_t)(int32_t)q[g.maxAxis], (int64_t)(int32_t)q[g.minAxis]};
}

// the grid point mapped back: getCoordinates (p * scaling + center, float)
V3 dequantize(const Grid& g, IV v) {
    float p[3];
    p[g.medAxis] = (float)v.x;
    p[g.maxAxis] = (float)v.y;
    p[g.minAxis] = (float)v.z;
    float o[3];
    for (int k = 0; k < 3; ++k) o[k] = p[k] * g.scaling[k] + g.center[k];
    return {o[0], o[1], o[2]};
}

// ---------------------------------------------------------------------------
// Exact incremental hull of grid points (|coordinate| <= 2^13, so every
// cross product and plane test below is exact in 64-bit integers)
// ---------------------------------------------------------------------------
struct HTri {
    int a, b, c;
    IV n;       // outward normal (b - a) x (c - a)
    int64_t d;  // plane n . x = d
    bool alive;
};

HTri make_tri(const std::vector<IV>& Q, int a, int b, int c) {
    HTri t;
    t.a = a;
    t.b = b;
    t.c = c;
    t.n = icross(isub(Q[b], Q[a]), isub(Q[c], Q[a]));
    t.d = idot(t.n, Q[a]);
    t.alive = true;
    return t;
}

bool exact_hull(const std::vector<IV>& Q, std::vector<HTri>& tris) {
    const int m = (int)Q.size();
    tris.clear();
    if (m < 4) return false;
    // initial tetrahedron: farthest point, largest triangle, largest volume
    const int i0 = 0;
    int i1 = -1, i2 = -1, i3 = -1;
    int64_t best = 0;
    for (int j = 1; j < m; ++j) {
        const IV d = isub(Q[j], Q[i0]);
        const int64_t l2 = idot(d, d);
        if (l2 > best) best = l2, i1 = j;
    }
    if (i1 < 0) return false;
    best = 0;
    for (int j = 1; j < m; ++j) {
        const IV c = icross(isub(Q[i1], Q[i0]), isub(Q[j], Q[i0]));
        const int64_t l2 = idot(c, c);
        if (l2 > best) best = l2, i2 = j;
    }
    if (i2 < 0) return false;
    const IV nrm = icross(isub(Q[i1], Q[i0]), isub(Q[i2], Q[i0]));
    best = 0;
    for (int j = 1; j < m; ++j) {
        const int64_t v = idot(nrm, isub(Q[j], Q[i0]));
        const int64_t av = v < 0 ? -v : v;
        if (av > best) best = av, i3 = j;
    }
    if (i3 < 0) return false;
    if (idot(nrm, isub(Q[i3], Q[i0])) > 0) {
        tris.push_back(make_tri(Q, i0, i2, i1));
        tris.push_back(make_tri(Q, i0, i1, i3));
        tris.push_back(make_tri(Q, i1, i2, i3));
        tris.push_back(make_tri(Q, i2, i0, i3));
    } else {
        tris.push_back(make_tri(Q, i0, i1, i2));
        tris.push_back(make_tri(Q, i0, i3, i1));
        tris.push_back(make_tri(Q, i1, i3, i2));
        tris.push_back(make_tri(Q, i2, i3, i0));
    }
    // the remaining points in a fixed pseudo-random order (an odd-step walk
    // through the indices), which keeps the visible sets small on average
    std::vector<int> order;
    order.reserve(m);
    uint64_t step = 0x9E3779B97F4A7C15ull % (uint64_t)m;
    while (step == 0 || std::gcd(step, (uint64_t)m) != 1) step = (step + 1) % (uint64_t)m;
    for (uint64_t k = 0, j = 0; k < (uint64_t)m; ++k, j = (j + step) % (uint64_t)m)
        if ((int)j != i0 && (int)j != i1 && (int)j != i2 && (int)j != i3) order.push_back((int)j);
    std::vector<int> visible;
    std::vector<std::pair<int, int>> edges;
    int alive = 4;
    for (int p : order) {
        visible.clear();
        for (int t = 0; t < (int)tris.size(); ++t)
            if (tris[t].alive && idot(tris[t].n, Q[p]) > tris[t].d) visible.push_back(t);
        if (visible.empty()) continue;  // inside the hull or on its surface
        edges.clear();
        for (int t : visible) {
            edges.push_back({tris[t].a, tris[t].b});
            edges.push_back({tris[t].b, tris[t].c});
            edges.push_back({tris[t].c, tris[t].a});
            tris[t].alive = false;
        }
        alive -= (int)visible.size();
        std::vector<std::pair<int, int>> sorted = edges;
        std::sort(sorted.begin(), sorted.end());
        // horizon: edges of the visible region whose reverse is not in it;
        // each gets a new triangle to p with the visible face's winding
        for (const auto& e : edges)
            if (!std::binary_search(sorted.begin(), sorted.end(), std::make_pair(e.second, e.first))) {
                tris.push_back(make_tri(Q, e.first, e.second, p));
                ++alive;
            }
        if ((int)tris.size() > 4 * alive + 64) {
            std::vector<HTri> keep;
            keep.reserve(alive);
            for (const HTri& t : tris)
                if (t.alive) keep.push_back(t);
            tris.swap(keep);
        }
    }
    std::vector<HTri> keep;
    for (const HTri& t : tris)
        if (t.alive) keep.push_back(t);
    tris.swap(keep);
    return true;
}

int64_t gcd64(int64_t a, int64_t b) {
    a = a < 0 ? -a : a;
    b = b < 0 ? -b : b;
    while (b) {
        const int64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Vertices of one planar face, strictly convex and counter-clockwise about
// the outward normal n, by a monotone chain on the two axes other than n's
// largest component (exact).
std::vector<int> planar_polygon(const std::vector<IV>& Q, const std::vector<int>& ids, IV n) {
    const int64_t ax = std::llabs(n.x), ay = std::llabs(n.y), az = std::llabs(n.z);
    const int k = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    const int64_t nk = k == 0 ? n.x : (k == 1 ? n.y : n.z);
    auto coord = [&](const IV& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); };
    struct P2 {
        int64_t u, v;
        int id;
    };
    std::vector<P2> q;
    for (int id : ids) q.push_back({coord(Q[id], (k + 1) % 3), coord(Q[id], (k + 2) % 3), id});
    std::sort(q.begin(), q.end(), [](const P2& a, const P2& b) { return a.u < b.u || (a.u == b.u && a.v < b.v); });
    auto crs = [](const P2& o, const P2& a, const P2& b) { return (a.u - o.u) * (b.v - o.v) - (a.v - o.v) * (b.u - o.u); };
    std::vector<P2> h(2 * q.size() + 1);
    size_t t = 0;
    for (size_t i = 0; i < q.size(); ++i) {
        while (t >= 2 && crs(h[t - 2], h[t - 1], q[i]) <= 0) --t;
        h[t++] = q[i];
    }
    for (size_t i = q.size() - 1, lo = t + 1; i > 0; --i) {
        while (t >= lo && crs(h[t - 2], h[t - 1], q[i - 1]) <= 0) --t;
        h[t++] = q[i - 1];
    }
    h.resize(t > 0 ? t - 1 : 0);
    // (axis k+1, axis k+2, axis k) is right-handed: counter-clockwise in
    // (u, v) is counter-clockwise about +axis k
    std::vector<int> r;
    for (const P2& e : h) r.push_back(e.id);
    if (nk < 0) std::reverse(r.begin(), r.end());
    return r;
}

// Order coplanar points counter-clockwise around normal n, keeping only the
// extreme points of their 2D convex hull (monotone chain); for the welded
// faces, whose points are not exactly coplanar.
std::vector<int> ccw_hull_2d(const std::vector<V3>& P, const std::vector<int>& ids, V3 n) {
    V3 a = std::fabs(n.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0};
    V3 u = norm(cross(n, a));
    V3 v = cross(n, u);
    struct Q {
        double x, y;
        int id;
    };
    std::vector<Q> q;
    for (int id : ids) q.push_back({dot(P[id], u), dot(P[id], v), id});
    std::sort(q.begin(), q.end(), [](const Q& a, const Q& b) {
        return a.x < b.x || (a.x == b.x && (a.y < b.y || (a.y == b.y && a.id < b.id)));
    });
    if (q.size() < 3) {
        std::vector<int> r;
        for (auto& e : q) r.push_back(e.id);
        return r;
    }
    auto crs = [](const Q& o, const Q& a, const Q& b) {
        return (a.x - o.x) * (b.y - o.y) - (a.y - o.y) * (b.x - o.x);
    };
    std::vector<Q> h(2 * q.size());
    size_t k = 0;
    for (size_t i = 0; i < q.size(); ++i) {
        while (k >= 2 && crs(h[k - 2], h[k - 1], q[i]) <= 1e-12) k--;
        h[k++] = q[i];
    }
    for (size_t i = q.size() - 1, t = k + 1; i > 0; --i) {
        while (k >= t && crs(h[k - 2], h[k - 1], q[i - 1]) <= 1e-12) k--;
        h[k++] = q[i - 1];
    }
    h.resize(k - 1);
    // (u, v, n) is right-handed, so increasing angle in (u, v) is CCW about n.
    std::vector<int> r;
    for (auto& e : h) r.push_back(e.id);
    return r;
}

struct RawFace {
    std::vector<int> idx;  // CCW seen from outside (indices into the grid points)
};

}  // namespace

bool compute_polyhedron(const float* pts_in, int n, Polyhedron& out, std::string* err) {
    out = Polyhedron();
    if (n < 4) {
        if (err) *err = "need at least 4 points";
        return false;
    }
    // 1. Grid points, duplicates merged (numbered by their first input point).
    const Grid G = make_grid(pts_in, n);
    std::vector<IV> Q;
    {
        std::unordered_map<uint64_t, int> seen;
        seen.reserve(2 * (size_t)n);
        for (int i = 0; i < n; ++i) {
            const IV v = quantize(G, pts_in + 3 * i);
            const uint64_t key = ((uint64_t)(v.x + 32768) << 32) | ((uint64_t)(v.y + 32768) << 16) |
                                 (uint64_t)(v.z + 32768);
            if (seen.emplace(key, (int)Q.size()).second) Q.push_back(v);
        }
    }
    std::vector<HTri> tris;
    if (!exact_hull(Q, tris)) {
        if (err) *err = "degenerate point set";
        return false;
    }
    // 2. Maximal planar faces: the triangles of one supporting plane.
    std::map<std::array<int64_t, 4>, std::vector<int>> byPlane;
    for (const HTri& t : tris) {
        const int64_t g = gcd64(gcd64(t.n.x, t.n.y), t.n.z);
        const std::array<int64_t, 4> key = {t.n.x / g, t.n.y / g, t.n.z / g, t.d / g};
        std::vector<int>& ids = byPlane[key];
        for (int id : {t.a, t.b, t.c})
            if (std::find(ids.begin(), ids.end(), id) == ids.end()) ids.push_back(id);
    }
    // the grid-to-world map is a per-axis scaling after an axis permutation;
    // when it reverses orientation the counter-clockwise order flips
    int perm[3] = {G.medAxis, G.maxAxis, G.minAxis};
    int inversions = 0;
    for (int a = 0; a < 3; ++a)
        for (int b = a + 1; b < 3; ++b)
            if (perm[a] > perm[b]) ++inversions;
    const double det = (inversions & 1 ? -1.0 : 1.0) * (double)G.scaling[0] * G.scaling[1] * G.scaling[2];
    std::vector<RawFace> planes;
    for (const auto& kv : byPlane) {
        const IV nn = {kv.first[0], kv.first[1], kv.first[2]};
        RawFace f;
        f.idx = planar_polygon(Q, kv.second, nn);
        if (det < 0) std::reverse(f.idx.begin(), f.idx.end());
        if (f.idx.size() >= 3) planes.push_back(f);
    }
    if (planes.size() < 4) {
        if (err) *err = "degenerate point set";
        return false;
    }
    std::vector<V3> P(Q.size());
    for (size_t i = 0; i < Q.size(); ++i) P[i] = dequantize(G, Q[i]);
    n = (int)Q.size();
    // Deterministic face order: by the sorted smallest vertex index, then normal.
    std::sort(planes.begin(), planes.end(), [](const RawFace& a, const RawFace& b) {
        std::vector<int> sa = a.idx, sb = b.idx;
        std::sort(sa.begin(), sa.end());
        std::sort(sb.begin(), sb.end());
        return sa < sb;
    });
    // 2. Hull vertices in input order.
    std::vector<int> used(n, 0);
    for (auto& f : planes)
        for (int id : f.idx) used[id] = 1;
    std::vector<int> remap(n, -1);
    std::vector<V3> verts;
    for (int i = 0; i < n; ++i)
        if (used[i]) {
            remap[i] = (int)verts.size();
            verts.push_back(P[i]);
        }
    // Faces with hull-vertex indices; plane from the first two edges of the
    // polygon, in float as btConvexUtility computes it (:56-108): normal =
    // normalized(normalized(e0) x normalized(e1)), w = -min over the face's
    // vertices of v . normal.
    struct TF {
        double plane[4];
        std::vector<int> idx;
    };
    auto fv = [&](int id) { return F3{(float)verts[id].x, (float)verts[id].y, (float)verts[id].z}; };
    std::vector<TF> tmp;
    for (auto& f : planes) {
        TF t;
        for (int id : f.idx) t.idx.push_back(remap[id]);
        const F3 e0 = fnormalized(fsub(fv(t.idx[1]), fv(t.idx[0])));
        const F3 e1 = fnormalized(fsub(fv(t.idx[2]), fv(t.idx[1])));
        const F3 nn = fnormalized(fcross(e0, e1));
        float pe = 1e30f;
        for (int id : t.idx) {
            const float eq = fdot(fv(id), nn);
            if (pe > eq) pe = eq;
        }
        t.plane[0] = nn.x;
        t.plane[1] = nn.y;
        t.plane[2] = nn.z;
        t.plane[3] = -pe;
        tmp.push_back(t);
    }
    // 3. Coplanar weld (threshold 0.999), reference face = last unprocessed.
    std::vector<int> todo;
    for (int i = 0; i < (int)tmp.size(); ++i) todo.push_back(i);
    std::vector<TF> faces;
    while (!todo.empty()) {
        int ref = todo.back();
        todo.pop_back();
        std::vector<int> group{ref};
        const F3 na{(float)tmp[ref].plane[0], (float)tmp[ref].plane[1], (float)tmp[ref].plane[2]};
        for (int j = (int)todo.size() - 1; j >= 0; --j) {
            int i = todo[j];
            const F3 nb{(float)tmp[i].plane[0], (float)tmp[i].plane[1], (float)tmp[i].plane[2]};
            if (fdot(na, nb) > 0.999f) {
                group.push_back(i);
                todo.erase(todo.begin() + j);
            }
        }
        bool merged = false;
        if (group.size() > 1) {
            std::vector<int> pts;
            V3 avg{0, 0, 0};
            for (int g : group) {
                avg = add(avg, V3{tmp[g].plane[0], tmp[g].plane[1], tmp[g].plane[2]});
                for (int id : tmp[g].idx)
                    if (std::find(pts.begin(), pts.end(), id) == pts.end()) pts.push_back(id);
            }
            avg = norm(avg);
            std::vector<int> hull = ccw_hull_2d(verts, pts, avg);
            bool reject = false;
            for (int id : pts) {
                if (std::find(hull.begin(), hull.end(), id) != hull.end()) continue;
                for (int j = 0; j < (int)tmp.size() && !reject; ++j) {
                    if (std::find(group.begin(), group.end(), j) != group.end()) continue;
                    if (std::find(tmp[j].idx.begin(), tmp[j].idx.end(), id) != tmp[j].idx.end())
                        reject = true;
                }
                if (reject) break;
            }
            if (!reject) {
                TF c;
                for (int q = 0; q < 4; ++q) c.plane[q] = tmp[group[0]].plane[q];
                c.idx = hull;
                faces.push_back(c);
                merged = true;
            }
        }
        if (!merged)
            for (int g : group) faces.push_back(tmp[g]);
    }
    // 4. Unique edges.
    std::vector<V3> uedges;
    for (auto& f : faces) {
        int nv = (int)f.idx.size();
        for (int j = 0; j < nv; ++j) {
            int a = f.idx[j], b = f.idx[(j + 1) % nv];
            int v0 = std::max(a, b), v1 = std::min(a, b);
            V3 e = norm(sub(verts[v1], verts[v0]));
            // float rounding like the reference's btVector3 edges
            V3 ef{(float)e.x, (float)e.y, (float)e.z};
            bool found = false;
            for (auto& u : uedges) {
                V3 dm = sub(u, ef), dp = add(u, ef);
                if ((std::fabs(dm.x) <= 1e-6 && std::fabs(dm.y) <= 1e-6 && std::fabs(dm.z) <= 1e-6) ||
                    (std::fabs(dp.x) <= 1e-6 && std::fabs(dp.y) <= 1e-6 && std::fabs(dp.z) <= 1e-6)) {
                    found = true;
                    break;
                }
            }
            if (!found) uedges.push_back(ef);
        }
    }
    // 5. Output.
    for (auto& v : verts) {
        out.vertices.push_back((float)v.x);
        out.vertices.push_back((float)v.y);
        out.vertices.push_back((float)v.z);
    }
    for (auto& f : faces) {
        Face ff;
        for (int q = 0; q < 4; ++q) ff.plane[q] = (float)f.plane[q];
        ff.indices = f.idx;
        out.faces.push_back(ff);
    }
    for (auto& e : uedges) {
        out.uniqueEdges.push_back((float)e.x);
        out.uniqueEdges.push_back((float)e.y);
        out.uniqueEdges.push_back((float)e.z);
    }
    double cx = 0, cy = 0, cz = 0;
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (size_t i = 0; i < verts.size(); ++i) {
        float vf[3] = {(float)verts[i].x, (float)verts[i].y, (float)verts[i].z};
        for (int q = 0; q < 3; ++q) {
            mn[q] = std::min(mn[q], vf[q]);
            mx[q] = std::max(mx[q], vf[q]);
        }
    }
    // vertex average accumulated in float like btVector3 (P2/CLPhysicsDemo.cpp:360-366)
    float acc[3] = {0, 0, 0};
    for (size_t i = 0; i < verts.size(); ++i) {
        acc[0] += (float)verts[i].x;
        acc[1] += (float)verts[i].y;
        acc[2] += (float)verts[i].z;
    }
    float inv = 1.f / (float)verts.size();
    out.localCenter[0] = acc[0] * inv;
    out.localCenter[1] = acc[1] * inv;
    out.localCenter[2] = acc[2] * inv;
    (void)cx; (void)cy; (void)cz;
    // inradius about the (float) local centre over the unwelded facets: the
    // support in each facet direction minus the centre's projection
    {
        const V3 lc{out.localCenter[0], out.localCenter[1], out.localCenter[2]};
        double r = 1e30;
        for (auto& t : tmp) {
            const V3 nn{t.plane[0], t.plane[1], t.plane[2]};
            double h = -1e30;
            for (auto& v : verts) h = std::max(h, dot(v, nn));
            r = std::min(r, h - dot(lc, nn));
        }
        out.inradius = r < 0.0 ? 0.0 : r;
    }
    for (int q = 0; q < 3; ++q) {
        out.aabbMin[q] = mn[q];
        out.aabbMax[q] = mx[q];
        out.mC[q] = mx[q] + mn[q];
        out.mE[q] = mx[q] - mn[q];
    }
    return true;
}

}  // namespace b3hull
