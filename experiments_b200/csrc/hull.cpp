// Convex-hull polyhedral features for registration (host side).
//
// Behaviour follows btConvexUtility::initializePolyhedralFeatures and
// ::initialize (P1/btConvexUtility.cpp:31-270, 339-513):
//   * hull of the point cloud; hull vertices keep their input order,
//   * faces wound counter-clockwise seen from outside, plane
//     (n, -min_v n.v) over the face's vertices,
//   * faces whose normals agree to dot > 0.999 are welded into one polygon
//     (2D hull of their points, plane of the group's reference face), unless
//     a dropped point is used by a face outside the group,
//   * unique edge directions: normalised (v[smaller] - v[larger]) deduped
//     by +/- within 1e-6 per component,
//   * local centre = average of the hull vertices
//     (CLPhysicsDemo::registerConvexPolyhedron, P2/CLPhysicsDemo.cpp:360-366).
// The hull itself is computed here by exhaustive plane search, which is exact
// for the few-dozen-point shapes this pipeline registers (the reference uses
// Bullet's btConvexHullComputer); faces, vertices and edges agree as sets.
#include "hull.h"

#include <algorithm>
#include <cmath>
#include <map>

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

struct RawFace {
    V3 n;
    double d;                 // plane: n.x = d
    std::vector<int> idx;     // CCW seen from outside (indices into input points)
};

// Order coplanar points counter-clockwise around normal n, keeping only the
// extreme points of their 2D convex hull (monotone chain).
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

}  // namespace

bool compute_polyhedron(const float* pts_in, int n, Polyhedron& out, std::string* err) {
    out = Polyhedron();
    if (n < 4) {
        if (err) *err = "need at least 4 points";
        return false;
    }
    std::vector<V3> P(n);
    double scale = 0;
    for (int i = 0; i < n; ++i) {
        P[i] = {pts_in[3 * i], pts_in[3 * i + 1], pts_in[3 * i + 2]};
        scale = std::max(scale, std::max(std::fabs(P[i].x), std::max(std::fabs(P[i].y), std::fabs(P[i].z))));
    }
    const double eps = 1e-7 * std::max(1.0, scale);
    // 1. Exhaustive supporting-plane search.
    std::vector<RawFace> planes;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            for (int k = j + 1; k < n; ++k) {
                V3 nn = cross(sub(P[j], P[i]), sub(P[k], P[i]));
                double l = len(nn);
                if (l < 1e-12 * std::max(1.0, scale * scale)) continue;
                nn = mul(nn, 1.0 / l);
                double d = dot(nn, P[i]);
                double mx = -1e300, mn = 1e300;
                for (int m = 0; m < n; ++m) {
                    double s = dot(nn, P[m]) - d;
                    mx = std::max(mx, s);
                    mn = std::min(mn, s);
                }
                if (mx <= eps) {
                } else if (mn >= -eps) {
                    nn = mul(nn, -1.0);
                    d = -d;
                } else {
                    continue;
                }
                bool dup = false;
                for (auto& f : planes)
                    if (dot(f.n, nn) > 1.0 - 1e-9 && std::fabs(f.d - d) < 4 * eps) {
                        dup = true;
                        break;
                    }
                if (!dup) planes.push_back({nn, d, {}});
            }
    if (planes.size() < 4) {
        if (err) *err = "degenerate point set";
        return false;
    }
    for (auto& f : planes) {
        std::vector<int> on;
        for (int m = 0; m < n; ++m)
            if (std::fabs(dot(f.n, P[m]) - f.d) <= 4 * eps) on.push_back(m);
        // drop duplicate input points (keep first)
        std::vector<int> uniq;
        for (int m : on) {
            bool same = false;
            for (int u : uniq)
                if (len(sub(P[m], P[u])) <= eps) same = true;
            if (!same) uniq.push_back(m);
        }
        f.idx = ccw_hull_2d(P, uniq, f.n);
    }
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
    // polygon (btConvexUtility: normal = e0 x e1, w = -min over face verts).
    struct TF {
        double plane[4];
        std::vector<int> idx;
    };
    std::vector<TF> tmp;
    for (auto& f : planes) {
        TF t;
        for (int id : f.idx) t.idx.push_back(remap[id]);
        V3 e0 = norm(sub(verts[t.idx[1]], verts[t.idx[0]]));
        V3 e1 = norm(sub(verts[t.idx[2]], verts[t.idx[1]]));
        V3 nn = norm(cross(e0, e1));
        double pe = 1e30;
        for (int id : t.idx) pe = std::min(pe, dot(verts[id], nn));
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
        V3 na{tmp[ref].plane[0], tmp[ref].plane[1], tmp[ref].plane[2]};
        for (int j = (int)todo.size() - 1; j >= 0; --j) {
            int i = todo[j];
            V3 nb{tmp[i].plane[0], tmp[i].plane[1], tmp[i].plane[2]};
            if (dot(na, nb) > 0.999) {
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
