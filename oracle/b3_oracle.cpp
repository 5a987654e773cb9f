// ORACLE — test infrastructure only. Single-threaded CPU restatement of the
// reference GPU rigid-body step (erwincoumans/experiments,
// opencl/gpu_rigidbody_pipeline2 and dependencies), used by tests/, the
// smoke check and bench.py's CPU baseline leg as the checker. Nothing in the
// product links or calls this file.
//
// Precision: the world AABB and cell hash are evaluated in FP32 with the
// same operation order as the device kernel (compiled with
// -ffp-contract=off), so cell keys, the stable sort and the pair set are
// bit-comparable when both start from the same FP32 state. Narrowphase,
// constraint setup, Jacobi iterations and integration run in FP64 (Real).
//
// Parity pins (see oracle/ref_shim.cpp and tests/test_oracle_pins.py):
//   * the Jacobi solver against the reference's own btPgsJacobiSolver
//     (P2/btPgsJacobiSolver.cpp) compiled from the reference sources,
//   * clipping + contact reduction against the reference host port
//     (P2/satClipHullContacts.cpp),
//   * hull tables against btConvexUtility (P1/btConvexUtility.cpp),
//   * analytic known-answer contact cases.
//
// Reference citations (paths relative to the reference project root):
//   AABB      opencl/broadphase_benchmark/broadphaseKernel.cl:91-113,293-331
//   hash      opencl/3dGridBroadphase/Shared/bt3dGridBroadphaseOCL.cl:4-48
//   pairs     opencl/3dGridBroadphase/Shared/bt3dGridBroadphaseOCL.cl:89-215
//   SAT       opencl/gpu_rigidbody_pipeline2/sat.cl:227-252,497-635,928-1262
//   clip      opencl/gpu_rigidbody_pipeline2/satClipHullContacts.cl:303-452,556-611
//   reduce    opencl/gpu_rigidbody_pipeline2/satClipHullContacts.cl:678-770,1958-2039
//   solver    opencl/gpu_rigidbody_pipeline2/btPgsJacobiSolver.cpp:124-155,505-592,
//             689-888,933-1080,1081-1370,1372-1823
//   integrate opencl/broadphase_benchmark/integrateKernel.cl:102-158
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef ORACLE_DUAL
// tangent-linear build: every Real carries a derivative along one direction
#include "b3_dual.h"
#define ORACLE_REAL b3dual::Dual
#endif
#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
typedef ORACLE_REAL Real;

// value and tangent of a Real, the same source for every build
inline double rval(double x) { return x; }
inline double rval(float x) { return x; }
inline double rtan(double) { return 0.0; }
inline double rtan(float) { return 0.0; }
inline void set_tan(double&, double) {}
inline void set_tan(float&, double) {}
#ifdef ORACLE_DUAL
inline double rval(const b3dual::Dual& x) { return x.v; }
inline double rtan(const b3dual::Dual& x) { return x.d; }
inline void set_tan(b3dual::Dual& x, double d) { x.d = d; }
#endif
// unqualified calls: the std overloads for double / float, the dual ones
// by argument-dependent lookup
using std::cos;
using std::fabs;
using std::sin;
using std::sqrt;

namespace {

struct V {
    Real x, y, z;
    V() : x(0), y(0), z(0) {}
    V(Real a, Real b, Real c) : x(a), y(b), z(c) {}
};
inline V operator+(V a, V b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V operator-(V a, V b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V operator-(V a) { return V(-a.x, -a.y, -a.z); }
inline V operator*(V a, Real s) { return V(a.x * s, a.y * s, a.z * s); }
inline Real dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(V a, V b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V mulv(V a, V b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V normalize(V a) {
    Real l = sqrt(dot(a, a));
    return l > 0 ? a * (1.0 / l) : a;
}
struct Q {
    Real x, y, z, w;
};
// qtMul / qtRotate (sat.cl:146-230) in Real
inline Q qmul(Q a, Q b) {
    V c = cross(V(a.x, a.y, a.z), V(b.x, b.y, b.z));
    Q r;
    r.x = c.x + a.w * b.x + b.w * a.x;
    r.y = c.y + a.w * b.y + b.w * a.y;
    r.z = c.z + a.w * b.z + b.w * a.z;
    r.w = a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z);
    return r;
}
inline V qrot(Q q, V v) {
    Q qi = {-q.x, -q.y, -q.z, q.w};
    Q vv = {v.x, v.y, v.z, 0};
    Q r = qmul(qmul(q, vv), qi);
    return V(r.x, r.y, r.z);
}
inline V qinvrot(Q q, V v) { return qrot(Q{-q.x, -q.y, -q.z, q.w}, v); }
inline uint64_t mix64(uint64_t h, uint64_t v) { return (h ^ (v + 0x9e3779b97f4a7c15ull)) * 0x100000001b3ull; }

}  // namespace

extern "C" {

// Shape tables (layout of the reference's ConvexPolyhedronCL / btGpuFace).
struct or_poly {
    float localCenter[4], extents[4], mC[4], mE[4];
    float radius;
    int faceOffset, numFaces, numVertices, vertexOffset, uniqueEdgesOffset, numUniqueEdges, unused;
};
struct or_face {
    float plane[4];
    int indexOffset, numIndices, pad[2];
};
struct or_contact {  // Contact4-like, FP64 (the exported layout)
    double pos[4][4];
    double normal[4];  // w = nPoints
    double friction;
    int pairIndex, bodyA, bodyB, pad;
};
struct or_contact_r {  // the same in Real (internal storage)
    Real pos[4][4];
    Real normal[4];
    Real friction;
    int pairIndex, bodyA, bodyB, pad;
};

struct or_config {
    float cellSize;
    int dims[3];
    int maxBodiesPerCell;
    int maxPairsPerBody;
    float gravity[3];
    float dt;
    int iterations;
    float erp;
    float contactBreaking;
    float contactProcessing;
    float slopOffset;
    float angularDamping;
    int frictionCombine;  // 0 = sqrt(a*b), 1 = a*b
    int numWorlds;
    int maxPairs;         // global pair capacity (0 = unlimited)
};

struct or_world {
    or_config cfg;
    int n;
    int cellBits;
    // static body data
    std::vector<Real> invMass, friction, restitution;  // set from FP32 inputs, or FP64 by or_set_params_f64
    std::vector<int> col, worldId, isLarge;
    std::vector<Real> invInertia;  // 3 per body
    // shapes
    std::vector<int> colShape;
    std::vector<or_poly> polys;
    std::vector<float> verts4, edges4, localAabb8;
    std::vector<or_face> faces;
    std::vector<int> indices;
    // state (FP64) and its FP32 image for the integer stages
    std::vector<Real> pos, quat, lin, ang;  // 4 per body
    // stage outputs
    std::vector<float> aabb;                 // 8 per body
    std::vector<uint32_t> keys, vals;        // sorted (small bodies)
    std::vector<int> pairs;                  // 2 per pair
    std::vector<or_contact_r> contacts;      // manifolds in pair order
    std::vector<Real> avgLin, avgAng;        // 3 per body (sum/count after the last average)
    std::vector<int> count;                  // copies per body
    // per-world signature of the discrete choices (pairs with manifolds,
    // clip size and reduced point indices, row clamp states), for telling
    // which worlds keep their active set under a perturbation
    std::vector<uint64_t> activeHash;   // row clamp states
    std::vector<uint64_t> topoHash;     // pairs with manifolds, clip sizes, reduced points
    long long pairOverflow, cellOverflow;
    // collidable table beyond the hulls (or_set_collidables): type, radius,
    // child count and shape index per collidable; the compounds' children
    std::vector<int> colType, colNum, colIndex;
    std::vector<float> colRadius;
    std::vector<float> childPose;   // 8 per child: position xyzw, orientation xyzw
    std::vector<int> childCol;
    int sap;  // broadphase: 0 = uniform grid, 1 = sweep and prune
    int gs;   // solver: 0 = Jacobi (pipeline2), 1 = batched Gauss-Seidel (the reference GPU solver)
    // batched Gauss-Seidel: per manifold its cell (xz, 16 x 16) and batch
    std::vector<int> gsCell, gsBatch;
    std::vector<double> gsApplied;  // per manifold: normal impulses [4], friction impulses [2]
};

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------
// FP32 stage: AABB + gravity + hash (exact operation order, no contraction)
// ---------------------------------------------------------------------------
inline float d3(const float a[4], const float b[4]) { return ((a[0] * b[0]) + (a[1] * b[1])) + (a[2] * b[2]); }

void qmul_f(const float a[4], const float b[4], float r[4]) {
    const float c0 = a[1] * b[2] - a[2] * b[1];
    const float c1 = a[2] * b[0] - a[0] * b[2];
    const float c2 = a[0] * b[1] - a[1] * b[0];
    r[0] = c0 + ((a[3] * b[0]) + (b[3] * a[0]));
    r[1] = c1 + ((a[3] * b[1]) + (b[3] * a[1]));
    r[2] = c2 + ((a[3] * b[2]) + (b[3] * a[2]));
    r[3] = (a[3] * b[3]) - d3(a, b);
}

void aabb_f32(const float p[4], const float q[4], const float* lmn, const float* lmx, float out[8]) {
    const float he[4] = {(lmx[0] - lmn[0]) * 0.5f, (lmx[1] - lmn[1]) * 0.5f, (lmx[2] - lmn[2]) * 0.5f, 0.f};
    const float lc[4] = {(lmx[0] + lmn[0]) * 0.5f, (lmx[1] + lmn[1]) * 0.5f, (lmx[2] + lmn[2]) * 0.5f, 0.f};
    const float qi[4] = {-q[0], -q[1], -q[2], q[3]};
    float t[4], wc[4];
    qmul_f(q, lc, t);
    qmul_f(t, qi, wc);
    wc[0] = wc[0] + p[0];
    wc[1] = wc[1] + p[1];
    wc[2] = wc[2] + p[2];
    const float x2 = q[0] * q[0], y2 = q[1] * q[1], z2 = q[2] * q[2];
    const float tx = 2.f * q[0], ty = 2.f * q[1], tw = 2.f * q[3];
    const float r0[4] = {std::fabs((1.f - 2.f * y2) - 2.f * z2), std::fabs(tx * q[1] - tw * q[2]),
                         std::fabs(tx * q[2] + tw * q[1]), 0.f};
    const float r1[4] = {std::fabs(tx * q[1] + tw * q[2]), std::fabs((1.f - 2.f * x2) - 2.f * z2),
                         std::fabs(ty * q[2] - tw * q[0]), 0.f};
    const float r2[4] = {std::fabs(tx * q[2] - tw * q[1]), std::fabs(ty * q[2] + tw * q[0]),
                         std::fabs((1.f - 2.f * x2) - 2.f * y2), 0.f};
    const float e[3] = {d3(r0, he), d3(r1, he), d3(r2, he)};
    for (int k = 0; k < 3; ++k) {
        out[k] = wc[k] - e[k];
        out[4 + k] = wc[k] + e[k];
    }
}

inline int gcoord(float c, float inv, int dim) { return ((int)std::floor(c * inv)) & (dim - 1); }

void stage_aabbs(or_world* w) {
    const int N = w->n;
    w->aabb.assign(8 * (size_t)N, 0.f);
    const float gdt[3] = {w->cfg.gravity[0] * w->cfg.dt, w->cfg.gravity[1] * w->cfg.dt, w->cfg.gravity[2] * w->cfg.dt};
    for (int i = 0; i < N; ++i) {
        float p[4] = {(float)w->pos[4 * i], (float)w->pos[4 * i + 1], (float)w->pos[4 * i + 2], 0.f};
        float q[4] = {(float)w->quat[4 * i], (float)w->quat[4 * i + 1], (float)w->quat[4 * i + 2], (float)w->quat[4 * i + 3]};
        const int c = w->col[i];
        float* o = &w->aabb[8 * (size_t)i];
        aabb_f32(p, q, &w->localAabb8[8 * c], &w->localAabb8[8 * c + 4], o);
        int id = i;
        memcpy(&o[3], &id, 4);
        int dyn = w->invMass[i] == 0.f ? 0 : 1;
        memcpy(&o[7], &dyn, 4);
        if (w->invMass[i] != 0.f)
            for (int k = 0; k < 3; ++k) w->lin[4 * i + k] += (Real)gdt[k];
    }
}

// Sweep-and-prune pairs over small proxies sorted by min along axis, each
// record (min x, y, z, id | max x, y, z, max.w) as float bits: per sorted
// proxy i, every large proxy overlapping it (pair (large id, id_i)), then
// every later j whose min along axis does not exceed i's max and whose AABB
// overlaps (pair (id_i, id_j)); computePairsKernelTwoArrays (BB/sap.cl:
// 65-90) and computePairsKernel (BB/sapFast.cl:48-150), with the device
// build's deterministic order. The overlap test is inclusive, x, z, y; the
// small-small test skips two max.w both 0 (BB/sapFast.cl:39-41).
inline bool sap_overlap(const float* a, const float* b) {
    bool o = true;
    o = (a[0] > b[4] || a[4] < b[0]) ? false : o;
    o = (a[2] > b[6] || a[6] < b[2]) ? false : o;
    o = (a[1] > b[5] || a[5] < b[1]) ? false : o;
    return o;
}
inline int fbits(float f) {
    int i;
    memcpy(&i, &f, 4);
    return i;
}
void sap_pairs(const std::vector<float>& sorted8, int n, int axis, const std::vector<float>& large8, int numLarge,
               std::vector<int>& pairs) {
    for (int i = 0; i < n; ++i) {
        const float* a = &sorted8[8 * (size_t)i];
        for (int l = 0; l < numLarge; ++l) {
            const float* L = &large8[8 * (size_t)l];
            if (sap_overlap(L, a)) {
                pairs.push_back(fbits(L[3]));
                pairs.push_back(fbits(a[3]));
            }
        }
        const float test = a[4 + axis];
        for (int j = i + 1; j < n; ++j) {
            const float* b = &sorted8[8 * (size_t)j];
            if (test < b[axis]) break;
            if (fbits(a[7]) == 0 && fbits(b[7]) == 0) continue;
            if (sap_overlap(a, b)) {
                pairs.push_back(fbits(a[3]));
                pairs.push_back(fbits(b[3]));
            }
        }
    }
}

// FloatFlip (BB/sap.cl:272-278)
inline uint32_t float_flip(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint32_t mask = (uint32_t)(-(int32_t)(u >> 31)) | 0x80000000u;
    return u ^ mask;
}

// btGpuSapBroadphase::calculateOverlappingPairs (P2/btGpuSapBroadphase.cpp:
// 97-485): dynamic bodies are the small proxies, sorted stably by
// FloatFlip(min.x); static bodies the large ones (P2/CLPhysicsDemo.cpp:
// 558-568). A small proxy's max.w is its body index (copyAabbsKernel,
// BB/sap.cl:290-299).
void stage_broadphase_sap(or_world* w) {
    const int N = w->n;
    std::vector<std::pair<uint32_t, int>> kv;
    std::vector<float> large8;
    int numLarge = 0;
    for (int i = 0; i < N; ++i) {
        if (w->invMass[i] != 0.f) {
            kv.push_back({float_flip(w->aabb[8 * (size_t)i]), i});
        } else {
            large8.insert(large8.end(), &w->aabb[8 * (size_t)i], &w->aabb[8 * (size_t)i] + 8);
            ++numLarge;
        }
    }
    std::stable_sort(kv.begin(), kv.end(), [](const std::pair<uint32_t, int>& a, const std::pair<uint32_t, int>& b) {
        return a.first < b.first;
    });
    std::vector<float> sorted8(8 * kv.size());
    w->keys.clear();
    w->vals.clear();
    for (size_t s = 0; s < kv.size(); ++s) {
        const int b = kv[s].second;
        memcpy(&sorted8[8 * s], &w->aabb[8 * (size_t)b], 8 * sizeof(float));
        memcpy(&sorted8[8 * s + 7], &b, 4);
        w->keys.push_back(kv[s].first);
        w->vals.push_back((uint32_t)b);
    }
    w->pairs.clear();
    w->pairOverflow = 0;
    w->cellOverflow = 0;
    sap_pairs(sorted8, (int)kv.size(), 0, large8, numLarge, w->pairs);
    if (w->cfg.maxPairs > 0 && (long long)w->pairs.size() / 2 > w->cfg.maxPairs) {
        w->pairOverflow += (long long)w->pairs.size() / 2 - w->cfg.maxPairs;
        w->pairs.resize(2 * (size_t)w->cfg.maxPairs);
    }
}

void stage_broadphase(or_world* w) {
    if (w->sap) {
        stage_broadphase_sap(w);
        return;
    }
    const int N = w->n;
    const float inv = 1.f / w->cfg.cellSize;
    const int dx = w->cfg.dims[0], dy = w->cfg.dims[1], dz = w->cfg.dims[2];
    struct KV {
        uint32_t k, v;
    };
    std::vector<KV> kv;
    for (int i = 0; i < N; ++i) {
        if (w->isLarge[i]) continue;
        const float* a = &w->aabb[8 * (size_t)i];
        const float cx = (a[0] + a[4]) * 0.5f, cy = (a[1] + a[5]) * 0.5f, cz = (a[2] + a[6]) * 0.5f;
        const int gx = gcoord(cx, inv, dx), gy = gcoord(cy, inv, dy), gz = gcoord(cz, inv, dz);
        const uint32_t h = (uint32_t)(gz * dy * dx + gy * dx + gx);
        kv.push_back({((uint32_t)w->worldId[i] << w->cellBits) | h, (uint32_t)i});
    }
    // stable LSD sort == stable sort by key (btRadixSort32CL::executeHost)
    std::stable_sort(kv.begin(), kv.end(), [](const KV& a, const KV& b) { return a.k < b.k; });
    const int ns = (int)kv.size();
    w->keys.resize(ns);
    w->vals.resize(ns);
    for (int i = 0; i < ns; ++i) {
        w->keys[i] = kv[i].k;
        w->vals[i] = kv[i].v;
    }
    // cell starts (first sorted index per key)
    std::vector<std::pair<uint32_t, int>> starts;
    for (int i = 0; i < ns; ++i)
        if (i == 0 || w->keys[i - 1] != w->keys[i]) starts.push_back({w->keys[i], i});
    auto find_start = [&](uint32_t h) -> int {
        auto it = std::lower_bound(starts.begin(), starts.end(), std::make_pair(h, -1));
        if (it == starts.end() || it->first != h) return -1;
        return it->second;
    };
    // large bodies per world
    std::vector<std::vector<int>> large(w->cfg.numWorlds);
    for (int i = 0; i < N; ++i)
        if (w->isLarge[i]) large[w->worldId[i]].push_back(i);
    auto overlap = [&](int a, int b) {
        const float* A = &w->aabb[8 * (size_t)a];
        const float* B = &w->aabb[8 * (size_t)b];
        return A[0] <= B[4] && B[0] <= A[4] && A[1] <= B[5] && B[1] <= A[5] && A[2] <= B[6] && B[2] <= A[6];
    };
    w->pairs.clear();
    w->pairOverflow = 0;
    w->cellOverflow = 0;
    const int cap = w->cfg.maxPairsPerBody - 1;  // curr_max
    for (int i = 0; i < ns; ++i) {
        const uint32_t self = w->vals[i];
        const uint32_t world = w->keys[i] >> w->cellBits;
        const float* a = &w->aabb[8 * (size_t)self];
        const float cx = (a[0] + a[4]) * 0.5f, cy = (a[1] + a[5]) * 0.5f, cz = (a[2] + a[6]) * 0.5f;
        const int gx = gcoord(cx, inv, dx), gy = gcoord(cy, inv, dy), gz = gcoord(cz, inv, dz);
        int cnt = 0;
        for (int oz = -1; oz <= 1; ++oz)
            for (int oy = -1; oy <= 1; ++oy)
                for (int ox = -1; ox <= 1; ++ox) {
                    const int xx = (gx + ox) & (dx - 1), yy = (gy + oy) & (dy - 1), zz = (gz + oz) & (dz - 1);
                    const uint32_t h = (world << w->cellBits) | (uint32_t)(zz * dy * dx + yy * dx + xx);
                    const int start = find_start(h);
                    if (start < 0) continue;
                    const int end = std::min(start + w->cfg.maxBodiesPerCell, ns);
                    int j = start;
                    bool full = false;
                    for (; j < end; ++j) {
                        if (w->keys[j] != h) break;
                        const uint32_t other = w->vals[j];
                        if (other < self && overlap((int)self, (int)other)) {
                            if (cnt >= cap) {
                                w->pairOverflow++;
                                full = true;
                                break;
                            }
                            w->pairs.push_back((int)self);
                            w->pairs.push_back((int)other);
                            ++cnt;
                        }
                    }
                    if (!full && j == end && end < ns && w->keys[end] == h) w->cellOverflow++;
                }
        for (int L : large[world]) {
            if (overlap((int)self, L)) {
                if (cnt >= cap) {
                    w->pairOverflow++;
                    break;
                }
                w->pairs.push_back((int)self);
                w->pairs.push_back(L);
                ++cnt;
            }
        }
    }
    // global capacity: the device keeps the first maxPairs pairs in order
    if (w->cfg.maxPairs > 0 && (long long)w->pairs.size() / 2 > w->cfg.maxPairs) {
        w->pairOverflow += (long long)w->pairs.size() / 2 - w->cfg.maxPairs;
        w->pairs.resize(2 * (size_t)w->cfg.maxPairs);
    }
}

// ---------------------------------------------------------------------------
// Narrowphase (FP64)
// ---------------------------------------------------------------------------
struct Body {
    V pos;
    Q q;
};

inline V vtx(const or_world* w, int i) { return V(w->verts4[4 * i], w->verts4[4 * i + 1], w->verts4[4 * i + 2]); }

// project (sat.cl:227-252)
void project(const or_world* w, const or_poly& h, const Body& b, V dir, Real& mn, Real& mx) {
    mn = std::numeric_limits<Real>::max();
    mx = -std::numeric_limits<Real>::max();
    const V ld = qinvrot(b.q, dir);
    const Real off = dot(b.pos, dir);
    for (int i = 0; i < h.numVertices; ++i) {
        const Real dp = dot(vtx(w, h.vertexOffset + i), ld);
        if (dp < mn) mn = dp;
        if (dp > mx) mx = dp;
    }
    if (mn > mx) std::swap(mn, mx);
    mn += off;
    mx += off;
}

// findSeparatingAxis (sat.cl:497-551); returns false if a face axis separates
// feature of the chosen separating axis (A face i, 1000 + B face i, or
// 100000 + 1000 e0 + e1 for an edge pair), for the active-set signature
int g_axisId = -1;

// Every axis projected by the search (depth, feature id, oriented normal):
// depths within kAxisTieTol of the minimum are tied and the first axis in
// the reference's order wins (its first minimum for axes tied in exact
// arithmetic, whose FP64 depths differ only by rounding).
constexpr double kAxisTieTol = 1e-10;
struct AxisRec {
    Real d;
    int id;
    V n;
};
thread_local std::vector<AxisRec> g_axes;

bool face_axes(const or_world* w, const or_poly& hA, const or_poly& hB, const Body& A, const Body& B, V D,
               V& sep, Real& dmin, int idBase) {
    for (int i = 0; i < hA.numFaces; ++i) {
        const or_face& f = w->faces[hA.faceOffset + i];
        V n = qrot(A.q, V(f.plane[0], f.plane[1], f.plane[2]));
        if (dot(D, n) < 0) n = -n;
        Real mn0, mx0, mn1, mx1;
        project(w, hA, A, n, mn0, mx0);
        project(w, hB, B, n, mn1, mx1);
        if (mx0 < mn1 || mx1 < mn0) return false;
        const Real d0 = mx0 - mn1, d1 = mx1 - mn0;
        const Real d = d0 < d1 ? d0 : d1;
        g_axes.push_back({d, idBase + i, n});
        if (d < dmin) {
            dmin = d;
            sep = n;
            g_axisId = idBase + i;
        }
    }
    if (dot(-D, sep) > 0) sep = -sep;
    return true;
}

// findSeparatingAxisEdgeEdge (sat.cl:556-635): never rejects
void edge_axes(const or_world* w, const or_poly& hA, const or_poly& hB, const Body& A, const Body& B, V D,
               V& sep, Real& dmin) {
    for (int e0 = 0; e0 < hA.numUniqueEdges; ++e0) {
        const float* ea = &w->edges4[4 * (hA.uniqueEdgesOffset + e0)];
        const V wa = qrot(A.q, V(ea[0], ea[1], ea[2]));
        for (int e1 = 0; e1 < hB.numUniqueEdges; ++e1) {
            const float* eb = &w->edges4[4 * (hB.uniqueEdgesOffset + e1)];
            const V wb = qrot(B.q, V(eb[0], eb[1], eb[2]));
            V c = cross(wa, wb);
            if (!(fabs(c.x) > 1e-6 || fabs(c.y) > 1e-6 || fabs(c.z) > 1e-6)) continue;
            c = normalize(c);
            if (dot(D, c) < 0) c = -c;
            Real mn0, mx0, mn1, mx1;
            project(w, hA, A, c, mn0, mx0);
            project(w, hB, B, c, mn1, mx1);
            const Real d0 = mx0 - mn1, d1 = mx1 - mn0;
            const Real d = d0 < d1 ? d0 : d1;
            g_axes.push_back({d, 100000 + 1000 * e0 + e1, c});
            if (d < dmin) {
                dmin = d;
                sep = c;
                g_axisId = 100000 + 1000 * e0 + e1;
            }
        }
    }
    if (dot(-D, sep) > 0) sep = -sep;
}

struct P4 {
    Real x, y, z, w;
};

// clipFace (satClipHullContacts.cl:303-351)
int clip_face(const std::vector<P4>& in, V pn, Real eq, std::vector<P4>& out) {
    out.clear();
    const int n = (int)in.size();
    if (n == 0) return 0;
    P4 first = in[n - 1];
    Real ds = pn.x * first.x + pn.y * first.y + pn.z * first.z + eq;
    for (int ve = 0; ve < n; ++ve) {
        const P4 end = in[ve];
        const Real de = pn.x * end.x + pn.y * end.y + pn.z * end.z + eq;
        if (ds < 0) {
            if (de < 0) {
                out.push_back(end);
            } else {
                const Real t = ds * 1.0 / (ds - de);
                out.push_back({first.x + (end.x - first.x) * t, first.y + (end.y - first.y) * t,
                               first.z + (end.z - first.z) * t, 0});
            }
        } else if (de < 0) {
            const Real t = ds * 1.0 / (ds - de);
            out.push_back({first.x + (end.x - first.x) * t, first.y + (end.y - first.y) * t,
                           first.z + (end.z - first.z) * t, 0});
            out.push_back(end);
        }
        first = end;
        ds = de;
    }
    if (out.size() > 64) out.resize(64);
    return (int)out.size();
}

#ifdef ORACLE_LOCAL_FRAME
// clipFace with the plane given by a normal and a point on it
int clip_face_pt(const std::vector<P4>& in, V pn, V a, std::vector<P4>& out) {
    out.clear();
    const int n = (int)in.size();
    if (n == 0) return 0;
    P4 first = in[n - 1];
    Real ds = pn.x * (first.x - a.x) + pn.y * (first.y - a.y) + pn.z * (first.z - a.z);
    for (int ve = 0; ve < n; ++ve) {
        const P4 end = in[ve];
        const Real de = pn.x * (end.x - a.x) + pn.y * (end.y - a.y) + pn.z * (end.z - a.z);
        if (ds < 0) {
            if (de < 0) {
                out.push_back(end);
            } else {
                const Real t = ds * 1.0 / (ds - de);
                out.push_back({first.x + (end.x - first.x) * t, first.y + (end.y - first.y) * t,
                               first.z + (end.z - first.z) * t, 0});
            }
        } else if (de < 0) {
            const Real t = ds * 1.0 / (ds - de);
            out.push_back({first.x + (end.x - first.x) * t, first.y + (end.y - first.y) * t,
                           first.z + (end.z - first.z) * t, 0});
            out.push_back(end);
        }
        first = end;
        ds = de;
    }
    if (out.size() > 64) out.resize(64);
    return (int)out.size();
}
#endif

constexpr double kFaceTieTol = 1e-10;

// The face of h (posed b) with the smallest sign * (n . sep), ties within
// kFaceTieTol to the lowest index; -1 for a hull without faces.
int extreme_face(const or_world* w, const or_poly& h, const Body& b, V sep, double sign) {
    std::vector<Real> d(h.numFaces);
    Real best = std::numeric_limits<Real>::max();
    for (int f = 0; f < h.numFaces; ++f) {
        const or_face& fc = w->faces[h.faceOffset + f];
        d[f] = (Real)sign * dot(qrot(b.q, V(fc.plane[0], fc.plane[1], fc.plane[2])), sep);
        if (d[f] < best) best = d[f];
    }
    for (int f = 0; f < h.numFaces; ++f)
        if (d[f] - best <= (Real)kFaceTieTol) return f;
    return -1;
}

// clipHullAgainstHull (satClipHullContacts.cl:556-611 with clipFaceAgainstHull :353-452)
int clip_hull_hull(const or_world* w, V sep, const or_poly& hA, const or_poly& hB, const Body& A, const Body& B,
                   Real minDist, Real maxDist, std::vector<P4>& out) {
    out.clear();
    // incident face of B: the largest n . sep; reference face of A: the
    // smallest. Faces within kFaceTieTol of the extreme are tied and the
    // lowest index wins, the reference's first extreme for faces tied in
    // exact arithmetic (their FP64 products differ only by rounding).
    const int closestB = extreme_face(w, hB, B, sep, -1.0);
    if (closestB < 0) return 0;
    std::vector<P4> in, tmp;
#ifdef ORACLE_LOCAL_FRAME
    // Same arithmetic in a frame centred on body A (numerics experiment for
    // the FP32 build only): clip planes as (normal, point), no plane constant.
    const V orgA = A.pos;
#else
    const V orgA(0, 0, 0);
#endif
    {
        const or_face& fb = w->faces[hB.faceOffset + closestB];
        for (int e = 0; e < fb.numIndices; ++e) {
            const V b = vtx(w, hB.vertexOffset + w->indices[fb.indexOffset + e]);
            const V wv = qrot(B.q, b) + (B.pos - orgA);
            in.push_back({wv.x, wv.y, wv.z, 0});
        }
    }
    const int closestA = extreme_face(w, hA, A, sep, 1.0);
    if (closestA < 0) return 0;
    const or_face& fa = w->faces[hA.faceOffset + closestA];
    const int nvA = fa.numIndices;
    // A reference face of two vertices (a mesh triangle's edge plane,
    // sat.cl:1083-1105) has two side planes that are one plane with opposite
    // orientations; clipFace keeps only points strictly inside (ds < 0), so
    // in exact arithmetic nothing is kept. The reference's FP32 outcome
    // there is rounding noise; the exact result is taken.
    if (nvA < 3) return 0;
    const V nA = V(fa.plane[0], fa.plane[1], fa.plane[2]);
    const V nAw = qrot(A.q, nA);
    for (int e0 = 0; e0 < nvA; ++e0) {
        const V a = vtx(w, hA.vertexOffset + w->indices[fa.indexOffset + e0]);
        const V b = vtx(w, hA.vertexOffset + w->indices[fa.indexOffset + (e0 + 1) % nvA]);
        const V we = qrot(A.q, a - b);
        const V pn = -cross(we, nAw);
#ifdef ORACLE_LOCAL_FRAME
        const V wa = qrot(A.q, a);
        clip_face_pt(in, pn, wa, tmp);
#else
        const V wa = qrot(A.q, a) + A.pos;
        const Real eq = -dot(wa, pn);
        clip_face(in, pn, eq, tmp);
#endif
        in.swap(tmp);
    }
#ifdef ORACLE_LOCAL_FRAME
    const Real eqA = (Real)fa.plane[3];
#else
    const Real eqA = (Real)fa.plane[3] - dot(nAw, A.pos);
#endif
    for (const P4& p : in) {
        Real depth = nAw.x * p.x + nAw.y * p.y + nAw.z * p.z + eqA;
        if (depth <= minDist) depth = minDist;
        if (depth <= maxDist) out.push_back({p.x + orgA.x, p.y + orgA.y, p.z + orgA.z, depth});
    }
    return (int)out.size();
}

// extractManifoldSequentialGlobal (satClipHullContacts.cl:678-770)
int reduce_manifold(const std::vector<P4>& p, V nearNormal, int idx[4]) {
    int n = (int)p.size();
    idx[0] = 0; idx[1] = 1; idx[2] = 2; idx[3] = 3;
    if (n == 0) return 0;
    if (n <= 4) return n;
    if (n > 64) n = 64;
    P4 c = {0, 0, 0, 0};
    for (int i = 0; i < n; ++i) {
        c.x += p[i].x; c.y += p[i].y; c.z += p[i].z; c.w += p[i].w;
    }
    c.x /= n; c.y /= n; c.z /= n; c.w /= n;
    const V cv(c.x, c.y, c.z);
    const V aV = V(p[0].x, p[0].y, p[0].z) - cv;
    V u = cross(nearNormal, aV);
    V v = cross(nearNormal, u);
    u = normalize(u);
    v = normalize(v);
    Real minW = std::numeric_limits<Real>::max();
    int minIndex = -1;
    Real md[4] = {FLT_MIN, FLT_MIN, FLT_MIN, FLT_MIN};
    for (int ie = 0; ie < n; ++ie) {
        if (p[ie].w < minW) {
            minW = p[ie].w;
            minIndex = ie;
        }
        const V r = V(p[ie].x, p[ie].y, p[ie].z) - cv;
        Real f = dot(u, r);
        if (f < md[0]) { md[0] = f; idx[0] = ie; }
        f = dot(-u, r);
        if (f < md[1]) { md[1] = f; idx[1] = ie; }
        f = dot(v, r);
        if (f < md[2]) { md[2] = f; idx[2] = ie; }
        f = dot(-v, r);
        if (f < md[3]) { md[3] = f; idx[3] = ie; }
    }
    if (idx[0] != minIndex && idx[1] != minIndex && idx[2] != minIndex && idx[3] != minIndex) idx[0] = minIndex;
    return 4;
}

Real combine_friction(Real a, Real b, int mode) { return mode == 1 ? a * b : sqrt(a * b); }

Body body_pose(const or_world* w, int i) {
    Body b;
    b.pos = V(w->pos[4 * i], w->pos[4 * i + 1], w->pos[4 * i + 2]);
    b.q = Q{w->quat[4 * i], w->quat[4 * i + 1], w->quat[4 * i + 2], w->quat[4 * i + 3]};
    return b;
}

// SAT, clip and reduction of hull hA at pose a against hull hB at pose b;
// the manifold is reported for bodies A and B.
bool contact_for_shapes(const or_world* w, int pairIndex, int A, int B, const or_poly& hA, const Body& a,
                        const or_poly& hB, const Body& b, or_contact_r& out);

bool contact_for_pair(const or_world* w, int pairIndex, int A, int B, or_contact_r& out) {
    if (w->invMass[A] == 0.f && w->invMass[B] == 0.f) return false;  // sat.cl:944-948
    return contact_for_shapes(w, pairIndex, A, B, w->polys[w->colShape[w->col[A]]], body_pose(w, A),
                              w->polys[w->colShape[w->col[B]]], body_pose(w, B), out);
}

bool contact_for_shapes(const or_world* w, int pairIndex, int A, int B, const or_poly& hA, const Body& a,
                        const or_poly& hB, const Body& b, or_contact_r& out) {
    const V c0 = qrot(a.q, V(hA.localCenter[0], hA.localCenter[1], hA.localCenter[2])) + a.pos;
    const V c1 = qrot(b.q, V(hB.localCenter[0], hB.localCenter[1], hB.localCenter[2])) + b.pos;
    const V D = c0 - c1;
    Real dmin = std::numeric_limits<Real>::max();
    V sep(0, 0, 0);
    bool haveAxis = false;
    {
        // track whether any axis was accepted (dmin updated)
        g_axisId = -1;
        g_axes.clear();
        if (!face_axes(w, hA, hB, a, b, D, sep, dmin, 0)) return false;
        if (!face_axes(w, hB, hA, b, a, D, sep, dmin, 1000)) return false;
        edge_axes(w, hA, hB, a, b, D, sep, dmin);
        haveAxis = dmin < std::numeric_limits<Real>::max();
        // ties: the first axis (in search order) within kAxisTieTol of the minimum
        for (const AxisRec& r : g_axes)
            if (r.d - dmin <= (Real)kAxisTieTol) {
                sep = r.n;
                g_axisId = r.id;
                if (dot(-D, sep) > 0) sep = -sep;
                break;
            }
    }
    if (!haveAxis) return false;
    std::vector<P4> pts;
    const int np = clip_hull_hull(w, sep, hA, hB, a, b, -1e30, (Real)w->cfg.contactBreaking, pts);
    if (np <= 0) return false;
    const V nrm = -sep;
    int idx[4];
    const int nr = reduce_manifold(pts, nrm, idx);
    out = or_contact_r();
    out.pad = (int)std::min<size_t>(pts.size(), 127) | (idx[0] << 7) | (idx[1] << 13) | (idx[2] << 19) | (idx[3] << 25);
    for (int k = 0; k < nr; ++k) {
        const P4& q = pts[idx[k]];
        out.pos[k][0] = q.x; out.pos[k][1] = q.y; out.pos[k][2] = q.z; out.pos[k][3] = q.w;
    }
    out.normal[0] = nrm.x; out.normal[1] = nrm.y; out.normal[2] = nrm.z; out.normal[3] = nr;
    out.friction = combine_friction(w->friction[A], w->friction[B], w->cfg.frictionCombine);
    out.pairIndex = pairIndex;
    out.bodyA = w->invMass[A] == 0.f ? -A : A;
    out.bodyB = w->invMass[B] == 0.f ? -B : B;
    return true;
}

// The pair's manifold goes into the per-world signature of discrete choices.
void record_topology(or_world* w, const or_contact_r& c) {
    const int A = std::abs(c.bodyA), B = std::abs(c.bodyB);
    uint64_t& h = w->topoHash[w->worldId[A]];
    h = mix64(h, ((uint64_t)A << 32) | (uint32_t)B);
    h = mix64(h, (uint32_t)c.pad);
    h = mix64(h, (uint64_t)(int64_t)g_axisId);
}

int col_type(const or_world* w, int col) { return w->colType.empty() ? 3 : w->colType[col]; }

inline int ibits(float f) {
    int i;
    memcpy(&i, &f, 4);
    return i;
}

// sphere-sphere branch of clipHullHullKernel (satClipHullContacts.cl:1078-1124)
bool sphere_sphere(const or_world* w, int slot, int A, int B, or_contact_r& out) {
    const Real rA = w->colRadius[w->col[A]], rB = w->colRadius[w->col[B]];
    const V pA = body_pose(w, A).pos, pB = body_pose(w, B).pos;
    const V diff = pA - pB;
    const Real len = sqrt(dot(diff, diff));
    if (!(len <= rA + rB)) return false;
    const Real dist = len - (rA + rB);
    V nB(1, 0, 0);
    if (len > 0.00001) nB = diff * (1 / len);
    const V cp = pB + nB * rB;
    out = or_contact_r();
    out.pos[0][0] = cp.x; out.pos[0][1] = cp.y; out.pos[0][2] = cp.z; out.pos[0][3] = dist;
    out.normal[0] = -nB.x; out.normal[1] = -nB.y; out.normal[2] = -nB.z; out.normal[3] = 1;
    out.friction = combine_friction(w->friction[A], w->friction[B], w->cfg.frictionCombine);
    out.pairIndex = slot;
    out.bodyA = w->invMass[A] == 0.f ? -A : A;
    out.bodyB = w->invMass[B] == 0.f ? -B : B;
    return true;
}

// computeContactPlaneConvex (satClipHullContacts.cl:957-1016) for a sphere:
// the sphere's point deepest along -n, its distance to the plane
// n . x = constant in the plane body's frame; a contact when below it. The
// manifold's A side is the plane's body, B the sphere's.
bool plane_sphere(const or_world* w, int slot, int P, int Sb, or_contact_r& out) {
    const float* pl = w->faces[w->colIndex[w->col[P]]].plane;
    const Real r = w->colRadius[w->col[Sb]];
    const Body bp = body_pose(w, P), bs = body_pose(w, Sb);
    const V n(pl[0], pl[1], pl[2]);
    const V cLocal = qinvrot(bp.q, bs.pos - bp.pos);
    const Real distance = dot(n, cLocal) - r - (Real)pl[3];
    if (!(distance < 0)) return false;
    const V nw = qrot(bp.q, n);
    const V pOnB = bs.pos - nw * r;
    out = or_contact_r();
    out.pos[0][0] = pOnB.x; out.pos[0][1] = pOnB.y; out.pos[0][2] = pOnB.z; out.pos[0][3] = distance;
    out.normal[0] = nw.x; out.normal[1] = nw.y; out.normal[2] = nw.z; out.normal[3] = 1;
    out.friction = combine_friction(w->friction[P], w->friction[Sb], w->cfg.frictionCombine);
    out.pairIndex = slot;
    out.bodyA = w->invMass[P] == 0.f ? -P : P;
    out.bodyB = w->invMass[Sb] == 0.f ? -Sb : Sb;
    return true;
}

// A sub-pair of a compound or mesh pair: bodies A and B (the manifold's
// sides) and per side either a compound child (>= 0) or, as -(poly + 1), a
// polytope at the body's own pose.
struct SubPair {
    int A, B, sa, sb;
};

// The child's pose: qtRotate(orn, childPos) + pos and qtMul(orn, childOrn)
// in FP32 (findCompoundPairsKernel, sat.cl:774-781), in the operation order
// the device uses, from the body's FP32 pose.
Body child_pose(const or_world* w, int body, int child) {
    const float p[4] = {(float)rval(w->pos[4 * body]), (float)rval(w->pos[4 * body + 1]),
                        (float)rval(w->pos[4 * body + 2]), 0.f};
    const float q[4] = {(float)rval(w->quat[4 * body]), (float)rval(w->quat[4 * body + 1]),
                        (float)rval(w->quat[4 * body + 2]), (float)rval(w->quat[4 * body + 3])};
    const float* cp = &w->childPose[8 * (size_t)child];
    const float* cq = cp + 4;
    const float v[4] = {cp[0], cp[1], cp[2], 0.f};
    const float qi[4] = {-q[0], -q[1], -q[2], q[3]};
    float t[4], r[4], o[4];
    qmul_f(q, v, t);
    qmul_f(t, qi, r);
    qmul_f(q, cq, o);
    Body b;
    b.pos = V(r[0] + p[0], r[1] + p[1], r[2] + p[2]);
    b.q = Q{o[0], o[1], o[2], o[3]};
    return b;
}

void side_of(const or_world* w, int body, int s, const or_poly*& h, Body& pose) {
    if (s >= 0) {
        h = &w->polys[w->colIndex[w->childCol[s]]];
        pose = child_pose(w, body, s);
    } else {
        h = &w->polys[-s - 1];
        pose = body_pose(w, body);
    }
}

// Sub-pairs of broadphase pair (A, B) in order: compound children (child
// of A outer, child of B inner; findCompoundPairsKernel, sat.cl:747-926,
// with no culling between children), or a mesh's triangles whose local AABB
// overlaps the hull's world AABB (findSeparatingAxisKernel, sat.cl:970-1012),
// the mesh taking side A whichever order the pair has.
void sub_pairs_of(const or_world* w, int A, int B, std::vector<SubPair>& out) {
    if (w->invMass[A] == 0.f && w->invMass[B] == 0.f) return;
    const int tA = col_type(w, w->col[A]), tB = col_type(w, w->col[B]);
    if (tA == 6 || tB == 6) {
        if ((tA != 6 && tA != 3) || (tB != 6 && tB != 3)) return;
        const int nA = tA == 6 ? w->colNum[w->col[A]] : 1;
        const int nB = tB == 6 ? w->colNum[w->col[B]] : 1;
        for (int i = 0; i < nA; ++i)
            for (int j = 0; j < nB; ++j) {
                const int sa = tA == 6 ? w->colIndex[w->col[A]] + i : -(w->colShape[w->col[A]] + 1);
                const int sb = tB == 6 ? w->colIndex[w->col[B]] + j : -(w->colShape[w->col[B]] + 1);
                out.push_back({A, B, sa, sb});
            }
        return;
    }
    int M = -1, H = -1;
    if (tA == 5 && tB == 3) M = A, H = B;
    else if (tB == 5 && tA == 3) M = B, H = A;
    if (M < 0) return;
    const or_poly& mesh = w->polys[w->colIndex[w->col[M]]];
    const float* bb = &w->aabb[8 * (size_t)H];
    for (int f = 0; f < mesh.numFaces; ++f) {
        const int tp = mesh.unused + f;
        const or_poly& t = w->polys[tp];
        float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) {
                const float v = w->verts4[4 * (size_t)(t.vertexOffset + i) + k];
                mn[k] = std::min(mn[k], v);
                mx[k] = std::max(mx[k], v);
            }
        bool overlap = true;
        overlap = (mn[0] > bb[4] || mx[0] < bb[0]) ? false : overlap;
        overlap = (mn[2] > bb[6] || mx[2] < bb[2]) ? false : overlap;
        overlap = (mn[1] > bb[5] || mx[1] < bb[1]) ? false : overlap;
        if (overlap) out.push_back({M, H, -(tp + 1), -(w->colShape[w->col[H]] + 1)});
    }
}

void stage_narrowphase(or_world* w) {
    w->contacts.clear();
    const int np = (int)w->pairs.size() / 2;
    std::vector<SubPair> subs;
    for (int p = 0; p < np; ++p) {
        const int A = w->pairs[2 * p], B = w->pairs[2 * p + 1];
        const int tA = col_type(w, w->col[A]), tB = col_type(w, w->col[B]);
        or_contact_r c;
        bool have = false;
        if (tA == 3 && tB == 3) {
            have = contact_for_pair(w, p, A, B, c);
        } else if (w->invMass[A] == 0.f && w->invMass[B] == 0.f) {
        } else if (tA == 7 && tB == 7) {
            have = sphere_sphere(w, p, A, B, c);
        } else if (tA == 7 && tB == 4) {
            have = plane_sphere(w, p, B, A, c);
        } else if (tA == 4 && tB == 7) {
            have = plane_sphere(w, p, A, B, c);
        } else {
            sub_pairs_of(w, A, B, subs);
        }
        if (have) {
            w->contacts.push_back(c);
            record_topology(w, c);
        }
    }
    // the sub-pairs' slots follow the pairs' within the pair capacity
    long long room = w->cfg.maxPairs > 0 ? (long long)w->cfg.maxPairs - np : (long long)subs.size();
    if (room < 0) room = 0;
    if ((long long)subs.size() > room) {
        w->pairOverflow += (long long)subs.size() - room;
        subs.resize((size_t)room);
    }
    for (size_t s = 0; s < subs.size(); ++s) {
        const SubPair& sp = subs[s];
        const or_poly* hA;
        const or_poly* hB;
        Body a, b;
        side_of(w, sp.A, sp.sa, hA, a);
        side_of(w, sp.B, sp.sb, hB, b);
        or_contact_r c;
        if (contact_for_shapes(w, np + (int)s, sp.A, sp.B, *hA, a, *hB, b, c)) {
            w->contacts.push_back(c);
            record_topology(w, c);
        }
    }
}

// ---------------------------------------------------------------------------
// Jacobi solver with velocity averaging (btPgsJacobiSolver, usePgs = false)
// ---------------------------------------------------------------------------
struct Row {
    V n, t1, t2;  // contactNormal, relpos1CrossNormal, relpos2CrossNormal
    Real rhs, jac, applied, lo, hi, mu;
    int normalIndex;  // friction rows: index of their normal row
};
struct Copy {
    int body;  // -1 for the shared static solver body
    V dv, dw;
};
struct MRows {
    int a, b;      // copy indices
    int A, B;      // body ids
    int nNormal;
    std::vector<Row> normal, fric;
};

void plane_space(V n, V& p, V& q) {
    const Real SQRT12 = 0.7071067811865475244008443621048490;
    if (fabs(n.z) > SQRT12) {
        const Real a = n.y * n.y + n.z * n.z;
        const Real k = 1.0 / sqrt(a);
        p = V(0, -n.z * k, n.y * k);
        q = V(a * k, -n.x * p.z, n.x * p.y);
    } else {
        const Real a = n.x * n.x + n.y * n.y;
        const Real k = 1.0 / sqrt(a);
        p = V(-n.y * k, n.x * k, 0);
        q = V(-n.z * p.y, n.z * p.x, a * k);
    }
}

int solve_row(Row& c, Copy& A, Copy& B, Real imA, Real imB, V iiA, V iiB) {
    int state = 0;
    Real delta = c.rhs;  // - applied * cfm (0)
    const Real dv1 = dot(c.n, A.dv) + dot(c.t1, A.dw);
    const Real dv2 = -dot(c.n, B.dv) + dot(c.t2, B.dw);
    delta -= dv1 * c.jac;
    delta -= dv2 * c.jac;
    const Real sum = c.applied + delta;
    if (sum < c.lo) {
        delta = c.lo - c.applied;
        c.applied = c.lo;
        state = 1;
    } else if (sum > c.hi) {
        delta = c.hi - c.applied;
        c.applied = c.hi;
        state = 2;
    } else {
        c.applied = sum;
    }
    A.dv = A.dv + c.n * (imA * delta);
    A.dw = A.dw + mulv(iiA, c.t1) * delta;
    B.dv = B.dv + (-c.n * imB) * delta;
    B.dw = B.dw + mulv(iiB, c.t2) * delta;
    return state;
}


// ---------------------------------------------------------------------------
// Batched Gauss-Seidel solver: the reference's GPU solver
// (P1/btGpuNarrowPhaseAndSolver.cpp:1073-1353 driving ST/Solver.cpp), in
// FP64. Structure followed: contacts binned to a 16 x 16 xz grid of cells
// (SetSortDataKernel, ST/solverSetup2.cl:457-478), cells solved in four
// parity classes (BatchSolveKernelContact, ST/solveContact.cl:418-426),
// batches of constraints without a shared dynamic body solved one after
// another, four contact iterations then four friction iterations
// (ST/Solver.cpp:561-700), Constraint4 set up by setConstraint4
// (ST/solverSetup.cl:520-609). The colouring is the sequential greedy pass
// of the reference's CPU batching (sortConstraintByBatch,
// P1/btGpuNarrowPhaseAndSolver.cpp:752-852) run over each parity class in
// (cell, manifold) order with exact body identities, so that no dynamic
// body appears twice in a batch anywhere in the class (the reference's GPU
// colouring is per cell, with atomics, and races on bodies shared by
// concurrently solved cells). Static means inverse mass 0.
// ---------------------------------------------------------------------------
namespace gs {

constexpr int kSplit = 16;          // SolverBase::N_SPLIT
constexpr int kIterations = 4;      // m_nIterations (:1330)
constexpr float kScale = 0.5f;      // 1 / (N_OBJ_PER_SPLIT * m_averageExtent) = 1 / (10 * 0.2)
constexpr double kFriction = 0.7;   // m_linear.w (solverSetup.cl:541), solveFriction.cl:319
constexpr double kDrift = 0.005;    // ConstraintCfg::m_positionDrift
constexpr double kPosCoeff = 0.2;   // ConstraintCfg::m_positionConstraintCoeff

struct M3 {
    V r[3];
};
inline V mul(const M3& m, V v) { return V(dot(m.r[0], v), dot(m.r[1], v), dot(m.r[2], v)); }

struct C4 {  // Constraint4 (ST/AdlConstraint4.h:23-47) in Real
    V linear;
    V worldPos[4];
    V center;
    Real jacCoeffInv[4], b[4], applied[4];
    Real fJacCoeffInv[2], fApplied[2];
    int A, B;
};

// world inverse inertia R diag(I^-1) R^T (setupBodiesKernel,
// broadphaseKernel.cl:189-201); static bodies have none
M3 world_inv_inertia(const or_world* w, int i) {
    M3 m;
    if (w->invMass[i] == 0.f) return m;
    const Q q = {w->quat[4 * i], w->quat[4 * i + 1], w->quat[4 * i + 2], w->quat[4 * i + 3]};
    const V c0 = qrot(q, V(1, 0, 0)), c1 = qrot(q, V(0, 1, 0)), c2 = qrot(q, V(0, 0, 1));
    const V d(w->invInertia[3 * i], w->invInertia[3 * i + 1], w->invInertia[3 * i + 2]);
    const V rows[3] = {V(c0.x, c1.x, c2.x), V(c0.y, c1.y, c2.y), V(c0.z, c1.z, c2.z)};
    for (int a = 0; a < 3; ++a) m.r[a] = V(dot(mulv(rows[a], d), rows[0]), dot(mulv(rows[a], d), rows[1]),
                                          dot(mulv(rows[a], d), rows[2]));
    return m;
}

// btPlaneSpace1 (solverSetup.cl:477-501)
void plane_space1(V n, V& p, V& q) {
    if (fabs(n.z) > 0.70710678) {
        const Real a = n.y * n.y + n.z * n.z;
        const Real k = 1.0 / sqrt(a);
        p = V(0, -n.z * k, n.y * k);
        q = V(a * k, -n.x * p.z, n.x * p.y);
    } else {
        const Real a = n.x * n.x + n.y * n.y;
        const Real k = 1.0 / sqrt(a);
        p = V(-n.y * k, n.x * k, 0);
        q = V(-n.z * p.y, n.z * p.x, a * k);
    }
}

// calcJacCoeff (solverSetup.cl:445-454) with setLinearAndAngular's angular
// parts; the inverse inertias are symmetric, so a^T I = I a
Real jac_coeff(V ang0, V ang1, Real imA, const M3& IA, Real imB, const M3& IB) {
    return -1.0 / (imA + dot(mul(IA, ang0), ang0) + imB + dot(mul(IB, ang1), ang1));
}

// setConstraint4 (solverSetup.cl:520-609), restitution 0
C4 set_constraint(const or_contact_r& c, V posA, V linA, V angA, Real imA, const M3& IA, V posB, V linB, V angB,
                  Real imB, const M3& IB, Real dt) {
    C4 d;
    d.A = std::abs(c.bodyA);
    d.B = std::abs(c.bodyB);
    const V n(c.normal[0], c.normal[1], c.normal[2]);
    const int np = (int)rval(c.normal[3]);
    d.linear = -n;
    for (int i = 0; i < 4; ++i) {
        d.applied[i] = 0;
        d.jacCoeffInv[i] = 0;
        d.b[i] = 0;
        d.worldPos[i] = V();
    }
    d.fJacCoeffInv[0] = d.fJacCoeffInv[1] = 0;
    d.fApplied[0] = d.fApplied[1] = 0;
    for (int ic = 0; ic < 4 && ic < np; ++ic) {
        const V p(c.pos[ic][0], c.pos[ic][1], c.pos[ic][2]);
        const V r0 = p - posA, r1 = p - posB;
        const V ang0 = -cross(r0, n), ang1 = cross(r1, n);
        d.jacCoeffInv[ic] = jac_coeff(ang0, ang1, imA, IA, imB, IB);
        // restitution e = 0: m_b is the position term alone
        d.b[ic] = (c.pos[ic][3] + kDrift) * kPosCoeff / dt;
        d.worldPos[ic] = p;
    }
    V center;
    for (int i = 0; i < np; ++i) center = center + V(c.pos[i][0], c.pos[i][1], c.pos[i][2]);
    center = center * (1.0 / (Real)np);
    V t[2];
    plane_space1(n, t[0], t[1]);
    for (int i = 0; i < 2; ++i) {
        const V ang0 = -cross(center - posA, t[i]), ang1 = cross(center - posB, t[i]);
        d.fJacCoeffInv[i] = jac_coeff(ang0, ang1, imA, IA, imB, IB);
    }
    d.center = center;
    (void)linA; (void)angA; (void)linB; (void)angB;
    return d;
}

struct BodyVel {
    V lin, ang;
};

// solveContact (solveContact.cl:272-309), accumulated impulse clamped to [0, inf)
void solve_contact(C4& cs, V posA, BodyVel& a, Real imA, const M3& IA, V posB, BodyVel& b, Real imB, const M3& IB) {
    const V n = -cs.linear;  // the argument -m_linear of setLinearAndAngular
    for (int ic = 0; ic < 4; ++ic) {
        if (cs.jacCoeffInv[ic] == 0) continue;
        const V r0 = cs.worldPos[ic] - posA, r1 = cs.worldPos[ic] - posB;
        const V lin = -n, ang0 = -cross(r0, n), ang1 = cross(r1, n);
        Real l = dot(cs.linear, a.lin) + dot(ang0, a.ang) + dot(-cs.linear, b.lin) + dot(ang1, b.ang) + cs.b[ic];
        l = l * cs.jacCoeffInv[ic];
        const Real prev = cs.applied[ic];
        Real upd = prev + l;
        if (upd < 0) upd = 0;
        l = upd - prev;
        cs.applied[ic] = upd;
        a.lin = a.lin + lin * (imA * l);
        b.lin = b.lin + (-lin) * (imB * l);
        a.ang = a.ang + mul(IA, ang0) * l;
        b.ang = b.ang + mul(IB, ang1) * l;
    }
}

// solveFrictionConstraint (solveFriction.cl:297-391): limits 0.7 times the
// sum of the contact impulses, then the angular damping about the normal
void solve_friction(C4& cs, V posA, BodyVel& a, Real imA, const M3& IA, V posB, BodyVel& b, Real imB, const M3& IB) {
    Real sum = 0;
    for (int j = 0; j < 4; ++j) sum = sum + cs.applied[j];
    const Real maxR = kFriction * sum, minR = -maxR;
    const V n = -cs.linear;
    V t[2];
    plane_space1(n, t[0], t[1]);
    const V r0 = cs.center - posA, r1 = cs.center - posB;
    for (int i = 0; i < 2; ++i) {
        const V lin = -t[i], ang0 = -cross(r0, t[i]), ang1 = cross(r1, t[i]);
        Real l = dot(lin, a.lin) + dot(ang0, a.ang) + dot(-lin, b.lin) + dot(ang1, b.ang);
        l = l * cs.fJacCoeffInv[i];
        const Real prev = cs.fApplied[i];
        Real upd = prev + l;
        if (upd < minR) upd = minR;
        if (upd > maxR) upd = maxR;
        l = upd - prev;
        cs.fApplied[i] = upd;
        a.lin = a.lin + lin * (imA * l);
        b.lin = b.lin + (-lin) * (imB * l);
        a.ang = a.ang + mul(IA, ang0) * l;
        b.ang = b.ang + mul(IB, ang1) * l;
    }
    const V ab = normalize(posB - posA), ac = normalize(cs.center - posA);
    if (dot(ab, ac) > 0.95 || imA == 0 || imB == 0) {
        const Real angNA = dot(n, a.ang), angNB = dot(n, b.ang);
        a.ang = a.ang - n * (angNA * 0.1);
        b.ang = b.ang - n * (angNB * 0.1);
    }
}

// cell of a manifold: the xz position of its dynamic body (A unless A is
// static), in FP32 as SetSortDataKernel computes it
int cell_of(const or_world* w, const or_contact_r& c) {
    const int A = std::abs(c.bodyA), B = std::abs(c.bodyB);
    const int body = w->invMass[A] != 0.f ? A : B;
    const float px = (float)w->pos[4 * body], pz = (float)w->pos[4 * body + 2];
    const int xi = (int)((px - (px < 0.f ? 1.f : 0.f)) * kScale) & (kSplit - 1);
    const int zi = (int)((pz - (pz < 0.f ? 1.f : 0.f)) * kScale) & (kSplit - 1);
    return xi + zi * kSplit;
}
inline int class_of(int cell) { return (cell & 1) + 2 * ((cell / kSplit) & 1); }

}  // namespace gs

void stage_solve_gs(or_world* w) {
    using namespace gs;
    const int N = w->n;
    const int M = (int)w->contacts.size();
    w->count.clear();  // integration applies no Jacobi averages
    w->gsCell.assign(M, 0);
    w->gsBatch.assign(M, -1);
    for (int m = 0; m < M; ++m) w->gsCell[m] = cell_of(w, w->contacts[m]);
    // each parity class in (cell, manifold) order
    std::vector<int> order(M);
    for (int m = 0; m < M; ++m) order[m] = m;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const int ka = class_of(w->gsCell[a]) * 256 + w->gsCell[a];
        const int kb = class_of(w->gsCell[b]) * 256 + w->gsCell[b];
        return ka < kb;
    });
    // greedy colouring per class (sortConstraintByBatch's pass, exact bodies)
    int nb[4] = {0, 0, 0, 0};
    std::vector<int> stamp(N, -1);
    for (int cls = 0; cls < 4; ++cls) {
        std::vector<int> rem;
        for (int m : order)
            if (class_of(w->gsCell[m]) == cls) rem.push_back(m);
        int b = 0;
        while (!rem.empty()) {
            std::vector<int> next;
            for (int m : rem) {
                const int A = std::abs(w->contacts[m].bodyA), B = std::abs(w->contacts[m].bodyB);
                const bool dA = w->invMass[A] != 0.f, dB = w->invMass[B] != 0.f;
                if ((!dA || stamp[A] != b) && (!dB || stamp[B] != b)) {
                    w->gsBatch[m] = b;
                    if (dA) stamp[A] = b;
                    if (dB) stamp[B] = b;
                } else {
                    next.push_back(m);
                }
            }
            rem.swap(next);
            ++b;
            // stamps of this pass must not alias the next class' batch 0
            if (rem.empty()) std::fill(stamp.begin(), stamp.end(), -1);
        }
        nb[cls] = b;
    }
    if (M == 0) return;
    // constraints, bodies' state at the solve
    std::vector<M3> Iw(N);
    for (int i = 0; i < N; ++i) Iw[i] = world_inv_inertia(w, i);
    auto posv = [&](int i) { return V(w->pos[4 * i], w->pos[4 * i + 1], w->pos[4 * i + 2]); };
    std::vector<BodyVel> vel(N);
    for (int i = 0; i < N; ++i) {
        if (w->invMass[i] == 0.f) continue;  // static bodies move with zero velocity
        vel[i].lin = V(w->lin[4 * i], w->lin[4 * i + 1], w->lin[4 * i + 2]);
        vel[i].ang = V(w->ang[4 * i], w->ang[4 * i + 1], w->ang[4 * i + 2]);
    }
    std::vector<C4> cs(M);
    for (int m = 0; m < M; ++m) {
        const or_contact_r& c = w->contacts[m];
        const int A = std::abs(c.bodyA), B = std::abs(c.bodyB);
        cs[m] = set_constraint(c, posv(A), vel[A].lin, vel[A].ang, (Real)w->invMass[A], Iw[A], posv(B), vel[B].lin,
                               vel[B].ang, (Real)w->invMass[B], Iw[B], (Real)w->cfg.dt);
    }
    // (class, batch) lists in class order
    std::vector<std::vector<int>> lists;
    for (int cls = 0; cls < 4; ++cls)
        for (int b = 0; b < nb[cls]; ++b) {
            std::vector<int> l;
            for (int m : order)
                if (class_of(w->gsCell[m]) == cls && w->gsBatch[m] == b) l.push_back(m);
            lists.push_back(l);
        }
    for (int phase = 0; phase < 2; ++phase)
        for (int it = 0; it < kIterations; ++it)
            for (const std::vector<int>& l : lists)
                for (int m : l) {
                    C4& c = cs[m];
                    const int A = c.A, B = c.B;
                    const Real imA = w->invMass[A], imB = w->invMass[B];
                    BodyVel a = vel[A], b = vel[B];
                    if (phase == 0) solve_contact(c, posv(A), a, imA, Iw[A], posv(B), b, imB, Iw[B]);
                    else solve_friction(c, posv(A), a, imA, Iw[A], posv(B), b, imB, Iw[B]);
                    // a static body's velocity is written as zero
                    vel[A] = imA != 0 ? a : BodyVel();
                    vel[B] = imB != 0 ? b : BodyVel();
                }
    w->gsApplied.assign(6 * (size_t)M, 0.0);
    for (int m = 0; m < M; ++m) {
        for (int k = 0; k < 4; ++k) w->gsApplied[6 * m + k] = rval(cs[m].applied[k]);
        for (int k = 0; k < 2; ++k) w->gsApplied[6 * m + 4 + k] = rval(cs[m].fApplied[k]);
    }
    for (int i = 0; i < N; ++i) {
        if (w->invMass[i] == 0.f) continue;
        w->lin[4 * i] = vel[i].lin.x; w->lin[4 * i + 1] = vel[i].lin.y; w->lin[4 * i + 2] = vel[i].lin.z;
        w->ang[4 * i] = vel[i].ang.x; w->ang[4 * i + 1] = vel[i].ang.y; w->ang[4 * i + 2] = vel[i].ang.z;
    }
}

void stage_solve(or_world* w) {
    if (w->gs) {
        stage_solve_gs(w);
        return;
    }
    const int N = w->n;
    const int M = (int)w->contacts.size();
    const Real dt = w->cfg.dt;
    // m_bodyCount (:1105-1129)
    w->count.assign(N, 0);
    for (const or_contact_r& c : w->contacts) {
        const int A = std::abs(c.bodyA), B = std::abs(c.bodyB);
        if (w->invMass[A] != 0.f) w->count[A]++;
        if (w->invMass[B] != 0.f) w->count[B]++;
    }
    std::vector<Copy> copies;
    std::vector<int> staticCopy(N, -1);
    auto get_copy = [&](int body) {
        if (w->invMass[body] == 0.f) {
            if (staticCopy[body] < 0) {
                staticCopy[body] = (int)copies.size();
                copies.push_back({-1, V(), V()});
            }
            return staticCopy[body];
        }
        copies.push_back({body, V(), V()});
        return (int)copies.size() - 1;
    };
    std::vector<MRows> ms;
    ms.reserve(M);
    for (const or_contact_r& c : w->contacts) {
        MRows m;
        m.A = std::abs(c.bodyA);
        m.B = std::abs(c.bodyB);
        m.a = get_copy(m.A);
        m.b = get_copy(m.B);
        const bool dynA = w->invMass[m.A] != 0.f, dynB = w->invMass[m.B] != 0.f;
        if (!dynA && !dynB) {
            ms.push_back(m);
            continue;
        }
        const Real imA = w->invMass[m.A], imB = w->invMass[m.B];
        const V iiA = dynA ? V(w->invInertia[3 * m.A], w->invInertia[3 * m.A + 1], w->invInertia[3 * m.A + 2]) : V();
        const V iiB = dynB ? V(w->invInertia[3 * m.B], w->invInertia[3 * m.B + 1], w->invInertia[3 * m.B + 2]) : V();
        const Real kA = dynA ? (Real)w->count[m.A] : 1.0, kB = dynB ? (Real)w->count[m.B] : 1.0;
        const V pA(w->pos[4 * m.A], w->pos[4 * m.A + 1], w->pos[4 * m.A + 2]);
        const V pB(w->pos[4 * m.B], w->pos[4 * m.B + 1], w->pos[4 * m.B + 2]);
        const V vA = dynA ? V(w->lin[4 * m.A], w->lin[4 * m.A + 1], w->lin[4 * m.A + 2]) : V();
        const V wA = dynA ? V(w->ang[4 * m.A], w->ang[4 * m.A + 1], w->ang[4 * m.A + 2]) : V();
        const V vB = dynB ? V(w->lin[4 * m.B], w->lin[4 * m.B + 1], w->lin[4 * m.B + 2]) : V();
        const V wB = dynB ? V(w->ang[4 * m.B], w->ang[4 * m.B + 1], w->ang[4 * m.B + 2]) : V();
        const Real restitution = (Real)w->restitution[m.A] * (Real)w->restitution[m.B];
        const V n = normalize(V(-c.normal[0], -c.normal[1], -c.normal[2]));
        const int npts = (int)rval(c.normal[3]);
        for (int j = 0; j < npts; ++j) {
            const Real dist = c.pos[j][3] + (Real)w->cfg.slopOffset;
            if (!(dist <= (Real)w->cfg.contactProcessing)) continue;
            const V posB(c.pos[j][0], c.pos[j][1], c.pos[j][2]);
            const V posA = posB + n * dist;
            const V r1 = posA - pA, r2 = posB - pB;
            const V t0 = cross(r1, n), t1 = cross(r2, n);
            const V angA = mulv(iiA, t0), angB = mulv(iiB, -t1);
            const Real d0 = imA + dot(n, cross(angA, r1));
            const Real d1 = imB + dot(n, cross(-angB, r2));
            Row row;
            row.n = n;
            row.t1 = t0;
            row.t2 = -t1;
            row.jac = 1.0 / (d0 + d1);
            const Real scaled = 1.0 / (d0 * kA + d1 * kB);
            const Real penetration = dist;
            const V vel = (vA + cross(wA, r1)) - (vB + cross(wB, r2));
            const Real relv0 = dot(n, vel);
            Real rest = restitution * -relv0;
            if (rest <= 0) rest = 0;
            const Real relv = (dot(n, vA) + dot(t0, wA)) + (-dot(n, vB) + dot(-t1, wB));
            Real posErr = 0, velErr = rest - relv;
            if (penetration > 0) velErr -= penetration / dt;
            else posErr = -penetration * (Real)w->cfg.erp / dt;
            row.rhs = posErr * scaled + velErr * scaled;
            row.applied = 0;
            row.lo = 0;
            row.hi = 1e10;
            row.mu = c.friction;
            row.normalIndex = -1;
            const int ni = (int)m.normal.size();
            m.normal.push_back(row);
            V d1v = vel - n * relv0, d2v;
            const Real lat = dot(d1v, d1v);
            // the setup's own branches belong to the active set too
            w->activeHash[w->worldId[m.A]] = mix64(w->activeHash[w->worldId[m.A]],
                                                   16 + (penetration > 0 ? 1 : 0) + (rest > 0 ? 2 : 0) +
                                                       (lat > (Real)FLT_EPSILON ? 4 : 0) + 8 * j);
            if (lat > (Real)FLT_EPSILON) {
                d1v = d1v * (1.0 / sqrt(lat));
                d2v = normalize(cross(d1v, n));
            } else {
                plane_space(n, d1v, d2v);
            }
            const V dirs[2] = {d2v, d1v};
            for (int q = 0; q < 2; ++q) {
                const V dir = dirs[q];
                Row f;
                f.n = dir;
                f.t1 = cross(r1, dir);
                f.t2 = cross(r2, -dir);
                const V aA = mulv(iiA, f.t1), aB = mulv(iiB, f.t2);
                const Real e0 = imA + dot(dir, cross(aA, r1));
                const Real e1 = imB + dot(dir, cross(-aB, r2));
                f.jac = 1.0 / (e0 + e1);
                const Real sc = 1.0 / (e0 * kA + e1 * kB);
                const Real rv = (dot(dir, vA) + dot(f.t1, wA)) + (-dot(dir, vB) + dot(f.t2, wB));
                f.rhs = (0 - rv) * sc;
                f.applied = 0;
                f.lo = 0;
                f.hi = 1e10;
                f.mu = c.friction;
                f.normalIndex = ni;
                m.fric.push_back(f);
            }
        }
        ms.push_back(m);
    }
    // iterations
    std::vector<V> sumL(N), sumA(N);
    auto average = [&]() {
        for (int i = 0; i < N; ++i) sumL[i] = sumA[i] = V();
        for (const Copy& cp : copies)
            if (cp.body >= 0) {
                sumL[cp.body] = sumL[cp.body] + cp.dv;
                sumA[cp.body] = sumA[cp.body] + cp.dw;
            }
        for (Copy& cp : copies)
            if (cp.body >= 0) {
                const Real f = 1.0 / (Real)w->count[cp.body];
                cp.dv = sumL[cp.body] * f;
                cp.dw = sumA[cp.body] * f;
            }
    };
    for (int it = 0; it < w->cfg.iterations; ++it) {
        for (MRows& m : ms) {
            const Real imA = w->invMass[m.A], imB = w->invMass[m.B];
            const bool dynA = imA != 0, dynB = imB != 0;
            const V iiA = dynA ? V(w->invInertia[3 * m.A], w->invInertia[3 * m.A + 1], w->invInertia[3 * m.A + 2]) : V();
            const V iiB = dynB ? V(w->invInertia[3 * m.B], w->invInertia[3 * m.B + 1], w->invInertia[3 * m.B + 2]) : V();
            uint64_t& h = w->activeHash[w->worldId[m.A]];
            for (Row& r : m.normal) h = mix64(h, (uint64_t)solve_row(r, copies[m.a], copies[m.b], imA, imB, iiA, iiB));
        }
        average();
        for (MRows& m : ms) {
            const Real imA = w->invMass[m.A], imB = w->invMass[m.B];
            const bool dynA = imA != 0, dynB = imB != 0;
            const V iiA = dynA ? V(w->invInertia[3 * m.A], w->invInertia[3 * m.A + 1], w->invInertia[3 * m.A + 2]) : V();
            const V iiB = dynB ? V(w->invInertia[3 * m.B], w->invInertia[3 * m.B + 1], w->invInertia[3 * m.B + 2]) : V();
            uint64_t& h = w->activeHash[w->worldId[m.A]];
            for (Row& r : m.fric) {
                const Real total = m.normal[r.normalIndex].applied;
                if (total > 0) {
                    r.lo = -(r.mu * total);
                    r.hi = r.mu * total;
                    h = mix64(h, 4 + (uint64_t)solve_row(r, copies[m.a], copies[m.b], imA, imB, iiA, iiB));
                } else {
                    h = mix64(h, 8);
                }
            }
        }
        average();
    }
    // finish: per copy, body velocity += sum / count (:1790-1803)
    w->avgLin.assign(3 * (size_t)N, 0);
    w->avgAng.assign(3 * (size_t)N, 0);
    for (int i = 0; i < N; ++i)
        if (w->count[i] > 0) {
            const Real f = 1.0 / (Real)w->count[i];
            w->avgLin[3 * i] = sumL[i].x * f;
            w->avgLin[3 * i + 1] = sumL[i].y * f;
            w->avgLin[3 * i + 2] = sumL[i].z * f;
            w->avgAng[3 * i] = sumA[i].x * f;
            w->avgAng[3 * i + 1] = sumA[i].y * f;
            w->avgAng[3 * i + 2] = sumA[i].z * f;
        }
    if (w->cfg.iterations == 0) {
        w->avgLin.assign(3 * (size_t)N, 0);
        w->avgAng.assign(3 * (size_t)N, 0);
    }
}

// integrateTransformsKernel2 (integrateKernel.cl:102-158) after copyVelocities
void stage_integrate(or_world* w) {
    const Real dt = w->cfg.dt;
    const Real thr = 0.25 * 3.14159254f;
    for (int i = 0; i < w->n; ++i) {
        if (w->invMass[i] == 0.f) continue;
        Real* v = &w->lin[4 * i];
        Real* a = &w->ang[4 * i];
        if (!w->count.empty() && w->count[i] > 0) {
            for (int c = 0; c < w->count[i]; ++c)
                for (int k = 0; k < 3; ++k) {
                    v[k] += w->avgLin[3 * i + k];
                    a[k] += w->avgAng[3 * i + k];
                }
        }
        for (int k = 0; k < 3; ++k) a[k] *= (Real)w->cfg.angularDamping;
        Real fAngle = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (fAngle * dt > thr) fAngle = thr / dt;
        Real s;
        if (fAngle < 0.001) s = 0.5 * dt - (dt * dt * dt) * 0.020833333333 * fAngle * fAngle;
        else s = sin(0.5 * fAngle * dt) / fAngle;
        const Real dq[4] = {a[0] * s, a[1] * s, a[2] * s, cos(fAngle * dt * 0.5)};
        Real* q = &w->quat[4 * i];
        Real r[4];
        r[0] = dq[3] * q[0] + dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1];
        r[1] = dq[3] * q[1] + dq[1] * q[3] + dq[2] * q[0] - dq[0] * q[2];
        r[2] = dq[3] * q[2] + dq[2] * q[3] + dq[0] * q[1] - dq[1] * q[0];
        r[3] = dq[3] * q[3] - dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2];
        const Real len = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
        if (len > 0) for (int k = 0; k < 4; ++k) q[k] = r[k] / len;
        else { q[0] = q[1] = q[2] = 0; q[3] = 1; }
        for (int k = 0; k < 3; ++k) w->pos[4 * i + k] += v[k] * dt;
    }
}

int ilog2(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) ++b;
    return b;
}

}  // namespace

extern "C" {

or_world* or_world_create(const or_config* cfg, int n, const float* invMass, const float* friction,
                          const float* restitution, const int* collidable, const int* worldId,
                          const int* isLarge, const float* invInertia4, int numCols, const int* colShape,
                          int numPolys, const or_poly* polys, int numVerts, const float* verts4, int numFaces,
                          const or_face* faces, int numIndices, const int* indices, int numEdges,
                          const float* edges4, const float* localAabb8) {
    or_world* w = new or_world();
    w->cfg = *cfg;
    w->n = n;
    w->cellBits = ilog2((uint64_t)cfg->dims[0] * cfg->dims[1] * cfg->dims[2]);
    w->invMass.assign(invMass, invMass + n);
    w->friction.assign(friction, friction + n);
    w->restitution.assign(restitution, restitution + n);
    w->col.assign(collidable, collidable + n);
    w->worldId.assign(worldId, worldId + n);
    w->activeHash.assign(std::max(1, cfg->numWorlds), 0ull);
    w->topoHash.assign(std::max(1, cfg->numWorlds), 0ull);
    w->isLarge.assign(isLarge, isLarge + n);
    w->invInertia.resize(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) w->invInertia[3 * i + k] = invInertia4[4 * i + k];
    w->colShape.assign(colShape, colShape + numCols);
    w->polys.assign(polys, polys + numPolys);
    w->verts4.assign(verts4, verts4 + 4 * (size_t)numVerts);
    w->faces.assign(faces, faces + numFaces);
    w->indices.assign(indices, indices + numIndices);
    w->edges4.assign(edges4, edges4 + 4 * (size_t)numEdges);
    w->localAabb8.assign(localAabb8, localAabb8 + 8 * (size_t)numCols);
    w->pos.assign(4 * (size_t)n, 0);
    w->quat.assign(4 * (size_t)n, 0);
    w->lin.assign(4 * (size_t)n, 0);
    w->ang.assign(4 * (size_t)n, 0);
    return w;
}

void or_world_destroy(or_world* w) { delete w; }

// The collidable table of a scene with shapes other than hulls: per
// collidable its type (B3_SHAPE_*), radius, child count and shape index,
// and the compounds' children (pose: position xyzw, orientation xyzw; the
// child's collidable).
void or_set_collidables(or_world* w, int numCols, const int* type, const float* radius, const int* numChildren,
                        const int* shapeIndex, int numChild, const float* childPose8, const int* childCol) {
    w->colType.assign(type, type + numCols);
    w->colRadius.assign(radius, radius + numCols);
    w->colNum.assign(numChildren, numChildren + numCols);
    w->colIndex.assign(shapeIndex, shapeIndex + numCols);
    w->childPose.assign(childPose8, childPose8 + 8 * (size_t)numChild);
    w->childCol.assign(childCol, childCol + numChild);
}

// FP64 body parameters (finite differences need perturbations finer than
// FP32 inputs resolve): inverse masses, friction coefficients and local
// inverse inertia diagonals (3 per body); NULL leaves a set unchanged.
void or_set_params_f64(or_world* w, const double* invMass, const double* friction, const double* invInertia3) {
    for (int i = 0; i < w->n; ++i) {
        if (invMass) w->invMass[i] = (Real)invMass[i];
        if (friction) w->friction[i] = (Real)friction[i];
        if (invInertia3)
            for (int k = 0; k < 3; ++k) w->invInertia[3 * i + k] = (Real)invInertia3[3 * i + k];
    }
}

// Per-world signatures of the discrete choices since the last reset:
// out[2k] = contact topology, out[2k+1] = row clamp states.
void or_active_hash(or_world* w, uint64_t* out, int numWorlds) {
    for (int k = 0; k < numWorlds && k < (int)w->activeHash.size(); ++k) {
        out[2 * k] = w->topoHash[k];
        out[2 * k + 1] = w->activeHash[k];
    }
}
void or_reset_active(or_world* w) {
    std::fill(w->activeHash.begin(), w->activeHash.end(), 0ull);
    std::fill(w->topoHash.begin(), w->topoHash.end(), 0ull);
}

void or_set_state_f32(or_world* w, const float* pos4, const float* quat4, const float* lin4, const float* ang4) {
    for (size_t i = 0; i < 4 * (size_t)w->n; ++i) {
        if (pos4) w->pos[i] = pos4[i];
        if (quat4) w->quat[i] = quat4[i];
        if (lin4) w->lin[i] = lin4[i];
        if (ang4) w->ang[i] = ang4[i];
    }
}
void or_set_state_f64(or_world* w, const double* pos4, const double* quat4, const double* lin4, const double* ang4) {
    for (size_t i = 0; i < 4 * (size_t)w->n; ++i) {
        if (pos4) w->pos[i] = pos4[i];
        if (quat4) w->quat[i] = quat4[i];
        if (lin4) w->lin[i] = lin4[i];
        if (ang4) w->ang[i] = ang4[i];
    }
}
void or_get_state(or_world* w, double* pos4, double* quat4, double* lin4, double* ang4) {
    for (size_t i = 0; i < 4 * (size_t)w->n; ++i) {
        if (pos4) pos4[i] = rval(w->pos[i]);
        if (quat4) quat4[i] = rval(w->quat[i]);
        if (lin4) lin4[i] = rval(w->lin[i]);
        if (ang4) ang4[i] = rval(w->ang[i]);
    }
}

// Tangent-linear build: derivative seeds of the initial velocities and of
// the body parameters (NULL leaves a set at zero derivative), and the
// derivatives of the state after the steps. The FP64 and FP32 builds carry
// no derivatives (set is a no-op, get returns zeros).
void or_set_tangent(or_world* w, const double* dlin4, const double* dang4, const double* dInvMass,
                    const double* dInvInertia3, const double* dFriction) {
    for (int i = 0; i < w->n; ++i) {
        for (int k = 0; k < 4; ++k) {
            set_tan(w->pos[4 * i + k], 0.0);
            set_tan(w->quat[4 * i + k], 0.0);
            set_tan(w->lin[4 * i + k], dlin4 ? dlin4[4 * i + k] : 0.0);
            set_tan(w->ang[4 * i + k], dang4 ? dang4[4 * i + k] : 0.0);
        }
        set_tan(w->invMass[i], dInvMass ? dInvMass[i] : 0.0);
        set_tan(w->friction[i], dFriction ? dFriction[i] : 0.0);
        for (int k = 0; k < 3; ++k) set_tan(w->invInertia[3 * i + k], dInvInertia3 ? dInvInertia3[3 * i + k] : 0.0);
    }
}
// Derivative seeds of the pose (position and quaternion, n x 4 each), set
// after or_set_tangent (which zeroes them): with them a run continues a
// tangent from any state, e.g. one step at a time along another trajectory.
void or_set_tangent_pose(or_world* w, const double* dpos4, const double* dquat4) {
    for (size_t i = 0; i < 4 * (size_t)w->n; ++i) {
        if (dpos4) set_tan(w->pos[i], dpos4[i]);
        if (dquat4) set_tan(w->quat[i], dquat4[i]);
    }
}
void or_get_tangent(or_world* w, double* dpos4, double* dquat4, double* dlin4, double* dang4) {
    for (size_t i = 0; i < 4 * (size_t)w->n; ++i) {
        if (dpos4) dpos4[i] = rtan(w->pos[i]);
        if (dquat4) dquat4[i] = rtan(w->quat[i]);
        if (dlin4) dlin4[i] = rtan(w->lin[i]);
        if (dang4) dang4[i] = rtan(w->ang[i]);
    }
}
// 0 = FP64, 1 = FP32, 2 = FP64 with tangents
int or_real_kind() {
#ifdef ORACLE_DUAL
    return 2;
#else
    return sizeof(Real) == 4 ? 1 : 0;
#endif
}

void or_stage_aabbs(or_world* w) { stage_aabbs(w); }
// 0 = uniform grid (default), 1 = sweep and prune
void or_set_broadphase(or_world* w, int kind) { w->sap = kind == 1 ? 1 : 0; }
// solver: 0 = Jacobi with velocity averaging, 1 = batched Gauss-Seidel
void or_set_solver(or_world* w, int kind) { w->gs = kind == 1 ? 1 : 0; }
// per manifold (in contact order) its cell and batch from the last
// batched Gauss-Seidel solve; returns the manifold count
int or_gs_batches(or_world* w, int* cellBatch2, int max) {
    const int n = (int)w->gsBatch.size();
    for (int m = 0; m < n && m < max; ++m) {
        cellBatch2[2 * m] = w->gsCell[m];
        cellBatch2[2 * m + 1] = w->gsBatch[m];
    }
    return n;
}
// per manifold the accumulated impulses of the last batched Gauss-Seidel
// solve: normal [4], friction [2]; returns the manifold count
int or_gs_applied(or_world* w, double* out6, int max) {
    const int n = (int)w->gsApplied.size() / 6;
    for (int m = 0; m < n && m < max; ++m)
        for (int k = 0; k < 6; ++k) out6[6 * m + k] = w->gsApplied[6 * m + k];
    return n;
}
// setConstraint4 on one manifold given the bodies' state (for pinning the
// restatement against recorded constraints): out = jacCoeffInv[4], b[4],
// center[3], fJacCoeffInv[2]
void or_gs_constraint(const double* pos4x4, const double* normal4, const double* posA3, const double* posB3,
                      double invMassA, double invMassB, const double* invInertiaA9, const double* invInertiaB9,
                      double dt, double* out13) {
    or_contact_r c = {};
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 4; ++k) c.pos[i][k] = pos4x4[4 * i + k];
    for (int k = 0; k < 4; ++k) c.normal[k] = normal4[k];
    gs::M3 IA, IB;
    for (int r = 0; r < 3; ++r) {
        IA.r[r] = V(invInertiaA9[3 * r], invInertiaA9[3 * r + 1], invInertiaA9[3 * r + 2]);
        IB.r[r] = V(invInertiaB9[3 * r], invInertiaB9[3 * r + 1], invInertiaB9[3 * r + 2]);
    }
    const gs::C4 d = gs::set_constraint(c, V(posA3[0], posA3[1], posA3[2]), V(), V(), invMassA, IA,
                                        V(posB3[0], posB3[1], posB3[2]), V(), V(), invMassB, IB, dt);
    for (int i = 0; i < 4; ++i) {
        out13[i] = rval(d.jacCoeffInv[i]);
        out13[4 + i] = rval(d.b[i]);
    }
    out13[8] = rval(d.center.x);
    out13[9] = rval(d.center.y);
    out13[10] = rval(d.center.z);
    out13[11] = rval(d.fJacCoeffInv[0]);
    out13[12] = rval(d.fJacCoeffInv[1]);
}
// computePairsKernel restatement on caller-sorted records (8 floats each):
// writes up to max pairs, returns the full count
int or_sap_sorted_pairs(const float* sorted8, int n, int axis, int* pairs2, int max) {
    std::vector<float> s(sorted8, sorted8 + 8 * (size_t)n), none;
    std::vector<int> p;
    sap_pairs(s, n, axis, none, 0, p);
    const int np = (int)p.size() / 2;
    if (pairs2) memcpy(pairs2, p.data(), 8 * (size_t)std::min(np, max));
    return np;
}
void or_stage_broadphase(or_world* w) { stage_broadphase(w); }
void or_stage_narrowphase(or_world* w) { stage_narrowphase(w); }
void or_stage_solve(or_world* w) { stage_solve(w); }
void or_stage_integrate(or_world* w) { stage_integrate(w); }

void or_step(or_world* w, int steps) {
    for (int s = 0; s < steps; ++s) {
        stage_aabbs(w);
        stage_broadphase(w);
        stage_narrowphase(w);
        stage_solve(w);
        stage_integrate(w);
    }
}

int or_get_aabbs(or_world* w, float* out8) {
    memcpy(out8, w->aabb.data(), sizeof(float) * w->aabb.size());
    return (int)w->aabb.size() / 8;
}
int or_get_sorted(or_world* w, uint32_t* keys, uint32_t* vals, int max) {
    const int n = std::min((int)w->keys.size(), max);
    if (keys) memcpy(keys, w->keys.data(), 4 * (size_t)n);
    if (vals) memcpy(vals, w->vals.data(), 4 * (size_t)n);
    return (int)w->keys.size();
}
int or_get_pairs(or_world* w, int* pairs2, int max) {
    const int n = std::min((int)w->pairs.size() / 2, max);
    if (pairs2) memcpy(pairs2, w->pairs.data(), 8 * (size_t)n);
    return (int)w->pairs.size() / 2;
}
or_contact export_contact(const or_contact_r& c) {
    or_contact o;
    for (int j = 0; j < 4; ++j) {
        for (int k = 0; k < 4; ++k) o.pos[j][k] = rval(c.pos[j][k]);
        o.normal[j] = rval(c.normal[j]);
    }
    o.friction = rval(c.friction);
    o.pairIndex = c.pairIndex;
    o.bodyA = c.bodyA;
    o.bodyB = c.bodyB;
    o.pad = c.pad;
    return o;
}
int or_get_contacts(or_world* w, or_contact* out, int max) {
    const int n = std::min((int)w->contacts.size(), max);
    if (out)
        for (int i = 0; i < n; ++i) out[i] = export_contact(w->contacts[i]);
    return (int)w->contacts.size();
}
void or_get_overflow(or_world* w, long long* pairOverflow, long long* cellOverflow) {
    *pairOverflow = w->pairOverflow;
    *cellOverflow = w->cellOverflow;
}
// Inject contacts (e.g. from the device) before or_stage_solve.
void or_set_contacts(or_world* w, const or_contact* c, int n) {
    w->contacts.assign((size_t)n, or_contact_r());
    for (int i = 0; i < n; ++i) {
        or_contact_r& r = w->contacts[i];
        for (int j = 0; j < 4; ++j) {
            for (int k = 0; k < 4; ++k) r.pos[j][k] = c[i].pos[j][k];
            r.normal[j] = c[i].normal[j];
        }
        r.friction = c[i].friction;
        r.pairIndex = c[i].pairIndex;
        r.bodyA = c[i].bodyA;
        r.bodyB = c[i].bodyB;
        r.pad = c[i].pad;
    }
}
// Inject pairs before or_stage_narrowphase.
void or_set_pairs(or_world* w, const int* pairs2, int n) { w->pairs.assign(pairs2, pairs2 + 2 * (size_t)n); }

// Single-pair narrowphase for known-answer tests: returns nPoints (0 = none).
int or_pair_contact(or_world* w, int A, int B, or_contact* out) {
    or_contact_r c;
    if (!contact_for_pair(w, 0, A, B, c)) return 0;
    *out = export_contact(c);
    return (int)rval(c.normal[3]);
}

// Clipping + reduction entry for the pin against the reference host port:
// clip the given incident polygon against reference face fa of polyA posed
// at (posA, qA); returns kept points (x, y, z, depth) and reduced indices.
int or_clip_reduce(or_world* w, int polyA, int faceA, const double* posA, const double* qA,
                   const double* polyIn4, int nIn, double maxDist, const double* nearNormal, double* out4,
                   int* idx4) {
    const or_poly& hA = w->polys[polyA];
    Body A;
    A.pos = V(posA[0], posA[1], posA[2]);
    A.q = Q{qA[0], qA[1], qA[2], qA[3]};
    const or_face& fa = w->faces[hA.faceOffset + faceA];
    std::vector<P4> in, tmp;
    for (int i = 0; i < nIn; ++i) in.push_back({polyIn4[4 * i], polyIn4[4 * i + 1], polyIn4[4 * i + 2], 0});
    const int nvA = fa.numIndices;
    const V nAw = qrot(A.q, V(fa.plane[0], fa.plane[1], fa.plane[2]));
    for (int e0 = 0; e0 < nvA; ++e0) {
        const V a = vtx(w, hA.vertexOffset + w->indices[fa.indexOffset + e0]);
        const V b = vtx(w, hA.vertexOffset + w->indices[fa.indexOffset + (e0 + 1) % nvA]);
        const V pn = -cross(qrot(A.q, a - b), nAw);
        const Real eq = -dot(qrot(A.q, a) + A.pos, pn);
        clip_face(in, pn, eq, tmp);
        in.swap(tmp);
    }
    const Real eqA = (Real)fa.plane[3] - dot(nAw, A.pos);
    std::vector<P4> pts;
    for (const P4& p : in) {
        Real depth = nAw.x * p.x + nAw.y * p.y + nAw.z * p.z + eqA;
        if (depth <= -1e30) depth = -1e30;
        if (depth <= maxDist) pts.push_back({p.x, p.y, p.z, depth});
    }
    for (size_t i = 0; i < pts.size(); ++i) {
        out4[4 * i] = rval(pts[i].x); out4[4 * i + 1] = rval(pts[i].y);
        out4[4 * i + 2] = rval(pts[i].z); out4[4 * i + 3] = rval(pts[i].w);
    }
    reduce_manifold(pts, V(nearNormal[0], nearNormal[1], nearNormal[2]), idx4);
    return (int)pts.size();
}

// clipFacesAndContactReductionKernel (satClipHullContacts.cl:1845-1952) for
// one pair given in world space, as the reference's own test data records
// it: the reference face's vertices vertsA4[0..nA) and normal normalA, the
// incident polygon polyB4[0..nB); side planes -cross(a - b, n) through a,
// Sutherland-Hodgman clip, then depth = n . p - n . a0, clamped at minDist
// and kept when <= maxDist. Writes (x, y, z, depth) and returns the count.
int or_clip_face_world(const double* vertsA4, int nA, const double* normalA, const double* polyB4, int nB,
                       double minDist, double maxDist, double* out4) {
    std::vector<P4> in, tmp;
    for (int i = 0; i < nB; ++i) in.push_back({polyB4[4 * i], polyB4[4 * i + 1], polyB4[4 * i + 2], 0});
    const V n(normalA[0], normalA[1], normalA[2]);
    for (int e0 = 0; e0 < nA; ++e0) {
        const V a(vertsA4[4 * e0], vertsA4[4 * e0 + 1], vertsA4[4 * e0 + 2]);
        const int e1 = (e0 + 1) % nA;
        const V b(vertsA4[4 * e1], vertsA4[4 * e1 + 1], vertsA4[4 * e1 + 2]);
        const V pn = -cross(a - b, n);
        const Real eq = -dot(a, pn);
        clip_face(in, pn, eq, tmp);
        in.swap(tmp);
    }
    const V a0(vertsA4[0], vertsA4[1], vertsA4[2]);
    const Real eqA = -dot(n, a0);
    int k = 0;
    for (const P4& p : in) {
        Real depth = n.x * p.x + n.y * p.y + n.z * p.z + eqA;
        if (depth <= minDist) depth = minDist;
        if (depth <= maxDist) {
            out4[4 * k] = rval(p.x); out4[4 * k + 1] = rval(p.y); out4[4 * k + 2] = rval(p.z);
            out4[4 * k + 3] = rval(depth);
            ++k;
        }
    }
    return k;
}

// Solver-only entry for the pin against the reference's btPgsJacobiSolver:
// solve the given manifolds with the given velocities and return the
// post-solve velocities (bodies' linVel/angVel after the finish step).
void or_solve_velocities(or_world* w, double* lin4, double* ang4) {
    stage_solve(w);
    for (int i = 0; i < w->n; ++i) {
        if (w->invMass[i] == 0.f || w->count[i] == 0) continue;
        for (int c = 0; c < w->count[i]; ++c)
            for (int k = 0; k < 3; ++k) {
                w->lin[4 * i + k] += w->avgLin[3 * i + k];
                w->ang[4 * i + k] += w->avgAng[3 * i + k];
            }
    }
    for (size_t i = 0; i < 4 * (size_t)w->n; ++i) {
        lin4[i] = rval(w->lin[i]);
        ang4[i] = rval(w->ang[i]);
    }
}

}  // extern "C"
