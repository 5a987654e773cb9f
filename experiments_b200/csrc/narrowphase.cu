// Convex-hull SAT narrowphase with face clipping and contact reduction,
// one warp per broadphase pair, for sm_100a.
//
// Semantics follow the reference GPU path
// (GpuSatCollision::computeConvexConvexContactsGPUSAT, P2/ConvexHullContact.cpp:1793):
//   findSeparatingAxisKernel  P2/sat.cl:928-1262
//     - static-static pairs are skipped (sat.cl:944-948)
//     - face normals of A, then of B, oriented along DeltaC2 = cA - cB;
//       any separating face axis rejects the pair (findSeparatingAxis :497-551)
//     - edge x edge axes (skip |cross| components <= 1e-6), never reject
//       (findSeparatingAxisEdgeEdge :556-635, result forced true :600-616)
//     - minimum depth over the axes in that order, first minimum wins
//   clipHullAgainstHull  P2/satClipHullContacts.cl:556-611
//     - incident face of B = max dot(nB, sep); reference face of A =
//       min dot(nA, sep); Sutherland-Hodgman against A's side planes
//       (clipFace :303-351); keep depth <= maxDist (0.02), clamp at minDist
//   contact reduction = extractManifoldSequentialGlobal
//     (P2/satClipHullContacts.cl:678-770): <= 4 points kept as is, else the
//     extreme points along +-u, +-v (arg-min with FLT_MIN start) and the
//     deepest point substituted into slot 0 if absent
//   Contact4 emission (newContactReductionKernel :1958-2039): normal = -sep,
//     static bodies carry a negative id.
//
// B200 mapping: the 32 lanes of a warp split the candidate axes (face
// normals and edge pairs), each projecting both hulls from L1-resident
// hull tables; a (depth, axis index) arg-min across lanes reproduces the
// sequential first-minimum choice. Clipping runs one polygon vertex per
// lane with a ballot prefix for the output slots, so the whole
// find-axis / clip / reduce chain is one kernel with no per-pair global
// scratch (the reference writes 3 x 64 x 16 B per pair between its kernels).
// Contacts go to the pair's own slot, so the manifold order is the pair
// order and every run is deterministic.
#include "b3_math.cuh"
#include "b3_world.h"
#include "b3_ff.cuh"

#include <algorithm>
#include <cfloat>

using namespace b3m;

namespace {

using namespace b3ff;

constexpr int kMaxPoly = 64;  // capacityWorldVerts (satClipHullContacts.cl:1027)
constexpr int kKeep = 4;      // near-minimum axis candidates kept per lane
constexpr int kMaxCand = 32;  // candidates refined in float-float per pair
constexpr int kPreChunk = 4;  // pairs per work grab of the sweep and the clip, prefetched by lanes
// shared memory of one sweep warp: the prefetched chunk and the candidates
constexpr int kSweepWarpSmem = 128 * kPreChunk + 4 * kMaxCand;
constexpr int kNone = 0x7fffffff;
// clip faces whose products with the axis differ by no more than this are
// tied (the lowest index wins), in the device's float-float ranking and in
// the oracle's FP64 one alike
constexpr float kFaceTieTol = 1e-10f;
// separating axes whose depths differ by no more than this (metres) are
// tied and the lowest axis index wins, in the float-float ranking and in the
// oracle's FP64 one alike
constexpr float kAxisTieTol = 1e-10f;
// pairSep[p].w: how the pair reached the exact stage
// pairSep[p].w: how the pair reached the exact stage
constexpr int kSepRefine = 0;      // near-minimum axes: float-float re-ranking
constexpr int kSepDecided = 1;     // FP32 axis (FP32 clip stage)
constexpr int kSepClipDoubt = 2;   // FP32 axis, clip or reduction in doubt: float-float clip
constexpr int kSepFaceTie = 3;     // FP32 axis, clip faces near-tied: float-float axis, then clip

struct NpParams {
    float minDist;
    float maxDist;
    // depth above which the solver skips a point (contactProcessing -
    // slopOffset, btPgsJacobiSolver.cpp:961): a depth this close to it in
    // FP32 is a decision in doubt as well
    float skipDist;
    int frictionCombine;
    int maxPairs;
};

// Per-pair context. The clip and float-float stages keep it in the warp's
// shared scratch (one copy per warp, written by lane 0): the functions that
// take it by reference are not inlined, and a per-thread copy would live in
// local memory, which at full occupancy does not fit L1.
struct PairCtx {
    int A, B;
    float invMassA, invMassB;
    const b3ConvexPolyhedron* pa;
    const b3ConvexPolyhedron* pb;
    float4 qA, qB;
    Mat3 RA, RB;
    ffmat FA, FB;  // float-float rotation matrices
    bool haveFF;   // FA/FB valid
    float3 posA, posB;
};

// Geometry of one FP32 clip (reference face side planes, incident face).
struct ClipGeom {
    const float4* sideN;   // per side plane k: normal (not unit)
    const float4* sideP;   // per side plane k: a point on it
    const float4* incV;    // incident face vertices, A frame
    b3Face fA, fB;
    Mat3 RA, RB;
    float3 rel;      // posB - posA
    float3 nAw;      // reference face normal (world)
    float3 nIn;      // incident face normal (world)
    float hIn;       // incident plane: nIn . x = hIn (A frame)
    float eIn;       // error bound of hIn
};

// Per-warp shared scratch: two float-float polygons (x, y, z, depth).
struct __align__(16) FfVert {
    float xh, xl, yh, yl, zh, zl, wh, wl;
};
struct __align__(16) WarpScratch {
    FfVert poly[2][kMaxPoly];
    FfVert planes[kMaxPoly];  // float-float clip planes (normal, constant)
    float4 sideN[kMaxPoly];   // FP32 clip: side plane normals of the reference face
    float4 sideP[kMaxPoly];   // FP32 clip: a point on each side plane
    float4 incV[kMaxPoly];    // FP32 clip: incident face vertices (A frame)
    PairCtx ctx;
    ClipGeom geom;
    int cand[kMaxCand];
    int refinedAxes, refinedClips;  // float-float fallbacks taken by this warp
};

__device__ __forceinline__ ff3 vget(const FfVert& v) { return {{v.xh, v.xl}, {v.yh, v.yl}, {v.zh, v.zl}}; }
__device__ __forceinline__ ff wget(const FfVert& v) { return {v.wh, v.wl}; }
__device__ __forceinline__ FfVert vput(ff3 p, ff w) {
    return {p.x.hi, p.x.lo, p.y.hi, p.y.lo, p.z.hi, p.z.lo, w.hi, w.lo};
}

__device__ __forceinline__ float combine_friction(float a, float b, int mode) {
    return mode == B3_FRICTION_PRODUCT ? a * b : sqrtf(a * b);
}

// |a| for error bounds and thresholds, rounded up: the approximate
// reciprocal square root is within a few ulps, which the factor covers
__device__ __forceinline__ float len_ub(float3 a) {
    const float d = dot(a, a);
    return d * rsqrtf(fmaxf(d, FLT_MIN)) * 1.000002f;
}

// Integer key whose signed order is the float order: -0 and +0 share a key
// (the sum with +0 turns -0 into +0) and a NaN never wins a minimum (or a
// maximum, with kNanMax).
constexpr int kNanMin = 0x7fffffff, kNanMax = (int)0x80000000;
__device__ __forceinline__ int fkey(float v, int nanKey) {
    const int k = __float_as_int(v + 0.f);
    return v != v ? nanKey : k ^ ((k >> 31) & 0x7fffffff);
}
__device__ __forceinline__ float fkey_inv(int k) { return __int_as_float(k ^ ((k >> 31) & 0x7fffffff)); }
__device__ __forceinline__ float warp_min(float v) {
    return fkey_inv(__reduce_min_sync(0xffffffffu, fkey(v, kNanMin)));
}
__device__ __forceinline__ float warp_max(float v) {
    return fkey_inv(__reduce_max_sync(0xffffffffu, fkey(v, kNanMax)));
}

// lexicographic (value, index) minimum across the warp: the minimum value,
// then the smallest index (as unsigned) among the lanes holding it
__device__ __forceinline__ void warp_argmin(float& v, int& idx) {
    const int k = fkey(v, kNanMin);
    const int km = __reduce_min_sync(0xffffffffu, k);
    idx = (int)__reduce_min_sync(0xffffffffu, k == km ? (unsigned)idx : 0xffffffffu);
    v = fkey_inv(km);
}
// the same for float-float values, ordered by (hi, lo)
__device__ __forceinline__ void warp_argmin_ff(ff& v, int& idx) {
    const int kh = fkey(v.hi, kNanMin);
    const int mh = __reduce_min_sync(0xffffffffu, kh);
    const int kl = kh == mh ? fkey(v.lo, kNanMin) : kNanMin;
    const int ml = __reduce_min_sync(0xffffffffu, kl);
    idx = (int)__reduce_min_sync(0xffffffffu, kh == mh && kl == ml ? (unsigned)idx : 0xffffffffu);
    v.hi = fkey_inv(mh);
    v.lo = fkey_inv(ml);
}

// Axis index space (sequential order of the reference): faces of A
// [0, FA), faces of B [FA, FA+FB), edge pairs e0*EB+e1 after that.
//
// Oriented world direction of axis idx and its FP32 depth error bound;
// false for a degenerate edge pair (|e0 x e1| components all <= 1e-6).
// lb: a lower bound of the axis' depth that the sweep compares against its
// depth windows. With D = cA - cB (the local centres in world space) and
// rin the hull's inradius about its local centre (ShapesDev.inradius),
// every axis n has
//   depth = min(maxA - minB, maxB - minA) >= rinA + rinB - |n . D|,
// since each hull's support about its centre is at least rin in every
// direction. rinSum carries a margin for the radii; the FP32 error of n . D
// and twice the axis' own depth error are subtracted too, so an axis whose
// bound exceeds the window can neither be the first minimum nor enter the
// near-minimum candidates (depth - err <= the minimum's depth + err).
__device__ __forceinline__ bool axis_dir(const PairCtx& c, const b3::ShapesDev& S, int idx, float3 D, float delta,
                                         float rinSum, float3& n, float& err, float& lb, bool& isFace,
                                         bool wantLb = true) {
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    const int FA = pa.numFaces, FB = pb.numFaces;
    const float lD = wantLb ? len_ub(D) : 0.f;
    if (idx < FA + FB) {
        isFace = true;
        const bool onA = idx < FA;
        const float4 pl = __ldg((const float4*)&S.faces[onA ? pa.faceOffset + idx : pb.faceOffset + idx - FA].plane[0]);
        n = mul(onA ? c.RA : c.RB, make_float3(pl.x, pl.y, pl.z));
        err = delta;
        lb = wantLb ? rinSum - fabsf(dot(D, n)) - 1e-5f * (1.f + lD) - 2.f * err : -FLT_MAX;
    } else {
        isFace = false;
        const int e = idx - FA - FB;
        const int EB = pb.numUniqueEdges;
        const int e0 = e / EB, e1 = e - e0 * EB;
        const float4 ea = __ldg(&S.edges[pa.uniqueEdgesOffset + e0]);
        const float4 eb = __ldg(&S.edges[pb.uniqueEdgesOffset + e1]);
        const float3 wa = mul(c.RA, f3(ea));
        const float3 wb = mul(c.RB, f3(eb));
        float3 cr = cross(wa, wb);
        if (!(fabsf(cr.x) > 1e-6f || fabsf(cr.y) > 1e-6f || fabsf(cr.z) > 1e-6f)) return false;
        const float cl = length(cr);
        n = cr * (1.f / cl);
        // direction error of the normalised FP32 cross product is ~ulp/sin,
        // sin = cl over the edges' lengths (w: 1 for a hull's unit edges, the
        // length of a mesh triangle's edge); its depth error scales with the
        // projected extents (delta / 1e-6)
        const float isin = ea.w * eb.w / cl;
        err = delta + 0.3f * delta * isin;
        lb = wantLb ? rinSum - fabsf(dot(D, n)) - 1e-5f * (1.f + lD) - 1e-6f * lD * isin - 2.f * err : -FLT_MAX;
    }
    if (dot(D, n) < 0.f) n = -n;
    return true;
}

// Two FP32 lanes in one 64-bit register, and the packed FP32x2 multiply
// and fused multiply-add (each half rounds as its scalar instruction would).
__device__ __forceinline__ unsigned long long pack2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// FP32 projection of polyhedron h (index pi) onto world axis dir relative to
// its own position, two vertices per packed FP32x2 instruction: x * d.x,
// then + y * d.y, then + z * d.z, each rounded once.
__device__ __forceinline__ void project_packed(const b3::ShapesDev& S, const b3ConvexPolyhedron& h, int pi,
                                               const Mat3& R, float3 dir, float& mn, float& mx) {
    const float3 ld = mul_t(R, dir);
    const unsigned long long lx = pack2(ld.x, ld.x), ly = pack2(ld.y, ld.y), lz = pack2(ld.z, ld.z);
    const int off = __ldg(&S.polyPack[pi]), np = (h.numVertices + 1) >> 1;
    float lo = FLT_MAX, hi = -FLT_MAX;
#pragma unroll 4
    for (int j = 0; j < np; ++j) {
        const float4 xy = __ldg(&S.vpXY[off + j]);
        const float2 z = __ldg(&S.vpZ[off + j]);
        unsigned long long d = mul2(pack2(xy.x, xy.y), lx);
        d = fma2(pack2(xy.z, xy.w), ly, d);
        d = fma2(pack2(z.x, z.y), lz, d);
        float d0, d1;
        unpack2(d, d0, d1);
        lo = fminf(lo, fminf(d0, d1));
        hi = fmaxf(hi, fmaxf(d0, d1));
    }
    mn = lo;
    mx = hi;
}

// FP32 depth along the oriented axis n (P2/sat.cl:227-252, relative to
// body A's position).
__device__ __forceinline__ float axis_depth(const PairCtx& c, const b3::ShapesDev& S, float3 rel, float3 n) {
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    float mn0, mx0, mn1, mx1;
    project_packed(S, pa, (int)(c.pa - S.polys), c.RA, n, mn0, mx0);
    project_packed(S, pb, (int)(c.pb - S.polys), c.RB, n, mn1, mx1);
    const float off = dot(rel, n);  // posB - posA along n
    mn1 += off;
    mx1 += off;
    return fminf(mx0 - mn1, mx1 - mn0);
}

// Direction and depth of axis idx; false for a degenerate edge pair.
__device__ __forceinline__ bool axis_f32(const PairCtx& c, const b3::ShapesDev& S, int idx, float3 D,
                                         float3 rel, float delta, float3& n, float& d, float& err, bool& isFace) {
    float lb;
    if (!axis_dir(c, S, idx, D, delta, 0.f, n, err, lb, isFace, false)) return false;
    d = axis_depth(c, S, rel, n);
    return true;
}

// float-float evaluation of one axis: oriented axis and depth; false if
// the edge pair is degenerate. vA / vB: the hulls' vertices (staged in
// shared memory by the caller, or the global tables).
__device__ __noinline__ bool axis_ff(const PairCtx& c, const b3::ShapesDev& S, const float4* vA, const float4* vB,
                                     int idx, ff3 Dff, ff3& n, ff& d, bool& isFace) {
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    const int FA = pa.numFaces, FB = pb.numFaces;
    if (idx < FA + FB) {
        isFace = true;
        const bool onA = idx < FA;
        const float4 pl = __ldg((const float4*)&S.faces[onA ? pa.faceOffset + idx : pb.faceOffset + idx - FA].plane[0]);
        n = mrot(onA ? c.FA : c.FB, make_float3(pl.x, pl.y, pl.z));
    } else {
        isFace = false;
        const int e = idx - FA - FB;
        const int EB = pb.numUniqueEdges;
        const int e0 = e / EB, e1 = e - e0 * EB;
        const float4 ea = __ldg(&S.edges[pa.uniqueEdgesOffset + e0]);
        const float4 eb = __ldg(&S.edges[pb.uniqueEdgesOffset + e1]);
        const ff3 wa = mrot(c.FA, make_float3(ea.x, ea.y, ea.z));
        const ff3 wb = mrot(c.FB, make_float3(eb.x, eb.y, eb.z));
        const ff3 cr = cross3(wa, wb);
        if (dot3(cr, cr).hi <= 0.f) return false;
        n = normalize3(cr);
    }
    if (dot3(Dff, n).hi < 0.f) n = neg3(n);
    // projections (P2/sat.cl:227-252) in float-float
    ff lo[2], hi[2];
    for (int h = 0; h < 2; ++h) {
        const b3ConvexPolyhedron& p = h == 0 ? pa : pb;
        const float4* verts = h == 0 ? vA : vB;
        const float3 pos = h == 0 ? c.posA : c.posB;
        const ff3 ld = mrot_t(h == 0 ? c.FA : c.FB, n);
        ff mn = mk(FLT_MAX), mx = mk(-FLT_MAX);
#pragma unroll 2
        for (int i = 0; i < p.numVertices; ++i) {
            const float4 v = verts[i];
            const ff dp = add(add(mulf(ld.x, v.x), mulf(ld.y, v.y)), mulf(ld.z, v.z));
            if (lt(dp, mn)) mn = dp;
            if (lt(mx, dp)) mx = dp;
        }
        const ff offs = add(add(mulf(n.x, pos.x), mulf(n.y, pos.y)), mulf(n.z, pos.z));
        lo[h] = add(mn, offs);
        hi[h] = add(mx, offs);
    }
    const ff d0 = sub(hi[0], lo[1]), d1 = sub(hi[1], lo[0]);
    d = lt(d0, d1) ? d0 : d1;
    return true;
}

// Separating-axis search (findSeparatingAxisKernel, P2/sat.cl:928-1262):
// FP32 sweep over all axes by the warp, then float-float refinement of every
// axis whose FP32 depth is within delta of the minimum. Returns false if a
// face axis separates or no axis exists.
// FP32 part: 0 = separated (or no axis), 1 = decided in FP32 (sepf),
// 2 = near-minimum candidates left in W.cand[0..count) for float-float.
template <bool kEarlyFaces>
__device__ __forceinline__ int sweep_axes(PairCtx& c, const b3::ShapesDev& S, int* cand, float3& sepf,
                                          int& count, int* ovfCounter) {
    const int lane = threadIdx.x & 31;
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    const float3 lcA = make_float3(pa.localCenter[0], pa.localCenter[1], pa.localCenter[2]);
    const float3 lcB = make_float3(pb.localCenter[0], pb.localCenter[1], pb.localCenter[2]);
    const float3 rel = c.posB - c.posA;
    const float3 D = mul(c.RA, lcA) - (mul(c.RB, lcB) + rel);
    const int nFace = pa.numFaces + pb.numFaces;
    const int nAxes = nFace + pa.numUniqueEdges * pb.numUniqueEdges;
    const float scale = 1.f + sqrtf(pa.mE[0] * pa.mE[0] + pa.mE[1] * pa.mE[1] + pa.mE[2] * pa.mE[2]) +
                        sqrtf(pb.mE[0] * pb.mE[0] + pb.mE[1] * pb.mE[1] + pb.mE[2] * pb.mE[2]) + len_ub(rel);
    // FP32 depth error bound for well-conditioned axes (a few ulps of the
    // largest projected coordinate); edge axes add a term inversely
    // proportional to |e0 x e1| (their normalisation amplifies rounding)
    const float delta = 1e-6f * scale;
    // kEarlyFaces, pairs with more than one lane-round of faces: first
    // test the face of A and the face of B best aligned with D (the
    // likeliest separating axes), with the warp splitting the vertices. A
    // separating face axis rejects the pair whichever face it is, and each
    // test computes the same FP32 depth as the full pass below, so an early
    // rejection here is the full pass' own verdict. (A template switch: the
    // launch picks it only for shape sets with such hulls, as its code
    // costs the cube-only sweeps a few per cent.)
    if (kEarlyFaces && nFace > 32) {
        const int FA = pa.numFaces;
        float bA = -1.f, bB = -1.f;
        int iA = kNone, iB = kNone;
        for (int f = lane; f < nFace; f += 32) {
            const bool onA = f < FA;
            const float4 pl = __ldg((const float4*)&S.faces[onA ? pa.faceOffset + f : pb.faceOffset + f - FA].plane[0]);
            const float a = fabsf(dot(D, mul(onA ? c.RA : c.RB, make_float3(pl.x, pl.y, pl.z))));
            if (onA) {
                if (a > bA) { bA = a; iA = f; }
            } else if (a > bB) {
                bB = a;
                iB = f;
            }
        }
        bA = -bA;
        bB = -bB;
        warp_argmin(bA, iA);
        warp_argmin(bB, iB);
        for (int t = 0; t < 2; ++t) {
            const int f = t == 0 ? iA : iB;
            if (f == kNone) continue;
            const bool onA = f < FA;
            const float4 pl = __ldg((const float4*)&S.faces[onA ? pa.faceOffset + f : pb.faceOffset + f - FA].plane[0]);
            float3 n = mul(onA ? c.RA : c.RB, make_float3(pl.x, pl.y, pl.z));
            if (dot(D, n) < 0.f) n = -n;
            float mn[2], mx[2];
            for (int h = 0; h < 2; ++h) {
                const b3ConvexPolyhedron& p = h == 0 ? pa : pb;
                const float3 ld = mul_t(h == 0 ? c.RA : c.RB, n);
                float lo = FLT_MAX, hi = -FLT_MAX;
                for (int i = lane; i < p.numVertices; i += 32) {
                    const float4 v = __ldg(&S.verts[p.vertexOffset + i]);
                    const float dp = v.x * ld.x + v.y * ld.y + v.z * ld.z;
                    lo = fminf(lo, dp);
                    hi = fmaxf(hi, dp);
                }
                mn[h] = warp_min(lo);
                mx[h] = warp_max(hi);
            }
            const float off = dot(rel, n);
            const float d = fminf(mx[0] - (mn[1] + off), (mx[1] + off) - mn[0]);
            if (d < -delta) return 0;
        }
    }
    float kd[kKeep];
    int ki[kKeep];
#pragma unroll
    for (int k = 0; k < kKeep; ++k) {
        kd[k] = FLT_MAX;
        ki[k] = kNone;
    }
    // face axes whose separation test is ambiguous in FP32 (|d| <= delta)
    int amb[2] = {kNone, kNone};
    bool ambOverflow = false;
    float sepMin = FLT_MAX;
    float upper = FLT_MAX;  // min over axes of (d + err): bounds the true minimum depth
    // Edge pairs are projected only when a lower bound of their depth
    // (axis_dir) reaches the best face axis (d + err): the others can
    // neither be the minimum nor a near-minimum candidate. The radii lose
    // 1e-4 m for their own rounding.
    float lbHi = FLT_MAX;
    const float rinSum = fmaxf(0.f, S.inradius[c.pa - S.polys] + S.inradius[c.pb - S.polys] - 1e-4f);
    // faces of A and B first; a separating face axis ends the search before
    // the edge pairs, as the reference returns early (P2/sat.cl:527-530)
    for (int pass = 0; pass < 2; ++pass) {
        const int i0 = pass == 0 ? 0 : nFace;
        const int i1 = pass == 0 ? nFace : nAxes;
        for (int idx = i0 + lane; idx < i1; idx += 32) {
            float3 n;
            float err, lb;
            bool isFace;
            if (!axis_dir(c, S, idx, D, delta, rinSum, n, err, lb, isFace, pass == 1) || lb > lbHi) continue;
            const float d = axis_depth(c, S, rel, n);
            if (isFace) {
                sepMin = fminf(sepMin, d);
                if (fabsf(d) <= delta) {
                    if (amb[0] == kNone) amb[0] = idx;
                    else if (amb[1] == kNone) amb[1] = idx;
                    else ambOverflow = true;
                }
            }
            upper = fminf(upper, d + err);
            const float lo = d - err;  // lower bound of this axis' depth
            if (!(lo < kd[kKeep - 1])) continue;  // also drops NaN
            // insertion into the lane's sorted keep list (indices increase)
            float cd = lo;
            int ci = idx;
#pragma unroll
            for (int k = 0; k < kKeep; ++k) {
                if (cd < kd[k]) {
                    const float td = kd[k];
                    const int ti = ki[k];
                    kd[k] = cd;
                    ki[k] = ci;
                    cd = td;
                    ci = ti;
                }
            }
        }
        if (pass == 0) {
            float sm0 = sepMin;
            int dz = 0;
            warp_argmin(sm0, dz);
            if (sm0 < -delta) return 0;
            lbHi = warp_min(upper);
        }
    }
    // clearly separated by a face axis
    float sm = sepMin;
    int dummy = 0;
    warp_argmin(sm, dummy);
    if (sm < -delta) return 0;
    float best = upper;
    int bi = 0;
    warp_argmin(best, bi);
    if (!(best < FLT_MAX)) return 0;
    const float lim = best;
    // collect candidates
    count = 0;
    bool overflow = kd[kKeep - 1] <= lim || ambOverflow;
    for (int k = 0; k < kKeep + 2; ++k) {
        const int id = k < kKeep ? ki[k] : amb[k - kKeep];
        const bool take = id != kNone && (k >= kKeep || kd[k] <= lim);
        const unsigned m = __ballot_sync(0xffffffffu, take);
        const int pos = count + __popc(m & b3dev::lanemask_lt());
        if (take && pos < kMaxCand) cand[pos] = id;
        count += __popc(m);
    }
    if (__any_sync(0xffffffffu, overflow) || count > kMaxCand) {
        // more near-minimum axes than the keep lists hold: rescan
        count = 0;
        for (int base = 0; base < nAxes; base += 32) {
            const int idx = base + lane;
            float3 n;
            float d = FLT_MAX, err = 0.f;
            bool isFace;
            bool take = false;
            if (idx < nAxes && axis_f32(c, S, idx, D, rel, delta, n, d, err, isFace))
                take = d - err <= lim || (isFace && fabsf(d) <= delta);
            const unsigned m = __ballot_sync(0xffffffffu, take);
            const int pos = count + __popc(m & b3dev::lanemask_lt());
            if (take && pos < kMaxCand) cand[pos] = idx;
            count += __popc(m);
        }
        if (count > kMaxCand) {
            if (lane == 0) atomicAdd(ovfCounter, 1);
            count = kMaxCand;
        }
    }
    __syncwarp();
    // A single well-conditioned winner needs no refinement: a face axis, or
    // an edge axis with |e0 x e1| >= 0.01 (FP32 normal error < 1e-5), whose
    // orientation test is not near zero.
    if (count == 1) {
        const int idx = cand[0];
        float3 n;
        float d, err;
        bool isFace;
        if (axis_f32(c, S, idx, D, rel, delta, n, d, err, isFace) && err <= 31.f * delta &&
            fabsf(dot(D, n)) > 1e-5f * (len_ub(D) + 1e-3f)) {
            if (dot(-D, n) > 0.f) n = -n;
            sepf = n;
            return 1;
        }
    }
    // Several candidates that are the same direction within 1e-5 (parallel
    // faces, or edge pairs spanning a face's normal): whichever the exact
    // arithmetic picks, the normal agrees within tolerance and the clip
    // faces follow from it, so the FP32 first minimum is kept. Candidates
    // that decide separation (|depth| near zero) still go to float-float.
    if (count <= 32) {
        float3 n = make_float3(0.f, 0.f, 0.f);
        float d = FLT_MAX, err = 0.f;
        bool isFace = false, ok = true;
        int myIdx = kNone;
        if (lane < count) {
            myIdx = cand[lane];
            ok = axis_f32(c, S, myIdx, D, rel, delta, n, d, err, isFace) && err <= 31.f * delta &&
                 !(isFace && fabsf(d) <= delta) && fabsf(dot(D, n)) > 1e-5f * (len_ub(D) + 1e-3f);
            if (!ok) myIdx = kNone;
        }
        const float3 n0 = make_float3(__shfl_sync(0xffffffffu, n.x, 0), __shfl_sync(0xffffffffu, n.y, 0),
                                      __shfl_sync(0xffffffffu, n.z, 0));
        if (lane < count && ok) {
            const float3 dd = n - n0;
            if (fmaxf(fabsf(dd.x), fmaxf(fabsf(dd.y), fabsf(dd.z))) > 1e-5f) ok = false;
        }
        if (__all_sync(0xffffffffu, ok)) {
            float bd = (lane < count) ? d : FLT_MAX;
            int bidx = (lane < count) ? myIdx : kNone;
            warp_argmin(bd, bidx);
            const unsigned who = __ballot_sync(0xffffffffu, lane < count && myIdx == bidx);
            const int src = __ffs(who) - 1;
            float3 w = make_float3(__shfl_sync(0xffffffffu, n.x, src), __shfl_sync(0xffffffffu, n.y, src),
                                   __shfl_sync(0xffffffffu, n.z, src));
            if (dot(-D, w) > 0.f) w = -w;
            sepf = w;
            return 1;
        }
    }
    return 2;
}

// Float-float rotation matrices of the pair, computed once per pair (the
// context is warp-shared: lane 0 stores, the warp synchronises).
__device__ __forceinline__ void ensure_ff(PairCtx& c) {
    const bool have = c.haveFF;
    __syncwarp();
    if (!have) {
        const ffmat a = quat_mat(c.qA), b = quat_mat(c.qB);
        if ((threadIdx.x & 31) == 0) {
            c.FA = a;
            c.FB = b;
            c.haveFF = true;
        }
        __syncwarp();
    }
}

// float-float re-ranking of the sweep's candidates
__device__ __noinline__ bool refine_axes(PairCtx& c, const b3::ShapesDev& S, WarpScratch& W, int count, ff3& sep) {
    const int lane = threadIdx.x & 31;
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    const float3 lcA = make_float3(pa.localCenter[0], pa.localCenter[1], pa.localCenter[2]);
    const float3 lcB = make_float3(pb.localCenter[0], pb.localCenter[1], pb.localCenter[2]);
    // float-float refinement of the candidates (matrices built only for
    // pairs that got this far)
    ensure_ff(c);
    const ff3 lcAw = mrot(c.FA, make_float3(lcA.x, lcA.y, lcA.z));
    const ff3 lcBw = mrot(c.FB, make_float3(lcB.x, lcB.y, lcB.z));
    const ff3 Dff = sub3(add3(lcAw, mk3(c.posA.x, c.posA.y, c.posA.z)), add3(lcBw, mk3(c.posB.x, c.posB.y, c.posB.z)));
    // both hulls' vertices staged in shared memory (the polygon buffers are
    // free until the clip): every candidate lane loops over them, and
    // dependent L2 loads would dominate the float-float projections
    const float4* vA = S.verts + pa.vertexOffset;
    const float4* vB = S.verts + pb.vertexOffset;
    constexpr int kStage = (int)(sizeof(W.poly) / sizeof(float4));
    if (pa.numVertices + pb.numVertices <= kStage) {
        float4* st = reinterpret_cast<float4*>(&W.poly[0][0]);
        for (int k = lane; k < pa.numVertices; k += 32) st[k] = __ldg(&vA[k]);
        for (int k = lane; k < pb.numVertices; k += 32) st[pa.numVertices + k] = __ldg(&vB[k]);
        __syncwarp();
        vA = st;
        vB = st + pa.numVertices;
    }
    ff bd = mk(FLT_MAX);
    int bidx = kNone;
    ff3 bn = mk3(0.f, 0.f, 0.f);
    bool fsep = false;
    if (lane < count) {
        const int idx = W.cand[lane];
        ff3 n;
        ff d;
        bool isFace;
        if (axis_ff(c, S, vA, vB, idx, Dff, n, d, isFace)) {
            if (isFace && d.hi < 0.f) fsep = true;
            bd = d;
            bidx = idx;
            bn = n;
        }
    }
    if (__any_sync(0xffffffffu, fsep)) return false;
    ff wd = bd;
    int widx = bidx;
    warp_argmin_ff(wd, widx);
    if (widx == kNone) return false;
    // depths within kAxisTieTol of the minimum are tied and the lowest axis
    // index wins: the reference's first minimum for axes tied in exact
    // arithmetic, whose FP64 depths differ only by rounding
    widx = (int)__reduce_min_sync(0xffffffffu, bidx != kNone && sub(bd, wd).hi <= kAxisTieTol ? (unsigned)bidx
                                                                                               : 0xffffffffu);
    const unsigned who = __ballot_sync(0xffffffffu, bidx == widx);
    const int src = __ffs(who) - 1;
    sep.x.hi = __shfl_sync(0xffffffffu, bn.x.hi, src);
    sep.x.lo = __shfl_sync(0xffffffffu, bn.x.lo, src);
    sep.y.hi = __shfl_sync(0xffffffffu, bn.y.hi, src);
    sep.y.lo = __shfl_sync(0xffffffffu, bn.y.lo, src);
    sep.z.hi = __shfl_sync(0xffffffffu, bn.z.hi, src);
    sep.z.lo = __shfl_sync(0xffffffffu, bn.z.lo, src);
    if (dot3(neg3(Dff), sep).hi > 0.f) sep = neg3(sep);
    return true;
}

// Whether reference face ai of A can keep a clipped point. A face of two
// vertices (a mesh triangle's edge plane, P2/sat.cl:1083-1105) has two side
// planes that are one plane with opposite orientations, and clipFace keeps
// only points strictly inside (ds < 0), so in exact arithmetic the clip
// keeps nothing (the reference's FP32 outcome there is rounding noise).
__device__ __forceinline__ bool ref_face_clips(const b3::ShapesDev& S, const PairCtx& c, int ai) {
    return S.faces[c.pa->faceOffset + ai].numIndices >= 3;
}

// Separating-axis search: the FP32 sweep, then the float-float re-ranking
// when the sweep leaves near-minimum candidates. exact: the axis is needed
// to float-float accuracy (clip faces near-tied along it), so a winner the
// FP32 sweep decided is re-evaluated in float-float too.
__device__ __noinline__ bool find_axis(PairCtx& c, const b3::ShapesDev& S, WarpScratch& W, ff3& sep, int* ovfCounter,
                                       bool exact = false) {
    float3 sepf;
    int count = 0;
    const int r = sweep_axes<false>(c, S, W.cand, sepf, count, ovfCounter);
    if (r == 0) return false;
    if (r == 1 && !(exact && count >= 1)) {
        sep = mk3(sepf.x, sepf.y, sepf.z);
        return true;
    }
    if ((threadIdx.x & 31) == 0) ++W.refinedAxes;
    return refine_axes(c, S, W, count, sep);
}

// One Sutherland-Hodgman step in float-float (clipFace,
// satClipHullContacts.cl:303-351), one polygon vertex per lane; output
// order identical to the sequential loop. Each lane evaluates its own
// vertex's plane distance once; the edge start takes it from the previous
// lane.
__device__ __noinline__ int clip_poly_ff(const FfVert* in, int nin, const FfVert& plane, FfVert* out, int* ovf) {
    const int lane = threadIdx.x & 31;
    const ff3 pn = vget(plane);
    const ff eq = wget(plane);
    int total = 0;
    for (int base = 0; base < nin; base += 32) {
        const int ve = base + lane;
        const int sv = ve == 0 ? nin - 1 : ve - 1;
        ff3 e = mk3(0.f, 0.f, 0.f), s = e;
        ff de = mk(0.f);
        if (ve < nin) {
            e = vget(in[ve]);
            s = vget(in[sv]);
            de = add(dot3(pn, e), eq);
        }
        // distance of the edge start: previous lane's, or recomputed at the
        // chunk boundary and for the wrap-around edge of a long polygon
        ff ds;
        ds.hi = __shfl_up_sync(0xffffffffu, de.hi, 1);
        ds.lo = __shfl_up_sync(0xffffffffu, de.lo, 1);
        const bool own = lane == 0;
        if (ve < nin && own) ds = add(dot3(pn, s), eq);
        int cnt = 0;
        ff3 o0 = mk3(0.f, 0.f, 0.f), o1 = o0;
        if (ve < nin) {
            const bool sNeg = ds.hi < 0.f, eNeg = de.hi < 0.f;
            if (sNeg || eNeg) {
                if (sNeg && eNeg) {
                    o0 = e;
                    cnt = 1;
                } else {
                    const ff t = div(ds, sub(ds, de));
                    o0 = add3(s, scale3(sub3(e, s), t));
                    cnt = 1;
                    if (!sNeg) {
                        o1 = e;
                        cnt = 2;
                    }
                }
            }
        }
        const unsigned b1 = __ballot_sync(0xffffffffu, cnt >= 1), b2 = __ballot_sync(0xffffffffu, cnt == 2);
        const unsigned below = b3dev::lanemask_lt();
        const int pos = total + __popc(b1 & below) + __popc(b2 & below);
        if (cnt >= 1) {
            if (pos < kMaxPoly) out[pos] = vput(o0, mk(0.f)); else atomicAdd(ovf, 1);
        }
        if (cnt == 2) {
            if (pos + 1 < kMaxPoly) out[pos + 1] = vput(o1, mk(0.f)); else atomicAdd(ovf, 1);
        }
        total += __popc(b1) + __popc(b2);
    }
    __syncwarp();
    return min(total, kMaxPoly);
}

// ---------------------------------------------------------------------------
// FP32 fast path with error bounds. Clipping runs in a frame centred on body
// A (magnitudes of about the hull size, not the world), planes are kept as
// (normal, point) so no large plane constant cancels, and every decision or
// intersection whose FP32 error bound exceeds ~1e-6 m marks the pair for the
// float-float path.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void put_f32(FfVert& v, float3 p, float w) {
    v = {p.x, 0.f, p.y, 0.f, p.z, 0.f, w, 0.f};
}
__device__ __forceinline__ float3 get_f32(const FfVert& v) { return make_float3(v.xh, v.yh, v.zh); }

// Every vertex of the polygon being clipped carries the two constraints it
// lies on (in FfVert.xl as two 16-bit tags): incident-face edge j (tag j)
// or side plane k of the reference face (tag kPlaneTag + k). An edge of the
// polygon lies on the tag its two ends share, so an intersection is
// recomputed from its defining primitives, not interpolated between
// already-rounded points: the original incident edge cut by plane k, or
// the corner of two side planes on the incident face plane. The output
// order is that of the sequential clip. A vertex also carries its own
// position error bound (FfVert.wl): later inside / outside decisions on it
// widen by that bound, and only the vertices that reach the output must
// keep within kCutBudget (an intermediate vertex that a later plane clips
// away cleanly may carry more).
constexpr int kPlaneTag = 64;
// error budget of one FP32 intersection in metres: with the FP32 rounding
// of world coordinates (< 4e-6 m up to 100 m) it stays inside the 1e-5 m
// contact tolerance against the FP64 restatement
constexpr float kCutBudget = 4e-6f;


// a . b with TwoProd / TwoSum compensation (Ogita-Rump-Oishi Dot2): the
// error is that of the rounded inputs only
__device__ __forceinline__ float dot2(float3 a, float3 b) {
    // products and sums through the _rn intrinsics: no contraction may fuse
    // them, or the error terms would be lost
    const float p0 = __fmul_rn(a.x, b.x), e0 = __fmaf_rn(a.x, b.x, -p0);
    const float p1 = __fmul_rn(a.y, b.y), e1 = __fmaf_rn(a.y, b.y, -p1);
    const float p2 = __fmul_rn(a.z, b.z), e2 = __fmaf_rn(a.z, b.z, -p2);
    float t = __fadd_rn(p0, p1);
    float z = __fsub_rn(t, p0);
    float s = __fadd_rn(__fsub_rn(p0, __fsub_rn(t, z)), __fsub_rn(p1, z));
    const float t2 = __fadd_rn(t, p2);
    z = __fsub_rn(t2, t);
    s = __fadd_rn(s, __fadd_rn(__fsub_rn(t, __fsub_rn(t2, z)), __fsub_rn(p2, z)));
    s = __fadd_rn(s, __fadd_rn(e0, __fadd_rn(e1, e2)));
    return __fadd_rn(t2, s);
}
__device__ __forceinline__ bool exact_axes(const Mat3& R) {
    const float m[9] = {R.r0.x, R.r0.y, R.r0.z, R.r1.x, R.r1.y, R.r1.z, R.r2.x, R.r2.y, R.r2.z};
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 9; ++i) ok = ok && (m[i] == 0.f || m[i] == 1.f || m[i] == -1.f);
    return ok;
}

__device__ __forceinline__ unsigned tag2(int a, int b) { return (unsigned)a | ((unsigned)b << 16); }
__device__ __forceinline__ unsigned vtag(const FfVert& v) { return __float_as_uint(v.xl); }
__device__ __forceinline__ void put_tagged(FfVert& v, float3 p, unsigned tags, float err = 0.f) {
    v = {p.x, __uint_as_float(tags), p.y, 0.f, p.z, 0.f, 0.f, err};
}
__device__ __forceinline__ float verr(const FfVert& v) { return v.wl; }
__device__ __forceinline__ int shared_tag(unsigned s, unsigned e) {
    const int s0 = (int)(s & 0xffffu), s1 = (int)(s >> 16), e0 = (int)(e & 0xffffu), e1 = (int)(e >> 16);
    if (s0 == e0 || s0 == e1) return s0;
    if (s1 == e0 || s1 == e1) return s1;
    return -1;
}
// incident face vertex j in A's frame
__device__ __forceinline__ float3 inc_vertex(const ClipGeom& G, int j) {
    return f3(G.incV[j % G.fB.numIndices]);
}
// side plane k of the reference face: normal (not unit) and a point on it
__device__ __forceinline__ void side_plane(const ClipGeom& G, int k, float3& pn, float3& ap) {
    pn = f3(G.sideN[k]);
    ap = f3(G.sideP[k]);
}

// Intersection of the polygon edge on constraint `tag` with side plane k,
// and its FP32 position error bound in *err; *bad for a degenerate cut (or
// an interpolated one over the budget).
__device__ float3 exact_cut(const ClipGeom& G, int tag, int k, float3 pn, float3 ap, float3 sv, float3 ev,
                            bool* bad, float* err) {
    const float pnl = len_ub(pn);
    if (tag >= 0 && tag < kPlaneTag) {
        // incident edge j cut by plane k, from its original end points
        const float3 a = inc_vertex(G, tag), b = inc_vertex(G, tag + 1);
        const float da = dot(pn, a - ap), db = dot(pn, b - ap);
        const float den = da - db;
        // FP32 error of da, db: the end points' transform (|R v| + |rel|)
        // and the anchor, a few ulps each
        const float base = len_ub(G.rel) + len_ub(ap) + 0.5f;
        const float ea = 2.4e-7f * pnl * (len_ub(a) + base);
        const float eb = 2.4e-7f * pnl * (len_ub(b) + base);
        // position error along the edge: t = da / (da - db) moves by
        // (|db| ea + |da| eb) / den^2 (at most max(ea, eb) / |den| when
        // da and db have opposite signs, as for a crossing edge), plus the
        // rounding of a + (b - a) t
        if (!(fabsf(den) > 0.f)) *bad = true;
        const float lba = len_ub(b - a);
        *err = lba * (fabsf(db) * ea + fabsf(da) * eb) / (den * den) + 2.4e-7f * (len_ub(a) + lba);
        const float t = da / den;
        return a + (b - a) * t;
    }
    if (tag >= kPlaneTag && G.fB.pad[0]) {
        // corner of side planes l and k on the (planar) incident face plane
        // (Cramer); a welded, non-planar face keeps the interpolation below
        float3 pl, al;
        side_plane(G, tag - kPlaneTag, pl, al);
        const float3 n1 = normalize(pl), n2 = normalize(pn), n3 = G.nIn;
        const float h1 = dot(n1, al), h2 = dot(n2, ap), h3 = G.hIn;
        const float3 c23 = cross(n2, n3), c31 = cross(n3, n1), c12 = cross(n1, n2);
        const float det = dot(n1, c23);
        const float3 p = (c23 * h1 + c31 * h2 + c12 * h3) * (1.f / det);
        const float e = 3.6e-7f * (fabsf(h1) + fabsf(h2) + fabsf(h3) + len_ub(p)) + G.eIn;
        if (!(fabsf(det) > 0.f)) *bad = true;
        *err = e / fabsf(det);
        return p;
    }
    // interpolation between the current end points (an edge along a side
    // plane of a non-planar incident face); no shared constraint means a
    // degenerate polygon, which the float-float path decides
    if (tag < 0) *bad = true;
    const float ds = dot(pn, sv - ap), de = dot(pn, ev - ap);
    const float den = ds - de;
    const float apl = len_ub(ap);
    const float es = 2.5e-7f * pnl * (1.f + len_ub(sv) + apl), ee = 2.5e-7f * pnl * (1.f + len_ub(ev) + apl);
    if (!(fabsf(den) > 0.f) || len_ub(ev - sv) * (es + ee) > kCutBudget * fabsf(den)) *bad = true;
    *err = kCutBudget;
    return sv + (ev - sv) * (ds / den);
}

__device__ __noinline__ int clip_poly_f32(const ClipGeom& G, const FfVert* in, int nin, int k, FfVert* out,
                                          bool* bad, int* ovf) {
    const int lane = threadIdx.x & 31;
    float3 pn, ap;
    side_plane(G, k, pn, ap);
    const float pnl = len_ub(pn);
    const float apl = len_ub(ap);
    const unsigned newTag = (unsigned)(kPlaneTag + k);
    int total = 0;
    for (int base = 0; base < nin; base += 32) {
        const int ve = base + lane;
        int cnt = 0;
        float3 o0 = make_float3(0.f, 0.f, 0.f), o1 = o0;
        unsigned t0 = 0, t1 = 0;
        float r0 = 0.f, r1 = 0.f;
        if (ve < nin) {
            const FfVert& S0 = in[ve == 0 ? nin - 1 : ve - 1];
            const FfVert& E0 = in[ve];
            const float3 sv = get_f32(S0), ev = get_f32(E0);
            const float ds = dot(pn, sv - ap);
            const float de = dot(pn, ev - ap);
            // inside / outside decisions: FP32 error of ds, de, and of the
            // vertices themselves
            const float es = 2.5e-7f * pnl * (1.f + len_ub(sv) + apl) + pnl * verr(S0);
            const float ee = 2.5e-7f * pnl * (1.f + len_ub(ev) + apl) + pnl * verr(E0);
            if (fabsf(ds) <= es || fabsf(de) <= ee) *bad = true;
            const bool sNeg = ds < 0.f, eNeg = de < 0.f;
            if (sNeg || eNeg) {
                if (sNeg && eNeg) {
                    o0 = ev;
                    t0 = vtag(E0);
                    r0 = verr(E0);
                    cnt = 1;
                } else {
                    const int tag = shared_tag(vtag(S0), vtag(E0));
                    o0 = exact_cut(G, tag, k, pn, ap, sv, ev, bad, &r0);
                    t0 = tag2(tag < 0 ? 0 : tag, newTag);
                    cnt = 1;
                    if (!sNeg) {
                        o1 = ev;
                        t1 = vtag(E0);
                        r1 = verr(E0);
                        cnt = 2;
                    }
                }
            }
        }
        // output slots: exclusive prefix of cnt (0, 1 or 2) from two ballots
        const unsigned b1 = __ballot_sync(0xffffffffu, cnt >= 1), b2 = __ballot_sync(0xffffffffu, cnt == 2);
        const unsigned below = b3dev::lanemask_lt();
        const int pos = total + __popc(b1 & below) + __popc(b2 & below);
        if (cnt >= 1) {
            if (pos < kMaxPoly) put_tagged(out[pos], o0, t0, r0); else atomicAdd(ovf, 1);
        }
        if (cnt == 2) {
            if (pos + 1 < kMaxPoly) put_tagged(out[pos + 1], o1, t1, r1); else atomicAdd(ovf, 1);
        }
        total += __popc(b1) + __popc(b2);
    }
    __syncwarp();
    return min(total, kMaxPoly);
}

__device__ __noinline__ int clip_f32(const PairCtx& c, const b3::ShapesDev& S, const NpParams& P, int ai, int bi,
                                     WarpScratch& W, int* outBuf, bool* doubt, int* ovf) {
    const int lane = threadIdx.x & 31;
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    if (ai == kNone || bi == kNone) return 0;
    {
        ClipGeom g;
        g.sideN = W.sideN;
        g.sideP = W.sideP;
        g.incV = W.incV;
        g.fB = S.faces[pb.faceOffset + bi];
        g.fA = S.faces[pa.faceOffset + ai];
        g.fB.numIndices = min(g.fB.numIndices, kMaxPoly);
        g.fA.numIndices = min(g.fA.numIndices, kMaxPoly);
        g.RA = c.RA;
        g.RB = c.RB;
        g.rel = c.posB - c.posA;
        g.nAw = mul(c.RA, make_float3(g.fA.plane[0], g.fA.plane[1], g.fA.plane[2]));
        g.nIn = mul(c.RB, make_float3(g.fB.plane[0], g.fB.plane[1], g.fB.plane[2]));
        // incident plane in A's frame: nIn . x = -d_B + nIn . (posB - posA);
        // rel is exact for nearby bodies, the dot is compensated, and the
        // rounding of nIn only matters when B is rotated (times |rel|)
        g.hIn = -g.fB.plane[3] + dot2(g.nIn, g.rel);
        g.eIn = 2.5e-7f * (fabsf(g.fB.plane[3]) + fabsf(g.hIn)) + (exact_axes(c.RB) ? 0.f : 2.4e-7f * len_ub(g.rel));
        if (lane == 0) W.geom = g;
        __syncwarp();
    }
    const ClipGeom& G = W.geom;
    int nIn = G.fB.numIndices;
    const int nvA = G.fA.numIndices;
    // per-pair tables in shared memory: incident vertices and side planes
    for (int k = lane; k < nIn; k += 32) {
        const float4 v = __ldg(&S.verts[pb.vertexOffset + S.indices[G.fB.indexOffset + k]]);
        W.incV[k] = f4(mul(c.RB, f3(v)) + G.rel);
    }
    for (int k = lane; k < nvA; k += 32) {
        const float4 a = __ldg(&S.verts[pa.vertexOffset + S.indices[G.fA.indexOffset + k]]);
        const float4 b = __ldg(&S.verts[pa.vertexOffset + S.indices[G.fA.indexOffset + (k + 1) % nvA]]);
        W.sideN[k] = f4(-cross(mul(c.RA, make_float3(a.x - b.x, a.y - b.y, a.z - b.z)), G.nAw));
        W.sideP[k] = f4(mul(c.RA, f3(a)));
    }
    __syncwarp();
    for (int k = lane; k < nIn; k += 32) {
        // vertex k lies on incident edges k-1 and k
        put_tagged(W.poly[0][k], inc_vertex(G, k), tag2((k + nIn - 1) % nIn, k));
    }
    __syncwarp();
    bool bad = false;
    int cur = 0;
    for (int e0 = 0; e0 < nvA; ++e0) {
        nIn = clip_poly_f32(G, W.poly[cur], nIn, e0, W.poly[cur ^ 1], &bad, ovf);
        cur ^= 1;
    }
    const float3 nAw = G.nAw;
    const b3Face& fA = G.fA;
    // keep points behind the witness face; in A's frame the plane constant is
    // the face's own (clipFaceAgainstHull :433-452)
    int total = 0;
    for (int base = 0; base < nIn; base += 32) {
        const int k = base + lane;
        bool keep = false;
        float3 p = make_float3(0.f, 0.f, 0.f);
        float depth = 0.f;
        if (k < nIn) {
            p = get_f32(W.poly[cur][k]);
            const float pe = verr(W.poly[cur][k]);
            // an output point keeps within the budget; its depth decisions
            // widen by its error
            if (!(pe <= kCutBudget)) bad = true;
            depth = dot(nAw, p) + fA.plane[3];
            const float eb = 5e-7f * (1.f + len_ub(p)) + pe;
            if (fabsf(depth - P.maxDist) <= eb || fabsf(depth - P.skipDist) <= eb) bad = true;
            if (depth <= P.minDist) depth = P.minDist;
            keep = depth <= P.maxDist;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        const int pos = total + __popc(m & b3dev::lanemask_lt());
        if (keep) put_f32(W.poly[cur ^ 1][pos], p + c.posA, depth);
        total += __popc(m);
    }
    __syncwarp();
    *doubt = __any_sync(0xffffffffu, bad);
    *outBuf = cur ^ 1;
    return total;
}

// count of lanes' values within gap of the warp minimum (near-tie test)
__device__ __forceinline__ int near_count(float best, float v, bool valid, float gap) {
    return __popc(__ballot_sync(0xffffffffu, valid && v <= best + gap));
}

// FP32 extractManifoldSequentialGlobal; *tie set when an arg-min is within
// the error of its inputs of another candidate or of the FLT_MIN threshold.
// The points carry the FP32 clip's error (the 4e-6 m cut budget plus the
// rounding of world coordinates); the directions u and v come from the
// first point minus the centre, so their error grows as that vector
// shortens. A tie sends the pair to the float-float clip and reduction.
__device__ __noinline__ int4 reduce_f32(const FfVert* p, int n, float3 nearNormal, bool* tie) {
    const int lane = threadIdx.x & 31;
    const float3 o = get_f32(p[0]);  // subtract a point first: world magnitudes cancel
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int k = lane; k < n; k += 32) s += get_f32(p[k]) - o;
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, q);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, q);
        s.z += __shfl_xor_sync(0xffffffffu, s.z, q);
    }
    const float3 cr = s * (1.f / (float)n);  // centre relative to o
    const float3 aV = -cr;
    float3 u = cross(nearNormal, aV);
    const float ul = length(u);
    float3 v = cross(nearNormal, u);
    u = normalize(u);
    v = normalize(v);
    // error bounds of the points (eP) and of the directions (du)
    float pm = 0.f, rm = 0.f;
    for (int k = lane; k < n; k += 32) {
        const float3 q = get_f32(p[k]);
        pm = fmaxf(pm, len_ub(q));
        rm = fmaxf(rm, len_ub((q - o) - cr));
    }
    pm = warp_max(pm);
    rm = warp_max(rm);
    const float eP = 4e-6f + 1.2e-7f * pm;
    const float du = 2.f * eP / fmaxf(ul, 1e-30f) + 4e-7f;
    float fw[2], fu[2], fv[2];
    float mw = FLT_MAX, f0 = FLT_MIN, f1 = FLT_MIN, f2 = FLT_MIN, f3v = FLT_MIN;
    int iw = kNone, i0 = kNone, i1 = kNone, i2 = kNone, i3 = kNone;
    // a second point per lane only past 32 points (n is warp-uniform)
    const int nj = n > 32 ? 2 : 1;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int k = lane + 32 * j;
        fw[j] = FLT_MAX; fu[j] = 0.f; fv[j] = 0.f;
        if (j < nj && k < n) {
            const float3 r = (get_f32(p[k]) - o) - cr;
            fw[j] = p[k].wh;
            fu[j] = dot(u, r);
            fv[j] = dot(v, r);
            if (fw[j] < mw) { mw = fw[j]; iw = k; }
            if (fu[j] < f0) { f0 = fu[j]; i0 = k; }
            if (-fu[j] < f1) { f1 = -fu[j]; i1 = k; }
            if (fv[j] < f2) { f2 = fv[j]; i2 = k; }
            if (-fv[j] < f3v) { f3v = -fv[j]; i3 = k; }
        }
    }
    warp_argmin(mw, iw);
    warp_argmin(f0, i0);
    warp_argmin(f1, i1);
    warp_argmin(f2, i2);
    warp_argmin(f3v, i3);
    const float gap = 2.f * (2.f * eP + rm * du) + 1e-6f, gapw = 2.f * eP + 1e-6f;
    // points within the gap of each extreme, over both rounds of lanes
    int cw = 0, c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        if (j >= nj) break;
        const bool ok = lane + 32 * j < n;
        cw += near_count(mw, fw[j], ok, gapw);
        c0 += near_count(f0, fu[j], ok, gap);
        c1 += near_count(f1, -fu[j], ok, gap);
        c2 += near_count(f2, fv[j], ok, gap);
        c3 += near_count(f3v, -fv[j], ok, gap);
    }
    const int worst = max(max(cw, c0), max(max(c1, c2), c3));
    // values near the FLT_MIN start (i.e. near zero) are ambiguous too
    *tie = worst > 1 || fabsf(f0) <= gap || fabsf(f1) <= gap || fabsf(f2) <= gap || fabsf(f3v) <= gap;
    int4 idx = make_int4(i0 == kNone ? 0 : i0, i1 == kNone ? 1 : i1, i2 == kNone ? 2 : i2, i3 == kNone ? 3 : i3);
    const int minIndex = iw == kNone ? -1 : iw;
    if (idx.x != minIndex && idx.y != minIndex && idx.z != minIndex && idx.w != minIndex) idx.x = minIndex;
    return idx;
}

// First face minimising sign * dot(R n_f, sep) (the reference's strict
// comparisons: the first extreme face wins). FP32 sweep, then faces within
// a small window of the FP32 extreme are re-ranked in float-float.
__device__ __noinline__ int select_face(const b3::ShapesDev& S, PairCtx& c, bool sideA, float3 sepf, ff3 sep,
                                        float sign, bool* tied = nullptr) {
    const b3ConvexPolyhedron& h = sideA ? *c.pa : *c.pb;
    const Mat3& R = sideA ? c.RA : c.RB;
    const int lane = threadIdx.x & 31;
    float bv = FLT_MAX;
    int bi = kNone;
    float d0 = FLT_MAX;  // this lane's first face
    for (int f = lane; f < h.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[h.faceOffset + f].plane[0]);
        const float d = sign * dot(mul(R, make_float3(pl.x, pl.y, pl.z)), sepf);
        if (f == lane) d0 = d;
        if (d < bv) { bv = d; bi = f; }
    }
    float wv = bv;
    int wi = bi;
    warp_argmin(wv, wi);
    if (wi == kNone) return kNone;
    const float lim = wv + 4e-6f;
    // near-ties only: count faces inside the window
    int inWin;
    if (h.numFaces <= 32) {
        inWin = __popc(__ballot_sync(0xffffffffu, d0 <= lim));
    } else {
        inWin = 0;
        for (int f = lane; f < h.numFaces; f += 32) {
            const float4 pl = __ldg((const float4*)&S.faces[h.faceOffset + f].plane[0]);
            if (sign * dot(mul(R, make_float3(pl.x, pl.y, pl.z)), sepf) <= lim) ++inWin;
        }
        inWin = __reduce_add_sync(0xffffffffu, inWin);
    }
    if (inWin <= 1) return wi;
    // faces within the window: the choice follows the axis to float-float
    // accuracy, which the caller may have only to FP32
    if (tied) *tied = true;
    ensure_ff(c);
    const ffmat& F = sideA ? c.FA : c.FB;
    ff rv = mk(FLT_MAX);
    int ri = kNone;
    for (int f = lane; f < h.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[h.faceOffset + f].plane[0]);
        const float3 nl = make_float3(pl.x, pl.y, pl.z);
        if (!(sign * dot(mul(R, nl), sepf) <= lim)) continue;
        ff d = dot3(mrot(F, nl), sep);
        if (sign < 0.f) d = neg(d);
        if (lt(d, rv)) { rv = d; ri = f; }
    }
    warp_argmin_ff(rv, ri);
    if (ri == kNone) return wi;
    // faces within kFaceTieTol of the extreme count as tied, and the lowest
    // index wins: the reference's first extreme for faces tied in exact
    // arithmetic, whose FP64 values differ only by rounding
    int lowest = ri;
    for (int f = lane; f < h.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[h.faceOffset + f].plane[0]);
        const float3 nl = make_float3(pl.x, pl.y, pl.z);
        if (f >= lowest || !(sign * dot(mul(R, nl), sepf) <= lim)) continue;
        ff d = dot3(mrot(F, nl), sep);
        if (sign < 0.f) d = neg(d);
        if (sub(d, rv).hi <= kFaceTieTol) lowest = f;
    }
    return (int)__reduce_min_sync(0xffffffffu, (unsigned)lowest);
}

// clipHullAgainstHull (satClipHullContacts.cl:556-611 + clipFaceAgainstHull
// :353-452) in float-float; kept points (x, y, z, depth) end in
// W.poly[*outBuf].
__device__ __noinline__ int clip_hull_hull(PairCtx& c, const b3::ShapesDev& S, const NpParams& P, ff3 sep,
                              int ai, int bi, WarpScratch& W, int* outBuf, int* ovf) {
    ensure_ff(c);
    const int lane = threadIdx.x & 31;
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    if (ai == kNone || bi == kNone) return 0;
    const b3Face fB = S.faces[pb.faceOffset + bi];
    const b3Face fA = S.faces[pa.faceOffset + ai];
    const ff3 posA = mk3(c.posA.x, c.posA.y, c.posA.z);
    const ff3 posB = mk3(c.posB.x, c.posB.y, c.posB.z);
    int nIn = min(fB.numIndices, kMaxPoly);
    for (int k = lane; k < nIn; k += 32) {
        const float4 v = __ldg(&S.verts[pb.vertexOffset + S.indices[fB.indexOffset + k]]);
        W.poly[0][k] = vput(add3(mrot(c.FB, make_float3(v.x, v.y, v.z)), posB), mk(0.f));
    }
    __syncwarp();
    int cur = 0;
    const ff3 nAw = mrot(c.FA, make_float3(fA.plane[0], fA.plane[1], fA.plane[2]));
    const int nvA = min(fA.numIndices, kMaxPoly);
    // side planes of the reference face, one per lane
    for (int e0 = lane; e0 < nvA; e0 += 32) {
        const float4 a = __ldg(&S.verts[pa.vertexOffset + S.indices[fA.indexOffset + e0]]);
        const float4 b = __ldg(&S.verts[pa.vertexOffset + S.indices[fA.indexOffset + (e0 + 1) % fA.numIndices]]);
        // a - b of two FP32 vertices is exact in float-float
        const ff3 edge = sub3(mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z));
        const ff3 we{add(add(mul(c.FA.m[0][0], edge.x), mul(c.FA.m[0][1], edge.y)), mul(c.FA.m[0][2], edge.z)),
                     add(add(mul(c.FA.m[1][0], edge.x), mul(c.FA.m[1][1], edge.y)), mul(c.FA.m[1][2], edge.z)),
                     add(add(mul(c.FA.m[2][0], edge.x), mul(c.FA.m[2][1], edge.y)), mul(c.FA.m[2][2], edge.z))};
        const ff3 pn = neg3(cross3(we, nAw));
        const ff3 wa = add3(mrot(c.FA, make_float3(a.x, a.y, a.z)), posA);
        W.planes[e0] = vput(pn, neg(dot3(wa, pn)));
    }
    __syncwarp();
    for (int e0 = 0; e0 < nvA; ++e0) {
        nIn = clip_poly_ff(W.poly[cur], nIn, W.planes[e0], W.poly[cur ^ 1], ovf);
        cur ^= 1;
    }
    // keep points behind the witness face (clipFaceAgainstHull :433-452)
    const ff eqA = sub(mk(fA.plane[3]), dot3(nAw, posA));
    const ff minD = mk(P.minDist), maxD = mk(P.maxDist);
    int total = 0;
    for (int base = 0; base < nIn; base += 32) {
        const int k = base + lane;
        bool keep = false;
        ff3 p = mk3(0.f, 0.f, 0.f);
        ff depth = mk(0.f);
        if (k < nIn) {
            p = vget(W.poly[cur][k]);
            depth = add(dot3(nAw, p), eqA);
            if (le(depth, minD)) depth = minD;
            keep = le(depth, maxD);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        const int pos = total + __popc(m & b3dev::lanemask_lt());
        if (keep) W.poly[cur ^ 1][pos] = vput(p, depth);
        total += __popc(m);
    }
    __syncwarp();
    *outBuf = cur ^ 1;
    return total;
}

// extractManifoldSequentialGlobal (P2/satClipHullContacts.cl:678-770) over
// n > 4 float-float points; returns the 4 chosen indices.
__device__ __noinline__ int4 reduce_manifold(const FfVert* p, int n, ff3 nearNormal) {
    const int lane = threadIdx.x & 31;
    // centre in point order (sequential float-float sum on every lane)
    ff3 s = mk3(0.f, 0.f, 0.f);
    for (int k = 0; k < n; ++k) s = add3(s, vget(p[k]));
    const ff invn = div(mk(1.f), mk((float)n));
    const ff3 center = scale3(s, invn);
    const ff3 aV = sub3(vget(p[0]), center);
    ff3 u = cross3(nearNormal, aV);
    ff3 v = cross3(nearNormal, u);
    u = normalize3(u);
    v = normalize3(v);
    ff mw = mk(FLT_MAX), f0 = mk(FLT_MIN), f1 = mk(FLT_MIN), f2 = mk(FLT_MIN), f3v = mk(FLT_MIN);
    int iw = kNone, i0 = kNone, i1 = kNone, i2 = kNone, i3 = kNone;
    for (int k = lane; k < n; k += 32) {
        const ff w = wget(p[k]);
        if (lt(w, mw)) { mw = w; iw = k; }
        const ff3 r = sub3(vget(p[k]), center);
        const ff du = dot3(u, r), dv = dot3(v, r);
        if (lt(du, f0)) { f0 = du; i0 = k; }
        if (lt(neg(du), f1)) { f1 = neg(du); i1 = k; }
        if (lt(dv, f2)) { f2 = dv; i2 = k; }
        if (lt(neg(dv), f3v)) { f3v = neg(dv); i3 = k; }
    }
    warp_argmin_ff(mw, iw);
    warp_argmin_ff(f0, i0);
    warp_argmin_ff(f1, i1);
    warp_argmin_ff(f2, i2);
    warp_argmin_ff(f3v, i3);
    int4 idx = make_int4(i0 == kNone ? 0 : i0, i1 == kNone ? 1 : i1, i2 == kNone ? 2 : i2, i3 == kNone ? 3 : i3);
    const int minIndex = iw == kNone ? -1 : iw;
    if (idx.x != minIndex && idx.y != minIndex && idx.z != minIndex && idx.w != minIndex) idx.x = minIndex;
    return idx;
}

// Per-pair context from the pair list; false for pairs the narrowphase skips
// (two static bodies, sat.cl:944-948, or non-hull collidables).
__device__ __forceinline__ bool pair_setup(PairCtx& c, int2 pr, const b3::BodiesDev& Bd, const b3::ShapesDev& S) {
    c.A = pr.x;
    c.B = pr.y;
    c.invMassA = Bd.invMass[c.A];
    c.invMassB = Bd.invMass[c.B];
    const b3Collidable colA = S.cols[Bd.collidable[c.A]];
    const b3Collidable colB = S.cols[Bd.collidable[c.B]];
    if ((c.invMassA == 0.f && c.invMassB == 0.f) || colA.shapeType != B3_SHAPE_CONVEX_HULL ||
        colB.shapeType != B3_SHAPE_CONVEX_HULL)
        return false;
    c.pa = &S.polys[colA.shapeIndex];
    c.pb = &S.polys[colB.shapeIndex];
    c.qA = Bd.quat[c.A];
    c.qB = Bd.quat[c.B];
    c.RA = quat_to_mat(c.qA);
    c.RB = quat_to_mat(c.qB);
    c.posA = f3(Bd.pos[c.A]);
    c.posB = f3(Bd.pos[c.B]);
    c.haveFF = false;
    return true;
}

// Setup data of one pair, loaded by one lane for a chunk of pairs: the
// chain of dependent loads (pair -> collidables -> shapes, poses) is paid
// once per chunk instead of once per pair.
struct __align__(16) PairPre {
    float4 qA, qB, pA, pB;
    float4 aux;        // the clip stage: the pair's separating axis
    int A, B;
    int shapeA, shapeB;  // shapeA < 0: a pair the narrowphase skips
    float invMassA, invMassB;
    int p;
    int pad[5];
};
static_assert(sizeof(PairPre) == 128, "PairPre: 128 bytes");
static_assert(sizeof(WarpScratch::planes) >= sizeof(PairPre) * kPreChunk, "clip chunk in the plane table");

__device__ __forceinline__ void pair_prefetch(PairPre& q, int p, int2 pr, const b3::BodiesDev& Bd,
                                              const b3::ShapesDev& S) {
    q.p = p;
    q.A = pr.x;
    q.B = pr.y;
    q.invMassA = Bd.invMass[pr.x];
    q.invMassB = Bd.invMass[pr.y];
    const b3Collidable colA = S.cols[Bd.collidable[pr.x]];
    const b3Collidable colB = S.cols[Bd.collidable[pr.y]];
    const bool ok = !(q.invMassA == 0.f && q.invMassB == 0.f) && colA.shapeType == B3_SHAPE_CONVEX_HULL &&
                    colB.shapeType == B3_SHAPE_CONVEX_HULL;
    q.shapeA = ok ? colA.shapeIndex : -1;
    q.shapeB = colB.shapeIndex;
    q.qA = Bd.quat[pr.x];
    q.qB = Bd.quat[pr.y];
    q.pA = Bd.pos[pr.x];
    q.pB = Bd.pos[pr.y];
}

// PairCtx of a prefetched pair (pair_setup's result); false for a skipped
// pair.
__device__ __forceinline__ bool pair_from_pre(PairCtx& c, const PairPre& q, const b3::ShapesDev& S) {
    if (q.shapeA < 0) return false;
    c.A = q.A;
    c.B = q.B;
    c.invMassA = q.invMassA;
    c.invMassB = q.invMassB;
    c.pa = &S.polys[q.shapeA];
    c.pb = &S.polys[q.shapeB];
    c.qA = q.qA;
    c.qB = q.qB;
    c.RA = quat_to_mat(c.qA);
    c.RB = quat_to_mat(c.qB);
    c.posA = f3(q.pA);
    c.posB = f3(q.pB);
    c.haveFF = false;
    return true;
}

// pair_setup into the warp-shared context: every lane computes, lane 0
// stores, the warp synchronises.
__device__ __forceinline__ void pair_setup_shared(PairCtx& c, int2 pr, const b3::BodiesDev& Bd,
                                                  const b3::ShapesDev& S) {
    PairCtx t;
    pair_setup(t, pr, Bd, S);
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        c.A = t.A;
        c.B = t.B;
        c.invMassA = t.invMassA;
        c.invMassB = t.invMassB;
        c.pa = t.pa;
        c.pb = t.pb;
        c.qA = t.qA;
        c.qB = t.qB;
        c.RA = t.RA;
        c.RB = t.RB;
        c.haveFF = false;
        c.posA = t.posA;
        c.posB = t.posB;
    }
    __syncwarp();
}

// One side of a sub-pair: a compound child (s >= 0: its hull at the pose
// qtRotate(q, childPos) + pos, qtMul(q, childOrn) in FP32,
// findCompoundPairsKernel P2/sat.cl:774-781, in the order the oracle
// evaluates) or a polytope at the body's pose (s = -(polytope + 1)).
__device__ __forceinline__ void sub_side(const b3::BodiesDev& Bd, const b3::ShapesDev& S, int body, int s, int& poly,
                                         float4& q, float4& pos) {
    const float4 bq = Bd.quat[body], bp = Bd.pos[body];
    if (s >= 0) {
        const b3ChildShape& ch = S.children[s];
        poly = S.cols[ch.shapeIndex].shapeIndex;
        const float4 cp = make_float4(ch.childPosition[0], ch.childPosition[1], ch.childPosition[2], 0.f);
        const float4 cq = make_float4(ch.childOrientation[0], ch.childOrientation[1], ch.childOrientation[2],
                                      ch.childOrientation[3]);
        const float4 r = b3m::qt_rotate_rn(bq, cp);
        pos = make_float4(b3m::arn(r.x, bp.x), b3m::arn(r.y, bp.y), b3m::arn(r.z, bp.z), 0.f);
        q = b3m::qt_mul_rn(bq, cq);
    } else {
        poly = -s - 1;
        q = bq;
        pos = bp;
    }
}

// Setup of the item in slot `slot`: a broadphase pair (slot = pair index),
// or with kSub the sub-pair slot - base of a compound or mesh pair.
template <bool kSub>
__device__ __forceinline__ void item_prefetch(PairPre& q, int slot, const int2* __restrict__ pairs,
                                              const int4* __restrict__ subs, int base, const b3::BodiesDev& Bd,
                                              const b3::ShapesDev& S) {
    if (!kSub) {
        pair_prefetch(q, slot, pairs[slot], Bd, S);
        return;
    }
    const int4 sp = subs[slot - base];
    q.p = slot;
    q.A = sp.x;
    q.B = sp.y;
    q.invMassA = Bd.invMass[sp.x];
    q.invMassB = Bd.invMass[sp.y];
    int pa, pb;
    sub_side(Bd, S, sp.x, sp.z, pa, q.qA, q.pA);
    sub_side(Bd, S, sp.y, sp.w, pb, q.qB, q.pB);
    q.shapeA = pa;
    q.shapeB = pb;
}

template <bool kSub>
__device__ __forceinline__ void item_setup_shared(PairCtx& c, int slot, const int2* __restrict__ pairs,
                                                  const int4* __restrict__ subs, int base, const b3::BodiesDev& Bd,
                                                  const b3::ShapesDev& S) {
    if (!kSub) {
        pair_setup_shared(c, pairs[slot], Bd, S);
        return;
    }
    PairPre q;
    item_prefetch<true>(q, slot, pairs, subs, base, Bd, S);
    PairCtx t;
    pair_from_pre(t, q, S);
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        c.A = t.A;
        c.B = t.B;
        c.invMassA = t.invMassA;
        c.invMassB = t.invMassB;
        c.pa = t.pa;
        c.pb = t.pb;
        c.qA = t.qA;
        c.qB = t.qB;
        c.RA = t.RA;
        c.RB = t.RB;
        c.haveFF = false;
        c.posA = t.posA;
        c.posB = t.posB;
    }
    __syncwarp();
}

// Contact4 of pair p from the kept points pts[0..nOut) and the chosen
// indices (newContactReductionKernel, P2/satClipHullContacts.cl:1958-2039).
__device__ __forceinline__ void emit_contact(int p, const PairCtx& c, const FfVert* pts, int nRed, int4 idx,
                                             float3 nrm, const b3::BodiesDev& Bd, const NpParams& P,
                                             b3Contact4* __restrict__ contacts, uint32_t* __restrict__ manifoldFlag) {
    const int lane = threadIdx.x & 31;
    b3Contact4* out = &contacts[p];
    if (lane < nRed) {
        const int k = lane == 0 ? idx.x : lane == 1 ? idx.y : lane == 2 ? idx.z : idx.w;
        const FfVert q = pts[k];
        *reinterpret_cast<float4*>(&out->worldPos[lane][0]) =
            make_float4(q.xh + q.xl, q.yh + q.yl, q.zh + q.zl, q.wh + q.wl);
    } else if (lane < 4) {
        *reinterpret_cast<float4*>(&out->worldPos[lane][0]) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (lane == 4) {
        *reinterpret_cast<float4*>(&out->worldNormal[0]) = make_float4(nrm.x, nrm.y, nrm.z, (float)nRed);
        out->friction = combine_friction(Bd.friction[c.A], Bd.friction[c.B], P.frictionCombine);
        out->pairIndex = p;
        out->bodyAPtrAndSignBit = c.invMassA == 0.f ? -c.A : c.A;
        out->bodyBPtrAndSignBit = c.invMassB == 0.f ? -c.B : c.B;
        manifoldFlag[p] = 1u;
    }
}

__device__ __forceinline__ int next_work(int32_t* counter, int limit, int chunk) {
    int w = 0;
    if ((threadIdx.x & 31) == 0) w = atomicAdd(counter, chunk);
    w = __shfl_sync(0xffffffffu, w, 0);
    return w < limit ? w : -1;
}

__device__ __forceinline__ int push(int* queue, int32_t* count, int p) {
    int slot = 0;
    if ((threadIdx.x & 31) == 0) {
        slot = atomicAdd(count, 1);
        queue[slot] = p;
    }
    return __shfl_sync(0xffffffffu, slot, 0);
}

// Stage 1, every pair: the FP32 separating-axis sweep. Separated pairs are
// finished here; pairs whose axis the sweep decides go to the FP32 clip
// queue with that axis; pairs with near-minimum candidates go to the
// float-float queue.
// kSub: the items are the sub-pairs of compound and mesh pairs, in the
// slots after the pairs' (slot = numPairs + sub-pair).
// Six blocks per SM (80 registers): with the projection loop unrolled the
// extra resident warps hide more of the vertex loads' latency than the
// spills cost (settled 131,072-body step: sweep 4.01 -> 3.46 ms).
template <bool kEarlyFaces, bool kSub>
__global__ void __launch_bounds__(128, 6)
k_np_sweep(const int2* __restrict__ pairs, const int4* __restrict__ subs, const int32_t* __restrict__ numPairsDev,
           b3::BodiesDev Bd, b3::ShapesDev S, uint32_t* __restrict__ manifoldFlag, float4* __restrict__ pairSep,
           int* __restrict__ fastQ, int* __restrict__ slowQ, int* __restrict__ cand, int candSlots,
           int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    const int lane = threadIdx.x & 31;
    unsigned char* wbase = np_smem + (size_t)(threadIdx.x >> 5) * kSweepWarpSmem;
    PairPre* pre = reinterpret_cast<PairPre*>(wbase);
    int* wcand = reinterpret_cast<int*>(wbase + sizeof(PairPre) * kPreChunk);
    const int numItems = kSub ? scalars[b3::S_NUM_SUB] : *numPairsDev;
    const int base = kSub ? *numPairsDev : 0;
    for (;;) {
        const int chunk = next_work(scalars + b3::S_NP_WORK, numItems, kPreChunk);
        if (chunk < 0) break;
        const int n = min(kPreChunk, numItems - chunk);
        if (lane < n) item_prefetch<kSub>(pre[lane], base + chunk + lane, pairs, subs, base, Bd, S);
        __syncwarp();
        for (int i = 0; i < n; ++i) {
            const int p = base + chunk + i;
            PairCtx c;
            int r = 0, count = 0;
            float3 sepf = make_float3(0.f, 0.f, 0.f);
            if (pair_from_pre(c, pre[i], S))
                r = sweep_axes<kEarlyFaces>(c, S, wcand, sepf, count, &counters->clipOverflow);
            if (r == 0) {
                if (lane == 0) manifoldFlag[p] = 0u;
            } else if (r == 1) {
                if (lane == 0) pairSep[p] = make_float4(sepf.x, sepf.y, sepf.z, (float)kSepDecided);
                push(fastQ, scalars + b3::S_NP_FAST, p);
            } else {
                // keep the near-minimum candidates for the exact stage
                const int slot = push(slowQ, scalars + b3::S_NP_SLOW, p);
                const bool kept = slot < candSlots;
                if (kept && lane < count) cand[(size_t)slot * kMaxCand + lane] = wcand[lane];
                if (lane == 0)
                    pairSep[p] = make_float4(__int_as_float(kept ? count : -1), 0.f, 0.f, (float)kSepRefine);
            }
            __syncwarp();
        }
    }
}

// Stage 2, pairs with an FP32 axis: face selection, clipping and reduction
// in FP32 with error bounds; any doubt sends the pair to the float-float
// queue instead. (Four blocks per SM, 128 registers, measured 4-5 % faster
// than five or six on the settled workloads.) The queue is the clip queue
// (scalars[countSlot] entries, work counter scalars[workSlot]): every pair
// with an FP32 axis, or the pairs the lane-group clip passed on.
template <bool kSub>
__global__ void __launch_bounds__(128, 4)
k_np_clip(const int2* __restrict__ pairs, const int4* __restrict__ subs, b3::BodiesDev Bd, b3::ShapesDev S, NpParams P,
          float4* __restrict__ pairSep, const int* __restrict__ clipQ, int countSlot, int workSlot,
          int* __restrict__ slowQ, b3Contact4* __restrict__ contacts, uint32_t* __restrict__ manifoldFlag,
          int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    const int lane = threadIdx.x & 31;
    WarpScratch& W = reinterpret_cast<WarpScratch*>(np_smem)[threadIdx.x >> 5];
    const int nFast = scalars[countSlot];
    // the prefetched chunk lives in the float-float plane table, which only
    // the exact stage uses
    PairPre* pre = reinterpret_cast<PairPre*>(W.planes);
    for (;;) {
        const int chunk = next_work(scalars + workSlot, nFast, kPreChunk);
        if (chunk < 0) break;
        const int n = min(kPreChunk, nFast - chunk);
        if (lane < n) {
            const int p = clipQ[chunk + lane];
            item_prefetch<kSub>(pre[lane], p, pairs, subs, scalars[b3::S_NUM_PAIRS], Bd, S);
            pre[lane].aux = pairSep[p];
        }
        __syncwarp();
        for (int i = 0; i < n; ++i) {
            const int p = pre[i].p;
            PairCtx& c = W.ctx;
            {
                PairCtx t;
                pair_from_pre(t, pre[i], S);
                if (lane == 0) c = t;
                __syncwarp();
            }
            const float4 s4 = pre[i].aux;
            const float3 sepf = make_float3(s4.x, s4.y, s4.z);
            const ff3 sep = mk3(sepf.x, sepf.y, sepf.z);
            // incident face of B: max dot(nB, sep); reference face of A: min dot(nA, sep)
            bool faceTie = false;
            const int bi = select_face(S, c, false, sepf, sep, -1.f, &faceTie);
            const int ai = select_face(S, c, true, sepf, sep, 1.f, &faceTie);
            int buf = 0;
            bool slow = false;
            int nOut = 0;
            if (!faceTie && ref_face_clips(S, c, ai))
                nOut = clip_f32(c, S, P, ai, bi, W, &buf, &slow, &counters->clipOverflow);
            int4 idx = make_int4(0, 1, 2, 3);
            int nRed = nOut;
            bool tie = false;
            if (!faceTie && !slow && nOut > 4) {
                idx = reduce_f32(W.poly[buf], min(nOut, kMaxPoly), -sepf, &tie);
                nRed = 4;
            }
            if (faceTie || slow || tie) {
                // the exact stage redoes the part in doubt: the axis (faces
                // near-tied along it), or the clip (its own doubt, or a
                // reduction decided by points within their error bound)
                if (lane == 0) pairSep[p].w = (float)(faceTie ? kSepFaceTie : kSepClipDoubt);
                push(slowQ, scalars + b3::S_NP_SLOW, p);
            } else if (nOut > 0) {
                emit_contact(p, c, W.poly[buf], nRed, idx, -sepf, Bd, P, contacts, manifoldFlag);
            } else if (lane == 0) {
                manifoldFlag[p] = 0u;
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// Stage 2 by lane groups: kClipGroup lanes per pair, four pairs per warp.
// A cube face clipped by a cube face keeps 4 to 8 of a warp's 32 lanes busy;
// a group of 8 lanes runs the same face selection, clip, depth filter,
// reduction and Contact4 with the same arithmetic in the same order (each
// per-vertex and per-face value is computed alike; compactions keep the
// sequential order; the centroid sum of at most 16 points associates as the
// 32-lane butterfly does, whose first step only adds zeros), so a pair gets
// the same bits from either. A pair whose faces or clipped polygon exceed
// the group's 16-vertex tables goes to the clip queue of the warp kernel,
// which redoes it from the start; a pair whose clip faces tie goes to the
// float-float stage, as from the warp kernel.
// ---------------------------------------------------------------------------
constexpr int kClipGroup = 8;                // lanes per pair
constexpr int kGroupPoly = 2 * kClipGroup;   // vertex capacity of a group's polygons and face tables

struct __align__(16) GroupScratch {
    FfVert poly[2][kGroupPoly];
    float4 sideN[kGroupPoly];
    float4 sideP[kGroupPoly];
    float4 incV[kGroupPoly];
    PairCtx ctx;
    ClipGeom geom;
    PairPre pre;
};

__device__ __forceinline__ int grp_lane() { return threadIdx.x & (kClipGroup - 1); }
__device__ __forceinline__ unsigned grp_mask() {
    return ((1u << kClipGroup) - 1u) << ((threadIdx.x & 31) & ~(kClipGroup - 1));
}
__device__ __forceinline__ float grp_max(float v, unsigned m) {
    return fkey_inv(__reduce_max_sync(m, fkey(v, kNanMax)));
}
// (value, index) minimum over the group, as warp_argmin
__device__ __forceinline__ void grp_argmin(float& v, int& idx, unsigned m) {
    const int k = fkey(v, kNanMin);
    const int km = __reduce_min_sync(m, k);
    idx = (int)__reduce_min_sync(m, k == km ? (unsigned)idx : 0xffffffffu);
    v = fkey_inv(km);
}

// select_face over the group's lanes; faces within the window of the FP32
// extreme only set *tied (the pair then goes to the float-float stage,
// which decides them).
__device__ __noinline__ int select_face_g(const b3::ShapesDev& S, const PairCtx& c, bool sideA, float3 sepf,
                                          float sign, bool* tied) {
    const b3ConvexPolyhedron& h = sideA ? *c.pa : *c.pb;
    const Mat3& R = sideA ? c.RA : c.RB;
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    float bv = FLT_MAX;
    int bi = kNone;
    float d0 = FLT_MAX;  // this lane's first face
    for (int f = gl; f < h.numFaces; f += kClipGroup) {
        const float4 pl = __ldg((const float4*)&S.faces[h.faceOffset + f].plane[0]);
        const float d = sign * dot(mul(R, make_float3(pl.x, pl.y, pl.z)), sepf);
        if (f == gl) d0 = d;
        if (d < bv) { bv = d; bi = f; }
    }
    float wv = bv;
    int wi = bi;
    grp_argmin(wv, wi, gm);
    if (wi == kNone) return kNone;
    const float lim = wv + 4e-6f;
    int inWin;
    if (h.numFaces <= kClipGroup) {
        inWin = __popc(__ballot_sync(gm, d0 <= lim));
    } else {
        inWin = 0;
        for (int f = gl; f < h.numFaces; f += kClipGroup) {
            const float4 pl = __ldg((const float4*)&S.faces[h.faceOffset + f].plane[0]);
            if (sign * dot(mul(R, make_float3(pl.x, pl.y, pl.z)), sepf) <= lim) ++inWin;
        }
        inWin = __reduce_add_sync(gm, inWin);
    }
    if (inWin > 1) *tied = true;
    return wi;
}

// clip_poly_f32 over the group; *over when the output exceeds kGroupPoly
// (nothing past it is written).
__device__ __noinline__ int clip_poly_f32_g(const ClipGeom& G, const FfVert* in, int nin, int k, FfVert* out,
                                            bool* bad, bool* over) {
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    float3 pn, ap;
    side_plane(G, k, pn, ap);
    const float pnl = len_ub(pn);
    const float apl = len_ub(ap);
    const unsigned newTag = (unsigned)(kPlaneTag + k);
    int total = 0;
    for (int base = 0; base < nin; base += kClipGroup) {
        const int ve = base + gl;
        int cnt = 0;
        float3 o0 = make_float3(0.f, 0.f, 0.f), o1 = o0;
        unsigned t0 = 0, t1 = 0;
        float r0 = 0.f, r1 = 0.f;
        if (ve < nin) {
            const FfVert& S0 = in[ve == 0 ? nin - 1 : ve - 1];
            const FfVert& E0 = in[ve];
            const float3 sv = get_f32(S0), ev = get_f32(E0);
            const float ds = dot(pn, sv - ap);
            const float de = dot(pn, ev - ap);
            const float es = 2.5e-7f * pnl * (1.f + len_ub(sv) + apl) + pnl * verr(S0);
            const float ee = 2.5e-7f * pnl * (1.f + len_ub(ev) + apl) + pnl * verr(E0);
            if (fabsf(ds) <= es || fabsf(de) <= ee) *bad = true;
            const bool sNeg = ds < 0.f, eNeg = de < 0.f;
            if (sNeg || eNeg) {
                if (sNeg && eNeg) {
                    o0 = ev;
                    t0 = vtag(E0);
                    r0 = verr(E0);
                    cnt = 1;
                } else {
                    const int tag = shared_tag(vtag(S0), vtag(E0));
                    o0 = exact_cut(G, tag, k, pn, ap, sv, ev, bad, &r0);
                    t0 = tag2(tag < 0 ? 0 : tag, newTag);
                    cnt = 1;
                    if (!sNeg) {
                        o1 = ev;
                        t1 = vtag(E0);
                        r1 = verr(E0);
                        cnt = 2;
                    }
                }
            }
        }
        const unsigned b1 = __ballot_sync(gm, cnt >= 1), b2 = __ballot_sync(gm, cnt == 2);
        const unsigned below = b3dev::lanemask_lt();
        const int pos = total + __popc(b1 & below) + __popc(b2 & below);
        if (cnt >= 1 && pos < kGroupPoly) put_tagged(out[pos], o0, t0, r0);
        if (cnt == 2 && pos + 1 < kGroupPoly) put_tagged(out[pos + 1], o1, t1, r1);
        total += __popc(b1) + __popc(b2);
    }
    __syncwarp(gm);
    if (total > kGroupPoly) *over = true;
    return min(total, kGroupPoly);
}

// clip_f32 over the group. *defer: a face or the clipped polygon exceeds the
// group's tables (nothing is decided; the warp kernel redoes the pair).
__device__ __noinline__ int clip_f32_g(const PairCtx& c, const b3::ShapesDev& S, const NpParams& P, int ai, int bi,
                                       GroupScratch& W, int* outBuf, bool* doubt, bool* defer) {
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    if (ai == kNone || bi == kNone) return 0;
    {
        ClipGeom g;
        g.sideN = W.sideN;
        g.sideP = W.sideP;
        g.incV = W.incV;
        g.fB = S.faces[pb.faceOffset + bi];
        g.fA = S.faces[pa.faceOffset + ai];
        g.fB.numIndices = min(g.fB.numIndices, kMaxPoly);
        g.fA.numIndices = min(g.fA.numIndices, kMaxPoly);
        g.RA = c.RA;
        g.RB = c.RB;
        g.rel = c.posB - c.posA;
        g.nAw = mul(c.RA, make_float3(g.fA.plane[0], g.fA.plane[1], g.fA.plane[2]));
        g.nIn = mul(c.RB, make_float3(g.fB.plane[0], g.fB.plane[1], g.fB.plane[2]));
        g.hIn = -g.fB.plane[3] + dot2(g.nIn, g.rel);
        g.eIn = 2.5e-7f * (fabsf(g.fB.plane[3]) + fabsf(g.hIn)) + (exact_axes(c.RB) ? 0.f : 2.4e-7f * len_ub(g.rel));
        if (gl == 0) W.geom = g;
        __syncwarp(gm);
    }
    const ClipGeom& G = W.geom;
    int nIn = G.fB.numIndices;
    const int nvA = G.fA.numIndices;
    if (nIn > kGroupPoly || nvA > kGroupPoly) {
        *defer = true;
        return 0;
    }
    for (int k = gl; k < nIn; k += kClipGroup) {
        const float4 v = __ldg(&S.verts[pb.vertexOffset + S.indices[G.fB.indexOffset + k]]);
        W.incV[k] = f4(mul(c.RB, f3(v)) + G.rel);
    }
    for (int k = gl; k < nvA; k += kClipGroup) {
        const float4 a = __ldg(&S.verts[pa.vertexOffset + S.indices[G.fA.indexOffset + k]]);
        const float4 b = __ldg(&S.verts[pa.vertexOffset + S.indices[G.fA.indexOffset + (k + 1) % nvA]]);
        W.sideN[k] = f4(-cross(mul(c.RA, make_float3(a.x - b.x, a.y - b.y, a.z - b.z)), G.nAw));
        W.sideP[k] = f4(mul(c.RA, f3(a)));
    }
    __syncwarp(gm);
    for (int k = gl; k < nIn; k += kClipGroup)
        put_tagged(W.poly[0][k], inc_vertex(G, k), tag2((k + nIn - 1) % nIn, k));
    __syncwarp(gm);
    bool bad = false, over = false;
    int cur = 0;
    for (int e0 = 0; e0 < nvA && !over; ++e0) {
        nIn = clip_poly_f32_g(G, W.poly[cur], nIn, e0, W.poly[cur ^ 1], &bad, &over);
        cur ^= 1;
    }
    if (over) {
        *defer = true;
        return 0;
    }
    const float3 nAw = G.nAw;
    const b3Face& fA = G.fA;
    int total = 0;
    for (int base = 0; base < nIn; base += kClipGroup) {
        const int k = base + gl;
        bool keep = false;
        float3 p = make_float3(0.f, 0.f, 0.f);
        float depth = 0.f;
        if (k < nIn) {
            p = get_f32(W.poly[cur][k]);
            const float pe = verr(W.poly[cur][k]);
            if (!(pe <= kCutBudget)) bad = true;
            depth = dot(nAw, p) + fA.plane[3];
            const float eb = 5e-7f * (1.f + len_ub(p)) + pe;
            if (fabsf(depth - P.maxDist) <= eb || fabsf(depth - P.skipDist) <= eb) bad = true;
            if (depth <= P.minDist) depth = P.minDist;
            keep = depth <= P.maxDist;
        }
        const unsigned m = __ballot_sync(gm, keep);
        const int pos = total + __popc(m & b3dev::lanemask_lt());
        if (keep) put_f32(W.poly[cur ^ 1][pos], p + c.posA, depth);
        total += __popc(m);
    }
    __syncwarp(gm);
    *doubt = __any_sync(gm, bad);
    *outBuf = cur ^ 1;
    return total;
}

// reduce_f32 over the group, for n <= kGroupPoly points (two per lane).
__device__ __noinline__ int4 reduce_f32_g(const FfVert* p, int n, float3 nearNormal, bool* tie) {
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    const float3 o = get_f32(p[0]);
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int k = gl; k < n; k += kClipGroup) s += get_f32(p[k]) - o;
#pragma unroll
    for (int q = kClipGroup / 2; q > 0; q >>= 1) {
        s.x += __shfl_xor_sync(gm, s.x, q);
        s.y += __shfl_xor_sync(gm, s.y, q);
        s.z += __shfl_xor_sync(gm, s.z, q);
    }
    const float3 cr = s * (1.f / (float)n);
    const float3 aV = -cr;
    float3 u = cross(nearNormal, aV);
    const float ul = length(u);
    float3 v = cross(nearNormal, u);
    u = normalize(u);
    v = normalize(v);
    float pm = 0.f, rm = 0.f;
    for (int k = gl; k < n; k += kClipGroup) {
        const float3 q = get_f32(p[k]);
        pm = fmaxf(pm, len_ub(q));
        rm = fmaxf(rm, len_ub((q - o) - cr));
    }
    pm = grp_max(pm, gm);
    rm = grp_max(rm, gm);
    const float eP = 4e-6f + 1.2e-7f * pm;
    const float du = 2.f * eP / fmaxf(ul, 1e-30f) + 4e-7f;
    float fw[2], fu[2], fv[2];
    float mw = FLT_MAX, f0 = FLT_MIN, f1 = FLT_MIN, f2 = FLT_MIN, f3v = FLT_MIN;
    int iw = kNone, i0 = kNone, i1 = kNone, i2 = kNone, i3 = kNone;
    const int nj = n > kClipGroup ? 2 : 1;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int k = gl + kClipGroup * j;
        fw[j] = FLT_MAX; fu[j] = 0.f; fv[j] = 0.f;
        if (j < nj && k < n) {
            const float3 r = (get_f32(p[k]) - o) - cr;
            fw[j] = p[k].wh;
            fu[j] = dot(u, r);
            fv[j] = dot(v, r);
            if (fw[j] < mw) { mw = fw[j]; iw = k; }
            if (fu[j] < f0) { f0 = fu[j]; i0 = k; }
            if (-fu[j] < f1) { f1 = -fu[j]; i1 = k; }
            if (fv[j] < f2) { f2 = fv[j]; i2 = k; }
            if (-fv[j] < f3v) { f3v = -fv[j]; i3 = k; }
        }
    }
    grp_argmin(mw, iw, gm);
    grp_argmin(f0, i0, gm);
    grp_argmin(f1, i1, gm);
    grp_argmin(f2, i2, gm);
    grp_argmin(f3v, i3, gm);
    const float gap = 2.f * (2.f * eP + rm * du) + 1e-6f, gapw = 2.f * eP + 1e-6f;
    int cw = 0, c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        if (j >= nj) break;
        const bool ok = gl + kClipGroup * j < n;
        cw += __popc(__ballot_sync(gm, ok && fw[j] <= mw + gapw));
        c0 += __popc(__ballot_sync(gm, ok && fu[j] <= f0 + gap));
        c1 += __popc(__ballot_sync(gm, ok && -fu[j] <= f1 + gap));
        c2 += __popc(__ballot_sync(gm, ok && fv[j] <= f2 + gap));
        c3 += __popc(__ballot_sync(gm, ok && -fv[j] <= f3v + gap));
    }
    const int worst = max(max(cw, c0), max(max(c1, c2), c3));
    *tie = worst > 1 || fabsf(f0) <= gap || fabsf(f1) <= gap || fabsf(f2) <= gap || fabsf(f3v) <= gap;
    int4 idx = make_int4(i0 == kNone ? 0 : i0, i1 == kNone ? 1 : i1, i2 == kNone ? 2 : i2, i3 == kNone ? 3 : i3);
    const int minIndex = iw == kNone ? -1 : iw;
    if (idx.x != minIndex && idx.y != minIndex && idx.z != minIndex && idx.w != minIndex) idx.x = minIndex;
    return idx;
}

// emit_contact by the group's lanes
__device__ __forceinline__ void emit_contact_g(int p, const PairCtx& c, const FfVert* pts, int nRed, int4 idx,
                                               float3 nrm, const b3::BodiesDev& Bd, const NpParams& P,
                                               b3Contact4* __restrict__ contacts, uint32_t* __restrict__ manifoldFlag) {
    const int gl = grp_lane();
    b3Contact4* out = &contacts[p];
    if (gl < nRed) {
        const int k = gl == 0 ? idx.x : gl == 1 ? idx.y : gl == 2 ? idx.z : idx.w;
        const FfVert q = pts[k];
        *reinterpret_cast<float4*>(&out->worldPos[gl][0]) =
            make_float4(q.xh + q.xl, q.yh + q.yl, q.zh + q.zl, q.wh + q.wl);
    } else if (gl < 4) {
        *reinterpret_cast<float4*>(&out->worldPos[gl][0]) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (gl == 4) {
        *reinterpret_cast<float4*>(&out->worldNormal[0]) = make_float4(nrm.x, nrm.y, nrm.z, (float)nRed);
        out->friction = combine_friction(Bd.friction[c.A], Bd.friction[c.B], P.frictionCombine);
        out->pairIndex = p;
        out->bodyAPtrAndSignBit = c.invMassA == 0.f ? -c.A : c.A;
        out->bodyBPtrAndSignBit = c.invMassB == 0.f ? -c.B : c.B;
        manifoldFlag[p] = 1u;
    }
}

// Stage 2 by lane groups over the clip queue: four pairs per warp per work
// grab, lane l < 4 prefetching group l's pair. Pairs the groups cannot hold
// go to deferQ for k_np_clip.
template <bool kSub>
__global__ void __launch_bounds__(128, 4)
k_np_clip_groups(const int2* __restrict__ pairs, const int4* __restrict__ subs, b3::BodiesDev Bd, b3::ShapesDev S,
                 NpParams P, float4* __restrict__ pairSep, const int* __restrict__ fastQ, int* __restrict__ slowQ,
                 int* __restrict__ deferQ, b3Contact4* __restrict__ contacts, uint32_t* __restrict__ manifoldFlag,
                 int32_t* __restrict__ scalars) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    constexpr int kPerWarp = 32 / kClipGroup;
    const int lane = threadIdx.x & 31;
    GroupScratch* Wg = reinterpret_cast<GroupScratch*>(np_smem) + (threadIdx.x >> 5) * kPerWarp;
    const int g = lane / kClipGroup;
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    GroupScratch& W = Wg[g];
    const int nFast = scalars[b3::S_NP_FAST];
    for (;;) {
        const int chunk = next_work(scalars + b3::S_NP_WORK2, nFast, kPerWarp);
        if (chunk < 0) break;
        const int n = min(kPerWarp, nFast - chunk);
        if (lane < n) {
            const int p = fastQ[chunk + lane];
            item_prefetch<kSub>(Wg[lane].pre, p, pairs, subs, scalars[b3::S_NUM_PAIRS], Bd, S);
            Wg[lane].pre.aux = pairSep[p];
        }
        __syncwarp();
        if (g < n) {
            const int p = W.pre.p;
            PairCtx& c = W.ctx;
            {
                PairCtx t;
                pair_from_pre(t, W.pre, S);
                __syncwarp(gm);
                if (gl == 0) c = t;
                __syncwarp(gm);
            }
            const float4 s4 = W.pre.aux;
            const float3 sepf = make_float3(s4.x, s4.y, s4.z);
            bool faceTie = false;
            const int bi = select_face_g(S, c, false, sepf, -1.f, &faceTie);
            const int ai = select_face_g(S, c, true, sepf, 1.f, &faceTie);
            int buf = 0;
            bool slow = false, defer = false;
            int nOut = 0;
            if (!faceTie && ref_face_clips(S, c, ai)) nOut = clip_f32_g(c, S, P, ai, bi, W, &buf, &slow, &defer);
            int4 idx = make_int4(0, 1, 2, 3);
            int nRed = nOut;
            bool tie = false;
            if (!defer && !faceTie && !slow && nOut > 4) {
                idx = reduce_f32_g(W.poly[buf], nOut, -sepf, &tie);
                nRed = 4;
            }
            if (defer) {
                if (gl == 0) deferQ[atomicAdd(scalars + b3::S_NP_DEFER, 1)] = p;
            } else if (faceTie || slow || tie) {
                if (gl == 0) {
                    pairSep[p].w = (float)(faceTie ? kSepFaceTie : kSepClipDoubt);
                    slowQ[atomicAdd(scalars + b3::S_NP_SLOW, 1)] = p;
                }
            } else if (nOut > 0) {
                emit_contact_g(p, c, W.poly[buf], nRed, idx, -sepf, Bd, P, contacts, manifoldFlag);
            } else if (gl == 0) {
                manifoldFlag[p] = 0u;
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// The float-float stages by lane groups, as the FP32 clip above: the ranking
// of a pair's near-tied axes (at most kClipGroup candidates, one per lane)
// and the float-float clip of a pair whose FP32 clip was in doubt. Each pair
// gets the warp kernels' bits (the same per-candidate, per-vertex and
// per-point arithmetic; order-independent reductions; compactions in the
// sequential order). Pairs outside the group tables (more candidates, faces
// or clipped points than they hold, or clip faces tied along the FP32 axis,
// whose axis the full search must redo) are passed to the warp kernels.
// ---------------------------------------------------------------------------
struct __align__(16) GroupScratchFF {
    FfVert poly[2][kGroupPoly];   // clip polygons; the ranking's staged vertices
    FfVert planes[kGroupPoly];    // float-float side planes
    PairCtx ctx;
    int cand[kClipGroup];
};

__device__ __forceinline__ void ensure_ff_g(PairCtx& c, unsigned gm) {
    const bool have = c.haveFF;
    __syncwarp(gm);
    if (!have) {
        const ffmat a = quat_mat(c.qA), b = quat_mat(c.qB);
        if (grp_lane() == 0) {
            c.FA = a;
            c.FB = b;
            c.haveFF = true;
        }
        __syncwarp(gm);
    }
}

// (hi, lo, index) minimum over the group, as warp_argmin_ff
__device__ __forceinline__ void grp_argmin_ff(ff& v, int& idx, unsigned m) {
    const int kh = fkey(v.hi, kNanMin);
    const int mh = __reduce_min_sync(m, kh);
    const int kl = kh == mh ? fkey(v.lo, kNanMin) : kNanMin;
    const int ml = __reduce_min_sync(m, kl);
    idx = (int)__reduce_min_sync(m, kh == mh && kl == ml ? (unsigned)idx : 0xffffffffu);
    v.hi = fkey_inv(mh);
    v.lo = fkey_inv(ml);
}

// PairCtx of item p into the group's shared context (every lane computes,
// the group leader stores)
template <bool kSub>
__device__ __forceinline__ void item_setup_group(PairCtx& c, int p, const int2* __restrict__ pairs,
                                                 const int4* __restrict__ subs, int base, const b3::BodiesDev& Bd,
                                                 const b3::ShapesDev& S, unsigned gm) {
    PairPre q;
    item_prefetch<kSub>(q, p, pairs, subs, base, Bd, S);
    PairCtx t;
    pair_from_pre(t, q, S);
    __syncwarp(gm);
    if (grp_lane() == 0) {
        c.A = t.A;
        c.B = t.B;
        c.invMassA = t.invMassA;
        c.invMassB = t.invMassB;
        c.pa = t.pa;
        c.pb = t.pb;
        c.qA = t.qA;
        c.qB = t.qB;
        c.RA = t.RA;
        c.RB = t.RB;
        c.haveFF = false;
        c.posA = t.posA;
        c.posB = t.posB;
    }
    __syncwarp(gm);
}

// refine_axes over the group, count <= kClipGroup candidates in W.cand
__device__ __noinline__ bool refine_axes_g(PairCtx& c, const b3::ShapesDev& S, GroupScratchFF& W, int count,
                                           ff3& sep) {
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    const float3 lcA = make_float3(pa.localCenter[0], pa.localCenter[1], pa.localCenter[2]);
    const float3 lcB = make_float3(pb.localCenter[0], pb.localCenter[1], pb.localCenter[2]);
    ensure_ff_g(c, gm);
    const ff3 lcAw = mrot(c.FA, make_float3(lcA.x, lcA.y, lcA.z));
    const ff3 lcBw = mrot(c.FB, make_float3(lcB.x, lcB.y, lcB.z));
    const ff3 Dff = sub3(add3(lcAw, mk3(c.posA.x, c.posA.y, c.posA.z)), add3(lcBw, mk3(c.posB.x, c.posB.y, c.posB.z)));
    const float4* vA = S.verts + pa.vertexOffset;
    const float4* vB = S.verts + pb.vertexOffset;
    constexpr int kStage = (int)(sizeof(W.poly) / sizeof(float4));
    if (pa.numVertices + pb.numVertices <= kStage) {
        float4* st = reinterpret_cast<float4*>(&W.poly[0][0]);
        for (int k = gl; k < pa.numVertices; k += kClipGroup) st[k] = __ldg(&vA[k]);
        for (int k = gl; k < pb.numVertices; k += kClipGroup) st[pa.numVertices + k] = __ldg(&vB[k]);
        __syncwarp(gm);
        vA = st;
        vB = st + pa.numVertices;
    }
    ff bd = mk(FLT_MAX);
    int bidx = kNone;
    ff3 bn = mk3(0.f, 0.f, 0.f);
    bool fsep = false;
    if (gl < count) {
        const int idx = W.cand[gl];
        ff3 n;
        ff d;
        bool isFace;
        if (axis_ff(c, S, vA, vB, idx, Dff, n, d, isFace)) {
            if (isFace && d.hi < 0.f) fsep = true;
            bd = d;
            bidx = idx;
            bn = n;
        }
    }
    if (__any_sync(gm, fsep)) return false;
    ff wd = bd;
    int widx = bidx;
    grp_argmin_ff(wd, widx, gm);
    if (widx == kNone) return false;
    widx = (int)__reduce_min_sync(gm, bidx != kNone && sub(bd, wd).hi <= kAxisTieTol ? (unsigned)bidx : 0xffffffffu);
    const unsigned who = __ballot_sync(gm, bidx == widx);
    const int src = __ffs(who) - 1;
    sep.x.hi = __shfl_sync(gm, bn.x.hi, src);
    sep.x.lo = __shfl_sync(gm, bn.x.lo, src);
    sep.y.hi = __shfl_sync(gm, bn.y.hi, src);
    sep.y.lo = __shfl_sync(gm, bn.y.lo, src);
    sep.z.hi = __shfl_sync(gm, bn.z.hi, src);
    sep.z.lo = __shfl_sync(gm, bn.z.lo, src);
    if (dot3(neg3(Dff), sep).hi > 0.f) sep = neg3(sep);
    return true;
}

// clip_poly_ff over the group; *over when the output exceeds kGroupPoly
__device__ __noinline__ int clip_poly_ff_g(const FfVert* in, int nin, const FfVert& plane, FfVert* out, bool* over) {
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    const ff3 pn = vget(plane);
    const ff eq = wget(plane);
    int total = 0;
    for (int base = 0; base < nin; base += kClipGroup) {
        const int ve = base + gl;
        const int sv = ve == 0 ? nin - 1 : ve - 1;
        ff3 e = mk3(0.f, 0.f, 0.f), s = e;
        ff de = mk(0.f);
        if (ve < nin) {
            e = vget(in[ve]);
            s = vget(in[sv]);
            de = add(dot3(pn, e), eq);
        }
        ff ds;
        ds.hi = __shfl_up_sync(gm, de.hi, 1, kClipGroup);
        ds.lo = __shfl_up_sync(gm, de.lo, 1, kClipGroup);
        if (ve < nin && gl == 0) ds = add(dot3(pn, s), eq);
        int cnt = 0;
        ff3 o0 = mk3(0.f, 0.f, 0.f), o1 = o0;
        if (ve < nin) {
            const bool sNeg = ds.hi < 0.f, eNeg = de.hi < 0.f;
            if (sNeg || eNeg) {
                if (sNeg && eNeg) {
                    o0 = e;
                    cnt = 1;
                } else {
                    const ff t = div(ds, sub(ds, de));
                    o0 = add3(s, scale3(sub3(e, s), t));
                    cnt = 1;
                    if (!sNeg) {
                        o1 = e;
                        cnt = 2;
                    }
                }
            }
        }
        const unsigned b1 = __ballot_sync(gm, cnt >= 1), b2 = __ballot_sync(gm, cnt == 2);
        const unsigned below = b3dev::lanemask_lt();
        const int pos = total + __popc(b1 & below) + __popc(b2 & below);
        if (cnt >= 1 && pos < kGroupPoly) out[pos] = vput(o0, mk(0.f));
        if (cnt == 2 && pos + 1 < kGroupPoly) out[pos + 1] = vput(o1, mk(0.f));
        total += __popc(b1) + __popc(b2);
    }
    __syncwarp(gm);
    if (total > kGroupPoly) *over = true;
    return min(total, kGroupPoly);
}

// clip_hull_hull over the group; *over: a face or the clipped polygon
// exceeds the group's tables (nothing decided)
__device__ __noinline__ int clip_hull_hull_g(PairCtx& c, const b3::ShapesDev& S, const NpParams& P, ff3 sep, int ai,
                                             int bi, GroupScratchFF& W, int* outBuf, bool* over) {
    const unsigned gm = grp_mask();
    ensure_ff_g(c, gm);
    const int gl = grp_lane();
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    if (ai == kNone || bi == kNone) return 0;
    const b3Face fB = S.faces[pb.faceOffset + bi];
    const b3Face fA = S.faces[pa.faceOffset + ai];
    const ff3 posA = mk3(c.posA.x, c.posA.y, c.posA.z);
    const ff3 posB = mk3(c.posB.x, c.posB.y, c.posB.z);
    int nIn = min(fB.numIndices, kMaxPoly);
    const int nvA = min(fA.numIndices, kMaxPoly);
    if (nIn > kGroupPoly || nvA > kGroupPoly) {
        *over = true;
        return 0;
    }
    for (int k = gl; k < nIn; k += kClipGroup) {
        const float4 v = __ldg(&S.verts[pb.vertexOffset + S.indices[fB.indexOffset + k]]);
        W.poly[0][k] = vput(add3(mrot(c.FB, make_float3(v.x, v.y, v.z)), posB), mk(0.f));
    }
    __syncwarp(gm);
    int cur = 0;
    const ff3 nAw = mrot(c.FA, make_float3(fA.plane[0], fA.plane[1], fA.plane[2]));
    for (int e0 = gl; e0 < nvA; e0 += kClipGroup) {
        const float4 a = __ldg(&S.verts[pa.vertexOffset + S.indices[fA.indexOffset + e0]]);
        const float4 b = __ldg(&S.verts[pa.vertexOffset + S.indices[fA.indexOffset + (e0 + 1) % fA.numIndices]]);
        const ff3 edge = sub3(mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z));
        const ff3 we{add(add(mul(c.FA.m[0][0], edge.x), mul(c.FA.m[0][1], edge.y)), mul(c.FA.m[0][2], edge.z)),
                     add(add(mul(c.FA.m[1][0], edge.x), mul(c.FA.m[1][1], edge.y)), mul(c.FA.m[1][2], edge.z)),
                     add(add(mul(c.FA.m[2][0], edge.x), mul(c.FA.m[2][1], edge.y)), mul(c.FA.m[2][2], edge.z))};
        const ff3 pn = neg3(cross3(we, nAw));
        const ff3 wa = add3(mrot(c.FA, make_float3(a.x, a.y, a.z)), posA);
        W.planes[e0] = vput(pn, neg(dot3(wa, pn)));
    }
    __syncwarp(gm);
    for (int e0 = 0; e0 < nvA && !*over; ++e0) {
        nIn = clip_poly_ff_g(W.poly[cur], nIn, W.planes[e0], W.poly[cur ^ 1], over);
        cur ^= 1;
    }
    if (*over) return 0;
    const ff eqA = sub(mk(fA.plane[3]), dot3(nAw, posA));
    const ff minD = mk(P.minDist), maxD = mk(P.maxDist);
    int total = 0;
    for (int base = 0; base < nIn; base += kClipGroup) {
        const int k = base + gl;
        bool keep = false;
        ff3 p = mk3(0.f, 0.f, 0.f);
        ff depth = mk(0.f);
        if (k < nIn) {
            p = vget(W.poly[cur][k]);
            depth = add(dot3(nAw, p), eqA);
            if (le(depth, minD)) depth = minD;
            keep = le(depth, maxD);
        }
        const unsigned m = __ballot_sync(gm, keep);
        const int pos = total + __popc(m & b3dev::lanemask_lt());
        if (keep) W.poly[cur ^ 1][pos] = vput(p, depth);
        total += __popc(m);
    }
    __syncwarp(gm);
    *outBuf = cur ^ 1;
    return total;
}

// reduce_manifold over the group
__device__ __noinline__ int4 reduce_manifold_g(const FfVert* p, int n, ff3 nearNormal) {
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    ff3 s = mk3(0.f, 0.f, 0.f);
    for (int k = 0; k < n; ++k) s = add3(s, vget(p[k]));
    const ff invn = div(mk(1.f), mk((float)n));
    const ff3 center = scale3(s, invn);
    const ff3 aV = sub3(vget(p[0]), center);
    ff3 u = cross3(nearNormal, aV);
    ff3 v = cross3(nearNormal, u);
    u = normalize3(u);
    v = normalize3(v);
    ff mw = mk(FLT_MAX), f0 = mk(FLT_MIN), f1 = mk(FLT_MIN), f2 = mk(FLT_MIN), f3v = mk(FLT_MIN);
    int iw = kNone, i0 = kNone, i1 = kNone, i2 = kNone, i3 = kNone;
    for (int k = gl; k < n; k += kClipGroup) {
        const ff w = wget(p[k]);
        if (lt(w, mw)) { mw = w; iw = k; }
        const ff3 r = sub3(vget(p[k]), center);
        const ff du = dot3(u, r), dv = dot3(v, r);
        if (lt(du, f0)) { f0 = du; i0 = k; }
        if (lt(neg(du), f1)) { f1 = neg(du); i1 = k; }
        if (lt(dv, f2)) { f2 = dv; i2 = k; }
        if (lt(neg(dv), f3v)) { f3v = neg(dv); i3 = k; }
    }
    grp_argmin_ff(mw, iw, gm);
    grp_argmin_ff(f0, i0, gm);
    grp_argmin_ff(f1, i1, gm);
    grp_argmin_ff(f2, i2, gm);
    grp_argmin_ff(f3v, i3, gm);
    int4 idx = make_int4(i0 == kNone ? 0 : i0, i1 == kNone ? 1 : i1, i2 == kNone ? 2 : i2, i3 == kNone ? 3 : i3);
    const int minIndex = iw == kNone ? -1 : iw;
    if (idx.x != minIndex && idx.y != minIndex && idx.z != minIndex && idx.w != minIndex) idx.x = minIndex;
    return idx;
}

// Stage 1b by lane groups: the sweep's near-tie entries with at most
// kClipGroup stored candidates; the others (slow-queue positions) go to
// deferQ for k_np_refine.
template <bool kSub>
__global__ void __launch_bounds__(128, 4)
k_np_refine_groups(const int2* __restrict__ pairs, const int4* __restrict__ subs, b3::BodiesDev Bd, b3::ShapesDev S,
                   float4* __restrict__ pairSep, int* __restrict__ fastQ, int* __restrict__ slowQ,
                   const int* __restrict__ cand, int* __restrict__ deferQ, uint32_t* __restrict__ manifoldFlag,
                   int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    constexpr int kPerWarp = 32 / kClipGroup;
    const int lane = threadIdx.x & 31;
    const int g = lane / kClipGroup;
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    GroupScratchFF& W = reinterpret_cast<GroupScratchFF*>(np_smem)[(threadIdx.x >> 5) * kPerWarp + g];
    const int nSlow = scalars[b3::S_NP_SLOW];  // the sweep's entries: the clip has not run
    int refined = 0;
    for (;;) {
        const int chunk = next_work(scalars + b3::S_NP_WORK4, nSlow, kPerWarp);
        if (chunk < 0) break;
        const int q = chunk + g;
        if (q < nSlow) {
            const int p = slowQ[q];
            const float4 s4 = pairSep[p];
            const int count = __float_as_int(s4.x);
            if ((int)s4.w == kSepRefine && count > 0) {
                if (count > kClipGroup) {
                    if (gl == 0) deferQ[atomicAdd(scalars + b3::S_NP_DEFER3, 1)] = q;
                } else {
                    PairCtx& c = W.ctx;
                    item_setup_group<kSub>(c, p, pairs, subs, scalars[b3::S_NUM_PAIRS], Bd, S, gm);
                    if (gl < count) W.cand[gl] = cand[(size_t)q * kMaxCand + gl];
                    __syncwarp(gm);
                    ff3 sep = mk3(0.f, 0.f, 0.f);
                    const bool haveAxis = refine_axes_g(c, S, W, count, sep);
                    ++refined;
                    if (gl == 0) {
                        slowQ[q] = -1;
                        if (haveAxis) {
                            const float3 sf = to_f3(sep);
                            pairSep[p] = make_float4(sf.x, sf.y, sf.z, (float)kSepDecided);
                            fastQ[atomicAdd(scalars + b3::S_NP_FAST, 1)] = p;
                        } else {
                            manifoldFlag[p] = 0u;
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
    if (gl == 0 && refined) atomicAdd(&counters->refinedAxes, refined);
}

// Stage 3 by lane groups: slow-queue entries whose FP32 clip was in doubt
// (the axis is the sweep's FP32 axis) get the float-float clip and
// reduction here; every other entry (slow-queue position) goes to deferQ
// for k_np_exact.
template <bool kSub>
__global__ void __launch_bounds__(128, 4)
k_np_exact_groups(const int2* __restrict__ pairs, const int4* __restrict__ subs, b3::BodiesDev Bd, b3::ShapesDev S,
                  NpParams P, const float4* __restrict__ pairSep, const int* __restrict__ slowQ,
                  int* __restrict__ deferQ, b3Contact4* __restrict__ contacts, uint32_t* __restrict__ manifoldFlag,
                  int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    constexpr int kPerWarp = 32 / kClipGroup;
    const int lane = threadIdx.x & 31;
    const int g = lane / kClipGroup;
    const int gl = grp_lane();
    const unsigned gm = grp_mask();
    GroupScratchFF& W = reinterpret_cast<GroupScratchFF*>(np_smem)[(threadIdx.x >> 5) * kPerWarp + g];
    const int nSlow = scalars[b3::S_NP_SLOW];
    int clips = 0;
    for (;;) {
        const int chunk = next_work(scalars + b3::S_NP_WORK3, nSlow, kPerWarp);
        if (chunk < 0) break;
        const int q = chunk + g;
        if (q < nSlow) {
            const int p = slowQ[q];
            if (p >= 0) {
                const float4 s4 = pairSep[p];
                bool defer = (int)s4.w != kSepClipDoubt;
                if (!defer) {
                    PairCtx& c = W.ctx;
                    item_setup_group<kSub>(c, p, pairs, subs, scalars[b3::S_NUM_PAIRS], Bd, S, gm);
                    const ff3 sep = mk3(s4.x, s4.y, s4.z);
                    const float3 sepf = to_f3(sep);
                    bool faceTie = false;
                    const int bi = select_face_g(S, c, false, sepf, -1.f, &faceTie);
                    const int ai = select_face_g(S, c, true, sepf, 1.f, &faceTie);
                    defer = faceTie;
                    if (!defer) {
                        int nOut = 0, buf = 0;
                        bool over = false, clipped = false;
                        if (ref_face_clips(S, c, ai)) {
                            nOut = clip_hull_hull_g(c, S, P, sep, ai, bi, W, &buf, &over);
                            clipped = true;
                        }
                        if (over) {
                            defer = true;
                        } else {
                            if (clipped) ++clips;
                            if (nOut > 0) {
                                const FfVert* pts = W.poly[buf];
                                const ff3 nrm = neg3(sep);
                                int4 idx = make_int4(0, 1, 2, 3);
                                int nRed = nOut;
                                if (nOut > 4) {
                                    bool tie = false;
                                    idx = reduce_f32_g(pts, nOut, to_f3(nrm), &tie);
                                    if (tie) idx = reduce_manifold_g(pts, nOut, nrm);
                                    nRed = 4;
                                }
                                emit_contact_g(p, c, pts, nRed, idx, to_f3(nrm), Bd, P, contacts, manifoldFlag);
                            } else if (gl == 0) {
                                manifoldFlag[p] = 0u;
                            }
                        }
                    }
                }
                if (defer && gl == 0) deferQ[atomicAdd(scalars + b3::S_NP_DEFER2, 1)] = q;
            }
        }
        __syncwarp();
    }
    if (gl == 0 && clips) atomicAdd(&counters->refinedClips, clips);
}

// Stage 1b, the sweep's near-minimum pairs with stored candidates: the
// float-float ranking of the candidates only. A pair with an axis then
// joins the FP32 clip queue with that axis (rounded to FP32, as the contact
// normal reports it); a pair without one is finished. Its slow-queue entry
// is cleared, so stage 3 only sees what is left. Pairs whose candidates
// did not fit the store keep their entry for stage 3's full search.
template <bool kSub>
__global__ void __launch_bounds__(128, 4)
k_np_refine(const int2* __restrict__ pairs, const int4* __restrict__ subs, b3::BodiesDev Bd, b3::ShapesDev S,
            float4* __restrict__ pairSep,
            int* __restrict__ fastQ, int* __restrict__ slowQ, const int* __restrict__ cand,
            const int* __restrict__ idxQ, int countSlot, int workSlot,
            uint32_t* __restrict__ manifoldFlag, int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    const int lane = threadIdx.x & 31;
    WarpScratch& W = reinterpret_cast<WarpScratch*>(np_smem)[threadIdx.x >> 5];
    // the sweep's entries (the clip has not run), or the slow-queue
    // positions in idxQ that the lane groups passed on
    const int nSlow = scalars[idxQ ? countSlot : b3::S_NP_SLOW];
    int refined = 0;
    for (;;) {
        const int i = next_work(scalars + workSlot, nSlow, 1);
        if (i < 0) break;
        const int q = idxQ ? idxQ[i] : i;
        const int p = slowQ[q];
        const float4 s4 = pairSep[p];
        const int count = __float_as_int(s4.x);
        if ((int)s4.w != kSepRefine || count <= 0) continue;
        PairCtx& c = W.ctx;
        item_setup_shared<kSub>(c, p, pairs, subs, scalars[b3::S_NUM_PAIRS], Bd, S);
        if (lane < count) W.cand[lane] = cand[(size_t)q * kMaxCand + lane];
        __syncwarp();
        ff3 sep = mk3(0.f, 0.f, 0.f);
        const bool haveAxis = refine_axes(c, S, W, count, sep);
        ++refined;
        if (lane == 0) {
            slowQ[q] = -1;
            if (haveAxis) {
                const float3 sf = to_f3(sep);
                pairSep[p] = make_float4(sf.x, sf.y, sf.z, (float)kSepDecided);
            } else {
                manifoldFlag[p] = 0u;
            }
        }
        if (haveAxis) push(fastQ, scalars + b3::S_NP_FAST, p);
        __syncwarp();
    }
    if (lane == 0 && refined) atomicAdd(&counters->refinedAxes, refined);
}

// Stage 3, the pairs either stage handed on: the whole chain with
// float-float refinement of the axis, the faces, the clip and the reduction.
template <bool kSub>
__global__ void __launch_bounds__(128, 4)
k_np_exact(const int2* __restrict__ pairs, const int4* __restrict__ subs, b3::BodiesDev Bd, b3::ShapesDev S,
           NpParams P,
           const float4* __restrict__ pairSep, const int* __restrict__ slowQ, const int* __restrict__ cand,
           const int* __restrict__ idxQ, int countSlot, int workSlot, b3Contact4* __restrict__ contacts,
           uint32_t* __restrict__ manifoldFlag, int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    const int lane = threadIdx.x & 31;
    WarpScratch& W = reinterpret_cast<WarpScratch*>(np_smem)[threadIdx.x >> 5];
    // every slow-queue entry, or the positions in idxQ that the lane groups
    // passed on
    const int nSlow = scalars[idxQ ? countSlot : b3::S_NP_SLOW];
    if (lane == 0) {
        W.refinedAxes = 0;
        W.refinedClips = 0;
    }
    __syncwarp();
    for (;;) {
        // one pair per grab: the queued pairs differ widely in cost
        const int chunk = next_work(scalars + workSlot, nSlow, 1);
        if (chunk < 0) break;
        const int chunkEnd = min(chunk + 1, nSlow);
        for (int i = chunk; i < chunkEnd; ++i) {
            const int q = idxQ ? idxQ[i] : i;
            const int p = slowQ[q];
            if (p < 0) continue;  // settled by the ranking stage
            PairCtx& c = W.ctx;
            item_setup_shared<kSub>(c, p, pairs, subs, scalars[b3::S_NUM_PAIRS], Bd, S);
            int nOut = 0, buf = 0;
            ff3 sep = mk3(0.f, 0.f, 0.f);
            const float4 s4 = pairSep[p];
            const int why = (int)s4.w;
            bool haveAxis;
            bool exactAxis = false;  // sep known to float-float accuracy
            if (why == kSepRefine) {
                const int count = __float_as_int(s4.x);
                if (count > 0) {
                    // the sweep's candidates: float-float ranking only
                    if (lane < count) W.cand[lane] = cand[(size_t)q * kMaxCand + lane];
                    __syncwarp();
                    if (lane == 0) ++W.refinedAxes;
                    haveAxis = refine_axes(c, S, W, count, sep);
                    exactAxis = true;
                } else {
                    haveAxis = find_axis(c, S, W, sep, &counters->clipOverflow);
                }
            } else if (why == kSepFaceTie) {
                // clip faces near-tied along the FP32 axis: the axis in float-float
                if (lane == 0) ++W.refinedAxes;
                haveAxis = find_axis(c, S, W, sep, &counters->clipOverflow, true);
                exactAxis = true;
            } else {
                // axis decided by the FP32 sweep
                sep = mk3(s4.x, s4.y, s4.z);
                haveAxis = true;
            }
            int ai = kNone, bi = kNone;
            if (haveAxis) {
                // incident face of B: max dot(nB, sep); reference face of A: min dot(nA, sep)
                bool faceTie = false;
                bi = select_face(S, c, false, to_f3(sep), sep, -1.f, &faceTie);
                ai = select_face(S, c, true, to_f3(sep), sep, 1.f, &faceTie);
                if (faceTie && !exactAxis) {
                    haveAxis = find_axis(c, S, W, sep, &counters->clipOverflow, true);
                    if (haveAxis) {
                        bi = select_face(S, c, false, to_f3(sep), sep, -1.f);
                        ai = select_face(S, c, true, to_f3(sep), sep, 1.f);
                    }
                }
            }
            if (haveAxis && ref_face_clips(S, c, ai)) {
                bool doubt = why == kSepClipDoubt || why == kSepFaceTie;
                if (!doubt) nOut = clip_f32(c, S, P, ai, bi, W, &buf, &doubt, &counters->clipOverflow);
                if (doubt) {
                    if (lane == 0) ++W.refinedClips;
                    nOut = clip_hull_hull(c, S, P, sep, ai, bi, W, &buf, &counters->clipOverflow);
                }
            }
            if (nOut > 0) {
                const FfVert* pts = W.poly[buf];
                const ff3 nrm = neg3(sep);
                int4 idx = make_int4(0, 1, 2, 3);
                int nRed = nOut;
                if (nOut > 4) {
                    bool tie = false;
                    idx = reduce_f32(pts, min(nOut, kMaxPoly), to_f3(nrm), &tie);
                    if (tie) idx = reduce_manifold(pts, nOut, nrm);
                    nRed = 4;
                }
                emit_contact(p, c, pts, nRed, idx, to_f3(nrm), Bd, P, contacts, manifoldFlag);
            } else if (lane == 0) {
                manifoldFlag[p] = 0u;
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        if (W.refinedAxes) atomicAdd(&counters->refinedAxes, W.refinedAxes);
        if (W.refinedClips) atomicAdd(&counters->refinedClips, W.refinedClips);
    }
}

// ---------------------------------------------------------------------------
// Spheres and planes (clipHullHullKernel's sphere branches,
// P2/satClipHullContacts.cl:957-1124): one manifold of one point per pair,
// decided in float-float (a body resting on a plane or a sphere sits at the
// contact threshold, where FP32 and FP64 decide apart)
// ---------------------------------------------------------------------------
__device__ void write_point_contact(b3Contact4* __restrict__ out, int slot, int A, int B, float3 pt, float depth,
                                    float3 n, const b3::BodiesDev& Bd, const NpParams& P) {
    *reinterpret_cast<float4*>(&out->worldPos[0][0]) = make_float4(pt.x, pt.y, pt.z, depth);
    for (int k = 1; k < 4; ++k) *reinterpret_cast<float4*>(&out->worldPos[k][0]) = make_float4(0.f, 0.f, 0.f, 0.f);
    *reinterpret_cast<float4*>(&out->worldNormal[0]) = make_float4(n.x, n.y, n.z, 1.f);
    out->friction = combine_friction(Bd.friction[A], Bd.friction[B], P.frictionCombine);
    out->pairIndex = slot;
    out->bodyAPtrAndSignBit = Bd.invMass[A] == 0.f ? -A : A;
    out->bodyBPtrAndSignBit = Bd.invMass[B] == 0.f ? -B : B;
}

__global__ void k_np_special(const int2* __restrict__ pairs, const int32_t* __restrict__ numPairsDev, b3::BodiesDev Bd,
                             b3::ShapesDev S, NpParams P, b3Contact4* __restrict__ contacts,
                             uint32_t* __restrict__ manifoldFlag) {
    const int np = *numPairsDev;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        const int2 pr = pairs[p];
        const int A = pr.x, B = pr.y;
        const b3Collidable cA = S.cols[Bd.collidable[A]], cB = S.cols[Bd.collidable[B]];
        const int tA = cA.shapeType, tB = cB.shapeType;
        if (!((tA == B3_SHAPE_SPHERE && (tB == B3_SHAPE_SPHERE || tB == B3_SHAPE_PLANE)) ||
              (tA == B3_SHAPE_PLANE && tB == B3_SHAPE_SPHERE)))
            continue;
        if (Bd.invMass[A] == 0.f && Bd.invMass[B] == 0.f) continue;
        const float4 pA4 = Bd.pos[A], pB4 = Bd.pos[B];
        bool hit = false;
        if (tA == B3_SHAPE_SPHERE && tB == B3_SHAPE_SPHERE) {
            // len = |posA - posB| <= rA + rB; normalOnSurfaceB = (posA - posB) / len
            const ff3 d = {two_sum(pA4.x, -pB4.x), two_sum(pA4.y, -pB4.y), two_sum(pA4.z, -pB4.z)};
            const ff rs = two_sum(cA.radius, cB.radius);
            const ff l2 = dot3(d, d);
            if (le(l2, mul(rs, rs))) {
                const ff len = sqrt_ff(l2);
                const float dist = val(sub(len, rs));
                float3 nB = make_float3(1.f, 0.f, 0.f);
                if (val(len) > 0.00001f) nB = to_f3(scale3(d, div(mk(1.f), len)));
                const float3 pt = make_float3(pB4.x, pB4.y, pB4.z) + nB * cB.radius;
                write_point_contact(&contacts[p], p, A, B, pt, dist, -nB, Bd, P);
                hit = true;
            }
        } else {
            // computeContactPlaneConvex with the plane's body on side A
            const int Pl = tA == B3_SHAPE_PLANE ? A : B, Sp = tA == B3_SHAPE_PLANE ? B : A;
            const b3Collidable cP = tA == B3_SHAPE_PLANE ? cA : cB, cS = tA == B3_SHAPE_PLANE ? cB : cA;
            const float4 pl = *reinterpret_cast<const float4*>(&S.faces[cP.shapeIndex].plane[0]);
            const float4 pP = Bd.pos[Pl], pS = Bd.pos[Sp];
            const ffmat R = quat_mat(Bd.quat[Pl]);
            const ff3 rel = {two_sum(pS.x, -pP.x), two_sum(pS.y, -pP.y), two_sum(pS.z, -pP.z)};
            const ff3 cl = mrot_t(R, rel);
            const ff dist = sub(sub(dot3(mk3(pl.x, pl.y, pl.z), cl), mk(cS.radius)), mk(pl.w));
            if (lt(dist, mk(0.f))) {
                const float3 nw = to_f3(mrot(R, make_float3(pl.x, pl.y, pl.z)));
                const float3 pt = make_float3(pS.x, pS.y, pS.z) - nw * cS.radius;
                write_point_contact(&contacts[p], p, Pl, Sp, pt, val(dist), nw, Bd, P);
                hit = true;
            }
        }
        if (hit) manifoldFlag[p] = 1u;
    }
}

// ---------------------------------------------------------------------------
// Compound and mesh pairs: sub-pairs in pair order (count, scan, write)
// ---------------------------------------------------------------------------
// A mesh triangle's local AABB against a body's world AABB (the reference
// culls so, P2/sat.cl:985-1012; inclusive)
__device__ __forceinline__ bool tri_overlaps(const float4* __restrict__ tv, float4 mn, float4 mx) {
    const float4 a = __ldg(&tv[0]), b = __ldg(&tv[1]), c = __ldg(&tv[2]);
    const float x0 = fminf(fminf(a.x, b.x), c.x), x1 = fmaxf(fmaxf(a.x, b.x), c.x);
    const float y0 = fminf(fminf(a.y, b.y), c.y), y1 = fmaxf(fmaxf(a.y, b.y), c.y);
    const float z0 = fminf(fminf(a.z, b.z), c.z), z1 = fmaxf(fmaxf(a.z, b.z), c.z);
    return !(x0 > mx.x || x1 < mn.x) && !(z0 > mx.z || z1 < mn.z) && !(y0 > mx.y || y1 < mn.y);
}

// What a pair expands into: compound x compound / hull (n child pairs), or
// mesh x hull (the mesh's triangles). kind 0 = nothing.
struct SubPlan {
    int kind;       // 1 compound, 2 mesh
    int A, B;       // manifold sides (the mesh body takes side A)
    int nA, nB;     // children per side (1 for a hull)
    int sA, sB;     // first child, or -(polytope + 1)
    int triBase;    // mesh: first triangle polytope
    int numTri, triVerts;
};

__device__ __forceinline__ SubPlan sub_plan(int2 pr, const b3::BodiesDev& Bd, const b3::ShapesDev& S) {
    SubPlan pl{};
    const int A = pr.x, B = pr.y;
    if (Bd.invMass[A] == 0.f && Bd.invMass[B] == 0.f) return pl;
    const b3Collidable cA = S.cols[Bd.collidable[A]], cB = S.cols[Bd.collidable[B]];
    const int tA = cA.shapeType, tB = cB.shapeType;
    if (tA == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS || tB == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS) {
        const bool okA = tA == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS || tA == B3_SHAPE_CONVEX_HULL;
        const bool okB = tB == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS || tB == B3_SHAPE_CONVEX_HULL;
        if (!okA || !okB) return pl;
        pl.kind = 1;
        pl.A = A;
        pl.B = B;
        pl.nA = tA == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS ? cA.numChildShapes : 1;
        pl.nB = tB == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS ? cB.numChildShapes : 1;
        pl.sA = tA == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS ? cA.shapeIndex : -(cA.shapeIndex + 1);
        pl.sB = tB == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS ? cB.shapeIndex : -(cB.shapeIndex + 1);
        return pl;
    }
    int M = -1, H = -1;
    b3Collidable cM{}, cH{};
    if (tA == B3_SHAPE_CONCAVE_TRIMESH && tB == B3_SHAPE_CONVEX_HULL) M = A, H = B, cM = cA, cH = cB;
    else if (tB == B3_SHAPE_CONCAVE_TRIMESH && tA == B3_SHAPE_CONVEX_HULL) M = B, H = A, cM = cB, cH = cA;
    if (M < 0) return pl;
    const b3ConvexPolyhedron& mesh = S.polys[cM.shapeIndex];
    pl.kind = 2;
    pl.A = M;
    pl.B = H;
    pl.numTri = mesh.numFaces;
    pl.triBase = mesh.unused;
    pl.triVerts = S.polys[mesh.unused].vertexOffset;
    pl.sB = -(cH.shapeIndex + 1);
    return pl;
}

// one warp per pair
__global__ void k_sub_count(const int2* __restrict__ pairs, const int32_t* __restrict__ numPairsDev, b3::BodiesDev Bd,
                            b3::ShapesDev S, const float4* __restrict__ aabbMin, const float4* __restrict__ aabbMax,
                            uint32_t* __restrict__ subCount) {
    const int np = *numPairsDev;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += warps) {
        const SubPlan pl = sub_plan(pairs[p], Bd, S);
        uint32_t cnt = 0;
        if (pl.kind == 1) {
            cnt = (uint32_t)(pl.nA * pl.nB);
        } else if (pl.kind == 2) {
            const float4 mn = aabbMin[pl.B], mx = aabbMax[pl.B];
            for (int base = 0; base < pl.numTri; base += 32) {
                const int f = base + lane;
                const bool ov = f < pl.numTri && tri_overlaps(S.verts + pl.triVerts + 3 * f, mn, mx);
                cnt += __popc(__ballot_sync(0xffffffffu, ov));
            }
        }
        if (lane == 0) subCount[p] = cnt;
    }
}

// the sub-pairs that fit the slots after the pairs'; the rest are counted
// as dropped pairs
__global__ void k_sub_total(int32_t* __restrict__ scalars, b3Counters* __restrict__ counters, int maxSlots) {
    const int P = scalars[b3::S_NUM_PAIRS];
    const uint32_t total = (uint32_t)scalars[b3::S_SUB_TOTAL];
    const uint32_t room = (uint32_t)max(0, maxSlots - P);
    const uint32_t n = min(total, room);
    if (total > n) atomicAdd(&counters->pairOverflow, (int)(total - n));
    scalars[b3::S_NUM_SUB] = (int32_t)n;
    scalars[b3::S_NUM_SLOTS] = P + (int32_t)n;
}

// one warp per pair, sub-pairs in order (children of A outer, of B inner;
// triangles in mesh order)
__global__ void k_sub_write(const int2* __restrict__ pairs, const int32_t* __restrict__ numPairsDev, b3::BodiesDev Bd,
                            b3::ShapesDev S, const float4* __restrict__ aabbMin, const float4* __restrict__ aabbMax,
                            const uint32_t* __restrict__ subOffset, const int32_t* __restrict__ scalars,
                            int4* __restrict__ subs) {
    const int np = *numPairsDev;
    const int n = scalars[b3::S_NUM_SUB];
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += warps) {
        const int off = (int)subOffset[p];
        if (off >= n) continue;
        const SubPlan pl = sub_plan(pairs[p], Bd, S);
        if (pl.kind == 1) {
            const int total = pl.nA * pl.nB;
            for (int k = lane; k < total && off + k < n; k += 32) {
                const int i = k / pl.nB, j = k - i * pl.nB;
                subs[off + k] = make_int4(pl.A, pl.B, pl.sA >= 0 ? pl.sA + i : pl.sA, pl.sB >= 0 ? pl.sB + j : pl.sB);
            }
        } else if (pl.kind == 2) {
            const float4 mn = aabbMin[pl.B], mx = aabbMax[pl.B];
            int run = 0;
            for (int base = 0; base < pl.numTri; base += 32) {
                const int f = base + lane;
                const bool ov = f < pl.numTri && tri_overlaps(S.verts + pl.triVerts + 3 * f, mn, mx);
                const unsigned m = __ballot_sync(0xffffffffu, ov);
                const int pos = off + run + __popc(m & b3dev::lanemask_lt());
                if (ov && pos < n) subs[pos] = make_int4(pl.A, pl.B, -(pl.triBase + f + 1), pl.sB);
                run += __popc(m);
            }
        }
    }
}

}  // namespace

namespace b3 {

// The four narrowphase stages over the pairs (kSub false) or the sub-pairs
// of compound and mesh pairs (kSub true).
template <bool kSub>
static int launch_np_stages(b3World_t* w, cudaStream_t st, const NpParams& P, bool early) {
    // work counters and queue lengths S_NP_WORK .. S_NP_WORK4, S_NP_DEFER .. S_NP_WORK7
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_NP_WORK, 0, sizeof(int32_t) * 6, st));
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_NP_DEFER, 0, sizeof(int32_t) * 6, st));
    const int threads = 32 * w->npWarpsPerBlock;
    const size_t smem = sizeof(WarpScratch) * w->npWarpsPerBlock;
    const size_t smemGroups = sizeof(GroupScratch) * (32 / kClipGroup) * w->npWarpsPerBlock;
    auto grid_of = [&](const void* k) -> int {
        int occ = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smem) != cudaSuccess || occ < 1) occ = 1;
        return w->ctx->numSMs * occ;
    };
    const b3::BodiesDev Bd = w->bodiesDev();
    const b3::ShapesDev S = w->shapesDev();
    int32_t* sc = w->d.scalars;
    const size_t smemSweep = (size_t)kSweepWarpSmem * w->npWarpsPerBlock;
    auto sweep = early ? k_np_sweep<true, kSub> : k_np_sweep<false, kSub>;
    int occS = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occS, sweep, threads, smemSweep) != cudaSuccess || occS < 1)
        occS = 1;
    // per-kernel events only in eagerly timed steps of the pairs (never inside a capture)
    const bool tk = !kSub && w->timing && w->npEv[0] != nullptr;
    if (tk) B3_CUDA(cudaEventRecord(w->npEv[0], st));
    sweep<<<w->ctx->numSMs * occS, threads, smemSweep, st>>>(
        w->d.pairs, w->d.subPairs, sc + S_NUM_PAIRS, Bd, S, w->d.manifoldFlag, w->d.pairSep, w->d.npFast,
        w->d.npSlow, w->d.npCand, std::min(w->cfg.maxPairs, kNpCandSlots), sc, w->d.counters);
    B3_CHECK_LAUNCH();
    if (tk) B3_CUDA(cudaEventRecord(w->npEv[1], st));
    const size_t smemFF = sizeof(GroupScratchFF) * (32 / kClipGroup) * w->npWarpsPerBlock;
    auto grid_ff = [&](const void* k) -> int {
        int occ = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smemFF) != cudaSuccess || occ < 1) occ = 1;
        return w->ctx->numSMs * occ;
    };
    if (w->clipGroups) {
        // lane groups for the rankings of up to 8 candidates; the rest by warps
        k_np_refine_groups<kSub><<<grid_ff((const void*)k_np_refine_groups<kSub>), threads, smemFF, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, w->d.pairSep, w->d.npFast, w->d.npSlow, w->d.npCand, w->d.npDefer3,
            w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
        k_np_refine<kSub><<<grid_of((const void*)k_np_refine<kSub>), threads, smem, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, w->d.pairSep, w->d.npFast, w->d.npSlow, w->d.npCand, w->d.npDefer3,
            S_NP_DEFER3, S_NP_WORK7, w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
    } else {
        k_np_refine<kSub><<<grid_of((const void*)k_np_refine<kSub>), threads, smem, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, w->d.pairSep, w->d.npFast, w->d.npSlow, w->d.npCand, nullptr, 0,
            S_NP_WORK4, w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
    }
    if (tk) B3_CUDA(cudaEventRecord(w->npEv[2], st));
    if (w->clipGroups) {
        // lane groups over the clip queue; what they pass on, by warps
        int occG = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occG, k_np_clip_groups<kSub>, threads, smemGroups) !=
                cudaSuccess || occG < 1)
            occG = 1;
        k_np_clip_groups<kSub><<<w->ctx->numSMs * occG, threads, smemGroups, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, P, w->d.pairSep, w->d.npFast, w->d.npSlow, w->d.npDefer,
            w->d.contacts, w->d.manifoldFlag, sc);
        B3_CHECK_LAUNCH();
        k_np_clip<kSub><<<grid_of((const void*)k_np_clip<kSub>), threads, smem, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, P, w->d.pairSep, w->d.npDefer, S_NP_DEFER, S_NP_WORK5, w->d.npSlow,
            w->d.contacts, w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
    } else {
        k_np_clip<kSub><<<grid_of((const void*)k_np_clip<kSub>), threads, smem, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, P, w->d.pairSep, w->d.npFast, S_NP_FAST, S_NP_WORK2, w->d.npSlow,
            w->d.contacts, w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
    }
    if (tk) B3_CUDA(cudaEventRecord(w->npEv[3], st));
    if (w->clipGroups) {
        // lane groups for the float-float clips of FP32 clips in doubt; the rest by warps
        k_np_exact_groups<kSub><<<grid_ff((const void*)k_np_exact_groups<kSub>), threads, smemFF, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, P, w->d.pairSep, w->d.npSlow, w->d.npDefer2, w->d.contacts,
            w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
        k_np_exact<kSub><<<grid_of((const void*)k_np_exact<kSub>), threads, smem, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, P, w->d.pairSep, w->d.npSlow, w->d.npCand, w->d.npDefer2, S_NP_DEFER2,
            S_NP_WORK6, w->d.contacts, w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
    } else {
        k_np_exact<kSub><<<grid_of((const void*)k_np_exact<kSub>), threads, smem, st>>>(
            w->d.pairs, w->d.subPairs, Bd, S, P, w->d.pairSep, w->d.npSlow, w->d.npCand, nullptr, 0, S_NP_WORK3,
            w->d.contacts, w->d.manifoldFlag, sc, w->d.counters);
        B3_CHECK_LAUNCH();
    }
    if (tk) B3_CUDA(cudaEventRecord(w->npEv[4], st));
    return B3_OK;
}

int launch_narrowphase(b3World_t* w, cudaStream_t st) {
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_NP_WORK, 0, sizeof(int32_t) * 6, st));
    if (w->cfg.maxPairs == 0 || w->bodies.empty()) return B3_OK;
    NpParams P;
    P.minDist = -1e30f;
    P.maxDist = w->sim.contactBreaking;
    P.skipDist = (float)((double)w->sim.contactProcessing - (double)w->sim.slopOffset);
    P.frictionCombine = w->sim.frictionCombine;
    P.maxPairs = w->cfg.maxPairs;
    // the early face test only where some pair can have more than 64 faces
    // (a hull may pair with another instance of itself); mesh triangles are
    // polytopes of 5 faces
    int maxFaces = 0;
    for (const b3Collidable& c : w->cols)
        if (c.shapeType == B3_SHAPE_CONVEX_HULL) maxFaces = std::max(maxFaces, w->polys[c.shapeIndex].numFaces);
    if (w->numMeshes) maxFaces = std::max(maxFaces, 5);
    const bool early = 2 * maxFaces > 64;
    const size_t smem = sizeof(WarpScratch) * w->npWarpsPerBlock;
    if (smem > 48 * 1024 && (size_t)w->npSmemAttr < smem) {
        // more than the default dynamic shared memory per block (8 warps);
        // set once per size, before any capture (the first step is eager)
        w->npSmemAttr = (int)smem;
        B3_CUDA(cudaFuncSetAttribute(k_np_clip<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        B3_CUDA(cudaFuncSetAttribute(k_np_exact<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        B3_CUDA(cudaFuncSetAttribute(k_np_refine<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        B3_CUDA(cudaFuncSetAttribute(k_np_clip<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        B3_CUDA(cudaFuncSetAttribute(k_np_exact<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        B3_CUDA(cudaFuncSetAttribute(k_np_refine<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    const size_t smemGroups = sizeof(GroupScratch) * (32 / kClipGroup) * w->npWarpsPerBlock;
    if (smemGroups > 48 * 1024 && (size_t)w->npGroupSmemAttr < smemGroups) {
        w->npGroupSmemAttr = (int)smemGroups;
        B3_CUDA(cudaFuncSetAttribute(k_np_clip_groups<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smemGroups));
        B3_CUDA(cudaFuncSetAttribute(k_np_clip_groups<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smemGroups));
    }
    const size_t smemFF = sizeof(GroupScratchFF) * (32 / kClipGroup) * w->npWarpsPerBlock;
    if (smemFF > 48 * 1024 && (size_t)w->npFFSmemAttr < smemFF) {
        w->npFFSmemAttr = (int)smemFF;
        for (const void* k : {(const void*)k_np_refine_groups<false>, (const void*)k_np_refine_groups<true>,
                              (const void*)k_np_exact_groups<false>, (const void*)k_np_exact_groups<true>})
            B3_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemFF));
    }
    {
        B3_TRY(launch_np_stages<false>(w, st, P, early));
        if (w->hasSubPairs()) {
            // expand compound and mesh pairs into sub-pairs, then their stages
            const b3::BodiesDev Bd = w->bodiesDev();
            const b3::ShapesDev S = w->shapesDev();
            const int g = w->ctx->numSMs * 4;
            k_sub_count<<<g, 256, 0, st>>>(w->d.pairs, w->d.scalars + S_NUM_PAIRS, Bd, S, w->d.aabbMin,
                                          w->d.aabbMax, w->d.subCount);
            B3_CHECK_LAUNCH();
            B3_TRY(exclusive_scan_u32(w->d.subCount, w->d.subOffset, w->d.scalars + S_NUM_PAIRS, w->cfg.maxPairs,
                                      (uint32_t*)(w->d.scalars + S_SUB_TOTAL), w->d.scanScratch,
                                      w->d.scanScratchBytes, w->d.scalars + S_ERR, st, w->ctx->numSMs));
            k_sub_total<<<1, 1, 0, st>>>(w->d.scalars, w->d.counters, w->cfg.maxPairs);
            B3_CHECK_LAUNCH();
            k_sub_write<<<g, 256, 0, st>>>(w->d.pairs, w->d.scalars + S_NUM_PAIRS, Bd, S, w->d.aabbMin, w->d.aabbMax,
                                          w->d.subOffset, w->d.scalars, w->d.subPairs);
            B3_CHECK_LAUNCH();
            B3_TRY(launch_np_stages<true>(w, st, P, early));
        }
    }
    if (w->hasSpheresPlanes()) {
        k_np_special<<<w->ctx->numSMs * 4, 256, 0, st>>>(w->d.pairs, w->d.scalars + S_NUM_PAIRS, w->bodiesDev(),
                                                          w->shapesDev(), P, w->d.contacts, w->d.manifoldFlag);
        B3_CHECK_LAUNCH();
    }
    return B3_OK;
}

}  // namespace b3
