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

#include <cfloat>

using namespace b3m;

namespace {

constexpr int kMaxPoly = 64;  // capacityWorldVerts (satClipHullContacts.cl:1027)
constexpr int kChunk = 4;     // pairs per work grab

struct NpParams {
    float minDist;
    float maxDist;
    int frictionCombine;
    int maxPairs;
};

struct __align__(16) WarpScratch {
    float4 poly[2][kMaxPoly];
};

__device__ __forceinline__ float combine_friction(float a, float b, int mode) {
    return mode == B3_FRICTION_PRODUCT ? a * b : sqrtf(a * b);
}

// project hull (local verts) onto world axis dir
__device__ __forceinline__ void project(const float4* __restrict__ verts, int off, int nv,
                                        const Mat3& R, float3 pos, float3 dir, float& mn, float& mx) {
    const float3 ld = mul_t(R, dir);
    const float offs = dot(pos, dir);
    float lo = FLT_MAX, hi = -FLT_MAX;
    for (int i = 0; i < nv; ++i) {
        const float4 v = __ldg(&verts[off + i]);
        const float dp = v.x * ld.x + v.y * ld.y + v.z * ld.z;
        lo = fminf(lo, dp);
        hi = fmaxf(hi, dp);
    }
    mn = lo + offs;
    mx = hi + offs;
}

// lexicographic (value, index) minimum across the warp
__device__ __forceinline__ void warp_argmin(float& v, int& idx) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov < v || (ov == v && (unsigned)oi < (unsigned)idx)) {
            v = ov;
            idx = oi;
        }
    }
}

struct PairCtx {
    int A, B;
    float invMassA, invMassB;
    const b3ConvexPolyhedron* pa;
    const b3ConvexPolyhedron* pb;
    Mat3 RA, RB;
    float3 posA, posB;
};

// Find the minimum-penetration axis. Returns false if separated / no axis.
__device__ bool find_axis(const PairCtx& c, const b3::ShapesDev& S, float3& sep) {
    const int lane = threadIdx.x & 31;
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    const float4 lcA = make_float4(pa.localCenter[0], pa.localCenter[1], pa.localCenter[2], 0.f);
    const float4 lcB = make_float4(pb.localCenter[0], pb.localCenter[1], pb.localCenter[2], 0.f);
    const float3 c0 = mul(c.RA, f3(lcA)) + c.posA;
    const float3 c1 = mul(c.RB, f3(lcB)) + c.posB;
    const float3 D = c0 - c1;
    float best = FLT_MAX;
    int bestIdx = 0x7fffffff;
    float3 bestAxis = make_float3(0.f, 0.f, 0.f);
    bool separated = false;
    // faces of A
    for (int f = lane; f < pa.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[pa.faceOffset + f].plane[0]);
        float3 n = mul(c.RA, make_float3(pl.x, pl.y, pl.z));
        if (dot(D, n) < 0.f) n = -n;
        float mn0, mx0, mn1, mx1;
        project(S.verts, pa.vertexOffset, pa.numVertices, c.RA, c.posA, n, mn0, mx0);
        project(S.verts, pb.vertexOffset, pb.numVertices, c.RB, c.posB, n, mn1, mx1);
        if (mx0 < mn1 || mx1 < mn0) separated = true;
        const float d = fminf(mx0 - mn1, mx1 - mn0);
        if (d < best) {
            best = d;
            bestIdx = f;
            bestAxis = n;
        }
    }
    if (__any_sync(0xffffffffu, separated)) return false;
    // faces of B (findSeparatingAxis(hullB, hullA, ...), same DeltaC2)
    for (int f = lane; f < pb.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[pb.faceOffset + f].plane[0]);
        float3 n = mul(c.RB, make_float3(pl.x, pl.y, pl.z));
        if (dot(D, n) < 0.f) n = -n;
        float mn0, mx0, mn1, mx1;
        project(S.verts, pb.vertexOffset, pb.numVertices, c.RB, c.posB, n, mn0, mx0);
        project(S.verts, pa.vertexOffset, pa.numVertices, c.RA, c.posA, n, mn1, mx1);
        if (mx0 < mn1 || mx1 < mn0) separated = true;
        const float d = fminf(mx0 - mn1, mx1 - mn0);
        if (d < best) {
            best = d;
            bestIdx = pa.numFaces + f;
            bestAxis = n;
        }
    }
    if (__any_sync(0xffffffffu, separated)) return false;
    // edge x edge
    const int EA = pa.numUniqueEdges, EB = pb.numUniqueEdges;
    const int base = pa.numFaces + pb.numFaces;
    for (int e = lane; e < EA * EB; e += 32) {
        const int e0 = e / EB, e1 = e - e0 * EB;
        const float4 ea = __ldg(&S.edges[pa.uniqueEdgesOffset + e0]);
        const float4 eb = __ldg(&S.edges[pb.uniqueEdgesOffset + e1]);
        const float3 wa = mul(c.RA, f3(ea));
        const float3 wb = mul(c.RB, f3(eb));
        float3 cr = cross(wa, wb);
        if (fabsf(cr.x) > 1e-6f || fabsf(cr.y) > 1e-6f || fabsf(cr.z) > 1e-6f) {
            cr = normalize(cr);
            if (dot(D, cr) < 0.f) cr = -cr;
            float mn0, mx0, mn1, mx1;
            project(S.verts, pa.vertexOffset, pa.numVertices, c.RA, c.posA, cr, mn0, mx0);
            project(S.verts, pb.vertexOffset, pb.numVertices, c.RB, c.posB, cr, mn1, mx1);
            const float d = fminf(mx0 - mn1, mx1 - mn0);
            if (d < best) {
                best = d;
                bestIdx = base + e;
                bestAxis = cr;
            }
        }
    }
    float bv = best;
    int bi = bestIdx;
    warp_argmin(bv, bi);
    if (bi == 0x7fffffff) return false;
    const unsigned who = __ballot_sync(0xffffffffu, bestIdx == bi && best == bv);
    const int src = __ffs(who) - 1;
    sep.x = __shfl_sync(0xffffffffu, bestAxis.x, src);
    sep.y = __shfl_sync(0xffffffffu, bestAxis.y, src);
    sep.z = __shfl_sync(0xffffffffu, bestAxis.z, src);
    if (dot(-D, sep) > 0.f) sep = -sep;
    return true;
}

// One Sutherland-Hodgman step: keep the part behind plane (n, eq).
// Warp-parallel, output order identical to the sequential loop.
__device__ int clip_poly(const float4* in, int nin, float3 pn, float eq, float4* out, int* ovf) {
    const int lane = threadIdx.x & 31;
    int total = 0;
    for (int base = 0; base < nin; base += 32) {
        const int ve = base + lane;
        int cnt = 0;
        float4 o0 = make_float4(0, 0, 0, 0), o1 = make_float4(0, 0, 0, 0);
        if (ve < nin) {
            const float4 s = in[ve == 0 ? nin - 1 : ve - 1];
            const float4 e = in[ve];
            const float ds = pn.x * s.x + pn.y * s.y + pn.z * s.z + eq;
            const float de = pn.x * e.x + pn.y * e.y + pn.z * e.z + eq;
            if (ds < 0.f) {
                if (de < 0.f) {
                    o0 = e;
                    cnt = 1;
                } else {
                    const float t = ds * 1.f / (ds - de);
                    o0 = make_float4(s.x + (e.x - s.x) * t, s.y + (e.y - s.y) * t, s.z + (e.z - s.z) * t, 0.f);
                    cnt = 1;
                }
            } else if (de < 0.f) {
                const float t = ds * 1.f / (ds - de);
                o0 = make_float4(s.x + (e.x - s.x) * t, s.y + (e.y - s.y) * t, s.z + (e.z - s.z) * t, 0.f);
                o1 = e;
                cnt = 2;
            }
        }
        // exclusive prefix of cnt across lanes
        int x = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const int pos = total + x - cnt;
        if (cnt >= 1) {
            if (pos < kMaxPoly) out[pos] = o0; else atomicAdd(ovf, 1);
        }
        if (cnt == 2) {
            if (pos + 1 < kMaxPoly) out[pos + 1] = o1; else atomicAdd(ovf, 1);
        }
        total += __shfl_sync(0xffffffffu, x, 31);
    }
    __syncwarp();
    return min(total, kMaxPoly);
}

// clipHullAgainstHull: returns the number of kept points, stored with
// w = depth in W.poly[*outBuf].
__device__ int clip_hull_hull(const PairCtx& c, const b3::ShapesDev& S, const NpParams& P,
                              float3 sep, WarpScratch& W, int* outBuf, int* ovf) {
    const int lane = threadIdx.x & 31;
    const b3ConvexPolyhedron& pa = *c.pa;
    const b3ConvexPolyhedron& pb = *c.pb;
    // incident face of B: max dot(nB, sep), first wins
    float bv = FLT_MAX;
    int bi = 0x7fffffff;
    for (int f = lane; f < pb.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[pb.faceOffset + f].plane[0]);
        const float d = -dot(mul(c.RB, make_float3(pl.x, pl.y, pl.z)), sep);
        if (d < bv) { bv = d; bi = f; }
    }
    warp_argmin(bv, bi);
    // reference face of A: min dot(nA, sep), first wins
    float av = FLT_MAX;
    int ai = 0x7fffffff;
    for (int f = lane; f < pa.numFaces; f += 32) {
        const float4 pl = __ldg((const float4*)&S.faces[pa.faceOffset + f].plane[0]);
        const float d = dot(mul(c.RA, make_float3(pl.x, pl.y, pl.z)), sep);
        if (d < av) { av = d; ai = f; }
    }
    warp_argmin(av, ai);
    if (ai == 0x7fffffff || bi == 0x7fffffff) return 0;
    const b3Face fB = S.faces[pb.faceOffset + bi];
    const b3Face fA = S.faces[pa.faceOffset + ai];
    int nIn = min(fB.numIndices, kMaxPoly);
    for (int k = lane; k < nIn; k += 32) {
        const float4 v = __ldg(&S.verts[pb.vertexOffset + S.indices[fB.indexOffset + k]]);
        W.poly[0][k] = f4(mul(c.RB, f3(v)) + c.posB);
    }
    __syncwarp();
    int cur = 0;
    const float3 nAw = mul(c.RA, make_float3(fA.plane[0], fA.plane[1], fA.plane[2]));
    const int nvA = fA.numIndices;
    for (int e0 = 0; e0 < nvA; ++e0) {
        const float4 a = __ldg(&S.verts[pa.vertexOffset + S.indices[fA.indexOffset + e0]]);
        const float4 b = __ldg(&S.verts[pa.vertexOffset + S.indices[fA.indexOffset + (e0 + 1) % nvA]]);
        const float3 we = mul(c.RA, make_float3(a.x - b.x, a.y - b.y, a.z - b.z));
        const float3 pn = -cross(we, nAw);
        const float3 wa = mul(c.RA, f3(a)) + c.posA;
        const float eq = -dot(wa, pn);
        nIn = clip_poly(W.poly[cur], nIn, pn, eq, W.poly[cur ^ 1], ovf);
        cur ^= 1;
    }
    // keep points behind the witness face (clipFaceAgainstHull :433-452)
    const float eqA = fA.plane[3] - dot(nAw, c.posA);
    int total = 0;
    for (int base = 0; base < nIn; base += 32) {
        const int k = base + lane;
        bool keep = false;
        float4 pt = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k < nIn) {
            pt = W.poly[cur][k];
            float depth = dot(nAw, f3(pt)) + eqA;
            if (depth <= P.minDist) depth = P.minDist;
            if (depth <= P.maxDist) {
                keep = true;
                pt.w = depth;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        const int pos = total + __popc(m & b3dev::lanemask_lt());
        if (keep) W.poly[cur ^ 1][pos] = pt;
        total += __popc(m);
    }
    __syncwarp();
    *outBuf = cur ^ 1;
    return total;
}

// extractManifoldSequentialGlobal (P2/satClipHullContacts.cl:678-770) over
// n > 4 points in p; returns the 4 chosen indices.
__device__ int4 reduce_manifold(const float4* p, int n, float3 nearNormal) {
    const int lane = threadIdx.x & 31;
    // centre (float4 incl. w)
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = lane; k < n; k += 32) {
        const float4 q = p[k];
        s.x += q.x; s.y += q.y; s.z += q.z; s.w += q.w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
        s.z += __shfl_xor_sync(0xffffffffu, s.z, o);
        s.w += __shfl_xor_sync(0xffffffffu, s.w, o);
    }
    const float inv = 1.f / (float)n;
    const float3 center = make_float3(s.x * inv, s.y * inv, s.z * inv);
    const float3 aV = f3(p[0]) - center;
    float3 u = cross(nearNormal, aV);
    float3 v = cross(nearNormal, u);
    u = normalize(u);
    v = normalize(v);
    float mw = FLT_MAX, f0 = FLT_MIN, f1 = FLT_MIN, f2 = FLT_MIN, f3v = FLT_MIN;
    int iw = -1, i0 = 0x7fffffff, i1 = 0x7fffffff, i2 = 0x7fffffff, i3 = 0x7fffffff;
    for (int k = lane; k < n; k += 32) {
        const float4 q = p[k];
        if (q.w < mw) { mw = q.w; iw = k; }
        const float3 r = f3(q) - center;
        const float du = dot(u, r), dv = dot(v, r);
        if (du < f0) { f0 = du; i0 = k; }
        if (-du < f1) { f1 = -du; i1 = k; }
        if (dv < f2) { f2 = dv; i2 = k; }
        if (-dv < f3v) { f3v = -dv; i3 = k; }
    }
    if (iw < 0) iw = 0x7fffffff;
    warp_argmin(mw, iw);
    warp_argmin(f0, i0);
    warp_argmin(f1, i1);
    warp_argmin(f2, i2);
    warp_argmin(f3v, i3);
    int4 idx = make_int4(i0 == 0x7fffffff ? 0 : i0, i1 == 0x7fffffff ? 1 : i1,
                         i2 == 0x7fffffff ? 2 : i2, i3 == 0x7fffffff ? 3 : i3);
    const int minIndex = (iw == 0x7fffffff) ? -1 : iw;
    if (idx.x != minIndex && idx.y != minIndex && idx.z != minIndex && idx.w != minIndex)
        idx.x = minIndex;
    return idx;
}

__global__ void __launch_bounds__(128)
k_narrowphase(const int2* __restrict__ pairs, const int32_t* __restrict__ numPairsDev,
              b3::BodiesDev Bd, b3::ShapesDev S, NpParams P, b3Contact4* __restrict__ contacts,
              uint32_t* __restrict__ manifoldFlag, int32_t* __restrict__ workCounter,
              b3Counters* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char np_smem[];
    const int lane = threadIdx.x & 31;
    WarpScratch& W = reinterpret_cast<WarpScratch*>(np_smem)[threadIdx.x >> 5];
    const int numPairs = *numPairsDev;
    for (;;) {
        int chunk = 0;
        if (lane == 0) chunk = atomicAdd(workCounter, kChunk);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
        if (chunk >= numPairs) break;
        const int chunkEnd = min(chunk + kChunk, numPairs);
        for (int p = chunk; p < chunkEnd; ++p) {
            const int2 pr = pairs[p];
            PairCtx c;
            c.A = pr.x;
            c.B = pr.y;
            c.invMassA = Bd.invMass[c.A];
            c.invMassB = Bd.invMass[c.B];
            const b3Collidable colA = S.cols[Bd.collidable[c.A]];
            const b3Collidable colB = S.cols[Bd.collidable[c.B]];
            int nOut = 0, buf = 0;
            float3 sep = make_float3(0.f, 0.f, 0.f);
            if (!(c.invMassA == 0.f && c.invMassB == 0.f) &&
                colA.shapeType == B3_SHAPE_CONVEX_HULL && colB.shapeType == B3_SHAPE_CONVEX_HULL) {
                c.pa = &S.polys[colA.shapeIndex];
                c.pb = &S.polys[colB.shapeIndex];
                c.RA = quat_to_mat(Bd.quat[c.A]);
                c.RB = quat_to_mat(Bd.quat[c.B]);
                c.posA = f3(Bd.pos[c.A]);
                c.posB = f3(Bd.pos[c.B]);
                if (find_axis(c, S, sep))
                    nOut = clip_hull_hull(c, S, P, sep, W, &buf, &counters->clipOverflow);
            }
            if (nOut > 0) {
                const float4* pts = W.poly[buf];
                const float3 nrm = -sep;
                int4 idx = make_int4(0, 1, 2, 3);
                int nRed = nOut;
                if (nOut > 4) {
                    idx = reduce_manifold(pts, nOut, nrm);
                    nRed = 4;
                }
                b3Contact4* out = &contacts[p];
                if (lane < nRed) {
                    const int k = lane == 0 ? idx.x : lane == 1 ? idx.y : lane == 2 ? idx.z : idx.w;
                    const float4 q = pts[k];
                    *reinterpret_cast<float4*>(&out->worldPos[lane][0]) = q;
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
            } else if (lane == 0) {
                manifoldFlag[p] = 0u;
            }
            __syncwarp();
        }
    }
}

}  // namespace

namespace b3 {

int launch_narrowphase(b3World_t* w, cudaStream_t st) {
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_NP_WORK, 0, sizeof(int32_t), st));
    if (w->cfg.maxPairs == 0 || w->bodies.empty()) return B3_OK;
    NpParams P;
    P.minDist = -1e30f;
    P.maxDist = w->sim.contactBreaking;
    P.frictionCombine = w->sim.frictionCombine;
    P.maxPairs = w->cfg.maxPairs;
    const int threads = 32 * w->npWarpsPerBlock;
    const size_t smem = sizeof(WarpScratch) * w->npWarpsPerBlock;
    int occ = 1;
    B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_narrowphase, threads, smem));
    occ = occ < 1 ? 1 : occ;
    const int grid = w->ctx->numSMs * occ;
    k_narrowphase<<<grid, threads, smem, st>>>(w->d.pairs, w->d.scalars + S_NUM_PAIRS,
                                              w->bodiesDev(), w->shapesDev(), P, w->d.contacts,
                                              w->d.manifoldFlag, w->d.scalars + S_NP_WORK,
                                              w->d.counters);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

}  // namespace b3
