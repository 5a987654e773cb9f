// ORACLE PIN SHIM — test infrastructure only. C entry points over the
// reference's host port of the clipping kernels
// (opencl/gpu_rigidbody_pipeline2/satClipHullContacts.cpp:406-462 clipHullAgainstHull,
// :540-697 extractManifoldSequential), compiled from the reference sources.
// The two structs below restate the host port's own layouts so this file
// can name the functions it links against.
#include "AdlMath.h"
#include "AdlQuaternion.h"
#include "LinearMath/btAlignedObjectArray.h"

struct ConvexPolyhedronCL {
    float4 m_localCenter;
    float4 m_extents;
    float4 mC;
    float4 mE;
    float m_radius;
    int m_faceOffset;
    int m_numFaces;
    int m_numVertices;
    int m_vertexOffset;
    int m_uniqueEdgesOffset;
    int m_numUniqueEdges;
    int m_unused;
};
struct btGpuFace {
    float4 m_plane;
    int m_indexOffset;
    int m_numIndices;
};

int clipHullAgainstHull(const float4& separatingNormal, const ConvexPolyhedronCL* hullA,
                        const ConvexPolyhedronCL* hullB, const float4& posA, const Quaternion& ornA,
                        const float4& posB, const Quaternion& ornB, float4* worldVertsB1, float4* worldVertsB2,
                        int capacityWorldVerts, const float minDist, float maxDist,
                        btAlignedObjectArray<float4>& vertices, btAlignedObjectArray<btGpuFace>& faces,
                        btAlignedObjectArray<int>& indices, float4* localContactsOut, int localContactCapacity);
int extractManifoldSequential(const float4* p, int nPoints, const float4& nearNormal, int4* contactIdx);

static float4 mk(const float* v) {
    float4 r;
    r.x = v[0]; r.y = v[1]; r.z = v[2]; r.w = v[3];
    return r;
}

// Hull tables in the reference layouts: polys (2), verts (xyzw), faces
// (plane[4], indexOffset, numIndices), indices. Bodies: pos (xyzw), quat.
// Returns the number of contact points (x, y, z, depth) and the reduced
// indices (contactIdx starts as 0,1,2,3 as in newContactReductionKernel).
extern "C" int ref_clip_reduce(const float* sep4, const int* polyA12, const int* polyB12, const float* polyAf16,
                               const float* polyBf16, const float* verts4, int numVerts, const float* facePlanes4,
                               const int* faceRanges2, int numFaces, const int* idx, int numIdx,
                               const float* posA4, const float* qA4, const float* posB4, const float* qB4,
                               float maxDist, float* out4, int* reduced4) {
    ConvexPolyhedronCL ha, hb;
    ha.m_localCenter = mk(polyAf16); ha.m_extents = mk(polyAf16 + 4); ha.mC = mk(polyAf16 + 8); ha.mE = mk(polyAf16 + 12);
    hb.m_localCenter = mk(polyBf16); hb.m_extents = mk(polyBf16 + 4); hb.mC = mk(polyBf16 + 8); hb.mE = mk(polyBf16 + 12);
    int* ia = &ha.m_faceOffset;
    int* ib = &hb.m_faceOffset;
    for (int k = 0; k < 7; ++k) { ia[k] = polyA12[k]; ib[k] = polyB12[k]; }
    ha.m_radius = 0; hb.m_radius = 0;
    btAlignedObjectArray<float4> V;
    for (int i = 0; i < numVerts; ++i) V.push_back(mk(verts4 + 4 * i));
    btAlignedObjectArray<btGpuFace> F;
    for (int i = 0; i < numFaces; ++i) {
        btGpuFace f;
        f.m_plane = mk(facePlanes4 + 4 * i);
        f.m_indexOffset = faceRanges2[2 * i];
        f.m_numIndices = faceRanges2[2 * i + 1];
        F.push_back(f);
    }
    btAlignedObjectArray<int> I;
    for (int i = 0; i < numIdx; ++i) I.push_back(idx[i]);
    float4 b1[64], b2[64], pts[64];
    const int n = clipHullAgainstHull(mk(sep4), &ha, &hb, mk(posA4), mk(qA4), mk(posB4), mk(qB4), b1, b2, 64,
                                      -1e30f, maxDist, V, F, I, pts, 64);
    for (int i = 0; i < n; ++i) {
        out4[4 * i] = pts[i].x; out4[4 * i + 1] = pts[i].y; out4[4 * i + 2] = pts[i].z; out4[4 * i + 3] = pts[i].w;
    }
    int4 ci;
    ci.x = 0; ci.y = 1; ci.z = 2; ci.w = 3;
    float4 nn = mk(sep4);
    nn.x = -nn.x; nn.y = -nn.y; nn.z = -nn.z;
    const int r = extractManifoldSequential(pts, n, nn, &ci);
    reduced4[0] = ci.x; reduced4[1] = ci.y; reduced4[2] = ci.z; reduced4[3] = ci.w;
    (void)r;
    return n;
}
