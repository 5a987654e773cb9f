// ORACLE PIN SHIM — test infrastructure only. C entry point over the
// reference's btConvexUtility::initializePolyhedralFeatures
// (opencl/gpu_rigidbody_pipeline/btConvexUtility.cpp:31-270) with
// btConvexHullComputer, compiled from the reference sources.
#include "btConvexUtility.h"

// Output: vertices (xyz), faces as (plane[4], numIndices) + flat indices,
// unique edges (xyz). Returns 0 or -1 if a capacity is too small.
extern "C" int ref_hull(const float* pts3, int n, float* verts3, int maxVerts, int* numVerts, float* planes4,
                        int* faceCounts, int maxFaces, int* numFaces, int* indices, int maxIndices,
                        float* edges3, int maxEdges, int* numEdges) {
    btAlignedObjectArray<btVector3> v;
    for (int i = 0; i < n; ++i) v.push_back(btVector3(pts3[3 * i], pts3[3 * i + 1], pts3[3 * i + 2]));
    btConvexUtility u;
    u.initializePolyhedralFeatures(&v[0], v.size(), true);
    if (u.m_vertices.size() > maxVerts || u.m_faces.size() > maxFaces || u.m_uniqueEdges.size() > maxEdges)
        return -1;
    *numVerts = u.m_vertices.size();
    for (int i = 0; i < u.m_vertices.size(); ++i)
        for (int k = 0; k < 3; ++k) verts3[3 * i + k] = u.m_vertices[i][k];
    *numFaces = u.m_faces.size();
    int idx = 0;
    for (int f = 0; f < u.m_faces.size(); ++f) {
        for (int k = 0; k < 4; ++k) planes4[4 * f + k] = u.m_faces[f].m_plane[k];
        faceCounts[f] = u.m_faces[f].m_indices.size();
        for (int j = 0; j < u.m_faces[f].m_indices.size(); ++j) {
            if (idx >= maxIndices) return -1;
            indices[idx++] = u.m_faces[f].m_indices[j];
        }
    }
    *numEdges = u.m_uniqueEdges.size();
    for (int i = 0; i < u.m_uniqueEdges.size(); ++i)
        for (int k = 0; k < 3; ++k) edges3[3 * i + k] = u.m_uniqueEdges[i][k];
    return 0;
}
