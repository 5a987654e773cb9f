// World object (rigid-body and collidable arrays, grid broadphase,
// narrowphase-and-solver) and stepSimulation orchestration.
//
// Mirrors CLPhysicsDemo (P2/CLPhysicsDemo.h:30-81, .cpp:205-943) and
// btGpuNarrowphaseAndSolver (P1/btGpuNarrowPhaseAndSolver.h:63-123) behind
// the C ABI in include/b3gpu.h. One step issues, on one stream and with no
// host synchronisation (so it can be captured as a CUDA graph):
//   k_step_begin -> k_aabb_hash -> radix sort -> k_cell_start -> k_find_pairs
//   -> k_narrowphase -> scan + k_manifold_emit -> radix sort -> k_body_ranges
//   -> k_setup_rows -> k_jacobi (persistent) -> k_integrate
// Every count that varies per step (pairs, manifolds, copies) stays on the
// device and is read by the next kernel; the reference instead blocks on
// clFinish more than 15 times and reads 3 counts back per step.
#include "b3_world.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>

namespace {

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }
int ilog2(uint64_t v) {
    int b = 0;
    while ((1ull << b) < v) ++b;
    return b;
}

__global__ void k_step_begin(int32_t* scalars, b3Counters* counters) {
    if (threadIdx.x == 0) {
        scalars[b3::S_STAMP] += 1;
        counters->steps += 1;
        counters->numContactPoints = 0;
        counters->numManifolds = 0;
        counters->numPairs = 0;
        counters->refinedAxes = 0;
        counters->refinedClips = 0;
        counters->pairOverflow = 0;
        counters->cellOverflow = 0;
        counters->clipOverflow = 0;
    }
}

__global__ void k_world_stats(b3::BodiesDev Bd, float4* out, int numWorlds) {
    // one warp-strided accumulation per body into its world (atomics; stats only)
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Bd.n) return;
    const float im = Bd.invMass[i];
    if (im == 0.f) return;
    const float m = 1.f / im;
    const float4 p = Bd.pos[i], v = Bd.linVel[i];
    const int w = Bd.worldId[i];
    atomicAdd(&out[2 * w].x, m * p.x);
    atomicAdd(&out[2 * w].y, m * p.y);
    atomicAdd(&out[2 * w].z, m * p.z);
    atomicAdd(&out[2 * w].w, m);
    atomicAdd(&out[2 * w + 1].x, 0.5f * m * (v.x * v.x + v.y * v.y + v.z * v.z));
}

template <typename T>
int dalloc(T*& p, size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) count = 1;
    B3_CUDA(cudaMalloc((void**)&p, sizeof(T) * count));
    return B3_OK;
}

void free_all(b3::DevBuffers& d) {
    void* ptrs[] = {d.pos, d.quat, d.linVel, d.angVel, d.invMass, d.friction, d.restitution,
                    d.invInertia, d.collidable, d.worldId, d.cols, d.polys, d.verts, d.faces,
                    d.indices, d.edges, d.localAabb, d.polyInradius, d.childShapes, d.vpXY, d.vpZ, d.polyPack, d.subPairs, d.subCount, d.subOffset, d.aabbMin, d.aabbMax, d.smallSlot,
                    d.largeStart, d.largeList, d.sapSmall, d.sapLarge, d.sapSorted, d.sapCount, d.sapOffset, d.keys, d.vals, d.keysAlt, d.valsAlt, d.cellTable,
                    d.pairs, d.contacts, d.manifoldFlag, d.pairSep, d.npFast, d.npSlow, d.npDefer, d.npDefer2, d.npDefer3, d.npCand, d.manifoldScan,
                    d.manifoldPair,
                    d.incKeys, d.incVals, d.incKeysAlt, d.incValsAlt, d.bodyIncStart,
                    d.bodyIncEnd, d.rows, d.manifoldHdr, d.incLin, d.incAng, d.avgLin, d.avgAng,
                    d.scalars, d.counters, d.sortScratch, d.incSortScratch, d.scanScratch,
                    d.worldStats, d.worldMStart, d.worldMEnd, d.gsCell, d.gsSlotBatch,
                    d.gsSlotOfManifold, d.gsMinRank, d.gsTaken, d.gsBatchCount, d.gsGroupCount, d.gsGroupFill,
                    d.gsGroupOffset, d.gsInertia};  // gsConstraints shares the row storage
    for (void* p : ptrs)
        if (p) cudaFree(p);
    d = b3::DevBuffers();
}

// btTransformAabb (LinearMath/btAabbUtil2.h) with margin, in double: the
// registration AABB used for the large-body test and the inertia.
void transform_aabb(const float lmin[3], const float lmax[3], float margin, const float pos[3],
                    const float q[4], float outMin[3], float outMax[3]) {
    double he[3], c[3];
    for (int k = 0; k < 3; ++k) {
        he[k] = 0.5 * ((double)lmax[k] - lmin[k]) + margin;
        c[k] = 0.5 * ((double)lmax[k] + lmin[k]);
    }
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double d = x * x + y * y + z * z + w * w;
    const double s = 2.0 / d;
    const double xs = x * s, ys = y * s, zs = z * s;
    const double wx = w * xs, wy = w * ys, wz = w * zs;
    const double xx = x * xs, xy = x * ys, xz = x * zs;
    const double yy = y * ys, yz = y * zs, zz = z * zs;
    const double Rm[3][3] = {{1.0 - (yy + zz), xy - wz, xz + wy},
                             {xy + wz, 1.0 - (xx + zz), yz - wx},
                             {xz - wy, yz + wx, 1.0 - (xx + yy)}};
    for (int r = 0; r < 3; ++r) {
        double cc = Rm[r][0] * c[0] + Rm[r][1] * c[1] + Rm[r][2] * c[2] + pos[r];
        double e = std::fabs(Rm[r][0]) * he[0] + std::fabs(Rm[r][1]) * he[1] + std::fabs(Rm[r][2]) * he[2];
        outMin[r] = (float)(cc - e);
        outMax[r] = (float)(cc + e);
    }
}

}  // namespace

b3::BodiesDev b3World_t::bodiesDev() const {
    b3::BodiesDev B;
    B.n = (int)bodies.size();
    B.pos = d.pos;
    B.quat = d.quat;
    B.linVel = d.linVel;
    B.angVel = d.angVel;
    B.invMass = d.invMass;
    B.collidable = d.collidable;
    B.friction = d.friction;
    B.restitution = d.restitution;
    B.invInertia = d.invInertia;
    B.worldId = d.worldId;
    return B;
}

b3::ShapesDev b3World_t::shapesDev() const {
    b3::ShapesDev S;
    S.cols = d.cols;
    S.polys = d.polys;
    S.verts = d.verts;
    S.faces = d.faces;
    S.indices = d.indices;
    S.edges = d.edges;
    S.localAabb = d.localAabb;
    S.inradius = d.polyInradius;
    S.children = d.childShapes;
    S.vpXY = d.vpXY;
    S.vpZ = d.vpZ;
    S.polyPack = d.polyPack;
    S.numPolys = (int)polys.size();
    S.numVerts = (int)verts4.size() / 4;
    S.numFaces = (int)faces.size();
    S.numIndices = (int)indices.size();
    S.numEdges = (int)edges4.size() / 4;
    return S;
}

extern "C" void b3_world_config_default(b3WorldConfig* c) {
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->maxBodies = 128 * 1024;
    c->maxPairs = 0;               // 0 = 8 x maxBodies
    c->numWorlds = 1;
    c->cellSize = 4.f;             // P2/CLPhysicsDemo.cpp:636 uses 4 m cells
    c->gridDims[0] = c->gridDims[1] = c->gridDims[2] = 128;
    c->maxBodiesPerCell = 128;
    c->maxPairsPerBody = 32;
    c->maxSmallProxySize = 100.f;
    c->gravity[0] = 0.f;
    c->gravity[1] = -9.8f;
    c->gravity[2] = 0.f;
    c->dt = 1.f / 60.f;
    c->solverIterations = 10;
    c->erp = 0.2f;
    c->contactBreaking = 0.02f;
    c->contactProcessing = 0.02f;
    c->linearSlopOffset = 0.01f;
    c->angularDamping = 0.99f;
    c->frictionCombine = B3_FRICTION_GEOMEAN;
    c->useGraph = 0;
}

extern "C" int b3_world_create(b3Context ctx, const b3WorldConfig* cfg, b3World* out) {
    if (!ctx || !cfg || !out) return B3_ERR_INVALID_ARG;
    *out = nullptr;
    const b3WorldConfig& c = *cfg;
    for (int k = 0; k < 3; ++k)
        if (!is_pow2(c.gridDims[k]) || c.gridDims[k] < 4) {
            b3_set_error("gridDims must be powers of two >= 4");
            return B3_ERR_INVALID_ARG;
        }
    if (c.maxBodies <= 0 || c.numWorlds <= 0 || c.cellSize <= 0.f || c.maxBodiesPerCell <= 0 ||
        c.maxPairsPerBody < 2 || c.maxPairsPerBody > 256 || c.dt <= 0.f || c.solverIterations < 0) {
        b3_set_error("invalid world configuration");
        return B3_ERR_INVALID_ARG;
    }
    const int cellBits = ilog2((uint64_t)c.gridDims[0] * c.gridDims[1] * c.gridDims[2]);
    const int worldBits = c.numWorlds > 1 ? ilog2((uint64_t)c.numWorlds) : 0;
    if (cellBits + worldBits > 32) {
        b3_set_error("world id + cell hash need %d > 32 key bits", cellBits + worldBits);
        return B3_ERR_INVALID_ARG;
    }
    if ((c.flags & ~(B3_WORLD_SAP_BROADPHASE | B3_WORLD_BATCHED_GS_SOLVER)) != 0 ||
        ((c.flags & B3_WORLD_SAP_BROADPHASE) && c.numWorlds != 1)) {
        b3_set_error("invalid world flags (the SAP broadphase takes one world)");
        return B3_ERR_INVALID_ARG;
    }
    b3World w = new b3World_t();
    w->ctx = ctx;
    w->cfg = c;
    w->sap = (c.flags & B3_WORLD_SAP_BROADPHASE) != 0;
    w->gs = (c.flags & B3_WORLD_BATCHED_GS_SOLVER) != 0;
    if (w->cfg.maxPairs <= 0) w->cfg.maxPairs = 8 * c.maxBodies;
    w->cellBits = cellBits;
    w->worldBits = worldBits;
    w->keyBits = w->sap ? 32 : std::max(1, cellBits + worldBits);
    w->invCell = 1.f / c.cellSize;
    w->sim.gravity = make_float3(c.gravity[0], c.gravity[1], c.gravity[2]);
    w->sim.dt = c.dt;
    w->sim.iterations = c.solverIterations;
    w->sim.erp = c.erp;
    w->sim.contactBreaking = c.contactBreaking;
    w->sim.contactProcessing = c.contactProcessing;
    w->sim.slopOffset = c.linearSlopOffset;
    w->sim.angularDamping = c.angularDamping;
    w->sim.frictionCombine = c.frictionCombine;
    *out = w;
    return B3_OK;
}

extern "C" int b3_world_destroy(b3World w) {
    if (!w) return B3_OK;
    if (w->ctx->device < 0) {
        delete w;
        return B3_OK;
    }
    cudaSetDevice(w->ctx->device);
    if (w->graphExec) cudaGraphExecDestroy(w->graphExec);
    if (w->graphStream) cudaStreamDestroy(w->graphStream);
    free_all(w->d);
    delete w;
    return B3_OK;
}

extern "C" int b3_register_convex_hull(b3World w, const float* vertices, int numVertices, int strideBytes,
                                       const float scaling[3], int* collidableOut) {
    if (!w || !vertices || numVertices < 4 || !collidableOut) return B3_ERR_INVALID_ARG;
    if (strideBytes <= 0) strideBytes = 3 * sizeof(float);
    std::vector<float> pts(3 * (size_t)numVertices);
    const unsigned char* base = (const unsigned char*)vertices;
    for (int i = 0; i < numVertices; ++i) {
        const float* v = (const float*)(base + (size_t)i * strideBytes);
        for (int k = 0; k < 3; ++k) pts[3 * i + k] = v[k] * (scaling ? scaling[k] : 1.f);
    }
    b3hull::Polyhedron P;
    std::string err;
    if (!b3hull::compute_polyhedron(pts.data(), numVertices, P, &err)) {
        b3_set_error("hull: %s", err.c_str());
        return B3_ERR_INVALID_ARG;
    }
    b3ConvexPolyhedron poly;
    memset(&poly, 0, sizeof(poly));
    for (int k = 0; k < 3; ++k) {
        poly.localCenter[k] = P.localCenter[k];
        poly.mC[k] = P.mC[k];
        poly.mE[k] = P.mE[k];
        poly.extents[k] = 0.5f * P.mE[k];
    }
    float r = 1e30f;
    for (auto& f : P.faces)
        r = std::min(r, std::fabs(f.plane[0] * P.localCenter[0] + f.plane[1] * P.localCenter[1] +
                                  f.plane[2] * P.localCenter[2] + f.plane[3]));
    poly.radius = r;
    // rounded down to float: a lower bound stays a lower bound
    float rin = (float)P.inradius;
    if ((double)rin > P.inradius) rin = std::nextafter(rin, 0.f);
    w->polyInradius.push_back(rin);
    poly.numVertices = (int)P.vertices.size() / 3;
    poly.vertexOffset = (int)w->verts4.size() / 4;
    for (int i = 0; i < poly.numVertices; ++i) {
        w->verts4.push_back(P.vertices[3 * i]);
        w->verts4.push_back(P.vertices[3 * i + 1]);
        w->verts4.push_back(P.vertices[3 * i + 2]);
        w->verts4.push_back(0.f);
    }
    poly.numFaces = (int)P.faces.size();
    poly.faceOffset = (int)w->faces.size();
    for (auto& f : P.faces) {
        b3Face ff;
        memset(&ff, 0, sizeof(ff));
        for (int k = 0; k < 4; ++k) ff.plane[k] = f.plane[k];
        ff.indexOffset = (int)w->indices.size();
        ff.numIndices = (int)f.indices.size();
        // pad[0] = 1 when every vertex lies on the stored plane (within
        // FP32 rounding); a welded face of near-coplanar triangles does not
        double off = 0.0, mag = 1.0;
        for (int id : f.indices) {
            const double x = P.vertices[3 * id], y = P.vertices[3 * id + 1], z = P.vertices[3 * id + 2];
            off = std::max(off, std::fabs(x * ff.plane[0] + y * ff.plane[1] + z * ff.plane[2] + ff.plane[3]));
            mag = std::max(mag, std::fabs(x) + std::fabs(y) + std::fabs(z));
        }
        ff.pad[0] = off <= 1e-6 * mag ? 1 : 0;
        for (int id : f.indices) w->indices.push_back(id);
        w->faces.push_back(ff);
    }
    poly.numUniqueEdges = (int)P.uniqueEdges.size() / 3;
    poly.uniqueEdgesOffset = (int)w->edges4.size() / 4;
    for (int i = 0; i < poly.numUniqueEdges; ++i) {
        w->edges4.push_back(P.uniqueEdges[3 * i]);
        w->edges4.push_back(P.uniqueEdges[3 * i + 1]);
        w->edges4.push_back(P.uniqueEdges[3 * i + 2]);
        w->edges4.push_back(1.f);  // w: the edge's length (unit edges)
    }
    b3Collidable col;
    col.numChildShapes = 0;
    col.radius = 0.f;
    col.shapeType = B3_SHAPE_CONVEX_HULL;
    col.shapeIndex = (int)w->polys.size();
    w->polys.push_back(poly);
    w->cols.push_back(col);
    for (int k = 0; k < 3; ++k) w->localAabb8.push_back(P.aabbMin[k]);
    w->localAabb8.push_back(0.f);
    for (int k = 0; k < 3; ++k) w->localAabb8.push_back(P.aabbMax[k]);
    w->localAabb8.push_back(0.f);
    w->shapesDirty = true;
    *collidableOut = (int)w->cols.size() - 1;
    return B3_OK;
}

// Appends a collidable with its local AABB; returns its index.
static int add_collidable(b3World w, int type, int shapeIndex, float radius, int numChildren, const float mn[3],
                          const float mx[3]) {
    b3Collidable col;
    col.numChildShapes = numChildren;
    col.radius = radius;
    col.shapeType = type;
    col.shapeIndex = shapeIndex;
    w->cols.push_back(col);
    for (int k = 0; k < 3; ++k) w->localAabb8.push_back(mn[k]);
    w->localAabb8.push_back(0.f);
    for (int k = 0; k < 3; ++k) w->localAabb8.push_back(mx[k]);
    w->localAabb8.push_back(0.f);
    w->shapesDirty = true;
    return (int)w->cols.size() - 1;
}

extern "C" int b3_register_sphere(b3World w, float radius, int* collidableOut) {
    if (!w || !collidableOut || !(radius > 0.f)) return B3_ERR_INVALID_ARG;
    const float mn[3] = {-radius, -radius, -radius}, mx[3] = {radius, radius, radius};
    // registerSphereShape: shapeIndex 0, the radius in the collidable
    *collidableOut = add_collidable(w, B3_SHAPE_SPHERE, 0, radius, 0, mn, mx);
    ++w->numSpheres;
    return B3_OK;
}

extern "C" int b3_register_plane(b3World w, const float normal[3], float planeConstant, int* collidableOut) {
    if (!w || !normal || !collidableOut) return B3_ERR_INVALID_ARG;
    // registerFace: the plane as one face of the shared face table
    b3Face f;
    memset(&f, 0, sizeof(f));
    for (int k = 0; k < 3; ++k) f.plane[k] = normal[k];
    f.plane[3] = planeConstant;
    const int face = (int)w->faces.size();
    w->faces.push_back(f);
    const float mn[3] = {-1e30f, -1e30f, -1e30f}, mx[3] = {1e30f, 1e30f, 1e30f};
    *collidableOut = add_collidable(w, B3_SHAPE_PLANE, face, planeConstant, 0, mn, mx);
    ++w->numPlanes;
    return B3_OK;
}

extern "C" int b3_register_compound(b3World w, const b3ChildShape* children, int numChildren, int* collidableOut) {
    if (!w || !children || numChildren <= 0 || !collidableOut) return B3_ERR_INVALID_ARG;
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < numChildren; ++i) {
        const int c = children[i].shapeIndex;
        if (c < 0 || c >= (int)w->cols.size() || w->cols[c].shapeType != B3_SHAPE_CONVEX_HULL) {
            b3_set_error("compound child %d: collidable %d is not a convex hull", i, c);
            return B3_ERR_INVALID_ARG;
        }
    }
    // the union of the children's local AABBs at their poses (btTransformAabb, margin 0)
    for (int i = 0; i < numChildren; ++i) {
        const float* la = &w->localAabb8[8 * (size_t)children[i].shapeIndex];
        float a[3], b[3];
        transform_aabb(la, la + 4, 0.f, children[i].childPosition, children[i].childOrientation, a, b);
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], a[k]);
            mx[k] = std::max(mx[k], b[k]);
        }
    }
    const int first = (int)w->childShapes.size();
    for (int i = 0; i < numChildren; ++i) w->childShapes.push_back(children[i]);
    *collidableOut = add_collidable(w, B3_SHAPE_COMPOUND_OF_CONVEX_HULLS, first, 0.f, numChildren, mn, mx);
    ++w->numCompounds;
    return B3_OK;
}

// float helpers in btVector3's operation order (the mesh's face planes)
static inline void fcross3(const float a[3], const float b[3], float r[3]) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline float fdot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void fnormalize3(float a[3]) {
    const float r = 1.f / std::sqrt(fdot3(a, a));
    for (int k = 0; k < 3; ++k) a[k] *= r;
}

extern "C" int b3_register_concave_mesh(b3World w, const float* vertices3, int numVertices, const int* indices,
                                        int numIndices, const float scaling[3], int* collidableOut) {
    if (!w || !vertices3 || numVertices < 3 || !indices || numIndices < 3 || numIndices % 3 != 0 || !collidableOut)
        return B3_ERR_INVALID_ARG;
    for (int i = 0; i < numIndices; ++i)
        if (indices[i] < 0 || indices[i] >= numVertices) {
            b3_set_error("mesh index %d out of range", i);
            return B3_ERR_INVALID_ARG;
        }
    const int numTri = numIndices / 3;
    std::vector<float> v(3 * (size_t)numVertices);
    for (int i = 0; i < numVertices; ++i)
        for (int k = 0; k < 3; ++k) v[3 * i + k] = vertices3[3 * i + k] * (scaling ? scaling[k] : 1.f);
    auto V = [&](int i) { return &v[3 * (size_t)i]; };
    // the mesh's own table entry (registerConcaveMeshShape): its vertices,
    // one face per triangle with the reference's plane, no unique edges
    b3ConvexPolyhedron mesh;
    memset(&mesh, 0, sizeof(mesh));
    mesh.numVertices = numVertices;
    mesh.vertexOffset = (int)w->verts4.size() / 4;
    for (int i = 0; i < numVertices; ++i) {
        for (int k = 0; k < 3; ++k) w->verts4.push_back(V(i)[k]);
        w->verts4.push_back(0.f);
    }
    mesh.faceOffset = (int)w->faces.size();
    mesh.numFaces = numTri;
    mesh.uniqueEdgesOffset = (int)w->edges4.size() / 4;
    mesh.numUniqueEdges = 0;
    std::vector<std::array<float, 4>> triPlane(numTri);
    for (int t = 0; t < numTri; ++t) {
        const float* a = V(indices[3 * t]);
        const float* b = V(indices[3 * t + 1]);
        const float* c = V(indices[3 * t + 2]);
        const float e0[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const float e1[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        float n[3];
        fcross3(e0, e1, n);
        if (!(fdot3(n, n) > 0.f)) {
            b3_set_error("mesh triangle %d is degenerate", t);
            return B3_ERR_INVALID_ARG;
        }
        fnormalize3(n);
        triPlane[t] = {n[0], n[1], n[2], -fdot3(n, a)};
        b3Face f;
        memset(&f, 0, sizeof(f));
        for (int k = 0; k < 4; ++k) f.plane[k] = triPlane[t][k];
        f.indexOffset = (int)w->indices.size();
        f.numIndices = 3;
        f.pad[0] = 1;
        for (int k = 0; k < 3; ++k) w->indices.push_back(indices[3 * t + k]);
        w->faces.push_back(f);
    }
    const int meshPoly = (int)w->polys.size();
    mesh.unused = meshPoly + 1;  // the first triangle polytope
    w->polys.push_back(mesh);
    w->polyInradius.push_back(0.f);
    // one polytope per triangle, as findSeparatingAxisKernel builds it
    // (P2/sat.cl:970-1100): vertices 0, 1, 2; faces front (the triangle's
    // plane; indices 0 1 2), back (-n, n . v0; 2 1 0), and for i = 0, 1, 2
    // the edge plane of vertices i and i-1 (normalize(n x (v[i-1] - v[i])),
    // -e . v[i]; indices i, i-1); unique edges v1-v0, v2-v1, v0-v2 as they
    // are (not normalised); local centre (v0 + v1 + v2) / 3
    for (int t = 0; t < numTri; ++t) {
        const float* tv[3] = {V(indices[3 * t]), V(indices[3 * t + 1]), V(indices[3 * t + 2])};
        const float n[3] = {triPlane[t][0], triPlane[t][1], triPlane[t][2]};
        b3ConvexPolyhedron tp;
        memset(&tp, 0, sizeof(tp));
        tp.numVertices = 3;
        tp.vertexOffset = (int)w->verts4.size() / 4;
        float lc[3] = {0.f, 0.f, 0.f}, mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
        for (int i = 0; i < 3; ++i) {
            for (int k = 0; k < 3; ++k) {
                w->verts4.push_back(tv[i][k]);
                lc[k] += tv[i][k];
                mn[k] = std::min(mn[k], tv[i][k]);
                mx[k] = std::max(mx[k], tv[i][k]);
            }
            w->verts4.push_back(0.f);
        }
        for (int k = 0; k < 3; ++k) {
            tp.localCenter[k] = lc[k] * (1.f / 3.f);
            tp.mC[k] = mx[k] + mn[k];
            tp.mE[k] = mx[k] - mn[k];
            tp.extents[k] = 0.5f * tp.mE[k];
        }
        tp.faceOffset = (int)w->faces.size();
        tp.numFaces = 5;
        auto add_face = [&](const float pl[4], std::initializer_list<int> ids) {
            b3Face f;
            memset(&f, 0, sizeof(f));
            for (int k = 0; k < 4; ++k) f.plane[k] = pl[k];
            f.indexOffset = (int)w->indices.size();
            f.numIndices = (int)ids.size();
            f.pad[0] = 1;
            for (int id : ids) w->indices.push_back(id);
            w->faces.push_back(f);
        };
        const float front[4] = {n[0], n[1], n[2], triPlane[t][3]};
        add_face(front, {0, 1, 2});
        const float back[4] = {-n[0], -n[1], -n[2], fdot3(n, tv[0])};
        add_face(back, {2, 1, 0});
        int prev = 2;
        for (int i = 0; i < 3; ++i) {
            const float d[3] = {tv[prev][0] - tv[i][0], tv[prev][1] - tv[i][1], tv[prev][2] - tv[i][2]};
            float e[3];
            fcross3(n, d, e);
            fnormalize3(e);
            const float pl[4] = {e[0], e[1], e[2], -fdot3(e, tv[i])};
            add_face(pl, {i, prev});
            prev = i;
        }
        tp.uniqueEdgesOffset = (int)w->edges4.size() / 4;
        tp.numUniqueEdges = 3;
        for (int i = 0; i < 3; ++i) {
            const float* a = tv[i];
            const float* b = tv[(i + 1) % 3];
            float e[3];
            for (int k = 0; k < 3; ++k) e[k] = b[k] - a[k];
            for (int k = 0; k < 3; ++k) w->edges4.push_back(e[k]);
            // w: the edge's length, rounded up (scales the sweep's error bound)
            w->edges4.push_back(std::nextafter((float)std::sqrt((double)e[0] * e[0] + (double)e[1] * e[1] +
                                                                (double)e[2] * e[2]), 1e30f));
        }
        tp.radius = 0.f;
        w->polys.push_back(tp);
        w->polyInradius.push_back(0.f);
    }
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < numVertices; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], V(i)[k]);
            mx[k] = std::max(mx[k], V(i)[k]);
        }
    *collidableOut = add_collidable(w, B3_SHAPE_CONCAVE_TRIMESH, meshPoly, 0.f, numTri, mn, mx);
    ++w->numMeshes;
    return B3_OK;
}

extern "C" int b3_get_child_shapes(b3World w, b3ChildShape* out, int max, int* count) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    *count = (int)w->childShapes.size();
    if (out) memcpy(out, w->childShapes.data(), sizeof(b3ChildShape) * std::min(max, *count));
    return B3_OK;
}

extern "C" int b3_register_body(b3World w, float mass, const float position[3], const float orientation[4],
                                int collidable, float friction, float restitution, int worldId, int* bodyOut) {
    if (!w || !position || !orientation || !bodyOut) return B3_ERR_INVALID_ARG;
    if (collidable < 0 || collidable >= (int)w->cols.size()) return B3_ERR_INVALID_ARG;
    if (worldId < 0 || worldId >= w->cfg.numWorlds) return B3_ERR_INVALID_ARG;
    if ((int)w->bodies.size() >= w->cfg.maxBodies) {
        b3_set_error("maxBodies (%d) reached", w->cfg.maxBodies);
        return B3_ERR_CAPACITY;
    }
    b3Body b;
    memset(&b, 0, sizeof(b));
    for (int k = 0; k < 3; ++k) b.pos[k] = position[k];
    for (int k = 0; k < 4; ++k) b.quat[k] = orientation[k];
    b.collidableIdx = (uint32_t)collidable;
    b.invMass = mass != 0.f ? 1.f / mass : 0.f;
    b.friction = friction;
    b.restitution = restitution;
    // registration AABB with 0.01 margin (P2/CLPhysicsDemo.cpp:538-548)
    float amin[3], amax[3];
    const float* la = &w->localAabb8[8 * (size_t)collidable];
    transform_aabb(la, la + 4, 0.01f, position, orientation, amin, amax);
    b3Inertia I;
    memset(&I, 0, sizeof(I));
    if (mass != 0.f) {
        // registerRigidBody (P1/btGpuNarrowPhaseAndSolver.cpp:610-641): full
        // extents, doubled, as the inertia box
        const float hx = amax[0] - amin[0], hy = amax[1] - amin[1], hz = amax[2] - amin[2];
        const float lx = 2.f * hx, ly = 2.f * hy, lz = 2.f * hz;
        const float ix = (mass / 12.0f) * (ly * ly + lz * lz);
        const float iy = (mass / 12.0f) * (lx * lx + lz * lz);
        const float iz = (mass / 12.0f) * (lx * lx + ly * ly);
        I.initInvInertia[0] = 1.f / ix;
        I.initInvInertia[5] = 1.f / iy;
        I.initInvInertia[10] = 1.f / iz;
        memcpy(I.invInertiaWorld, I.initInvInertia, sizeof(I.initInvInertia));
    }
    w->bodies.push_back(b);
    w->inertias.push_back(I);
    w->worldIds.push_back(worldId);
    for (int k = 0; k < 3; ++k) w->regAabb.push_back(amin[k]);
    for (int k = 0; k < 3; ++k) w->regAabb.push_back(amax[k]);
    w->written = false;
    *bodyOut = (int)w->bodies.size() - 1;
    return B3_OK;
}

extern "C" int b3_register_bodies(b3World w, int n, const float* masses, const float* positions3,
                                  const float* orientations4, const int* collidables, const float* frictions,
                                  const float* restitutions, const int* worldIds, int* firstBodyOut) {
    if (!w || n < 0 || (n > 0 && (!masses || !positions3 || !orientations4 || !collidables)))
        return B3_ERR_INVALID_ARG;
    if ((int64_t)w->bodies.size() + n > w->cfg.maxBodies) {
        b3_set_error("maxBodies (%d) reached", w->cfg.maxBodies);
        return B3_ERR_CAPACITY;
    }
    if (firstBodyOut) *firstBodyOut = (int)w->bodies.size();
    for (int i = 0; i < n; ++i) {
        int id = 0;
        B3_TRY(b3_register_body(w, masses[i], positions3 + 3 * (size_t)i, orientations4 + 4 * (size_t)i,
                                collidables[i], frictions ? frictions[i] : 1.f,
                                restitutions ? restitutions[i] : 0.f, worldIds ? worldIds[i] : 0, &id));
    }
    return B3_OK;
}

static int ensure_capacity(b3World w) {
    const int N = (int)w->bodies.size();
    const int cap = w->cfg.maxPairs;
    auto& d = w->d;
    if (!d.cellTable) {
        const size_t cells = (size_t)w->cfg.numWorlds << w->cellBits;
        B3_TRY(dalloc(d.cellTable, cells));
        B3_TRY(dalloc(d.scalars, b3::S_NUM_SCALARS));
        B3_TRY(dalloc(d.counters, 1));
        B3_CUDA(cudaMemset(d.cellTable, 0, sizeof(uint2) * cells));
        B3_CUDA(cudaMemset(d.scalars, 0, sizeof(int32_t) * b3::S_NUM_SCALARS));
        B3_CUDA(cudaMemset(d.counters, 0, sizeof(b3Counters)));
    }
    if (w->capBodies < N || !d.pos) {
        const int nb = std::max(N, 1);
        B3_TRY(dalloc(d.pos, nb));
        B3_TRY(dalloc(d.quat, nb));
        B3_TRY(dalloc(d.linVel, nb));
        B3_TRY(dalloc(d.angVel, nb));
        B3_TRY(dalloc(d.invMass, nb));
        B3_TRY(dalloc(d.friction, nb));
        B3_TRY(dalloc(d.restitution, nb));
        B3_TRY(dalloc(d.invInertia, nb));
        B3_TRY(dalloc(d.collidable, nb));
        B3_TRY(dalloc(d.worldId, nb));
        B3_TRY(dalloc(d.aabbMin, nb));
        B3_TRY(dalloc(d.aabbMax, nb));
        B3_TRY(dalloc(d.smallSlot, nb));
        if (w->sap) {
            B3_TRY(dalloc(d.sapSmall, nb));
            B3_TRY(dalloc(d.sapLarge, nb));
            B3_TRY(dalloc(d.sapSorted, 2 * (size_t)nb));
            B3_TRY(dalloc(d.sapCount, (size_t)nb + 1));
            B3_TRY(dalloc(d.sapOffset, (size_t)nb + 1));
        }
        B3_TRY(dalloc(d.keys, nb));
        B3_TRY(dalloc(d.vals, nb));
        B3_TRY(dalloc(d.keysAlt, nb));
        B3_TRY(dalloc(d.valsAlt, nb));
        B3_TRY(dalloc(d.bodyIncStart, nb));
        B3_TRY(dalloc(d.bodyIncEnd, nb));
        B3_TRY(dalloc(d.avgLin, nb));
        B3_TRY(dalloc(d.avgAng, nb));
        if (w->gs) {
            B3_TRY(dalloc(d.gsMinRank, 4 * (size_t)nb));
            B3_TRY(dalloc(d.gsTaken, 4 * (size_t)nb));
            B3_TRY(dalloc(d.gsInertia, 3 * (size_t)nb));
        }
        d.sortScratchBytes = b3::radix_scratch_bytes(nb, w->keyBits);
        B3_TRY(dalloc((unsigned char*&)d.sortScratch, d.sortScratchBytes));
        w->capBodies = nb;
    }
    if (!d.pairs) {
        const size_t c = std::max(cap, 1);
        B3_TRY(dalloc(d.pairs, c));
        B3_TRY(dalloc(d.contacts, c));
        B3_TRY(dalloc(d.manifoldFlag, c));
        B3_TRY(dalloc(d.pairSep, c));
        B3_TRY(dalloc(d.npFast, c));
        B3_TRY(dalloc(d.npSlow, c));
        B3_TRY(dalloc(d.npDefer, c));
        B3_TRY(dalloc(d.npDefer2, c));
        B3_TRY(dalloc(d.npDefer3, c));
        B3_TRY(dalloc(d.npCand, (size_t)std::min<size_t>(c, b3::kNpCandSlots) * 32));
        B3_TRY(dalloc(d.manifoldScan, c));
        B3_TRY(dalloc(d.manifoldPair, c));
        B3_TRY(dalloc(d.incKeys, 2 * c));
        B3_TRY(dalloc(d.incVals, 2 * c));
        B3_TRY(dalloc(d.incKeysAlt, 2 * c));
        B3_TRY(dalloc(d.incValsAlt, 2 * c));
        B3_TRY(dalloc(d.rows, 40 * c));
        B3_TRY(dalloc(d.incLin, 4 * c));  // [2 phase buffers][2 sides][capacity]
        B3_TRY(dalloc(d.incAng, 4 * c));
        if (w->gs) {
            static_assert(sizeof(b3Constraint4) <= 40 * sizeof(float4), "Constraint4 fits a manifold's rows");
            d.gsConstraints = reinterpret_cast<b3Constraint4*>(d.rows);
            B3_TRY(dalloc(d.gsCell, c));
            B3_TRY(dalloc(d.gsSlotBatch, c));
            B3_TRY(dalloc(d.gsSlotOfManifold, c));
            B3_TRY(dalloc(d.gsBatchCount, 16));
            B3_TRY(dalloc(d.gsGroupCount, 4 * (size_t)b3::kGsMaxBatch));
            B3_TRY(dalloc(d.gsGroupFill, 4 * (size_t)b3::kGsMaxBatch));
            B3_TRY(dalloc(d.gsGroupOffset, 4 * (size_t)b3::kGsMaxBatch + 1));
        }
        const size_t tiles = (w->cfg.maxBodies + 31) / 32 + 16;  // pair-search tiles, 32 bodies at the least
        d.scanScratchBytes = std::max(b3::scan_scratch_bytes(std::max<int64_t>(cap, w->cfg.maxBodies + 1)),
                                      tiles * 8 + 256);
        B3_TRY(dalloc((unsigned char*&)d.scanScratch, d.scanScratchBytes));
    }
    // body-id key bits for the copy sort must cover the sentinel numBodies
    w->bodyBits = std::max(1, ilog2((uint64_t)N + 1));
    const size_t incBytes = std::max(b3::radix_scratch_bytes(2LL * cap, w->bodyBits),
                                     w->gs ? b3::radix_scratch_bytes(cap, 10) : (size_t)0);
    if (incBytes > d.incSortScratchBytes) {
        d.incSortScratchBytes = incBytes;
        B3_TRY(dalloc((unsigned char*&)d.incSortScratch, incBytes));
    }
    if (w->hasSubPairs() && !d.subPairs) {
        const size_t c = std::max(cap, 1);
        B3_TRY(dalloc(d.subPairs, c));
        B3_TRY(dalloc(d.subCount, c));
        B3_TRY(dalloc(d.subOffset, c));
    }
    if (!d.worldStats) B3_TRY(dalloc(d.worldStats, 2 * (size_t)w->cfg.numWorlds));
    if (!d.worldMStart) {
        B3_TRY(dalloc(d.worldMStart, (size_t)w->cfg.numWorlds));
        B3_TRY(dalloc(d.worldMEnd, (size_t)w->cfg.numWorlds));
    }
    return B3_OK;
}

static int upload_shapes(b3World w, cudaStream_t st) {
    auto& d = w->d;
    B3_TRY(dalloc(d.cols, w->cols.size()));
    B3_TRY(dalloc(d.polys, w->polys.size()));
    B3_TRY(dalloc(d.verts, w->verts4.size() / 4));
    B3_TRY(dalloc(d.faces, w->faces.size()));
    B3_TRY(dalloc(d.indices, w->indices.size()));
    B3_TRY(dalloc(d.edges, w->edges4.size() / 4 + 1));
    B3_TRY(dalloc(d.localAabb, w->localAabb8.size() / 4));
    B3_TRY(dalloc(d.polyInradius, w->polyInradius.size()));
    B3_CUDA(cudaMemcpyAsync(d.cols, w->cols.data(), sizeof(b3Collidable) * w->cols.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.polys, w->polys.data(), sizeof(b3ConvexPolyhedron) * w->polys.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.verts, w->verts4.data(), sizeof(float) * w->verts4.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.faces, w->faces.data(), sizeof(b3Face) * w->faces.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.indices, w->indices.data(), sizeof(int) * w->indices.size(), cudaMemcpyHostToDevice, st));
    if (!w->edges4.empty())
        B3_CUDA(cudaMemcpyAsync(d.edges, w->edges4.data(), sizeof(float) * w->edges4.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.localAabb, w->localAabb8.data(), sizeof(float) * w->localAabb8.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.polyInradius, w->polyInradius.data(), sizeof(float) * w->polyInradius.size(),
                            cudaMemcpyHostToDevice, st));
    // vertex pairs per polyhedron (the packed projection's layout)
    w->vpXY.clear();
    w->vpZ.clear();
    w->polyPack.assign(w->polys.size(), 0);
    for (size_t p = 0; p < w->polys.size(); ++p) {
        const b3ConvexPolyhedron& h = w->polys[p];
        w->polyPack[p] = (int)(w->vpZ.size() / 2);
        for (int j = 0; j < h.numVertices; j += 2) {
            const float* a = &w->verts4[4 * (size_t)(h.vertexOffset + j)];
            const float* b = &w->verts4[4 * (size_t)(h.vertexOffset + std::min(j + 1, h.numVertices - 1))];
            w->vpXY.insert(w->vpXY.end(), {a[0], b[0], a[1], b[1]});
            w->vpZ.insert(w->vpZ.end(), {a[2], b[2]});
        }
    }
    B3_TRY(dalloc(d.vpXY, w->vpXY.size() / 4 + 1));
    B3_TRY(dalloc(d.vpZ, w->vpZ.size() / 2 + 1));
    B3_TRY(dalloc(d.polyPack, w->polyPack.size() + 1));
    if (!w->vpXY.empty()) {
        B3_CUDA(cudaMemcpyAsync(d.vpXY, w->vpXY.data(), sizeof(float) * w->vpXY.size(), cudaMemcpyHostToDevice, st));
        B3_CUDA(cudaMemcpyAsync(d.vpZ, w->vpZ.data(), sizeof(float) * w->vpZ.size(), cudaMemcpyHostToDevice, st));
    }
    if (!w->polyPack.empty())
        B3_CUDA(cudaMemcpyAsync(d.polyPack, w->polyPack.data(), sizeof(int) * w->polyPack.size(),
                                cudaMemcpyHostToDevice, st));
    B3_TRY(dalloc(d.childShapes, w->childShapes.size()));
    if (!w->childShapes.empty())
        B3_CUDA(cudaMemcpyAsync(d.childShapes, w->childShapes.data(), sizeof(b3ChildShape) * w->childShapes.size(),
                                cudaMemcpyHostToDevice, st));
    w->shapesDirty = false;
    return B3_OK;
}

extern "C" int b3_write_bodies(b3World w, void* stream) {
    if (!w) return B3_ERR_INVALID_ARG;
    if (w->cols.empty()) return B3_ERR_STATE;
    if (w->ctx->device < 0) {
        b3_set_error("host-only context");
        return B3_ERR_NO_DEVICE;
    }
    cudaStream_t st = as_stream(stream);
    B3_CUDA(cudaSetDevice(w->ctx->device));
    B3_TRY(ensure_capacity(w));
    B3_TRY(upload_shapes(w, st));
    const int N = (int)w->bodies.size();
    std::vector<float4> pos(N), quat(N), lv(N), av(N), ii(N);
    std::vector<float> im(N), fr(N), rs(N);
    std::vector<int> col(N);
    for (int i = 0; i < N; ++i) {
        const b3Body& b = w->bodies[i];
        pos[i] = make_float4(b.pos[0], b.pos[1], b.pos[2], 0.f);
        quat[i] = make_float4(b.quat[0], b.quat[1], b.quat[2], b.quat[3]);
        lv[i] = make_float4(b.linVel[0], b.linVel[1], b.linVel[2], 0.f);
        av[i] = make_float4(b.angVel[0], b.angVel[1], b.angVel[2], 0.f);
        im[i] = b.invMass;
        fr[i] = b.friction;
        rs[i] = b.restitution;
        col[i] = (int)b.collidableIdx;
        const b3Inertia& I = w->inertias[i];
        ii[i] = make_float4(I.initInvInertia[0], I.initInvInertia[5], I.initInvInertia[10], 0.f);
    }
    // small / large classification (btGpu3DGridBroadphase::isLargeProxy,
    // G3/btGpu3DGridBroadphase.cpp:385-391): half-diagonal > maxSmallProxySize/2
    w->smallSlotHost.assign(N, -1);
    std::vector<std::vector<int>> large(w->cfg.numWorlds);
    int ns = 0;
    for (int i = 0; i < N; ++i) {
        const float* a = &w->regAabb[6 * (size_t)i];
        const double dx = a[3] - a[0], dy = a[4] - a[1], dz = a[5] - a[2];
        const double r = 0.5 * std::sqrt(dx * dx + dy * dy + dz * dz);
        if (r > 0.5 * w->cfg.maxSmallProxySize) large[w->worldIds[i]].push_back(i);
        else w->smallSlotHost[i] = ns++;
    }
    if (w->sap) {
        // sweep and prune: dynamic bodies are the sorted small proxies,
        // static ones the large proxies (P2/CLPhysicsDemo.cpp:558-568); no
        // grid hashing
        w->smallSlotHost.assign(N, -1);
        for (auto& l : large) l.clear();
        w->sapSmallHost.clear();
        w->sapLargeHost.clear();
        for (int i = 0; i < N; ++i) (w->bodies[i].invMass != 0.f ? w->sapSmallHost : w->sapLargeHost).push_back(i);
        ns = (int)w->sapSmallHost.size();
    }
    w->numSmall = ns;
    w->largeStartHost.assign(w->cfg.numWorlds + 1, 0);
    w->largeListHost.clear();
    for (int k = 0; k < w->cfg.numWorlds; ++k) {
        w->largeStartHost[k] = (int)w->largeListHost.size();
        for (int id : large[k]) w->largeListHost.push_back(id);
    }
    w->largeStartHost[w->cfg.numWorlds] = (int)w->largeListHost.size();
    auto& d = w->d;
    B3_TRY(dalloc(d.largeStart, w->largeStartHost.size()));
    B3_TRY(dalloc(d.largeList, std::max<size_t>(1, w->largeListHost.size())));
    B3_CUDA(cudaMemcpyAsync(d.largeStart, w->largeStartHost.data(), sizeof(int) * w->largeStartHost.size(), cudaMemcpyHostToDevice, st));
    if (!w->largeListHost.empty())
        B3_CUDA(cudaMemcpyAsync(d.largeList, w->largeListHost.data(), sizeof(int) * w->largeListHost.size(), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.smallSlot, w->smallSlotHost.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    if (w->sap) {
        if (!w->sapSmallHost.empty())
            B3_CUDA(cudaMemcpyAsync(d.sapSmall, w->sapSmallHost.data(), sizeof(int) * w->sapSmallHost.size(),
                                    cudaMemcpyHostToDevice, st));
        if (!w->sapLargeHost.empty())
            B3_CUDA(cudaMemcpyAsync(d.sapLarge, w->sapLargeHost.data(), sizeof(int) * w->sapLargeHost.size(),
                                    cudaMemcpyHostToDevice, st));
    }
    B3_CUDA(cudaMemcpyAsync(d.pos, pos.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.quat, quat.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.linVel, lv.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.angVel, av.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.invMass, im.data(), sizeof(float) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.friction, fr.data(), sizeof(float) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.restitution, rs.data(), sizeof(float) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.invInertia, ii.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.collidable, col.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemcpyAsync(d.worldId, w->worldIds.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemsetAsync(d.avgLin, 0, sizeof(float4) * N, st));
    B3_CUDA(cudaMemsetAsync(d.avgAng, 0, sizeof(float4) * N, st));
    B3_CUDA(cudaMemsetAsync(d.bodyIncStart, 0, sizeof(uint32_t) * N, st));
    B3_CUDA(cudaMemsetAsync(d.bodyIncEnd, 0, sizeof(uint32_t) * N, st));
    const int32_t hs[1] = {ns};
    B3_CUDA(cudaMemcpyAsync(d.scalars + b3::S_NUM_SMALL, hs, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    B3_CUDA(cudaMemsetAsync(d.counters, 0, sizeof(b3Counters), st));
    B3_CUDA(cudaStreamSynchronize(st));
    if (w->graphExec) {
        cudaGraphExecDestroy(w->graphExec);
        w->graphExec = nullptr;
    }
    w->graphValid = false;
    w->written = true;
    return B3_OK;
}

extern "C" int b3_write_velocities(b3World w, const float* linVel3, const float* angVel3, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    const int N = (int)w->bodies.size();
    cudaStream_t st = as_stream(stream);
    std::vector<float4> t(N);
    if (linVel3) {
        for (int i = 0; i < N; ++i) t[i] = make_float4(linVel3[3 * i], linVel3[3 * i + 1], linVel3[3 * i + 2], 0.f);
        B3_CUDA(cudaMemcpyAsync(w->d.linVel, t.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
        B3_CUDA(cudaStreamSynchronize(st));
    }
    if (angVel3) {
        for (int i = 0; i < N; ++i) t[i] = make_float4(angVel3[3 * i], angVel3[3 * i + 1], angVel3[3 * i + 2], 0.f);
        B3_CUDA(cudaMemcpyAsync(w->d.angVel, t.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
        B3_CUDA(cudaStreamSynchronize(st));
    }
    return B3_OK;
}

// ---------------------------------------------------------------------------
// Step orchestration
// ---------------------------------------------------------------------------
static int step_begin(b3World w, cudaStream_t st) {
    k_step_begin<<<1, 32, 0, st>>>(w->d.scalars, w->d.counters);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

// One eager step; with a tape, the Jacobi solve records its phases.
int b3::run_step(b3World_t* w, cudaStream_t st, const JacobiTape* tape) {
    B3_TRY(step_begin(w, st));
    B3_TRY(b3::launch_aabb_hash(w, st));
    B3_TRY(b3::launch_sort_and_cells(w, st));
    B3_TRY(b3::launch_find_pairs(w, st));
    B3_TRY(b3::launch_narrowphase(w, st));
    B3_TRY(b3::launch_manifolds(w, st));
    B3_TRY(b3::launch_solver_taped(w, st, tape));
    B3_TRY(b3::launch_integrate(w, st));
    return B3_OK;
}

static int run_one_step(b3World w, cudaStream_t st) { return b3::run_step(w, st, nullptr); }

static int run_one_step_timed(b3World w, cudaStream_t st) {
    cudaEvent_t ev[9];
    for (auto& e : ev) B3_CUDA(cudaEventCreate(&e));
    for (auto& e : w->npEv) B3_CUDA(cudaEventCreate(&e));
    B3_CUDA(cudaEventCreate(&w->setupEv));
    B3_CUDA(cudaEventRecord(ev[0], st));
    B3_TRY(step_begin(w, st));
    B3_TRY(b3::launch_aabb_hash(w, st));
    B3_CUDA(cudaEventRecord(ev[1], st));
    B3_TRY(b3::launch_sort_and_cells(w, st));
    B3_CUDA(cudaEventRecord(ev[2], st));
    B3_TRY(b3::launch_find_pairs(w, st));
    B3_CUDA(cudaEventRecord(ev[3], st));
    B3_TRY(b3::launch_narrowphase(w, st));
    B3_CUDA(cudaEventRecord(ev[4], st));
    B3_TRY(b3::launch_manifolds(w, st));
    B3_CUDA(cudaEventRecord(ev[5], st));
    B3_TRY(b3::launch_solver(w, st));
    B3_CUDA(cudaEventRecord(ev[6], st));
    B3_TRY(b3::launch_integrate(w, st));
    B3_CUDA(cudaEventRecord(ev[7], st));
    B3_CUDA(cudaEventSynchronize(ev[7]));
    // 7 stages, the narrowphase's four kernels (sweep, refine, clip, exact),
    // then the Jacobi solve's row setup and its iterations
    w->stageMs.assign(13, 0.f);
    for (int k = 0; k < 7; ++k) cudaEventElapsedTime(&w->stageMs[k], ev[k], ev[k + 1]);
    if (w->cfg.maxPairs > 0 && !w->bodies.empty()) {
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&w->stageMs[7 + k], w->npEv[k], w->npEv[k + 1]);
        if (!w->gs) {
            cudaEventElapsedTime(&w->stageMs[11], ev[5], w->setupEv);
            cudaEventElapsedTime(&w->stageMs[12], w->setupEv, ev[6]);
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (auto& e : w->npEv) {
        cudaEventDestroy(e);
        e = nullptr;
    }
    cudaEventDestroy(w->setupEv);
    w->setupEv = nullptr;
    return B3_OK;
}

extern "C" int b3_step(b3World w, int numSteps, void* stream) {
    if (!w || numSteps < 0) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    B3_CUDA(cudaSetDevice(w->ctx->device));
    cudaStream_t st = as_stream(stream);
    int done = 0;
    if (w->cfg.useGraph && !w->timing && numSteps > 0) {
        if (!w->graphValid) {
            // first step eagerly (sets kernel attributes), then capture one step
            B3_TRY(run_one_step(w, st));
            done = 1;
            if (!w->graphStream) B3_CUDA(cudaStreamCreateWithFlags(&w->graphStream, cudaStreamNonBlocking));
            B3_CUDA(cudaStreamSynchronize(st));
            cudaGraph_t g = nullptr;
            B3_CUDA(cudaStreamBeginCapture(w->graphStream, cudaStreamCaptureModeThreadLocal));
            int s = run_one_step(w, w->graphStream);
            cudaError_t ce = cudaStreamEndCapture(w->graphStream, &g);
            if (s != B3_OK) return s;
            if (ce != cudaSuccess) {
                b3_set_error("graph capture failed: %s", cudaGetErrorString(ce));
                return B3_ERR_CUDA;
            }
            if (w->graphExec) cudaGraphExecDestroy(w->graphExec);
            {
                size_t nn = 0;
                cudaGraphGetNodes(g, nullptr, &nn);
                std::vector<cudaGraphNode_t> nodes(nn);
                if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
                int kn = 0;
                for (auto nd : nodes) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kn;
                }
                w->kernelsPerStep = kn;
            }
            cudaError_t ie = cudaGraphInstantiate(&w->graphExec, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) {
                b3_set_error("graph instantiate failed: %s", cudaGetErrorString(ie));
                return B3_ERR_CUDA;
            }
            w->graphValid = true;
        }
        for (int i = done; i < numSteps; ++i) B3_CUDA(cudaGraphLaunch(w->graphExec, st));
        return B3_OK;
    }
    for (int i = 0; i < numSteps; ++i) {
        if (w->timing) B3_TRY(run_one_step_timed(w, st));
        else B3_TRY(run_one_step(w, st));
    }
    return B3_OK;
}

extern "C" int b3_stage_aabbs(b3World w, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    B3_TRY(step_begin(w, st));
    return b3::launch_aabb_hash(w, st);
}
extern "C" int b3_stage_broadphase(b3World w, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    B3_TRY(b3::launch_sort_and_cells(w, st));
    return b3::launch_find_pairs(w, st);
}
extern "C" int b3_stage_narrowphase(b3World w, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    B3_TRY(b3::launch_narrowphase(w, st));
    return b3::launch_manifolds(w, st);
}
extern "C" int b3_stage_solve(b3World w, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    return b3::launch_solver(w, as_stream(stream));
}
extern "C" int b3_stage_integrate(b3World w, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    return b3::launch_integrate(w, as_stream(stream));
}

// Entry points under the reference object API's names.
extern "C" int b3_grid_broadphase_calculate_overlapping_pairs(b3World w, void* stream) {
    return b3_stage_broadphase(w, stream);
}

extern "C" int b3_grid_broadphase_get_pair_count(b3World w, int* count, void* stream) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    int np = 0;
    B3_CUDA(cudaMemcpyAsync(&np, w->d.scalars + b3::S_NUM_PAIRS, 4, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    *count = np;
    return B3_OK;
}

extern "C" int b3_narrowphase_compute_contacts(b3World w, const int32_t* d_pairs, int numPairs, void* stream) {
    if (!w) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    if (d_pairs) {
        if (numPairs < 0) return B3_ERR_INVALID_ARG;
        if (numPairs > w->cfg.maxPairs) {
            b3_set_error("b3_narrowphase_compute_contacts: %d pairs exceed maxPairs %d", numPairs, w->cfg.maxPairs);
            return B3_ERR_CAPACITY;
        }
        if (numPairs > 0)
            B3_CUDA(cudaMemcpyAsync(w->d.pairs, d_pairs, (size_t)numPairs * sizeof(int2), cudaMemcpyDeviceToDevice,
                                    st));
        // pageable source: the copy is staged before the call returns
        B3_CUDA(cudaMemcpyAsync(w->d.scalars + b3::S_NUM_PAIRS, &numPairs, 4, cudaMemcpyHostToDevice, st));
    }
    B3_TRY(b3::launch_narrowphase(w, st));
    return b3::launch_manifolds(w, st);
}

extern "C" int b3_solver_solve_jacobi(b3World w, void* stream) { return b3_stage_solve(w, stream); }

extern "C" int b3_integrate(b3World w, void* stream) { return b3_stage_integrate(w, stream); }

extern "C" int b3_batch_world_offsets(b3World w, int* offsets, int maxWorlds, int* numWorlds) {
    if (!w || !numWorlds) return B3_ERR_INVALID_ARG;
    const int nw = w->cfg.numWorlds > 0 ? w->cfg.numWorlds : 1;
    *numWorlds = nw;
    if (!offsets) return B3_OK;
    if (maxWorlds < nw + 1) return B3_ERR_CAPACITY;
    std::vector<int> cnt(nw + 1, 0);
    for (int id : w->worldIds) {
        if (id < 0 || id >= nw) return B3_ERR_STATE;
        ++cnt[id + 1];
    }
    for (int k = 0; k < nw; ++k) cnt[k + 1] += cnt[k];
    for (int k = 0; k <= nw; ++k) offsets[k] = cnt[k];
    return B3_OK;
}

// ---------------------------------------------------------------------------
// Reads
// ---------------------------------------------------------------------------
extern "C" int b3_get_num_bodies(b3World w, int* n) {
    if (!w || !n) return B3_ERR_INVALID_ARG;
    *n = (int)w->bodies.size();
    return B3_OK;
}

extern "C" int b3_read_state(b3World w, float* pos4, float* quat4, float* linVel4, float* angVel4, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    const size_t N = w->bodies.size();
    cudaStream_t st = as_stream(stream);
    if (pos4) B3_CUDA(cudaMemcpyAsync(pos4, w->d.pos, 16 * N, cudaMemcpyDeviceToHost, st));
    if (quat4) B3_CUDA(cudaMemcpyAsync(quat4, w->d.quat, 16 * N, cudaMemcpyDeviceToHost, st));
    if (linVel4) B3_CUDA(cudaMemcpyAsync(linVel4, w->d.linVel, 16 * N, cudaMemcpyDeviceToHost, st));
    if (angVel4) B3_CUDA(cudaMemcpyAsync(angVel4, w->d.angVel, 16 * N, cudaMemcpyDeviceToHost, st));
    int32_t err = 0;
    B3_CUDA(cudaMemcpyAsync(&err, w->d.scalars + b3::S_ERR, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    if (err) {
        b3_set_error("a bounded device wait gave up; the state read is not valid");
        return B3_ERR_TIMEOUT;
    }
    return B3_OK;
}

// Asynchronous on the stream: the copies read pinned host buffers when the
// stream reaches them (keep them unchanged until then); pageable buffers are
// staged before the call returns.
extern "C" int b3_write_state(b3World w, const float* pos4, const float* quat4, const float* linVel4,
                              const float* angVel4, void* stream) {
    if (!w || !w->written) return B3_ERR_STATE;
    const size_t N = w->bodies.size();
    cudaStream_t st = as_stream(stream);
    if (pos4) B3_CUDA(cudaMemcpyAsync(w->d.pos, pos4, 16 * N, cudaMemcpyHostToDevice, st));
    if (quat4) B3_CUDA(cudaMemcpyAsync(w->d.quat, quat4, 16 * N, cudaMemcpyHostToDevice, st));
    if (linVel4) B3_CUDA(cudaMemcpyAsync(w->d.linVel, linVel4, 16 * N, cudaMemcpyHostToDevice, st));
    if (angVel4) B3_CUDA(cudaMemcpyAsync(w->d.angVel, angVel4, 16 * N, cudaMemcpyHostToDevice, st));
    return B3_OK;
}

extern "C" int b3_read_bodies(b3World w, b3Body* out, int maxBodies, void* stream) {
    if (!w || !out) return B3_ERR_INVALID_ARG;
    const int N = std::min((int)w->bodies.size(), maxBodies);
    if (!w->written) {
        // before the first write: the records as registered (host only)
        for (int i = 0; i < N; ++i) out[i] = w->bodies[i];
        return B3_OK;
    }
    std::vector<float4> p(w->bodies.size()), q(p.size()), l(p.size()), a(p.size());
    B3_TRY(b3_read_state(w, (float*)p.data(), (float*)q.data(), (float*)l.data(), (float*)a.data(), stream));
    for (int i = 0; i < N; ++i) {
        b3Body b = w->bodies[i];
        memcpy(b.pos, &p[i], 16);
        b.pos[3] = 0.f;
        memcpy(b.quat, &q[i], 16);
        memcpy(b.linVel, &l[i], 16);
        memcpy(b.angVel, &a[i], 16);
        out[i] = b;
    }
    return B3_OK;
}

extern "C" int b3_get_counters(b3World w, b3Counters* out, void* stream) {
    if (!w || !out) return B3_ERR_INVALID_ARG;
    if (!w->d.counters) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    B3_CUDA(cudaMemcpyAsync(out, w->d.counters, sizeof(b3Counters), cudaMemcpyDeviceToHost, st));
    int32_t err = 0;
    B3_CUDA(cudaMemcpyAsync(&err, w->d.scalars + b3::S_ERR, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    if (err && out->timeouts == 0) out->timeouts = 1;
    if (err) {
        b3_set_error("a bounded device wait gave up (%d timeouts); results since are not valid",
                     (int)out->timeouts);
        return B3_ERR_TIMEOUT;
    }
    return B3_OK;
}

extern "C" int b3_set_wait_limits(b3World w, int spinLimit, int holdMicros) {
    if (!w || spinLimit < 0 || holdMicros < 0 || holdMicros > 1000000) return B3_ERR_INVALID_ARG;
    w->waitSpinLimit = spinLimit == 0 ? b3::kDefaultSpinLimit : spinLimit;
    w->waitHoldMicros = holdMicros;
    w->graphValid = false;  // the limits are launch arguments of the captured step
    return B3_OK;
}

extern "C" int b3_reset_counters(b3World w, void* stream) {
    if (!w || !w->d.counters) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    B3_CUDA(cudaMemsetAsync(w->d.counters, 0, sizeof(b3Counters), st));
    B3_CUDA(cudaMemsetAsync(w->d.scalars + b3::S_ERR, 0, sizeof(int32_t), st));
    B3_CUDA(cudaStreamSynchronize(st));
    return B3_OK;
}

extern "C" int b3_get_aabbs(b3World w, float* out8, int maxBodies, void* stream) {
    if (!w || !out8) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    const int N = std::min((int)w->bodies.size(), maxBodies);
    std::vector<float4> mn(N), mx(N);
    cudaStream_t st = as_stream(stream);
    B3_CUDA(cudaMemcpyAsync(mn.data(), w->d.aabbMin, 16 * (size_t)N, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaMemcpyAsync(mx.data(), w->d.aabbMax, 16 * (size_t)N, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < N; ++i) {
        memcpy(out8 + 8 * (size_t)i, &mn[i], 16);
        memcpy(out8 + 8 * (size_t)i + 4, &mx[i], 16);
    }
    return B3_OK;
}

extern "C" int b3_get_sorted_hash(b3World w, uint32_t* keys, uint32_t* values, int max, int* count, void* stream) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    const int n = std::min(w->numSmall, max);
    cudaStream_t st = as_stream(stream);
    if (keys && n) B3_CUDA(cudaMemcpyAsync(keys, w->d.keys, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (values && n) B3_CUDA(cudaMemcpyAsync(values, w->d.vals, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    *count = w->numSmall;
    return B3_OK;
}

extern "C" int b3_get_pairs(b3World w, int32_t* pairs2, int max, int* count, void* stream) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    int32_t np = 0;
    B3_CUDA(cudaMemcpyAsync(&np, w->d.scalars + b3::S_NUM_PAIRS, 4, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    *count = np;
    const int n = std::min(np, max);
    if (pairs2 && n > 0) {
        B3_CUDA(cudaMemcpyAsync(pairs2, w->d.pairs, 8 * (size_t)n, cudaMemcpyDeviceToHost, st));
        B3_CUDA(cudaStreamSynchronize(st));
    }
    return B3_OK;
}

extern "C" int b3_get_contacts(b3World w, b3Contact4* out, int max, int* count, void* stream) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    int32_t s[b3::S_NUM_SCALARS] = {};
    B3_CUDA(cudaMemcpyAsync(s, w->d.scalars, sizeof(s), cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    // manifold slots: the pairs', then the sub-pairs' of compound and mesh pairs
    const int np = w->hasSubPairs() ? s[b3::S_NUM_SLOTS] : s[b3::S_NUM_PAIRS];
    const int nm = s[b3::S_NUM_MANIFOLDS];
    *count = nm;
    if (!out || nm <= 0 || max <= 0) return B3_OK;
    std::vector<uint32_t> flag(np);
    std::vector<b3Contact4> all(np);
    if (np > 0) {
        B3_CUDA(cudaMemcpyAsync(flag.data(), w->d.manifoldFlag, 4 * (size_t)np, cudaMemcpyDeviceToHost, st));
        B3_CUDA(cudaMemcpyAsync(all.data(), w->d.contacts, sizeof(b3Contact4) * (size_t)np, cudaMemcpyDeviceToHost, st));
        B3_CUDA(cudaStreamSynchronize(st));
    }
    int k = 0;
    for (int p = 0; p < np && k < max; ++p)
        if (flag[p]) out[k++] = all[p];
    return B3_OK;
}

extern "C" int b3_get_shape_sizes(b3World w, int* numCollidables, int* numPolys, int* numVertices,
                                  int* numFaces, int* numIndices, int* numEdges) {
    if (!w) return B3_ERR_INVALID_ARG;
    if (numCollidables) *numCollidables = (int)w->cols.size();
    if (numPolys) *numPolys = (int)w->polys.size();
    if (numVertices) *numVertices = (int)w->verts4.size() / 4;
    if (numFaces) *numFaces = (int)w->faces.size();
    if (numIndices) *numIndices = (int)w->indices.size();
    if (numEdges) *numEdges = (int)w->edges4.size() / 4;
    return B3_OK;
}

extern "C" int b3_get_shapes(b3World w, b3Collidable* cols, b3ConvexPolyhedron* polys, float* vertices4,
                             b3Face* faces, int* indices, float* edges4, float* localAabbs8) {
    if (!w) return B3_ERR_INVALID_ARG;
    if (cols) memcpy(cols, w->cols.data(), sizeof(b3Collidable) * w->cols.size());
    if (polys) memcpy(polys, w->polys.data(), sizeof(b3ConvexPolyhedron) * w->polys.size());
    if (vertices4) memcpy(vertices4, w->verts4.data(), sizeof(float) * w->verts4.size());
    if (faces) memcpy(faces, w->faces.data(), sizeof(b3Face) * w->faces.size());
    if (indices) memcpy(indices, w->indices.data(), sizeof(int) * w->indices.size());
    if (edges4) memcpy(edges4, w->edges4.data(), sizeof(float) * w->edges4.size());
    if (localAabbs8) memcpy(localAabbs8, w->localAabb8.data(), sizeof(float) * w->localAabb8.size());
    return B3_OK;
}

extern "C" int b3_get_inertias(b3World w, b3Inertia* out, int maxBodies) {
    if (!w || !out) return B3_ERR_INVALID_ARG;
    const int n = std::min((int)w->inertias.size(), maxBodies);
    memcpy(out, w->inertias.data(), sizeof(b3Inertia) * n);
    return B3_OK;
}

extern "C" int b3_get_device_buffer(b3World w, int which, void** d_ptr, int64_t* bytes) {
    if (!w || !d_ptr) return B3_ERR_INVALID_ARG;
    const int64_t N = (int64_t)w->bodies.size();
    void* p = nullptr;
    int64_t b = 0;
    switch (which) {
        case B3_BUF_POS: p = w->d.pos; b = 16 * N; break;
        case B3_BUF_QUAT: p = w->d.quat; b = 16 * N; break;
        case B3_BUF_LINVEL: p = w->d.linVel; b = 16 * N; break;
        case B3_BUF_ANGVEL: p = w->d.angVel; b = 16 * N; break;
        case B3_BUF_AABB_MIN: p = w->d.aabbMin; b = 16 * N; break;
        case B3_BUF_AABB_MAX: p = w->d.aabbMax; b = 16 * N; break;
        case B3_BUF_PAIRS: p = w->d.pairs; b = 8 * (int64_t)w->cfg.maxPairs; break;
        case B3_BUF_CONTACTS: p = w->d.contacts; b = (int64_t)sizeof(b3Contact4) * w->cfg.maxPairs; break;
        case B3_BUF_COUNTERS: p = w->d.counters; b = sizeof(b3Counters); break;
        case B3_BUF_INVMASS: p = w->d.invMass; b = 4 * N; break;
        default: return B3_ERR_INVALID_ARG;
    }
    *d_ptr = p;
    if (bytes) *bytes = b;
    return B3_OK;
}

extern "C" int b3_set_stage_timing(b3World w, int enable) {
    if (!w) return B3_ERR_INVALID_ARG;
    w->timing = enable != 0;
    return B3_OK;
}

extern "C" int b3_get_stage_times(b3World w, float* ms, int max, int* count) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    *count = (int)w->stageMs.size();
    for (int i = 0; i < std::min(max, *count); ++i) ms[i] = w->stageMs[i];
    return B3_OK;
}

namespace b3 {
int launch_world_stats(b3World_t* w, cudaStream_t st) {
    const int N = (int)w->bodies.size();
    B3_CUDA(cudaMemsetAsync(w->d.worldStats, 0, sizeof(float4) * 2 * w->cfg.numWorlds, st));
    if (N == 0) return B3_OK;
    k_world_stats<<<(N + 255) / 256, 256, 0, st>>>(w->bodiesDev(), w->d.worldStats, w->cfg.numWorlds);
    B3_CHECK_LAUNCH();
    return B3_OK;
}
}  // namespace b3

extern "C" int b3_batch_world_stats(b3World w, float* out4, int numWorlds, void* stream) {
    if (!w || !out4 || numWorlds <= 0) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    B3_TRY(b3::launch_world_stats(w, st));
    const int nw = std::min(numWorlds, w->cfg.numWorlds);
    std::vector<float4> s(2 * (size_t)w->cfg.numWorlds);
    B3_CUDA(cudaMemcpyAsync(s.data(), w->d.worldStats, sizeof(float4) * s.size(), cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < nw; ++k) {
        const float m = s[2 * k].w;
        out4[4 * k + 0] = m > 0 ? s[2 * k].x / m : 0.f;
        out4[4 * k + 1] = m > 0 ? s[2 * k].y / m : 0.f;
        out4[4 * k + 2] = m > 0 ? s[2 * k].z / m : 0.f;
        out4[4 * k + 3] = s[2 * k + 1].x;
    }
    return B3_OK;
}

// Autotuner: coordinate descent over the launch shapes of the tunable
// kernels on the world's current scene. Each trial restores the body state
// and counters, runs one untimed step and then trialSteps timed eager steps
// (CUDA events on the stream); the fastest value of each knob is kept, the
// state is restored and the step graph is recaptured on the next b3_step.
extern "C" int b3_autotune(b3World w, int trialSteps, void* stream) {
    if (!w || trialSteps <= 0) return B3_ERR_INVALID_ARG;
    if (!w->written) return B3_ERR_STATE;
    B3_CUDA(cudaSetDevice(w->ctx->device));
    cudaStream_t st = as_stream(stream);
    const size_t N = w->bodies.size();
    float4* save = nullptr;
    B3_CUDA(cudaMalloc((void**)&save, 4 * N * sizeof(float4)));
    float4* bufs[4] = {w->d.pos, w->d.quat, w->d.linVel, w->d.angVel};
    b3Counters ctr;
    int rc = B3_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto restore = [&]() -> int {
        for (int k = 0; k < 4; ++k)
            B3_CUDA(cudaMemcpyAsync(bufs[k], save + k * N, N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        B3_CUDA(cudaMemcpyAsync(w->d.counters, &ctr, sizeof(ctr), cudaMemcpyHostToDevice, st));
        return B3_OK;
    };
    auto trial = [&](float* ms) -> int {
        B3_TRY(restore());
        B3_TRY(b3::run_step(w, st, nullptr));
        B3_TRY(restore());
        B3_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < trialSteps; ++i) B3_TRY(b3::run_step(w, st, nullptr));
        B3_CUDA(cudaEventRecord(e1, st));
        B3_CUDA(cudaEventSynchronize(e1));
        B3_CUDA(cudaEventElapsedTime(ms, e0, e1));
        ++w->tunedTrials;
        return B3_OK;
    };
    struct Knob {
        int* v;
        int n;
        int cand[3];
    };
    // the narrowphase CTA size and the FP32 clip form by whole-step trials;
    // with the batched Gauss-Seidel solver also its grid width (solverMode).
    // The Jacobi launch shapes interact (a one-knob-at-a-time descent stops
    // in a local optimum), so they are searched jointly below on the solve
    // alone.
    Knob knobs[] = {{&w->npWarpsPerBlock, 3, {1, 2, 4}}, {&w->clipGroups, 2, {0, 1, 0}}, {&w->solverMode, 2, {0, 1, 0}}};
    const int numKnobs = w->gs ? 3 : 2;
    // one solve from the current contacts, timed (the solve leaves the body
    // state alone: the finish happens in the integration)
    auto solve_trial = [&](float* ms) -> int {
        B3_TRY(b3::launch_solver(w, st));
        B3_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < 3; ++i) B3_TRY(b3::launch_solver(w, st));
        B3_CUDA(cudaEventRecord(e1, st));
        B3_CUDA(cudaEventSynchronize(e1));
        B3_CUDA(cudaEventElapsedTime(ms, e0, e1));
        ++w->tunedTrials;
        return B3_OK;
    };
    // three pair searches over the same sorted keys, timed
    auto pair_trial = [&](float* ms) -> int {
        B3_TRY(b3::launch_find_pairs(w, st));
        B3_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < 3; ++i) B3_TRY(b3::launch_find_pairs(w, st));
        B3_CUDA(cudaEventRecord(e1, st));
        B3_CUDA(cudaEventSynchronize(e1));
        B3_CUDA(cudaEventElapsedTime(ms, e0, e1));
        ++w->tunedTrials;
        return B3_OK;
    };
    do {
        for (int k = 0; k < 4 && rc == B3_OK; ++k)
            if (cudaMemcpyAsync(save + k * N, bufs[k], N * sizeof(float4), cudaMemcpyDeviceToDevice, st) !=
                cudaSuccess)
                rc = B3_ERR_CUDA;
        if (rc != B3_OK) break;
        if (cudaMemcpyAsync(&ctr, w->d.counters, sizeof(ctr), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess) {
            rc = B3_ERR_CUDA;
            break;
        }
        for (int ki = 0; ki < numKnobs; ++ki) {
            Knob& kb = knobs[ki];
            int best = *kb.v;
            float bestMs = 1e30f;
            for (int ci = 0; ci < kb.n; ++ci) {
                const int c = kb.cand[ci];
                *kb.v = c;
                float ms = 0.f;
                if ((rc = trial(&ms)) != B3_OK) break;
                if (ms < bestMs) {
                    bestMs = ms;
                    best = c;
                }
            }
            *kb.v = best;
            if (rc != B3_OK) break;
        }
        if (rc == B3_OK && !w->sap) {
            // grid pair search: thread per body or warp per body, each timed
            // on three searches over the same sorted keys
            rc = restore();
            if (rc == B3_OK) rc = step_begin(w, st);
            if (rc == B3_OK) rc = b3::launch_aabb_hash(w, st);
            if (rc == B3_OK) rc = b3::launch_sort_and_cells(w, st);
            int bp = w->pairSearchMode;
            float bestMs = 1e30f;
            for (int m = 0; m < 2 && rc == B3_OK; ++m) {
                w->pairSearchMode = m;
                float ms = 0.f;
                if ((rc = pair_trial(&ms)) != B3_OK) break;
                if (ms < bestMs) {
                    bestMs = ms;
                    bp = m;
                }
            }
            w->pairSearchMode = bp;
        }
        if (rc == B3_OK && !w->gs) {
            // Jacobi: CTA size x blocks per SM x gather (x mode for batched
            // worlds), every combination timed on the same contacts
            rc = restore();
            if (rc == B3_OK) rc = step_begin(w, st);
            if (rc == B3_OK) rc = b3::launch_aabb_hash(w, st);
            if (rc == B3_OK) rc = b3::launch_sort_and_cells(w, st);
            if (rc == B3_OK) rc = b3::launch_find_pairs(w, st);
            if (rc == B3_OK) rc = b3::launch_narrowphase(w, st);
            if (rc == B3_OK) rc = b3::launch_manifolds(w, st);
            int bt = w->solverThreads, bo = w->solverOccCap, bg = w->solverGather, bm = w->solverMode;
            float bestMs = 1e30f;
            const int modes = w->cfg.numWorlds > 1 ? 2 : 1;  // per-world solver only for batched worlds
            for (int m = 0; m < modes && rc == B3_OK; ++m)
                for (int t : {64, 128, 256})
                    for (int o : {1, 2, 4, 8})
                        for (int g = 0; g < 2 && rc == B3_OK; ++g) {
                            if (m == 1 && o > 1) continue;  // the per-world grid ignores the cap
                            w->solverMode = m;
                            w->solverThreads = t;
                            w->solverOccCap = o;
                            w->solverGather = g;
                            float ms = 0.f;
                            if ((rc = solve_trial(&ms)) != B3_OK) break;
                            if (ms < bestMs) {
                                bestMs = ms;
                                bt = t, bo = o, bg = g, bm = m;
                            }
                        }
            w->solverThreads = bt, w->solverOccCap = bo, w->solverGather = bg, w->solverMode = bm;
        }
        if (rc == B3_OK) rc = restore();
        if (rc == B3_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = B3_ERR_CUDA;
    } while (false);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(save);
    w->graphValid = false;  // recapture with the chosen shapes
    return rc;
}

extern "C" int b3_set_tuning(b3World w, const int* values, int count) {
    if (!w || !values || count < 3) return B3_ERR_INVALID_ARG;
    const int np = values[0], st = values[2], cap = count >= 5 ? values[4] : w->solverOccCap;
    const int mode = count >= 7 ? values[6] : w->solverMode;
    const int gather = count >= 8 ? values[7] : w->solverGather;
    const int pairMode = count >= 9 ? values[8] : w->pairSearchMode;
    const int clipG = count >= 10 ? values[9] : w->clipGroups;
    if ((np != 1 && np != 2 && np != 4) || (st != 64 && st != 128 && st != 256) || cap < 1 || cap > 8 ||
        (mode != 0 && mode != 1) || (gather != 0 && gather != 1) || (pairMode != 0 && pairMode != 1) ||
        (clipG != 0 && clipG != 1))
        return B3_ERR_INVALID_ARG;
    w->npWarpsPerBlock = np;
    w->solverThreads = st;
    w->solverOccCap = cap;
    w->solverMode = mode;
    w->solverGather = gather;
    w->pairSearchMode = pairMode;
    w->clipGroups = clipG;
    w->graphValid = false;
    return B3_OK;
}

extern "C" int b3_get_tuning(b3World w, int* values, int max, int* count) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    int v[10] = {w->npWarpsPerBlock, w->pairThreads, w->solverThreads, w->kernelsPerStep, w->solverOccCap,
                 w->tunedTrials, w->solverMode, w->solverGather, w->pairSearchMode, w->clipGroups};
    *count = 10;
    for (int i = 0; i < std::min(10, max); ++i) values[i] = v[i];
    return B3_OK;
}

// Adjoint entry points are implemented in adjoint.cu.
