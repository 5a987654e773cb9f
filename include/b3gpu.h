/*
 * b3gpu.h — C ABI of the B200-native rigid-body step.
 *
 * This is the drop-in boundary for the reference GPU rigid-body pipeline
 * (erwincoumans/experiments, opencl/gpu_rigidbody_pipeline2 and its
 * dependencies). Every entry point is plain C: opaque handles, plain
 * pointers and sizes, int status codes (0 = OK), no exceptions across the
 * ABI and no torch types. Device pointers are CUDA device pointers; streams
 * are cudaStream_t passed as void* (NULL = legacy default stream). Nothing
 * synchronises implicitly except the *_read_* / *_get_* calls that copy to
 * host memory and b3_sync.
 *
 * Citations name files relative to the reference project root:
 *   P2/ = opencl/gpu_rigidbody_pipeline2/   P1/ = opencl/gpu_rigidbody_pipeline/
 *   BB/ = opencl/broadphase_benchmark/      G3/ = opencl/3dGridBroadphase/Shared/
 *   ST/ = dynamics/basic_demo/Stubs/         PR/ = opencl/primitives/AdlPrimitives/
 */
#ifndef B3GPU_H
#define B3GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status codes                                                         */
/* ------------------------------------------------------------------ */
enum {
    B3_OK = 0,
    B3_ERR_INVALID_ARG = 1,
    B3_ERR_CUDA = 2,            /* a CUDA runtime call failed */
    B3_ERR_CAPACITY = 3,        /* a fixed capacity would be exceeded */
    B3_ERR_NO_DEVICE = 4,       /* no CUDA device / extension not usable */
    B3_ERR_STATE = 5,           /* call out of order (e.g. step before write) */
    B3_ERR_TIMEOUT = 6,         /* a device-side bounded wait gave up */
    B3_ERR_UNSUPPORTED = 7
};

/* ------------------------------------------------------------------ */
/* Reference-layout data types (byte-compatible where noted)            */
/* ------------------------------------------------------------------ */

/* RigidBodyBase::Body, ST/AdlRigidBody.h:26-45 (80 bytes, same layout). */
typedef struct b3Body {
    float pos[4];          /* w unused (0) */
    float quat[4];         /* x, y, z, w */
    float linVel[4];
    float angVel[4];
    uint32_t collidableIdx;
    float invMass;
    float restitution;
    float friction;
} b3Body;

/* RigidBodyBase::Inertia, ST/AdlRigidBody.h:47-59 (96 bytes, same layout:
 * two 3x4 row-major matrices, world then local inverse inertia). */
typedef struct b3Inertia {
    float invInertiaWorld[12];
    float initInvInertia[12];
} b3Inertia;

/* btCollidable, P1/btCollidable.h:5-11 (16 bytes, same layout). */
typedef struct b3Collidable {
    int numChildShapes;
    float radius;
    int shapeType;         /* B3_SHAPE_* */
    int shapeIndex;
} b3Collidable;

/* Shape types, the values of the reference's CollisionShape enum
 * (P2/sat.cl:1-5, P2/satClipHullContacts.cl:4-5). What shapeIndex, radius
 * and numChildShapes hold for each:
 *   CONVEX_HULL: shapeIndex = its b3ConvexPolyhedron;
 *   PLANE: shapeIndex = its b3Face (normal, constant), radius = constant;
 *   CONCAVE_TRIMESH: shapeIndex = its b3ConvexPolyhedron, whose faces are
 *     the triangles and whose `unused` field holds the first of the
 *     per-triangle polytopes (see b3_register_concave_mesh),
 *     numChildShapes = number of triangles;
 *   COMPOUND_OF_CONVEX_HULLS: shapeIndex = first b3ChildShape,
 *     numChildShapes = number of children;
 *   SPHERE: radius. */
enum {
    B3_SHAPE_CONVEX_HULL = 3,
    B3_SHAPE_PLANE = 4,
    B3_SHAPE_CONCAVE_TRIMESH = 5,
    B3_SHAPE_COMPOUND_OF_CONVEX_HULLS = 6,
    B3_SHAPE_SPHERE = 7
};

/* btGpuChildShape (P2/sat.cl:21-29, 48 bytes, same layout): a child of a
 * compound, a convex hull collidable at a pose relative to the compound's
 * body (position xyz, orientation quaternion xyzw). */
typedef struct b3ChildShape {
    float childPosition[4];
    float childOrientation[4];
    int shapeIndex;        /* collidable of a convex hull */
    int unused[3];
} b3ChildShape;

/* ConvexPolyhedronCL, P2/ConvexPolyhedronCL.h:15-31 (96 bytes, same layout). */
typedef struct b3ConvexPolyhedron {
    float localCenter[4];
    float extents[4];
    float mC[4];
    float mE[4];
    float radius;
    int faceOffset;
    int numFaces;
    int numVertices;
    int vertexOffset;
    int uniqueEdgesOffset;
    int numUniqueEdges;
    int unused;
} b3ConvexPolyhedron;

/* btGpuFace, P2/ConvexPolyhedronCL.h:6-13 (plane + index range; padded to
 * 32 bytes like the reference's 16-byte aligned struct). */
typedef struct b3Face {
    float plane[4];        /* outward normal xyz, w = plane constant */
    int indexOffset;
    int numIndices;
    int pad[2];
} b3Face;

/* Contact manifold, after Contact4 (ST/AdlContact4.h:26-59), 96 bytes.
 * worldPos[k].w = penetration depth (negative = penetrating);
 * worldNormal.w = number of points (1..4), normal points from A to B.
 * Differences from the reference: friction is a float (the reference packs
 * u16 restitution + u16 friction), the combined restitution is derived from
 * the two bodies in the solver, and m_batchIdx holds the broadphase pair
 * index. Body fields carry a negative sign for static bodies. */
typedef struct b3Contact4 {
    float worldPos[4][4];
    float worldNormal[4];
    float friction;
    int pairIndex;
    int bodyAPtrAndSignBit;
    int bodyBPtrAndSignBit;
} b3Contact4;

/* Constraint4, ST/AdlConstraint4.h:23-47 (176 bytes, same layout): one
 * manifold as the batched Gauss-Seidel solver holds it. linear = -normal
 * (w = friction coefficient), jacCoeffInv = -1 / effective mass per point
 * (0 for an unused point), b = position correction per point, appliedRambdaDt
 * = accumulated normal impulses, center and fJacCoeffInv / fAppliedRambdaDt
 * the two friction directions at the manifold centre. bodyA / bodyB are
 * body indices (no sign), batchIdx the batch within the parity class. */
typedef struct b3Constraint4 {
    float linear[4];
    float worldPos[4][4];
    float center[4];
    float jacCoeffInv[4];
    float b[4];
    float appliedRambdaDt[4];
    float fJacCoeffInv[2];
    float fAppliedRambdaDt[2];
    uint32_t bodyA;
    uint32_t bodyB;
    int32_t batchIdx;
    uint32_t padding;
} b3Constraint4;

/* Step diagnostics (the reference truncates silently; the build counts).
 * Every count is of the last step, except timeouts and steps, which
 * accumulate until b3_reset_counters. */
typedef struct b3Counters {
    int32_t numPairs;            /* broadphase pairs this step */
    int32_t numManifolds;        /* contact manifolds this step */
    int32_t numContactPoints;    /* sum of manifold points */
    int32_t pairOverflow;        /* pairs dropped this step: per-body or global cap */
    int32_t cellOverflow;        /* candidates skipped by the per-cell cap this step */
    int32_t timeouts;            /* bounded device waits that gave up */
    int32_t clipOverflow;        /* clipped polygons truncated to 64 verts this step */
    int32_t steps;               /* steps executed since write_bodies */
    int32_t refinedAxes;         /* pairs whose axis choice was re-ranked in float-float */
    int32_t refinedClips;        /* pairs whose clipping was redone in float-float */
} b3Counters;

/* ------------------------------------------------------------------ */
/* Context (device + default stream)                                    */
/* ------------------------------------------------------------------ */
typedef struct b3Context_t* b3Context;

/* Replaces btOpenCLUtils::createContextFromType + clCreateCommandQueue
 * (opencl/basic_initialize/btOpenCLUtils.h:33-56). device = -1 creates a
 * host-only context: shape and body registration work, anything that
 * touches the GPU returns B3_ERR_NO_DEVICE. */
int b3_context_create(int device, b3Context* out);
int b3_context_destroy(b3Context ctx);
int b3_sync(b3Context ctx, void* stream);
/* Library + device description, one line (driver, SM count). */
int b3_context_info(b3Context ctx, char* buf, int buflen);
/* Last error message of this thread (static storage). */
const char* b3_last_error(void);

/* ------------------------------------------------------------------ */
/* GPU primitives (device pointers, caller-owned)                       */
/* ------------------------------------------------------------------ */

/* btFillCL::execute (BB/btFillCL.h:85-126, PR/Fill/FillKernels.cl:47-96):
 * dst[offset + i] = value for i < n. */
int b3_fill_u32(b3Context ctx, uint32_t* d_dst, uint32_t value, int64_t n, int64_t offset, void* stream);
/* FillInt2Kernel: dst[offset + i] = (x, y). */
int b3_fill_int2(b3Context ctx, int32_t* d_dst_int2, int32_t x, int32_t y, int64_t n, int64_t offset, void* stream);

/* btPrefixScanCL::execute (BB/btPrefixScanCL.cpp:46-98): exclusive scan
 * d_dst[i] = sum_{j<i} d_src[j]; optional total written to d_sum (device)
 * and/or *h_sum (host, synchronising). In-place allowed. No size limit
 * (the reference's top level holds 2,048 blocks x 256). */
int b3_prefix_scan_u32(b3Context ctx, const uint32_t* d_src, uint32_t* d_dst, int64_t n,
                       uint32_t* d_sum, uint32_t* h_sum, void* stream);

/* Exclusive scan that allocates nothing. It has no counterpart in the
 * reference. For callers that cannot call cudaMalloc (an engine that owns
 * all GPU memory through its own pool, a real-time loop that must never
 * allocate, a plug-in whose allocator belongs to another runtime): same
 * result as b3_prefix_scan_u32, but the scratch is a fixed 33 KB device
 * array inside the library, so no context is needed either.
 * Limit: n <= 16,777,216 (larger n returns B3_ERR_CAPACITY). All calls on
 * a device share that array: calls that overlap on the GPU race, so keep
 * them on one stream. The first call on a device looks up the array's
 * address; make it before any stream capture. The total goes to d_sum
 * (device, may be NULL). d_err (device, may be NULL) receives 0 after a
 * valid scan and 1 if a bounded wait inside the scan gave up, in which case
 * d_dst and d_sum are not valid. */
int b3_prefix_scan_u32_static(const uint32_t* d_src, uint32_t* d_dst, int64_t n, uint32_t* d_sum,
                              int32_t* d_err, void* stream);

/* btRadixSort32CL::execute (BB/btRadixSort32CL.cpp:161-535): stable LSD
 * key-value sort of n (key, value) pairs, in place. Only the low key_bits
 * bits of the keys are sorted (1..32); keys must not use higher bits unless
 * key_bits = 32. Onesweep with 8-bit digits: ceil(key_bits/8) passes. */
int b3_radix_sort32_kv(b3Context ctx, uint32_t* d_keys, uint32_t* d_values, int64_t n,
                       int key_bits, void* stream);
/* Keys-only variant (RadixSort32 keys-only benchmark,
 * opencl/primitives/AdlTest/RadixSortBenchmark.h:64). */
int b3_radix_sort32_keys(b3Context ctx, uint32_t* d_keys, int64_t n, int key_bits, void* stream);
/* btRadixSort32CL::execute(keysIn, keysOut, valuesIn, valuesOut, n, sortBits)
 * (BB/btRadixSort32CL.h:67-68): out of place. The inputs are only read; the
 * stably sorted keys and values land in the outputs, which must not be the
 * inputs. d_values_in / d_values_out may both be NULL (keys only). The
 * reference declares this form with an empty body
 * (BB/btRadixSort32CL.cpp:151-155); this is the sort its signature names. */
int b3_radix_sort32_kv_out(b3Context ctx, const uint32_t* d_keys_in, uint32_t* d_keys_out,
                           const uint32_t* d_values_in, uint32_t* d_values_out, int64_t n, int key_bits,
                           void* stream);
/* btRadixSort32CL::execute(btOpenCLArray<btSortData>& keyValuesInOut,
 * sortBits) (BB/btRadixSort32CL.h:70): the grid broadphase's and the batched
 * solver's form. d_key_values holds n btSortData records (BB/btRadixSort32CL.h:
 * 7-11: int m_key, int m_value; 8 bytes, 8-byte aligned), sorted in place
 * by the low key_bits bits of m_key taken as unsigned, stably. */
int b3_radix_sort32_sortdata(b3Context ctx, int32_t* d_key_values, int64_t n, int key_bits, void* stream);

/* btBoundSearchCL::execute (BB/btBoundSearchCL.cpp:78-136,
 * PR/Search/BoundSearchKernels.cl:42-104) over sorted keys.
 * mode 0 = LOWER: d_dst[k] = first index with key == k (untouched if absent)
 * mode 1 = UPPER: d_dst[k] = one past the last index with key == k
 * mode 2 = COUNT: d_dst[k] = number of keys equal to k (fills 0 first).
 * Keys >= n_dst are ignored (the reference would write out of range). */
int b3_bound_search(b3Context ctx, const uint32_t* d_sorted_keys, int64_t n_src,
                    uint32_t* d_dst, int64_t n_dst, int mode, void* stream);
/* btBoundSearchCL::execute(btOpenCLArray<btSortData>& src, nSrc, dst, nDst,
 * option) (BB/btBoundSearchCL.h:60): the same search over btSortData records
 * sorted by m_key (8-byte aligned), modes as b3_bound_search. One difference
 * follows the reference's SearchSortDataUpperKernel
 * (PR/Search/BoundSearchKernels.cl:66-86): in UPPER mode, when no record has
 * key 0, d_dst[0] is set to 0. Keys >= n_dst are skipped (the reference
 * writes past d_dst for them). */
int b3_bound_search_sortdata(b3Context ctx, const int32_t* d_sorted_key_values, int64_t n_src, uint32_t* d_dst,
                             int64_t n_dst, int mode, void* stream);

/* ------------------------------------------------------------------ */
/* World: rigid-body & collidable arrays, grid broadphase,              */
/* narrowphase-and-solver, stepSimulation                               */
/* ------------------------------------------------------------------ */
typedef struct b3World_t* b3World;

enum { B3_FRICTION_GEOMEAN = 0, B3_FRICTION_PRODUCT = 1 };

typedef struct b3WorldConfig {
    int32_t maxBodies;            /* capacity (no 128K cap, P1/btGpuNarrowPhaseAndSolver.h:24) */
    int32_t maxPairs;             /* dense pair-list capacity */
    int32_t numWorlds;            /* 1 = plain step; >1 = batched independent worlds */
    float   cellSize;             /* grid cell edge (m) */
    int32_t gridDims[3];          /* per-world grid, powers of two (G3/bt3dGridBroadphaseOCL.cl:7-9) */
    int32_t maxBodiesPerCell;     /* bucket cap, reference maxSmallProxiesPerCell */
    int32_t maxPairsPerBody;      /* per-body cap, reference maxPairsPerSmallProxy */
    float   maxSmallProxySize;    /* AABB half-diagonal > half this => large body */
    float   gravity[3];
    float   dt;
    int32_t solverIterations;     /* btContactSolverInfo::m_numIterations */
    float   erp;                  /* Baumgarte factor, m_erp (0.2) */
    float   contactBreaking;      /* clip keep threshold maxDist (0.02) */
    float   contactProcessing;    /* solver distance threshold (0.02) */
    float   linearSlopOffset;     /* distance = depth + this (0.01, P2/btPgsJacobiSolver.cpp:124-155) */
    float   angularDamping;       /* per-step factor (0.99, BB/integrateKernel.cl:124-126) */
    int32_t frictionCombine;      /* B3_FRICTION_* */
    int32_t useGraph;             /* capture the step as a CUDA graph */
    int32_t flags;                /* B3_WORLD_* bits, 0 = defaults */
} b3WorldConfig;

/* flags: B3_WORLD_SAP_BROADPHASE selects the sweep-and-prune broadphase of
 * gpu_rigidbody_pipeline2 (its default, P2/CLPhysicsDemo.cpp:17) in place of
 * the uniform grid: dynamic bodies are the sorted small proxies, static
 * bodies the large proxies (P2/CLPhysicsDemo.cpp:558-568). One world only
 * (numWorlds = 1), as in the reference. */
enum { B3_WORLD_SAP_BROADPHASE = 1 };
/* flags: B3_WORLD_BATCHED_GS_SOLVER selects the reference's GPU solver
 * (btGpuNarrowphaseAndSolver::solveContacts, P1/btGpuNarrowPhaseAndSolver.cpp:
 * 1073-1353, with ST/Solver.cpp) in place of pipeline2's Jacobi solver:
 * manifolds binned to a 16 x 16 grid of 2 m xz cells by their dynamic body
 * (SetSortDataKernel, ST/solverSetup2.cl:457-478), cells taken in four
 * parity classes (ST/solveContact.cl:418-426), each class coloured into
 * batches without a shared dynamic body, Constraint4 set up per manifold
 * (ST/solverSetup.cl:520-609), then 4 contact and 4 friction Gauss-Seidel
 * iterations, batch after batch (ST/Solver.cpp:561-700), writing body
 * velocities directly. The colouring is the greedy pass of the reference's
 * CPU batching (sortConstraintByBatch, P1/btGpuNarrowPhaseAndSolver.cpp:
 * 752-852) over each class in (cell, manifold) order with exact body
 * identities: deterministic, and free of the reference GPU colouring's
 * races between concurrently solved cells. */
enum { B3_WORLD_BATCHED_GS_SOLVER = 2 };

/* Defaults: reference constants (P2/CLPhysicsDemo.cpp:603-653,
 * BB/integrateKernel.cl:102-158, P2/btPgsJacobiSolver.cpp:171-191). */
void b3_world_config_default(b3WorldConfig* cfg);

int b3_world_create(b3Context ctx, const b3WorldConfig* cfg, b3World* out);
int b3_world_destroy(b3World w);

/* CLPhysicsDemo::registerConvexPolyhedron (P2/CLPhysicsDemo.cpp:491-531 ->
 * btConvexUtility::initializePolyhedralFeatures P1/btConvexUtility.cpp:31-270
 * -> btGpuNarrowphaseAndSolver::registerConvexHullShape
 * P1/btGpuNarrowPhaseAndSolver.cpp:423-490): convex hull of the scaled
 * points, coplanar face weld, unique edges; local centre = vertex average
 * (P2/CLPhysicsDemo.cpp:360-366). Returns the collidable index. */
/* btGpuSapBroadphase::calculateOverlappingPairs (P2/btGpuSapBroadphase.cpp:
 * 97-485) for a world created with B3_WORLD_SAP_BROADPHASE, from the world
 * AABBs of b3_stage_aabbs (initializeGpuAabbsFull); b3_stage_broadphase of
 * such a world runs the same. Steps: FloatFlip keys
 * of the small proxies' minimum x (flipFloatKernel, BB/sap.cl:301-311),
 * stable 32-bit radix sort, sorted copy (scatterKernel :313-320), then the
 * pairs: for each sorted small proxy i, first every large proxy whose AABB
 * overlaps it (computePairsKernelTwoArrays :65-90; pair = (large id, small
 * id)), then every later proxy j whose minimum x does not exceed i's
 * maximum x and whose AABB overlaps (computePairsKernel, BB/sapFast.cl:
 * 48-150; pair = (id_i, id_j)). The reference appends both sets with
 * atomics in an unspecified order; here the order is the one just given
 * (deterministic). Pairs beyond maxPairs are counted in pairOverflow. The
 * pair list replaces the world's (b3_get_device_buffer B3_BUF_PAIRS). */
int b3_sap_broadphase_calculate_overlapping_pairs(b3World w, void* stream);

/* computePairsKernel (BB/sapFast.cl:48-150) on a caller-sorted array of
 * n AABBs in the reference's btAabbCL layout (8 floats per AABB: min xyz,
 * min w = proxy id as int bits, max xyz, max w), sorted by minimum along
 * axis (0..2): for each i, every later j whose minimum along axis does not
 * exceed i's maximum and whose AABB overlaps (inclusive, x, z, y) gives the
 * pair (id_i, id_j), in order of i then j. Writes min(count, maxPairs) pairs
 * to d_pairs (int2) and the full count to *d_count (device int). Takes the
 * context for its scratch (allocated per call); synchronises the stream. */
int b3_sap_compute_pairs(b3Context ctx, const float* d_sortedAabbs, int n, int axis, int32_t* d_pairs,
                         int maxPairs, int32_t* d_count, void* stream);

int b3_register_convex_hull(b3World w, const float* vertices, int numVertices, int strideBytes,
                            const float scaling[3], int* collidableOut);

/* CLPhysicsDemo::registerSphereShape (P2/CLPhysicsDemo.cpp:420-456): a
 * sphere of the given radius (> 0); local AABB +-radius. Spheres collide
 * with spheres and planes (clipHullHullKernel, P2/satClipHullContacts.cl:
 * 1057-1124); the reference has no sphere-hull contact, nor has this. */
int b3_register_sphere(b3World w, float radius, int* collidableOut);
/* CLPhysicsDemo::registerPlaneShape (:459-490) -> registerFace
 * (P1/btGpuNarrowPhaseAndSolver.cpp:252-262): the plane n . x = constant
 * in the body's frame (n of unit length), unbounded (local AABB +-1e30).
 * Planes collide with spheres only, as there. */
int b3_register_plane(b3World w, const float normal[3], float planeConstant, int* collidableOut);
/* CLPhysicsDemo::registerCompoundShape (P2/CLPhysicsDemo.cpp:217-285) ->
 * registerCompoundShape (P1/btGpuNarrowPhaseAndSolver.cpp:237-250): a
 * compound of n convex hull children (each child's shapeIndex a
 * convex-hull collidable registered before). Local AABB: the union of the
 * children's AABBs at their poses. A compound pair expands into one pair
 * per child (per child pair for compound-compound) with no culling between
 * children (findCompoundPairsKernel, P2/sat.cl:747-926), each tested and
 * clipped as two hulls at the composed poses; every child pair with
 * contact points gives its own manifold. Compounds collide with hulls and
 * compounds. */
int b3_register_compound(b3World w, const b3ChildShape* children, int numChildren, int* collidableOut);
/* CLPhysicsDemo::registerConcaveMesh (P2/CLPhysicsDemo.cpp:288-330) ->
 * registerConcaveMeshShape (P1/btGpuNarrowPhaseAndSolver.cpp:264-333): a
 * triangle mesh (numIndices / 3 triangles, vertices scaled by scaling),
 * normally the shape of a static body. Each triangle's plane is
 * normalize((v1 - v0) x (v2 - v0)), -n . v0. Against a convex hull, every
 * triangle whose local AABB overlaps the hull's world AABB is tested as the
 * reference builds it in findSeparatingAxisKernel (P2/sat.cl:970-1191): a
 * polytope of the 3 vertices, the front and back faces, 3 edge planes and
 * the 3 edges, clipped as a hull (clipHullHullConcaveConvexKernel,
 * P2/satClipHullContacts.cl:1387); each triangle with contact points gives
 * its own manifold. These polytopes are registered here, after the mesh's
 * own table entry. The reference's test takes the mesh's local triangle
 * AABBs as world ones (a mesh body at the origin, unrotated), and so does
 * this. The reference tests a mesh only when it is the pair's first body;
 * here either order is tested, the mesh body taking the manifold's A side. */
int b3_register_concave_mesh(b3World w, const float* vertices3, int numVertices, const int* indices,
                             int numIndices, const float scaling[3], int* collidableOut);

/* CLPhysicsDemo::registerPhysicsInstance (P2/CLPhysicsDemo.cpp:533-599) ->
 * btGpuNarrowphaseAndSolver::registerRigidBody (P1/...cpp:566-657):
 * mass 0 = static. Inverse inertia from the registration AABB (margin
 * 0.01) with full extents, as the reference does. worldId selects the
 * independent world in batched mode (0 for plain). Returns the body id. */
int b3_register_body(b3World w, float mass, const float position[3], const float orientation[4],
                     int collidable, float friction, float restitution, int worldId, int* bodyOut);

/* btBulletDataExtractor::convertAllObjects (P2/BulletDataExtractor.cpp:
 * 456-721) on a .bullet scene file as bullet2's btDefaultSerializer writes it
 * (single precision, little endian), read by this library's own parser of
 * the format (chunks and the DNA1 struct catalogue, fields found by name as
 * bParse's btBulletFile does). Registers, in file order, the box shapes (the
 * unit cube scaled by halfDimensions * localScaling + margin) and convex
 * hulls (points times localScaling); spheres, planes and other shapes are
 * skipped, as there. Then the rigid bodies, grouped by shape in shape order:
 * mass 1 / inverseMass, position and orientation from the world transform,
 * friction 1 (registerRigidBody, P1/btGpuNarrowPhaseAndSolver.cpp:577).
 * Static bodies are dropped unless keepStaticObjects, and then, as the demo
 * does, a 50 x 50 grid of static ground tiles is added. Call before
 * b3_write_bodies; *numBodiesOut = bodies added. The whole file is read and
 * checked before anything is registered: a file that fails (truncated or
 * inconsistent records, a degenerate hull, a hull record of more than 65,536
 * points, more bodies than the world's capacity) returns an error and leaves
 * the world as it was. */
int b3_load_bullet_file(b3World w, const char* path, int keepStaticObjects, int* numBodiesOut);

/* Flags of b3_load_bullet_file_ex. */
enum {
    B3_BULLET_KEEP_STATIC_OBJECTS = 1, /* keepStaticObjects of b3_load_bullet_file */
    /* also convert sphere shapes (radius = implicitShapeDimensions.x *
     * localScaling.x) and static plane shapes (n . x = constant) into this
     * library's sphere and plane shapes, where the reference's extractor
     * skips them (createSphereShape / createPlaneShape return -1,
     * P2/BulletDataExtractor.cpp:999-1010); their bodies register like the
     * others. A plane body is static, so it is kept only with
     * B3_BULLET_KEEP_STATIC_OBJECTS. */
    B3_BULLET_SPHERES_AND_PLANES = 2
};
/* b3_load_bullet_file with flags (B3_BULLET_*); flags 0 or
 * B3_BULLET_KEEP_STATIC_OBJECTS give exactly b3_load_bullet_file. */
int b3_load_bullet_file_ex(b3World w, const char* path, int flags, int* numBodiesOut);

/* Bulk form of b3_register_body for n bodies (arrays of n, xyz / xyzw
 * packed); writes the id of the first new body. */
int b3_register_bodies(b3World w, int n, const float* masses, const float* positions3,
                       const float* orientations4, const int* collidables, const float* frictions,
                       const float* restitutions, const int* worldIds, int* firstBodyOut);

/* Upload all registered bodies, inertias and collidables
 * (CLPhysicsDemo::writeBodiesToGpu P2/CLPhysicsDemo.cpp:205-216). */
int b3_write_bodies(b3World w, void* stream);
/* Bulk velocity write (CLPhysicsDemo::setObjectLinearVelocity generalised):
 * xyz triples for each body, NULL to leave unchanged. Host pointers. */
int b3_write_velocities(b3World w, const float* linVel3, const float* angVel3, void* stream);

/* CLPhysicsDemo::stepSimulation (P2/CLPhysicsDemo.cpp:740-943): AABB+hash,
 * sort, cell start, pair search, gravity, SAT+clip+reduce, constraint
 * setup, Jacobi solve with velocity averaging, integrate; n steps. */
int b3_step(b3World w, int numSteps, void* stream);

/* Read bodies back in the reference Body layout (host, synchronising);
 * before the first b3_write_bodies, the records as registered. Reports
 * B3_ERR_TIMEOUT as b3_read_state does. */
int b3_read_bodies(b3World w, b3Body* out, int maxBodies, void* stream);
/* Read SoA state (host float4 arrays, NULL to skip; synchronising).
 * Returns B3_ERR_TIMEOUT (arrays filled) when a bounded device wait has
 * given up since the last b3_reset_counters: the state is not valid. */
int b3_read_state(b3World w, float* pos4, float* quat4, float* linVel4, float* angVel4, void* stream);
/* Write SoA state (host float4 arrays, NULL to skip). Asynchronous on the
 * stream: pinned host buffers are read when the stream reaches the copies
 * and must stay unchanged until then; pageable buffers are staged before
 * the call returns. */
int b3_write_state(b3World w, const float* pos4, const float* quat4, const float* linVel4,
                   const float* angVel4, void* stream);
int b3_get_num_bodies(b3World w, int* n);
/* Step diagnostics (synchronising). Returns B3_ERR_TIMEOUT, with *out
 * filled and out->timeouts >= 1, when a bounded device wait has given up
 * since the last b3_reset_counters; the step results since are not valid.
 * The error stays set (later solves stop at their first grid barrier) until
 * b3_reset_counters. */
int b3_get_counters(b3World w, b3Counters* out, void* stream);
/* Bounded waits of the persistent Jacobi solve (its grid barriers): a
 * waiter gives up after spinLimit polls (0 = the default, 4,194,304 polls
 * of about 64 ns each). holdMicros > 0 makes block 0 of the solve arrive at
 * its first grid barrier that many microseconds late, which, with a small
 * spinLimit, exercises the give-up path (tests only; at most 1 s).
 * No reference counterpart: the reference's waits are clFinish calls. */
int b3_set_wait_limits(b3World w, int spinLimit, int holdMicros);
int b3_reset_counters(b3World w, void* stream);

/* --- stage entry points (each one stage of stepSimulation) --- */
/* setupGpuAabbsFull + gravity (BB/broadphaseKernel.cl:293-331,163-213). */
int b3_stage_aabbs(b3World w, void* stream);
/* btGridBroadphaseCl::calculateOverlappingPairs (BB/btGridBroadphaseCL.cpp:135-238):
 * hash, radix sort, cell start, 27-cell + large-body pair search, compaction. */
int b3_stage_broadphase(b3World w, void* stream);
/* btGpuNarrowphaseAndSolver::computeContacts (P1/...cpp:873-1070) via
 * GpuSatCollision::computeConvexConvexContactsGPUSAT (P2/ConvexHullContact.cpp:1793). */
int b3_stage_narrowphase(b3World w, void* stream);
/* btPgsJacobiSolver::solveGroup (P2/btPgsJacobiSolver.cpp:195-215):
 * setup, iterations with velocity averaging, finish. */
int b3_stage_solve(b3World w, void* stream);
/* integrateTransformsKernel2 (BB/integrateKernel.cl:102-158). */
int b3_stage_integrate(b3World w, void* stream);

/* --- the same stages under the reference object API's names --- */
/* btGridBroadphaseCl::calculateOverlappingPairs (BB/btGridBroadphaseCL.cpp:135-238);
 * same as b3_stage_broadphase (uses the AABBs of b3_stage_aabbs). */
int b3_grid_broadphase_calculate_overlapping_pairs(b3World w, void* stream);
/* btGridBroadphaseCl::getNumOverlap (BB/btGridBroadphaseCL.h:48-51):
 * pairs found by the last broadphase (synchronising). */
int b3_grid_broadphase_get_pair_count(b3World w, int* count, void* stream);
/* btGpuNarrowphaseAndSolver::computeContacts(pairs, nPairs, aabbs, nObjects)
 * (P1/btGpuNarrowPhaseAndSolver.h:101): contacts for caller-provided device
 * pairs (int2 (self, other), numPairs <= maxPairs; copied into the world's
 * pair buffer), or for the world's own broadphase pairs when d_pairs is
 * NULL. Also builds the manifold list the solver consumes. */
int b3_narrowphase_compute_contacts(b3World w, const int32_t* d_pairs, int numPairs, void* stream);
/* btPgsJacobiSolver::solveContacts (P2/btPgsJacobiSolver.cpp:171-189) on the
 * device: same as b3_stage_solve. */
int b3_solver_solve_jacobi(b3World w, void* stream);
/* Solver::batchContacts + convertToConstraints + solveContactConstraint
 * (ST/Solver.cpp:561-761, 842-925) for a world created with
 * B3_WORLD_BATCHED_GS_SOLVER: same as b3_stage_solve of such a world. */
int b3_solver_solve_batched_gs(b3World w, void* stream);
/* integrateTransformsKernel2 (BB/integrateKernel.cl:102-158): same as
 * b3_stage_integrate. */
int b3_integrate(b3World w, void* stream);

/* --- stage outputs (host copies, synchronising) --- */
/* Batched Gauss-Seidel solver: per manifold (manifold order of
 * b3_get_contacts) its cell (x + 16 z) and batch, 2 ints each, and its
 * Constraint4 after the last solve (applied impulses included). */
int b3_get_gs_batches(b3World w, int32_t* cellBatch2, int max, int* count, void* stream);
int b3_get_gs_constraints(b3World w, b3Constraint4* out, int max, int* count, void* stream);
/* World AABBs, 2 float4 per body (min.w = body id bits, max.w = dynamic flag). */
int b3_get_aabbs(b3World w, float* out8, int maxBodies, void* stream);
/* Sorted (cell key, body id) of the small bodies; returns count. */
int b3_get_sorted_hash(b3World w, uint32_t* keys, uint32_t* values, int max, int* count, void* stream);
/* Broadphase pairs (x = self, y = other); returns count. */
int b3_get_pairs(b3World w, int32_t* pairs2, int max, int* count, void* stream);
/* Contact manifolds in pair order; returns count. */
int b3_get_contacts(b3World w, b3Contact4* out, int max, int* count, void* stream);
/* Shape tables after registration (for checking / interop). */
int b3_get_shape_sizes(b3World w, int* numCollidables, int* numPolys, int* numVertices,
                       int* numFaces, int* numIndices, int* numEdges);
int b3_get_shapes(b3World w, b3Collidable* cols, b3ConvexPolyhedron* polys, float* vertices4,
                  b3Face* faces, int* indices, float* edges4, float* localAabbs8);
/* The compounds' child shapes (all of them, in registration order);
 * *count = their number. */
int b3_get_child_shapes(b3World w, b3ChildShape* out, int max, int* count);
int b3_get_inertias(b3World w, b3Inertia* out, int maxBodies);

/* --- device buffers (borrowed views, like getBodiesGpu / getContactsGpu,
 *     P1/btGpuNarrowPhaseAndSolver.h:104-111) --- */
enum {
    B3_BUF_POS = 0, B3_BUF_QUAT = 1, B3_BUF_LINVEL = 2, B3_BUF_ANGVEL = 3,
    B3_BUF_AABB_MIN = 4, B3_BUF_AABB_MAX = 5, B3_BUF_PAIRS = 6, B3_BUF_CONTACTS = 7,
    B3_BUF_COUNTERS = 8, B3_BUF_INVMASS = 9
};
int b3_get_device_buffer(b3World w, int which, void** d_ptr, int64_t* bytes);

/* CUDA-event timing of each stage of the last timed step (ms): 13 values,
 * the 7 stages (AABB + hash, cell sort, pair search, narrowphase, manifolds,
 * solve, integrate), the narrowphase's 4 kernels (separating-axis sweep,
 * float-float ranking, FP32 clip, float-float path), then the Jacobi
 * solve's row setup and its iterations (0 for the Gauss-Seidel solver). */
int b3_set_stage_timing(b3World w, int enable);
int b3_get_stage_times(b3World w, float* ms, int max, int* count);

/* ------------------------------------------------------------------ */
/* Batched worlds: thousands of independent worlds in one launch per    */
/* stage. World ids go into the high bits of the cell keys, pair and    */
/* contact arrays are segmented by world. Configure with numWorlds > 1  */
/* in b3WorldConfig and pass worldId to b3_register_body.               */
/* ------------------------------------------------------------------ */
/* Per-world aggregate: centre of mass and kinetic energy, 4 floats per
 * world (x, y, z, KE) computed on device; host output. */
int b3_batch_world_stats(b3World w, float* out4, int numWorlds, void* stream);
/* Body-count prefix sums per world: offsets[k+1] - offsets[k] bodies carry
 * worldId k (numWorlds + 1 entries; bodies registered in world order occupy
 * [offsets[k], offsets[k+1])). offsets NULL = query numWorlds only. Used to
 * partition worlds across GPUs by body count. */
int b3_batch_world_offsets(b3World w, int* offsets, int maxWorlds, int* numWorlds);
/* Autotuner over the launch shapes of the tunable kernels on the current
 * scene: the narrowphase warps per CTA (1/2/4) and the lane-group form by
 * trials of trialSteps eager steps from the same saved state; then the grid
 * pair search form
 * (thread or warp per body), each timed on three searches over the same
 * sorted keys; then the Jacobi launch shapes
 * jointly, every combination of CTA size (64/128/256), persistent blocks
 * per SM (1/2/4/8), body-average gather (one-at-a-time / four-wide) and,
 * for batched worlds, mode (grid-barrier / block-per-world), each timed on
 * three solves of the same contacts (the knobs interact, so they are not
 * tuned one at a time). With the batched Gauss-Seidel solver its grid width
 * is tuned by step trials instead. Timing uses CUDA events; the fastest
 * shapes are kept, the body state and counters are restored, and the step
 * graph is recaptured on the next b3_step. Synchronises the stream. */
int b3_autotune(b3World w, int trialSteps, void* stream);
/* values: narrowphase warps per CTA, pair-search CTA size, solver CTA size,
 * kernel launches per step of the captured step graph (0 before capture),
 * Jacobi blocks per SM cap, configurations timed by the autotuner, Jacobi
 * mode (0 = persistent grid with grid barriers, 1 = one block per world
 * with block barriers; batched worlds only, bit-identical results), Jacobi
 * body-average gather (0 = one copy at a time, 1 = four loads in flight;
 * bit-identical results), grid pair search form (0 = one thread per body
 * over its 27 cells, 1 = one warp per body, a lane per cell; the same pair
 * list and overflow counts bit for bit), narrowphase lane groups (0 = one
 * warp per pair in the FP32 clip and the float-float stages, 1 = eight-lane
 * groups there, four pairs per warp, with the warp form for pairs that do
 * not fit a group's 16-vertex tables or 8 candidates; bit-identical
 * results). */
int b3_get_tuning(b3World w, int* values, int max, int* count);
/* Set the tunables in b3_get_tuning's order (count >= 3; the pair-search
 * CTA size, the launch count and the trial count are read-only, indices 4,
 * 6, 7, 8 and 9 are optional):
 * narrowphase warps per CTA 1/2/4, Jacobi CTA size 64/128/256, Jacobi
 * blocks per SM cap 1..8, Jacobi mode 0/1, Jacobi gather 0/1, pair search
 * form 0/1, lane groups 0/1. */
int b3_set_tuning(b3World w, const int* values, int count);

/* ------------------------------------------------------------------ */
/* Adjoint (reverse mode)                                               */
/* ------------------------------------------------------------------ */
typedef struct b3Adjoint_t* b3Adjoint;

/* Forward run of numSteps steps with body-state checkpoints every
 * checkpointEvery steps; the backward pass recomputes each segment and
 * records its tape (contacts, active sets, clamp masks, iterates). */
int b3_adjoint_create(b3World w, int numSteps, int checkpointEvery, b3Adjoint* out);
int b3_adjoint_destroy(b3Adjoint a);
int b3_adjoint_forward(b3Adjoint a, void* stream);
/* Seed: dLoss/d(final state) as float4 arrays (host; NULL = zero). */
int b3_adjoint_backward(b3Adjoint a, const float* dPos4, const float* dQuat4, const float* dLinVel4,
                        const float* dAngVel4, void* stream);
/* Gradients w.r.t. initial linear/angular velocities (float4 per body),
 * masses and friction coefficients (float per body). Host outputs. */
int b3_adjoint_gradients(b3Adjoint a, float* dLinVel4, float* dAngVel4, float* dMass, float* dFriction);
/* Diagnostics of the last backward pass: contact points or axes that matched
 * no feature of the clip (differentiated as rigidly attached instead). */
int b3_adjoint_info(b3Adjoint a, int* unclassified);

#ifdef __cplusplus
}
#endif

#endif /* B3GPU_H */
