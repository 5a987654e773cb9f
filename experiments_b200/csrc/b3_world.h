// World object: host mirrors of the registered bodies and shapes, device
// buffers (structure-of-arrays, float4 streams), and the per-stage launchers.
#pragma once

#include "b3_internal.h"
#include "hull.h"

#include <vector>

namespace b3 {

// Device views passed by value to the kernels.
struct BodiesDev {
    int n;
    float4* pos;
    float4* quat;
    float4* linVel;
    float4* angVel;
    const float* invMass;
    const int* collidable;
    const float* friction;
    const float* restitution;
    const float4* invInertia;  // local diagonal inverse inertia (xyz)
    const int* worldId;
};

struct ShapesDev {
    const b3Collidable* cols;
    const b3ConvexPolyhedron* polys;
    const float4* verts;
    const b3Face* faces;
    const int* indices;
    const float4* edges;
    const float4* localAabb;  // 2 per collidable (min, max)
    const float* inradius;    // per polyhedron: lower bound of its support about localCenter
    const b3ChildShape* children;  // the compounds' children
    // the hulls' vertices two at a time for the packed FP32x2 projection:
    // pair j of polyhedron p at polyPack[p] + j holds (x0, x1, y0, y1) in
    // vpXY and (z0, z1) in vpZ (an odd count repeats the last vertex)
    const float4* vpXY;
    const float2* vpZ;
    const int* polyPack;
    int numPolys, numVerts, numFaces, numIndices, numEdges;
};

struct SimParams {
    float3 gravity;
    float dt;
    int iterations;
    float erp;
    float contactBreaking;
    float contactProcessing;
    float slopOffset;
    float angularDamping;
    int frictionCombine;
};

// Device buffers owned by a world.
struct DevBuffers {
    // bodies
    float4 *pos = nullptr, *quat = nullptr, *linVel = nullptr, *angVel = nullptr;
    float *invMass = nullptr, *friction = nullptr, *restitution = nullptr;
    float4* invInertia = nullptr;
    int *collidable = nullptr, *worldId = nullptr;
    // shapes
    b3Collidable* cols = nullptr;
    b3ConvexPolyhedron* polys = nullptr;
    float4* verts = nullptr;
    b3Face* faces = nullptr;
    int* indices = nullptr;
    float4* edges = nullptr;
    float4* localAabb = nullptr;
    float* polyInradius = nullptr;
    b3ChildShape* childShapes = nullptr;
    float4* vpXY = nullptr;  // vertex pairs (x0, x1, y0, y1)
    float2* vpZ = nullptr;   // vertex pairs (z0, z1)
    int* polyPack = nullptr; // per polyhedron: its first vertex pair
    // compound and mesh pairs: sub-pair records (body A, body B, side A,
    // side B; a side is a child shape >= 0 or -(polytope + 1)), per pair
    // counts and their exclusive scan
    int4* subPairs = nullptr;
    uint32_t* subCount = nullptr;
    uint32_t* subOffset = nullptr;
    // broadphase
    float4 *aabbMin = nullptr, *aabbMax = nullptr;
    int* smallSlot = nullptr;      // body -> slot in the hash arrays, -1 = large
    int* largeStart = nullptr;     // per world CSR over largeList
    int* largeList = nullptr;
    // sweep-and-prune broadphase (B3_WORLD_SAP_BROADPHASE)
    int* sapSmall = nullptr;          // dynamic bodies (small proxies), body order
    int* sapLarge = nullptr;          // static bodies (large proxies), body order
    float4* sapSorted = nullptr;      // small AABBs sorted by min x: (min, max) per proxy
    uint32_t* sapCount = nullptr;     // pairs per sorted proxy, then their offsets
    uint32_t* sapOffset = nullptr;
    uint32_t *keys = nullptr, *vals = nullptr, *keysAlt = nullptr, *valsAlt = nullptr;
    uint2* cellTable = nullptr;    // (stamp, first sorted index) per (world, cell)
    int2* pairs = nullptr;
    // narrowphase
    b3Contact4* contacts = nullptr;   // one slot per pair
    uint32_t* manifoldFlag = nullptr; // per pair: 1 if a manifold was emitted
    float4* pairSep = nullptr;        // per pair: FP32 separating axis of the sweep
    int* npFast = nullptr;            // queue: pairs whose axis the FP32 sweep decided
    int* npSlow = nullptr;            // queue: pairs for the float-float path
    int* npDefer = nullptr;           // queue: clip pairs the lane groups pass to the warp clip
    int* npDefer2 = nullptr;          // queue: slow-queue positions for the warp float-float stage
    int* npDefer3 = nullptr;          // queue: slow-queue positions for the warp ranking
    int* npCand = nullptr;            // near-minimum axes of queued pairs (kNpCandSlots x 32)
    uint32_t* manifoldScan = nullptr; // exclusive scan of the flags
    int* manifoldPair = nullptr;      // manifold -> pair slot
    // solver
    uint32_t *incKeys = nullptr, *incVals = nullptr, *incKeysAlt = nullptr, *incValsAlt = nullptr;
    uint32_t *bodyIncStart = nullptr, *bodyIncEnd = nullptr;
    float4* rows = nullptr;           // constraint rows, see solver.cu
    float4* manifoldHdr = nullptr;    // per manifold header
    float4 *incLin = nullptr, *incAng = nullptr;   // per manifold side increments
    float4 *avgLin = nullptr, *avgAng = nullptr;   // per body averaged delta velocity
    // scalars (device): [0] numSmall, [1] numPairs, [2] numManifolds, [3] numInc,
    // [4] stamp, [5] sort error flag, [6..7] barrier, [8] tile counter
    int32_t* scalars = nullptr;
    b3Counters* counters = nullptr;
    void* sortScratch = nullptr;
    size_t sortScratchBytes = 0;
    void* incSortScratch = nullptr;
    size_t incSortScratchBytes = 0;
    void* scanScratch = nullptr;
    size_t scanScratchBytes = 0;
    float4* worldStats = nullptr;
    int *worldMStart = nullptr, *worldMEnd = nullptr;  // per world: manifold range (batched solver)
    // batched Gauss-Seidel solver (B3_WORLD_BATCHED_GS_SOLVER); the
    // Constraint4 records live in the Jacobi row storage, which that solver
    // does not use
    int* gsCell = nullptr;            // per manifold: cell x + 16 z
    int* gsSlotBatch = nullptr;       // per sorted slot: batch
    int* gsSlotOfManifold = nullptr;  // per manifold: index of its Constraint4
    int* gsMinRank = nullptr;         // [4][bodies]
    int* gsTaken = nullptr;           // [4][bodies]
    int* gsBatchCount = nullptr;      // [4] batches per class, then 5 round counters
    uint32_t* gsGroupCount = nullptr; // [4 * kGsMaxBatch]
    uint32_t* gsGroupFill = nullptr;  // [4 * kGsMaxBatch]
    uint32_t* gsGroupOffset = nullptr;  // [4 * kGsMaxBatch + 1]
    float4* gsInertia = nullptr;      // [3][bodies] world inverse inertia rows
    b3Constraint4* gsConstraints = nullptr;
};

enum ScalarSlot {
    S_NUM_SMALL = 0,
    S_NUM_PAIRS = 1,
    S_NUM_MANIFOLDS = 2,
    S_NUM_INC = 3,
    S_STAMP = 4,
    S_ERR = 5,
    S_BAR_COUNT = 6,
    S_BAR_GEN = 7,
    S_TILE = 8,
    S_NP_WORK = 9,
    S_NP_FAST = 10,       // pairs queued for the FP32 clip
    S_NP_SLOW = 11,       // pairs queued for the float-float path
    S_NP_WORK2 = 12,
    S_NP_WORK3 = 13,
    S_NP_WORK4 = 14,
    S_NUM_SUB = 15,       // sub-pairs of compound and mesh pairs this step (after the capacity cut)
    S_NUM_SLOTS = 16,     // manifold slots: pairs, then sub-pairs
    S_SUB_TOTAL = 17,     // sub-pairs before the capacity cut
    S_NP_DEFER = 18,      // clip-queue pairs the lane-group clip passed to the warp clip
    S_NP_WORK5 = 19,
    S_NP_DEFER2 = 20,     // slow-queue positions the lane-group float-float clip passed to k_np_exact
    S_NP_WORK6 = 21,
    S_NP_DEFER3 = 22,     // slow-queue positions the lane-group ranking passed to k_np_refine
    S_NP_WORK7 = 23,
    S_NUM_SCALARS = 24
};

}  // namespace b3

struct b3World_t {
    b3Context ctx = nullptr;
    b3WorldConfig cfg{};
    int cellBits = 0, worldBits = 0, keyBits = 0, bodyBits = 0;
    float invCell = 1.f;

    // host mirrors
    std::vector<b3Body> bodies;
    std::vector<b3Inertia> inertias;
    std::vector<b3Collidable> cols;
    std::vector<b3ConvexPolyhedron> polys;
    std::vector<float> verts4, edges4, localAabb8;
    std::vector<float> polyInradius;
    std::vector<float> vpXY, vpZ;  // vertex pairs, built at upload
    std::vector<int> polyPack;
    std::vector<b3ChildShape> childShapes;  // children of the compounds
    int numSpheres = 0, numPlanes = 0, numCompounds = 0, numMeshes = 0;
    bool hasSpheresPlanes() const { return numSpheres > 0 && (numSpheres > 1 || numPlanes > 0); }
    bool hasSubPairs() const { return numCompounds + numMeshes > 0; }
    std::vector<b3Face> faces;
    std::vector<int> indices;
    std::vector<int> worldIds;
    std::vector<float> regAabb;   // registration AABB per body (6 floats)
    std::vector<int> smallSlotHost, largeStartHost, largeListHost;
    int numSmall = 0;
    bool sap = false;    // sweep-and-prune broadphase in place of the grid
    bool gs = false;     // batched Gauss-Seidel solver in place of Jacobi
    std::vector<int> sapSmallHost, sapLargeHost;
    int capBodies = 0;   // allocated body capacity on device
    int capInc = 0;
    bool written = false;
    bool shapesDirty = true;

    b3::DevBuffers d;
    b3::SimParams sim{};

    // CUDA graph of one step
    cudaGraphExec_t graphExec = nullptr;
    cudaStream_t graphStream = nullptr;
    bool graphValid = false;

    // stage timing; with it on, the narrowphase also records one event
    // after each of its four kernels (npEv[0] before the sweep) and the
    // Jacobi solve one after its row setup (setupEv)
    bool timing = false;
    std::vector<float> stageMs;
    cudaEvent_t npEv[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t setupEv = nullptr;

    // tunables (autotuner)
    int npWarpsPerBlock = 4;   // narrowphase warps per CTA
    int kernelsPerStep = 0;    // kernel nodes in the captured step graph
    int pairThreads = 128;     // pair-search CTA size
    int solverThreads = 256;   // Jacobi CTA size
    int solverOccCap = 4;      // Jacobi persistent blocks per SM (at most)
    int solverMode = 0;        // Jacobi: 0 = grid barriers, 1 = one block per world (batched);
                               // batched Gauss-Seidel: grid width 0 = manifolds / 8, 1 = manifolds / 64
    int solverGather = 0;      // Jacobi body averages: 0 = one copy at a time, 1 = four loads in flight
    int pairSearchMode = 0;    // grid pair search: 0 = thread per body, 1 = warp per body
    int clipGroups = 1;        // clip and float-float stages: 0 = a warp per pair, 1 = 8-lane groups
                               // (a warp per pair for what does not fit)
    int tunedTrials = 0;       // configurations the autotuner timed
    int npSmemAttr = 0;        // dynamic shared memory attribute set on the narrowphase kernels
    int npGroupSmemAttr = 0;   // the same for the lane-group clip
    int npFFSmemAttr = 0;      // and for the lane-group float-float stages

    int cooperativeOk = 1;

    // bounded waits of the persistent Jacobi kernel (b3_set_wait_limits)
    int waitSpinLimit = b3::kDefaultSpinLimit;
    int waitHoldMicros = 0;

    b3::BodiesDev bodiesDev() const;
    b3::ShapesDev shapesDev() const;
};

namespace b3 {
// slots of the narrowphase candidate store (pairs queued for float-float
// axis ranking beyond this recompute their FP32 sweep)
constexpr int kNpCandSlots = 1 << 20;
constexpr int kGsMaxBatch = 1024;  // batches per parity class (batched Gauss-Seidel)

// Record of one Jacobi solve for the reverse sweep: every phase's solver-body
// copies (both sides of every manifold) and the row impulses after it.
struct JacobiTape {
    float4* copyLin;   // [2 * iterations][2 sides][maxPairs]
    float4* copyAng;
    float4* lamN;      // [iterations][maxPairs]: normal rows 0..3 after each normal phase
    float4* lamF;      // [iterations][2][maxPairs]: friction rows 0..7 after each friction phase
};

// stage launchers (world.cu / broadphase.cu / narrowphase.cu / solver.cu)
int launch_aabb_hash(b3World_t* w, cudaStream_t st);
int launch_sort_and_cells(b3World_t* w, cudaStream_t st);
int launch_find_pairs(b3World_t* w, cudaStream_t st);
// sweep-and-prune counterparts (sap.cu), called by the two above in SAP mode
int launch_sap_sort(b3World_t* w, cudaStream_t st);
int launch_sap_pairs(b3World_t* w, cudaStream_t st);
int launch_narrowphase(b3World_t* w, cudaStream_t st);
int launch_manifolds(b3World_t* w, cudaStream_t st);
int launch_solver(b3World_t* w, cudaStream_t st);
int launch_solver_taped(b3World_t* w, cudaStream_t st, const JacobiTape* tape);
int launch_integrate(b3World_t* w, cudaStream_t st);
int launch_gs_solver(b3World_t* w, cudaStream_t st);
int launch_world_stats(b3World_t* w, cudaStream_t st);
// one eager step (world.cu); tape may be null
int run_step(b3World_t* w, cudaStream_t st, const JacobiTape* tape);
}  // namespace b3
