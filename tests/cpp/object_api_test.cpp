// Host program that drives the library through the C++ object API
// (include/b3gpu.hpp), the way a caller of the reference's objects would.
//
//   object_api_test host   registration and inspection on a host-only
//                          context; device calls must report NO_DEVICE
//   object_api_test gpu    primitives and a 120-step cube stack on device 0,
//                          stage by stage and through stepSimulation
//
// Prints "OK" and returns 0 when every check passes.
#include "b3gpu.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#define EXPECT(c)                                                              \
    do {                                                                       \
        if (!(c)) {                                                            \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #c);         \
            return 1;                                                          \
        }                                                                      \
    } while (0)

static const float kCube[8][4] = {{-0.5f, -0.5f, -0.5f, 0}, {0.5f, -0.5f, -0.5f, 0}, {-0.5f, 0.5f, -0.5f, 0},
                                  {0.5f, 0.5f, -0.5f, 0},   {-0.5f, -0.5f, 0.5f, 0}, {0.5f, -0.5f, 0.5f, 0},
                                  {-0.5f, 0.5f, 0.5f, 0},   {0.5f, 0.5f, 0.5f, 0}};

// A static 40 x 1 x 40 ground box and a 4 x 4 x 4 stack of unit cubes.
static int build_stack(b3::World& w) {
    const float groundScale[3] = {40.f, 1.f, 40.f};
    const float one[3] = {1.f, 1.f, 1.f};
    const int ground = w.registerConvexPolyhedron(&kCube[0][0], 8, 16, groundScale);
    const int cube = w.registerConvexPolyhedron(&kCube[0][0], 8, 16, one);
    const float q[4] = {0, 0, 0, 1};
    const float g[3] = {0, -0.5f, 0};
    w.registerPhysicsInstance(0.f, g, q, ground, 0.6f);
    for (int y = 0; y < 4; ++y)
        for (int z = 0; z < 4; ++z)
            for (int x = 0; x < 4; ++x) {
                const float p[3] = {(x - 1.5f) * 1.05f, 0.5f + y * 1.05f, (z - 1.5f) * 1.05f};
                w.registerPhysicsInstance(1.f, p, q, cube, 0.6f);
            }
    return 65;
}

static b3WorldConfig stack_config() {
    b3WorldConfig cfg = b3::World::defaultConfig();
    cfg.gridDims[0] = cfg.gridDims[1] = cfg.gridDims[2] = 16;
    cfg.cellSize = 1.f;
    cfg.maxSmallProxySize = 4.f;
    return cfg;
}

static int host_mode(const char* bulletFile) {
    b3::Context ctx(-1);
    if (bulletFile) {
        // createScene's file path: the shapes and bodies of a .bullet scene
        b3WorldConfig cfg = stack_config();
        cfg.maxBodies = 64;
        b3::World wf(ctx, cfg);
        EXPECT(wf.loadBulletFile(bulletFile, true) == 41 && wf.numBodies() == 41);
    }
    {
        // the other shape kinds: sphere, plane, a compound of two cubes, a
        // two-triangle mesh; each is a collidable of its reference shape type
        b3::World ws(ctx, stack_config());
        const float one[3] = {1.f, 1.f, 1.f};
        const int cube = ws.registerConvexPolyhedron(&kCube[0][0], 8, 16, one);
        const int sphere = ws.registerSphereShape(0.5f);
        const float up[3] = {0.f, 1.f, 0.f};
        const int plane = ws.registerPlaneShape(up, 0.f);
        b3ChildShape kids[2] = {};
        kids[0].childPosition[0] = 0.55f;
        kids[1].childPosition[0] = -0.55f;
        kids[0].childOrientation[3] = kids[1].childOrientation[3] = 1.f;
        kids[0].shapeIndex = kids[1].shapeIndex = cube;
        const int compound = ws.registerCompoundShape(kids, 2);
        const float sq[12] = {-5, 0, 5, 5, 0, 5, -5, 0, -5, 5, 0, -5};
        const int tris[6] = {0, 1, 2, 2, 1, 3};
        const int mesh = ws.registerConcaveMesh(sq, 4, tris, 6);
        std::vector<b3Collidable> cols(8);
        EXPECT(b3_get_shapes(ws.handle(), cols.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == 0);
        EXPECT(cols[sphere].shapeType == B3_SHAPE_SPHERE && cols[sphere].radius == 0.5f);
        EXPECT(cols[plane].shapeType == B3_SHAPE_PLANE);
        EXPECT(cols[compound].shapeType == B3_SHAPE_COMPOUND_OF_CONVEX_HULLS && cols[compound].numChildShapes == 2);
        EXPECT(cols[mesh].shapeType == B3_SHAPE_CONCAVE_TRIMESH && cols[mesh].numChildShapes == 2);
        ws.setWaitLimits(1000);
        ws.setWaitLimits(0);
    }
    b3::World w(ctx, stack_config());
    EXPECT(build_stack(w) == w.numBodies());
    b3::GpuNarrowphaseAndSolver np(w);
    bool threw = false;
    try {
        np.writeAllBodiesToGpu();
    } catch (const b3::Error& e) {
        threw = e.code() == B3_ERR_NO_DEVICE;
    }
    EXPECT(threw);
    return 0;
}

static int gpu_mode() {
    b3::Context ctx(0);
    // --- primitives ---
    const int n = 1 << 20;
    std::mt19937 rng(7);
    std::vector<uint32_t> keys(n), vals(n);
    for (int i = 0; i < n; ++i) {
        keys[i] = rng() & 0xFFFFF;
        vals[i] = i;
    }
    uint32_t *dk = nullptr, *dv = nullptr, *ds = nullptr;
    EXPECT(cudaMalloc(&dk, n * 4) == cudaSuccess && cudaMalloc(&dv, n * 4) == cudaSuccess &&
           cudaMalloc(&ds, n * 4) == cudaSuccess);
    cudaMemcpy(dk, keys.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, vals.data(), n * 4, cudaMemcpyHostToDevice);
    b3::RadixSort32 sort(ctx);
    sort.execute(dk, dv, n, 20);
    std::vector<uint32_t> sk(n), sv(n);
    cudaMemcpy(sk.data(), dk, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(sv.data(), dv, n * 4, cudaMemcpyDeviceToHost);
    std::vector<uint32_t> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    for (int i = 0; i < n; ++i) EXPECT(sv[i] == order[i] && sk[i] == keys[order[i]]);
    b3::Fill fill(ctx);
    fill.execute(ds, 3u, n);
    b3::PrefixScan scan(ctx);
    uint32_t total = 0;
    scan.execute(ds, ds, n, &total);
    EXPECT(total == 3u * n);
    uint32_t last = 0;
    cudaMemcpy(&last, ds + n - 1, 4, cudaMemcpyDeviceToHost);
    EXPECT(last == 3u * (n - 1));
    b3::BoundSearch bs(ctx);
    bs.execute(dk, n, ds, 1 << 20, b3::BoundSearch::COUNT);
    std::vector<uint32_t> cnt(1 << 20);
    cudaMemcpy(cnt.data(), ds, 4 << 20, cudaMemcpyDeviceToHost);
    uint64_t sum = 0;
    for (uint32_t c : cnt) sum += c;
    EXPECT(sum == (uint64_t)n);
    // btSortData form: the same keys and values interleaved, sorted in place,
    // then bound-searched; and the out-of-place four-array form
    std::vector<b3::SortData> kv(n);
    for (int i = 0; i < n; ++i) kv[i] = {(int)keys[i], (int)vals[i]};
    b3::SortData* dkv = nullptr;
    uint32_t *dko = nullptr, *dvo = nullptr, *dlo = nullptr;
    EXPECT(cudaMalloc(&dkv, n * 8) == cudaSuccess && cudaMalloc(&dko, n * 4) == cudaSuccess &&
           cudaMalloc(&dvo, n * 4) == cudaSuccess && cudaMalloc(&dlo, 4 << 20) == cudaSuccess);
    cudaMemcpy(dkv, kv.data(), n * 8, cudaMemcpyHostToDevice);
    sort.execute(dkv, n, 20);
    cudaMemcpy(kv.data(), dkv, n * 8, cudaMemcpyDeviceToHost);
    for (int i = 0; i < n; ++i) EXPECT((uint32_t)kv[i].m_key == sk[i] && (uint32_t)kv[i].m_value == sv[i]);
    bs.execute(dkv, n, dlo, 1 << 20, b3::BoundSearch::COUNT);
    std::vector<uint32_t> cnt2(1 << 20);
    cudaMemcpy(cnt2.data(), dlo, 4 << 20, cudaMemcpyDeviceToHost);
    EXPECT(cnt2 == cnt);
    cudaMemcpy(dk, keys.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, vals.data(), n * 4, cudaMemcpyHostToDevice);
    sort.execute(dk, dko, dv, dvo, n, 20);
    std::vector<uint32_t> ok(n), ov(n), ik(n);
    cudaMemcpy(ok.data(), dko, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(ov.data(), dvo, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(ik.data(), dk, n * 4, cudaMemcpyDeviceToHost);
    EXPECT(ok == sk && ov == sv && ik == keys);
    cudaFree(dkv);
    cudaFree(dko);
    cudaFree(dvo);
    cudaFree(dlo);
    cudaFree(dk);
    cudaFree(dv);
    cudaFree(ds);

    // --- stage by stage, through the reference-named objects ---
    b3::World w(ctx, stack_config());
    build_stack(w);
    b3::GridBroadphase bp(w);
    b3::GpuNarrowphaseAndSolver np(w);
    np.writeAllBodiesToGpu();
    w.computeAabbs();
    bp.calculateOverlappingPairs();
    const int pairs = bp.getNumOverlap();
    EXPECT(pairs >= 16);
    np.computeContacts();
    np.solveContacts();
    np.integrate();
    EXPECT(np.getNumContactsGpu() >= 16);  // the bottom layer touches the ground

    // --- stepSimulation ---
    w.stepSimulation(120);
    std::vector<b3Body> bodies = w.readBodies();
    float minY = 1e9f, maxSpeed = 0.f;
    for (size_t i = 1; i < bodies.size(); ++i) {
        minY = std::min(minY, bodies[i].pos[1]);
        const float* v = bodies[i].linVel;
        maxSpeed = std::max(maxSpeed, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
    EXPECT(minY > 0.4f);        // resting on the ground, not through it
    EXPECT(maxSpeed < 0.5f);    // settled
    b3Counters c = w.counters();
    EXPECT(c.timeouts == 0 && c.pairOverflow == 0);

    // --- the sweep-and-prune broadphase (pipeline2's default) ---
    b3WorldConfig sapCfg = stack_config();
    sapCfg.flags = B3_WORLD_SAP_BROADPHASE;
    b3::World ws(ctx, sapCfg);
    build_stack(ws);
    b3::GpuSapBroadphase sap(ws);
    b3::GpuNarrowphaseAndSolver nps(ws);
    nps.writeAllBodiesToGpu();
    ws.computeAabbs();
    sap.calculateOverlappingPairs();
    EXPECT(sap.getNumOverlap() == pairs);  // the same stack, the same overlaps
    ws.stepSimulation(120);
    std::vector<b3Body> sb = ws.readBodies();
    float sapMinY = 1e9f;
    for (size_t i = 1; i < sb.size(); ++i) sapMinY = std::min(sapMinY, sb[i].pos[1]);
    EXPECT(sapMinY > 0.4f);

    // --- the reference's GPU solver (batched Gauss-Seidel) ---
    b3WorldConfig gsCfg = stack_config();
    gsCfg.flags = B3_WORLD_BATCHED_GS_SOLVER;
    b3::World wg(ctx, gsCfg);
    build_stack(wg);
    b3::GpuNarrowphaseAndSolver npg(wg);
    b3::BatchedSolver gs(wg);
    npg.writeAllBodiesToGpu();
    wg.computeAabbs();
    b3::GridBroadphase bpg(wg);
    bpg.calculateOverlappingPairs();
    npg.computeContacts();
    gs.solveContactConstraint();
    npg.integrate();
    const int nm = gs.getConstraints(nullptr, 0);
    EXPECT(nm >= 16);
    std::vector<b3Constraint4> cs(nm);
    std::vector<int32_t> cb(2 * (size_t)nm);
    EXPECT(gs.getConstraints(cs.data(), nm) == nm && gs.getBatches(cb.data(), nm) == nm);
    for (int m = 0; m < nm; ++m) {
        EXPECT(cs[m].batchIdx == cb[2 * m + 1] && cs[m].batchIdx >= 0);
        EXPECT(cs[m].jacCoeffInv[0] < 0.f && cs[m].linear[3] == 0.7f);
    }
    wg.stepSimulation(120);
    std::vector<b3Body> gb = wg.readBodies();
    float gsMinY = 1e9f;
    for (size_t i = 1; i < gb.size(); ++i) gsMinY = std::min(gsMinY, gb[i].pos[1]);
    EXPECT(gsMinY > 0.4f);
    EXPECT(wg.counters().timeouts == 0);
    return 0;
}

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    int rc = 1;
    try {
        rc = gpu ? gpu_mode() : host_mode(argc > 2 ? argv[2] : nullptr);
    } catch (const std::exception& e) {
        std::printf("FAILED: %s\n", e.what());
        return 1;
    }
    if (rc == 0) std::printf("OK\n");
    return rc;
}
