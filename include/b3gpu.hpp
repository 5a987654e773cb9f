/* C++ object API over the C ABI of b3gpu.h, with classes named after the
 * reference pipeline's objects so that host code written against them maps
 * one to one:
 *
 *   b3::Context                  the (cl_context, cl_device_id, cl_command_queue)
 *                                triple the reference objects take
 *   b3::RadixSort32              btRadixSort32CL        (BB/btRadixSort32CL.h:63)
 *   b3::PrefixScan               btPrefixScanCL         (BB/btPrefixScanCL.h:29)
 *   b3::Fill                     btFillCL               (BB/btFillCL.h)
 *   b3::BoundSearch              btBoundSearchCL        (BB/btBoundSearchCL.h:56)
 *   b3::World                    CLPhysicsDemo          (P2/CLPhysicsDemo.cpp:603-943):
 *                                registration, writeBodiesToGpu, stepSimulation
 *   b3::GridBroadphase           btGridBroadphaseCl     (BB/btGridBroadphaseCL.h:54-63)
 *   b3::GpuSapBroadphase         btGpuSapBroadphase     (P2/btGpuSapBroadphase.h)
 *   b3::GpuNarrowphaseAndSolver  btGpuNarrowphaseAndSolver (P1/btGpuNarrowPhaseAndSolver.h:82-111)
 *
 * Device buffers are raw CUDA device pointers (the reference's cl_mem);
 * streams are cudaStream_t passed as void* (0 = the default stream). Calls
 * that fail throw b3::Error carrying the status code and b3_last_error();
 * nothing throws across the C ABI itself.
 */
#pragma once

#include "b3gpu.h"

#include <stdexcept>
#include <string>
#include <vector>

namespace b3 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& where)
        : std::runtime_error(where + ": status " + std::to_string(code) + " (" +
                             (b3_last_error() ? b3_last_error() : "") + ")"),
          code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc, const char* where) {
    if (rc != B3_OK) throw Error(rc, where);
}

class Context {
public:
    /* device >= 0: that CUDA device; -1: host-only (registration and
     * inspection work, device calls report B3_ERR_NO_DEVICE). */
    explicit Context(int device = 0) { check(b3_context_create(device, &h_), "b3_context_create"); }
    ~Context() {
        if (h_) b3_context_destroy(h_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    b3Context handle() const { return h_; }
    void sync(void* stream = nullptr) { check(b3_sync(h_, stream), "b3_sync"); }

private:
    b3Context h_ = nullptr;
};

/* btRadixSort32CL::execute(keyValues, sortBits): stable LSD sort of
 * (key, value) pairs by the low sortBits bits of the key. */
/* btSortData (BB/btRadixSort32CL.h:7-11): one (key, value) record of the
 * sorts and bound searches, 8 bytes. */
struct SortData {
    int m_key;
    int m_value;
};
static_assert(sizeof(SortData) == 8, "btSortData is 8 bytes");

class RadixSort32 {
public:
    explicit RadixSort32(Context& ctx) : ctx_(ctx) {}
    void execute(uint32_t* d_keys, uint32_t* d_values, int64_t n, int sortBits = 32, void* stream = nullptr) {
        check(b3_radix_sort32_kv(ctx_.handle(), d_keys, d_values, n, sortBits, stream), "RadixSort32::execute");
    }
    void executeKeys(uint32_t* d_keys, int64_t n, int sortBits = 32, void* stream = nullptr) {
        check(b3_radix_sort32_keys(ctx_.handle(), d_keys, n, sortBits, stream), "RadixSort32::executeKeys");
    }
    /* execute(keysIn, keysOut, valuesIn, valuesOut, n, sortBits): out of place. */
    void execute(const uint32_t* d_keysIn, uint32_t* d_keysOut, const uint32_t* d_valuesIn, uint32_t* d_valuesOut,
                 int64_t n, int sortBits = 32, void* stream = nullptr) {
        check(b3_radix_sort32_kv_out(ctx_.handle(), d_keysIn, d_keysOut, d_valuesIn, d_valuesOut, n, sortBits, stream),
              "RadixSort32::execute");
    }
    /* execute(keyValuesInOut, sortBits): n btSortData records in place. */
    void execute(SortData* d_keyValues, int64_t n, int sortBits = 32, void* stream = nullptr) {
        check(b3_radix_sort32_sortdata(ctx_.handle(), reinterpret_cast<int32_t*>(d_keyValues), n, sortBits, stream),
              "RadixSort32::execute");
    }

private:
    Context& ctx_;
};

/* btPrefixScanCL::execute(src, dst, n, sum): exclusive scan; *sum (host,
 * optional) receives the total. */
class PrefixScan {
public:
    explicit PrefixScan(Context& ctx) : ctx_(ctx) {}
    void execute(const uint32_t* d_src, uint32_t* d_dst, int64_t n, uint32_t* sum = nullptr,
                 void* stream = nullptr) {
        check(b3_prefix_scan_u32(ctx_.handle(), d_src, d_dst, n, nullptr, sum, stream), "PrefixScan::execute");
    }

private:
    Context& ctx_;
};

/* btFillCL::execute(buffer, value, n, offset). */
class Fill {
public:
    explicit Fill(Context& ctx) : ctx_(ctx) {}
    void execute(uint32_t* d_dst, uint32_t value, int64_t n, int64_t offset = 0, void* stream = nullptr) {
        check(b3_fill_u32(ctx_.handle(), d_dst, value, n, offset, stream), "Fill::execute");
    }
    void execute(int32_t* d_dst_int2, int32_t x, int32_t y, int64_t n, int64_t offset = 0, void* stream = nullptr) {
        check(b3_fill_int2(ctx_.handle(), d_dst_int2, x, y, n, offset, stream), "Fill::execute");
    }

private:
    Context& ctx_;
};

/* btBoundSearchCL::execute(src, nSrc, dst, nDst, option). */
class BoundSearch {
public:
    enum Option { BOUND_LOWER = 0, BOUND_UPPER = 1, COUNT = 2 };
    explicit BoundSearch(Context& ctx) : ctx_(ctx) {}
    void execute(const uint32_t* d_sortedKeys, int64_t nSrc, uint32_t* d_dst, int64_t nDst, Option option,
                 void* stream = nullptr) {
        check(b3_bound_search(ctx_.handle(), d_sortedKeys, nSrc, d_dst, nDst, (int)option, stream),
              "BoundSearch::execute");
    }
    /* execute(src, nSrc, dst, nDst, option) over btSortData records. */
    void execute(const SortData* d_src, int64_t nSrc, uint32_t* d_dst, int64_t nDst, Option option = BOUND_LOWER,
                 void* stream = nullptr) {
        check(b3_bound_search_sortdata(ctx_.handle(), reinterpret_cast<const int32_t*>(d_src), nSrc, d_dst, nDst,
                                       (int)option, stream),
              "BoundSearch::execute");
    }

private:
    Context& ctx_;
};

/* The rigid-body world: CLPhysicsDemo's registration and stepSimulation. */
class World {
public:
    World(Context& ctx, const b3WorldConfig& cfg) { check(b3_world_create(ctx.handle(), &cfg, &h_), "b3_world_create"); }
    static b3WorldConfig defaultConfig() {
        b3WorldConfig c;
        b3_world_config_default(&c);
        return c;
    }
    ~World() {
        if (h_) b3_world_destroy(h_);
    }
    World(const World&) = delete;
    World& operator=(const World&) = delete;
    b3World handle() const { return h_; }

    /* CLPhysicsDemo::registerConvexPolyhedron: returns the collidable id. */
    /* createScene's file path (P2/BulletDataExtractor.cpp:456-721): the
     * shapes and rigid bodies of a .bullet file (b3_load_bullet_file);
     * returns the bodies added. */
    int loadBulletFile(const char* path, bool keepStaticObjects = false) {
        int n = 0;
        check(b3_load_bullet_file(h_, path, keepStaticObjects ? 1 : 0, &n), "loadBulletFile");
        return n;
    }
    /* The same with B3_BULLET_* flags (b3_load_bullet_file_ex): e.g. with
     * B3_BULLET_SPHERES_AND_PLANES the file's spheres and static planes
     * register too. */
    int loadBulletFileFlags(const char* path, int flags) {
        int n = 0;
        check(b3_load_bullet_file_ex(h_, path, flags, &n), "loadBulletFileFlags");
        return n;
    }
    int registerConvexPolyhedron(const float* vertices, int numVertices, int strideBytes = 16,
                                 const float* scaling3 = nullptr) {
        int c = -1;
        check(b3_register_convex_hull(h_, vertices, numVertices, strideBytes, scaling3, &c),
              "registerConvexPolyhedron");
        return c;
    }
    /* CLPhysicsDemo::registerSphereShape / registerPlaneShape /
     * registerCompoundShape / registerConcaveMesh: return the collidable
     * id (b3_register_sphere, _plane, _compound, _concave_mesh). */
    int registerSphereShape(float radius) {
        int c = -1;
        check(b3_register_sphere(h_, radius, &c), "registerSphereShape");
        return c;
    }
    int registerPlaneShape(const float* normal3, float planeConstant) {
        int c = -1;
        check(b3_register_plane(h_, normal3, planeConstant, &c), "registerPlaneShape");
        return c;
    }
    int registerCompoundShape(const b3ChildShape* children, int numChildren) {
        int c = -1;
        check(b3_register_compound(h_, children, numChildren, &c), "registerCompoundShape");
        return c;
    }
    int registerConcaveMesh(const float* vertices3, int numVertices, const int* indices, int numIndices,
                            const float* scaling3 = nullptr) {
        const float one[3] = {1.f, 1.f, 1.f};
        int c = -1;
        check(b3_register_concave_mesh(h_, vertices3, numVertices, indices, numIndices, scaling3 ? scaling3 : one,
                                       &c),
              "registerConcaveMesh");
        return c;
    }
    /* Bounded waits of the persistent solve (b3_set_wait_limits). */
    void setWaitLimits(int spinLimit, int holdMicros = 0) {
        check(b3_set_wait_limits(h_, spinLimit, holdMicros), "setWaitLimits");
    }
    /* CLPhysicsDemo::registerPhysicsInstance: mass 0 = static. */
    int registerPhysicsInstance(float mass, const float* position3, const float* orientation4, int collidable,
                                float friction = 0.6f, float restitution = 0.f, int worldId = 0) {
        int b = -1;
        check(b3_register_body(h_, mass, position3, orientation4, collidable, friction, restitution, worldId, &b),
              "registerPhysicsInstance");
        return b;
    }
    void writeBodiesToGpu(void* stream = nullptr) { check(b3_write_bodies(h_, stream), "writeBodiesToGpu"); }
    void stepSimulation(int numSteps = 1, void* stream = nullptr) {
        check(b3_step(h_, numSteps, stream), "stepSimulation");
    }
    int numBodies() const {
        int n = 0;
        check(b3_get_num_bodies(h_, &n), "b3_get_num_bodies");
        return n;
    }
    std::vector<b3Body> readBodies(void* stream = nullptr) const {
        std::vector<b3Body> out((size_t)numBodies());
        check(b3_read_bodies(h_, out.data(), (int)out.size(), stream), "readBodies");
        return out;
    }
    b3Counters counters(void* stream = nullptr) const {
        b3Counters c;
        check(b3_get_counters(h_, &c, stream), "b3_get_counters");
        return c;
    }
    /* Borrowed device views (getBodiesGpu and friends). */
    void* deviceBuffer(int which, int64_t* bytes = nullptr) const {
        void* p = nullptr;
        int64_t nb = 0;
        check(b3_get_device_buffer(h_, which, &p, &nb), "b3_get_device_buffer");
        if (bytes) *bytes = nb;
        return p;
    }
    /* setupGpuAabbsFull + gravity: the stage before the broadphase. */
    void computeAabbs(void* stream = nullptr) { check(b3_stage_aabbs(h_, stream), "b3_stage_aabbs"); }

private:
    b3World h_ = nullptr;
};

/* btGridBroadphaseCl over a world's bodies (AABBs from World::computeAabbs). */
class GridBroadphase {
public:
    explicit GridBroadphase(World& w) : w_(w) {}
    void calculateOverlappingPairs(void* stream = nullptr) {
        check(b3_grid_broadphase_calculate_overlapping_pairs(w_.handle(), stream), "calculateOverlappingPairs");
    }
    int getNumOverlap(void* stream = nullptr) const {
        int n = 0;
        check(b3_grid_broadphase_get_pair_count(w_.handle(), &n, stream), "getNumOverlap");
        return n;
    }
    /* int2 (self, other) pairs on the device. */
    int32_t* getOverlappingPairBuffer() const { return (int32_t*)w_.deviceBuffer(B3_BUF_PAIRS); }
    float* getAabbMinBuffer() const { return (float*)w_.deviceBuffer(B3_BUF_AABB_MIN); }
    float* getAabbMaxBuffer() const { return (float*)w_.deviceBuffer(B3_BUF_AABB_MAX); }

private:
    World& w_;
};

/* btGpuSapBroadphase (P2/btGpuSapBroadphase.h) over a world created with
 * B3_WORLD_SAP_BROADPHASE: dynamic bodies are its small proxies, static
 * bodies its large proxies. */
class GpuSapBroadphase {
public:
    explicit GpuSapBroadphase(World& w) : w_(w) {}
    void calculateOverlappingPairs(void* stream = nullptr) {
        check(b3_sap_broadphase_calculate_overlapping_pairs(w_.handle(), stream), "calculateOverlappingPairs");
    }
    int getNumOverlap(void* stream = nullptr) const {
        int n = 0;
        check(b3_grid_broadphase_get_pair_count(w_.handle(), &n, stream), "getNumOverlap");
        return n;
    }
    /* int2 pairs on the device: (static id, dynamic id) or (id_i, id_j) in
     * sorted order. */
    int32_t* getOverlappingPairBuffer() const { return (int32_t*)w_.deviceBuffer(B3_BUF_PAIRS); }
    float* getAabbMinBuffer() const { return (float*)w_.deviceBuffer(B3_BUF_AABB_MIN); }
    float* getAabbMaxBuffer() const { return (float*)w_.deviceBuffer(B3_BUF_AABB_MAX); }

private:
    World& w_;
};

/* Solver (ST/Solver.h:104-158), the reference's batched Gauss-Seidel GPU
 * solver, over a world created with B3_WORLD_BATCHED_GS_SOLVER:
 * solveContactConstraint runs batching, convertToConstraints and the 4 + 4
 * iterations (the world's solve stage); getBatches / getConstraints read
 * each manifold's (cell, batch) and Constraint4 after it. */
class BatchedSolver {
public:
    explicit BatchedSolver(World& w) : w_(w) {}
    void solveContactConstraint(void* stream = nullptr) {
        check(b3_solver_solve_batched_gs(w_.handle(), stream), "solveContactConstraint");
    }
    int getBatches(int32_t* cellBatch2, int max, void* stream = nullptr) const {
        int n = 0;
        check(b3_get_gs_batches(w_.handle(), cellBatch2, max, &n, stream), "getBatches");
        return n;
    }
    int getConstraints(b3Constraint4* out, int max, void* stream = nullptr) const {
        int n = 0;
        check(b3_get_gs_constraints(w_.handle(), out, max, &n, stream), "getConstraints");
        return n;
    }

private:
    World& w_;
};

/* btGpuNarrowphaseAndSolver over a world: contacts, Jacobi solve, integrate. */
class GpuNarrowphaseAndSolver {
public:
    explicit GpuNarrowphaseAndSolver(World& w) : w_(w) {}
    int registerConvexHullShape(const float* vertices, int numVertices, int strideBytes = 16,
                                const float* scaling3 = nullptr) {
        return w_.registerConvexPolyhedron(vertices, numVertices, strideBytes, scaling3);
    }
    int registerRigidBody(int collidable, float mass, const float* position3, const float* orientation4,
                          float friction = 0.6f, int worldId = 0) {
        return w_.registerPhysicsInstance(mass, position3, orientation4, collidable, friction, 0.f, worldId);
    }
    void writeAllBodiesToGpu(void* stream = nullptr) { w_.writeBodiesToGpu(stream); }
    /* computeContacts(pairs, nPairs, ...): d_pairs NULL = the world's own
     * broadphase pairs. */
    void computeContacts(const int32_t* d_pairs = nullptr, int numPairs = 0, void* stream = nullptr) {
        check(b3_narrowphase_compute_contacts(w_.handle(), d_pairs, numPairs, stream), "computeContacts");
    }
    void solveContacts(void* stream = nullptr) { check(b3_solver_solve_jacobi(w_.handle(), stream), "solveContacts"); }
    void integrate(void* stream = nullptr) { check(b3_integrate(w_.handle(), stream), "integrate"); }
    int getNumContactsGpu(void* stream = nullptr) const { return (int)w_.counters(stream).numManifolds; }
    b3Contact4* getContactsGpu() const { return (b3Contact4*)w_.deviceBuffer(B3_BUF_CONTACTS); }
    float* getBodiesPositionsGpu() const { return (float*)w_.deviceBuffer(B3_BUF_POS); }

private:
    World& w_;
};

}  // namespace b3
