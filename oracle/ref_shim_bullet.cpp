// REFERENCE CPU BASELINE SHIM — test and benchmark infrastructure only.
// C entry points over the reference's own CPU rigid-body pipeline,
// bullet2's btDiscreteDynamicsWorld (btDbvtBroadphase +
// btSequentialImpulseConstraintSolver, 10 iterations), compiled from the
// reference's bullet2/ sources by oracle/build.py. bench.py times it as the
// CPU baseline of the step: boxes become btBoxShape, other hulls
// btConvexHullShape of the same points; every independent world of a
// batched scene is its own btDiscreteDynamicsWorld.
#include "btBulletDynamicsCommon.h"

#include <cmath>
#include <cstdio>
#include <vector>

namespace {

struct RefWorld {
    btDefaultCollisionConfiguration* config = nullptr;
    btCollisionDispatcher* dispatcher = nullptr;
    btDbvtBroadphase* broadphase = nullptr;
    btSequentialImpulseConstraintSolver* solver = nullptr;
    btDiscreteDynamicsWorld* world = nullptr;
};

struct RefScene {
    std::vector<RefWorld> worlds;
    std::vector<btCollisionShape*> shapes;
    std::vector<btRigidBody*> bodies;
    std::vector<int> bodyWorld;
    std::vector<btDefaultMotionState*> motions;
    float dt = 1.f / 60.f;
};

// An axis-aligned box given by its 8 corner points becomes a btBoxShape.
// One point (r, 0, 0) is a btSphereShape of radius r; two points (normal,
// then (constant, 0, 0)) a btStaticPlaneShape n . x = constant.
btCollisionShape* make_shape(const float* p, int n) {
    if (n == 1) return new btSphereShape(p[0]);
    if (n == 2) return new btStaticPlaneShape(btVector3(p[0], p[1], p[2]), p[3]);
    if (n == 8) {
        float lo[3] = {p[0], p[1], p[2]}, hi[3] = {p[0], p[1], p[2]};
        for (int i = 1; i < 8; ++i)
            for (int k = 0; k < 3; ++k) {
                lo[k] = std::fmin(lo[k], p[3 * i + k]);
                hi[k] = std::fmax(hi[k], p[3 * i + k]);
            }
        bool box = true;
        for (int i = 0; i < 8 && box; ++i)
            for (int k = 0; k < 3; ++k)
                if (p[3 * i + k] != lo[k] && p[3 * i + k] != hi[k]) box = false;
        if (box && std::fabs(lo[0] + hi[0]) < 1e-6f && std::fabs(lo[1] + hi[1]) < 1e-6f &&
            std::fabs(lo[2] + hi[2]) < 1e-6f)
            return new btBoxShape(btVector3(hi[0], hi[1], hi[2]));
    }
    btConvexHullShape* h = new btConvexHullShape();
    for (int i = 0; i < n; ++i) h->addPoint(btVector3(p[3 * i], p[3 * i + 1], p[3 * i + 2]));
    return h;
}

}  // namespace

extern "C" {

void* rb_create(int numShapes, const int* shapeOffsets, const float* points3, int numBodies, const int* shape,
                const float* mass, const float* pos3, const float* quat4, const float* friction, const float* lin3,
                const float* ang3, const int* worldId, int numWorlds, float dt, int iterations, float gx, float gy,
                float gz) {
    RefScene* s = new RefScene();
    s->dt = dt;
    s->worlds.resize(numWorlds < 1 ? 1 : numWorlds);
    for (RefWorld& w : s->worlds) {
        w.config = new btDefaultCollisionConfiguration();
        w.dispatcher = new btCollisionDispatcher(w.config);
        w.broadphase = new btDbvtBroadphase();
        w.solver = new btSequentialImpulseConstraintSolver();
        w.world = new btDiscreteDynamicsWorld(w.dispatcher, w.broadphase, w.solver, w.config);
        w.world->setGravity(btVector3(gx, gy, gz));
        w.world->getSolverInfo().m_numIterations = iterations;
    }
    for (int k = 0; k < numShapes; ++k)
        s->shapes.push_back(make_shape(points3 + 3 * shapeOffsets[k], shapeOffsets[k + 1] - shapeOffsets[k]));
    for (int i = 0; i < numBodies; ++i) {
        btCollisionShape* sh = s->shapes[shape[i]];
        btVector3 inertia(0, 0, 0);
        if (mass[i] > 0.f) sh->calculateLocalInertia(mass[i], inertia);
        btTransform t;
        t.setIdentity();
        t.setOrigin(btVector3(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]));
        t.setRotation(btQuaternion(quat4[4 * i], quat4[4 * i + 1], quat4[4 * i + 2], quat4[4 * i + 3]));
        btDefaultMotionState* ms = new btDefaultMotionState(t);
        btRigidBody::btRigidBodyConstructionInfo info(mass[i], ms, sh, inertia);
        info.m_friction = friction[i];
        btRigidBody* b = new btRigidBody(info);
        if (mass[i] > 0.f) {
            b->setLinearVelocity(btVector3(lin3[3 * i], lin3[3 * i + 1], lin3[3 * i + 2]));
            b->setAngularVelocity(btVector3(ang3[3 * i], ang3[3 * i + 1], ang3[3 * i + 2]));
        }
        int wid = worldId ? worldId[i] : 0;
        if (wid < 0 || wid >= (int)s->worlds.size()) wid = 0;
        s->worlds[wid].world->addRigidBody(b);
        s->bodies.push_back(b);
        s->bodyWorld.push_back(wid);
        s->motions.push_back(ms);
    }
    return s;
}

void rb_step(void* h, int steps) {
    RefScene* s = (RefScene*)h;
    for (int i = 0; i < steps; ++i)
        for (RefWorld& w : s->worlds) w.world->stepSimulation(s->dt, 0);
}

// Positions of the bodies (xyz) after the steps taken.
void rb_positions(void* h, float* pos3) {
    RefScene* s = (RefScene*)h;
    for (size_t i = 0; i < s->bodies.size(); ++i) {
        const btVector3& o = s->bodies[i]->getCenterOfMassPosition();
        pos3[3 * i] = o.x();
        pos3[3 * i + 1] = o.y();
        pos3[3 * i + 2] = o.z();
    }
}

// The first world serialised by bullet2's own btDefaultSerializer into a
// .bullet file at path (the reference's scene file format); 0 on success.
int rb_write_bullet(void* h, const char* path) {
    RefScene* s = (RefScene*)h;
    btDefaultSerializer* ser = new btDefaultSerializer();
    s->worlds[0].world->serialize(ser);
    FILE* f = fopen(path, "wb");
    if (!f) {
        delete ser;
        return 1;
    }
    const size_t n = fwrite(ser->getBufferPointer(), ser->getCurrentBufferSize(), 1, f);
    fclose(f);
    delete ser;
    return n == 1 ? 0 : 1;
}

void rb_destroy(void* h) {
    RefScene* s = (RefScene*)h;
    for (size_t i = 0; i < s->bodies.size(); ++i) {
        s->worlds[s->bodyWorld[i]].world->removeRigidBody(s->bodies[i]);
        delete s->bodies[i];
        delete s->motions[i];
    }
    for (btCollisionShape* sh : s->shapes) delete sh;
    for (RefWorld& w : s->worlds) {
        delete w.world;
        delete w.solver;
        delete w.broadphase;
        delete w.dispatcher;
        delete w.config;
    }
    delete s;
}

}  // extern "C"
