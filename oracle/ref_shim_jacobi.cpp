// ORACLE PIN SHIM — test infrastructure only. C entry point over the
// reference's own btPgsJacobiSolver (opencl/gpu_rigidbody_pipeline2/
// btPgsJacobiSolver.cpp), compiled from the reference sources by
// oracle/build.py. Used to pin the oracle's Jacobi restatement.
#include "btPgsJacobiSolver.h"
#include "AdlRigidBody.h"
#include "AdlContact4.h"

extern "C" int ref_jacobi_solve(int numBodies, void* bodies80, void* inertias96, int numContacts,
                                void* contacts96) {
    if (sizeof(RigidBodyBase::Body) != 80 || sizeof(RigidBodyBase::Inertia) != 96 || sizeof(Contact4) != 96)
        return -1;
    btPgsJacobiSolver solver;
    solver.solveContacts(numBodies, (RigidBodyBase::Body*)bodies80, (RigidBodyBase::Inertia*)inertias96,
                         numContacts, (Contact4*)contacts96);
    return 0;
}

// The solver's translation unit emits btTypedConstraint's vtable, which names
// serialize(); joints are compiled out (DISABLE_JOINTS) and no constraint
// object is ever created, so this definition only satisfies the linker.
#include "BulletDynamics/ConstraintSolver/btTypedConstraint.h"
const char* btTypedConstraint::serialize(void*, btSerializer*) const { return 0; }
