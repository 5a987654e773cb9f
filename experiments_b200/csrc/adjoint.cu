// Adjoint (reverse-mode) form of the step: placeholder until the adjoint
// kernels land; every entry point reports B3_ERR_UNSUPPORTED.
#include "b3_world.h"

struct b3Adjoint_t {
    b3World w = nullptr;
};

extern "C" int b3_adjoint_create(b3World w, int numSteps, int checkpointEvery, b3Adjoint* out) {
    (void)w; (void)numSteps; (void)checkpointEvery;
    if (out) *out = nullptr;
    return B3_ERR_UNSUPPORTED;
}
extern "C" int b3_adjoint_destroy(b3Adjoint a) { delete a; return B3_OK; }
extern "C" int b3_adjoint_forward(b3Adjoint a, void* stream) { (void)a; (void)stream; return B3_ERR_UNSUPPORTED; }
extern "C" int b3_adjoint_backward(b3Adjoint a, const float* dPos4, const float* dQuat4, const float* dLinVel4,
                                   const float* dAngVel4, void* stream) {
    (void)a; (void)dPos4; (void)dQuat4; (void)dLinVel4; (void)dAngVel4; (void)stream;
    return B3_ERR_UNSUPPORTED;
}
extern "C" int b3_adjoint_gradients(b3Adjoint a, float* dLinVel4, float* dAngVel4, float* dMass, float* dFriction) {
    (void)a; (void)dLinVel4; (void)dAngVel4; (void)dMass; (void)dFriction;
    return B3_ERR_UNSUPPORTED;
}
