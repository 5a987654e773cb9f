// Shared by the Jacobi solver (solver.cu) and its adjoint (adjoint.cu):
// constraint-row storage, the solver view of the world's buffers, the row
// update, the per-body averaging and the bounded grid barrier.
#pragma once
#include "b3_math.cuh"
#include "b3_world.h"

namespace b3solver {

using namespace b3m;

// Row storage: kRowSlots float4 streams of length maxManifolds.
//  slot 0..3   header: (A,B,nRows,flags as int), (invMassA, invMassB, mu, -),
//              (invInertiaA.xyz, countA), (invInertiaB.xyz, countB)
//  normal row j (j<4):   4 + 3j + {0,1,2}
//  friction row r (r<8): 16 + 3r + {0,1,2}; r = 2j + {0: dir2, 1: dir1}
//  each row: (n.xyz, rhs), (r1xn.xyz, jacDiagABInv), (r2xn.xyz, applied)
constexpr int kRowSlots = 40;
constexpr int kNormal0 = 4;
constexpr int kFric0 = 16;

struct SolverView {
    float4* rows;       // [kRowSlots][cap]
    int cap;            // manifold capacity (stride)
    float4* copyLin;    // [2][cap]
    float4* copyAng;    // [2][cap]
    float4* avgLin;     // [N]
    float4* avgAng;     // [N]
    const uint32_t* incVals;   // sorted copy ids (2m + side)
    const uint32_t* incStart;  // per body
    const uint32_t* incEnd;
    const int32_t* numManifolds;
    int numBodies;
    // bounded waits of the persistent Jacobi kernel: polls of a grid
    // barrier before it gives up, and (testing the give-up path only) how
    // long block 0 holds back before its first barrier, in microseconds
    int spinLimit;
    int holdMicros;
};

__device__ __forceinline__ float4& R(const SolverView& v, int slot, int m) {
    return v.rows[(size_t)slot * v.cap + m];
}

// btPlaneSpace1 (LinearMath/btVector3.h), published construction of two
// unit tangents orthogonal to n.
__device__ __forceinline__ void plane_space(float3 n, float3& p, float3& q) {
    const float SQRT12 = 0.7071067811865475244008443621048490f;
    if (fabsf(n.z) > SQRT12) {
        const float a = n.y * n.y + n.z * n.z;
        const float k = rsqrtf(a);
        p = make_float3(0.f, -n.z * k, n.y * k);
        q = make_float3(a * k, -n.x * p.z, n.x * p.y);
    } else {
        const float a = n.x * n.x + n.y * n.y;
        const float k = rsqrtf(a);
        p = make_float3(-n.y * k, n.x * k, 0.f);
        q = make_float3(-n.z * p.y, n.z * p.x, a * k);
    }
}

// ---------------------------------------------------------------------------
// Persistent-kernel helpers
// ---------------------------------------------------------------------------
// Every block arrives, the last one releases the others. A waiter gives up
// after spinLimit polls: it sets *err, counts a timeout and the kernel's
// blocks leave at this or their next barrier (an error set by anyone makes
// every barrier fail), so the launch always ends.
__device__ __forceinline__ bool grid_barrier(uint32_t* count, uint32_t* gen, uint32_t nblocks,
                                             int32_t* err, b3Counters* counters,
                                             int spinLimit = b3dev::kSpinLimit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const uint32_t g = b3dev::ld_acquire_u32(gen);
        __threadfence();
        const uint32_t arrived = atomicAdd(count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(count, 0u);
            __threadfence();
            b3dev::st_release_u32(gen, g + 1u);
        } else {
            int spins = 0;
            while (b3dev::ld_acquire_u32(gen) == g) {
                if (++spins > spinLimit) {
                    atomicExch(err, 1);
                    atomicAdd(&counters->timeouts, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (*(volatile int32_t*)err) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ void solve_row(const float4 r0, const float4 r1, float4& r2, float lo, float hi,
                                          float imA, float imB, float3 iiA, float3 iiB,
                                          float3& dvA, float3& dwA, float3& dvB, float3& dwB) {
    const float3 n = f3(r0), t1 = f3(r1), t2 = f3(r2);
    const float rhs = r0.w, jac = r1.w, applied = r2.w;
    float delta = rhs;  // - applied * cfm (cfm = 0)
    const float dv1 = dot(n, dvA) + dot(t1, dwA);
    const float dv2 = -dot(n, dvB) + dot(t2, dwB);
    delta -= dv1 * jac;
    delta -= dv2 * jac;
    const float sum = applied + delta;
    float na;
    if (sum < lo) {
        delta = lo - applied;
        na = lo;
    } else if (sum > hi) {
        delta = hi - applied;
        na = hi;
    } else {
        na = sum;
    }
    r2.w = na;
    dvA += n * (imA * delta);
    dwA += mulv(iiA, t1) * delta;
    dvB += (-n * imB) * delta;
    dwB += mulv(iiB, t2) * delta;
}

// Averaged delta velocity of body b over its copies in buffer buf
// (averageVelocities, P2/btPgsJacobiSolver.cpp:1683-1720): copies in
// manifold order, sum then multiply by 1/count.
__device__ __forceinline__ void body_average_se(const SolverView& V, uint32_t s, uint32_t e, int buf, float3& lin,
                                                float3& ang) {
    float3 sl = make_float3(0.f, 0.f, 0.f), sa = sl;
    for (uint32_t i = s; i < e; ++i) {
        const uint32_t cid = V.incVals[i];
        const size_t at = (size_t)(buf * 2 + (int)(cid & 1u)) * V.cap + (cid >> 1);
        sl += f3(V.copyLin[at]);
        sa += f3(V.copyAng[at]);
    }
    const float factor = 1.f / (float)(e - s);
    lin = sl * factor;
    ang = sa * factor;
}
__device__ __forceinline__ void body_average(const SolverView& V, int b, int buf, float3& lin, float3& ang) {
    body_average_se(V, V.incStart[b], V.incEnd[b], buf, lin, ang);
}

// One body's average given its incidence range, with the loads issued four
// copies at a time (copy ids, then the copies): the same copies, order and
// operations as body_average, hence the same result.
__device__ __forceinline__ void body_average_range(const SolverView& V, uint32_t s, uint32_t e, int buf, float3& lin,
                                                   float3& ang) {
    float3 sl = make_float3(0.f, 0.f, 0.f), sa = sl;
    for (uint32_t i0 = s; i0 < e; i0 += 4) {
        uint32_t cid[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) cid[u] = i0 + u < e ? V.incVals[i0 + u] : 0u;
        float4 cl[4], ca[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u < e) {
                const size_t at = (size_t)(buf * 2 + (int)(cid[u] & 1u)) * V.cap + (cid[u] >> 1);
                cl[u] = V.copyLin[at];
                ca[u] = V.copyAng[at];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u < e) {
                sl += f3(cl[u]);
                sa += f3(ca[u]);
            }
        }
    }
    const float factor = 1.f / (float)(e - s);
    lin = sl * factor;
    ang = sa * factor;
}

SolverView solver_view(b3World_t* w);

}  // namespace b3solver
