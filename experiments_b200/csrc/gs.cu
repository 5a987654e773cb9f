// Batched Gauss-Seidel contact solver: the reference's GPU solver
// (btGpuNarrowphaseAndSolver::solveContacts, P1/btGpuNarrowPhaseAndSolver.cpp:
// 1073-1353, driving ST/Solver.cpp) for worlds created with
// B3_WORLD_BATCHED_GS_SOLVER.
//
// Per step, after the manifolds:
//   k_gs_keys      cell of each manifold on the 16 x 16 xz grid from its
//                  dynamic body (SetSortDataKernel, ST/solverSetup2.cl:457-478)
//                  and its parity class (BatchSolveKernelContact's cell
//                  mapping, ST/solveContact.cl:418-426); radix sort by
//                  (class, cell), stable, so each class lists its manifolds
//                  in (cell, manifold) order
//   k_gs_colour    greedy colouring of every class at once, persistent and
//                  cooperative: batch after batch, rounds of "a manifold
//                  joins when it is the first undecided manifold of each of
//                  its dynamic bodies; manifolds sharing a body with a
//                  joined one wait for the next batch", which reproduces the
//                  sequential greedy pass of sortConstraintByBatch
//                  (P1/btGpuNarrowPhaseAndSolver.cpp:752-852) run over the
//                  class in order, with exact body identities
//   k_gs_inertia   world inverse inertia R diag(I^-1) R^T per body
//                  (setupBodiesKernel, broadphaseKernel.cl:189-201)
//   k_gs_setup     Constraint4 per manifold (setConstraint4,
//                  ST/solverSetup.cl:520-609), stored grouped by
//                  (class, batch) (counting sort)
//   k_gs_solve     4 contact then 4 friction iterations; in each, the
//                  classes in order and their batches in order, every batch
//                  solved in parallel (no dynamic body twice), grid
//                  barriers in between (ST/Solver.cpp:561-700;
//                  solveContact.cl:272-365, solveFriction.cl:297-391)
// Velocities are written to the bodies directly; integration then applies
// no Jacobi averages.
#include <algorithm>

#include "b3_internal.h"
#include "b3_math.cuh"
#include "b3_world.h"
#include "solver_common.cuh"

using namespace b3m;
using b3solver::grid_barrier;

namespace {

constexpr int kSplit = 16;        // SolverBase::N_SPLIT
constexpr int kIterations = 4;    // m_nIterations (P1/btGpuNarrowPhaseAndSolver.cpp:1330)
constexpr float kScale = 0.5f;    // 1 / (N_OBJ_PER_SPLIT * m_averageExtent) = 1 / (10 * 0.2)
constexpr float kFriction = 0.7f; // m_linear.w (ST/solverSetup.cl:541), ST/solveFriction.cl:319
constexpr float kDrift = 0.005f;  // ConstraintCfg::m_positionDrift
constexpr float kPosCoeff = 0.2f; // ConstraintCfg::m_positionConstraintCoeff
constexpr int kNone = 0x7fffffff;

__device__ __forceinline__ int class_of(int cell) { return (cell & 1) + 2 * ((cell / kSplit) & 1); }

// cell and class of every manifold; keys (class, cell), values manifold
__global__ void k_gs_keys(const b3Contact4* __restrict__ contacts, const int* __restrict__ manifoldPair,
                          const int32_t* __restrict__ numManifolds, const float4* __restrict__ pos,
                          const float* __restrict__ invMass, uint32_t* __restrict__ keys,
                          uint32_t* __restrict__ vals, int* __restrict__ cellOf) {
    const int M = *numManifolds;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const b3Contact4& c = contacts[manifoldPair[m]];
        const int A = abs(c.bodyAPtrAndSignBit), B = abs(c.bodyBPtrAndSignBit);
        // the dynamic body's position (A unless A is static)
        const int body = invMass[A] != 0.f ? A : B;
        const float4 p = pos[body];
        const int xi = (int)((p.x - (p.x < 0.f ? 1.f : 0.f)) * kScale) & (kSplit - 1);
        const int zi = (int)((p.z - (p.z < 0.f ? 1.f : 0.f)) * kScale) & (kSplit - 1);
        const int cell = xi + zi * kSplit;
        keys[m] = (uint32_t)((class_of(cell) << 8) | cell);
        vals[m] = (uint32_t)m;
        cellOf[m] = cell;
    }
}

struct ColourView {
    const uint32_t* keys;     // sorted (class << 8 | cell)
    const uint32_t* vals;     // sorted manifold ids
    const b3Contact4* contacts;
    const int* manifoldPair;
    const float* invMass;
    const int32_t* numManifolds;
    int numBodies;
    int* minRank;             // [4][numBodies]: first undecided slot per body this round
    int* taken;               // [4][numBodies]: batch + 1 of the last batch that took the body
    int* slotBatch;           // per slot: batch, -1 undecided, -2 waiting for the next batch
    int* batchCount;          // [4]: batches per class
    int* roundCount;          // [5]: undecided after a round (three in rotation: a block may
                              // still read the last round's while block 0 clears the next),
                              // then waiting after a batch (two)
    uint32_t* bar;            // barrier count, generation
    int32_t* err;
    b3Counters* counters;
    int maxBatch;
};

__device__ __forceinline__ void slot_bodies(const ColourView& V, int s, int& cls, int& a, int& b) {
    cls = (int)(V.keys[s] >> 8);
    const b3Contact4& c = V.contacts[V.manifoldPair[V.vals[s]]];
    const int A = abs(c.bodyAPtrAndSignBit), B = abs(c.bodyBPtrAndSignBit);
    a = V.invMass[A] != 0.f ? A : -1;  // dynamic bodies only
    b = V.invMass[B] != 0.f ? B : -1;
}

__global__ void __launch_bounds__(256) k_gs_colour(ColourView V) {
    const int M = *V.numManifolds;
    const int N = V.numBodies;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    uint32_t* cnt = V.bar;
    uint32_t* gen = V.bar + 1;
    for (int s = tid; s < M; s += stride) V.slotBatch[s] = -1;
    if (tid < 4) V.batchCount[tid] = 0;
    if (tid < 5) V.roundCount[tid] = 0;
    if (!grid_barrier(cnt, gen, gridDim.x, V.err, V.counters)) return;
    int round = 0;
    for (int batch = 0;; ++batch) {
        if (batch >= V.maxBatch) {
            if (tid == 0) atomicExch(V.err, 2);
            return;
        }
        for (;; ++round) {
            // A: the first undecided slot of every dynamic body
            if (tid == 0) V.roundCount[(round + 1) % 3] = 0;
            for (int s = tid; s < M; s += stride) {
                if (__ldcg(&V.slotBatch[s]) != -1) continue;
                int cls, a, b;
                slot_bodies(V, s, cls, a, b);
                if (a >= 0) atomicMin(&V.minRank[cls * N + a], s);
                if (b >= 0) atomicMin(&V.minRank[cls * N + b], s);
            }
            if (!grid_barrier(cnt, gen, gridDim.x, V.err, V.counters)) return;
            // B: join where first on every dynamic body
            for (int s = tid; s < M; s += stride) {
                if (__ldcg(&V.slotBatch[s]) != -1) continue;
                int cls, a, b;
                slot_bodies(V, s, cls, a, b);
                if ((a < 0 || __ldcg(&V.minRank[cls * N + a]) == s) && (b < 0 || __ldcg(&V.minRank[cls * N + b]) == s)) {
                    __stcg(&V.slotBatch[s], batch);
                    if (a >= 0) __stcg(&V.taken[cls * N + a], batch + 1);
                    if (b >= 0) __stcg(&V.taken[cls * N + b], batch + 1);
                    atomicMax(&V.batchCount[cls], batch + 1);
                }
            }
            if (!grid_barrier(cnt, gen, gridDim.x, V.err, V.counters)) return;
            // C: wait when a body was taken; clear the ranks; count the rest
            int undecided = 0;
            for (int s = tid; s < M; s += stride) {
                const int sb = __ldcg(&V.slotBatch[s]);
                if (sb != -1 && sb != -2 && sb != batch) continue;
                int cls, a, b;
                slot_bodies(V, s, cls, a, b);
                if (a >= 0) __stcg(&V.minRank[cls * N + a], kNone);
                if (b >= 0) __stcg(&V.minRank[cls * N + b], kNone);
                if (sb != -1) continue;
                if ((a >= 0 && __ldcg(&V.taken[cls * N + a]) == batch + 1) ||
                    (b >= 0 && __ldcg(&V.taken[cls * N + b]) == batch + 1)) {
                    __stcg(&V.slotBatch[s], -2);
                } else {
                    ++undecided;
                }
            }
            if (undecided) atomicAdd(&V.roundCount[round % 3], undecided);
            if (!grid_barrier(cnt, gen, gridDim.x, V.err, V.counters)) return;
            if (__ldcg(&V.roundCount[round % 3]) == 0) {
                ++round;
                break;
            }
        }
        // the waiting slots are the next batch's undecided ones
        if (tid == 0) V.roundCount[3 + ((batch + 1) & 1)] = 0;
        int waiting = 0;
        for (int s = tid; s < M; s += stride)
            if (__ldcg(&V.slotBatch[s]) == -2) {
                __stcg(&V.slotBatch[s], -1);
                ++waiting;
            }
        if (waiting) atomicAdd(&V.roundCount[3 + (batch & 1)], waiting);
        if (!grid_barrier(cnt, gen, gridDim.x, V.err, V.counters)) return;
        if (__ldcg(&V.roundCount[3 + (batch & 1)]) == 0) return;
    }
}

// world inverse inertia rows per body (zero for static bodies)
__global__ void k_gs_inertia(b3::BodiesDev Bd, float4* __restrict__ Iw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Bd.n) return;
    float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0, r2 = r0;
    if (Bd.invMass[i] != 0.f) {
        const Mat3 R = quat_to_mat(Bd.quat[i]);
        const float3 d = f3(Bd.invInertia[i]);
        // (R diag(d) R^T)_ab = sum_k R_ak d_k R_bk
        const float3 a0 = make_float3(R.r0.x * d.x, R.r0.y * d.y, R.r0.z * d.z);
        const float3 a1 = make_float3(R.r1.x * d.x, R.r1.y * d.y, R.r1.z * d.z);
        const float3 a2 = make_float3(R.r2.x * d.x, R.r2.y * d.y, R.r2.z * d.z);
        r0 = make_float4(dot(a0, R.r0), dot(a0, R.r1), dot(a0, R.r2), 0.f);
        r1 = make_float4(dot(a1, R.r0), dot(a1, R.r1), dot(a1, R.r2), 0.f);
        r2 = make_float4(dot(a2, R.r0), dot(a2, R.r1), dot(a2, R.r2), 0.f);
    }
    Iw[3 * i + 0] = r0;
    Iw[3 * i + 1] = r1;
    Iw[3 * i + 2] = r2;
}

struct M3 {
    float3 r0, r1, r2;
};
__device__ __forceinline__ M3 load_iw(const float4* Iw, int i) {
    return M3{f3(__ldg(&Iw[3 * i])), f3(__ldg(&Iw[3 * i + 1])), f3(__ldg(&Iw[3 * i + 2]))};
}
__device__ __forceinline__ float3 mul(const M3& m, float3 v) {
    return make_float3(dot(m.r0, v), dot(m.r1, v), dot(m.r2, v));
}

// calcJacCoeff (ST/solverSetup.cl:445-454); symmetric inverse inertias
__device__ __forceinline__ float jac_coeff(float3 ang0, float3 ang1, float imA, const M3& IA, float imB,
                                           const M3& IB) {
    return -1.f / (imA + dot(mul(IA, ang0), ang0) + imB + dot(mul(IB, ang1), ang1));
}

// btPlaneSpace1 as the solver kernels write it (ST/solverSetup.cl:477-501)
__device__ __forceinline__ void plane_space1(float3 n, float3& p, float3& q) {
    if (fabsf(n.z) > 0.70710678f) {
        const float a = n.y * n.y + n.z * n.z;
        const float k = 1.f / sqrtf(a);
        p = make_float3(0.f, -n.z * k, n.y * k);
        q = make_float3(a * k, -n.x * p.z, n.x * p.y);
    } else {
        const float a = n.x * n.x + n.y * n.y;
        const float k = 1.f / sqrtf(a);
        p = make_float3(-n.y * k, n.x * k, 0.f);
        q = make_float3(-n.z * p.y, n.z * p.x, a * k);
    }
}

// per (class, batch) key: counts, then offsets (exclusive scan), then the
// constraints scattered to their group with setConstraint4
__global__ void k_gs_count(const uint32_t* __restrict__ keys, const int* __restrict__ slotBatch,
                           const int32_t* __restrict__ numManifolds, int maxBatch, uint32_t* __restrict__ groupCount) {
    const int M = *numManifolds;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < M; s += gridDim.x * blockDim.x) {
        const int cls = (int)(keys[s] >> 8);
        const int b = slotBatch[s];
        if (b >= 0 && b < maxBatch) atomicAdd(&groupCount[cls * maxBatch + b], 1u);
    }
}

// exclusive scan of the group counts, one block (groups <= 4 * 1024)
__global__ void __launch_bounds__(1024) k_gs_offsets(const uint32_t* __restrict__ count, uint32_t* __restrict__ offset,
                                                     int groups) {
    __shared__ uint32_t warpSum[32];
    const int per = (groups + blockDim.x - 1) / blockDim.x;
    const int i0 = threadIdx.x * per;
    uint32_t local = 0;
    for (int i = i0; i < min(i0 + per, groups); ++i) local += count[i];
    // inclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) / 32;
        uint32_t v = lane < nw ? warpSum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane < nw) warpSum[lane] = v;
    }
    __syncthreads();
    uint32_t run = x - local + (wid > 0 ? warpSum[wid - 1] : 0u);
    for (int i = i0; i < min(i0 + per, groups); ++i) {
        offset[i] = run;
        run += count[i];
    }
    if (threadIdx.x == blockDim.x - 1) offset[groups] = run;
}

struct SetupParams {
    float dtInv;
    int maxBatch;
};

__global__ void k_gs_setup(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                           const int* __restrict__ slotBatch, const int32_t* __restrict__ numManifolds,
                           const uint32_t* __restrict__ groupOffset, uint32_t* __restrict__ groupFill,
                           const b3Contact4* __restrict__ contacts, const int* __restrict__ manifoldPair,
                           b3::BodiesDev Bd, const float4* __restrict__ Iw, b3Constraint4* __restrict__ cs,
                           int* __restrict__ slotOfManifold, SetupParams P) {
    const int M = *numManifolds;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < M; s += gridDim.x * blockDim.x) {
        const int cls = (int)(keys[s] >> 8);
        const int batch = slotBatch[s];
        const int m = (int)vals[s];
        if (batch < 0 || batch >= P.maxBatch) {  // colouring stopped (error flag set)
            slotOfManifold[m] = -1;
            continue;
        }
        const int g = cls * P.maxBatch + batch;
        const int q = (int)(groupOffset[g] + atomicAdd(&groupFill[g], 1u));
        slotOfManifold[m] = q;
        const b3Contact4 c = contacts[manifoldPair[m]];
        const int A = abs(c.bodyAPtrAndSignBit), B = abs(c.bodyBPtrAndSignBit);
        const float imA = Bd.invMass[A], imB = Bd.invMass[B];
        const M3 IA = load_iw(Iw, A), IB = load_iw(Iw, B);
        const float3 posA = f3(Bd.pos[A]), posB = f3(Bd.pos[B]);
        const float3 n = make_float3(c.worldNormal[0], c.worldNormal[1], c.worldNormal[2]);
        const int np = (int)c.worldNormal[3];
        b3Constraint4 d;
        d.bodyA = (uint32_t)A;
        d.bodyB = (uint32_t)B;
        d.batchIdx = batch;
        d.padding = 0u;
        d.linear[0] = -n.x;
        d.linear[1] = -n.y;
        d.linear[2] = -n.z;
        d.linear[3] = kFriction;
#pragma unroll
        for (int ic = 0; ic < 4; ++ic) {
            d.appliedRambdaDt[ic] = 0.f;
            d.jacCoeffInv[ic] = 0.f;
            d.b[ic] = 0.f;
            d.worldPos[ic][0] = d.worldPos[ic][1] = d.worldPos[ic][2] = d.worldPos[ic][3] = 0.f;
            if (ic < np) {
                const float3 p = make_float3(c.worldPos[ic][0], c.worldPos[ic][1], c.worldPos[ic][2]);
                const float3 ang0 = -cross(p - posA, n), ang1 = cross(p - posB, n);
                d.jacCoeffInv[ic] = jac_coeff(ang0, ang1, imA, IA, imB, IB);
                // restitution 0: the position term alone
                d.b[ic] = (c.worldPos[ic][3] + kDrift) * kPosCoeff * P.dtInv;
                d.worldPos[ic][0] = p.x;
                d.worldPos[ic][1] = p.y;
                d.worldPos[ic][2] = p.z;
                d.worldPos[ic][3] = c.worldPos[ic][3];
            }
        }
        float3 center = make_float3(0.f, 0.f, 0.f);
        for (int i = 0; i < np; ++i) center += make_float3(c.worldPos[i][0], c.worldPos[i][1], c.worldPos[i][2]);
        center = center * (1.f / (float)np);
        float3 t[2];
        plane_space1(n, t[0], t[1]);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const float3 ang0 = -cross(center - posA, t[i]), ang1 = cross(center - posB, t[i]);
            d.fJacCoeffInv[i] = jac_coeff(ang0, ang1, imA, IA, imB, IB);
            d.fAppliedRambdaDt[i] = 0.f;
        }
        d.center[0] = center.x;
        d.center[1] = center.y;
        d.center[2] = center.z;
        d.center[3] = 0.f;
        cs[q] = d;
    }
}

struct SolveView {
    b3Constraint4* cs;
    const uint32_t* groupOffset;  // [4 * maxBatch + 1]
    const int* batchCount;        // [4]
    int maxBatch;
    float4* pos;
    float4* linVel;
    float4* angVel;
    const float* invMass;
    const float4* Iw;
    uint32_t* bar;
    int32_t* err;
    b3Counters* counters;
};

__device__ __forceinline__ float3 ldv(const float4* p) {
    const float4 v = __ldcg(p);
    return make_float3(v.x, v.y, v.z);
}

// One constraint with the data that does not change during the solve:
// its Constraint4 record and its bodies' positions, inverse masses and world
// inverse inertias. The solve fetches the next batch's before each barrier,
// so that after it only the velocities are still to be loaded.
struct Pending {
    int q;  // constraint index, -1 for none
    union {
        b3Constraint4 c;
        float4 raw[11];
    };
    int A, B;
    float imA, imB;
    float3 posA, posB;
    M3 IA, IB;
};
static_assert(sizeof(b3Constraint4) == 11 * sizeof(float4), "Constraint4 is 176 bytes");

__device__ __forceinline__ void fetch(const SolveView& V, int q, Pending& P) {
    P.q = q;
    if (q < 0) return;
    const float4* src = reinterpret_cast<const float4*>(V.cs + q);
#pragma unroll
    for (int k = 0; k < 11; ++k) P.raw[k] = src[k];
    P.A = (int)P.c.bodyA;
    P.B = (int)P.c.bodyB;
    P.imA = V.invMass[P.A];
    P.imB = V.invMass[P.B];
    P.posA = f3(V.pos[P.A]);
    P.posB = f3(V.pos[P.B]);
    P.IA = load_iw(V.Iw, P.A);
    P.IB = load_iw(V.Iw, P.B);
}

// the constraint, contact (phase 0) or friction (phase 1); a static
// body's velocity is read and written as zero
__device__ void solve_one(const SolveView& V, Pending& P, int phase) {
    b3Constraint4& c = P.c;
    const int A = P.A, B = P.B;
    const float imA = P.imA, imB = P.imB;
    const bool dA = imA != 0.f, dB = imB != 0.f;
    float3 vA = dA ? ldv(&V.linVel[A]) : make_float3(0.f, 0.f, 0.f);
    float3 wA = dA ? ldv(&V.angVel[A]) : make_float3(0.f, 0.f, 0.f);
    float3 vB = dB ? ldv(&V.linVel[B]) : make_float3(0.f, 0.f, 0.f);
    float3 wB = dB ? ldv(&V.angVel[B]) : make_float3(0.f, 0.f, 0.f);
    const float3 posA = P.posA, posB = P.posB;
    const M3& IA = P.IA;
    const M3& IB = P.IB;
    const float3 lin = make_float3(c.linear[0], c.linear[1], c.linear[2]);
    const float3 n = -lin;
    float4* dst = reinterpret_cast<float4*>(V.cs + P.q);
    if (phase == 0) {
        // solveContact (ST/solveContact.cl:272-309): impulses clamped to [0, inf)
#pragma unroll
        for (int ic = 0; ic < 4; ++ic) {
            if (c.jacCoeffInv[ic] == 0.f) continue;
            const float3 p = make_float3(c.worldPos[ic][0], c.worldPos[ic][1], c.worldPos[ic][2]);
            const float3 ang0 = -cross(p - posA, n), ang1 = cross(p - posB, n);
            float l = dot(lin, vA) + dot(ang0, wA) + dot(-lin, vB) + dot(ang1, wB) + c.b[ic];
            l *= c.jacCoeffInv[ic];
            const float prev = c.appliedRambdaDt[ic];
            const float upd = fmaxf(prev + l, 0.f);
            l = upd - prev;
            c.appliedRambdaDt[ic] = upd;
            vA += lin * (imA * l);
            vB += -lin * (imB * l);
            wA += mul(IA, ang0) * l;
            wB += mul(IB, ang1) * l;
        }
        dst[8] = P.raw[8];  // appliedRambdaDt
    } else {
        // solveFrictionConstraint (ST/solveFriction.cl:297-391)
        if (c.fJacCoeffInv[0] == 0.f && c.fJacCoeffInv[1] == 0.f) return;
        const float sum = ((c.appliedRambdaDt[0] + c.appliedRambdaDt[1]) + c.appliedRambdaDt[2]) + c.appliedRambdaDt[3];
        const float maxR = kFriction * sum, minR = -maxR;
        float3 t[2];
        plane_space1(n, t[0], t[1]);
        const float3 center = make_float3(c.center[0], c.center[1], c.center[2]);
        const float3 r0 = center - posA, r1 = center - posB;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const float3 fl = -t[i], ang0 = -cross(r0, t[i]), ang1 = cross(r1, t[i]);
            float l = dot(fl, vA) + dot(ang0, wA) + dot(-fl, vB) + dot(ang1, wB);
            l *= c.fJacCoeffInv[i];
            const float prev = c.fAppliedRambdaDt[i];
            const float upd = fminf(fmaxf(prev + l, minR), maxR);
            l = upd - prev;
            c.fAppliedRambdaDt[i] = upd;
            vA += fl * (imA * l);
            vB += -fl * (imB * l);
            wA += mul(IA, ang0) * l;
            wB += mul(IB, ang1) * l;
        }
        // angular damping about the normal (:368-379)
        const float3 ab = normalize(posB - posA), ac = normalize(center - posA);
        if (dot(ab, ac) > 0.95f || !dA || !dB) {
            const float angNA = dot(n, wA), angNB = dot(n, wB);
            wA -= n * (angNA * 0.1f);
            wB -= n * (angNB * 0.1f);
        }
        dst[9] = P.raw[9];  // fJacCoeffInv, fAppliedRambdaDt
    }
    __stcg(&V.linVel[A], dA ? make_float4(vA.x, vA.y, vA.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f));
    __stcg(&V.angVel[A], dA ? make_float4(wA.x, wA.y, wA.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f));
    __stcg(&V.linVel[B], dB ? make_float4(vB.x, vB.y, vB.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f));
    __stcg(&V.angVel[B], dB ? make_float4(wB.x, wB.y, wB.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f));
}

// (class, batch) group of step j of an iteration (classes in order, their
// batches in order)
__device__ __forceinline__ int group_of(int j, const int nb[4], int maxBatch) {
    int cls = 0;
    while (cls < 3 && j >= nb[cls]) {
        j -= nb[cls];
        ++cls;
    }
    return cls * maxBatch + j;
}

__global__ void __launch_bounds__(256) k_gs_solve(SolveView V) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    int nb[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) nb[c] = min(__ldcg(&V.batchCount[c]), V.maxBatch);
    const int G = nb[0] + nb[1] + nb[2] + nb[3];  // batch steps per iteration
    const int steps = 2 * kIterations * G;        // contact iterations, then friction
    if (steps == 0) return;
    int g = group_of(0, nb, V.maxBatch);
    int q0 = (int)V.groupOffset[g], q1 = (int)V.groupOffset[g + 1];
    Pending P;
    fetch(V, q0 + tid < q1 ? q0 + tid : -1, P);
    for (int k = 0; k < steps; ++k) {
        const int phase = k / (kIterations * G);
        if (P.q >= 0) solve_one(V, P, phase);
        for (int q = q0 + tid + stride; q < q1; q += stride) {
            Pending T;
            fetch(V, q, T);
            solve_one(V, T, phase);
        }
        // the next batch's records and static body data: no thread of this
        // batch writes them (a record belongs to its own thread)
        if (k + 1 < steps) {
            g = group_of((k + 1) % G, nb, V.maxBatch);
            q0 = (int)V.groupOffset[g];
            q1 = (int)V.groupOffset[g + 1];
            fetch(V, q0 + tid < q1 ? q0 + tid : -1, P);
        }
        if (!grid_barrier(V.bar, V.bar + 1, gridDim.x, V.err, V.counters)) return;
    }
}

int cooperative_grid(const void* kern, int threads, int numSMs, long long work) {
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, 0) != cudaSuccess || occ < 1) occ = 1;
    const long long want = std::max<long long>(1, (work + threads - 1) / threads);
    return (int)std::min<long long>((long long)numSMs * occ, want);
}

int launch_cooperative(const void* kern, int grid, int threads, void** args, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    B3_CUDA(cudaLaunchKernelExC(&cfg, kern, args));
    return B3_OK;
}

}  // namespace

namespace b3 {

int launch_gs_solver(b3World_t* w, cudaStream_t st) {
    if (w->cfg.maxPairs == 0 || w->bodies.empty()) return B3_OK;
    auto& d = w->d;
    const int N = (int)w->bodies.size();
    const int cap = w->cfg.maxPairs;
    const int maxBatch = kGsMaxBatch;
    const int32_t* M = d.scalars + S_NUM_MANIFOLDS;
    const int g = w->ctx->numSMs * 8;
    // 1. cells and classes, sorted by (class, cell)
    k_gs_keys<<<g, 256, 0, st>>>(d.contacts, d.manifoldPair, M, d.pos, d.invMass, d.incKeys, d.incVals, d.gsCell);
    B3_CHECK_LAUNCH();
    bool alt = false;
    B3_TRY(radix_sort_pairs(d.incKeys, d.incVals, d.incKeysAlt, d.incValsAlt, M, cap, 10, d.incSortScratch,
                            d.incSortScratchBytes, d.scalars + S_ERR, st, &alt, w->ctx->numSMs));
    const uint32_t* keys = alt ? d.incKeysAlt : d.incKeys;
    const uint32_t* vals = alt ? d.incValsAlt : d.incVals;
    // 2. colouring
    B3_CUDA(cudaMemsetAsync(d.gsMinRank, 0x7f, sizeof(int) * 4 * (size_t)N, st));  // 0x7f7f7f7f: no rank
    B3_CUDA(cudaMemsetAsync(d.gsTaken, 0, sizeof(int) * 4 * (size_t)N, st));
    B3_CUDA(cudaMemsetAsync(d.scalars + S_BAR_COUNT, 0, sizeof(int32_t) * 2, st));
    ColourView CV;
    CV.keys = keys;
    CV.vals = vals;
    CV.contacts = d.contacts;
    CV.manifoldPair = d.manifoldPair;
    CV.invMass = d.invMass;
    CV.numManifolds = M;
    CV.numBodies = N;
    CV.minRank = d.gsMinRank;
    CV.taken = d.gsTaken;
    CV.slotBatch = d.gsSlotBatch;
    CV.batchCount = d.gsBatchCount;
    CV.roundCount = d.gsBatchCount + 4;  // 5 more ints
    CV.bar = (uint32_t*)(d.scalars + S_BAR_COUNT);
    CV.err = d.scalars + S_ERR;
    CV.counters = d.counters;
    CV.maxBatch = maxBatch;
    const long long estM = std::min<long long>((long long)cap, 3LL * N);
    {
        // the narrow width of the solve (solverMode 1) also narrows the
        // colouring: each round passes over every slot, but costs three
        // barriers
        const int grid = cooperative_grid((const void*)k_gs_colour, 256, w->ctx->numSMs,
                                          w->solverMode == 1 ? estM / 8 : estM);
        void* args[] = {&CV};
        B3_TRY(launch_cooperative((const void*)k_gs_colour, grid, 256, args, st));
    }
    // 3. groups (class, batch): counts, offsets, constraints
    const int groups = 4 * maxBatch;
    B3_CUDA(cudaMemsetAsync(d.gsGroupCount, 0, sizeof(uint32_t) * groups, st));
    B3_CUDA(cudaMemsetAsync(d.gsGroupFill, 0, sizeof(uint32_t) * groups, st));
    k_gs_count<<<g, 256, 0, st>>>(keys, d.gsSlotBatch, M, maxBatch, d.gsGroupCount);
    B3_CHECK_LAUNCH();
    k_gs_offsets<<<1, 1024, 0, st>>>(d.gsGroupCount, d.gsGroupOffset, groups);
    B3_CHECK_LAUNCH();
    k_gs_inertia<<<(N + 255) / 256, 256, 0, st>>>(w->bodiesDev(), d.gsInertia);
    B3_CHECK_LAUNCH();
    SetupParams SP;
    SP.dtInv = 1.f / w->sim.dt;
    SP.maxBatch = maxBatch;
    k_gs_setup<<<g, 128, 0, st>>>(keys, vals, d.gsSlotBatch, M, d.gsGroupOffset, d.gsGroupFill, d.contacts,
                                  d.manifoldPair, w->bodiesDev(), d.gsInertia, d.gsConstraints, d.gsSlotOfManifold,
                                  SP);
    B3_CHECK_LAUNCH();
    // 4. Gauss-Seidel iterations
    B3_CUDA(cudaMemsetAsync(d.scalars + S_BAR_COUNT, 0, sizeof(int32_t) * 2, st));
    SolveView SV;
    SV.cs = d.gsConstraints;
    SV.groupOffset = d.gsGroupOffset;
    SV.batchCount = d.gsBatchCount;
    SV.maxBatch = maxBatch;
    SV.pos = d.pos;
    SV.linVel = d.linVel;
    SV.angVel = d.angVel;
    SV.invMass = d.invMass;
    SV.Iw = d.gsInertia;
    SV.bar = (uint32_t*)(d.scalars + S_BAR_COUNT);
    SV.err = d.scalars + S_ERR;
    SV.counters = d.counters;
    {
        // a batch holds a fraction of the manifolds, and fewer blocks make
        // each grid barrier cheaper: the autotuner picks the width
        // (solverMode 0: manifolds / 8 threads, 1: manifolds / 64)
        const void* kg = (const void*)k_gs_solve;
        const int grid = cooperative_grid(kg, 256, w->ctx->numSMs, estM / (w->solverMode == 1 ? 64 : 8));
        void* args[] = {&SV};
        B3_TRY(launch_cooperative(kg, grid, 256, args, st));
    }
    return B3_OK;
}

}  // namespace b3

extern "C" int b3_solver_solve_batched_gs(b3World w, void* stream) {
    if (!w) return B3_ERR_INVALID_ARG;
    if (!w->gs) {
        b3_set_error("the world was not created with B3_WORLD_BATCHED_GS_SOLVER");
        return B3_ERR_STATE;
    }
    return b3_stage_solve(w, stream);
}

extern "C" int b3_get_gs_batches(b3World w, int32_t* cellBatch2, int max, int* count, void* stream) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    if (!w->gs) return B3_ERR_STATE;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = (cudaStream_t)stream;
    int32_t nm = 0;
    B3_CUDA(cudaMemcpyAsync(&nm, w->d.scalars + b3::S_NUM_MANIFOLDS, 4, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    *count = nm;
    if (!cellBatch2 || nm <= 0 || max <= 0) return B3_OK;
    const int n = std::min(nm, max);
    std::vector<int> cell(nm), slot(nm);
    std::vector<b3Constraint4> cs(nm);
    B3_CUDA(cudaMemcpyAsync(cell.data(), w->d.gsCell, 4 * (size_t)nm, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaMemcpyAsync(slot.data(), w->d.gsSlotOfManifold, 4 * (size_t)nm, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaMemcpyAsync(cs.data(), w->d.gsConstraints, sizeof(b3Constraint4) * (size_t)nm,
                            cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < n; ++m) {
        cellBatch2[2 * m] = cell[m];
        cellBatch2[2 * m + 1] = slot[m] >= 0 && slot[m] < nm ? cs[slot[m]].batchIdx : -1;
    }
    return B3_OK;
}

extern "C" int b3_get_gs_constraints(b3World w, b3Constraint4* out, int max, int* count, void* stream) {
    if (!w || !count) return B3_ERR_INVALID_ARG;
    if (!w->gs) return B3_ERR_STATE;
    if (!w->written) return B3_ERR_STATE;
    cudaStream_t st = (cudaStream_t)stream;
    int32_t nm = 0;
    B3_CUDA(cudaMemcpyAsync(&nm, w->d.scalars + b3::S_NUM_MANIFOLDS, 4, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    *count = nm;
    if (!out || nm <= 0 || max <= 0) return B3_OK;
    std::vector<int> slot(nm);
    std::vector<b3Constraint4> cs(nm);
    B3_CUDA(cudaMemcpyAsync(slot.data(), w->d.gsSlotOfManifold, 4 * (size_t)nm, cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaMemcpyAsync(cs.data(), w->d.gsConstraints, sizeof(b3Constraint4) * (size_t)nm,
                            cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < std::min(nm, max); ++m) out[m] = slot[m] >= 0 && slot[m] < nm ? cs[slot[m]] : b3Constraint4{};
    return B3_OK;
}
