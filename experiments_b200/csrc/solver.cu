// Contact-to-constraint setup, Jacobi contact/friction solver with velocity
// averaging, and transform integration, for sm_100a.
//
// Solver semantics are btPgsJacobiSolver with usePgs = false
// (P2/btPgsJacobiSolver.cpp:35), as solveContacts configures it (:171-191):
// 10 iterations, splitImpulse off, erp 0.2, linearSlop 0, solver mode
// WARMSTARTING | SIMD | USE_2_FRICTION_DIRECTIONS (btContactSolverInfo.h:72-90
// defaults plus :180), which means
//   * one solver-body copy per (manifold, dynamic body); a static body is a
//     single shared solver body with zero inverse mass (getOrInitSolverBody
//     :689-722); m_bodyCount[b] = number of manifolds touching b (:1105-1129)
//   * per point (skipped if depth + 0.01 > 0.02, :124-155 and :961):
//     normal row (setupContactConstraint :725-888) with Baumgarte rhs and the
//     count-scaled denominator relaxation/(d0*countA + d1*countB), then two
//     friction rows, direction 2 first, along the relative tangential velocity
//     when its squared length exceeds FLT_EPSILON, else btPlaneSpace1(n)
//     (convertContact :933-1080, setupFrictionConstraint :505-592)
//   * inverse inertia used by the rows is the body's local diagonal inverse
//     inertia (getInvInertiaTensorWorld returns m_initInvInertia, :51-66)
//   * each iteration: all normal rows (lower limit 0), averageVelocities,
//     all friction rows clamped to +-mu*lambda_n (skipped while lambda_n <= 0),
//     averageVelocities (solveSingleIteration :1372-1614,
//     solveGroupCacheFriendlyIterations :1656-1681, averageVelocities :1683-1720)
//   * finish: every copy of a dynamic body adds sum/count to the body
//     velocity (solveGroupCacheFriendlyFinish :1790-1803), so a body with k
//     copies receives k times the averaged delta.
// Impulses reach every solver body (the SIMD row solvers used by this
// solver mode have no per-body guard).
//
// B200 mapping: rows within a copy are Gauss-Seidel, copies are independent,
// so one thread owns one manifold and solves its rows in order, keeping the
// two copies' delta velocities in registers. The per-body average is a
// deterministic segmented sum over the body's copies in manifold order (the
// copy list is a stable radix sort of (body, copy) entries). All 4 phases x
// iterations run in one persistent cooperative kernel separated by a grid
// barrier whose wait is bounded. Rows are stored structure-of-arrays
// (row slot major) so each phase streams them with coalesced float4 loads.
#include "solver_common.cuh"

#include <algorithm>
#include <cfloat>

using namespace b3m;
using namespace b3solver;

namespace {

// ---------------------------------------------------------------------------
// Manifold compaction: manifold index = exclusive scan of per-pair flags.
// ---------------------------------------------------------------------------
__global__ void k_manifold_emit(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ scan,
                                const int32_t* __restrict__ numPairsDev,
                                const b3Contact4* __restrict__ contacts, const float* __restrict__ invMass,
                                int numBodies, int* __restrict__ manifoldPair,
                                uint32_t* __restrict__ incKeys, uint32_t* __restrict__ incVals,
                                int32_t* __restrict__ scalars, b3Counters* __restrict__ counters) {
    const int np = *numPairsDev;
    const int M = scalars[b3::S_NUM_MANIFOLDS];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scalars[b3::S_NUM_INC] = 2 * M;
        counters->numManifolds = M;
    }
    int pts = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        if (!flag[p]) continue;
        const int m = (int)scan[p];
        manifoldPair[m] = p;
        const b3Contact4& c = contacts[p];
        const int a = abs(c.bodyAPtrAndSignBit), b = abs(c.bodyBPtrAndSignBit);
        // copies exist for dynamic bodies only; static ones get the
        // out-of-range key numBodies and sort past every body
        incKeys[2 * m] = invMass[a] != 0.f ? (uint32_t)a : (uint32_t)numBodies;
        incVals[2 * m] = 2u * m;
        incKeys[2 * m + 1] = invMass[b] != 0.f ? (uint32_t)b : (uint32_t)numBodies;
        incVals[2 * m + 1] = 2u * m + 1u;
        pts += (int)c.worldNormal[3];
    }
    if (pts) atomicAdd(&counters->numContactPoints, pts);
}

__global__ void k_body_ranges(const uint32_t* __restrict__ keys, const int32_t* __restrict__ nDev,
                              uint32_t* __restrict__ start, uint32_t* __restrict__ end, int numBodies) {
    const int n = *nDev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        if (k >= (uint32_t)numBodies) continue;
        if (i == 0 || keys[i - 1] != k) start[k] = (uint32_t)i;
        if (i == n - 1 || keys[i + 1] != k) end[k] = (uint32_t)(i + 1);
    }
}

// ---------------------------------------------------------------------------
// Constraint setup (one thread per manifold)
// ---------------------------------------------------------------------------
struct SetupParams {
    float dt;
    float erp;
    float contactProcessing;
    float slopOffset;
};

__device__ __forceinline__ void setup_friction_row(const SolverView& V, int slot, int m, float3 dir,
                                                   float3 r1, float3 r2, float imA, float imB,
                                                   float3 iiA, float3 iiB, float cA, float cB,
                                                   float3 vA, float3 wA, float3 vB, float3 wB) {
    const float3 t1 = cross(r1, dir);
    const float3 t2 = cross(r2, -dir);
    const float3 angA = mulv(iiA, t1);
    const float3 angB = mulv(iiB, t2);
    const float d0 = imA + dot(dir, cross(angA, r1));
    const float d1 = imB + dot(dir, cross(-angB, r2));
    const float denom = 1.f / (d0 + d1);
    const float scaled = 1.f / (d0 * cA + d1 * cB);
    const float relv = (dot(dir, vA) + dot(t1, wA)) + (-dot(dir, vB) + dot(t2, wB));
    const float rhs = (0.f - relv) * scaled;
    R(V, slot + 0, m) = make_float4(dir.x, dir.y, dir.z, rhs);
    R(V, slot + 1, m) = make_float4(t1.x, t1.y, t1.z, denom);
    R(V, slot + 2, m) = make_float4(t2.x, t2.y, t2.z, 0.f);
}

__global__ void k_setup_rows(b3::BodiesDev Bd, SolverView V, const int* __restrict__ manifoldPair,
                             const b3Contact4* __restrict__ contacts, SetupParams SP) {
    const int M = *V.numManifolds;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const b3Contact4 c = contacts[manifoldPair[m]];
        const int A = abs(c.bodyAPtrAndSignBit), B = abs(c.bodyBPtrAndSignBit);
        const float imA = Bd.invMass[A], imB = Bd.invMass[B];
        const bool dynA = imA != 0.f, dynB = imB != 0.f;
        const float kA = dynA ? (float)(V.incEnd[A] - V.incStart[A]) : 1.f;
        const float kB = dynB ? (float)(V.incEnd[B] - V.incStart[B]) : 1.f;
        const float3 iiA = dynA ? f3(Bd.invInertia[A]) : make_float3(0.f, 0.f, 0.f);
        const float3 iiB = dynB ? f3(Bd.invInertia[B]) : make_float3(0.f, 0.f, 0.f);
        const float3 pA = f3(Bd.pos[A]), pB = f3(Bd.pos[B]);
        // solver body velocities (static bodies contribute zero)
        const float3 vA = dynA ? f3(Bd.linVel[A]) : make_float3(0.f, 0.f, 0.f);
        const float3 wA = dynA ? f3(Bd.angVel[A]) : make_float3(0.f, 0.f, 0.f);
        const float3 vB = dynB ? f3(Bd.linVel[B]) : make_float3(0.f, 0.f, 0.f);
        const float3 wB = dynB ? f3(Bd.angVel[B]) : make_float3(0.f, 0.f, 0.f);
        const float restitution = Bd.restitution[A] * Bd.restitution[B];
        const float mu = c.friction;
        int nRows = 0;
        const int npts = (int)c.worldNormal[3];
        const bool solve = dynA || dynB;
        float3 n = normalize(make_float3(-c.worldNormal[0], -c.worldNormal[1], -c.worldNormal[2]));
        for (int j = 0; j < npts && solve; ++j) {
            const float depth = c.worldPos[j][3];
            const float dist = depth + SP.slopOffset;
            if (!(dist <= SP.contactProcessing)) continue;
            const float3 posB = make_float3(c.worldPos[j][0], c.worldPos[j][1], c.worldPos[j][2]);
            const float3 posA = posB + n * dist;
            const float3 r1 = posA - pA;
            const float3 r2 = posB - pB;
            const float3 t0 = cross(r1, n);
            const float3 t1 = cross(r2, n);
            const float3 angA = mulv(iiA, t0);
            const float3 angB = mulv(iiB, -t1);
            const float d0 = imA + dot(n, cross(angA, r1));
            const float d1 = imB + dot(n, cross(-angB, r2));
            const float denom = 1.f / (d0 + d1);
            const float scaled = 1.f / (d0 * kA + d1 * kB);
            const float penetration = dist;  // + linearSlop (0)
            const float3 vel1 = vA + cross(wA, r1);
            const float3 vel2 = vB + cross(wB, r2);
            const float3 vel = vel1 - vel2;
            const float relv0 = dot(n, vel);
            float rest = restitution * -relv0;
            if (rest <= 0.f) rest = 0.f;
            const float v1n = dot(n, vA) + dot(t0, wA);
            const float v2n = -dot(n, vB) + dot(-t1, wB);
            const float relv = v1n + v2n;
            float posErr = 0.f;
            float velErr = rest - relv;
            if (penetration > 0.f) {
                velErr -= penetration / SP.dt;
            } else {
                posErr = -penetration * SP.erp / SP.dt;
            }
            const float rhs = posErr * scaled + velErr * scaled;
            const int s = kNormal0 + 3 * nRows;
            R(V, s + 0, m) = make_float4(n.x, n.y, n.z, rhs);
            R(V, s + 1, m) = make_float4(t0.x, t0.y, t0.z, denom);
            R(V, s + 2, m) = make_float4(-t1.x, -t1.y, -t1.z, 0.f);
            // friction directions (convertContact :1015-1049)
            float3 d1v = vel - n * relv0;
            const float lat = dot(d1v, d1v);
            float3 d2v;
            if (lat > FLT_EPSILON) {
                d1v = d1v * (1.f / sqrtf(lat));
                d2v = normalize(cross(d1v, n));
            } else {
                plane_space(n, d1v, d2v);
            }
            const int fs = kFric0 + 3 * (2 * nRows);
            setup_friction_row(V, fs, m, d2v, r1, r2, imA, imB, iiA, iiB, kA, kB, vA, wA, vB, wB);
            setup_friction_row(V, fs + 3, m, d1v, r1, r2, imA, imB, iiA, iiB, kA, kB, vA, wA, vB, wB);
            ++nRows;
        }
        R(V, 0, m) = make_float4(__int_as_float(A), __int_as_float(B), __int_as_float(nRows),
                                 __int_as_float((dynA ? 1 : 0) | (dynB ? 2 : 0)));
        R(V, 1, m) = make_float4(imA, imB, mu, 0.f);
        R(V, 2, m) = make_float4(iiA.x, iiA.y, iiA.z, kA);
        R(V, 3, m) = make_float4(iiB.x, iiB.y, iiB.z, kB);
    }
}

// ---------------------------------------------------------------------------
// Persistent Jacobi kernel
// ---------------------------------------------------------------------------
constexpr int kJacobiHeads = 4;         // manifolds per thread whose headers stay in shared memory
constexpr int kJacobiMaxThreads = 256;  // k_jacobi's largest CTA

// What a manifold's solve reads that no phase changes: its header (bodies,
// row count, dynamic flags) and its bodies' incidence ranges.
struct MHead {
    int A, B, nRows, dyn;
    uint32_t sA, eA, sB, eB;
};

__device__ __forceinline__ void load_head(const SolverView& V, int m, MHead& H) {
    const float4 h0 = R(V, 0, m);
    H.nRows = __float_as_int(h0.z);
    H.A = __float_as_int(h0.x);
    H.B = __float_as_int(h0.y);
    H.dyn = __float_as_int(h0.w);
    H.sA = H.eA = H.sB = H.eB = 0u;
    if (H.dyn & 1) {
        H.sA = V.incStart[H.A];
        H.eA = V.incEnd[H.A];
    }
    if (H.dyn & 2) {
        H.sB = V.incStart[H.B];
        H.eB = V.incEnd[H.B];
    }
}

// One phase for one manifold: start each copy from its body's average of
// the previous phase (zero in the first phase), solve the manifold's normal
// or friction rows in order, store both copies in buffer outBuf. A copy of a
// manifold without rows keeps the average, as in the reference.
template <bool TAPE, bool GATHER4>
__device__ __forceinline__ void solve_manifold_h(const SolverView& V, int m, const MHead& H, bool friction,
                                                 bool first, int inBuf, int outBuf, const b3::JacobiTape& T,
                                                 int phase) {
    {
        const int nRows = H.nRows;
        const int dyn = H.dyn;
        float3 dvA = make_float3(0.f, 0.f, 0.f), dwA = dvA, dvB = dvA, dwB = dvA;
        if (!first) {
            if (GATHER4) {
                // the copies four at a time (same sums as body_average)
                if (dyn & 1) body_average_range(V, H.sA, H.eA, inBuf, dvA, dwA);
                if (dyn & 2) body_average_range(V, H.sB, H.eB, inBuf, dvB, dwB);
            } else {
                if (dyn & 1) body_average_se(V, H.sA, H.eA, inBuf, dvA, dwA);
                if (dyn & 2) body_average_se(V, H.sB, H.eB, inBuf, dvB, dwB);
            }
        }
        float lam[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (nRows > 0) {
            const float4 h1 = R(V, 1, m);
            const float4 h2 = R(V, 2, m);
            const float4 h3 = R(V, 3, m);
            const float imA = h1.x, imB = h1.y, mu = h1.z;
            const float3 iiA = f3(h2), iiB = f3(h3);
            if (!friction) {
                for (int j = 0; j < nRows; ++j) {
                    const int s = kNormal0 + 3 * j;
                    const float4 r0 = R(V, s, m), r1 = R(V, s + 1, m);
                    float4 r2 = R(V, s + 2, m);
                    solve_row(r0, r1, r2, 0.f, 1e10f, imA, imB, iiA, iiB, dvA, dwA, dvB, dwB);
                    R(V, s + 2, m).w = r2.w;
                    if (TAPE) lam[j] = r2.w;
                }
            } else {
                for (int j = 0; j < nRows; ++j) {
                    const float total = R(V, kNormal0 + 3 * j + 2, m).w;
                    if (TAPE) {
                        lam[2 * j] = R(V, kFric0 + 3 * (2 * j) + 2, m).w;
                        lam[2 * j + 1] = R(V, kFric0 + 3 * (2 * j + 1) + 2, m).w;
                    }
                    if (!(total > 0.f)) continue;
                    const float lim = mu * total;
                    for (int q = 0; q < 2; ++q) {
                        const int s = kFric0 + 3 * (2 * j + q);
                        const float4 r0 = R(V, s, m), r1 = R(V, s + 1, m);
                        float4 r2 = R(V, s + 2, m);
                        solve_row(r0, r1, r2, -lim, lim, imA, imB, iiA, iiB, dvA, dwA, dvB, dwB);
                        R(V, s + 2, m).w = r2.w;
                        if (TAPE) lam[2 * j + q] = r2.w;
                    }
                }
            }
        }
        if (dyn & 1) {
            const size_t at = (size_t)(outBuf * 2 + 0) * V.cap + m;
            V.copyLin[at] = f4(dvA);
            V.copyAng[at] = f4(dwA);
        }
        if (dyn & 2) {
            const size_t at = (size_t)(outBuf * 2 + 1) * V.cap + m;
            V.copyLin[at] = f4(dvB);
            V.copyAng[at] = f4(dwB);
        }
        if (TAPE) {
            // every phase's copies and the impulses after it, for the
            // reverse sweep (both sides, zero for a static side)
            const size_t a0 = (size_t)(phase * 2 + 0) * V.cap + m, a1 = (size_t)(phase * 2 + 1) * V.cap + m;
            T.copyLin[a0] = f4(dvA);
            T.copyAng[a0] = f4(dwA);
            T.copyLin[a1] = f4(dvB);
            T.copyAng[a1] = f4(dwB);
            const int it = phase >> 1;
            if (!friction) {
                T.lamN[(size_t)it * V.cap + m] = make_float4(lam[0], lam[1], lam[2], lam[3]);
            } else {
                T.lamF[(size_t)(2 * it) * V.cap + m] = make_float4(lam[0], lam[1], lam[2], lam[3]);
                T.lamF[(size_t)(2 * it + 1) * V.cap + m] = make_float4(lam[4], lam[5], lam[6], lam[7]);
            }
        }
    }
}

template <bool TAPE, bool GATHER4>
__device__ __forceinline__ void solve_manifold(const SolverView& V, int m, bool friction, bool first, int inBuf,
                                               int outBuf, const b3::JacobiTape& T, int phase) {
    MHead H;
    load_head(V, m, H);
    solve_manifold_h<TAPE, GATHER4>(V, m, H, friction, first, inBuf, outBuf, T, phase);
}

template <bool TAPE, bool GATHER4>
__device__ void manifold_phase(const SolverView& V, int M, bool friction, bool first, int inBuf, int outBuf,
                               const b3::JacobiTape& T, int phase) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x)
        solve_manifold<TAPE, GATHER4>(V, m, friction, first, inBuf, outBuf, T, phase);
}

// Phases p = 0 .. 2*iterations-1 alternate normal (even) and friction (odd)
// rows; the averaging of the reference happens at the start of the next
// phase from the double-buffered copies, so phases are separated by one
// bounded grid barrier each.
//
// GATHER4 (a tuning choice): each copy's body averages are gathered with
// their loads issued four at a time. Shorter dependent-load chains per
// phase, more registers per thread: the autotuner weighs the two.
template <bool TAPE, bool GATHER4>
__global__ void __launch_bounds__(256)
k_jacobi(SolverView V, int iterations, uint32_t* bar, int32_t* err, b3Counters* counters, b3::JacobiTape T) {
    const int M = *V.numManifolds;
    const uint32_t nb = gridDim.x;
    const int phases = 2 * iterations;
    const int m0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    // the headers and incidence ranges of this thread's first kJacobiHeads
    // manifolds stay in shared memory for every phase: after each barrier
    // only the copy ids and the copies remain to be loaded from L2
    __shared__ MHead heads[kJacobiHeads][kJacobiMaxThreads];
    for (int k = 0; k < kJacobiHeads; ++k)
        if (m0 + k * stride < M) load_head(V, m0 + k * stride, heads[k][threadIdx.x]);
    for (int p = 0; p < phases; ++p) {
        if (p == 1 && V.holdMicros > 0 && blockIdx.x == 0 && threadIdx.x == 0) {
            // test of the give-up path: block 0 arrives late (bounded sleep)
            for (int i = 0; i < V.holdMicros; ++i) __nanosleep(1000);
        }
        if (p > 0 && !grid_barrier(bar, bar + 1, nb, err, counters, V.spinLimit)) return;
        const bool friction = (p & 1) != 0, first = p == 0;
        const int inBuf = (p - 1) & 1, outBuf = p & 1;
        int k = 0;
        for (int m = m0; m < M; m += stride, ++k) {
            MHead H;
            if (k < kJacobiHeads) H = heads[k][threadIdx.x];
            else load_head(V, m, H);
            solve_manifold_h<TAPE, GATHER4>(V, m, H, friction, first, inBuf, outBuf, T, p);
        }
    }
}

// Batched worlds: the manifolds of one world are contiguous (the pair list
// follows the world-major cell keys) and touch only that world's bodies, so
// a block can run all phases of a world by itself with block barriers in
// place of grid barriers. Same per-manifold arithmetic and averaging order
// as k_jacobi, hence bit-identical results.
// Span [start, end) of each world's manifolds. When a world's manifolds are
// not contiguous (pairs between two large bodies come after the tiles) the
// span covers foreign manifolds, which k_jacobi_worlds skips: every
// manifold is still solved by its own world's block only.
__global__ void k_world_ranges(SolverView V, const int* __restrict__ worldId, int* __restrict__ start,
                               int* __restrict__ end) {
    const int M = *V.numManifolds;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const int w = worldId[__float_as_int(R(V, 0, m).x)];
        if (m == 0 || worldId[__float_as_int(R(V, 0, m - 1).x)] != w) atomicMin(&start[w], m);
        if (m == M - 1 || worldId[__float_as_int(R(V, 0, m + 1).x)] != w) atomicMax(&end[w], m + 1);
    }
}

template <bool TAPE, bool GATHER4>
__global__ void __launch_bounds__(256)
k_jacobi_worlds(SolverView V, int iterations, const int* __restrict__ start, const int* __restrict__ end,
                int numWorlds, const int* __restrict__ worldId, b3::JacobiTape T) {
    const int phases = 2 * iterations;
    for (int w = blockIdx.x; w < numWorlds; w += gridDim.x) {
        const int s = start[w], e = end[w];
        if (s >= e) continue;
        for (int p = 0; p < phases; ++p) {
            if (p > 0) __syncthreads();
            for (int m = s + (int)threadIdx.x; m < e; m += blockDim.x)
                if (worldId[__float_as_int(R(V, 0, m).x)] == w)
                    solve_manifold<TAPE, GATHER4>(V, m, (p & 1) != 0, p == 0, (p - 1) & 1, p & 1, T, p);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Integration (copyVelocitiesKernel + integrateTransformsKernel2)
// ---------------------------------------------------------------------------
struct IntegrateParams {
    float dt;
    float damping;
    float threshold;  // BT_GPU_ANGULAR_MOTION_THRESHOLD = 0.25 * pi
};

__global__ void k_integrate(b3::BodiesDev Bd, SolverView V, int finalBuf, IntegrateParams P, int applySolve) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Bd.n) return;
    if (Bd.invMass[i] == 0.f) return;
    float4 v = Bd.linVel[i];
    float4 w = Bd.angVel[i];
    // solveGroupCacheFriendlyFinish (:1790-1803): each of the k copies adds
    // sum/k of the last averaging to the body velocity
    if (applySolve && V.incEnd[i] > V.incStart[i]) {
        const uint32_t k = V.incEnd[i] - V.incStart[i];
        float3 sl, sa;
        body_average(V, i, finalBuf, sl, sa);
        for (uint32_t c = 0; c < k; ++c) {
            v.x += sl.x; v.y += sl.y; v.z += sl.z;
            w.x += sa.x; w.y += sa.y; w.z += sa.z;
        }
    }
    v.w = 0.f;
    w.x *= P.damping;
    w.y *= P.damping;
    w.z *= P.damping;
    w.w = 0.f;
    float fAngle = sqrtf(w.x * w.x + w.y * w.y + w.z * w.z);
    if (fAngle * P.dt > P.threshold) fAngle = P.threshold / P.dt;
    float s;
    if (fAngle < 0.001f) {
        s = 0.5f * P.dt - (P.dt * P.dt * P.dt) * 0.020833333333f * fAngle * fAngle;
    } else {
        s = sinf(0.5f * fAngle * P.dt) / fAngle;
    }
    const float4 dorn = make_float4(w.x * s, w.y * s, w.z * s, cosf(fAngle * P.dt * 0.5f));
    const float4 q0 = Bd.quat[i];
    float4 q = quat_mult(dorn, q0);
    const float len = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (len > 0.f) {
        const float il = 1.f / len;
        q.x *= il; q.y *= il; q.z *= il; q.w *= il;
    } else {
        q = make_float4(0.f, 0.f, 0.f, 1.f);
    }
    float4 p = Bd.pos[i];
    p.x += v.x * P.dt;
    p.y += v.y * P.dt;
    p.z += v.z * P.dt;
    Bd.pos[i] = p;
    Bd.quat[i] = q;
    Bd.linVel[i] = v;
    Bd.angVel[i] = w;
}

}  // namespace

SolverView b3solver::solver_view(b3World_t* w) {
    SolverView V;
    V.rows = w->d.rows;
    V.cap = w->cfg.maxPairs;
    V.copyLin = w->d.incLin;
    V.copyAng = w->d.incAng;
    V.avgLin = w->d.avgLin;
    V.avgAng = w->d.avgAng;
    V.incVals = w->d.incVals;
    V.incStart = w->d.bodyIncStart;
    V.incEnd = w->d.bodyIncEnd;
    V.numManifolds = w->d.scalars + b3::S_NUM_MANIFOLDS;
    V.numBodies = (int)w->bodies.size();
    V.spinLimit = w->waitSpinLimit;
    V.holdMicros = w->waitHoldMicros;
    return V;
}

namespace b3 {

int launch_manifolds(b3World_t* w, cudaStream_t st) {
    const int N = (int)w->bodies.size();
    const int cap = w->cfg.maxPairs;
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_NUM_MANIFOLDS, 0, sizeof(int32_t) * 2, st));
    B3_CUDA(cudaMemsetAsync(w->d.bodyIncStart, 0, sizeof(uint32_t) * N, st));
    B3_CUDA(cudaMemsetAsync(w->d.bodyIncEnd, 0, sizeof(uint32_t) * N, st));
    if (cap == 0 || N == 0) return B3_OK;
    // manifold slots: the pairs', then (compound and mesh worlds) the sub-pairs'
    const int32_t* slots = w->d.scalars + (w->hasSubPairs() ? S_NUM_SLOTS : S_NUM_PAIRS);
    B3_TRY(exclusive_scan_u32(w->d.manifoldFlag, w->d.manifoldScan, slots, cap,
                              (uint32_t*)(w->d.scalars + S_NUM_MANIFOLDS), w->d.scanScratch,
                              w->d.scanScratchBytes, w->d.scalars + S_ERR, st, w->ctx->numSMs));
    const int g = w->ctx->numSMs * 8;
    k_manifold_emit<<<g, 256, 0, st>>>(w->d.manifoldFlag, w->d.manifoldScan, slots,
                                      w->d.contacts, w->d.invMass, N, w->d.manifoldPair, w->d.incKeys,
                                      w->d.incVals, w->d.scalars, w->d.counters);
    B3_CHECK_LAUNCH();
    if (w->gs) return B3_OK;  // body incidences serve the Jacobi averaging only
    bool alt = false;
    B3_TRY(radix_sort_pairs(w->d.incKeys, w->d.incVals, w->d.incKeysAlt, w->d.incValsAlt,
                            w->d.scalars + S_NUM_INC, 2LL * cap, w->bodyBits, w->d.incSortScratch,
                            w->d.incSortScratchBytes, w->d.scalars + S_ERR, st, &alt, w->ctx->numSMs));
    if (alt) {
        B3_CUDA(cudaMemcpyAsync(w->d.incKeys, w->d.incKeysAlt, sizeof(uint32_t) * 2 * (size_t)cap,
                                cudaMemcpyDeviceToDevice, st));
        B3_CUDA(cudaMemcpyAsync(w->d.incVals, w->d.incValsAlt, sizeof(uint32_t) * 2 * (size_t)cap,
                                cudaMemcpyDeviceToDevice, st));
    }
    k_body_ranges<<<g, 256, 0, st>>>(w->d.incKeys, w->d.scalars + S_NUM_INC, w->d.bodyIncStart,
                                    w->d.bodyIncEnd, N);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

int launch_solver(b3World_t* w, cudaStream_t st) { return launch_solver_taped(w, st, nullptr); }

int launch_solver_taped(b3World_t* w, cudaStream_t st, const JacobiTape* tape) {
    if (w->cfg.maxPairs == 0 || w->bodies.empty()) return B3_OK;
    if (w->gs) {
        if (tape) {
            b3_set_error("the adjoint form runs the Jacobi solver only");
            return B3_ERR_UNSUPPORTED;
        }
        return launch_gs_solver(w, st);
    }
    SolverView V = solver_view(w);
    SetupParams SP;
    SP.dt = w->sim.dt;
    SP.erp = w->sim.erp;
    SP.contactProcessing = w->sim.contactProcessing;
    SP.slopOffset = w->sim.slopOffset;
    const int g = w->ctx->numSMs * 8;
    k_setup_rows<<<g, 128, 0, st>>>(w->bodiesDev(), V, w->d.manifoldPair, w->d.contacts, SP);
    B3_CHECK_LAUNCH();
    if (w->timing && w->setupEv) B3_CUDA(cudaEventRecord(w->setupEv, st));
    if (w->solverMode == 1 && w->cfg.numWorlds > 1) {
        // one block per world at a time, block barriers between phases
        const int nw = w->cfg.numWorlds;
        B3_CUDA(cudaMemsetAsync(w->d.worldMStart, 0x7f, sizeof(int) * nw, st));  // 0x7f7f7f7f: above any index
        B3_CUDA(cudaMemsetAsync(w->d.worldMEnd, 0, sizeof(int) * nw, st));
        k_world_ranges<<<w->ctx->numSMs * 4, 256, 0, st>>>(V, w->d.worldId, w->d.worldMStart, w->d.worldMEnd);
        B3_CHECK_LAUNCH();
        const int threads = w->solverThreads;
        // the taped forward keeps the plain gather (same results either way)
        const void* kw = tape ? (const void*)k_jacobi_worlds<true, false>
                              : (w->solverGather ? (const void*)k_jacobi_worlds<false, true>
                                                 : (const void*)k_jacobi_worlds<false, false>);
        int occ = 1;
        B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kw, threads, 0));
        occ = occ < 1 ? 1 : occ;
        const int grid = std::min(nw, w->ctx->numSMs * occ);
        int iters = w->sim.iterations;
        int nwv = nw;
        JacobiTape T = tape ? *tape : JacobiTape{};
        int* ws = w->d.worldMStart;
        int* we = w->d.worldMEnd;
        const int* wid = w->d.worldId;
        void* args[] = {&V, &iters, &ws, &we, &nwv, &wid, &T};
        B3_CUDA(cudaLaunchKernel(kw, dim3(grid), dim3(threads), args, 0, st));
        return B3_OK;
    }
    // persistent cooperative Jacobi
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_BAR_COUNT, 0, sizeof(int32_t) * 2, st));
    const int threads = w->solverThreads;
    int occ = 1;
    const void* kern = tape ? (const void*)k_jacobi<true, false>
                            : (w->solverGather ? (const void*)k_jacobi<false, true> : (const void*)k_jacobi<false, false>);
    B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, 0));
    occ = occ < 1 ? 1 : occ;
    occ = occ > w->solverOccCap ? w->solverOccCap : occ;
    // size the persistent grid to the expected manifold count (about 3 per
    // body): fewer blocks make each grid barrier cheaper on small scenes
    const long long est = std::min<long long>((long long)w->cfg.maxPairs, 3LL * (long long)w->bodies.size());
    const int want = (int)std::max<long long>(1, (est + threads - 1) / threads);
    const int grid = std::min(w->ctx->numSMs * occ, want);
    int iters = w->sim.iterations;
    uint32_t* bar = (uint32_t*)(w->d.scalars + S_BAR_COUNT);
    int32_t* err = w->d.scalars + S_ERR;
    b3Counters* ctr = w->d.counters;
    JacobiTape T = tape ? *tape : JacobiTape{};
    void* args[] = {&V, &iters, &bar, &err, &ctr, &T};
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

int launch_integrate(b3World_t* w, cudaStream_t st) {
    const int N = (int)w->bodies.size();
    if (N == 0) return B3_OK;
    IntegrateParams P;
    P.dt = w->sim.dt;
    P.damping = w->sim.angularDamping;
    P.threshold = 0.25f * 3.14159254f;
    const int iters = w->sim.iterations;
    // the batched Gauss-Seidel solver leaves final velocities in the bodies
    k_integrate<<<(N + 255) / 256, 256, 0, st>>>(w->bodiesDev(), solver_view(w), (2 * iters - 1) & 1, P,
                                                iters > 0 && !w->gs ? 1 : 0);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

}  // namespace b3
