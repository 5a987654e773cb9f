// Adjoint (reverse-mode) form of the rigid-body step, for sm_100a.
//
// Gradients of a scalar loss of the final state with respect to the initial
// linear and angular velocities, the masses and the friction coefficients
// of the dynamic bodies, through every step of the plain pipeline:
//
//   integration   x' = x + v2 dt, q' = exp(phi(w2)) q (world-frame exp map
//                 with the 0.25 pi / dt clamp), v2 = v1 + dv, w2 = d (w + dw)
//   Jacobi solve  piecewise linear in the rows: the reverse sweep replays
//                 each phase from its recorded inputs (averaged copies and
//                 impulses) to recover the clamp masks, then runs the rows
//                 backwards; friction bounds carry mu and the normal impulse
//   constraint    rows (n, rhs, r x n, 1/diag) as functions of the contact
//   setup         points, normal, depths, positions, velocities, inverse
//                 masses / inertias: differentiated in forward mode, one
//                 dual-number pass per input, through the same arithmetic
//   contact       points, depths and normal as functions of both poses: each
//   geometry      reduced point is classified as an incident vertex, an
//                 incident edge cut by a side plane of the reference face, or
//                 a corner of two side planes on the incident face plane, and
//                 the normal as a face normal of A or B or an edge-edge cross
//                 product; then differentiated in forward mode over the 12
//                 pose directions (dx, dtheta of both bodies)
//   gravity       v1 = v + g dt (identity for the gradient)
//
// The discrete choices of the step (pair set, separating axis, clip
// topology, point selection, row activity, clamp masks) are held fixed, so
// the gradient is that of the smooth piece the trajectory lies on; finite
// differences agree with it on worlds whose active set does not change.
//
// Memory: body state is checkpointed every K steps; the reverse pass
// recomputes each segment from its checkpoint, storing the K pre-step
// states, then re-runs every step of the segment once more with the Jacobi
// tape (every phase's solver-body copies and impulses) before reversing it.
// The inverse inertia is the inverse mass times a fixed shape factor (the
// registration AABB rule), so its gradient folds into the mass gradient.
#include "solver_common.cuh"

#include <cfloat>
#include <vector>

using namespace b3m;
using namespace b3solver;

namespace {

// the float3 operators stay visible next to the dual-number ones below
using b3m::operator+;
using b3m::operator-;
using b3m::operator*;
using b3m::operator+=;
using b3m::operator-=;

// ---------------------------------------------------------------------------
// Dual numbers (value + one tangent) for the forward-mode derivatives
// ---------------------------------------------------------------------------
struct Du {
    float v, d;
};
__device__ __forceinline__ Du du(float v, float d = 0.f) { return Du{v, d}; }
__device__ __forceinline__ Du operator+(Du a, Du b) { return Du{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Du operator-(Du a, Du b) { return Du{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Du operator-(Du a) { return Du{-a.v, -a.d}; }
__device__ __forceinline__ Du operator*(Du a, Du b) { return Du{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Du operator*(Du a, float s) { return Du{a.v * s, a.d * s}; }
__device__ __forceinline__ Du operator/(Du a, Du b) {
    const float r = 1.f / b.v;
    const float q = a.v * r;
    return Du{q, (a.d - q * b.d) * r};
}
__device__ __forceinline__ Du dsqrt(Du a) {
    const float s = sqrtf(a.v);
    return Du{s, s > 0.f ? 0.5f * a.d / s : 0.f};
}
__device__ __forceinline__ Du drsqrt(Du a) {
    const float r = rsqrtf(a.v);
    return Du{r, -0.5f * a.d * r * r * r};
}

struct D3 {
    Du x, y, z;
};
__device__ __forceinline__ D3 d3(float3 v, float3 t) { return D3{du(v.x, t.x), du(v.y, t.y), du(v.z, t.z)}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator-(D3 a) { return D3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ D3 operator*(D3 a, Du s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Du ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 dmulv(D3 a, D3 b) { return D3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ D3 dnormalize(D3 a) {
    const Du l2 = ddot(a, a);
    return l2.v > 0.f ? a * drsqrt(l2) : a;
}
__device__ __forceinline__ float3 tan3(D3 a) { return make_float3(a.x.d, a.y.d, a.z.d); }

// btPlaneSpace1 in dual numbers (same branches as plane_space)
__device__ void dplane_space(D3 n, D3& p, D3& q) {
    const float SQRT12 = 0.7071067811865475244008443621048490f;
    if (fabsf(n.z.v) > SQRT12) {
        const Du a = n.y * n.y + n.z * n.z;
        const Du k = drsqrt(a);
        p = D3{du(0.f), -n.z * k, n.y * k};
        q = D3{a * k, -n.x * p.z, n.x * p.y};
    } else {
        const Du a = n.x * n.x + n.y * n.y;
        const Du k = drsqrt(a);
        p = D3{-n.y * k, n.x * k, du(0.f)};
        q = D3{-n.z * p.y, n.z * p.x, a * k};
    }
}

// ---------------------------------------------------------------------------
// Adjoint buffers
// ---------------------------------------------------------------------------
constexpr int kContrib = 5;  // float4 per (manifold, side): (gx, gim), (gth, gmu), gv, gw, gii

struct AdjView {
    float4 *gX, *gTh, *gV, *gW;   // per body: adjoint of the state (x, rotation, v, w)
    float4 *gDv, *gDw;            // per body: adjoint of the solver's velocity change
    float* gInvMass;              // per body accumulators over all steps
    float* gMu;
    float4* rowAdj;               // [kRowSlots][cap], layout of the rows
    float4 *gInLin, *gInAng;      // [2 parity][2 sides][cap]: adjoint of each phase's inputs
    float4* gLam;                 // [3][cap]: adjoint of the row impulses
    float4* contrib;              // [kContrib][2 sides][cap]
    int cap;
};

struct StepParams {
    float dt;
    float damping;
    float threshold;
    float3 gravity;
    float erp;
    float contactProcessing;
    float slopOffset;
    int frictionCombine;
    int iterations;
};

// Rodrigues rotation of v by the rotation vector phi
__device__ __forceinline__ float3 rotvec(float3 phi, float3 v) {
    const float a = length(phi);
    if (a < 1e-12f) return v + cross(phi, v);
    const float3 k = phi * (1.f / a);
    const float c = cosf(a), s = sinf(a);
    return v * c + cross(k, v) * s + k * (dot(k, v) * (1.f - c));
}

// ---------------------------------------------------------------------------
// Seeds: dL/dq -> world rotation adjoint 0.5 vec(gq (x) q*)
// ---------------------------------------------------------------------------
__global__ void k_adj_seed(int n, const float4* __restrict__ quat, const float4* __restrict__ gq,
                           float4* __restrict__ gTh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 q = quat[i];
    const float4 g = gq[i];
    const float4 qc = make_float4(-q.x, -q.y, -q.z, q.w);
    const float4 r = quat_mult(g, qc);
    gTh[i] = make_float4(0.5f * r.x, 0.5f * r.y, 0.5f * r.z, 0.f);
}

// ---------------------------------------------------------------------------
// Integration adjoint (one thread per body)
// ---------------------------------------------------------------------------
__global__ void k_adj_integrate(int n, const float* __restrict__ invMass, const float4* __restrict__ angVelPost,
                                const uint32_t* __restrict__ incStart, const uint32_t* __restrict__ incEnd,
                                AdjView A, StepParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || invMass[i] == 0.f) return;
    const float3 gx = f3(A.gX[i]), gth = f3(A.gTh[i]);
    const float3 gvPost = f3(A.gV[i]), gwPost = f3(A.gW[i]);
    const float3 w2 = f3(angVelPost[i]);
    // v2 feeds x' and the next state
    const float3 gv2 = gvPost + gx * P.dt;
    // q' = exp(phi) q: dtheta' = R(phi) dtheta + J_l(phi) dphi
    const float wl = length(w2);
    const bool clamped = wl * P.dt > P.threshold;
    const float ang = clamped ? P.threshold : wl * P.dt;
    const float3 axis = wl > 0.f ? w2 * (1.f / wl) : make_float3(0.f, 0.f, 0.f);
    const float3 phi = axis * ang;
    const float3 gthPre = rotvec(-phi, gth);
    // J_l^T g = g - c1 phi x g + c2 phi x (phi x g)
    float c1, c2;
    if (ang < 1e-3f) {
        c1 = 0.5f - ang * ang / 24.f;
        c2 = 1.f / 6.f - ang * ang / 120.f;
    } else {
        c1 = (1.f - cosf(ang)) / (ang * ang);
        c2 = (ang - sinf(ang)) / (ang * ang * ang);
    }
    const float3 pg = cross(phi, gth);
    const float3 gphi = gth - pg * c1 + cross(phi, pg) * c2;
    float3 gw2 = gwPost;
    if (clamped) {
        // phi = threshold * w2 / |w2|
        gw2 += (gphi - axis * dot(axis, gphi)) * (P.threshold / wl);
    } else {
        gw2 += gphi * P.dt;
    }
    // w2 = damping (w + dw), v2 = v1 + dv (dv, dw only with solver copies)
    const float3 gw = gw2 * P.damping;
    A.gX[i] = f4(gx);
    A.gTh[i] = f4(gthPre);
    A.gV[i] = f4(gv2);
    A.gW[i] = f4(gw);
    const bool solved = incEnd[i] > incStart[i];
    A.gDv[i] = f4(solved ? gv2 : make_float3(0.f, 0.f, 0.f));
    A.gDw[i] = f4(solved ? gw : make_float3(0.f, 0.f, 0.f));
}

// ---------------------------------------------------------------------------
// Jacobi adjoint: persistent cooperative kernel, phases in reverse
// ---------------------------------------------------------------------------
__device__ __forceinline__ void adj_average(const SolverView& V, const float4* gl, const float4* ga, int b, int buf,
                                            float3& lin, float3& ang) {
    const uint32_t s = V.incStart[b], e = V.incEnd[b];
    float3 sl = make_float3(0.f, 0.f, 0.f), sa = sl;
    for (uint32_t i = s; i < e; ++i) {
        const uint32_t cid = V.incVals[i];
        const size_t at = (size_t)(buf * 2 + (int)(cid & 1u)) * V.cap + (cid >> 1);
        sl += f3(gl[at]);
        sa += f3(ga[at]);
    }
    const float factor = 1.f / (float)(e - s);
    lin = sl * factor;
    ang = sa * factor;
}

__device__ __forceinline__ void add4(float4& a, float3 v, float w = 0.f) {
    a.x += v.x; a.y += v.y; a.z += v.z; a.w += w;
}

__device__ void reverse_phase(const SolverView& V, const b3::JacobiTape& T, const AdjView& A, int m, int p,
                              int phases) {
    const float4 h0 = R(V, 0, m);
    const int nRows = __float_as_int(h0.z);
    const int bA = __float_as_int(h0.x), bB = __float_as_int(h0.y);
    const int dyn = __float_as_int(h0.w);
    const bool friction = (p & 1) != 0;
    const bool last = p == phases - 1;
    // adjoint of this phase's copy outputs
    float3 gvA = make_float3(0.f, 0.f, 0.f), gwA = gvA, gvB = gvA, gwB = gvA;
    if (dyn & 1) {
        if (last) { gvA = f3(A.gDv[bA]); gwA = f3(A.gDw[bA]); }
        else adj_average(V, A.gInLin, A.gInAng, bA, (p + 1) & 1, gvA, gwA);
    }
    if (dyn & 2) {
        if (last) { gvB = f3(A.gDv[bB]); gwB = f3(A.gDw[bB]); }
        else adj_average(V, A.gInLin, A.gInAng, bB, (p + 1) & 1, gvB, gwB);
    }
    const size_t cap = (size_t)V.cap;
    float4 gLam0 = last ? make_float4(0.f, 0.f, 0.f, 0.f) : A.gLam[m];
    float4 gLam1 = last ? make_float4(0.f, 0.f, 0.f, 0.f) : A.gLam[cap + m];
    float4 gLam2 = last ? make_float4(0.f, 0.f, 0.f, 0.f) : A.gLam[2 * cap + m];
    if (last) {
        // first touch of this manifold in this step's reverse sweep
        for (int s = 0; s < kRowSlots; ++s) A.rowAdj[(size_t)s * cap + m] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (nRows > 0) {
        const float4 h1 = R(V, 1, m), h2 = R(V, 2, m), h3 = R(V, 3, m);
        const float imA = h1.x, imB = h1.y, mu = h1.z;
        const float3 iiA = f3(h2), iiB = f3(h3);
        // inputs of the phase
        float3 dvA = make_float3(0.f, 0.f, 0.f), dwA = dvA, dvB = dvA, dwB = dvA;
        if (p > 0) {
            SolverView Vt = V;
            Vt.copyLin = T.copyLin;
            Vt.copyAng = T.copyAng;
            if (dyn & 1) body_average(Vt, bA, p - 1, dvA, dwA);
            if (dyn & 2) body_average(Vt, bB, p - 1, dvB, dwB);
        }
        const int it = p >> 1;
        float lam[8], lamN[4] = {0.f, 0.f, 0.f, 0.f};
        if (!friction) {
            const float4 l = it > 0 ? T.lamN[(size_t)(it - 1) * cap + m] : make_float4(0.f, 0.f, 0.f, 0.f);
            lam[0] = l.x; lam[1] = l.y; lam[2] = l.z; lam[3] = l.w;
        } else {
            const float4 l0 = it > 0 ? T.lamF[(size_t)(2 * it - 2) * cap + m] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 l1 = it > 0 ? T.lamF[(size_t)(2 * it - 1) * cap + m] : make_float4(0.f, 0.f, 0.f, 0.f);
            lam[0] = l0.x; lam[1] = l0.y; lam[2] = l0.z; lam[3] = l0.w;
            lam[4] = l1.x; lam[5] = l1.y; lam[6] = l1.z; lam[7] = l1.w;
            const float4 n4 = T.lamN[(size_t)it * cap + m];
            lamN[0] = n4.x; lamN[1] = n4.y; lamN[2] = n4.z; lamN[3] = n4.w;
        }
        // replay: per row the applied change, the clamp state and J.dv
        float dpr[8], jdv[8];
        int st[8];
        const int nr = friction ? 2 * nRows : nRows;
        for (int r = 0; r < nr; ++r) {
            st[r] = -1;  // skipped
            const int j = friction ? (r >> 1) : r;
            float lo = 0.f, hi = 1e10f;
            if (friction) {
                if (!(lamN[j] > 0.f)) continue;
                hi = mu * lamN[j];
                lo = -hi;
            }
            const int s = friction ? kFric0 + 3 * r : kNormal0 + 3 * r;
            const float4 r0 = R(V, s, m), r1 = R(V, s + 1, m), r2 = R(V, s + 2, m);
            const float3 n = f3(r0), t1 = f3(r1), t2 = f3(r2);
            const float rhs = r0.w, jac = r1.w;
            const float dv1 = dot(n, dvA) + dot(t1, dwA);
            const float dv2 = -dot(n, dvB) + dot(t2, dwB);
            jdv[r] = dv1 + dv2;
            float delta = rhs;
            delta -= dv1 * jac;
            delta -= dv2 * jac;
            const float sum = lam[r] + delta;
            float na;
            if (sum < lo) { na = lo; st[r] = 1; }
            else if (sum > hi) { na = hi; st[r] = 2; }
            else { na = sum; st[r] = 0; }
            const float d = na - lam[r];
            dpr[r] = d;
            lam[r] = na;
            dvA += n * (imA * d);
            dwA += mulv(iiA, t1) * d;
            dvB += (-n * imB) * d;
            dwB += mulv(iiB, t2) * d;
        }
        // reverse
        float gl[8];
        if (!friction) { gl[0] = gLam0.x; gl[1] = gLam0.y; gl[2] = gLam0.z; gl[3] = gLam0.w; }
        else {
            gl[0] = gLam1.x; gl[1] = gLam1.y; gl[2] = gLam1.z; gl[3] = gLam1.w;
            gl[4] = gLam2.x; gl[5] = gLam2.y; gl[6] = gLam2.z; gl[7] = gLam2.w;
        }
        float glN[4] = {gLam0.x, gLam0.y, gLam0.z, gLam0.w};
        float gimA = 0.f, gimB = 0.f, gmu = 0.f;
        float3 giiA = make_float3(0.f, 0.f, 0.f), giiB = giiA;
        for (int r = nr - 1; r >= 0; --r) {
            if (st[r] < 0) continue;
            const int j = friction ? (r >> 1) : r;
            const int s = friction ? kFric0 + 3 * r : kNormal0 + 3 * r;
            const float4 r0 = R(V, s, m), r1 = R(V, s + 1, m), r2 = R(V, s + 2, m);
            const float3 n = f3(r0), t1 = f3(r1), t2 = f3(r2);
            const float jac = r1.w;
            const float d = dpr[r];
            const float3 ktA = mulv(iiA, t1), ktB = mulv(iiB, t2);
            // inputs of this row (step back through its update)
            const float3 dvAi = dvA - n * (imA * d), dwAi = dwA - ktA * d;
            const float3 dvBi = dvB + n * (imB * d), dwBi = dwB - ktB * d;
            const float S = imA * dot(n, gvA) + dot(ktA, gwA) - imB * dot(n, gvB) + dot(ktB, gwB);
            float3 gn = (gvA * imA - gvB * imB) * d;
            float3 gt1 = mulv(iiA, gwA) * d;
            float3 gt2 = mulv(iiB, gwB) * d;
            gimA += d * dot(n, gvA);
            gimB -= d * dot(n, gvB);
            giiA += mulv(t1, gwA) * d;
            giiB += mulv(t2, gwB) * d;
            const float gna = gl[r] + S;
            float glIn = -S;
            float grhs = 0.f, gjac = 0.f;
            if (st[r] == 0) {
                glIn += gna;
                const float gdelta = gna;
                grhs = gdelta;
                gjac = -gdelta * jdv[r];
                gn += (dvAi - dvBi) * (-gdelta * jac);
                gt1 += dwAi * (-gdelta * jac);
                gt2 += dwBi * (-gdelta * jac);
                gvA += n * (-gdelta * jac);
                gwA += t1 * (-gdelta * jac);
                gvB += n * (gdelta * jac);
                gwB += t2 * (-gdelta * jac);
            } else if (friction) {
                // bound +-mu * lambda_n
                const float sg = st[r] == 2 ? 1.f : -1.f;
                gmu += sg * lamN[j] * gna;
                glN[j] += sg * mu * gna;
            }
            gl[r] = glIn;
            float4& a0 = A.rowAdj[(size_t)s * cap + m];
            float4& a1 = A.rowAdj[(size_t)(s + 1) * cap + m];
            float4& a2 = A.rowAdj[(size_t)(s + 2) * cap + m];
            add4(a0, gn, grhs);
            add4(a1, gt1, gjac);
            add4(a2, gt2, 0.f);
            dvA = dvAi; dwA = dwAi; dvB = dvBi; dwB = dwBi;
        }
        float4& hA = A.rowAdj[cap + m];
        hA.x += gimA; hA.y += gimB; hA.z += gmu;
        add4(A.rowAdj[2 * cap + m], giiA, 0.f);
        add4(A.rowAdj[3 * cap + m], giiB, 0.f);
        if (!friction) {
            gLam0 = make_float4(gl[0], gl[1], gl[2], gl[3]);
        } else {
            gLam1 = make_float4(gl[0], gl[1], gl[2], gl[3]);
            gLam2 = make_float4(gl[4], gl[5], gl[6], gl[7]);
            gLam0 = make_float4(glN[0], glN[1], glN[2], glN[3]);
        }
    }
    A.gLam[m] = gLam0;
    A.gLam[cap + m] = gLam1;
    A.gLam[2 * cap + m] = gLam2;
    // adjoint of the phase inputs (the averages read at its start)
    if (p > 0) {
        const size_t a0 = (size_t)((p & 1) * 2 + 0) * cap + m, a1 = (size_t)((p & 1) * 2 + 1) * cap + m;
        if (dyn & 1) { A.gInLin[a0] = f4(gvA); A.gInAng[a0] = f4(gwA); }
        if (dyn & 2) { A.gInLin[a1] = f4(gvB); A.gInAng[a1] = f4(gwB); }
    }
}

__global__ void __launch_bounds__(256)
k_jacobi_adjoint(SolverView V, b3::JacobiTape T, AdjView A, int iterations, uint32_t* bar, int32_t* err,
                 b3Counters* counters) {
    const int M = *V.numManifolds;
    const uint32_t nb = gridDim.x;
    const int phases = 2 * iterations;
    for (int p = phases - 1; p >= 0; --p) {
        if (p < phases - 1 && !grid_barrier(bar, bar + 1, nb, err, counters)) return;
        for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x)
            reverse_phase(V, T, A, m, p, phases);
    }
}

// ---------------------------------------------------------------------------
// Constraint-setup and contact-geometry adjoint (one thread per manifold)
// ---------------------------------------------------------------------------
struct SetupIn {
    D3 xA, xB, vA, wA, vB, wB;
    Du imA, imB;
    D3 iiA, iiB;
    D3 n;
    D3 p[4];
    Du depth[4];
};

// k_setup_rows restated in dual numbers; returns the tangent of the rows
// contracted with their adjoint.
__device__ float setup_tangent(const SetupIn& I, const SolverView& V, const AdjView& A, int m, int npts, float kA,
                               float kB, float restitution, const StepParams& P) {
    const size_t cap = (size_t)V.cap;
    float acc = 0.f;
    int nRows = 0;
    for (int j = 0; j < npts; ++j) {
        const Du dist = I.depth[j] + du(P.slopOffset);
        if (!(dist.v <= P.contactProcessing)) continue;
        const D3 n = I.n;
        const D3 posB = I.p[j];
        const D3 posA = posB + n * dist;
        const D3 r1 = posA - I.xA;
        const D3 r2 = posB - I.xB;
        const D3 t0 = dcross(r1, n);
        const D3 t1 = dcross(r2, n);
        const D3 angA = dmulv(I.iiA, t0);
        const D3 angB = dmulv(I.iiB, -t1);
        const Du d0 = I.imA + ddot(n, dcross(angA, r1));
        const Du d1 = I.imB + ddot(n, dcross(-angB, r2));
        const Du denom = du(1.f) / (d0 + d1);
        const Du scaled = du(1.f) / (d0 * kA + d1 * kB);
        const D3 vel1 = I.vA + dcross(I.wA, r1);
        const D3 vel2 = I.vB + dcross(I.wB, r2);
        const D3 vel = vel1 - vel2;
        const Du relv0 = ddot(n, vel);
        Du rest = relv0 * (-restitution);
        if (rest.v <= 0.f) rest = du(0.f);
        const Du v1n = ddot(n, I.vA) + ddot(t0, I.wA);
        const Du v2n = -ddot(n, I.vB) + ddot(-t1, I.wB);
        const Du relv = v1n + v2n;
        Du posErr = du(0.f);
        Du velErr = rest - relv;
        if (dist.v > 0.f) velErr = velErr - dist * (1.f / P.dt);
        else posErr = -dist * (P.erp / P.dt);
        const Du rhs = posErr * scaled + velErr * scaled;
        {
            const int s = kNormal0 + 3 * nRows;
            const float4 g0 = A.rowAdj[(size_t)s * cap + m];
            const float4 g1 = A.rowAdj[(size_t)(s + 1) * cap + m];
            const float4 g2 = A.rowAdj[(size_t)(s + 2) * cap + m];
            acc += dot(f3(g0), tan3(n)) + g0.w * rhs.d + dot(f3(g1), tan3(t0)) + g1.w * denom.d -
                   dot(f3(g2), tan3(t1));
        }
        D3 d1v = vel - n * relv0;
        const Du lat = ddot(d1v, d1v);
        D3 d2v;
        if (lat.v > FLT_EPSILON) {
            d1v = d1v * (du(1.f) / dsqrt(lat));
            d2v = dnormalize(dcross(d1v, n));
        } else {
            dplane_space(n, d1v, d2v);
        }
        for (int q = 0; q < 2; ++q) {
            const D3 dir = q == 0 ? d2v : d1v;
            const D3 ft1 = dcross(r1, dir);
            const D3 ft2 = dcross(r2, -dir);
            const D3 fA = dmulv(I.iiA, ft1);
            const D3 fB = dmulv(I.iiB, ft2);
            const Du e0 = I.imA + ddot(dir, dcross(fA, r1));
            const Du e1 = I.imB + ddot(dir, dcross(-fB, r2));
            const Du fden = du(1.f) / (e0 + e1);
            const Du fsc = du(1.f) / (e0 * kA + e1 * kB);
            const Du frel = (ddot(dir, I.vA) + ddot(ft1, I.wA)) + (-ddot(dir, I.vB) + ddot(ft2, I.wB));
            const Du frhs = -frel * fsc;
            const int s = kFric0 + 3 * (2 * nRows + q);
            const float4 g0 = A.rowAdj[(size_t)s * cap + m];
            const float4 g1 = A.rowAdj[(size_t)(s + 1) * cap + m];
            const float4 g2 = A.rowAdj[(size_t)(s + 2) * cap + m];
            acc += dot(f3(g0), tan3(dir)) + g0.w * frhs.d + dot(f3(g1), tan3(ft1)) + g1.w * fden.d +
                   dot(f3(g2), tan3(ft2));
        }
        ++nRows;
    }
    return acc;
}

// Contact geometry of one manifold as a function of the two poses.
enum PointKind { PK_VERTEX = 0, PK_EDGE = 1, PK_CORNER = 2, PK_ATTACHED = 3 };
enum AxisKind { AX_FACE_A = 0, AX_FACE_B = 1, AX_EDGES = 2, AX_ATTACHED = 3 };

struct GeoPoint {
    int kind;
    int i0, i1;   // vertex / edge endpoints (incident face slots) or planes k, l
    int k;        // side plane for an edge point
    float3 local; // attached fallback: the point in B's frame
};

struct Geo {
    int faceA, faceB;       // reference face (A), incident face (B)
    int axisKind, ax0, ax1; // face index or edge pair
    float axisSign;
    float3 nLocalA;         // fallback: the axis in A's frame
    GeoPoint pt[4];
};

__device__ __forceinline__ float3 vtx(const b3::ShapesDev& S, const b3ConvexPolyhedron& h, int local) {
    return f3(S.verts[h.vertexOffset + local]);
}
__device__ __forceinline__ int face_vertex(const b3::ShapesDev& S, const b3Face& f, int k) {
    return S.indices[f.indexOffset + k];
}

// Pose with a first-order perturbation: world-relative-to-origin vector of a
// body-attached local vector u (rotation part only) and a point.
struct PoseD {
    Mat3 R;
    D3 x;      // position relative to the origin, with tangent
    float3 th; // rotation tangent (dtheta)
};
__device__ __forceinline__ D3 pose_dir(const PoseD& P, float3 u) {
    const float3 r = mul(P.R, u);
    return d3(r, cross(P.th, r));
}
__device__ __forceinline__ D3 pose_point(const PoseD& P, float3 u) { return P.x + pose_dir(P, u); }

// 3 x 3 solve M p = h by Cramer's rule, rows a, b, c
__device__ D3 solve3(D3 a, D3 b, D3 c, Du ha, Du hb, Du hc) {
    const D3 bc = dcross(b, c), ca = dcross(c, a), ab = dcross(a, b);
    const Du det = ddot(a, bc);
    const Du inv = du(1.f) / det;
    return (bc * ha + ca * hb + ab * hc) * inv;
}

__device__ void geo_eval(const Geo& G, const b3::ShapesDev& S, const b3ConvexPolyhedron& hA,
                         const b3ConvexPolyhedron& hB, const PoseD& PA, const PoseD& PB, int npts, D3& nOut,
                         D3* pOut, Du* depthOut) {
    const b3Face fa = S.faces[hA.faceOffset + G.faceA];
    const b3Face fb = S.faces[hB.faceOffset + G.faceB];
    // separating axis
    if (G.axisKind == AX_FACE_A) {
        const b3Face f = S.faces[hA.faceOffset + G.ax0];
        nOut = pose_dir(PA, make_float3(f.plane[0], f.plane[1], f.plane[2])) * du(G.axisSign);
    } else if (G.axisKind == AX_FACE_B) {
        const b3Face f = S.faces[hB.faceOffset + G.ax0];
        nOut = pose_dir(PB, make_float3(f.plane[0], f.plane[1], f.plane[2])) * du(G.axisSign);
    } else if (G.axisKind == AX_EDGES) {
        const D3 ea = pose_dir(PA, f3(S.edges[hA.uniqueEdgesOffset + G.ax0]));
        const D3 eb = pose_dir(PB, f3(S.edges[hB.uniqueEdgesOffset + G.ax1]));
        nOut = dnormalize(dcross(ea, eb)) * du(G.axisSign);
    } else {
        // not matched to a feature: rotates with A
        nOut = pose_dir(PA, G.nLocalA);
    }
    const float3 nAl = make_float3(fa.plane[0], fa.plane[1], fa.plane[2]);
    const D3 nAw = pose_dir(PA, nAl);
    const int nvA = fa.numIndices;
    for (int j = 0; j < npts; ++j) {
        const GeoPoint& g = G.pt[j];
        D3 p;
        if (g.kind == PK_VERTEX) {
            p = pose_point(PB, vtx(S, hB, face_vertex(S, fb, g.i0)));
        } else if (g.kind == PK_EDGE) {
            const D3 a = pose_point(PB, vtx(S, hB, face_vertex(S, fb, g.i0)));
            const D3 b = pose_point(PB, vtx(S, hB, face_vertex(S, fb, g.i1)));
            const float3 va = vtx(S, hA, face_vertex(S, fa, g.k));
            const float3 vb = vtx(S, hA, face_vertex(S, fa, (g.k + 1) % nvA));
            const D3 pn = -dcross(pose_dir(PA, va - vb), nAw);
            const D3 P0 = pose_point(PA, va);
            const D3 u = b - a;
            const Du t = ddot(pn, P0 - a) / ddot(pn, u);
            p = a + u * t;
        } else if (g.kind == PK_CORNER) {
            const float3 ka = vtx(S, hA, face_vertex(S, fa, g.i0));
            const float3 kb = vtx(S, hA, face_vertex(S, fa, (g.i0 + 1) % nvA));
            const float3 la = vtx(S, hA, face_vertex(S, fa, g.i1));
            const float3 lb = vtx(S, hA, face_vertex(S, fa, (g.i1 + 1) % nvA));
            const D3 pk = -dcross(pose_dir(PA, ka - kb), nAw);
            const D3 pl = -dcross(pose_dir(PA, la - lb), nAw);
            const D3 nBw = pose_dir(PB, make_float3(fb.plane[0], fb.plane[1], fb.plane[2]));
            const D3 Pk = pose_point(PA, ka), Pl = pose_point(PA, la);
            const D3 Pb = pose_point(PB, vtx(S, hB, face_vertex(S, fb, 0)));
            p = solve3(pk, pl, nBw, ddot(pk, Pk), ddot(pl, Pl), ddot(nBw, Pb));
        } else {
            p = pose_point(PB, g.local);
        }
        pOut[j] = p;
        depthOut[j] = ddot(nAw, p - PA.x) + du(fa.plane[3]);
    }
}

// The corner of side planes k, l on the incident face plane is well defined
// (the three normals are not close to coplanar).
__device__ bool corner_ok(const b3::ShapesDev& S, const b3ConvexPolyhedron& hA, const b3ConvexPolyhedron& hB,
                          const b3Face& fa, const b3Face& fb, const Mat3& RA, const Mat3& RB, float3 nAw, int k,
                          int l) {
    const int nvA = fa.numIndices;
    const float3 ka = vtx(S, hA, face_vertex(S, fa, k)), kb = vtx(S, hA, face_vertex(S, fa, (k + 1) % nvA));
    const float3 la = vtx(S, hA, face_vertex(S, fa, l)), lb = vtx(S, hA, face_vertex(S, fa, (l + 1) % nvA));
    const float3 pk = normalize(-cross(mul(RA, ka - kb), nAw));
    const float3 pl = normalize(-cross(mul(RA, la - lb), nAw));
    const float3 nb = mul(RB, make_float3(fb.plane[0], fb.plane[1], fb.plane[2]));
    return fabsf(dot(pk, cross(pl, nb))) > 1e-3f;
}

// Classify the manifold's points against reference face G.faceA and
// incident face G.faceB (values only); returns how many points fit neither
// an incident vertex, an incident edge cut by a side plane, nor a corner of
// two side planes.
__device__ int geo_points(Geo& G, const b3::ShapesDev& S, const b3ConvexPolyhedron& hA, const b3ConvexPolyhedron& hB,
                          const Mat3& RA, const Mat3& RB, float3 xB, const float3* p, int npts) {
    int miss = 0;
    // origin at body A's position (p and xB are given relative to it)
    const b3Face fa = S.faces[hA.faceOffset + G.faceA];
    const b3Face fb = S.faces[hB.faceOffset + G.faceB];
    const int nvA = fa.numIndices, nvB = fb.numIndices;
    const float3 nAw = mul(RA, make_float3(fa.plane[0], fa.plane[1], fa.plane[2]));
    const float tol = 5e-5f;
    for (int j = 0; j < npts; ++j) {
        GeoPoint& g = G.pt[j];
        g.kind = PK_ATTACHED;
        g.local = mul_t(RB, p[j] - xB);
        float bestV = tol;
        for (int i = 0; i < nvB; ++i) {
            const float3 w = mul(RB, vtx(S, hB, face_vertex(S, fb, i))) + xB;
            const float e = length(w - p[j]);
            if (e < bestV) { bestV = e; g.kind = PK_VERTEX; g.i0 = i; }
        }
        if (g.kind == PK_VERTEX) continue;
        // side planes containing the point
        int on[2] = {-1, -1};
        float onErr[2] = {tol, tol};
        for (int k = 0; k < nvA; ++k) {
            const float3 va = vtx(S, hA, face_vertex(S, fa, k));
            const float3 vb = vtx(S, hA, face_vertex(S, fa, (k + 1) % nvA));
            float3 pn = -cross(mul(RA, va - vb), nAw);
            const float l = length(pn);
            if (l <= 0.f) continue;
            pn = pn * (1.f / l);
            const float e = fabsf(dot(pn, p[j] - mul(RA, va)));
            if (e < onErr[0]) { onErr[1] = onErr[0]; on[1] = on[0]; onErr[0] = e; on[0] = k; }
            else if (e < onErr[1]) { onErr[1] = e; on[1] = k; }
        }
        if (on[0] < 0) { ++miss; continue; }
        // an incident edge through the point, crossing the side plane
        // (not lying in it: the intersection must be well defined)
        const float3 vk = vtx(S, hA, face_vertex(S, fa, on[0]));
        const float3 vk1 = vtx(S, hA, face_vertex(S, fa, (on[0] + 1) % nvA));
        const float3 pnk = normalize(-cross(mul(RA, vk - vk1), nAw));
        int edge = -1;
        float bestE = tol;
        for (int i = 0; i < nvB; ++i) {
            const float3 a = mul(RB, vtx(S, hB, face_vertex(S, fb, i))) + xB;
            const float3 b = mul(RB, vtx(S, hB, face_vertex(S, fb, (i + 1) % nvB))) + xB;
            const float3 u = b - a;
            const float uu = dot(u, u);
            if (uu <= 0.f) continue;
            if (fabsf(dot(pnk, u)) < 1e-3f * sqrtf(uu)) continue;
            const float t = dot(p[j] - a, u) / uu;
            if (t < -1e-4f || t > 1.f + 1e-4f) continue;
            const float e = length(a + u * t - p[j]);
            if (e < bestE) { bestE = e; edge = i; }
        }
        if (edge >= 0) {
            g.kind = PK_EDGE;
            g.i0 = edge;
            g.i1 = (edge + 1) % nvB;
            g.k = on[0];
        } else if (on[1] >= 0 && corner_ok(S, hA, hB, fa, fb, RA, RB, nAw, on[0], on[1])) {
            g.kind = PK_CORNER;
            g.i0 = on[0];
            g.i1 = on[1];
        } else {
            ++miss;
        }
    }
    return miss;
}

// Faces of h whose sign * (n . sep) is within the forward's FP32 window
// (4e-6) of the extreme, extreme first: clipHullAgainstHull's choice, or
// its candidates where faces tie within FP32 (the forward decides those in
// float-float, exact ties to the lowest index).
__device__ int face_candidates(const b3::ShapesDev& S, const b3ConvexPolyhedron& h, const Mat3& R, float3 sep,
                               float sign, int* out, int maxOut) {
    float best = FLT_MAX;
    int bi = 0;
    for (int f = 0; f < h.numFaces; ++f) {
        const b3Face fc = S.faces[h.faceOffset + f];
        const float d = sign * dot(mul(R, make_float3(fc.plane[0], fc.plane[1], fc.plane[2])), sep);
        if (d < best) { best = d; bi = f; }
    }
    int n = 0;
    out[n++] = bi;
    for (int f = 0; f < h.numFaces && n < maxOut; ++f) {
        if (f == bi) continue;
        const b3Face fc = S.faces[h.faceOffset + f];
        const float d = sign * dot(mul(R, make_float3(fc.plane[0], fc.plane[1], fc.plane[2])), sep);
        if (d <= best + 4e-6f) out[n++] = f;
    }
    return n;
}

// Classify the stored manifold against the forward poses (values only).
__device__ void geo_classify(Geo& G, const b3::ShapesDev& S, const b3ConvexPolyhedron& hA,
                             const b3ConvexPolyhedron& hB, const Mat3& RA, const Mat3& RB, float3 xB, float3 sep,
                             const float3* p, int npts, int* unclassified) {
    // separating axis: the feature whose direction matches sep best
    float best = 1e-4f;
    G.axisKind = AX_ATTACHED;
    G.ax0 = G.ax1 = 0;
    G.axisSign = 1.f;
    G.nLocalA = mul_t(RA, sep);
    for (int side = 0; side < 2; ++side) {
        const b3ConvexPolyhedron& h = side ? hB : hA;
        const Mat3& R = side ? RB : RA;
        for (int f = 0; f < h.numFaces; ++f) {
            const b3Face fc = S.faces[h.faceOffset + f];
            const float3 nw = mul(R, make_float3(fc.plane[0], fc.plane[1], fc.plane[2]));
            for (int sg = 0; sg < 2; ++sg) {
                const float s = sg ? -1.f : 1.f;
                const float3 dlt = nw * s - sep;
                const float e = fmaxf(fabsf(dlt.x), fmaxf(fabsf(dlt.y), fabsf(dlt.z)));
                if (e < best) { best = e; G.axisKind = side ? AX_FACE_B : AX_FACE_A; G.ax0 = f; G.axisSign = s; }
            }
        }
    }
    for (int ea = 0; ea < hA.numUniqueEdges; ++ea) {
        const float3 a = mul(RA, f3(S.edges[hA.uniqueEdgesOffset + ea]));
        for (int eb = 0; eb < hB.numUniqueEdges; ++eb) {
            const float3 b = mul(RB, f3(S.edges[hB.uniqueEdgesOffset + eb]));
            const float3 c = cross(a, b);
            const float l = length(c);
            if (l < 1e-6f) continue;
            const float3 cn = c * (1.f / l);
            for (int sg = 0; sg < 2; ++sg) {
                const float s = sg ? -1.f : 1.f;
                const float3 dlt = cn * s - sep;
                const float e = fmaxf(fabsf(dlt.x), fmaxf(fabsf(dlt.y), fabsf(dlt.z)));
                if (e < best) { best = e; G.axisKind = AX_EDGES; G.ax0 = ea; G.ax1 = eb; G.axisSign = s; }
            }
        }
    }
    if (G.axisKind == AX_ATTACHED) atomicAdd(unclassified, 1);
    // reference / incident faces: clipHullAgainstHull's choice, trying the
    // faces tied within FP32 until the points fit one pair of them
    int candA[4], candB[4];
    const int nA = face_candidates(S, hA, RA, sep, 1.f, candA, 4);
    const int nB = face_candidates(S, hB, RB, sep, -1.f, candB, 4);
    int bestMiss = 1 << 30, bestA = candA[0], bestB = candB[0];
    for (int ia = 0; ia < nA && bestMiss > 0; ++ia)
        for (int ib = 0; ib < nB && bestMiss > 0; ++ib) {
            G.faceA = candA[ia];
            G.faceB = candB[ib];
            const int miss = geo_points(G, S, hA, hB, RA, RB, xB, p, npts);
            if (miss < bestMiss) { bestMiss = miss; bestA = candA[ia]; bestB = candB[ib]; }
        }
    G.faceA = bestA;
    G.faceB = bestB;
    const int miss = geo_points(G, S, hA, hB, RA, RB, xB, p, npts);
    if (miss) atomicAdd(unclassified, miss);
}

struct ManifoldArgs {
    b3::BodiesDev Bd;       // invMass, invInertia, friction, restitution
    const float4* pos;      // pre-step state
    const float4* quat;
    const float4* linVel;   // before gravity
    const float4* angVel;
    b3::ShapesDev S;
    const int* manifoldPair;
    const b3Contact4* contacts;
    int* unclassified;
};

__global__ void __launch_bounds__(128)
k_adj_manifold(SolverView V, AdjView A, ManifoldArgs MA, StepParams P) {
    const int M = *V.numManifolds;
    const size_t cap = (size_t)V.cap;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const float4 h0 = R(V, 0, m);
        const int bA = __float_as_int(h0.x), bB = __float_as_int(h0.y);
        const int dyn = __float_as_int(h0.w);
        const float4 h1 = R(V, 1, m), h2 = R(V, 2, m), h3 = R(V, 3, m);
        const float kA = h2.w, kB = h3.w;
        const b3Contact4 c = MA.contacts[MA.manifoldPair[m]];
        const int npts = (int)c.worldNormal[3];
        const bool dynA = dyn & 1, dynB = dyn & 2;
        // forward values; positions relative to body A's position
        const float3 oA = f3(MA.pos[bA]);
        const float3 xB = f3(MA.pos[bB]) - oA;
        const float3 g = P.gravity * P.dt;
        const float3 vA = dynA ? f3(MA.linVel[bA]) + g : make_float3(0.f, 0.f, 0.f);
        const float3 wA = dynA ? f3(MA.angVel[bA]) : make_float3(0.f, 0.f, 0.f);
        const float3 vB = dynB ? f3(MA.linVel[bB]) + g : make_float3(0.f, 0.f, 0.f);
        const float3 wB = dynB ? f3(MA.angVel[bB]) : make_float3(0.f, 0.f, 0.f);
        const float3 iiA = f3(h2), iiB = f3(h3);
        const float imA = h1.x, imB = h1.y;
        const float3 n0 = normalize(make_float3(-c.worldNormal[0], -c.worldNormal[1], -c.worldNormal[2]));
        float3 p0[4];
        float dep0[4];
        for (int j = 0; j < 4; ++j) {
            p0[j] = make_float3(c.worldPos[j][0], c.worldPos[j][1], c.worldPos[j][2]) - oA;
            dep0[j] = c.worldPos[j][3];
        }
        const float restitution = MA.Bd.restitution[bA] * MA.Bd.restitution[bB];
        // --- setup: one forward-mode pass per input ---------------------
        // inputs: xA 0-2, xB 3-5, vA 6-8, wA 9-11, vB 12-14, wB 15-17, imA 18,
        // imB 19, iiA 20-22, iiB 23-25, n 26-28, p 29-40, depth 41-44
        float gin[45];
        const float3 z3 = make_float3(0.f, 0.f, 0.f);
        for (int k = 0; k < 45; ++k) {
            gin[k] = 0.f;
            const bool aSide = (k < 3) || (k >= 6 && k < 12) || k == 18 || (k >= 20 && k < 23);
            const bool bSide = (k >= 3 && k < 6) || (k >= 12 && k < 18) || k == 19 || (k >= 23 && k < 26);
            if ((aSide && !dynA) || (bSide && !dynB)) continue;
            if (k >= 29 && k < 41 && (k - 29) / 3 >= npts) continue;
            if (k >= 41 && k - 41 >= npts) continue;
            auto e = [&](int base) {
                return make_float3(k == base ? 1.f : 0.f, k == base + 1 ? 1.f : 0.f, k == base + 2 ? 1.f : 0.f);
            };
            SetupIn I;
            I.xA = d3(z3, e(0));
            I.xB = d3(xB, e(3));
            I.vA = d3(vA, e(6));
            I.wA = d3(wA, e(9));
            I.vB = d3(vB, e(12));
            I.wB = d3(wB, e(15));
            I.imA = du(imA, k == 18 ? 1.f : 0.f);
            I.imB = du(imB, k == 19 ? 1.f : 0.f);
            I.iiA = d3(iiA, e(20));
            I.iiB = d3(iiB, e(23));
            I.n = d3(n0, e(26));
            for (int j = 0; j < 4; ++j) {
                I.p[j] = d3(p0[j], e(29 + 3 * j));
                I.depth[j] = du(dep0[j], k == 41 + j ? 1.f : 0.f);
            }
            gin[k] = setup_tangent(I, V, A, m, npts, kA, kB, restitution, P);
        }
        // header adjoints from the solve (inverse masses, inertias, mu)
        const float4 ga1 = A.rowAdj[cap + m];
        const float4 ga2 = A.rowAdj[2 * cap + m];
        const float4 ga3 = A.rowAdj[3 * cap + m];
        float gimA = ga1.x + gin[18], gimB = ga1.y + gin[19];
        float3 giiA = f3(ga2) + make_float3(gin[20], gin[21], gin[22]);
        float3 giiB = f3(ga3) + make_float3(gin[23], gin[24], gin[25]);
        const float gmu = ga1.z;
        // --- geometry: 12 pose directions -------------------------------
        float3 gxA = make_float3(gin[0], gin[1], gin[2]), gxB = make_float3(gin[3], gin[4], gin[5]);
        float3 gthA = z3, gthB = z3;
        const int colA = MA.Bd.collidable[bA], colB = MA.Bd.collidable[bB];
        const b3ConvexPolyhedron hA = MA.S.polys[MA.S.cols[colA].shapeIndex];
        const b3ConvexPolyhedron hB = MA.S.polys[MA.S.cols[colB].shapeIndex];
        const Mat3 RA = quat_to_mat(MA.quat[bA]), RB = quat_to_mat(MA.quat[bB]);
        Geo G;
        geo_classify(G, MA.S, hA, hB, RA, RB, xB, n0, p0, npts, MA.unclassified);
        const float3 gn = make_float3(gin[26], gin[27], gin[28]);
        for (int k = 0; k < 12; ++k) {
            const int body = k < 6 ? 0 : 1;
            if ((body == 0 && !dynA) || (body == 1 && !dynB)) continue;
            const int kk = k % 6;
            const float3 ex = make_float3(kk == 0 ? 1.f : 0.f, kk == 1 ? 1.f : 0.f, kk == 2 ? 1.f : 0.f);
            const float3 et = make_float3(kk == 3 ? 1.f : 0.f, kk == 4 ? 1.f : 0.f, kk == 5 ? 1.f : 0.f);
            PoseD PA, PB;
            PA.R = RA;
            PB.R = RB;
            PA.x = d3(z3, body == 0 ? ex : z3);
            PA.th = body == 0 ? et : z3;
            PB.x = d3(xB, body == 1 ? ex : z3);
            PB.th = body == 1 ? et : z3;
            D3 nD, pD[4];
            Du dD[4];
            geo_eval(G, MA.S, hA, hB, PA, PB, npts, nD, pD, dD);
            float acc = dot(gn, tan3(nD));
            for (int j = 0; j < npts; ++j)
                acc += gin[29 + 3 * j] * pD[j].x.d + gin[30 + 3 * j] * pD[j].y.d + gin[31 + 3 * j] * pD[j].z.d +
                       gin[41 + j] * dD[j].d;
            if (!isfinite(acc)) {
                // a degenerate feature slipped through the classification
                atomicAdd(MA.unclassified, 1);
                acc = 0.f;
            }
            float* dst = body == 0 ? (kk < 3 ? &gxA.x : &gthA.x) : (kk < 3 ? &gxB.x : &gthB.x);
            dst[kk % 3] += acc;
        }
        // --- friction of the pair -> the bodies' coefficients -----------
        const float muA = MA.Bd.friction[bA], muB = MA.Bd.friction[bB];
        float gmuA, gmuB;
        if (P.frictionCombine == 1) {
            gmuA = gmu * muB;
            gmuB = gmu * muA;
        } else {
            const float mc = sqrtf(muA * muB);
            gmuA = mc > 0.f ? gmu * 0.5f * mc / muA : 0.f;
            gmuB = mc > 0.f ? gmu * 0.5f * mc / muB : 0.f;
        }
        // --- per-copy contributions --------------------------------------
        for (int side = 0; side < 2; ++side) {
            if (!(dyn & (1 << side))) continue;
            const size_t slot = (size_t)(2 * m + side);
            const size_t stride = 2 * cap;
            float4* C = A.contrib;
            if (side == 0) {
                C[0 * stride + slot] = f4(gxA, gimA);
                C[1 * stride + slot] = f4(gthA, gmuA);
                C[2 * stride + slot] = make_float4(gin[6], gin[7], gin[8], 0.f);
                C[3 * stride + slot] = make_float4(gin[9], gin[10], gin[11], 0.f);
                C[4 * stride + slot] = f4(giiA, 0.f);
            } else {
                C[0 * stride + slot] = f4(gxB, gimB);
                C[1 * stride + slot] = f4(gthB, gmuB);
                C[2 * stride + slot] = make_float4(gin[12], gin[13], gin[14], 0.f);
                C[3 * stride + slot] = make_float4(gin[15], gin[16], gin[17], 0.f);
                C[4 * stride + slot] = f4(giiB, 0.f);
            }
        }
    }
}

// Sum each dynamic body's per-copy contributions (deterministic order).
__global__ void k_adj_gather(int n, const float* __restrict__ invMass, const float4* __restrict__ invInertia,
                             SolverView V, AdjView A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || invMass[i] == 0.f) return;
    const uint32_t s = V.incStart[i], e = V.incEnd[i];
    if (e <= s) return;
    float4 sx = make_float4(0.f, 0.f, 0.f, 0.f), sth = sx, sv = sx, sw = sx, sii = sx;
    const size_t stride = 2 * (size_t)V.cap;
    for (uint32_t k = s; k < e; ++k) {
        const uint32_t slot = V.incVals[k];
        const float4 a = A.contrib[slot], b = A.contrib[stride + slot], c = A.contrib[2 * stride + slot];
        const float4 d = A.contrib[3 * stride + slot], f = A.contrib[4 * stride + slot];
        sx.x += a.x; sx.y += a.y; sx.z += a.z; sx.w += a.w;
        sth.x += b.x; sth.y += b.y; sth.z += b.z; sth.w += b.w;
        sv.x += c.x; sv.y += c.y; sv.z += c.z;
        sw.x += d.x; sw.y += d.y; sw.z += d.z;
        sii.x += f.x; sii.y += f.y; sii.z += f.z;
    }
    add4(A.gX[i], make_float3(sx.x, sx.y, sx.z));
    add4(A.gTh[i], make_float3(sth.x, sth.y, sth.z));
    add4(A.gV[i], make_float3(sv.x, sv.y, sv.z));
    add4(A.gW[i], make_float3(sw.x, sw.y, sw.z));
    // inverse inertia = inverse mass x shape factor
    const float im = invMass[i];
    const float3 ii = f3(invInertia[i]);
    A.gInvMass[i] += sx.w + (sii.x * ii.x + sii.y * ii.y + sii.z * ii.z) / im;
    A.gMu[i] += sth.w;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct b3Adjoint_t {
    b3World w = nullptr;
    int numSteps = 0, K = 1, N = 0, cap = 0, iterations = 0;
    int numCkpt = 0;
    float4* ckpt = nullptr;   // [numCkpt][4][N]
    float4* seg = nullptr;    // [K][4][N]
    b3::JacobiTape tape{};
    float4 *gX = nullptr, *gTh = nullptr, *gV = nullptr, *gW = nullptr, *gDv = nullptr, *gDw = nullptr;
    float *gInvMass = nullptr, *gMu = nullptr;
    float4 *rowAdj = nullptr, *gInLin = nullptr, *gInAng = nullptr, *gLam = nullptr, *contrib = nullptr;
    float4* seedQ = nullptr;
    int* unclassified = nullptr;
    bool forwardDone = false, backwardDone = false;
    std::vector<void*> owned;
};

namespace {

template <typename T>
int aalloc(b3Adjoint_t* a, T*& p, size_t count) {
    if (count == 0) count = 1;
    B3_CUDA(cudaMalloc((void**)&p, sizeof(T) * count));
    a->owned.push_back((void*)p);
    return B3_OK;
}

int copy_state(b3World_t* w, float4* dst, cudaStream_t st, bool toWorld) {
    const size_t N = w->bodies.size();
    float4* bufs[4] = {w->d.pos, w->d.quat, w->d.linVel, w->d.angVel};
    for (int k = 0; k < 4; ++k) {
        if (toWorld)
            B3_CUDA(cudaMemcpyAsync(bufs[k], dst + k * N, N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        else
            B3_CUDA(cudaMemcpyAsync(dst + k * N, bufs[k], N * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    }
    return B3_OK;
}

AdjView adj_view(b3Adjoint_t* a) {
    AdjView A;
    A.gX = a->gX; A.gTh = a->gTh; A.gV = a->gV; A.gW = a->gW;
    A.gDv = a->gDv; A.gDw = a->gDw;
    A.gInvMass = a->gInvMass; A.gMu = a->gMu;
    A.rowAdj = a->rowAdj; A.gInLin = a->gInLin; A.gInAng = a->gInAng; A.gLam = a->gLam;
    A.contrib = a->contrib;
    A.cap = a->cap;
    return A;
}

StepParams step_params(b3World_t* w) {
    StepParams P;
    P.dt = w->sim.dt;
    P.damping = w->sim.angularDamping;
    P.threshold = 0.25f * 3.14159254f;
    P.gravity = w->sim.gravity;
    P.erp = w->sim.erp;
    P.contactProcessing = w->sim.contactProcessing;
    P.slopOffset = w->sim.slopOffset;
    P.frictionCombine = w->sim.frictionCombine;
    P.iterations = w->sim.iterations;
    return P;
}

// Reverse one step whose pre-step state is in `pre` ([4][N]); the world's
// buffers hold that step re-run with the tape.
int reverse_step(b3Adjoint_t* a, const float4* pre, cudaStream_t st) {
    b3World_t* w = a->w;
    const int N = a->N;
    const StepParams P = step_params(w);
    SolverView V = solver_view(w);
    AdjView A = adj_view(a);
    k_adj_integrate<<<(N + 255) / 256, 256, 0, st>>>(N, w->d.invMass, w->d.angVel, w->d.bodyIncStart,
                                                    w->d.bodyIncEnd, A, P);
    B3_CHECK_LAUNCH();
    if (a->iterations > 0) {
        B3_CUDA(cudaMemsetAsync(w->d.scalars + b3::S_BAR_COUNT, 0, sizeof(int32_t) * 2, st));
        const int threads = 256;
        int occ = 1;
        B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_adjoint, threads, 0));
        occ = occ < 1 ? 1 : (occ > 4 ? 4 : occ);
        const long long est = std::min<long long>((long long)w->cfg.maxPairs, 3LL * (long long)N);
        const int want = (int)std::max<long long>(1, (est + threads - 1) / threads);
        const int grid = std::min(w->ctx->numSMs * occ, want);
        int iters = a->iterations;
        uint32_t* bar = (uint32_t*)(w->d.scalars + b3::S_BAR_COUNT);
        int32_t* err = w->d.scalars + b3::S_ERR;
        b3Counters* ctr = w->d.counters;
        b3::JacobiTape T = a->tape;
        void* args[] = {&V, &T, &A, &iters, &bar, &err, &ctr};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(threads);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        B3_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_jacobi_adjoint, args));
    }
    ManifoldArgs MA;
    MA.Bd = w->bodiesDev();
    MA.pos = pre;
    MA.quat = pre + N;
    MA.linVel = pre + 2 * (size_t)N;
    MA.angVel = pre + 3 * (size_t)N;
    MA.S = w->shapesDev();
    MA.manifoldPair = w->d.manifoldPair;
    MA.contacts = w->d.contacts;
    MA.unclassified = a->unclassified;
    if (a->iterations > 0) {
        const int g = w->ctx->numSMs * 4;
        k_adj_manifold<<<g, 128, 0, st>>>(V, A, MA, P);
        B3_CHECK_LAUNCH();
        k_adj_gather<<<(N + 255) / 256, 256, 0, st>>>(N, w->d.invMass, w->d.invInertia, V, A);
        B3_CHECK_LAUNCH();
    }
    return B3_OK;
}

}  // namespace

extern "C" int b3_adjoint_create(b3World w, int numSteps, int checkpointEvery, b3Adjoint* out) {
    if (!w || !out || numSteps <= 0 || checkpointEvery <= 0) return B3_ERR_INVALID_ARG;
    *out = nullptr;
    if (!w->written) return B3_ERR_STATE;
    if (w->gs) {
        b3_set_error("the adjoint form differentiates the Jacobi solver; this world runs batched Gauss-Seidel");
        return B3_ERR_UNSUPPORTED;
    }
    if (w->numSpheres || w->numPlanes || w->numCompounds || w->numMeshes) {
        b3_set_error("the adjoint form differentiates hull-hull contact geometry; this world has spheres, planes, "
                     "compounds or meshes");
        return B3_ERR_UNSUPPORTED;
    }
    B3_CUDA(cudaSetDevice(w->ctx->device));
    b3Adjoint_t* a = new b3Adjoint_t();
    a->w = w;
    a->numSteps = numSteps;
    a->K = std::min(checkpointEvery, numSteps);
    a->N = (int)w->bodies.size();
    a->cap = w->cfg.maxPairs;
    a->iterations = w->sim.iterations;
    a->numCkpt = (numSteps + a->K - 1) / a->K;
    const size_t N = (size_t)a->N, cap = (size_t)a->cap;
    const size_t phases = 2 * (size_t)a->iterations;
    int rc = B3_OK;
    // HBM sizing: checkpoints, one segment of pre-step states, the tape of
    // one step and the adjoint buffers, checked against free device memory
    {
        const size_t f4 = sizeof(float4);
        const size_t need = f4 * ((size_t)a->numCkpt * 4 * N + (size_t)a->K * 4 * N + phases * 4 * cap +
                                  (size_t)a->iterations * 3 * cap + 7 * N + (size_t)kRowSlots * cap + 8 * cap +
                                  3 * cap + (size_t)kContrib * 2 * cap) +
                            2 * sizeof(float) * N;
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess && need > freeB / 100 * 95) {
            delete a;
            b3_set_error("adjoint needs %.2f GB, %.2f GB free", need / 1e9, freeB / 1e9);
            return B3_ERR_CAPACITY;
        }
    }
    auto fail = [&](int r) {
        for (void* p : a->owned) cudaFree(p);
        delete a;
        return r;
    };
    if ((rc = aalloc(a, a->ckpt, (size_t)a->numCkpt * 4 * N)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->seg, (size_t)a->K * 4 * N)) != B3_OK) return fail(rc);
    if (phases > 0) {
        if ((rc = aalloc(a, a->tape.copyLin, phases * 2 * cap)) != B3_OK) return fail(rc);
        if ((rc = aalloc(a, a->tape.copyAng, phases * 2 * cap)) != B3_OK) return fail(rc);
        if ((rc = aalloc(a, a->tape.lamN, (size_t)a->iterations * cap)) != B3_OK) return fail(rc);
        if ((rc = aalloc(a, a->tape.lamF, (size_t)a->iterations * 2 * cap)) != B3_OK) return fail(rc);
    }
    float4** pb[] = {&a->gX, &a->gTh, &a->gV, &a->gW, &a->gDv, &a->gDw, &a->seedQ};
    for (auto p : pb)
        if ((rc = aalloc(a, *p, N)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->gInvMass, N)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->gMu, N)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->rowAdj, (size_t)kRowSlots * cap)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->gInLin, 4 * cap)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->gInAng, 4 * cap)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->gLam, 3 * cap)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->contrib, (size_t)kContrib * 2 * cap)) != B3_OK) return fail(rc);
    if ((rc = aalloc(a, a->unclassified, 1)) != B3_OK) return fail(rc);
    *out = a;
    return B3_OK;
}

extern "C" int b3_adjoint_destroy(b3Adjoint a) {
    if (!a) return B3_OK;
    for (void* p : a->owned) cudaFree(p);
    delete a;
    return B3_OK;
}

extern "C" int b3_adjoint_forward(b3Adjoint a, void* stream) {
    if (!a) return B3_ERR_INVALID_ARG;
    b3World_t* w = a->w;
    B3_CUDA(cudaSetDevice(w->ctx->device));
    cudaStream_t st = as_stream(stream);
    const size_t N = (size_t)a->N;
    for (int t = 0; t < a->numSteps; ++t) {
        if (t % a->K == 0) B3_TRY(copy_state(w, a->ckpt + (size_t)(t / a->K) * 4 * N, st, false));
        B3_TRY(b3_step(w, 1, stream));
    }
    a->forwardDone = true;
    a->backwardDone = false;
    return B3_OK;
}

extern "C" int b3_adjoint_backward(b3Adjoint a, const float* dPos4, const float* dQuat4, const float* dLinVel4,
                                   const float* dAngVel4, void* stream) {
    if (!a) return B3_ERR_INVALID_ARG;
    if (!a->forwardDone) return B3_ERR_STATE;
    b3World_t* w = a->w;
    B3_CUDA(cudaSetDevice(w->ctx->device));
    cudaStream_t st = as_stream(stream);
    const size_t N = (size_t)a->N;
    const size_t bytes = N * sizeof(float4);
    // seeds (dL/dq is turned into a world-rotation adjoint at the final pose)
    float4* dst[4] = {a->gX, a->seedQ, a->gV, a->gW};
    const float* src[4] = {dPos4, dQuat4, dLinVel4, dAngVel4};
    for (int k = 0; k < 4; ++k) {
        if (src[k]) B3_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyHostToDevice, st));
        else B3_CUDA(cudaMemsetAsync(dst[k], 0, bytes, st));
    }
    k_adj_seed<<<(int)((N + 255) / 256), 256, 0, st>>>((int)N, w->d.quat, a->seedQ, a->gTh);
    B3_CHECK_LAUNCH();
    B3_CUDA(cudaMemsetAsync(a->gInvMass, 0, N * sizeof(float), st));
    B3_CUDA(cudaMemsetAsync(a->gMu, 0, N * sizeof(float), st));
    B3_CUDA(cudaMemsetAsync(a->unclassified, 0, sizeof(int), st));
    for (int sgi = a->numCkpt - 1; sgi >= 0; --sgi) {
        const int t0 = sgi * a->K;
        const int t1 = std::min(t0 + a->K, a->numSteps);
        // recompute the segment's pre-step states from its checkpoint
        B3_TRY(copy_state(w, a->ckpt + (size_t)sgi * 4 * N, st, true));
        for (int t = t0; t < t1; ++t) {
            B3_TRY(copy_state(w, a->seg + (size_t)(t - t0) * 4 * N, st, false));
            if (t + 1 < t1) B3_TRY(b3::run_step(w, st, nullptr));
        }
        for (int t = t1 - 1; t >= t0; --t) {
            const float4* pre = a->seg + (size_t)(t - t0) * 4 * N;
            B3_TRY(copy_state(w, const_cast<float4*>(pre), st, true));
            B3_TRY(b3::run_step(w, st, &a->tape));
            B3_TRY(reverse_step(a, pre, st));
        }
    }
    // leave the world at the final state of the forward run
    B3_TRY(copy_state(w, a->ckpt + (size_t)(a->numCkpt - 1) * 4 * N, st, true));
    for (int t = (a->numCkpt - 1) * a->K; t < a->numSteps; ++t) B3_TRY(b3::run_step(w, st, nullptr));
    a->backwardDone = true;
    return B3_OK;
}

extern "C" int b3_adjoint_gradients(b3Adjoint a, float* dLinVel4, float* dAngVel4, float* dMass, float* dFriction) {
    if (!a) return B3_ERR_INVALID_ARG;
    if (!a->backwardDone) return B3_ERR_STATE;
    b3World_t* w = a->w;
    B3_CUDA(cudaSetDevice(w->ctx->device));
    const size_t N = (size_t)a->N;
    B3_CUDA(cudaDeviceSynchronize());
    if (dLinVel4) B3_CUDA(cudaMemcpy(dLinVel4, a->gV, N * sizeof(float4), cudaMemcpyDeviceToHost));
    if (dAngVel4) B3_CUDA(cudaMemcpy(dAngVel4, a->gW, N * sizeof(float4), cudaMemcpyDeviceToHost));
    if (dMass || dFriction) {
        std::vector<float> gim(N), gmu(N);
        B3_CUDA(cudaMemcpy(gim.data(), a->gInvMass, N * sizeof(float), cudaMemcpyDeviceToHost));
        B3_CUDA(cudaMemcpy(gmu.data(), a->gMu, N * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < N; ++i) {
            const float im = w->bodies[i].invMass;
            // invMass = 1 / mass  ->  dL/dmass = -dL/dinvMass * invMass^2
            if (dMass) dMass[i] = im != 0.f ? -gim[i] * im * im : 0.f;
            if (dFriction) dFriction[i] = im != 0.f ? gmu[i] : 0.f;
        }
    }
    return B3_OK;
}

extern "C" int b3_adjoint_info(b3Adjoint a, int* unclassified) {
    if (!a || !unclassified) return B3_ERR_INVALID_ARG;
    B3_CUDA(cudaMemcpy(unclassified, a->unclassified, sizeof(int), cudaMemcpyDeviceToHost));
    return B3_OK;
}
