// Small vector / quaternion helpers for the device kernels.
//
// Two flavours:
//   * default helpers (FMA contraction allowed) for the narrowphase, solver
//     and integrator, whose results are checked within tolerance;
//   * *_rn helpers built from __fmul_rn/__fadd_rn/__fsub_rn, which the
//     compiler never fuses, for the AABB + cell-hash stage whose integer
//     outputs (cell keys, sort order, pair set) must be bit-identical to the
//     single-threaded restatement evaluating the same operation sequence.
// Quaternion conventions follow the reference kernels: qtMul/qtRotate in
// BB/broadphaseKernel.cl:19-47 and P2/sat.cl:146-230 (q = x,y,z,w).
#pragma once
#include <cuda_runtime.h>

namespace b3m {

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(float3 v, float w = 0.f) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 mulv(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3& operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ float3& operator-=(float3& a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) {
    float l2 = dot(a, a);
    return l2 > 0.f ? a * rsqrtf(l2) : a;
}

// Rotation matrix of a unit quaternion (rows), for rotating many vectors.
struct Mat3 {
    float3 r0, r1, r2;
};
__device__ __forceinline__ Mat3 quat_to_mat(float4 q) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    Mat3 m;
    m.r0 = make_float3(1.f - 2.f * (y * y + z * z), 2.f * (x * y - w * z), 2.f * (x * z + w * y));
    m.r1 = make_float3(2.f * (x * y + w * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - w * x));
    m.r2 = make_float3(2.f * (x * z - w * y), 2.f * (y * z + w * x), 1.f - 2.f * (x * x + y * y));
    return m;
}
__device__ __forceinline__ float3 mul(const Mat3& m, float3 v) {
    return make_float3(dot(m.r0, v), dot(m.r1, v), dot(m.r2, v));
}
// R^T v
__device__ __forceinline__ float3 mul_t(const Mat3& m, float3 v) {
    return make_float3(m.r0.x * v.x + m.r1.x * v.y + m.r2.x * v.z,
                       m.r0.y * v.x + m.r1.y * v.y + m.r2.y * v.z,
                       m.r0.z * v.x + m.r1.z * v.y + m.r2.z * v.z);
}

// Quaternion product as in quatMult (BB/integrateKernel.cl:3-11).
__device__ __forceinline__ float4 quat_mult(float4 q1, float4 q2) {
    float4 q;
    q.x = q1.w * q2.x + q1.x * q2.w + q1.y * q2.z - q1.z * q2.y;
    q.y = q1.w * q2.y + q1.y * q2.w + q1.z * q2.x - q1.x * q2.z;
    q.z = q1.w * q2.z + q1.z * q2.w + q1.x * q2.y - q1.y * q2.x;
    q.w = q1.w * q2.w - q1.x * q2.x - q1.y * q2.y - q1.z * q2.z;
    return q;
}

// ---------------------------------------------------------------------------
// Non-contracting (bit-reproducible) helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mrn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float arn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float srn(float a, float b) { return __fsub_rn(a, b); }
// dot of xyz, evaluated ((x*x' + y*y') + z*z')
__device__ __forceinline__ float dot3_rn(float4 a, float4 b) {
    return arn(arn(mrn(a.x, b.x), mrn(a.y, b.y)), mrn(a.z, b.z));
}
__device__ __forceinline__ float4 cross3_rn(float4 a, float4 b) {
    return make_float4(srn(mrn(a.y, b.z), mrn(a.z, b.y)), srn(mrn(a.z, b.x), mrn(a.x, b.z)),
                       srn(mrn(a.x, b.y), mrn(a.y, b.x)), 0.f);
}
// qtMul (BB/broadphaseKernel.cl:19-27): ans = cross(a,b); ans += a.w*b + b.w*a;
// ans.w = a.w*b.w - dot3(a,b)
__device__ __forceinline__ float4 qt_mul_rn(float4 a, float4 b) {
    float4 c = cross3_rn(a, b);
    float4 r;
    r.x = arn(c.x, arn(mrn(a.w, b.x), mrn(b.w, a.x)));
    r.y = arn(c.y, arn(mrn(a.w, b.y), mrn(b.w, a.y)));
    r.z = arn(c.z, arn(mrn(a.w, b.z), mrn(b.w, a.z)));
    r.w = srn(mrn(a.w, b.w), dot3_rn(a, b));
    return r;
}
// qtRotate (BB/broadphaseKernel.cl:35-43)
__device__ __forceinline__ float4 qt_rotate_rn(float4 q, float4 v) {
    float4 qinv = make_float4(-q.x, -q.y, -q.z, q.w);
    float4 vc = make_float4(v.x, v.y, v.z, 0.f);
    return qt_mul_rn(qt_mul_rn(q, vc), qinv);
}

}  // namespace b3m
