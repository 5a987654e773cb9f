// Float-float ("double-single") arithmetic for the numerically sensitive
// parts of the narrowphase, built from the error-free transformations
// TwoSum (Knuth) and TwoProduct via fused multiply-add (Dekker/Ogita-Rump-
// Oishi). A value is hi + lo with |lo| <= ulp(hi)/2, about 48 significant
// bits, all on the FP32 pipes.
//
// Why: the reference's clipping and axis formulas are ill-conditioned for
// nearly parallel edges and planes (for example two stacked boxes whose side
// edges cross a clip plane at a grazing angle). Evaluated in plain FP32 the
// contact points then move by up to ~1e-3 m and edge-edge normals by ~1e-3
// relative to the exact result; the same formulas in float-float agree with
// an FP64 evaluation to ~1e-12 before the final rounding to FP32.
#pragma once
#include <cuda_runtime.h>

namespace b3ff {

struct ff {
    float hi, lo;
};
struct ff3 {
    ff x, y, z;
};
struct ffq {
    ff x, y, z, w;
};

__device__ __forceinline__ ff mk(float a) { return {a, 0.f}; }
__device__ __forceinline__ float val(ff a) { return a.hi + a.lo; }

__device__ __forceinline__ ff two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return {s, e};
}
__device__ __forceinline__ ff fast_two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    return {s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ ff two_prod(float a, float b) {
    const float p = __fmul_rn(a, b);
    return {p, __fmaf_rn(a, b, -p)};
}
__device__ __forceinline__ ff add(ff a, ff b) {
    ff s = two_sum(a.hi, b.hi);
    const ff t = two_sum(a.lo, b.lo);
    s.lo = __fadd_rn(s.lo, t.hi);
    s = fast_two_sum(s.hi, s.lo);
    s.lo = __fadd_rn(s.lo, t.lo);
    return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ ff neg(ff a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ ff sub(ff a, ff b) { return add(a, neg(b)); }
__device__ __forceinline__ ff mul(ff a, ff b) {
    ff p = two_prod(a.hi, b.hi);
    p.lo = __fmaf_rn(a.hi, b.lo, __fmaf_rn(a.lo, b.hi, p.lo));
    return fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ ff mulf(ff a, float b) {
    ff p = two_prod(a.hi, b);
    p.lo = __fmaf_rn(a.lo, b, p.lo);
    return fast_two_sum(p.hi, p.lo);
}
__device__ __noinline__ ff div(ff a, ff b) {
    const float q1 = __fdiv_rn(a.hi, b.hi);
    const ff r = sub(a, mulf(b, q1));
    const float q2 = __fdiv_rn(r.hi, b.hi);
    const ff r2 = sub(r, mulf(b, q2));
    const float q3 = __fdiv_rn(r2.hi, b.hi);
    ff q = fast_two_sum(q1, q2);
    return add(q, mk(q3));
}
__device__ __noinline__ ff sqrt_ff(ff a) {
    if (a.hi <= 0.f) return mk(0.f);
    const float s = __fsqrt_rn(a.hi);
    // one Newton step: s + (a - s^2) / (2 s)
    const ff e = sub(a, two_prod(s, s));
    return add(mk(s), mk(__fdiv_rn(e.hi, 2.f * s)));
}
__device__ __forceinline__ bool lt(ff a, ff b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
__device__ __forceinline__ bool le(ff a, ff b) { return !lt(b, a); }
__device__ __forceinline__ bool eq(ff a, ff b) { return a.hi == b.hi && a.lo == b.lo; }

__device__ __forceinline__ ff3 mk3(float x, float y, float z) { return {mk(x), mk(y), mk(z)}; }
__device__ __forceinline__ ff3 add3(ff3 a, ff3 b) { return {add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
__device__ __forceinline__ ff3 sub3(ff3 a, ff3 b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
__device__ __forceinline__ ff3 neg3(ff3 a) { return {neg(a.x), neg(a.y), neg(a.z)}; }
__device__ __forceinline__ ff3 scale3(ff3 a, ff s) { return {mul(a.x, s), mul(a.y, s), mul(a.z, s)}; }
__device__ __noinline__ ff dot3(ff3 a, ff3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
__device__ __noinline__ ff3 cross3(ff3 a, ff3 b) {
    return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)),
            sub(mul(a.x, b.y), mul(a.y, b.x))};
}
__device__ __noinline__ ff3 normalize3(ff3 a) {
    const ff l2 = dot3(a, a);
    if (l2.hi <= 0.f) return a;
    const ff l = sqrt_ff(l2);
    return {div(a.x, l), div(a.y, l), div(a.z, l)};
}
__device__ __forceinline__ float3 to_f3(ff3 a) { return make_float3(val(a.x), val(a.y), val(a.z)); }

// Quaternion product qtMul (P2/sat.cl:146-155) and rotation qtRotate
// (:203-210), the same sequence the oracle evaluates.
__device__ __forceinline__ ffq qmul(ffq a, ffq b) {
    const ff3 av{a.x, a.y, a.z}, bv{b.x, b.y, b.z};
    const ff3 c = cross3(av, bv);
    ffq r;
    r.x = add(add(c.x, mul(a.w, b.x)), mul(b.w, a.x));
    r.y = add(add(c.y, mul(a.w, b.y)), mul(b.w, a.y));
    r.z = add(add(c.z, mul(a.w, b.z)), mul(b.w, a.z));
    r.w = sub(mul(a.w, b.w), dot3(av, bv));
    return r;
}
__device__ __forceinline__ ff3 qrot(float4 q, ff3 v) {
    const ffq qq{mk(q.x), mk(q.y), mk(q.z), mk(q.w)};
    const ffq qi{mk(-q.x), mk(-q.y), mk(-q.z), mk(q.w)};
    const ffq vv{v.x, v.y, v.z, mk(0.f)};
    const ffq r = qmul(qmul(qq, vv), qi);
    return {r.x, r.y, r.z};
}
__device__ __forceinline__ ff3 qinvrot(float4 q, ff3 v) {
    return qrot(make_float4(-q.x, -q.y, -q.z, q.w), v);
}

// Matrix of v -> q v q* (q need not be unit: the homogeneous form equals the
// quaternion sandwich term for term), entries exact products of the FP32
// quaternion components summed in float-float.
struct ffmat {
    ff m[3][3];
};
__device__ __noinline__ ffmat quat_mat(float4 q) {
    const ff xx = two_prod(q.x, q.x), yy = two_prod(q.y, q.y), zz = two_prod(q.z, q.z), ww = two_prod(q.w, q.w);
    const ff xy = two_prod(q.x, q.y), xz = two_prod(q.x, q.z), yz = two_prod(q.y, q.z);
    const ff wx = two_prod(q.w, q.x), wy = two_prod(q.w, q.y), wz = two_prod(q.w, q.z);
    auto dbl = [](ff a) { return ff{2.f * a.hi, 2.f * a.lo}; };
    ffmat R;
    R.m[0][0] = sub(add(ww, xx), add(yy, zz));
    R.m[0][1] = dbl(sub(xy, wz));
    R.m[0][2] = dbl(add(xz, wy));
    R.m[1][0] = dbl(add(xy, wz));
    R.m[1][1] = sub(add(ww, yy), add(xx, zz));
    R.m[1][2] = dbl(sub(yz, wx));
    R.m[2][0] = dbl(sub(xz, wy));
    R.m[2][1] = dbl(add(yz, wx));
    R.m[2][2] = sub(add(ww, zz), add(xx, yy));
    return R;
}
// R v for an FP32 vector
__device__ __noinline__ ff3 mrot(const ffmat& R, float3 v) {
    ff3 r;
    r.x = add(add(mulf(R.m[0][0], v.x), mulf(R.m[0][1], v.y)), mulf(R.m[0][2], v.z));
    r.y = add(add(mulf(R.m[1][0], v.x), mulf(R.m[1][1], v.y)), mulf(R.m[1][2], v.z));
    r.z = add(add(mulf(R.m[2][0], v.x), mulf(R.m[2][1], v.y)), mulf(R.m[2][2], v.z));
    return r;
}
// R^T v for a float-float vector
__device__ __noinline__ ff3 mrot_t(const ffmat& R, ff3 v) {
    ff3 r;
    r.x = add(add(mul(R.m[0][0], v.x), mul(R.m[1][0], v.y)), mul(R.m[2][0], v.z));
    r.y = add(add(mul(R.m[0][1], v.x), mul(R.m[1][1], v.y)), mul(R.m[2][1], v.z));
    r.z = add(add(mul(R.m[0][2], v.x), mul(R.m[1][2], v.y)), mul(R.m[2][2], v.z));
    return r;
}

}  // namespace b3ff
