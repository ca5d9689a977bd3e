// Device helpers shared by the SPH forward (sph.cu) and derivative (sph_grad.cu) passes: the cubic
// spline kernel, its gradient and the viscosity Laplacian with the reference's FP32 rounding
// (density/device.cuh:26-43, 72-76), the prediction with the collision box (sph/pcisph.cu:26-45)
// and the per-particle prologue of every pass.
#pragma once

#include "gather.cuh"
#include "sph_launch.h"

namespace pbf {
namespace sph {
namespace detail {

using namespace gather_detail;

// x*y + ... as the reference's dot(a, b) compiles (density/device.cuh, domain/device.cuh:56-58):
// fma(a.z, b.z, fma(a.x, b.x, a.y * b.y)).
__device__ __forceinline__ float dot_xfirst(const f3 a, const f3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)));
}

// Cubic spline weight at distance `distance` < h (density/device.cuh:26-34).
__device__ __forceinline__ float cubic_inside(const float distance, const SphConstants& k) {
    const float q = __fdiv_rn(distance, k.h);
    if (q <= 0.5F) {
        // 6 q q q - 6 q q + 1 with the shared product t = 6 q q: fma(t, q, -t) + 1
        const float t = __fmul_rn(__fmul_rn(6.0F, q), q);
        return __fmul_rn(k.cubic_coefficient, __fadd_rn(__fmaf_rn(t, q, -t), 1.0F));
    }
    const float difference = __fsub_rn(1.0F, q);
    return __fmul_rn(__fmul_rn(__fmul_rn(k.cubic_coefficient_2, difference), difference), difference);
}

// Scale of the cubic gradient, grad W = d * s, at 0 < distance < h (density/device.cuh:36-42).
__device__ __forceinline__ float cubic_gradient_scale(const float distance, const SphConstants& k) {
    const float q = __fdiv_rn(distance, k.h);
    float derivative;
    if (q <= 0.5F) {
        derivative = __fmaf_rn(__fmul_rn(18.0F, q), q, -__fmul_rn(12.0F, q));
    } else {
        const float difference = __fsub_rn(1.0F, q);
        derivative = __fmul_rn(__fmul_rn(-6.0F, difference), difference);
    }
    return __fdiv_rn(__fmul_rn(k.cubic_coefficient, derivative), __fmul_rn(k.h, distance));
}

// Viscosity Laplacian at distance < h (density/device.cuh:72-76).
__device__ __forceinline__ float laplacian_inside(const float distance, const SphConstants& k) {
    return __fdiv_rn(__fmul_rn(45.0F, __fsub_rn(k.h, distance)), k.laplacian_denominator);
}

// predict (sph/pcisph.cu:26-45, the same body as integrate, sph/common.cu:302-320):
// v* = v + dt a, x* = x + dt v*, then the collision box of the step.
__device__ __forceinline__ void predict(const f3 x, const f3 v, const f3 a, const float dt, const Box& box,
                                        const SphConstants& k, f3& xo, f3& vo) {
    f3 vel = fma3(dt, a, v);
    f3 pos = fma3(dt, vel, x);
    const bool cx = pos.x < box.min_x || pos.x > box.max_x;
    const bool cy = pos.y < box.min_y || pos.y > box.max_y;
    const bool cz = pos.z < box.min_z || pos.z > box.max_z;
    pos.x = fminf(box.max_x, fmaxf(box.min_x, pos.x));
    pos.y = fminf(box.max_y, fmaxf(box.min_y, pos.y));
    pos.z = fminf(box.max_z, fmaxf(box.min_z, pos.z));
    if (k.no_slip != 0u && (cx || cy || cz)) {
        vel = mk(k.box_vx, k.box_vy, k.box_vz);
    } else {
        if (cx) vel.x = k.box_vx;
        if (cy) vel.y = k.box_vy;
        if (cz) vel.z = k.box_vz;
    }
    xo = pos;
    vo = vel;
}

// Largest |x* - x| of the particles predicted by one pass, as the bits of a non-negative float
// (their unsigned order is the float order): a warp maximum, then one atomic per warp.
__device__ __forceinline__ void record_displacement(unsigned int* word, const f3 predicted, const f3 x) {
    const float d = __fsqrt_rn(sq_xfirst(sub(predicted, x)));
    const unsigned int bits = __float_as_uint(d);   // d >= 0 or NaN (NaN bits exceed every finite bound)
    const unsigned int mask = __activemask();
    const unsigned int m = __reduce_max_sync(mask, bits);
    if ((threadIdx.x & 31u) == static_cast<unsigned int>(__ffs(mask) - 1)) atomicMax(word, m);
}

struct Own {
    Particle p;
    f3 x;
    float mass;
    float4 pa;   // (rest density, viscosity, surface tension, method parameter 0)
    const SphConstants* k;
};

__device__ __forceinline__ Own own(const SphStep& st) {
    Own o;
    o.p = locate(st.g);
    if (!o.p.active) return o;
    const float4 xi = st.topology[o.p.s];
    o.x = xyz(xi);
    o.mass = xi.w;
    o.pa = st.g.params_a[o.p.s];
    o.k = st.constants + o.p.scene->constants;
    return o;
}


// ------------------------------------------------------------------ derivatives (sph_grad.cu)
// FP32 kernel values with the forward passes' rounding.
__device__ __forceinline__ float cubic_value(const f3 d, const SphConstants& k) {
    const float r = __fsqrt_rn(sq_xfirst(d));
    return r >= k.h ? 0.0F : cubic_inside(r, k);
}
__device__ __forceinline__ f3 cubic_gradient_value(const f3 d, const SphConstants& k) {
    const float r = __fsqrt_rn(sq_xfirst(d));
    if (r == 0.0F || r >= k.h) return mk(0.0F, 0.0F, 0.0F);
    return scale(d, cubic_gradient_scale(r, k));
}
__device__ __forceinline__ float laplacian_value(const f3 d, const SphConstants& k) {
    const float r = __fsqrt_rn(sq_xfirst(d));
    return r >= k.h ? 0.0F : laplacian_inside(r, k);
}

// Directional derivative of the cubic gradient along the displacement tangent t
// (density/device.cuh:45-57), FP32.
// The tangents are held to FP32 rounding against the reference, not to its bits, so the distance
// and its reciprocal come from one reciprocal square root and the divisions by h and r become
// products with their reciprocals (1/h is loop-invariant in every caller).
__device__ __forceinline__ f3 cubic_gradient_tangent(const f3 d, const f3 t, const SphConstants& k) {
    const float r2 = dot(d, d);
    const float c = k.cubic_coefficient;
    const float inverse_h = 1.0F / k.h;
    if (r2 == 0.0F) return times(t, -12.0F * c * inverse_h * inverse_h);
    const float inverse_r = rsqrtf(r2);
    const float r = r2 * inverse_r;
    if (r >= k.h) return mk(0.0F, 0.0F, 0.0F);
    const float q = r * inverse_h;
    const float first = q <= 0.5F ? 18.0F * q * q - 12.0F * q : -6.0F * (1.0F - q) * (1.0F - q);
    const float second = q <= 0.5F ? 36.0F * q - 12.0F : 12.0F * (1.0F - q);
    const float radial_tangent = dot(d, t) * inverse_r;
    const float radial = c * first * inverse_h * inverse_r;
    const float radial_derivative = c * inverse_h * inverse_r * (second * inverse_h - first * inverse_r);
    return times(t, radial) + times(d, radial_derivative * radial_tangent);
}

// Directional derivative of the viscosity Laplacian (density/device.cuh:78-82), FP32.
__device__ __forceinline__ float laplacian_tangent(const f3 d, const f3 t, const SphConstants& k) {
    const float r2 = dot(d, d);
    if (r2 == 0.0F) return 0.0F;
    const float inverse_r = rsqrtf(r2);
    if (r2 * inverse_r >= k.h) return 0.0F;
    return -45.0F * dot(d, t) * inverse_r * (1.0F / k.laplacian_denominator);
}

// Hessian of the cubic kernel, in FP64 from the FP32 squared distance (density/device.cuh:59-70;
// the h h products are float there, and so in SphConstants::inverse_hh_d).
// CubicHessian is its scalar part for one displacement, shared by every vector the Hessian is
// applied to; H(-d) v = H(d) v exactly, because every step is sign-symmetric.
// The adjoint is held to FP64 rounding against the reference, not to its bits: one double
// reciprocal square root per pair replaces the square root and the divisions.  The support test
// stays exact, because for a float r2 and a float h, sqrt(r2) >= h in FP64 exactly when r2 >= h h
// (h h is exact in FP64, and a float r2 below it keeps sqrt(r2) more than half an FP64 ulp below h).
struct CubicHessian {
    double inverse_r, radial, radial_derivative, center;
    int kind;   // 0 outside the support, 1 at zero distance, 2 inside
};

__device__ __forceinline__ CubicHessian cubic_hessian(const f3 d, const SphConstants& k) {
    CubicHessian H{};
    const double r2 = static_cast<double>(sq_xfirst(d));
    const double c = k.cubic_coefficient_d;
    if (r2 == 0.0) {
        H.kind = 1;
        H.center = -12.0 * c * k.inverse_hh_d;
        return H;
    }
    if (r2 >= k.support_squared_d) return H;
    const double inverse_r = rsqrt(r2);
    const double q = r2 * inverse_r * k.inverse_h_d;
    const double first = q <= 0.5 ? 18.0 * q * q - 12.0 * q : -6.0 * (1.0 - q) * (1.0 - q);
    const double second = q <= 0.5 ? 36.0 * q - 12.0 : 12.0 * (1.0 - q);
    const double scale = c * inverse_r;
    H.inverse_r = inverse_r;
    H.radial = scale * first * k.inverse_h_d;                                            // c first / (h r)
    H.radial_derivative = scale * (second * k.inverse_hh_d - first * k.inverse_h_d * inverse_r);  // c (second / (hh r) - first / (h r r))
    H.kind = 2;
    return H;
}

__device__ __forceinline__ d3 hessian_times(const CubicHessian& H, const f3 d, const d3 v) {
    if (H.kind == 1) return times(v, H.center);
    if (H.kind == 0) return {0.0, 0.0, 0.0};
    return times(v, H.radial) + times(d, H.radial_derivative * dot(v, d) * H.inverse_r);
}

// Gradient of the viscosity Laplacian times `scalar`, in FP64 (density/device.cuh:84-88); -45 / (pi h^6)
// is the per-scene constant SphConstants::laplacian_scale_d, and the support test is the exact one above.
__device__ __forceinline__ d3 laplacian_gradient(const f3 d, const SphConstants& k, const double scalar) {
    const double r2 = static_cast<double>(sq_xfirst(d));
    if (r2 == 0.0 || r2 >= k.support_squared_d) return {0.0, 0.0, 0.0};
    return times(d, k.laplacian_scale_d * scalar * rsqrt(r2));
}

// The unclamped prediction's collision mask (sph/pcisph.cu:20-24, 69-71).
__device__ __forceinline__ void collision_mask(const f3 x, const f3 v, const f3 a, const float dt, const Box& box, bool& cx,
                                               bool& cy, bool& cz) {
    const f3 pos = fma3(dt, fma3(dt, a, v), x);
    cx = pos.x < box.min_x || pos.x > box.max_x;
    cy = pos.y < box.min_y || pos.y > box.max_y;
    cz = pos.z < box.min_z || pos.z > box.max_z;
}
}  // namespace detail
}  // namespace sph
}  // namespace pbf
