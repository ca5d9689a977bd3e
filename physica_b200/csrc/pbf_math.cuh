// Device vector math for the PBF kernels.
//
// Bit-exact parity with the reference kernels needs every per-pair expression to round
// exactly as the reference's compiled kernels do.  nvcc contracts a*b+c into fused
// multiply-adds by default, and which product it fuses depends on the surrounding code,
// so the FP32 arithmetic here is written with explicit round-to-nearest intrinsics
// (__fmaf_rn, __fmul_rn, __fadd_rn, __fsub_rn, __fdiv_rn, __fsqrt_rn), which the compiler
// never re-contracts.  The fused forms were determined by comparing each pass against
// the reference kernels on identical inputs, e.g.
//   squared distance          fma(dz, dz, fma(dx, dx, dy * dy))
//   cross product component   fma(a.y, b.z, -(a.z * b.y))
//   accumulations             fma(factor, term, accumulator)
//   |S|^2 after the lambda loop and |eta| after the normal loop
//                             fma(z, z, fma(y, y, x * x))
// The FP64 helpers of the adjoint keep the operand order of the reference's
// domain/device.cuh:103-157 and pbf/pbf.cu:45-54.  Names and structure are this library's own.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pbf {

struct f3 { float x, y, z; };
struct d3 { double x, y, z; };

__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 xyz(const float4 v) { return {v.x, v.y, v.z}; }

// ---------------------------------------------------------------- FP32, pinned rounding
__device__ __forceinline__ f3 add(const f3 a, const f3 b) {
    return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 sub(const f3 a, const f3 b) {
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 scale(const f3 v, const float s) {
    return {__fmul_rn(s, v.x), __fmul_rn(s, v.y), __fmul_rn(s, v.z)};
}
// acc + s * v, fused
__device__ __forceinline__ f3 fma3(const float s, const f3 v, const f3 acc) {
    return {__fmaf_rn(s, v.x, acc.x), __fmaf_rn(s, v.y, acc.y), __fmaf_rn(s, v.z, acc.z)};
}
// x*x + y*y + z*z as fma(z, z, fma(x, x, y*y))
__device__ __forceinline__ float sq_xfirst(const f3 d) {
    return __fmaf_rn(d.z, d.z, __fmaf_rn(d.x, d.x, __fmul_rn(d.y, d.y)));
}
// x*x + y*y + z*z as fma(z, z, fma(y, y, x*x))
__device__ __forceinline__ float sq_yfirst(const f3 d) {
    return __fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, __fmul_rn(d.x, d.x)));
}
// a x b with each component fma(p, q, -(r * s))
__device__ __forceinline__ f3 cross_f(const f3 a, const f3 b) {
    return {__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
            __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x))};
}

// ------------------------------------------------------------------- FP64 (adjoint)
__device__ __forceinline__ f3 operator+(const f3 a, const f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(const f3 a, const f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator+(const d3 a, const d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(const d3 a, const d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }

// factor * component, factor on the left (as the reference's scale()).
__device__ __forceinline__ f3 times(const f3 v, const float s) { return {s * v.x, s * v.y, s * v.z}; }
__device__ __forceinline__ d3 times(const f3 v, const double s) { return {s * v.x, s * v.y, s * v.z}; }
__device__ __forceinline__ d3 times(const d3 v, const double s) { return {s * v.x, s * v.y, s * v.z}; }

__device__ __forceinline__ float dot(const f3 a, const f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double dot(const d3 a, const f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double dot(const d3 a, const d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ f3 cross(const f3 a, const f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 cross(const f3 a, const d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 cross(const d3 a, const f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 cross(const d3 a, const d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// The float value of pi used by the reference kernels (density/device.cuh:8).
constexpr float kPi = 3.14159265358979323846F;

// Per-scene constants, derived on the device once so they come from the same
// device powf / division the reference evaluates inline.
struct KernelConstants {
    float h;              // support radius
    float h2;             // h * h
    float poly6_denominator;   // 64 pi h2 h2 h2 h h h           (density/device.cuh:15)
    float poly6_grad_denominator; // 32 pi h2 h2 h2 h h h        (density/device.cuh:23)
    float spiky_coefficient;   // -45 / (pi powf(h, 6))          (pbf/pbf.cu:30)
    float spiky_threshold;     // smallest r2 with sqrtf(r2) >= h: spiky is non-zero iff 0 < r2 < this
    float union_threshold;     // max(h2, spiky_threshold)
    float hessian_threshold;   // smallest r2 with sqrt((double)r2) >= h: the FP64 spiky Hessian is non-zero iff 0 < r2 < this
    float adjoint_threshold;   // max(spiky_threshold, hessian_threshold)
    float list_threshold;      // max of all: every kernel term of every pass is zero at r2 >= this
    float poly6_radial_coefficient; // 315 / (64 pi powf(h, 9))  (pbf/pbf.cu:22)
    double spiky_coefficient_d;    // -45 / (pi pow(h, 6)) in FP64 (pbf/pbf.cu:52)
};

// ------------------------------------------------------------ FP32 kernel functions
// Squared distance of a displacement, with the reference's rounding.
__device__ __forceinline__ float squared(const f3 d) { return sq_xfirst(d); }

// poly6 weight (density/device.cuh:10-16) for a squared distance already below h2.
__device__ __forceinline__ float poly6_inside(const float r2, const KernelConstants& k) {
    const float difference = __fsub_rn(k.h2, r2);
    return __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(315.0F, difference), difference), difference), k.poly6_denominator);
}

__device__ __forceinline__ float poly6(const f3 d, const KernelConstants& k) {
    const float r2 = squared(d);
    if (r2 >= k.h2) return 0.0F;
    return poly6_inside(r2, k);
}

// poly6 gradient (density/device.cuh:18-24).
__device__ __forceinline__ f3 poly6_gradient(const f3 d, const KernelConstants& k) {
    const float r2 = squared(d);
    if (r2 >= k.h2) return {0.0F, 0.0F, 0.0F};
    const float difference = __fsub_rn(k.h2, r2);
    return scale(d, __fdiv_rn(__fmul_rn(__fmul_rn(-945.0F, difference), difference), k.poly6_grad_denominator));
}

// Spiky gradient (pbf/pbf.cu:26-32) of a displacement of length `distance` (0 < distance < h).
__device__ __forceinline__ f3 spiky_gradient_at(const f3 d, const float distance, const KernelConstants& k) {
    const float difference = __fsub_rn(k.h, distance);
    return scale(d, __fdiv_rn(__fmul_rn(__fmul_rn(k.spiky_coefficient, difference), difference), distance));
}

__device__ __forceinline__ f3 spiky_gradient(const f3 d, const KernelConstants& k) {
    const float distance = __fsqrt_rn(squared(d));
    if (distance == 0.0F || distance >= k.h) return {0.0F, 0.0F, 0.0F};
    return spiky_gradient_at(d, distance, k);
}

// ------------------------------------------------------------------ FP64 helpers of the adjoint
__device__ __forceinline__ d3 ld3(const double4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ double4 st3(const d3 v) { return make_double4(v.x, v.y, v.z, 0.0); }

// Spiky Hessian applied to a vector, in FP64 (pbf/pbf.cu:45-54 evaluation order).
// The adjoint is held to FP64 rounding against the reference, so the distance and its reciprocal
// come from one reciprocal square root rather than a square root and a division; the support test
// is the exact one on the squared distance.
__device__ __forceinline__ d3 spiky_hessian_product(const f3 d, const d3 v, const KernelConstants& k) {
    const float r2f = squared(d);
    if (r2f == 0.0F || r2f >= k.hessian_threshold) return {0.0, 0.0, 0.0};   // sqrt((double)r2) == 0 or >= h
    const double r2 = r2f;
    const double inverse = rsqrt(r2);
    const double distance = r2 * inverse;
    const d3 direction = times(d, inverse);
    const double projection = dot(direction, v);
    const d3 direction_tangent = times(v - times(direction, projection), inverse);
    const double difference = k.h - distance;
    return times(times(direction, -2.0 * difference * projection) + times(direction_tangent, difference * difference),
                 k.spiky_coefficient_d);
}

// d/dr of poly6 along a radius (pbf/pbf.cu:18-24).
// H(d) v1 and H(d) v2 (as spiky_hessian_product) sharing one distance, inverse and direction.
// The spiky Hessian is even, H(-d) = H(d), and every step of the product is sign-symmetric, so
// H(-d) v equals H(d) v exactly: the reverse term of a pair uses the forward term's setup.
__device__ __forceinline__ void spiky_hessian_products(const f3 d, const d3 v1, const d3 v2, const KernelConstants& k, d3& out1,
                                                       d3& out2) {
    const float r2f = squared(d);
    if (r2f == 0.0F || r2f >= k.hessian_threshold) {   // sqrt((double)r2) == 0 or >= h
        out1 = out2 = {0.0, 0.0, 0.0};
        return;
    }
    const double r2 = r2f;
    const double inverse = rsqrt(r2);
    const double distance = r2 * inverse;
    const d3 direction = times(d, inverse);
    const double difference = k.h - distance;
    auto product = [&](const d3 v) {
        const double projection = dot(direction, v);
        const d3 direction_tangent = times(v - times(direction, projection), inverse);
        return times(times(direction, -2.0 * difference * projection) + times(direction_tangent, difference * difference),
                     k.spiky_coefficient_d);
    };
    out1 = product(v1);
    out2 = product(v2);
}

__device__ __forceinline__ float poly6_radial_derivative(const float radius, const KernelConstants& k) {
    if (radius >= k.h) return 0.0F;
    const float difference = __fmaf_rn(-radius, radius, __fmul_rn(k.h, k.h));
    return __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(-6.0F, k.poly6_radial_coefficient), radius), difference), difference);
}

// Artificial pressure s_corr = -strength (W(d)/W(radius))^exponent and its derivatives (pbf/pbf.cu:56-71).
struct ArtificialPressure {
    float value, d_strength, d_exponent, d_radius;
    f3 gradient;
};

__device__ __forceinline__ ArtificialPressure artificial_pressure(const f3 d, const KernelConstants& k, const float strength,
                                                                  const float exponent, const float radius) {
    ArtificialPressure a;
    const float reference = poly6(mk(radius, 0.0F, 0.0F), k);
    const float kernel = poly6(d, k);
    if (kernel == 0.0F) {
        a.value = a.d_strength = a.d_exponent = a.d_radius = 0.0F;
        a.gradient = {0.0F, 0.0F, 0.0F};
        return a;
    }
    const float ratio = __fdiv_rn(kernel, reference);
    const float power = powf(ratio, exponent);
    a.value = __fmul_rn(-strength, power);
    a.d_strength = -power;
    a.d_exponent = __fmul_rn(a.value, logf(ratio));
    a.d_radius = __fdiv_rn(__fmul_rn(__fmul_rn(-a.value, exponent), poly6_radial_derivative(radius, k)), reference);
    a.gradient = scale(poly6_gradient(d, k),
                       __fdiv_rn(__fmul_rn(__fmul_rn(-strength, exponent), powf(ratio, exponent - 1.0F)), reference));
    return a;
}

}  // namespace pbf
