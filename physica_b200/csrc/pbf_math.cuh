// Device vector math for the PBF kernels.
//
// Bit-exact parity with the reference kernels needs every per-pair expression to be
// evaluated with the same operations in the same order, so that nvcc contracts
// multiply-adds the same way (default --fmad=true, IEEE division and square root).
// The helpers below therefore keep the operand order of the reference's
// domain/device.cuh:103-157 (component-wise add/sub, factor * component scaling,
// x*x + y*y + z*z dot products, the y-z / z-x / x-y cross product) and the kernel
// functions keep the evaluation order of density/device.cuh:10-24 and
// pbf/pbf.cu:18-71.  Names and structure are this library's own.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pbf {

struct f3 { float x, y, z; };
struct d3 { double x, y, z; };

__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 xyz(const float4 v) { return {v.x, v.y, v.z}; }

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

__device__ __forceinline__ float norm(const f3 a) { return sqrtf(dot(a, a)); }

// The float value of pi used by the reference kernels (density/device.cuh:8).
constexpr float kPi = 3.14159265358979323846F;

// Per-solver constants, derived on the device once so they come from the same
// device powf / division the reference evaluates inline.
struct KernelConstants {
    float h;              // support radius
    float h2;             // h * h
    float poly6_denominator;   // 64 pi h2 h2 h2 h h h           (density/device.cuh:15)
    float poly6_grad_denominator; // 32 pi h2 h2 h2 h h h        (density/device.cuh:23)
    float spiky_coefficient;   // -45 / (pi powf(h, 6))          (pbf/pbf.cu:30)
    float spiky_threshold;     // smallest r2 with sqrtf(r2) >= h: spiky is non-zero iff 0 < r2 < this
    float union_threshold;     // max(h2, spiky_threshold): any kernel non-zero needs r2 below it
    float poly6_radial_coefficient; // 315 / (64 pi powf(h, 9))  (pbf/pbf.cu:22)
    double spiky_coefficient_d;    // -45 / (pi pow(h, 6)) in FP64 (pbf/pbf.cu:52)
};

// poly6 weight for a squared distance already known to be below h2.
__device__ __forceinline__ float poly6_inside(const float r2, const KernelConstants& k) {
    const float difference = k.h2 - r2;
    return 315.0F * difference * difference * difference / k.poly6_denominator;
}

// poly6 kernel (zero outside the support).
__device__ __forceinline__ float poly6(const f3 d, const KernelConstants& k) {
    const float r2 = dot(d, d);
    if (r2 >= k.h2) return 0.0F;
    return poly6_inside(r2, k);
}

__device__ __forceinline__ f3 poly6_gradient(const f3 d, const KernelConstants& k) {
    const float r2 = dot(d, d);
    if (r2 >= k.h2) return {0.0F, 0.0F, 0.0F};
    const float difference = k.h2 - r2;
    return times(d, -945.0F * difference * difference / k.poly6_grad_denominator);
}

// Spiky gradient from a displacement whose length is `distance` (0 < distance < h).
__device__ __forceinline__ f3 spiky_gradient_at(const f3 d, const float distance, const KernelConstants& k) {
    const float difference = k.h - distance;
    return times(d, k.spiky_coefficient * difference * difference / distance);
}

__device__ __forceinline__ f3 spiky_gradient(const f3 d, const KernelConstants& k) {
    const float distance = norm(d);
    if (distance == 0.0F || distance >= k.h) return {0.0F, 0.0F, 0.0F};
    return spiky_gradient_at(d, distance, k);
}

}  // namespace pbf
