// Forward-mode substep (PBF::jvp_step, pbf/pbf.cpp:193-215) over cell-sorted particles.
//
// The reference recomputes every Jacobi iteration beside its tangent kernels.  The differentiable
// forward here records every iterate and its primal fields (x_k, density, gradient sum S,
// denominator D, lambda, collision mask, and the post-loop fields), so the tangent sweep only runs
// the tangent passes, each over the ordered neighbour list the forward stored for that iterate:
//   seed: predict JVP (pbf.cu:80-84) and the sorted parameter tangents
//   per iteration k:
//     density JVP (density/density.cu:42-66) + lambda JVP (pbf.cu:129-178), one pass
//     correction JVP (pbf.cu:290-333) + project JVP (pbf.cu:433-442), and on the last
//     iteration reconstruct JVP (pbf.cu:462-466)
//   vorticity JVP (pbf.cu:499-526) + magnitude JVP (pbf.cu:595-599)
//   normal JVP (pbf.cu:601-631) + confinement JVP (pbf.cu:680-686)
//   XSPH JVP (pbf.cu:723-754)
// Tangents are FP32, as in the reference.  Every pair outside a term's support contributes an
// exact zero there, so the in-support lists give the same sums up to FP32 rounding.
#include "engine.h"
#include "gather.cuh"

namespace pbf {

struct TangentWorkspace {
    DeviceArena arena;
    float4* x[2] = {nullptr, nullptr};   // iterate position tangents (ping-pong), sorted
    float4* x_state = nullptr;           // position tangent of the input state, sorted
    float* lambda = nullptr;             // lambda tangent of the current iteration
    float4* velocity = nullptr;          // reconstructed-velocity tangent
    float4* vorticity = nullptr;         // (vorticity tangent, magnitude tangent)
    float4* confined = nullptr;          // confined-velocity tangent
    float4* params_a = nullptr;          // tangents of (mass, rest density, relaxation, xsph viscosity)
    float4* params_b = nullptr;          // tangents of (s_corr strength, exponent, radius, vorticity confinement)
};

void destroy_tangent_workspace(void* workspace) { delete static_cast<TangentWorkspace*>(workspace); }

namespace {

using namespace gather_detail;

inline unsigned blocks_of(const uint32_t n, const unsigned block) { return (n + block - 1) / block; }

// Caller-side FP32 parameter tangents (original order); a null pointer is a zero tangent.
struct ParamTangent {
    const float* masses;
    const float* rest_densities;
    const float* relaxation;
    const float* strength;
    const float* exponent;
    const float* radius;
    const float* xsph;
    const float* vorticity;
};

__device__ __forceinline__ float or_zero(const float* p, const uint32_t i) { return p ? p[i] : 0.0F; }

__device__ __forceinline__ f3 masked(f3 a, const uint32_t mask) {
    if ((mask & 1u) != 0u) a.x = 0.0F;
    if ((mask & 2u) != 0u) a.y = 0.0F;
    if ((mask & 4u) != 0u) a.z = 0.0F;
    return a;
}

// Directional derivative of the spiky gradient (pbf.cu:34-43) for 0 < distance < h.
__device__ __forceinline__ f3 spiky_gradient_tangent(const f3 d, const f3 dd, const float distance, const KernelConstants& k) {
    const f3 direction = times(d, 1.0F / distance);
    const float radial = dot(direction, dd);
    const f3 direction_tangent = times(dd + times(direction, -radial), 1.0F / distance);
    const float difference = k.h - distance;
    return times(times(direction, -2.0F * difference * radial) + times(direction_tangent, difference * difference),
                 k.spiky_coefficient);
}

// The spiky gradient (pbf.cu:26-32) and its directional derivative (pbf.cu:34-43) of one pair with
// 0 < r2 < spiky_threshold, sharing one reciprocal square root.  The tangent passes are held to FP32
// rounding against the reference, not to its bits, so they need not repeat its IEEE square root
// and divisions pair by pair.
__device__ __forceinline__ void spiky_pair(const f3 d, const f3 dd, const float r2, const KernelConstants& k, f3& gradient,
                                           f3& gradient_dot) {
    const float inverse = rsqrtf(r2);
    const float distance = r2 * inverse;
    const f3 direction = times(d, inverse);
    const float difference = k.h - distance;
    const float radial = dot(direction, dd);
    gradient = times(direction, k.spiky_coefficient * difference * difference);
    const f3 direction_tangent = times(dd + times(direction, -radial), inverse);
    gradient_dot = times(times(direction, -2.0F * difference * radial) + times(direction_tangent, difference * difference),
                         k.spiky_coefficient);
}

// ------------------------------------------------------------------- seed
__global__ void tangent_seed_kernel(const uint32_t count, const uint32_t* __restrict__ sorted_index, const int4* __restrict__ cell,
                                    const SceneDesc* __restrict__ scenes, const Field3 x_dot, const Field3 v_dot,
                                    const Field3 a_dot, const ParamTangent pt, float4* __restrict__ x0,
                                    float4* __restrict__ x_state, float4* __restrict__ params_a, float4* __restrict__ params_b) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint32_t i = sorted_index[s];
    const float dt = scenes[cell[s].w].time_step;
    const f3 xd = mk(x_dot.x[i], x_dot.y[i], x_dot.z[i]);
    const f3 vd = mk(v_dot.x[i], v_dot.y[i], v_dot.z[i]);
    const f3 ad = mk(a_dot.x[i], a_dot.y[i], a_dot.z[i]);
    const f3 predicted = xd + times(vd + times(ad, dt), dt);
    x0[s] = make_float4(predicted.x, predicted.y, predicted.z, 0.0F);
    x_state[s] = make_float4(xd.x, xd.y, xd.z, 0.0F);
    params_a[s] = make_float4(or_zero(pt.masses, i), or_zero(pt.rest_densities, i), or_zero(pt.relaxation, i), or_zero(pt.xsph, i));
    params_b[s] = make_float4(or_zero(pt.strength, i), or_zero(pt.exponent, i), or_zero(pt.radius, i), or_zero(pt.vorticity, i));
}

struct Pair {
    float4 q;    // neighbour position and mass
    float4 qd;   // neighbour position tangent
    float4 aux;  // pass-specific neighbour data
};

// ------------------------------------------------------ density + lambda
struct DensityLambdaJvpArgs {
    GatherCommon g;
    StoredList list;
    const float4* pos;
    const float4* x_dot;
    const float4* params_a_dot;
    const float* density;
    const float4* gsum_denom;
    float* lambda_dot;
};

struct DensityLambdaJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    const float4* __restrict__ x_dot;
    const float4* __restrict__ params_a_dot;
    f3 x, xd;
    uint32_t self;
    float rest, rest_dot, inverse_rest;
    KernelConstants k;
    float density_dot, denominator_dot;
    f3 gsum_dot;

    __device__ __forceinline__ Pair prefetch(const uint32_t t) const {
        if (t & kBoundaryBit) return {boundary[t & ~kBoundaryBit], make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0)};
        return {pos[t], x_dot[t], params_a_dot[t]};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const Pair& in) {
        const f3 d = x - xyz(in.q);
        const f3 dd = xd - xyz(in.qd);
        const float r2 = squared(d);
        if (t & kBoundaryBit) {
            // boundary particle b (density/density.cu:59-63, pbf.cu:164-169); it does not move with
            // the inputs, so the displacement tangent is x_dot_i
            const float volume = in.q.w;
            if (r2 < k.h2) density_dot += volume * (rest_dot * poly6_inside(r2, k) + rest * dot(poly6_gradient(d, k), xd));
            const float distance = sqrtf(r2);
            if (distance == 0.0F || distance >= k.h) return;
            gsum_dot = gsum_dot + times(spiky_gradient_tangent(d, xd, distance, k), volume);
            return;
        }
        const float mass_dot = in.aux.x;
        if (r2 < k.h2) density_dot += mass_dot * poly6_inside(r2, k) + in.q.w * dot(poly6_gradient(d, k), dd);
        if (t == self) return;
        // one reciprocal square root per pair and the reciprocal rest density instead of IEEE
        // divisions (the 1M tangent step: 10.65 -> 9.65 ms; 1.6e-7 relative to the reference
        // before and after)
        if (r2 == 0.0F || r2 >= k.spiky_threshold) return;   // sqrtf(r2) == 0 or >= h
        f3 gradient, gradient_dot;
        spiky_pair(d, dd, r2, k, gradient, gradient_dot);
        const float coefficient = in.q.w * inverse_rest;
        const float coefficient_dot = (mass_dot - in.q.w * rest_dot * inverse_rest) * inverse_rest;
        const f3 ng = times(gradient, coefficient);
        const f3 ng_dot = times(gradient, coefficient_dot) + times(gradient_dot, coefficient);
        gsum_dot = gsum_dot + ng_dot;
        denominator_dot += 2.0F * dot(ng, ng_dot);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

// Resident 128-thread blocks per SM the register budget of the tangent's list-replay passes is
// sized for (a compile-time tuning knob; 0 leaves the register count to the compiler).  At 1M
// particles the tangent step took 8.46 ms with the compiler's registers (61-72), 8.47 at a
// one-block minimum (62-88), 8.53 at 9 (56 registers) and 9.78 at 10 (48).
#ifndef PBF_JVP_MIN_BLOCKS
#define PBF_JVP_MIN_BLOCKS 0
#endif
__global__ void __launch_bounds__(kBlock, PBF_JVP_MIN_BLOCKS) density_lambda_jvp_kernel(const DensityLambdaJvpArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    DensityLambdaJvpOp op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    op.x_dot = a.x_dot;
    op.params_a_dot = a.params_a_dot;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.xd = xyz(a.x_dot[p.s]);
    const float4 pa = a.g.params_a[p.s];
    const float4 pad = a.params_a_dot[p.s];
    op.rest = pa.x;
    op.rest_dot = pad.y;
    op.inverse_rest = 1.0F / pa.x;
    op.density_dot = 0.0F;
    op.denominator_dot = pad.z;   // relaxation tangent
    op.gsum_dot = mk(0.0F, 0.0F, 0.0F);
    replay(op, p, a.g, a.list);
    const float4 gd = a.gsum_denom[p.s];
    const float denominator_dot = op.denominator_dot + 2.0F * dot(xyz(gd), op.gsum_dot);
    const float density = a.density[p.s];
    const float constraint = density / op.rest - 1.0F;
    const float constraint_dot = op.density_dot / op.rest - density * op.rest_dot / (op.rest * op.rest);
    a.lambda_dot[p.s] = -constraint_dot / gd.w + constraint * denominator_dot / (gd.w * gd.w);
}

// ---------------------------------------------------- correction + project
struct CorrectionJvpArgs {
    GatherCommon g;
    StoredList list;
    const float4* pos;
    const float4* x_dot;
    const float* lambda;
    const float* lambda_dot;
    const float4* params_a_dot;
    const float4* params_b_dot;
    const uint8_t* mask;
    float4* x_dot_next;
    int last;
    const uint32_t* sorted_index;
    const float4* x_state;
    float4* velocity_dot;      // reconstructed-velocity tangent (last iteration)
    MutField3 out_positions;   // next-state position tangent (last iteration)
};

struct CorrectionPair {
    float4 q, qd;
    float lambda, lambda_dot, mass_dot;
};

struct CorrectionJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    const float4* __restrict__ x_dot;
    const float* __restrict__ lambda;
    const float* __restrict__ lambda_dot;
    const float4* __restrict__ params_a_dot;
    f3 x, xd;
    uint32_t self;
    float rest, rest_dot, inverse_rest, lambda_i, lambda_dot_i;
    float strength, exponent, radius, strength_dot, exponent_dot, radius_dot;
    bool artificial;
    KernelConstants k;
    f3 result;

    __device__ __forceinline__ CorrectionPair prefetch(const uint32_t t) const {
        if (t & kBoundaryBit) return {boundary[t & ~kBoundaryBit], make_float4(0, 0, 0, 0), 0.0F, 0.0F, 0.0F};
        return {pos[t], x_dot[t], lambda[t], lambda_dot[t], params_a_dot[t].x};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const CorrectionPair& in) {
        if (t == self) return;
        const f3 d = x - xyz(in.q);
        const f3 dd = xd - xyz(in.qd);
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.spiky_threshold) return;   // both spiky terms vanish (sqrtf(r2) == 0 or >= h)
        const float distance = sqrtf(r2);
        float art = 0.0F, art_dot = 0.0F;
        if (artificial) {
            const ArtificialPressure ap = artificial_pressure(d, k, strength, exponent, radius);
            art = ap.value;
            art_dot = dot(ap.gradient, dd) + ap.d_strength * strength_dot + ap.d_exponent * exponent_dot + ap.d_radius * radius_dot;
        }
        if (t & kBoundaryBit) {
            // boundary particle b (pbf.cu:321-330)
            const float multiplier = lambda_i + art;
            result = result + times(times(spiky_gradient_at(d, distance, k), lambda_dot_i + art_dot) +
                                        times(spiky_gradient_tangent(d, dd, distance, k), multiplier),
                                    in.q.w);
            return;
        }
        f3 gradient, gradient_dot;
        spiky_pair(d, dd, r2, k, gradient, gradient_dot);
        const float coefficient = in.q.w * inverse_rest;
        const float coefficient_dot = (in.mass_dot - in.q.w * rest_dot * inverse_rest) * inverse_rest;
        const float multiplier = lambda_i + in.lambda + art;
        const float multiplier_dot = lambda_dot_i + in.lambda_dot + art_dot;
        result = result + times(gradient, coefficient_dot * multiplier + coefficient * multiplier_dot) +
                 times(gradient_dot, coefficient * multiplier);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

// Seven resident blocks per SM (at most 72 registers, a few spilled) against 88 registers and five
// blocks unbounded: the pass waits on its neighbours' loads, and the extra warps hide more of that
// (the 1M tangent step fell from 11.54 to 10.64 ms; 80 and 64 registers were slower).
__global__ void __launch_bounds__(kBlock, 7) correction_jvp_kernel(const CorrectionJvpArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    CorrectionJvpOp op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    op.x_dot = a.x_dot;
    op.lambda = a.lambda;
    op.lambda_dot = a.lambda_dot;
    op.params_a_dot = a.params_a_dot;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.xd = xyz(a.x_dot[p.s]);
    const float4 pa = a.g.params_a[p.s], pb = a.g.params_b[p.s];
    const float4 pad = a.params_a_dot[p.s], pbd = a.params_b_dot[p.s];
    op.rest = pa.x;
    op.inverse_rest = 1.0F / pa.x;
    op.rest_dot = pad.y;
    op.lambda_i = a.lambda[p.s];
    op.lambda_dot_i = a.lambda_dot[p.s];
    op.strength = pb.x;
    op.exponent = pb.y;
    op.radius = pb.z;
    op.strength_dot = pbd.x;
    op.exponent_dot = pbd.y;
    op.radius_dot = pbd.z;
    // With zero strength and zero s_corr tangents every s_corr term and tangent is zero.
    op.artificial = pb.x != 0.0F || pbd.x != 0.0F || pbd.y != 0.0F || pbd.z != 0.0F;
    op.result = mk(0.0F, 0.0F, 0.0F);
    replay(op, p, a.g, a.list);
    const f3 next = masked(op.xd + op.result, a.mask[p.s]);
    a.x_dot_next[p.s] = make_float4(next.x, next.y, next.z, 0.0F);
    if (!a.last) return;
    const uint32_t i = a.sorted_index[p.s];
    a.out_positions.x[i] = next.x;
    a.out_positions.y[i] = next.y;
    a.out_positions.z[i] = next.z;
    const f3 v = times(next - xyz(a.x_state[p.s]), p.scene->inverse_time_step);
    a.velocity_dot[p.s] = make_float4(v.x, v.y, v.z, 0.0F);
}

// Reconstruct JVP when no Jacobi iteration runs (K = 0).
__global__ void tangent_reconstruct_kernel(const uint32_t count, const int4* __restrict__ cell, const SceneDesc* __restrict__ scenes,
                                           const uint32_t* __restrict__ sorted_index, const float4* __restrict__ x_dot,
                                           const float4* __restrict__ x_state, float4* __restrict__ velocity_dot,
                                           const MutField3 out_positions) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const f3 xd = xyz(x_dot[s]);
    const uint32_t i = sorted_index[s];
    out_positions.x[i] = xd.x;
    out_positions.y[i] = xd.y;
    out_positions.z[i] = xd.z;
    const f3 v = times(xd - xyz(x_state[s]), scenes[cell[s].w].inverse_time_step);
    velocity_dot[s] = make_float4(v.x, v.y, v.z, 0.0F);
}

// -------------------------------------------------------------- vorticity
struct VorticityJvpArgs {
    GatherCommon g;
    StoredList list;
    const float4* pos;
    const float4* x_dot;
    const float4* velocity;
    const float4* velocity_dot;
    const float4* vorticity;
    float4* vorticity_dot;
};

struct VorticityJvpOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ x_dot;
    const float4* __restrict__ velocity;
    const float4* __restrict__ velocity_dot;
    f3 x, xd, v, vd;
    uint32_t self;
    KernelConstants k;
    f3 result;

    struct Data {
        float4 q, qd, w, wd;
    };
    __device__ __forceinline__ Data prefetch(const uint32_t t) const { return {pos[t], x_dot[t], velocity[t], velocity_dot[t]}; }
    __device__ __forceinline__ void apply(const uint32_t t, const Data& in) {
        if (t == self) return;
        const f3 d = x - xyz(in.q);
        const f3 dd = xd - xyz(in.qd);
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.spiky_threshold) return;   // sqrtf(r2) == 0 or >= h
        f3 gradient, gradient_dot;
        spiky_pair(d, dd, r2, k, gradient, gradient_dot);
        const f3 difference = xyz(in.w) - v;
        const f3 difference_dot = xyz(in.wd) - vd;
        result = result + cross(difference_dot, gradient) + cross(difference, gradient_dot);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_JVP_MIN_BLOCKS) vorticity_jvp_kernel(const VorticityJvpArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    VorticityJvpOp op;
    op.pos = a.pos;
    op.x_dot = a.x_dot;
    op.velocity = a.velocity;
    op.velocity_dot = a.velocity_dot;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.xd = xyz(a.x_dot[p.s]);
    op.v = xyz(a.velocity[p.s]);
    op.vd = xyz(a.velocity_dot[p.s]);
    op.result = mk(0.0F, 0.0F, 0.0F);
    replay(op, p, a.g, a.list);
    const float4 w = a.vorticity[p.s];   // (omega, |omega|)
    const float magnitude_dot = w.w > 0.0F ? dot(xyz(w), op.result) / w.w : 0.0F;
    a.vorticity_dot[p.s] = make_float4(op.result.x, op.result.y, op.result.z, magnitude_dot);
}

// ------------------------------------------------------ normal + confinement
struct NormalJvpArgs {
    GatherCommon g;
    StoredList list;
    const float4* pos;
    const float4* x_dot;
    const float4* vorticity;       // (omega, |omega|)
    const float4* vorticity_dot;   // (omega dot, |omega| dot)
    const float4* normal;          // (N, |eta|)
    const float4* velocity_dot;
    const float4* params_b_dot;
    float4* confined_dot;
};

struct NormalJvpOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ x_dot;
    const float4* __restrict__ vorticity;
    const float4* __restrict__ vorticity_dot;
    f3 x, xd;
    float magnitude, magnitude_dot;
    uint32_t self;
    KernelConstants k;
    f3 result;

    struct Data {
        float4 q, qd;
        float m, md;
    };
    __device__ __forceinline__ Data prefetch(const uint32_t t) const {
        return {pos[t], x_dot[t], vorticity[t].w, vorticity_dot[t].w};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const Data& in) {
        if (t == self) return;
        const f3 d = x - xyz(in.q);
        const f3 dd = xd - xyz(in.qd);
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.spiky_threshold) return;   // sqrtf(r2) == 0 or >= h
        f3 gradient, gradient_dot;
        spiky_pair(d, dd, r2, k, gradient, gradient_dot);
        result = result + times(gradient, in.md - magnitude_dot) + times(gradient_dot, in.m - magnitude);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_JVP_MIN_BLOCKS) normal_jvp_kernel(const NormalJvpArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    NormalJvpOp op;
    op.pos = a.pos;
    op.x_dot = a.x_dot;
    op.vorticity = a.vorticity;
    op.vorticity_dot = a.vorticity_dot;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.xd = xyz(a.x_dot[p.s]);
    const float4 w = a.vorticity[p.s], wd = a.vorticity_dot[p.s];
    op.magnitude = w.w;
    op.magnitude_dot = wd.w;
    op.result = mk(0.0F, 0.0F, 0.0F);
    replay(op, p, a.g, a.list);
    const float4 nrm = a.normal[p.s];
    const f3 normal = xyz(nrm);
    const f3 normal_dot = nrm.w == 0.0F ? mk(0.0F, 0.0F, 0.0F)
                                        : times(op.result + times(normal, -dot(normal, op.result)), 1.0F / nrm.w);
    // confinement JVP: v_c = v_r + (N x omega) (dt eps)
    const f3 omega = xyz(w), omega_dot = xyz(wd);
    const f3 force = cross(normal, omega);
    const f3 force_dot = cross(normal_dot, omega) + cross(normal, omega_dot);
    const float dt = p.scene->time_step;
    const float eps = a.g.params_a[p.s].w, eps_dot = a.params_b_dot[p.s].w;
    const f3 vc = xyz(a.velocity_dot[p.s]) + times(times(force, eps_dot) + times(force_dot, eps), dt);
    a.confined_dot[p.s] = make_float4(vc.x, vc.y, vc.z, 0.0F);
}

// ------------------------------------------------------------------- XSPH
struct XsphJvpArgs {
    GatherCommon g;
    StoredList list;
    const float4* pos;
    const float4* x_dot;
    const float4* confined;
    const float4* confined_dot;
    const float4* params_a_dot;
    const uint32_t* sorted_index;
    MutField3 out_velocities;
};

struct XsphJvpOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ x_dot;
    const float4* __restrict__ confined;
    const float4* __restrict__ confined_dot;
    f3 x, xd, v, vd;
    uint32_t self;
    KernelConstants k;
    f3 smoothing, smoothing_dot;

    struct Data {
        float4 q, qd, w, wd;
    };
    __device__ __forceinline__ Data prefetch(const uint32_t t) const { return {pos[t], x_dot[t], confined[t], confined_dot[t]}; }
    __device__ __forceinline__ void apply(const uint32_t t, const Data& in) {
        if (t == self) return;
        const f3 d = x - xyz(in.q);
        const float r2 = squared(d);
        if (r2 >= k.h2) return;
        const f3 dd = xd - xyz(in.qd);
        const float weight = poly6_inside(r2, k);
        const float weight_dot = dot(poly6_gradient(d, k), dd);
        const f3 difference = xyz(in.w) - v;
        const f3 difference_dot = xyz(in.wd) - vd;
        smoothing = smoothing + times(difference, weight);
        smoothing_dot = smoothing_dot + times(difference_dot, weight) + times(difference, weight_dot);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_JVP_MIN_BLOCKS) xsph_jvp_kernel(const XsphJvpArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    XsphJvpOp op;
    op.pos = a.pos;
    op.x_dot = a.x_dot;
    op.confined = a.confined;
    op.confined_dot = a.confined_dot;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.xd = xyz(a.x_dot[p.s]);
    op.v = xyz(a.confined[p.s]);
    op.vd = xyz(a.confined_dot[p.s]);
    op.smoothing = mk(0.0F, 0.0F, 0.0F);
    op.smoothing_dot = mk(0.0F, 0.0F, 0.0F);
    replay(op, p, a.g, a.list);
    const float c = a.g.params_a[p.s].z, c_dot = a.params_a_dot[p.s].w;
    const f3 out = op.vd + (times(op.smoothing, c_dot) + times(op.smoothing_dot, c));
    const uint32_t i = a.sorted_index[p.s];
    a.out_velocities.x[i] = out.x;
    a.out_velocities.y[i] = out.y;
    a.out_velocities.z[i] = out.z;
}

bool has3(const pbf_vector_field& f) { return f.x && f.y && f.z; }

}  // namespace

int Engine::tangent(const pbf_particle_state* state, const StepRecord& r, const pbf_particle_state_tangent* state_tangent,
                    const pbf_control* control_tangent, const pbf_parameter_tangent* parameter_tangent,
                    pbf_particle_state_tangent* next_state_tangent) {
    if (!differentiable()) {
        set_error("jvp_step needs PBF_EXECUTION_DIFFERENTIABLE");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    if (!state || !state_tangent || !control_tangent || !next_state_tangent) {
        set_error("null argument");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!r.valid || r.step_index != state->step_index) {
        set_error("the step cache does not hold the forward step of this state");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    const uint32_t n = count_, K = iterations_;
    if (n == 0) return PBF_SUCCESS;
    if (!has3(state_tangent->positions) || !has3(state_tangent->velocities) || !has3(control_tangent->external_accelerations) ||
        !has3(next_state_tangent->positions) || !has3(next_state_tangent->velocities)) {
        set_error("null tangent field");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    auto* ws = static_cast<TangentWorkspace*>(tangent_);
    if (!ws) {
        ws = new TangentWorkspace();
        ws->arena.set_stream(stream_);
        cudaError_t e = cudaSuccess;
        ws->x[0] = ws->arena.alloc<float4>(n, e);
        ws->x[1] = ws->arena.alloc<float4>(n, e);
        ws->x_state = ws->arena.alloc<float4>(n, e);
        ws->lambda = ws->arena.alloc<float>(n, e);
        ws->velocity = ws->arena.alloc<float4>(n, e);
        ws->vorticity = ws->arena.alloc<float4>(n, e);
        ws->confined = ws->arena.alloc<float4>(n, e);
        ws->params_a = ws->arena.alloc<float4>(n, e);
        ws->params_b = ws->arena.alloc<float4>(n, e);
        if (e != cudaSuccess) {
            delete ws;
            return check(e, "tangent workspace");
        }
        tangent_ = ws;
    }
    ParamTangent pt{};
    if (parameter_tangent) {
        pt = {parameter_tangent->masses, parameter_tangent->rest_densities, parameter_tangent->relaxation,
              parameter_tangent->artificial_pressure_strength, parameter_tangent->artificial_pressure_exponent,
              parameter_tangent->artificial_pressure_radius, parameter_tangent->xsph_viscosity,
              parameter_tangent->vorticity_confinement};
    }
    const GatherCommon gc = gather_common(r);
    // Passes that replay the same list run in alternating block orders, each starting on the entries
    // the previous pass read last (still in L2).
    GatherCommon gc_reverse = gc;
    gc_reverse.reverse = 1;
    const unsigned block = shape_.block;
    const unsigned blocks = blocks_of(n, block);
    const MutField3 out_x{next_state_tangent->positions.x, next_state_tangent->positions.y, next_state_tangent->positions.z};
    const MutField3 out_v{next_state_tangent->velocities.x, next_state_tangent->velocities.y, next_state_tangent->velocities.z};

    timer_.begin(stream_, kPassTangentSeed);
    tangent_seed_kernel<<<blocks_of(n, 256), 256, 0, stream_>>>(
        n, r.sorted_index, r.cell, d_scenes_,
        {state_tangent->positions.x, state_tangent->positions.y, state_tangent->positions.z},
        {state_tangent->velocities.x, state_tangent->velocities.y, state_tangent->velocities.z},
        {control_tangent->external_accelerations.x, control_tangent->external_accelerations.y,
         control_tangent->external_accelerations.z},
        pt, ws->x[0], ws->x_state, ws->params_a, ws->params_b);
    timer_.end(stream_, kPassTangentSeed);
    count_launch();
    const bool keep = r.keeps_all(true);
    Segment* sg = nullptr;
    if (!keep)
        if (int rc = segment_workspace(&sg)) return rc;
    for (uint32_t k = 0; k < K; ++k) {
        const float4* xk;
        StoredList list;
        const float* lambda_k;
        const float* density_k;
        const float4* gsum_k;
        if (keep) {
            xk = r.iterate(k, K, true);
            list = StoredList{r.list_entries[k], r.list_counts[k], r.list_capacity};
            lambda_k = r.lambda[k];
            density_k = r.density[k];
            gsum_k = r.gsum[k];
        } else {
            // Checkpoint recomputation: the primal iterations run again in order (pbf/pbf.cpp:198-212),
            // one at a time in the segment workspace's first slot, the iterates in its two ping-pong
            // buffers (iterate 0 is x*).
            xk = k == 0 ? r.topology : sg->positions[(k - 1u) & 1u];
            list = StoredList{sg->list_entries[0], sg->list_counts[0], kListCapacity};
            lambda_k = sg->lambda[0];
            density_k = sg->density[0];
            gsum_k = sg->gsum[0];
            ListScanArgs scan{gc, xk, list, 1};
            if (k > 0) scan.packed = packed_;   // written by the previous primal correction
            DensityLambdaArgs d{gc, xk, sg->lambda[0], sg->density[0], sg->gsum[0], nullptr, list};
            if (fuses_density(shape_, scan)) {
                if (int rc = check(launch_scan_density_lambda(stream_, scan, d, shape_), "recompute: scan + density/lambda"))
                    return rc;
            } else {
                if (int rc = check(launch_list_scan(stream_, scan, shape_), "recompute: neighbour list scan")) return rc;
                if (int rc = check(launch_density_lambda(stream_, d, shape_.block), "recompute: density/lambda")) return rc;
            }
        }
        DensityLambdaJvpArgs dl{gc, list, xk, ws->x[k & 1u], ws->params_a, density_k, gsum_k, ws->lambda};
        timer_.begin(stream_, kPassDensityLambdaJvp);
        density_lambda_jvp_kernel<<<blocks, block, 0, stream_>>>(dl);
        timer_.end(stream_, kPassDensityLambdaJvp);
        if (!keep && k + 1u < K) {   // the next primal iterate (the last one, x_K, is kept)
            CorrectionArgs c{gc, xk, sg->lambda[0], sg->positions[k & 1u], nullptr, 0, Field3{}, r.sorted_index, MutField3{},
                             nullptr, list};
            c.packed = packed_;
            if (int rc = check(launch_correction(stream_, c, shape_.block), "recompute: correction/project")) return rc;
        }
        CorrectionJvpArgs ca{gc_reverse, list, xk, ws->x[k & 1u], lambda_k, ws->lambda, ws->params_a, ws->params_b, r.mask[k],
                             ws->x[(k + 1u) & 1u], k + 1u == K ? 1 : 0, r.sorted_index, ws->x_state, ws->velocity, out_x};
        timer_.begin(stream_, kPassCorrectionJvp);
        correction_jvp_kernel<<<blocks, block, 0, stream_>>>(ca);
        timer_.end(stream_, kPassCorrectionJvp);
        count_launch(2);
    }
    const float4* x_dot_K = ws->x[K & 1u];
    if (K == 0) {
        tangent_reconstruct_kernel<<<blocks_of(n, 256), 256, 0, stream_>>>(n, r.cell, d_scenes_, r.sorted_index, x_dot_K,
                                                                           ws->x_state, ws->velocity, out_x);
        count_launch();
    }
    const float4* xK = r.iterate(K, K, true);
    const StoredList post{r.list_entries[keep ? K : 0u], r.list_counts[keep ? K : 0u], r.list_capacity};
    VorticityJvpArgs va{gc, post, xK, x_dot_K, r.velocity, ws->velocity, r.vorticity, ws->vorticity};
    timer_.begin(stream_, kPassVorticityJvp);
    vorticity_jvp_kernel<<<blocks, block, 0, stream_>>>(va);
    timer_.end(stream_, kPassVorticityJvp);
    NormalJvpArgs na{gc_reverse, post, xK, x_dot_K, r.vorticity, ws->vorticity, r.normal, ws->velocity, ws->params_b, ws->confined};
    timer_.begin(stream_, kPassNormalJvp);
    normal_jvp_kernel<<<blocks, block, 0, stream_>>>(na);
    timer_.end(stream_, kPassNormalJvp);
    XsphJvpArgs xa{gc, post, xK, x_dot_K, r.confined, ws->confined, ws->params_a, r.sorted_index, out_v};
    timer_.begin(stream_, kPassXsphJvp);
    xsph_jvp_kernel<<<blocks, block, 0, stream_>>>(xa);
    timer_.end(stream_, kPassXsphJvp);
    count_launch(3);
    return check(cudaGetLastError(), "jvp_step");
}

}  // namespace pbf
