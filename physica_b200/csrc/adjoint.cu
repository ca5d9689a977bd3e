// Reverse-mode substep (PBF::vjp_step, pbf/pbf.cpp:217-258) over cell-sorted particles.
//
// The differentiable forward records every Jacobi iterate and its primal fields (x_k,
// density, gradient sum S, denominator D, lambda, collision mask), so the reverse sweep
// recomputes nothing.  Each adjoint pass is the reference's pull formulation (a particle
// adds both its own i->j terms and the reverse j->i terms, so no atomics) with its FP64
// expressions, over the same ordered neighbour gather as the forward passes:
//   xsph VJP (pbf.cu:756-790) + confinement VJP (pbf.cu:688-698) + normalised-input adjoint
//   normal VJP (pbf.cu:633-672)
//   vorticity VJP (pbf.cu:528-563) + reconstruct VJP (pbf.cu:468-474) + project VJP (pbf.cu:444-454)
//   per iteration, last to first:
//     correction VJP (pbf.cu:335-415)
//     lambda VJP (pbf.cu:180-252, its two neighbour loops)
//     density VJP (density/density.cu:69-102) + project VJP of the previous iteration,
//     or predict VJP (pbf.cu:86-93) after the first iteration.
// Buffers that the reference clears before accumulating into them are written as
// 0.0 + contribution, which reproduces its values including the sign of zero.
#include "engine.h"
#include "gather.cuh"

namespace pbf {

struct AdjointWorkspace {
    DeviceArena arena;
    double4* x[2] = {nullptr, nullptr};   // position adjoint ping-pong
    double4* correction = nullptr;
    double4* output_velocity = nullptr;   // next-state velocity adjoint in sorted order
    double4* vorticity = nullptr;
    double4* velocity = nullptr;          // reconstructed-velocity adjoint
    double4* eta = nullptr;               // adjoint of the unnormalised vorticity-magnitude gradient
    double* lambda = nullptr;
    double* density = nullptr;
    double* constraint_weight = nullptr;   // lambda adjoint x C / D^2 of each particle (the lambda VJP's db)
    float4* gradient_sum_rest = nullptr;   // (S, rho0) of each particle, the lambda VJP's per-neighbour inputs
    float2* s_corr = nullptr;             // (W(s_corr radius), 1 when the strength is zero and the power stays finite)
    float4* reverse = nullptr;            // (rho0, s_corr strength, exponent, zero-strength flag): a neighbour's
                                          // reverse-term inputs in one load
};

void destroy_adjoint_workspace(void* workspace) { delete static_cast<AdjointWorkspace*>(workspace); }

namespace {

using namespace gather_detail;

// Caller-side FP64 outputs (original order); null pointers are skipped.
struct ParamAdjoint {
    double* masses;
    double* rest_densities;
    double* relaxation;
    double* strength;
    double* exponent;
    double* radius;
    double* xsph;
    double* vorticity;
};

// Per-pair quotients whose varying operand mostly repeats (uniform masses and rest densities): the
// last quotient is kept and reused while that operand's bits repeat.  The operands are then the
// same, so the correctly rounded quotient is the same.
struct DividendCache {   // x / divisor for varying x
    uint32_t key = 0xffffffffu;
    float value = 0.0F;
    __device__ __forceinline__ float operator()(const float x, const float divisor) {
        if (__float_as_uint(x) != key) {
            key = __float_as_uint(x);
            value = x / divisor;
        }
        return value;
    }
};
struct DivisorCache {    // dividend / y and 1 / y in FP64 for varying y
    uint32_t key = 0xffffffffu;
    float value = 0.0F;
    double reciprocal = 0.0;
    __device__ __forceinline__ void update(const float dividend, const float y) {
        if (__float_as_uint(y) != key) {
            key = __float_as_uint(y);
            value = dividend / y;
            reciprocal = 1.0 / static_cast<double>(y);
        }
    }
};

__device__ __forceinline__ void add_to(double* p, const uint32_t i, const double v) {
    if (p) p[i] += v;
}

__device__ __forceinline__ d3 cleared_plus(const d3 v) { return {0.0 + v.x, 0.0 + v.y, 0.0 + v.z}; }

__device__ __forceinline__ d3 masked(d3 a, const uint32_t mask) {
    if ((mask & 1u) != 0u) a.x = 0.0;
    if ((mask & 2u) != 0u) a.y = 0.0;
    if ((mask & 4u) != 0u) a.z = 0.0;
    return a;
}

__device__ __forceinline__ d3 normalized_input_adjoint(const f3 normal, const float normalizer, const d3 normal_adjoint) {
    if (normalizer == 0.0F) return {0.0, 0.0, 0.0};
    return times(normal_adjoint + times(normal, -dot(normal_adjoint, normal)), 1.0 / normalizer);
}

// Project VJP of one iteration (pbf.cu:444-454) into cleared buffers, or the predict VJP.
struct Tail {
    const uint8_t* mask;        // mask of the iteration being entered; null: predict VJP instead
    double4* next_position;     // position adjoint of that iteration (written 0 + masked)
    double4* correction;
    AdjField3 previous_position;
    AdjField3 previous_velocity;
    AdjField3 control;
};

__device__ __forceinline__ void finish(const Tail& t, const uint32_t s, const uint32_t i, const d3 x, const float dt) {
    if (t.mask) {
        const d3 a = masked(x, t.mask[s]);
        t.next_position[s] = st3(cleared_plus(a));
        t.correction[s] = st3(cleared_plus(a));
        return;
    }
    // predict VJP: x* = x + dt v + dt^2 (g + a)
    t.previous_position.x[i] += x.x;
    t.previous_position.y[i] += x.y;
    t.previous_position.z[i] += x.z;
    const d3 v = times(x, static_cast<double>(dt));
    t.previous_velocity.x[i] += v.x;
    t.previous_velocity.y[i] += v.y;
    t.previous_velocity.z[i] += v.z;
    const d3 c = times(x, static_cast<double>(dt * dt));
    t.control.x[i] += c.x;
    t.control.y[i] += c.y;
    t.control.z[i] += c.z;
}

// ----------------------------------------------------------------- seed
__global__ void seed_kernel(const GatherCommon g, const uint32_t* __restrict__ sorted_index, const ConstAdjField3 next_x,
                            const ConstAdjField3 next_v, double4* __restrict__ x, double4* __restrict__ out_v,
                            float2* __restrict__ s_corr, float4* __restrict__ reverse) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.count) return;
    const uint32_t i = sorted_index[s];
    x[s] = make_double4(next_x.x[i], next_x.y[i], next_x.z[i], 0.0);
    out_v[s] = make_double4(next_v.x[i], next_v.y[i], next_v.z[i], 0.0);
    // s_corr of this particle: the reference weight W(radius) and whether its strength is zero
    // with every power (W/W(radius))^exponent finite.  Then s_corr = -strength * power is a zero
    // whose sign is that of -strength, and its gradient and its exponent and radius derivatives
    // vanish; only the strength derivative -power remains (pbf/pbf.cu:56-71).
    const KernelConstants k = g.constants[g.scenes[g.cell[s].w].constants];
    const float4 pb = g.params_b[s];
    const float reference = poly6(mk(pb.z, 0.0F, 0.0F), k);
    bool zero_strength = pb.x == 0.0F && pb.y >= 0.0F && reference > 0.0F;
    if (zero_strength) {
        const float largest = powf(__fdiv_rn(poly6_inside(0.0F, k), reference), pb.y);
        zero_strength = largest < 1e30F;
    }
    s_corr[s] = make_float2(reference, zero_strength ? 1.0F : 0.0F);
    reverse[s] = make_float4(g.params_a[s].x, pb.x, pb.y, zero_strength ? 1.0F : 0.0F);
}

// ------------------------------------------------------- XSPH + confinement
struct XsphVjpArgs {
    GatherCommon g;
    StoredList list;
    const uint32_t* sorted_index;
    const float4* pos;
    const float4* confined;
    const float4* vorticity;
    const float4* normal;
    const double4* output_velocity;
    double4* x;
    double4* velocity;
    double4* vorticity_adjoint;
    double4* eta;
    ParamAdjoint pa;
};

struct XsphVjpOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ confined;
    const double4* __restrict__ output_velocity;
    const float4* __restrict__ params_a;
    f3 x, v;
    d3 ob;
    float viscosity;
    uint32_t self;
    KernelConstants k;
    d3 pc, vc;
    double cc;

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t == self) return;
        const f3 d = sub(x, xyz(pos[t]));
        if (squared(d) >= k.h2) return;
        const f3 vj = xyz(confined[t]);
        const f3 difference = vj - v;
        const float weight = poly6(d, k);
        const f3 gradient = poly6_gradient(d, k);
        vc = vc + times(ob, -viscosity * weight);
        pc = pc + times(gradient, viscosity * dot(ob, difference));
        cc += weight * dot(ob, difference);
        const d3 rob = ld3(output_velocity[t]);
        const f3 rdiff = v - vj;
        // W(-d) = W(d) and grad W(-d) = -grad W(d), exactly (the same squared distance; every
        // component is a product whose sign alone flips)
        const float rweight = weight;
        const float rviscosity = params_a[t].z;
        vc = vc + times(rob, rviscosity * rweight);
        pc = pc + times(scale(gradient, -1.0F), -rviscosity * dot(rob, rdiff));
    }
};

// Resident 128-thread blocks per SM the register budgets of the post-loop reverse passes and of
// the density VJP are sized for (compile-time tuning knobs; 0 leaves the register count to the
// compiler).  Measured (64k rollout / 32-scene batched rollout, grad-steps/s): the compiler's
// registers 721 / 35.2; a one-block minimum 724 / 34.6; the post-loop passes at 6 (80 registers)
// 721 / 35.3; the density VJP at 10 (48) 720 / 34.9.
#ifndef PBF_POST_VJP_MIN_BLOCKS
#define PBF_POST_VJP_MIN_BLOCKS 0
#endif
#ifndef PBF_DENSITY_VJP_MIN_BLOCKS
#define PBF_DENSITY_VJP_MIN_BLOCKS 0
#endif
__global__ void __launch_bounds__(kBlock, PBF_POST_VJP_MIN_BLOCKS) xsph_vjp_kernel(const XsphVjpArgs a) {
    uint32_t half;
    const Particle p = locate_pair(a.g, half);
    XsphVjpOp op;
    op.pos = a.pos;
    op.confined = a.confined;
    op.output_velocity = a.output_velocity;
    op.params_a = a.g.params_a;
    op.self = p.s;
    op.k = p.k;
    const float4 pa = p.active ? a.g.params_a[p.s] : make_float4(0, 0, 0, 0);
    op.x = p.active ? xyz(a.pos[p.s]) : mk(0, 0, 0);
    op.v = p.active ? xyz(a.confined[p.s]) : mk(0, 0, 0);
    op.ob = p.active ? ld3(a.output_velocity[p.s]) : d3{0, 0, 0};
    op.viscosity = pa.z;
    op.pc = {0.0, 0.0, 0.0};
    op.vc = {0.0, 0.0, 0.0};
    op.cc = 0.0;
    replay_pair(op, p, a.g, a.list, half);
    op.pc = pair_sum(op.pc);
    op.vc = op.ob + pair_sum(op.vc);
    op.cc = pair_sum(op.cc);
    if (!p.active || half) return;
    const uint32_t i = a.sorted_index[p.s];
    a.x[p.s] = st3(ld3(a.x[p.s]) + op.pc);
    add_to(a.pa.xsph, i, op.cc);
    // confinement VJP on the confined-velocity adjoint (a cleared buffer + the XSPH contribution)
    const d3 vcbar = cleared_plus(op.vc);
    const f3 vorticity = xyz(a.vorticity[p.s]);
    const float4 nrm = a.normal[p.s];
    const f3 normal = xyz(nrm);
    const float dt = p.scene->time_step;
    a.velocity[p.s] = st3(cleared_plus(vcbar));
    a.vorticity_adjoint[p.s] = st3(cleared_plus(times(cross(vcbar, normal), dt * pa.w)));
    const d3 normal_adjoint = cleared_plus(times(cross(vorticity, vcbar), dt * pa.w));
    add_to(a.pa.vorticity, i, dt * dot(vcbar, cross(normal, vorticity)));
    a.eta[p.s] = st3(normalized_input_adjoint(normal, nrm.w, normal_adjoint));
}

// ---------------------------------------------------------------- normal
struct NormalVjpArgs {
    GatherCommon g;
    StoredList list;
    const float4* pos;
    const float4* vorticity;
    const double4* eta;
    double4* x;
    double4* vorticity_adjoint;
};

struct NormalVjpOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ vorticity;
    const double4* __restrict__ eta;
    f3 x;
    float magnitude;
    d3 eb;
    uint32_t self;
    KernelConstants k;
    d3 pc;
    double mc;

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t == self) return;
        const f3 d = sub(x, xyz(pos[t]));
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.adjoint_threshold) return;
        const f3 gradient = spiky_gradient(d, k);
        const float magnitude_j = vorticity[t].w;
        const float difference = magnitude_j - magnitude;
        const f3 rg = scale(gradient, -1.0F);   // spiky_gradient(-d), exactly
        const d3 reb = ld3(eta[t]);
        const float rdiff = magnitude - magnitude_j;
        d3 hessian, reverse_hessian;   // H(d) applied to both sides' adjoints; H(-d) = H(d)
        spiky_hessian_products(d, times(eb, difference), times(reb, rdiff), k, hessian, reverse_hessian);
        pc = pc + hessian;
        mc -= dot(eb, gradient);
        pc = pc + times(reverse_hessian, -1.0);
        mc += dot(reb, rg);
    }
};

__global__ void __launch_bounds__(kBlock, PBF_POST_VJP_MIN_BLOCKS) normal_vjp_kernel(const NormalVjpArgs a) {
    uint32_t half;
    const Particle p = locate_pair(a.g, half);
    NormalVjpOp op;
    op.pos = a.pos;
    op.vorticity = a.vorticity;
    op.eta = a.eta;
    op.self = p.s;
    op.k = p.k;
    const float4 wi = p.active ? a.vorticity[p.s] : make_float4(0, 0, 0, 0);
    op.x = p.active ? xyz(a.pos[p.s]) : mk(0, 0, 0);
    op.magnitude = wi.w;
    op.eb = p.active ? ld3(a.eta[p.s]) : d3{0, 0, 0};
    op.pc = {0.0, 0.0, 0.0};
    op.mc = 0.0;
    replay_pair(op, p, a.g, a.list, half);
    op.pc = pair_sum(op.pc);
    op.mc = pair_sum(op.mc);
    if (!p.active || half) return;
    a.x[p.s] = st3(ld3(a.x[p.s]) + op.pc);
    if (wi.w > 0.0F) a.vorticity_adjoint[p.s] = st3(ld3(a.vorticity_adjoint[p.s]) + times(xyz(wi), op.mc / wi.w));
}

// ------------------------------------------------------------- vorticity
struct VorticityVjpArgs {
    GatherCommon g;
    StoredList list;
    const uint32_t* sorted_index;
    const float4* pos;
    const float4* velocity;
    const double4* vorticity_adjoint;
    double4* x;
    double4* velocity_adjoint;
    Tail tail;
};

struct VorticityVjpOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ velocity;
    const double4* __restrict__ vorticity_adjoint;
    f3 x, v;
    d3 wb;
    uint32_t self;
    KernelConstants k;
    d3 pc, vc;

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t == self) return;
        const f3 d = sub(x, xyz(pos[t]));
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.adjoint_threshold) return;
        const f3 gradient = spiky_gradient(d, k);
        const f3 vj = xyz(velocity[t]);
        const f3 difference = vj - v;
        const d3 rwb = ld3(vorticity_adjoint[t]);
        const f3 rg = scale(gradient, -1.0F);   // spiky_gradient(-d), exactly
        const f3 rdiff = v - vj;
        d3 hessian, reverse_hessian;   // H(d) applied to both sides' adjoints; H(-d) = H(d)
        spiky_hessian_products(d, cross(wb, difference), cross(rwb, rdiff), k, hessian, reverse_hessian);
        vc = vc + cross(wb, gradient);
        pc = pc + hessian;
        vc = vc + cross(rg, rwb);
        pc = pc + times(reverse_hessian, -1.0);
    }
};

__global__ void __launch_bounds__(kBlock, PBF_POST_VJP_MIN_BLOCKS) vorticity_vjp_kernel(const VorticityVjpArgs a) {
    uint32_t half;
    const Particle p = locate_pair(a.g, half);
    VorticityVjpOp op;
    op.pos = a.pos;
    op.velocity = a.velocity;
    op.vorticity_adjoint = a.vorticity_adjoint;
    op.self = p.s;
    op.k = p.k;
    op.x = p.active ? xyz(a.pos[p.s]) : mk(0, 0, 0);
    op.v = p.active ? xyz(a.velocity[p.s]) : mk(0, 0, 0);
    op.wb = p.active ? ld3(a.vorticity_adjoint[p.s]) : d3{0, 0, 0};
    op.pc = {0.0, 0.0, 0.0};
    op.vc = {0.0, 0.0, 0.0};
    replay_pair(op, p, a.g, a.list, half);
    op.pc = pair_sum(op.pc);
    op.vc = pair_sum(op.vc);
    if (!p.active || half) return;
    const uint32_t i = a.sorted_index[p.s];
    d3 xb = ld3(a.x[p.s]) + op.pc;
    const d3 vr = ld3(a.velocity_adjoint[p.s]) + op.vc;
    // reconstruct VJP: v = (x_c - x) / dt
    const d3 contribution = times(vr, static_cast<double>(p.scene->inverse_time_step));
    const d3 back = times(contribution, -1.0);
    a.tail.previous_position.x[i] += back.x;
    a.tail.previous_position.y[i] += back.y;
    a.tail.previous_position.z[i] += back.z;
    xb = xb + contribution;
    finish(a.tail, p.s, i, xb, p.scene->time_step);
}

// s_corr of a pair whose particle has zero strength (its s_corr table entry is 1): the value is a
// zero with the sign of -strength (or +0 outside the poly6 support, as the reference's early
// return), and only the strength derivative -power is non-zero; `weight` is W(d) = W(-d).
__device__ __forceinline__ ArtificialPressure zero_strength_pressure(const float weight, const float reference,
                                                                     const float strength, const float exponent,
                                                                     const bool with_derivative) {
    ArtificialPressure a;
    a.d_exponent = a.d_radius = 0.0F;
    a.gradient = {0.0F, 0.0F, 0.0F};
    a.value = a.d_strength = 0.0F;
    if (weight == 0.0F) return a;
    if (with_derivative) {
        const float power = powf(__fdiv_rn(weight, reference), exponent);
        a.value = __fmul_rn(-strength, power);
        a.d_strength = -power;
    } else {
        a.value = -strength;   // -strength * power for a finite power >= 0
    }
    return a;
}

// ------------------------------------------------------------ correction
struct CorrectionVjpArgs {
    GatherCommon g;
    StoredList list;
    const uint32_t* sorted_index;
    const float4* pos;
    const float2* s_corr;
    const float4* reverse;
    const float* lambda;
    const double4* correction;
    double4* x;
    double* lambda_adjoint;
    ParamAdjoint pa;
    // For each particle the correction VJP also writes lambda_adjoint * (rho / rho0 - 1) / D^2, the
    // factor the lambda VJP (pbf.cu:180-200) applies to the particle's own gradient terms and, for
    // every neighbour, to that neighbour's: evaluated once per particle instead of once per pair.
    const float* density;
    const float4* gsum;          // (S, D)
    double* constraint_weight;
    float4* gradient_sum_rest;   // (S, rho0): the lambda VJP reads a neighbour's in one load
};

struct CorrectionVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    float reference_i;
    bool zero_strength_i;
    const float* __restrict__ lambda;
    const double4* __restrict__ correction;
    const float4* __restrict__ params_b;
    const float4* __restrict__ reverse;
    f3 x;
    float mass, rest_density, lambda_i, strength, exponent, radius;
    d3 ob;
    uint32_t self;
    KernelConstants k;
    d3 pc;
    double lc, mc, rc, sc, ec, qc;
    DividendCache own_ratio;      // m_j / rho0_i
    DivisorCache reverse_ratio;   // m_i / rho0_j

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t == self) return;
        if (t & kBoundaryBit) {
            boundary_term(boundary[t & ~kBoundaryBit]);
            return;
        }
        const float4 q = pos[t];
        const f3 d = sub(x, xyz(q));
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.adjoint_threshold) return;
        const f3 gradient = spiky_gradient(d, k);
        const f3 rg = scale(gradient, -1.0F);   // spiky_gradient(-d), exactly
        const float weight = r2 >= k.h2 ? 0.0F : poly6_inside(r2, k);   // W(d) = W(-d)
        const ArtificialPressure ap = zero_strength_i ? zero_strength_pressure(weight, reference_i, strength, exponent, true)
                                                      : artificial_pressure(d, k, strength, exponent, radius);
        const float4 rv = reverse[t];   // (rho0_j, strength_j, exponent_j, zero-strength flag)
        const ArtificialPressure rap = rv.w != 0.0F ? zero_strength_pressure(weight, 1.0F, rv.y, rv.z, false)
                                                    : artificial_pressure(scale(d, -1.0F), k, rv.y, rv.z, params_b[t].z);
        const float coefficient = own_ratio(q.w, rest_density);
        const float lambda_j = lambda[t];
        const float multiplier = lambda_i + lambda_j + ap.value;
        const double scalar_adjoint = coefficient * dot(ob, gradient);
        const float rrest = rv.x;
        reverse_ratio.update(mass, rrest);
        const float rcoefficient = reverse_ratio.value;
        const float rmultiplier = lambda_j + lambda_i + rap.value;
        const d3 rob = ld3(correction[t]);
        const double rscalar = rcoefficient * dot(rob, rg);
        d3 hessian, reverse_hessian;   // H(d) applied to both sides' adjoints; H(-d) = H(d)
        spiky_hessian_products(d, times(ob, coefficient * multiplier), times(rob, rcoefficient * rmultiplier), k, hessian,
                               reverse_hessian);
        pc = pc + hessian;
        pc = pc + times(ap.gradient, scalar_adjoint);
        lc += scalar_adjoint;
        rc += dot(ob, times(gradient, coefficient * multiplier));   // divided by -rho0_i once, at the end
        sc += scalar_adjoint * ap.d_strength;
        ec += scalar_adjoint * ap.d_exponent;
        qc += scalar_adjoint * ap.d_radius;
        pc = pc + times(reverse_hessian, -1.0);
        pc = pc + times(rap.gradient, -rscalar);
        lc += rscalar;
        mc += dot(rob, times(rg, rmultiplier / rrest));
    }
    // boundary particle (position at the step's time, volume): pbf.cu:390-405
    __device__ __forceinline__ void boundary_term(const float4 q) {
        const f3 d = sub(x, xyz(q));
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.adjoint_threshold) return;
        const f3 gradient = spiky_gradient(d, k);
        const ArtificialPressure ap = artificial_pressure(d, k, strength, exponent, radius);
        const float volume = q.w;
        const float multiplier = lambda_i + ap.value;
        const double scalar_adjoint = volume * dot(ob, gradient);
        pc = pc + spiky_hessian_product(d, times(ob, volume * multiplier), k);
        pc = pc + times(ap.gradient, scalar_adjoint);
        lc += scalar_adjoint;
        sc += scalar_adjoint * ap.d_strength;
        ec += scalar_adjoint * ap.d_exponent;
        qc += scalar_adjoint * ap.d_radius;
    }
};

// Four resident blocks per SM (at most 128 registers) hide more latency than the unbounded 144.
// 5 blocks per SM (96 registers, 616 bytes of spills) took the 64k rollout from 720 to 644 grad-steps/s.
#ifndef PBF_CORRECTION_VJP_MIN_BLOCKS
#define PBF_CORRECTION_VJP_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kBlock, PBF_CORRECTION_VJP_MIN_BLOCKS) correction_vjp_kernel(const CorrectionVjpArgs a) {
    uint32_t half;
    const Particle p = locate_pair(a.g, half);
    CorrectionVjpOp op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    const float2 si = p.active ? a.s_corr[p.s] : make_float2(1.0F, 0.0F);
    op.reference_i = si.x;
    op.zero_strength_i = si.y != 0.0F;
    op.lambda = a.lambda;
    op.correction = a.correction;
    op.params_b = a.g.params_b;
    op.reverse = a.reverse;
    op.self = p.s;
    op.k = p.k;
    const float4 xi = p.active ? a.pos[p.s] : make_float4(0, 0, 0, 0);
    const float4 pa = p.active ? a.g.params_a[p.s] : make_float4(1, 0, 0, 0);
    const float4 pb = p.active ? a.g.params_b[p.s] : make_float4(0, 0, 0, 0);
    op.x = xyz(xi);
    op.mass = xi.w;
    op.rest_density = pa.x;
    op.lambda_i = p.active ? a.lambda[p.s] : 0.0F;
    op.strength = pb.x;
    op.exponent = pb.y;
    op.radius = pb.z;
    op.ob = p.active ? ld3(a.correction[p.s]) : d3{0, 0, 0};
    op.pc = {0.0, 0.0, 0.0};
    op.lc = op.mc = op.rc = op.sc = op.ec = op.qc = 0.0;
    replay_pair(op, p, a.g, a.list, half);
    op.pc = pair_sum(op.pc);
    op.lc = pair_sum(op.lc);
    op.mc = pair_sum(op.mc);
    op.rc = pair_sum(op.rc);
    op.sc = pair_sum(op.sc);
    op.ec = pair_sum(op.ec);
    op.qc = pair_sum(op.qc);
    if (!p.active || half) return;
    const uint32_t i = a.sorted_index[p.s];
    a.x[p.s] = st3(ld3(a.x[p.s]) + op.pc);
    const double lb = 0.0 + op.lc;
    a.lambda_adjoint[p.s] = lb;
    const double constraint = static_cast<double>(a.density[p.s]) / pa.x - 1.0;
    const float4 gsum = a.gsum[p.s];
    const float denominator = gsum.w;
    a.constraint_weight[p.s] = lb * constraint / (static_cast<double>(denominator) * denominator);
    a.gradient_sum_rest[p.s] = make_float4(gsum.x, gsum.y, gsum.z, pa.x);
    add_to(a.pa.masses, i, op.mc);
    add_to(a.pa.rest_densities, i, -op.rc / pa.x);
    add_to(a.pa.strength, i, op.sc);
    add_to(a.pa.exponent, i, op.ec);
    add_to(a.pa.radius, i, op.qc);
}

// ---------------------------------------------------------------- lambda
struct LambdaVjpArgs {
    GatherCommon g;
    StoredList list;
    const uint32_t* sorted_index;
    const float4* pos;
    const float* density;
    const float4* gsum;          // (S, D)
    const double* lambda_adjoint;
    const double* constraint_weight;
    const float4* gradient_sum_rest;
    double4* x;
    double* density_adjoint;
    ParamAdjoint pa;
};

struct LambdaVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    const float* __restrict__ density;
    const float4* __restrict__ gradient_sum_rest;
    const double* __restrict__ constraint_weight;
    f3 x;
    float mass, rest_density;
    double db;
    d3 sb;
    uint32_t self;
    KernelConstants k;
    d3 pc;
    double mc;
    double rc_pairs;   // the second neighbour loop's terms (pbf.cu:233-246), summed in this loop
    f3 self_gradient;
    DividendCache own_ratio;      // m_j / rho0_i
    DivisorCache reverse_ratio;   // m_i / rho0_j and 1 / rho0_j

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t == self) return;
        if (t & kBoundaryBit) {
            // boundary particle: Hessian of V_b W applied to the self-gradient adjoint (pbf.cu:226-230)
            const float4 q = boundary[t & ~kBoundaryBit];
            const f3 d = sub(x, xyz(q));
            const float r2 = squared(d);
            if (r2 == 0.0F || r2 >= k.adjoint_threshold) return;
            pc = pc + spiky_hessian_product(d, times(sb, static_cast<double>(q.w)), k);
            return;
        }
        const float4 q = pos[t];
        const f3 d = sub(x, xyz(q));
        const float r2 = squared(d);
        if (r2 == 0.0F || r2 >= k.adjoint_threshold) return;
        const f3 gradient = spiky_gradient(d, k);
        const float coefficient = own_ratio(q.w, rest_density);
        const f3 neighbor_gradient = times(gradient, -coefficient);
        const d3 neighbor_gradient_adjoint = times(neighbor_gradient, 2.0 * db);
        const d3 gradient_adjoint = times(sb - neighbor_gradient_adjoint, coefficient);
        self_gradient = fma3(coefficient, gradient, self_gradient);
        rc_pairs += dot(neighbor_gradient_adjoint, neighbor_gradient);   // divided by -rho0_i once, at the end
        const float4 gj = gradient_sum_rest[t];   // (S_j, rho0_j)
        const float rrest = gj.w;
        const double rdb = constraint_weight[t];   // the neighbour's db, as its own lambda VJP forms it
        const d3 rsb = times(xyz(gj), 2.0 * rdb);
        const f3 rg = scale(gradient, -1.0F);   // spiky_gradient(-d), exactly
        reverse_ratio.update(mass, rrest);
        const float rcoefficient = reverse_ratio.value;
        const f3 rneighbor_gradient = times(rg, -rcoefficient);
        const d3 rneighbor_gradient_adjoint = times(rneighbor_gradient, 2.0 * rdb);
        const d3 rgradient_adjoint = times(rsb - rneighbor_gradient_adjoint, rcoefficient);
        d3 hessian, reverse_hessian;   // H(d) applied to both sides' adjoints; H(-d) = H(d)
        spiky_hessian_products(d, gradient_adjoint, rgradient_adjoint, k, hessian, reverse_hessian);
        pc = pc + hessian;
        pc = pc + times(reverse_hessian, -1.0);
        mc += dot(rsb - rneighbor_gradient_adjoint, rg) * reverse_ratio.reciprocal;
    }
};

#ifndef PBF_LAMBDA_VJP_MIN_BLOCKS
#define PBF_LAMBDA_VJP_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kBlock, PBF_LAMBDA_VJP_MIN_BLOCKS) lambda_vjp_kernel(const LambdaVjpArgs a) {
    const Particle p = locate(a.g);
    LambdaVjpOp op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    op.density = a.density;
    op.gradient_sum_rest = a.gradient_sum_rest;
    op.constraint_weight = a.constraint_weight;
    op.self = p.s;
    op.k = p.k;
    const float4 xi = p.active ? a.pos[p.s] : make_float4(0, 0, 0, 0);
    const float4 pa = p.active ? a.g.params_a[p.s] : make_float4(1, 0, 0, 0);
    const float4 gi = p.active ? a.gsum[p.s] : make_float4(0, 0, 0, 1);
    const float rho = p.active ? a.density[p.s] : 0.0F;
    const double lb = p.active ? a.lambda_adjoint[p.s] : 0.0;
    op.x = xyz(xi);
    op.mass = xi.w;
    op.rest_density = pa.x;
    op.db = p.active ? a.constraint_weight[p.s] : 0.0;   // lb (rho / rho0 - 1) / D^2
    op.sb = times(xyz(gi), 2.0 * op.db);
    op.pc = {0.0, 0.0, 0.0};
    op.mc = 0.0;
    op.rc_pairs = 0.0;
    op.self_gradient = mk(0.0F, 0.0F, 0.0F);
    replay(op, p, a.g, a.list);
    // The reference sums the rest-density adjoint in a second neighbour loop after the first
    // (pbf.cu:233-246); its per-pair terms need nothing the first loop lacks, so they are summed
    // there and added here (FP64 rounding of a different summation order).
    double rc = lb * rho / (static_cast<double>(gi.w) * pa.x * pa.x);
    rc -= dot(op.sb, op.self_gradient) / pa.x;
    rc += -op.rc_pairs / pa.x;
    if (!p.active) return;
    const uint32_t i = a.sorted_index[p.s];
    a.x[p.s] = st3(ld3(a.x[p.s]) + op.pc);
    a.density_adjoint[p.s] = 0.0 - lb / (static_cast<double>(gi.w) * pa.x);
    add_to(a.pa.masses, i, op.mc);
    add_to(a.pa.rest_densities, i, rc);
    add_to(a.pa.relaxation, i, op.db);
}

// --------------------------------------------------------------- density
struct DensityVjpArgs {
    GatherCommon g;
    StoredList list;
    const uint32_t* sorted_index;
    const float4* pos;
    const double* density_adjoint;
    double4* x;
    ParamAdjoint pa;
    Tail tail;
};

struct DensityVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    const double* __restrict__ density_adjoint;
    f3 x;
    float mass, rest_density;
    double ob;
    KernelConstants k;
    d3 pc;
    double mc, rc;

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t & kBoundaryBit) {
            // boundary particle: rho0_i V_b W (density/density.cu:93-98)
            const float4 q = boundary[t & ~kBoundaryBit];
            const f3 d = sub(x, xyz(q));
            if (squared(d) >= k.h2) return;
            const float volume = q.w;
            pc = pc + times(poly6_gradient(d, k), ob * rest_density * volume);
            rc += ob * volume * poly6(d, k);
            return;
        }
        const float4 q = pos[t];
        const f3 d = sub(x, xyz(q));
        if (squared(d) >= k.h2) return;
        const f3 gradient = poly6_gradient(d, k);
        const double rb = density_adjoint[t];
        pc = pc + times(gradient, ob * q.w + rb * mass);
        mc += rb * poly6(d, k);
    }
};

__global__ void __launch_bounds__(kBlock, PBF_DENSITY_VJP_MIN_BLOCKS) density_vjp_kernel(const DensityVjpArgs a) {
    uint32_t half;
    const Particle p = locate_pair(a.g, half);
    DensityVjpOp op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    op.density_adjoint = a.density_adjoint;
    op.k = p.k;
    const float4 xi = p.active ? a.pos[p.s] : make_float4(0, 0, 0, 0);
    op.x = xyz(xi);
    op.mass = xi.w;
    op.rest_density = p.active ? a.g.params_a[p.s].x : 1.0F;
    op.ob = p.active ? a.density_adjoint[p.s] : 0.0;
    op.pc = {0.0, 0.0, 0.0};
    op.mc = 0.0;
    op.rc = 0.0;
    replay_pair(op, p, a.g, a.list, half);
    op.pc = pair_sum(op.pc);
    op.mc = pair_sum(op.mc);
    op.rc = pair_sum(op.rc);
    if (!p.active || half) return;
    const uint32_t i = a.sorted_index[p.s];
    const d3 xb = ld3(a.x[p.s]) + op.pc;
    add_to(a.pa.masses, i, op.mc);
    add_to(a.pa.rest_densities, i, op.rc);
    finish(a.tail, p.s, i, xb, p.scene->time_step);
}

inline unsigned grid_of(const uint32_t n, const unsigned block) { return (n + block - 1) / block; }

__global__ void accumulate6_kernel(const size_t count, const ConstAdjField3 s0, const ConstAdjField3 s1, const AdjField3 d0,
                                   const AdjField3 d1, const int fields) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double* src[6] = {s0.x, s0.y, s0.z, s1.x, s1.y, s1.z};
    double* dst[6] = {d0.x, d0.y, d0.z, d1.x, d1.y, d1.z};
    for (int f = 0; f < fields; ++f) dst[f][i] += src[f][i];
}

// Neumaier-compensated FP64 summation with a fixed reduction tree (deterministic for a given
// launch shape): one block per segment [first, first + count).
struct Compensated {
    double sum, carry;
};

__device__ __forceinline__ Compensated add_value(Compensated a, const double v) {
    const double t = a.sum + v;
    if (fabs(a.sum) >= fabs(v)) a.carry += (a.sum - t) + v;
    else a.carry += (v - t) + a.sum;
    a.sum = t;
    return a;
}

__device__ __forceinline__ Compensated combine(Compensated a, const Compensated b) {
    a = add_value(a, b.sum);
    a.carry += b.carry;
    return a;
}

__global__ void segment_sum_kernel(const double* __restrict__ values, const uint32_t* __restrict__ first,
                                   const uint32_t* __restrict__ count, const uint32_t single_count, double* __restrict__ out) {
    __shared__ double sums[256];
    __shared__ double carries[256];
    const uint32_t seg = blockIdx.x;
    const uint32_t begin = first ? first[seg] : 0u;
    const uint32_t n = count ? count[seg] : single_count;
    Compensated c{0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) c = add_value(c, values[begin + i]);
    sums[threadIdx.x] = c.sum;
    carries[threadIdx.x] = c.carry;
    __syncthreads();
    for (uint32_t stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            const Compensated r = combine({sums[threadIdx.x], carries[threadIdx.x]},
                                          {sums[threadIdx.x + stride], carries[threadIdx.x + stride]});
            sums[threadIdx.x] = r.sum;
            carries[threadIdx.x] = r.carry;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[seg] = sums[0] + carries[0];
}

}  // namespace

cudaError_t launch_segment_sums(cudaStream_t stream, const double* values, const uint32_t* first, const uint32_t* count,
                                const uint32_t segments, const uint32_t single_count, double* out) {
    if (segments == 0) return cudaSuccess;
    segment_sum_kernel<<<segments, 256, 0, stream>>>(values, first, count, single_count, out);
    count_launch();
    return cudaGetLastError();
}

// domain/domain.cu:8-29: FP64 dst += src over up to six fields.
cudaError_t launch_accumulate(cudaStream_t stream, const size_t count, const double* const* src, double* const* dst,
                              const int fields) {
    if (count == 0) return cudaSuccess;
    const ConstAdjField3 s0{src[0], fields > 1 ? src[1] : nullptr, fields > 2 ? src[2] : nullptr};
    const ConstAdjField3 s1{fields > 3 ? src[3] : nullptr, fields > 4 ? src[4] : nullptr, fields > 5 ? src[5] : nullptr};
    const AdjField3 d0{dst[0], fields > 1 ? dst[1] : nullptr, fields > 2 ? dst[2] : nullptr};
    const AdjField3 d1{fields > 3 ? dst[3] : nullptr, fields > 4 ? dst[4] : nullptr, fields > 5 ? dst[5] : nullptr};
    accumulate6_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(count, s0, s1, d0, d1,
                                                                                     fields < 6 ? fields : 6);
    count_launch();
    return cudaGetLastError();
}

static bool has3(const pbf_vector_adjoint_field& f) { return f.x && f.y && f.z; }

int Engine::reverse(const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                    const StepRecord& r, const pbf_particle_state_adjoint* next_adjoint,
                    pbf_particle_state_adjoint* previous_adjoint, pbf_control_adjoint* control_adjoint,
                    pbf_parameter_adjoint* parameter_adjoint) {
    (void)control;
    (void)parameters;
    if (!differentiable()) {
        set_error("vjp_step needs PBF_EXECUTION_DIFFERENTIABLE");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    if (!state || !next_adjoint || !previous_adjoint || !control_adjoint) {
        set_error("null argument");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!r.valid || r.step_index != state->step_index) {
        set_error("the step cache does not hold the forward step of this state");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    const uint32_t n = count_, K = iterations_;
    if (n == 0) return PBF_SUCCESS;
    if (!has3(next_adjoint->positions) || !has3(next_adjoint->velocities) || !has3(previous_adjoint->positions) ||
        !has3(previous_adjoint->velocities) || !has3(control_adjoint->external_accelerations)) {
        set_error("null adjoint field");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    auto* ws = static_cast<AdjointWorkspace*>(adjoint_);
    if (!ws) {
        ws = new AdjointWorkspace();
        ws->arena.set_stream(stream_);
        cudaError_t e = cudaSuccess;
        ws->x[0] = ws->arena.alloc<double4>(n, e);
        ws->x[1] = ws->arena.alloc<double4>(n, e);
        ws->correction = ws->arena.alloc<double4>(n, e);
        ws->output_velocity = ws->arena.alloc<double4>(n, e);
        ws->vorticity = ws->arena.alloc<double4>(n, e);
        ws->velocity = ws->arena.alloc<double4>(n, e);
        ws->eta = ws->arena.alloc<double4>(n, e);
        ws->lambda = ws->arena.alloc<double>(n, e);
        ws->density = ws->arena.alloc<double>(n, e);
        ws->constraint_weight = ws->arena.alloc<double>(n, e);
        ws->gradient_sum_rest = ws->arena.alloc<float4>(n, e);
        ws->s_corr = ws->arena.alloc<float2>(n, e);
        ws->reverse = ws->arena.alloc<float4>(n, e);
        if (e != cudaSuccess) {
            delete ws;
            return check(e, "adjoint workspace");
        }
        adjoint_ = ws;
    }
    ParamAdjoint pa{};
    if (parameter_adjoint) {
        pa = {parameter_adjoint->masses, parameter_adjoint->rest_densities, parameter_adjoint->relaxation,
              parameter_adjoint->artificial_pressure_strength, parameter_adjoint->artificial_pressure_exponent,
              parameter_adjoint->artificial_pressure_radius, parameter_adjoint->xsph_viscosity,
              parameter_adjoint->vorticity_confinement};
    }
    const GatherCommon gc = gather_common(r);
    // Passes that replay the same list run in alternating block orders, each starting on the entries
    // the previous pass read last (still in L2).
    GatherCommon gc_reverse = gc;
    gc_reverse.reverse = 1;
    const AdjField3 prev_x{previous_adjoint->positions.x, previous_adjoint->positions.y, previous_adjoint->positions.z};
    const AdjField3 prev_v{previous_adjoint->velocities.x, previous_adjoint->velocities.y, previous_adjoint->velocities.z};
    const AdjField3 ctrl{control_adjoint->external_accelerations.x, control_adjoint->external_accelerations.y,
                         control_adjoint->external_accelerations.z};
    const float4* xK = r.iterate(K, K, true);
    const unsigned blocks = grid_of(n, kBlock);
    const unsigned pair_blocks = grid_of(2u * n, kBlock);   // the passes with two lanes per particle
    const bool keep = r.keeps_all(true);
    // A checkpoint-recompute record keeps one list: the post-loop list.
    const StoredList post_list{r.list_entries[keep ? K : 0u], r.list_counts[keep ? K : 0u], r.list_capacity};

    timer_.begin(stream_, kPassSeed);
    seed_kernel<<<grid_of(n, 256), 256, 0, stream_>>>(
        gc, r.sorted_index, {next_adjoint->positions.x, next_adjoint->positions.y, next_adjoint->positions.z},
        {next_adjoint->velocities.x, next_adjoint->velocities.y, next_adjoint->velocities.z}, ws->x[0], ws->output_velocity,
        ws->s_corr, ws->reverse);
    timer_.end(stream_, kPassSeed);
    XsphVjpArgs xa{gc, post_list, r.sorted_index, xK, r.confined, r.vorticity, r.normal, ws->output_velocity, ws->x[0], ws->velocity,
                   ws->vorticity, ws->eta, pa};
    timer_.begin(stream_, kPassXsphVjp);
    xsph_vjp_kernel<<<pair_blocks, kBlock, 0, stream_>>>(xa);
    timer_.end(stream_, kPassXsphVjp);
    NormalVjpArgs na{gc_reverse, post_list, xK, r.vorticity, ws->eta, ws->x[0], ws->vorticity};
    timer_.begin(stream_, kPassNormalVjp);
    normal_vjp_kernel<<<pair_blocks, kBlock, 0, stream_>>>(na);
    timer_.end(stream_, kPassNormalVjp);
    Tail tail{K ? r.mask[K - 1] : nullptr, ws->x[1], ws->correction, prev_x, prev_v, ctrl};
    VorticityVjpArgs va{gc, post_list, r.sorted_index, xK, r.velocity, ws->vorticity, ws->x[0], ws->velocity, tail};
    timer_.begin(stream_, kPassVorticityVjp);
    vorticity_vjp_kernel<<<pair_blocks, kBlock, 0, stream_>>>(va);
    timer_.end(stream_, kPassVorticityVjp);
    count_launch(4);
    // Checkpoint recomputation (pbf/pbf.cpp:232-245): before the iterations of a segment between two
    // kept iterates are reversed, its lists and per-iteration fields are recomputed from the first.
    uint32_t segment_first = 0;
    for (uint32_t k = K; k-- > 0;) {
        double4* acc = ws->x[(K - k) & 1u];
        double4* other = ws->x[(K - k + 1) & 1u];
        const float4* xk;
        StoredList it_list;
        const float* lambda_k;
        const float* density_k;
        const float4* gsum_k;
        if (keep) {
            xk = r.iterate(k, K, true);
            it_list = StoredList{r.list_entries[k], r.list_counts[k], r.list_capacity};
            lambda_k = r.lambda[k];
            density_k = r.density[k];
            gsum_k = r.gsum[k];
        } else {
            if (k + 1 == K || r.is_checkpoint(k + 1, K)) {   // the last iteration of a segment: recompute it
                segment_first = k / r.checkpoint_interval * r.checkpoint_interval;
                if (int rc = recompute_segment(r, segment_first, k + 1 - segment_first)) return rc;
            }
            const uint32_t j = k - segment_first;
            xk = segment_iterate(r, segment_first, j);
            it_list = StoredList{segment_->list_entries[j], segment_->list_counts[j], kListCapacity};
            lambda_k = segment_->lambda[j];
            density_k = segment_->density[j];
            gsum_k = segment_->gsum[j];
        }
        CorrectionVjpArgs ca{gc, it_list, r.sorted_index, xk, ws->s_corr, ws->reverse, lambda_k, ws->correction, acc,
                             ws->lambda, pa, density_k, gsum_k, ws->constraint_weight, ws->gradient_sum_rest};
        timer_.begin(stream_, kPassCorrectionVjp);
        correction_vjp_kernel<<<pair_blocks, kBlock, 0, stream_>>>(ca);
        timer_.end(stream_, kPassCorrectionVjp);
        LambdaVjpArgs la{gc_reverse, it_list, r.sorted_index, xk, density_k, gsum_k, ws->lambda, ws->constraint_weight,
                         ws->gradient_sum_rest, acc, ws->density, pa};
        timer_.begin(stream_, kPassLambdaVjp);
        lambda_vjp_kernel<<<blocks, kBlock, 0, stream_>>>(la);
        timer_.end(stream_, kPassLambdaVjp);
        Tail t{k ? r.mask[k - 1] : nullptr, other, ws->correction, prev_x, prev_v, ctrl};
        DensityVjpArgs da{gc, it_list, r.sorted_index, xk, ws->density, acc, pa, t};
        timer_.begin(stream_, kPassDensityVjp);
        density_vjp_kernel<<<pair_blocks, kBlock, 0, stream_>>>(da);
        timer_.end(stream_, kPassDensityVjp);
        count_launch(3);
    }
    return check(cudaGetLastError(), "vjp_step");
}

}  // namespace pbf
