// Reverse (FP64) and tangent (FP32) passes of the SPH substep: SPH<Method>::vjp_step and
// ::jvp_step (sph/sph.ixx:356-365) for WCSPH, PCISPH, IISPH and DFSPH.
//
// Every reverse pass is a pull formulation like the reference's (sph/common.cu:98-163, 239-300,
// sph/wcsph.cu:242-304, 389-436, density/density.cu:68-99): particle i gathers its own terms and the
// cross terms of the pairs (j, i) from its neighbours' adjoints, so nothing is scattered and no
// atomics are needed.  Pairs are visited in the forward's stencil order over the same stored lists
// (or the stencil walk where the forward walked), with the reference's per-pair expressions and its
// FP32 / FP64 type mix: the kernel values and gradients are FP32 with the forward passes' rounding,
// products with adjoints FP64.  Candidates beyond the support contribute exact zeros there.
//
// Launch sequences (sph_engine.cu):
//   WCSPH   integrate (sph/common.cu:344-366) -> forces (surface + viscosity + pressure + EOS)
//           -> density
//   PCISPH / IISPH / DFSPH
//           final prediction -> per iteration, newest first: pressure + pressure update, then
//           predicted density + the prediction that produced it -> non-pressure -> density
#include "sph_math.cuh"

// Resident 128-thread blocks per SM the register budgets of the reverse and tangent list-replay
// passes are sized for (compile-time tuning knobs; 0 leaves the register count to the compiler).
// At 1M particles, ms per tangent step WCSPH / PCISPH / DFSPH on one box: the compiler's registers
// 2.35 / 8.91 / 15.36; these budgets 1.89 / 7.75 / 13.20.  Gradient steps: 3.28 / 10.74 / 17.81
// against 3.01 / 10.63 / 17.62 (the WCSPH force VJP at 168 registers instead of 220).  Measured
// and not kept: the pressure and non-pressure VJPs at 96 registers (spilling; PCISPH gradient
// 10.63 -> 11.02), the density VJP at 48 (0.4 % slower), the density tangents at 14 (32; slower
// than at 12).
#ifndef PBF_SPH_DENSITY_VJP_MIN_BLOCKS
#define PBF_SPH_DENSITY_VJP_MIN_BLOCKS 0
#endif
#ifndef PBF_SPH_DENSITY_JVP_MIN_BLOCKS
#define PBF_SPH_DENSITY_JVP_MIN_BLOCKS 12
#endif
#ifndef PBF_SPH_PRESSURE_JVP_MIN_BLOCKS
#define PBF_SPH_PRESSURE_JVP_MIN_BLOCKS 8
#endif
#ifndef PBF_WCSPH_FORCE_VJP_MIN_BLOCKS
#define PBF_WCSPH_FORCE_VJP_MIN_BLOCKS 3
#endif
#ifndef PBF_WCSPH_FORCE_JVP_MIN_BLOCKS
#define PBF_WCSPH_FORCE_JVP_MIN_BLOCKS 6
#endif
#ifndef PBF_SPH_PRESSURE_VJP_MIN_BLOCKS
#define PBF_SPH_PRESSURE_VJP_MIN_BLOCKS 0
#endif
#ifndef PBF_SPH_NON_PRESSURE_VJP_MIN_BLOCKS
#define PBF_SPH_NON_PRESSURE_VJP_MIN_BLOCKS 0
#endif
#ifndef PBF_SPH_NON_PRESSURE_JVP_MIN_BLOCKS
#define PBF_SPH_NON_PRESSURE_JVP_MIN_BLOCKS 8
#endif

namespace pbf {
namespace sph {

namespace {

using namespace gather_detail;
using namespace detail;

__device__ __forceinline__ void add_to(double* p, const uint32_t i, const double v) {
    if (p) p[i] += v;
}
__device__ __forceinline__ void add_to(const AdjField3 f, const uint32_t i, const d3 v) {
    f.x[i] += v.x;
    f.y[i] += v.y;
    f.z[i] += v.z;
}
__device__ __forceinline__ d3 ld(const double4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ double4 st4(const d3 v) { return make_double4(v.x, v.y, v.z, 0.0); }
__device__ __forceinline__ d3 neg(const d3 v) { return {-v.x, -v.y, -v.z}; }
__device__ __forceinline__ f3 negf(const f3 v) { return {-1.0F * v.x, -1.0F * v.y, -1.0F * v.z}; }

// --------------------------------------------------------------- per-pair reverse terms
// viscosity_reverse (sph/wcsph.cu:37-66): the adjoint of one Monaghan viscosity term.
struct ViscosityTerms {
    d3 displacement, velocity_difference;
    double neighbor_mass, first_density, second_density, first_viscosity, second_viscosity, first_speed, second_speed;
};

__device__ __forceinline__ ViscosityTerms viscosity_reverse(const f3 d, const f3 vd, const float first_density,
                                                          const float second_density, const float first_viscosity,
                                                          const float second_viscosity, const float first_speed,
                                                          const float second_speed, const float neighbor_mass,
                                                          const SphConstants& k, const d3 adjoint, const CubicHessian& H) {
    ViscosityTerms r{};
    const double compression = dot_xfirst(vd, d);
    if (compression >= 0.0) return r;
    const float h = k.h;
    const double denominator = static_cast<double>(sq_xfirst(d)) + 0.01 * h * h;
    const double viscosity = 0.5 * (first_viscosity + second_viscosity);
    const double speed = 0.5 * (first_speed + second_speed);
    const double density_sum = first_density + second_density;
    const double nu = 2.0 * viscosity * h * speed / density_sum;
    const double pi = -nu * compression / denominator;
    const f3 gradient = cubic_gradient_value(d, k);
    r.neighbor_mass = -pi * dot(adjoint, gradient);
    const double pi_adjoint = -neighbor_mass * dot(adjoint, gradient);
    const d3 gradient_adjoint = times(adjoint, -neighbor_mass * pi);
    r.displacement = hessian_times(H, d, gradient_adjoint);
    const double nu_adjoint = -compression * pi_adjoint / denominator;
    const double compression_adjoint = -nu * pi_adjoint / denominator;
    const double denominator_adjoint = nu * compression * pi_adjoint / (denominator * denominator);
    r.velocity_difference = times(d, compression_adjoint);
    r.displacement = r.displacement + (times(vd, compression_adjoint) + times(d, 2.0 * denominator_adjoint));
    const double viscosity_adjoint = 2.0 * h * speed * nu_adjoint / density_sum;
    const double speed_adjoint = 2.0 * viscosity * h * nu_adjoint / density_sum;
    const double density_adjoint = -nu * nu_adjoint / density_sum;
    r.first_viscosity = r.second_viscosity = 0.5 * viscosity_adjoint;
    r.first_speed = r.second_speed = 0.5 * speed_adjoint;
    r.first_density = r.second_density = density_adjoint;
    return r;
}

// surface_reverse (sph/wcsph.cu:68-84): the adjoint of one cohesion / adhesion term.
struct SurfaceTerms {
    d3 displacement;
    double first_mass, second_mass, tension;
};

__device__ __forceinline__ SurfaceTerms surface_reverse(const f3 d, const float first_mass, const float second_mass,
                                                        const float tension, const SphConstants& k, const d3 adjoint) {
    SurfaceTerms r{};
    const float distance = __fsqrt_rn(sq_xfirst(d));
    if (distance >= k.h) return r;
    const bool far = distance > k.diameter;
    const float weight = far ? cubic_inside(distance, k) : k.contact_weight;
    const double factor = -static_cast<double>(tension) * second_mass * weight / first_mass;
    const double factor_adjoint = dot(adjoint, d);
    r.displacement = times(adjoint, factor);
    if (far)
        r.displacement = r.displacement +
                         times(scale(d, cubic_gradient_scale(distance, k)), -static_cast<double>(tension) * second_mass * factor_adjoint / first_mass);
    r.tension = -second_mass * weight * factor_adjoint / first_mass;
    r.second_mass = -tension * weight * factor_adjoint / first_mass;
    r.first_mass = tension * second_mass * weight * factor_adjoint / (first_mass * first_mass);
    return r;
}

// ------------------------------------------------------------------ WCSPH integrate (reverse)
struct IntegrateVjpArgs {
    SphStep st;
    const float4* total;        // the total acceleration of the step
    ConstAdjField3 next_x, next_v;
    AdjField3 x, v, control;    // caller adjoints, original order (accumulated)
    double4* acceleration;      // total-acceleration adjoint (sorted)
};

// integrate_vjp (sph/common.cu:344-366) and the control adjoint (sph/sph.cpp:244).
__global__ void integrate_vjp_kernel(const IntegrateVjpArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.st.g.count) return;
    const uint32_t i = a.st.sorted_index[s];
    const SceneDesc& sc = a.st.g.scenes[a.st.g.cell[s].w];
    const SphConstants& k = a.st.constants[sc.constants];
    bool cx, cy, cz;
    collision_mask(xyz(a.st.topology[s]), xyz(a.st.velocity[s]), xyz(a.total[s]), sc.time_step, sc.box, cx, cy, cz);
    const float dt = sc.time_step;
    const d3 pb = {cx ? 0.0 : a.next_x.x[i], cy ? 0.0 : a.next_x.y[i], cz ? 0.0 : a.next_x.z[i]};
    d3 vb = {a.next_v.x[i] + dt * pb.x, a.next_v.y[i] + dt * pb.y, a.next_v.z[i] + dt * pb.z};
    if (k.no_slip != 0u && (cx || cy || cz)) {
        vb = {0.0, 0.0, 0.0};
    } else {
        if (cx) vb.x = 0.0;
        if (cy) vb.y = 0.0;
        if (cz) vb.z = 0.0;
    }
    add_to(a.x, i, pb);
    add_to(a.v, i, vb);
    const d3 ab = {dt * vb.x, dt * vb.y, dt * vb.z};
    a.acceleration[s] = st4(ab);
    add_to(a.control, i, ab);
}

// ------------------------------------------------------------------ WCSPH forces (reverse)
struct ParameterAdjoints {
    double* masses;
    double* rest_densities;
    double* viscosities;
    double* surface_tensions;
    double* method0;   // WCSPH speed of sound / relaxation of PCISPH, IISPH, DFSPH divergence
    double* method1;   // WCSPH Tait exponent / DFSPH density relaxation
    double* method2;   // WCSPH boundary surface tension
};

struct ForceVjpArgs {
    SphStep st;
    const float* pressure;
    const double4* acceleration;   // total-acceleration adjoint (sorted)
    AdjField3 x, v;
    ParameterAdjoints pa;
    double* density_adjoint;       // sorted, written
};

struct ForceVjpData {
    float4 q, v, aux;
    float p;
    double4 adjoint;
};

// surface_vjp (sph/wcsph.cu:389-436), viscosity_vjp (sph/wcsph.cu:242-304) and pressure_vjp
// (sph/common.cu:239-300) in one walk, each with its own accumulators so every sum keeps the
// reference's order.
struct ForceVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    const float4* __restrict__ aux;
    const float* __restrict__ pressure;
    const double4* __restrict__ acceleration;
    const float4* __restrict__ boundary;
    const float4* __restrict__ boundary_velocity;
    uint32_t self;
    f3 x, v;
    float mass, rest, density, viscosity, speed, tension, boundary_tension;
    double first_term;
    d3 adjoint;
    SphConstants k;
    // surface
    d3 s_position;
    double s_mass, s_rest, s_tension, s_boundary_tension;
    // viscosity
    d3 v_position, v_velocity;
    double v_mass, v_rest, v_density, v_viscosity, v_speed;
    // pressure
    d3 p_position;
    double p_mass, p_rest, first_term_adjoint;

    __device__ __forceinline__ ForceVjpData prefetch(const uint32_t t) const {
        ForceVjpData d;
        if (t & kBoundaryBit) {
            d.q = boundary[t & ~kBoundaryBit];
            d.v = boundary_velocity[t & ~kBoundaryBit];
            d.aux = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
            d.p = 0.0F;
            d.adjoint = make_double4(0.0, 0.0, 0.0, 0.0);
            return d;
        }
        d.q = pos[t];
        d.v = vel[t];
        d.aux = aux[t];
        d.p = pressure[t];
        d.adjoint = acceleration[t];
        return d;
    }
    __device__ __forceinline__ void apply(const uint32_t t, const ForceVjpData& d) {
        const f3 disp = sub(x, xyz(d.q));
        // every term vanishes once sqrt((double) r2) >= h (the FP64 Hessian's support, the widest)
        const CubicHessian H = cubic_hessian(disp, k);
        if (H.kind == 0) return;
        const f3 dv = sub(v, xyz(d.v));
        if (t & kBoundaryBit) {
            const float volume = d.q.w;
            const float boundary_mass = __fmul_rn(rest, volume);
            const SurfaceTerms sl = surface_reverse(disp, mass, boundary_mass, boundary_tension, k, adjoint);
            s_position = s_position + sl.displacement;
            s_mass += sl.first_mass;
            s_rest += sl.second_mass * volume;
            s_boundary_tension += sl.tension;
            const ViscosityTerms vl =
                viscosity_reverse(disp, dv, density, density, viscosity, viscosity, speed, speed, boundary_mass, k, adjoint, H);
            v_position = v_position + vl.displacement;
            v_velocity = v_velocity + vl.velocity_difference;
            v_rest += vl.neighbor_mass * volume;
            v_density += vl.first_density + vl.second_density;
            v_viscosity += vl.first_viscosity + vl.second_viscosity;
            v_speed += vl.first_speed + vl.second_speed;
            const f3 gradient = cubic_gradient_value(disp, k);
            const double factor = static_cast<double>(__fmul_rn(-rest, volume)) * first_term;
            const double factor_adjoint = dot(adjoint, gradient);
            p_rest -= factor_adjoint * volume * first_term;
            first_term_adjoint -= factor_adjoint * rest * volume;
            p_position = p_position + hessian_times(H, disp, times(adjoint, factor));
            return;
        }
        if (t == self) return;
        const float mj = d.q.w;
        const d3 cross = ld(d.adjoint);
        // surface: own term and the term of j's acceleration (sph/wcsph.cu:404-411)
        const SurfaceTerms sl = surface_reverse(disp, mass, mj, tension, k, adjoint);
        s_position = s_position + sl.displacement;
        s_mass += sl.first_mass;
        s_tension += sl.tension;
        const SurfaceTerms sc = surface_reverse(negf(disp), mj, mass, d.aux.w, k, cross);
        s_position = s_position + neg(sc.displacement);
        s_mass += sc.second_mass;
        // viscosity (sph/wcsph.cu:266-281)
        const ViscosityTerms vl =
            viscosity_reverse(disp, dv, density, d.aux.x, viscosity, d.aux.y, speed, d.aux.z, mj, k, adjoint, H);
        v_position = v_position + vl.displacement;
        v_velocity = v_velocity + vl.velocity_difference;
        v_density += vl.first_density;
        v_viscosity += vl.first_viscosity;
        v_speed += vl.first_speed;
        const ViscosityTerms vc =
            viscosity_reverse(negf(disp), negf(dv), d.aux.x, density, d.aux.y, viscosity, d.aux.z, speed, mass, k, cross, H);
        v_position = v_position + neg(vc.displacement);
        v_velocity = v_velocity + neg(vc.velocity_difference);
        v_mass += vc.neighbor_mass;
        v_density += vc.second_density;
        v_viscosity += vc.second_viscosity;
        v_speed += vc.second_speed;
        // pressure (sph/common.cu:263-277)
        const f3 gradient = cubic_gradient_value(disp, k);
        const double second_term = static_cast<double>(d.p) / (d.aux.x * d.aux.x);
        const double sum = first_term + second_term;
        const double local_factor = -mj * sum;
        const double local_factor_adjoint = dot(adjoint, gradient);
        first_term_adjoint -= mj * local_factor_adjoint;
        p_position = p_position + hessian_times(H, disp, times(adjoint, local_factor));
        const double cross_projection = dot(cross, gradient);
        p_mass += sum * cross_projection;
        first_term_adjoint += mass * cross_projection;
        p_position = p_position + hessian_times(H, disp, times(cross, mass * sum));
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_WCSPH_FORCE_VJP_MIN_BLOCKS) wcsph_force_vjp_kernel(const ForceVjpArgs a) {
    const SphStep& st = a.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    const uint32_t i = st.sorted_index[s];
    ForceVjpOp op{};
    op.pos = st.topology;
    op.vel = st.velocity;
    op.aux = st.aux;
    op.pressure = a.pressure;
    op.acceleration = a.acceleration;
    op.boundary = st.g.boundary;
    op.boundary_velocity = st.boundary_velocity;
    op.self = s;
    op.x = o.x;
    op.v = xyz(st.velocity[s]);
    const float4 au = st.aux[s];
    const float4 pb = st.g.params_b[s];
    op.mass = o.mass;
    op.rest = o.pa.x;
    op.density = au.x;
    op.viscosity = o.pa.y;
    op.speed = o.pa.w;
    op.tension = o.pa.z;
    op.boundary_tension = pb.y;
    const float p = a.pressure[s];
    op.first_term = static_cast<double>(p) / (au.x * au.x);
    op.adjoint = ld(a.acceleration[s]);
    op.k = *o.k;
    replay(op, o.p, st.g, st.list);
    // the reference's kernels accumulate in the order surface, viscosity, pressure (sph/sph.cpp:245-247)
    add_to(a.x, i, op.s_position);
    add_to(a.x, i, op.v_position);
    add_to(a.x, i, op.p_position);
    add_to(a.v, i, op.v_velocity);
    const ParameterAdjoints& pa = a.pa;
    add_to(pa.masses, i, op.s_mass);
    add_to(pa.masses, i, op.v_mass);
    add_to(pa.masses, i, op.p_mass);
    add_to(pa.rest_densities, i, op.s_rest);
    add_to(pa.rest_densities, i, op.v_rest);
    add_to(pa.rest_densities, i, op.p_rest);
    add_to(pa.surface_tensions, i, op.s_tension);
    add_to(pa.method2, i, op.s_boundary_tension);
    add_to(pa.viscosities, i, op.v_viscosity);
    add_to(pa.method0, i, op.v_speed);
    const float rho = au.x;
    double density_adjoint = op.v_density;
    const double pressure_adjoint = op.first_term_adjoint / (rho * rho);
    density_adjoint -= 2.0 * op.first_term_adjoint * p / (rho * rho * rho);
    // Tait equation of state (sph/wcsph.cu:119-134)
    const double dd = rho, rest = o.pa.x, speed = o.pa.w, exponent = pb.x;
    const double ratio = dd / rest;
    const double powered = pow(ratio, exponent);
    const double difference = powered - 1.0;
    density_adjoint += pressure_adjoint * speed * speed * pow(ratio, exponent - 1.0);
    add_to(pa.rest_densities, i, pressure_adjoint * (speed * speed * difference / exponent - speed * speed * powered));
    add_to(pa.method0, i, pressure_adjoint * 2.0 * rest * speed * difference / exponent);
    add_to(pa.method1, i, pressure_adjoint * rest * speed * speed * (exponent * powered * log(ratio) - difference) /
                              (exponent * exponent));
    a.density_adjoint[s] = density_adjoint;
}

// ------------------------------------------------------------------ density (reverse)
struct DensityVjpArgs {
    SphStep st;
    const float4* positions;          // x (step density) or x*_k (predicted density), with mass
    const double* density_adjoint;    // sorted
    int walk;                         // 0 replay the list, 1 walk the stencil, 2 decide from the displacement slot
    uint32_t displacement_slot;
    AdjField3 x, v;
    ParameterAdjoints pa;
    // predicted density: the prediction's reverse (predict_vjp, sph/pcisph.cu:67-103)
    int predicted;
    const float4* acceleration;       // the pressure acceleration the prediction used
    const float4* base;               // DFSPH's divergence acceleration added to it, or null
    double4* non_pressure_adjoint;
    double4* acceleration_adjoint;    // of `acceleration`
    double4* base_adjoint;            // of `base`, or null
};

struct DensityVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    const double* __restrict__ density_adjoint;
    f3 x;
    float mass, rest;
    double own;
    SphConstants k;
    d3 position;
    double mass_sum, rest_sum;

    __device__ __forceinline__ float4 prefetch(const uint32_t t) const {
        return (t & kBoundaryBit) ? boundary[t & ~kBoundaryBit] : pos[t];
    }
    __device__ __forceinline__ void apply(const uint32_t t, const float4 q) {
        const f3 d = sub(x, xyz(q));
        const float r = __fsqrt_rn(sq_xfirst(d));
        if (r >= k.h) return;
        const f3 gradient = r == 0.0F ? mk(0.0F, 0.0F, 0.0F) : scale(d, cubic_gradient_scale(r, k));
        const float w = cubic_inside(r, k);
        if (t & kBoundaryBit) {   // density/density.cu:92-97
            const float volume = q.w;
            position = position + times(gradient, own * rest * volume);
            rest_sum += own * volume * w;
            return;
        }
        const double other = density_adjoint[t];   // density/density.cu:86-90
        position = position + times(gradient, own * q.w + other * mass);
        mass_sum += other * w;
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_SPH_DENSITY_VJP_MIN_BLOCKS) density_vjp_kernel(const DensityVjpArgs a) {
    const SphStep& st = a.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    const uint32_t i = st.sorted_index[s];
    DensityVjpOp op{};
    op.pos = a.positions;
    op.boundary = st.g.boundary;
    op.density_adjoint = a.density_adjoint;
    const float4 xi = a.positions[s];
    op.x = xyz(xi);
    op.mass = o.mass;
    op.rest = o.pa.x;
    op.own = a.density_adjoint[s];
    op.k = *o.k;
    bool walk_all = a.walk == 1;
    if (a.walk == 2) walk_all = !(__fmul_rn(2.0F, __uint_as_float(st.displacement[a.displacement_slot])) <= o.k->skin_bound);
    if (walk_all) walk(op, o.p, st.g);
    else replay(op, o.p, st.g, st.list);
    add_to(a.pa.masses, i, op.mass_sum);
    add_to(a.pa.rest_densities, i, op.rest_sum);
    if (!a.predicted) {
        add_to(a.x, i, op.position);
        return;
    }
    const SceneDesc& sc = *o.p.scene;
    const float dt = sc.time_step;
    const f3 acceleration = a.base ? add(xyz(a.base[s]), xyz(a.acceleration[s])) : xyz(a.acceleration[s]);
    bool cx, cy, cz;
    collision_mask(o.x, xyz(st.velocity[s]), add(xyz(st.non_pressure[s]), acceleration), dt, sc.box, cx, cy, cz);
    const d3 pb = {cx ? 0.0 : op.position.x, cy ? 0.0 : op.position.y, cz ? 0.0 : op.position.z};
    d3 vb = {dt * pb.x, dt * pb.y, dt * pb.z};   // the predicted velocity's adjoint is zero here
    if (op.k.no_slip != 0u && (cx || cy || cz)) {
        vb = {0.0, 0.0, 0.0};
    } else {
        if (cx) vb.x = 0.0;
        if (cy) vb.y = 0.0;
        if (cz) vb.z = 0.0;
    }
    add_to(a.x, i, pb);
    add_to(a.v, i, vb);
    const d3 ab = {dt * vb.x, dt * vb.y, dt * vb.z};
    a.non_pressure_adjoint[s] = st4(ld(a.non_pressure_adjoint[s]) + ab);
    a.acceleration_adjoint[s] = st4(ld(a.acceleration_adjoint[s]) + ab);
    if (a.base_adjoint) a.base_adjoint[s] = st4(ld(a.base_adjoint[s]) + ab);
}

// ------------------------------------------------------------------ final prediction (reverse)
struct PredictVjpArgs {
    SphStep st;
    const float4* acceleration;
    const float4* base;
    ConstAdjField3 next_x, next_v;
    AdjField3 x, v;
    double4* non_pressure_adjoint;
    double4* acceleration_adjoint;   // written (not accumulated)
    double4* base_adjoint;           // written (DFSPH), or null
    const double* next_warm;         // DFSPH: the density phase's warm-pressure adjoint (original order), or null
    double* pressure_adjoint;        // sorted, written with next_warm (or 0)
};

__global__ void predict_vjp_kernel(const PredictVjpArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.st.g.count) return;
    const uint32_t i = a.st.sorted_index[s];
    const SceneDesc& sc = a.st.g.scenes[a.st.g.cell[s].w];
    const SphConstants& k = a.st.constants[sc.constants];
    const float dt = sc.time_step;
    const f3 acceleration = a.base ? add(xyz(a.base[s]), xyz(a.acceleration[s])) : xyz(a.acceleration[s]);
    bool cx, cy, cz;
    collision_mask(xyz(a.st.topology[s]), xyz(a.st.velocity[s]), add(xyz(a.st.non_pressure[s]), acceleration), dt, sc.box, cx,
                   cy, cz);
    const d3 pb = {cx ? 0.0 : a.next_x.x[i], cy ? 0.0 : a.next_x.y[i], cz ? 0.0 : a.next_x.z[i]};
    d3 vb = {a.next_v.x[i] + dt * pb.x, a.next_v.y[i] + dt * pb.y, a.next_v.z[i] + dt * pb.z};
    if (k.no_slip != 0u && (cx || cy || cz)) {
        vb = {0.0, 0.0, 0.0};
    } else {
        if (cx) vb.x = 0.0;
        if (cy) vb.y = 0.0;
        if (cz) vb.z = 0.0;
    }
    add_to(a.x, i, pb);
    add_to(a.v, i, vb);
    const d3 ab = {dt * vb.x, dt * vb.y, dt * vb.z};
    a.non_pressure_adjoint[s] = st4(ld(a.non_pressure_adjoint[s]) + ab);
    a.acceleration_adjoint[s] = st4(ab);
    if (a.base_adjoint) a.base_adjoint[s] = st4(ab);
    if (a.pressure_adjoint) a.pressure_adjoint[s] = a.next_warm ? a.next_warm[i] : 0.0;
}

// ------------------------------------------------------------------ pressure + update (reverse)
struct PressureVjpArgs {
    SphStep st;
    const float* pressure;            // p_k
    const double4* acceleration_adjoint;   // of a_k (sorted)
    double* pressure_adjoint;         // p_k's adjoint (sorted): holds the later iteration's part, completed here
    double* density_adjoint;          // sorted, accumulated
    AdjField3 x;
    ParameterAdjoints pa;
    // the pressure update that produced p_k (pressure_update_vjp, sph/pcisph.cu:113-128,
    // sph/iisph.cu:113-129, sph/dfsph.cu:113-129); method 0 = none (an iteration-0 pressure)
    uint32_t method;
    uint32_t relaxation;              // 0: params_a.w, 1: params_b.x
    uint32_t target;                  // 0 rest density, 1 density
    const float* previous_pressure;   // p_(k-1)
    const float* predicted_density;   // rho*_k
    double* previous_pressure_adjoint;   // accumulated
    double* predicted_density_adjoint;   // written
    double* relaxation_adjoint;       // original order
    double* warm_adjoint;             // iteration-0 pressure of a DFSPH phase: the warm start's adjoint (written), or null
};

struct PressureVjpData {
    float4 q;
    float p, rho;
    double4 adjoint;
};

struct PressureVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ aux;
    const float* __restrict__ pressure;
    const double4* __restrict__ acceleration_adjoint;
    const float4* __restrict__ boundary;
    uint32_t self;
    f3 x;
    float mass, rest;
    double first_term;
    d3 adjoint;
    SphConstants k;
    d3 position;
    double mass_sum, rest_sum, first_term_adjoint;

    __device__ __forceinline__ PressureVjpData prefetch(const uint32_t t) const {
        if (t & kBoundaryBit) return {boundary[t & ~kBoundaryBit], 0.0F, 0.0F, make_double4(0.0, 0.0, 0.0, 0.0)};
        return {pos[t], pressure[t], aux[t].x, acceleration_adjoint[t]};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const PressureVjpData& d) {
        const f3 disp = sub(x, xyz(d.q));
        const CubicHessian H = cubic_hessian(disp, k);
        if (H.kind == 0) return;
        const f3 gradient = cubic_gradient_value(disp, k);
        if (t & kBoundaryBit) {   // sph/common.cu:279-290
            const float volume = d.q.w;
            const double factor = static_cast<double>(__fmul_rn(-rest, volume)) * first_term;
            const double factor_adjoint = dot(adjoint, gradient);
            rest_sum -= factor_adjoint * volume * first_term;
            first_term_adjoint -= factor_adjoint * rest * volume;
            position = position + hessian_times(H, disp, times(adjoint, factor));
            return;
        }
        if (t == self) return;
        const float mj = d.q.w;
        const double second_term = static_cast<double>(d.p) / (d.rho * d.rho);
        const double sum = first_term + second_term;
        const double local_factor = -mj * sum;
        const double local_factor_adjoint = dot(adjoint, gradient);
        first_term_adjoint -= mj * local_factor_adjoint;
        position = position + hessian_times(H, disp, times(adjoint, local_factor));
        const d3 cross = ld(d.adjoint);
        const double cross_projection = dot(cross, gradient);
        mass_sum += sum * cross_projection;
        first_term_adjoint += mass * cross_projection;
        position = position + hessian_times(H, disp, times(cross, mass * sum));
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_SPH_PRESSURE_VJP_MIN_BLOCKS) pressure_vjp_kernel(const PressureVjpArgs a) {
    const SphStep& st = a.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    const uint32_t i = st.sorted_index[s];
    PressureVjpOp op{};
    op.pos = st.topology;
    op.aux = st.aux;
    op.pressure = a.pressure;
    op.acceleration_adjoint = a.acceleration_adjoint;
    op.boundary = st.g.boundary;
    op.self = s;
    op.x = o.x;
    op.mass = o.mass;
    op.rest = o.pa.x;
    const float rho = st.aux[s].x;
    const float p = a.pressure[s];
    op.first_term = static_cast<double>(p) / (rho * rho);
    op.adjoint = ld(a.acceleration_adjoint[s]);
    op.k = *o.k;
    replay(op, o.p, st.g, st.list);
    add_to(a.x, i, op.position);
    add_to(a.pa.masses, i, op.mass_sum);
    add_to(a.pa.rest_densities, i, op.rest_sum);
    const double pressure_adjoint = a.pressure_adjoint[s] + op.first_term_adjoint / (rho * rho);
    double density_adjoint = a.density_adjoint[s] - 2.0 * op.first_term_adjoint * p / (rho * rho * rho);
    a.pressure_adjoint[s] = pressure_adjoint;
    if (a.warm_adjoint) a.warm_adjoint[i] = pressure_adjoint;
    if (a.method != 0u) {
        const float4 pb = st.g.params_b[s];
        const float relaxation = a.relaxation == 0u ? o.pa.w : pb.x;
        const float rest = o.pa.x;
        const float target = a.target == 1u ? rho : rest;
        const double error = static_cast<double>(a.predicted_density[s]) - target;
        const double volume = static_cast<double>(o.mass) / (a.method == kPcisph ? rest : rho);
        const double dt = o.p.scene->time_step;
        const double delta = 1.0 / (2.0 * dt * dt * volume * volume * o.k->reference_gradient_norm);
        const double candidate = a.previous_pressure[s] + relaxation * delta * error;
        double predicted_adjoint = 0.0;
        if (candidate > 0.0) {
            a.previous_pressure_adjoint[s] += pressure_adjoint;
            predicted_adjoint = relaxation * delta * pressure_adjoint;
            if (a.method == kPcisph) {
                add_to(a.pa.rest_densities, i, relaxation * delta * pressure_adjoint * (-1.0 + 2.0 * error / rest));
            } else {
                if (a.target == 1u) density_adjoint -= relaxation * delta * pressure_adjoint;
                else add_to(a.pa.rest_densities, i, -(relaxation * delta * pressure_adjoint));
                density_adjoint += 2.0 * relaxation * delta * error * pressure_adjoint / rho;
            }
            add_to(a.pa.masses, i, -(2.0 * relaxation * delta * error * pressure_adjoint / o.mass));
            add_to(a.relaxation_adjoint, i, delta * error * pressure_adjoint);
        }
        a.predicted_density_adjoint[s] = predicted_adjoint;
    }
    a.density_adjoint[s] = density_adjoint;
}

// ------------------------------------------------------------------ non-pressure (reverse)
struct NonPressureVjpArgs {
    SphStep st;
    const double4* adjoint;       // of the non-pressure acceleration (sorted)
    AdjField3 x, v, control;
    double* density_adjoint;      // sorted, accumulated
    ParameterAdjoints pa;
};

struct NonPressureVjpData {
    float4 q, v, aux;
    double4 adjoint;
};

// non_pressure_vjp (sph/common.cu:98-163)
struct NonPressureVjpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    const float4* __restrict__ aux;
    const double4* __restrict__ adjoint_of;
    const float4* __restrict__ boundary;
    const float4* __restrict__ boundary_velocity;
    uint32_t self;
    f3 x, v;
    float mass, density, viscosity;
    d3 adjoint;
    SphConstants k;
    d3 position, velocity;
    double density_sum, mass_sum, viscosity_sum;

    __device__ __forceinline__ NonPressureVjpData prefetch(const uint32_t t) const {
        if (t & kBoundaryBit)
            return {boundary[t & ~kBoundaryBit], boundary_velocity[t & ~kBoundaryBit], make_float4(0.0F, 0.0F, 0.0F, 0.0F),
                    make_double4(0.0, 0.0, 0.0, 0.0)};
        return {pos[t], vel[t], aux[t], adjoint_of[t]};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const NonPressureVjpData& d) {
        const f3 disp = sub(x, xyz(d.q));
        if (static_cast<double>(sq_xfirst(disp)) >= k.support_squared_d) return;   // sqrt(r2) >= h, exactly
        const f3 difference = sub(xyz(d.v), v);
        const float laplacian = laplacian_value(disp, k);
        if (t & kBoundaryBit) {   // sph/common.cu:145-155
            const float volume = d.q.w;
            const float weight = __fmul_rn(__fmul_rn(viscosity, volume), laplacian);
            const double weight_adjoint = dot(adjoint, difference);
            velocity = velocity + times(adjoint, -weight);
            viscosity_sum += weight_adjoint * volume * laplacian;
            position = position + laplacian_gradient(disp, k, weight_adjoint * viscosity * volume);
            return;
        }
        if (t == self) return;
        const float mj = d.q.w, rho_j = d.aux.x;
        const float mu = __fmul_rn(0.5F, __fadd_rn(viscosity, d.aux.y));
        const float weight = __fdiv_rn(__fmul_rn(__fmul_rn(mu, mj), laplacian), rho_j);
        const double weight_adjoint = dot(adjoint, difference);
        velocity = velocity + times(adjoint, -weight);
        const double viscosity_adjoint = weight_adjoint * mj * laplacian / rho_j;
        viscosity_sum += 0.5 * viscosity_adjoint;
        position = position + laplacian_gradient(disp, k, weight_adjoint * mu * mj / rho_j);
        const d3 cross = ld(d.adjoint);
        const float cross_weight = __fdiv_rn(__fmul_rn(__fmul_rn(mu, mass), laplacian), density);
        const double cross_weight_adjoint = dot(cross, scale(difference, -1.0F));
        velocity = velocity + times(cross, cross_weight);
        mass_sum += cross_weight_adjoint * mu * laplacian / density;
        density_sum -= cross_weight_adjoint * mu * mass * laplacian / (density * density);
        viscosity_sum += 0.5 * cross_weight_adjoint * mass * laplacian / density;
        position = position + laplacian_gradient(disp, k, cross_weight_adjoint * mu * mass / density);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_SPH_NON_PRESSURE_VJP_MIN_BLOCKS) non_pressure_vjp_kernel(const NonPressureVjpArgs a) {
    const SphStep& st = a.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    const uint32_t i = st.sorted_index[s];
    NonPressureVjpOp op{};
    op.pos = st.topology;
    op.vel = st.velocity;
    op.aux = st.aux;
    op.adjoint_of = a.adjoint;
    op.boundary = st.g.boundary;
    op.boundary_velocity = st.boundary_velocity;
    op.self = s;
    op.x = o.x;
    op.v = xyz(st.velocity[s]);
    op.mass = o.mass;
    op.density = st.aux[s].x;
    op.viscosity = o.pa.y;
    op.adjoint = ld(a.adjoint[s]);
    op.k = *o.k;
    replay(op, o.p, st.g, st.list);
    add_to(a.x, i, op.position);
    add_to(a.v, i, op.velocity);
    add_to(a.control, i, op.adjoint);
    a.density_adjoint[s] += op.density_sum;
    add_to(a.pa.masses, i, op.mass_sum);
    add_to(a.pa.viscosities, i, op.viscosity_sum);
}

// A phase switch of DFSPH's reverse: the divergence phase's last acceleration adjoint is the
// divergence acceleration's, and its last pressure adjoint the next warm divergence pressure's.
__global__ void phase_seed_kernel(const uint32_t count, const uint32_t* __restrict__ sorted_index, const double4* __restrict__ from,
                                  double4* __restrict__ acceleration_adjoint, const double* __restrict__ next_warm,
                                  double* __restrict__ pressure_adjoint) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    acceleration_adjoint[s] = from[s];
    pressure_adjoint[s] = next_warm ? next_warm[sorted_index[s]] : 0.0;
}

inline unsigned grid_of(const uint32_t n, const unsigned block) { return (n + block - 1u) / block; }
unsigned block_of(const unsigned block) {
    return block >= 32u && block <= static_cast<unsigned>(kBlock) && block % 32u == 0u ? block : static_cast<unsigned>(kBlock);
}

}  // namespace

// ================================================================== launchers
cudaError_t launch_integrate_vjp(cudaStream_t stream, const SphStep& st, const float4* total, ConstAdjField3 next_x,
                                 ConstAdjField3 next_v, AdjField3 x, AdjField3 v, AdjField3 control, double4* acceleration) {
    if (st.g.count == 0) return cudaSuccess;
    integrate_vjp_kernel<<<grid_of(st.g.count, 256), 256, 0, stream>>>(
        IntegrateVjpArgs{st, total, next_x, next_v, x, v, control, acceleration});
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_wcsph_force_vjp(cudaStream_t stream, const SphStep& st, const float* pressure, const double4* acceleration,
                                   AdjField3 x, AdjField3 v, const SphParameterAdjoints& pa, double* density_adjoint,
                                   const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    const ParameterAdjoints p{pa.masses, pa.rest_densities, pa.viscosities, pa.surface_tensions, pa.method0, pa.method1, pa.method2};
    wcsph_force_vjp_kernel<<<grid_of(st.g.count, b), b, 0, stream>>>(ForceVjpArgs{st, pressure, acceleration, x, v, p, density_adjoint});
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_density_vjp(cudaStream_t stream, const DensityVjpLaunch& d, const unsigned block) {
    if (d.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    const SphParameterAdjoints& pa = d.pa;
    const DensityVjpArgs a{d.st,
                           d.positions,
                           d.density_adjoint,
                           d.walk,
                           d.displacement_slot,
                           d.x,
                           d.v,
                           {pa.masses, pa.rest_densities, pa.viscosities, pa.surface_tensions, pa.method0, pa.method1, pa.method2},
                           d.predicted,
                           d.acceleration,
                           d.base,
                           d.non_pressure_adjoint,
                           d.acceleration_adjoint,
                           d.base_adjoint};
    density_vjp_kernel<<<grid_of(d.st.g.count, b), b, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_predict_vjp(cudaStream_t stream, const SphStep& st, const float4* acceleration, const float4* base,
                               ConstAdjField3 next_x, ConstAdjField3 next_v, AdjField3 x, AdjField3 v, double4* non_pressure_adjoint,
                               double4* acceleration_adjoint, double4* base_adjoint, const double* next_warm,
                               double* pressure_adjoint) {
    if (st.g.count == 0) return cudaSuccess;
    predict_vjp_kernel<<<grid_of(st.g.count, 256), 256, 0, stream>>>(PredictVjpArgs{
        st, acceleration, base, next_x, next_v, x, v, non_pressure_adjoint, acceleration_adjoint, base_adjoint, next_warm,
        pressure_adjoint});
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pressure_vjp(cudaStream_t stream, const PressureVjpLaunch& d, const unsigned block) {
    if (d.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    const SphParameterAdjoints& pa = d.pa;
    const PressureVjpArgs a{d.st,
                            d.pressure,
                            d.acceleration_adjoint,
                            d.pressure_adjoint,
                            d.density_adjoint,
                            d.x,
                            {pa.masses, pa.rest_densities, pa.viscosities, pa.surface_tensions, pa.method0, pa.method1, pa.method2},
                            d.method,
                            d.relaxation,
                            d.target,
                            d.previous_pressure,
                            d.predicted_density,
                            d.previous_pressure_adjoint,
                            d.predicted_density_adjoint,
                            d.relaxation_adjoint,
                            d.warm_adjoint};
    pressure_vjp_kernel<<<grid_of(d.st.g.count, b), b, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_non_pressure_vjp(cudaStream_t stream, const SphStep& st, const double4* adjoint, AdjField3 x, AdjField3 v,
                                    AdjField3 control, double* density_adjoint, const SphParameterAdjoints& pa,
                                    const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    const ParameterAdjoints p{pa.masses, pa.rest_densities, pa.viscosities, pa.surface_tensions, pa.method0, pa.method1, pa.method2};
    non_pressure_vjp_kernel<<<grid_of(st.g.count, b), b, 0, stream>>>(NonPressureVjpArgs{st, adjoint, x, v, control, density_adjoint, p});
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_phase_seed(cudaStream_t stream, const uint32_t count, const uint32_t* sorted_index, const double4* from,
                              double4* acceleration_adjoint, const double* next_warm, double* pressure_adjoint) {
    if (count == 0) return cudaSuccess;
    phase_seed_kernel<<<grid_of(count, 256), 256, 0, stream>>>(count, sorted_index, from, acceleration_adjoint, next_warm,
                                                                pressure_adjoint);
    count_launch();
    return cudaGetLastError();
}

}  // namespace sph
}  // namespace pbf

// ================================================================== tangent passes (FP32)
namespace pbf {
namespace sph {

namespace {

using namespace gather_detail;
using namespace detail;

// Sorted tangents of the inputs: positions and masses, velocities, and the parameters packed as
// params_a / params_b.
__global__ void tangent_seed_kernel(const SphTangentStep t, const Field3 x, const Field3 v, const SphParameterTangents pt) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= t.st.g.count) return;
    const uint32_t i = t.st.sorted_index[s];
    auto get = [i](const float* p) { return p ? p[i] : 0.0F; };
    t.x[s] = make_float4(x.x[i], x.y[i], x.z[i], get(pt.masses));
    t.v[s] = make_float4(v.x[i], v.y[i], v.z[i], 0.0F);
    t.params_a[s] = make_float4(get(pt.rest_densities), get(pt.viscosities), get(pt.surface_tensions), get(pt.method0));
    t.params_b[s] = make_float4(get(pt.method1), get(pt.method2), 0.0F, 0.0F);
}

// density_jvp (density/density.cu:42-66): sum of dm_j W + m_j grad W . (dx_i - dx_j), boundary
// V_b (drho0_i W + rho0_i grad W . dx_i).
struct DensityJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ tangent;
    const float4* __restrict__ boundary;
    f3 x, dx;
    float rest, drest;
    SphConstants k;
    float result;

    __device__ __forceinline__ void process(const uint32_t t) {
        if (t & kBoundaryBit) {
            const float4 q = boundary[t & ~kBoundaryBit];
            const f3 d = x - xyz(q);
            const float w = cubic_value(d, k);
            if (w == 0.0F) return;
            result += q.w * (drest * w + rest * dot(cubic_gradient_value(d, k), dx));
            return;
        }
        const float4 q = pos[t];
        const f3 d = x - xyz(q);
        const float w = cubic_value(d, k);
        if (w == 0.0F) return;
        const float4 tq = tangent[t];
        result += tq.w * w + q.w * dot(cubic_gradient_value(d, k), dx - xyz(tq));
    }
    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
};

// The density tangent at the step's positions (+ WCSPH's equation of state, sph/wcsph.cu:102-117;
// DFSPH: the divergence phase's warm-start pressure tangent).
__global__ void __launch_bounds__(kBlock, PBF_SPH_DENSITY_JVP_MIN_BLOCKS) density_jvp_kernel(const SphTangentStep t, const uint32_t method, const float* warm) {
    const SphStep& st = t.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    DensityJvpOp op{};
    op.pos = st.topology;
    op.tangent = t.x;
    op.boundary = st.g.boundary;
    op.x = o.x;
    op.dx = xyz(t.x[s]);
    op.rest = o.pa.x;
    op.drest = t.params_a[s].x;
    op.k = *o.k;
    replay(op, o.p, st.g, st.list);
    const float drho = op.result;
    t.density[s] = drho;
    float dp = 0.0F;
    if (method == kWcsph) {
        const float rho = st.aux[s].x, rest = o.pa.x, speed = o.pa.w, exponent = st.g.params_b[s].x;
        const float4 ta = t.params_a[s], tb = t.params_b[s];
        const float ratio = rho / rest;
        const float powered = powf(ratio, exponent);
        const float difference = powered - 1.0F;
        const float d_density = speed * speed * powf(ratio, exponent - 1.0F);
        const float d_rest = speed * speed * difference / exponent - speed * speed * powered;
        const float d_speed = 2.0F * rest * speed * difference / exponent;
        const float d_exponent = rest * speed * speed * (exponent * powered * logf(ratio) - difference) / (exponent * exponent);
        dp = d_density * drho + d_rest * ta.x + d_speed * ta.w + d_exponent * tb.x;
    } else if (warm) {
        dp = warm[st.sorted_index[s]];
    }
    t.pressure[s] = dp;
}

// pressure_jvp (sph/common.cu:196-237) of one pair, FP32.
__device__ __forceinline__ f3 pressure_pair_jvp(const f3 d, const f3 dd, const float factor, const float dfactor,
                                                const SphConstants& k) {
    return times(cubic_gradient_value(d, k), dfactor) + times(cubic_gradient_tangent(d, dd, k), factor);
}

struct ForceJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    const float4* __restrict__ aux;
    const float* __restrict__ pressure;
    const float4* __restrict__ tx;
    const float4* __restrict__ tv;
    const float4* __restrict__ tpa;
    const float* __restrict__ tdensity;
    const float* __restrict__ tpressure;
    const float4* __restrict__ boundary;
    const float4* __restrict__ boundary_velocity;
    uint32_t self;
    f3 x, v, dx, dv;
    float mass, dmass, rest, drest, density, ddensity, viscosity, dviscosity, speed, dspeed, tension, dtension;
    float boundary_tension, dboundary_tension, first, dfirst;
    SphConstants k;
    f3 rp, rv, rs;   // pressure, viscosity and surface tangents

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        const float h = k.h;
        if (t & kBoundaryBit) {
            const uint32_t b = t & ~kBoundaryBit;
            const float4 q = boundary[b];
            const f3 d = x - xyz(q);
            const float distance = sqrtf(dot(d, d));
            if (distance >= h) return;
            const float volume = q.w;
            // pressure (sph/common.cu:225-232)
            rp = rp + pressure_pair_jvp(d, dx, -rest * volume * first, -volume * (drest * first + rest * dfirst), k);
            // viscosity (sph/wcsph.cu:222-238)
            const f3 vd = v - xyz(boundary_velocity[b]);
            const float compression = dot(vd, d);
            if (compression < 0.0F) {
                const float dcompression = dot(dv, d) + dot(vd, dx);
                const float denominator = dot(d, d) + 0.01F * h * h;
                const float ddenominator = 2.0F * dot(d, dx);
                const float nu = viscosity * h * speed / density;
                const float dnu = h * (dviscosity * speed + viscosity * dspeed) / density - nu * ddensity / density;
                const float pi = -nu * compression / denominator;
                const float dpi = -(dnu * compression + nu * dcompression) / denominator +
                                  nu * compression * ddenominator / (denominator * denominator);
                const float m = rest * volume, dm = drest * volume;
                rv = rv + times(cubic_gradient_value(d, k), -(dm * pi + m * dpi)) + times(cubic_gradient_tangent(d, dx, k), -m * pi);
            }
            // adhesion (sph/wcsph.cu:371-384)
            const float weight = distance > k.diameter ? cubic_inside(distance, k) : k.contact_weight;
            const float dweight = distance > k.diameter ? dot(cubic_gradient_value(d, k), dx) : 0.0F;
            const float m = rest * volume, dm = drest * volume;
            const float factor = -boundary_tension * m * weight / mass;
            const float dfactor = -dboundary_tension * m * weight / mass - boundary_tension * dm * weight / mass -
                                  boundary_tension * m * dweight / mass + boundary_tension * m * weight * dmass / (mass * mass);
            rs = rs + times(d, dfactor) + times(dx, factor);
            return;
        }
        if (t == self) return;
        const float4 q = pos[t];
        const f3 d = x - xyz(q);
        const float distance = sqrtf(dot(d, d));
        if (distance >= h) return;
        const float4 tq = tx[t];
        const f3 dd = dx - xyz(tq);
        const float mj = q.w, dmj = tq.w;
        const float4 au = aux[t];
        const float rho_j = au.x, drho_j = tdensity[t];
        // pressure (sph/common.cu:214-222)
        const float pj = pressure[t];
        const float second = pj / (rho_j * rho_j);
        const float dsecond = tpressure[t] / (rho_j * rho_j) - 2.0F * pj * drho_j / (rho_j * rho_j * rho_j);
        rp = rp + pressure_pair_jvp(d, dd, -mj * (first + second), -dmj * (first + second) - mj * (dfirst + dsecond), k);
        // viscosity (sph/wcsph.cu:196-220)
        const f3 vd = v - xyz(vel[t]);
        const float compression = dot(vd, d);
        if (compression < 0.0F) {
            const float4 tpj = tpa[t];
            const f3 dvd = dv - xyz(tv[t]);
            const float dcompression = dot(dvd, d) + dot(vd, dd);
            const float denominator = dot(d, d) + 0.01F * h * h;
            const float ddenominator = 2.0F * dot(d, dd);
            const float alpha = 0.5F * (viscosity + au.y), dalpha = 0.5F * (dviscosity + tpj.y);
            const float c = 0.5F * (speed + au.z), dc = 0.5F * (dspeed + tpj.w);
            const float density_sum = density + rho_j, ddensity_sum = ddensity + drho_j;
            const float nu = 2.0F * alpha * h * c / density_sum;
            const float dnu = 2.0F * h * (dalpha * c + alpha * dc) / density_sum - nu * ddensity_sum / density_sum;
            const float pi = -nu * compression / denominator;
            const float dpi = -(dnu * compression + nu * dcompression) / denominator +
                              nu * compression * ddenominator / (denominator * denominator);
            rv = rv + times(cubic_gradient_value(d, k), -(dmj * pi + mj * dpi)) + times(cubic_gradient_tangent(d, dd, k), -mj * pi);
        }
        // cohesion (sph/wcsph.cu:355-368)
        const float weight = distance > k.diameter ? cubic_inside(distance, k) : k.contact_weight;
        const float dweight = distance > k.diameter ? dot(cubic_gradient_value(d, k), dd) : 0.0F;
        const float factor = -tension * mj * weight / mass;
        const float dfactor = -dtension * mj * weight / mass - tension * dmj * weight / mass - tension * mj * dweight / mass +
                              tension * mj * weight * dmass / (mass * mass);
        rs = rs + times(d, dfactor) + times(dd, factor);
    }
};

// The prediction's tangent (sph/pcisph.cu:46-66; integrate_jvp, sph/common.cu:322-342).
__device__ __forceinline__ void predict_tangent(const f3 x, const f3 v, const f3 a, const f3 dx, const f3 dv, const f3 da,
                                                const float dt, const Box& box, const SphConstants& k, f3& out_x, f3& out_v) {
    bool cx, cy, cz;
    collision_mask(x, v, a, dt, box, cx, cy, cz);
    f3 tv = dv + times(da, dt);
    f3 tx = dx + times(tv, dt);
    if (cx) tx.x = 0.0F;
    if (cy) tx.y = 0.0F;
    if (cz) tx.z = 0.0F;
    if (k.no_slip != 0u && (cx || cy || cz)) {
        tv = mk(0.0F, 0.0F, 0.0F);
    } else {
        if (cx) tv.x = 0.0F;
        if (cy) tv.y = 0.0F;
        if (cz) tv.z = 0.0F;
    }
    out_x = tx;
    out_v = tv;
}

__global__ void __launch_bounds__(kBlock, PBF_WCSPH_FORCE_JVP_MIN_BLOCKS) wcsph_force_jvp_kernel(const SphTangentStep t, const float* pressure,
                                                                 const float4* total, const Field3 control_tangent,
                                                                 const MutField3 out_x, const MutField3 out_v) {
    const SphStep& st = t.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    ForceJvpOp op{};
    op.pos = st.topology;
    op.vel = st.velocity;
    op.aux = st.aux;
    op.pressure = pressure;
    op.tx = t.x;
    op.tv = t.v;
    op.tpa = t.params_a;
    op.tdensity = t.density;
    op.tpressure = t.pressure;
    op.boundary = st.g.boundary;
    op.boundary_velocity = st.boundary_velocity;
    op.self = s;
    op.x = o.x;
    op.v = xyz(st.velocity[s]);
    const float4 txs = t.x[s], ta = t.params_a[s], tb = t.params_b[s];
    op.dx = xyz(txs);
    op.dv = xyz(t.v[s]);
    op.mass = o.mass;
    op.dmass = txs.w;
    op.rest = o.pa.x;
    op.drest = ta.x;
    const float4 au = st.aux[s];
    op.density = au.x;
    op.ddensity = t.density[s];
    op.viscosity = o.pa.y;
    op.dviscosity = ta.y;
    op.speed = o.pa.w;
    op.dspeed = ta.w;
    op.tension = o.pa.z;
    op.dtension = ta.z;
    op.boundary_tension = st.g.params_b[s].y;
    op.dboundary_tension = tb.y;
    const float p = pressure[s];
    op.first = p / (au.x * au.x);
    op.dfirst = t.pressure[s] / (au.x * au.x) - 2.0F * p * op.ddensity / (au.x * au.x * au.x);
    op.k = *o.k;
    op.rp = op.rv = op.rs = mk(0.0F, 0.0F, 0.0F);
    replay(op, o.p, st.g, st.list);
    const uint32_t i = st.sorted_index[s];
    const f3 da = op.rp + op.rv + op.rs + mk(control_tangent.x[i], control_tangent.y[i], control_tangent.z[i]);
    const SceneDesc& sc = *o.p.scene;
    f3 tx, tv;
    predict_tangent(o.x, op.v, xyz(total[s]), op.dx, op.dv, da, sc.time_step, sc.box, op.k, tx, tv);
    out_x.x[i] = tx.x;
    out_x.y[i] = tx.y;
    out_x.z[i] = tx.z;
    out_v.x[i] = tv.x;
    out_v.y[i] = tv.y;
    out_v.z[i] = tv.z;
}

// non_pressure_jvp (sph/common.cu:49-96) and, for PCISPH / IISPH, the first prediction's tangent.
struct NonPressureJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    const float4* __restrict__ aux;
    const float4* __restrict__ tx;
    const float4* __restrict__ tv;
    const float4* __restrict__ tpa;
    const float* __restrict__ tdensity;
    const float4* __restrict__ boundary;
    const float4* __restrict__ boundary_velocity;
    uint32_t self;
    f3 x, v, dx, dv;
    float viscosity, dviscosity;
    SphConstants k;
    f3 result;

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t & kBoundaryBit) {
            const uint32_t b = t & ~kBoundaryBit;
            const float4 q = boundary[b];
            const f3 d = x - xyz(q);
            const float laplacian = laplacian_value(d, k);
            const float dlaplacian = laplacian_tangent(d, dx, k);
            if (laplacian == 0.0F && dlaplacian == 0.0F) return;
            const float weight = viscosity * q.w * laplacian;
            const float dweight = q.w * (dviscosity * laplacian + viscosity * dlaplacian);
            const f3 difference = xyz(boundary_velocity[b]) - v;
            result = result + times(difference, dweight) + times(dv, -weight);
            return;
        }
        if (t == self) return;
        const float4 q = pos[t];
        const f3 d = x - xyz(q);
        const float laplacian = laplacian_value(d, k);
        if (laplacian == 0.0F) return;
        const float4 tq = tx[t];
        const f3 dd = dx - xyz(tq);
        const float dlaplacian = laplacian_tangent(d, dd, k);
        const float4 au = aux[t];
        const float mu = 0.5F * (viscosity + au.y), dmu = 0.5F * (dviscosity + tpa[t].y);
        const float mass = q.w, dmass = tq.w, density = au.x, ddensity = tdensity[t];
        const float weight = mu * mass * laplacian / density;
        const float dweight = dmu * mass * laplacian / density + mu * dmass * laplacian / density + mu * mass * dlaplacian / density -
                              mu * mass * laplacian * ddensity / (density * density);
        const f3 difference = xyz(vel[t]) - v;
        const f3 ddifference = xyz(tv[t]) - dv;
        result = result + times(difference, dweight) + times(ddifference, weight);
    }
};

__global__ void __launch_bounds__(kBlock, PBF_SPH_NON_PRESSURE_JVP_MIN_BLOCKS) non_pressure_jvp_kernel(const SphTangentStep t, const Field3 control_tangent,
                                                                  const int mode, const MutField3 out_x, const MutField3 out_v) {
    const SphStep& st = t.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    const uint32_t i = st.sorted_index[s];
    NonPressureJvpOp op{};
    op.pos = st.topology;
    op.vel = st.velocity;
    op.aux = st.aux;
    op.tx = t.x;
    op.tv = t.v;
    op.tpa = t.params_a;
    op.tdensity = t.density;
    op.boundary = st.g.boundary;
    op.boundary_velocity = st.boundary_velocity;
    op.self = s;
    op.x = o.x;
    op.v = xyz(st.velocity[s]);
    op.dx = xyz(t.x[s]);
    op.dv = xyz(t.v[s]);
    op.viscosity = o.pa.y;
    op.dviscosity = t.params_a[s].y;
    op.k = *o.k;
    op.result = mk(control_tangent.x[i], control_tangent.y[i], control_tangent.z[i]);
    replay(op, o.p, st.g, st.list);
    t.non_pressure[s] = make_float4(op.result.x, op.result.y, op.result.z, 0.0F);
    if (mode == 0) return;
    const SceneDesc& sc = *o.p.scene;
    f3 tx, tv;
    predict_tangent(o.x, op.v, xyz(st.non_pressure[s]), op.dx, op.dv, op.result, sc.time_step, sc.box, op.k, tx, tv);
    if (mode == 1) {
        t.predicted[s] = make_float4(tx.x, tx.y, tx.z, 0.0F);
        return;
    }
    out_x.x[i] = tx.x;
    out_x.y[i] = tx.y;
    out_x.z[i] = tx.z;
    out_v.x[i] = tv.x;
    out_v.y[i] = tv.y;
    out_v.z[i] = tv.z;
}

// density_jvp at a prediction (x*, its tangent) and the pressure update's tangent
// (sph/pcisph.cu:113-122, sph/iisph.cu:113-123, sph/dfsph.cu:113-123).
struct PredictedDensityJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ predicted;
    const float4* __restrict__ tpredicted;
    const float4* __restrict__ tx;
    const float4* __restrict__ boundary;
    f3 x, dx;
    float rest, drest;
    SphConstants k;
    float result;

    __device__ __forceinline__ float4 prefetch(const uint32_t t) const {
        return (t & kBoundaryBit) ? boundary[t & ~kBoundaryBit] : predicted[t];
    }
    __device__ __forceinline__ void apply(const uint32_t t, const float4 q) {
        const f3 d = x - xyz(q);
        const float w = cubic_value(d, k);
        if (w == 0.0F) return;
        if (t & kBoundaryBit) {
            result += q.w * (drest * w + rest * dot(cubic_gradient_value(d, k), dx));
            return;
        }
        result += tx[t].w * w + q.w * dot(cubic_gradient_value(d, k), dx - xyz(tpredicted[t]));
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

__global__ void __launch_bounds__(kBlock, PBF_SPH_DENSITY_JVP_MIN_BLOCKS) predicted_density_jvp_kernel(const SphTangentStep t, const PredictedJvp u) {
    const SphStep& st = t.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    PredictedDensityJvpOp op{};
    op.predicted = u.predicted;
    op.tpredicted = t.predicted;
    op.tx = t.x;
    op.boundary = st.g.boundary;
    op.x = xyz(u.predicted[s]);
    op.dx = xyz(t.predicted[s]);
    op.rest = o.pa.x;
    op.drest = t.params_a[s].x;
    op.k = *o.k;
    const float displacement = __uint_as_float(st.displacement[u.displacement_slot]);
    if (__fmul_rn(2.0F, displacement) <= o.k->skin_bound) replay(op, o.p, st.g, st.list);
    else walk(op, o.p, st.g);
    const float dpredicted = op.result;
    const float rho = st.aux[s].x, drho = t.density[s];
    const float4 ta = t.params_a[s], tb = t.params_b[s];
    const float relaxation = u.relaxation == 0u ? o.pa.w : st.g.params_b[s].x;
    const float drelaxation = u.relaxation == 0u ? ta.w : tb.x;
    const float rest = o.pa.x, drest = ta.x;
    const float target = u.target == 1u ? rho : rest, dtarget = u.target == 1u ? drho : drest;
    const float error = u.predicted_density[s] - target;
    const bool pcisph = u.method == kPcisph;
    const float volume = o.mass / (pcisph ? rest : rho);
    const float dt = o.p.scene->time_step;
    const float delta = 1.0F / (2.0F * dt * dt * volume * volume * o.k->reference_gradient_norm);
    const float ddelta = -2.0F * delta * (t.x[s].w / o.mass - (pcisph ? drest / rest : drho / rho));
    const float candidate = u.previous_pressure[s] + relaxation * delta * error;
    const float previous = t.pressure[s];
    t.pressure[s] = candidate > 0.0F ? previous + drelaxation * delta * error + relaxation * ddelta * error +
                                           relaxation * delta * (dpredicted - dtarget)
                                     : 0.0F;
}

// pressure_jvp (sph/common.cu:196-237) of iterate k and the next prediction's tangent.
struct PressureJvpOp {
    static constexpr bool kBoundary = true;
    const float4* __restrict__ pos;
    const float4* __restrict__ aux;
    const float* __restrict__ pressure;
    const float4* __restrict__ tx;
    const float* __restrict__ tdensity;
    const float* __restrict__ tpressure;
    const float4* __restrict__ boundary;
    uint32_t self;
    f3 x, dx;
    float rest, drest, first, dfirst;
    SphConstants k;
    f3 result;

    __device__ __forceinline__ uint32_t prefetch(const uint32_t t) const { return t; }
    __device__ __forceinline__ void apply(const uint32_t t, uint32_t) { process(t); }
    __device__ __forceinline__ void process(const uint32_t t) {
        if (t & kBoundaryBit) {
            const float4 q = boundary[t & ~kBoundaryBit];
            const f3 d = x - xyz(q);
            if (dot(d, d) >= k.h * k.h * 1.0001F) return;
            result = result + pressure_pair_jvp(d, dx, -rest * q.w * first, -q.w * (drest * first + rest * dfirst), k);
            return;
        }
        if (t == self) return;
        const float4 q = pos[t];
        const f3 d = x - xyz(q);
        if (dot(d, d) >= k.h * k.h * 1.0001F) return;
        const float4 tq = tx[t];
        const float rho_j = aux[t].x, pj = pressure[t];
        const float second = pj / (rho_j * rho_j);
        const float dsecond = tpressure[t] / (rho_j * rho_j) - 2.0F * pj * tdensity[t] / (rho_j * rho_j * rho_j);
        result = result + pressure_pair_jvp(d, dx - xyz(tq), -q.w * (first + second),
                                            -tq.w * (first + second) - q.w * (dfirst + dsecond), k);
    }
};

__global__ void __launch_bounds__(kBlock, PBF_SPH_PRESSURE_JVP_MIN_BLOCKS) pressure_jvp_kernel(const SphTangentStep t, const PressureJvp u) {
    const SphStep& st = t.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    PressureJvpOp op{};
    op.pos = st.topology;
    op.aux = st.aux;
    op.pressure = u.pressure;
    op.tx = t.x;
    op.tdensity = t.density;
    op.tpressure = t.pressure;
    op.boundary = st.g.boundary;
    op.self = s;
    op.x = o.x;
    op.dx = xyz(t.x[s]);
    op.rest = o.pa.x;
    op.drest = t.params_a[s].x;
    const float rho = st.aux[s].x, drho = t.density[s], p = u.pressure[s];
    op.first = p / (rho * rho);
    op.dfirst = t.pressure[s] / (rho * rho) - 2.0F * p * drho / (rho * rho * rho);
    op.k = *o.k;
    op.result = mk(0.0F, 0.0F, 0.0F);
    replay(op, o.p, st.g, st.list);
    const uint32_t i = st.sorted_index[s];
    f3 dacceleration = op.result;
    if (u.store) u.store[s] = make_float4(dacceleration.x, dacceleration.y, dacceleration.z, 0.0F);
    f3 acceleration = xyz(u.acceleration[s]);
    if (u.base) {
        acceleration = add(xyz(u.base[s]), acceleration);
        dacceleration = xyz(u.base_tangent[s]) + dacceleration;
    }
    if (u.warm_out) u.warm_out[i] = t.pressure[s];
    if (u.next_pressure) u.next_pressure[s] = u.next_warm ? u.next_warm[i] : 0.0F;
    const SceneDesc& sc = *o.p.scene;
    f3 tx, tv;
    predict_tangent(o.x, xyz(st.velocity[s]), add(xyz(st.non_pressure[s]), acceleration), op.dx, xyz(t.v[s]),
                    xyz(t.non_pressure[s]) + dacceleration, sc.time_step, sc.box, op.k, tx, tv);
    if (!u.last) {
        t.predicted[s] = make_float4(tx.x, tx.y, tx.z, 0.0F);
        return;
    }
    u.out_x.x[i] = tx.x;
    u.out_x.y[i] = tx.y;
    u.out_x.z[i] = tx.z;
    u.out_v.x[i] = tv.x;
    u.out_v.y[i] = tv.y;
    u.out_v.z[i] = tv.z;
}

}  // namespace

cudaError_t launch_tangent_seed(cudaStream_t stream, const SphTangentStep& t, const Field3 x, const Field3 v,
                                const SphParameterTangents& pt) {
    if (t.st.g.count == 0) return cudaSuccess;
    tangent_seed_kernel<<<grid_of(t.st.g.count, 256), 256, 0, stream>>>(t, x, v, pt);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_density_jvp(cudaStream_t stream, const SphTangentStep& t, const uint32_t method, const float* warm,
                               const unsigned block) {
    if (t.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    density_jvp_kernel<<<grid_of(t.st.g.count, b), b, 0, stream>>>(t, method, warm);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_wcsph_force_jvp(cudaStream_t stream, const SphTangentStep& t, const float* pressure, const float4* total,
                                   const Field3 control_tangent, const MutField3 out_x, const MutField3 out_v, const unsigned block) {
    if (t.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    wcsph_force_jvp_kernel<<<grid_of(t.st.g.count, b), b, 0, stream>>>(t, pressure, total, control_tangent, out_x, out_v);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_non_pressure_jvp(cudaStream_t stream, const SphTangentStep& t, const Field3 control_tangent, const int mode,
                                    const MutField3 out_x, const MutField3 out_v, const unsigned block) {
    if (t.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    non_pressure_jvp_kernel<<<grid_of(t.st.g.count, b), b, 0, stream>>>(t, control_tangent, mode, out_x, out_v);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_predicted_density_jvp(cudaStream_t stream, const SphTangentStep& t, const PredictedJvp& u, const unsigned block) {
    if (t.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    predicted_density_jvp_kernel<<<grid_of(t.st.g.count, b), b, 0, stream>>>(t, u);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pressure_jvp(cudaStream_t stream, const SphTangentStep& t, const PressureJvp& u, const unsigned block) {
    if (t.st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    pressure_jvp_kernel<<<grid_of(t.st.g.count, b), b, 0, stream>>>(t, u);
    count_launch();
    return cudaGetLastError();
}

}  // namespace sph
}  // namespace pbf
