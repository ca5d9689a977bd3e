// Forward substep of the SPH family (WCSPH, PCISPH, IISPH, DFSPH) over cell-sorted particles.
//
// Reference kernels and the fused passes that replace them:
//   density (density/density.cu:18-40, cubic kernel)
//     [+ Tait equation of state (sph/wcsph.cu:92-100) for WCSPH]          -> sph_density_kernel
//   pressure (sph/common.cu:165-194) + artificial viscosity (sph/wcsph.cu:136-174)
//     + surface (sph/wcsph.cu:306-339) + external (sph/wcsph.cu:86-90)
//     + the three adds (sph/common.cu:368-374) + integrate (sph/common.cu:302-320) -> wcsph_force_kernel
//   non-pressure (sph/common.cu:14-47) [+ the first prediction with zero
//     pressure acceleration (sph/pcisph.cu:26-45)]                         -> non_pressure_kernel
//   predicted density (density::sph_forward at x*, topology x)
//     + pressure update (sph/pcisph.cu:104-110, sph/iisph.cu:104-110,
//       sph/dfsph.cu:104-110)                                             -> predicted_density_kernel
//   pressure (sph/common.cu:165-194) [+ DFSPH's add (sph/common.cu:368-374)]
//     + predict / integrate (sph/pcisph.cu:26-45)                         -> pressure_kernel
//
// Each per-particle sum runs over the particle's stored list (gather.cuh) in the reference's
// stencil order with the reference's per-pair expressions, so it equals the reference's sum bit
// for bit: a candidate outside the cubic support contributes an exact zero there.  The
// predicted density is evaluated at predicted positions whose distances differ from the list's,
// so that pass walks the full stencil of the input positions, as the reference does.
#include <cmath>

#include "sph_math.cuh"

namespace pbf {
namespace sph {

namespace {

using namespace gather_detail;
using namespace detail;

// Resident 128-thread blocks per SM the register budgets of the list-replay passes are sized for
// (compile-time tuning knobs; 0 leaves the register count to the compiler).  The density passes'
// per-entry work is a few multiply-adds, so they wait on their neighbours' loads and gain from
// more resident warps even with a few spills.  At 1M particles, ms per substep WCSPH / PCISPH /
// DFSPH on one box: the compiler's registers (the force pass bounded to 4 blocks) 0.89 / 2.43 /
// 3.85; these budgets 0.71 / 2.32 / 3.68.  Also measured, each against its neighbours in a sweep:
// density at 12 (40 registers) or 20 (24) slower than at 14 (32); pressure at 12 (40) slower than
// at 10 (48); the non-pressure pass at 8 (64 instead of 72) no change; the force pass at 7 (72,
// spilling) slower than at 6 (80, 24 resident warps instead of 20 at 88).
#ifndef PBF_SPH_DENSITY_MIN_BLOCKS
#define PBF_SPH_DENSITY_MIN_BLOCKS 14
#endif
#ifndef PBF_SPH_NON_PRESSURE_MIN_BLOCKS
#define PBF_SPH_NON_PRESSURE_MIN_BLOCKS 0
#endif
#ifndef PBF_SPH_PRESSURE_MIN_BLOCKS
#define PBF_SPH_PRESSURE_MIN_BLOCKS 10
#endif
#ifndef PBF_WCSPH_FORCE_MIN_BLOCKS
#define PBF_WCSPH_FORCE_MIN_BLOCKS 6
#endif

// ------------------------------------------------------------------ density (+ Tait EOS)
template <bool WithBoundary>
struct DensityOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    f3 x;
    float rest_density;
    SphConstants k;
    float density;

    __device__ __forceinline__ float4 prefetch(const uint32_t t) const {
        if constexpr (WithBoundary) return (t & kBoundaryBit) ? boundary[t & ~kBoundaryBit] : pos[t];
        return pos[t];
    }
    __device__ __forceinline__ void apply(const uint32_t t, const float4 q) {
        const float distance = __fsqrt_rn(sq_xfirst(sub(x, xyz(q))));
        if (distance >= k.h) return;
        const float w = cubic_inside(distance, k);
        // fluid: density += m_j W; boundary: density += rho0_i V_b W (density/density.cu:30-37)
        if (WithBoundary && (t & kBoundaryBit)) density = __fmaf_rn(__fmul_rn(rest_density, q.w), w, density);
        else density = __fmaf_rn(q.w, w, density);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

template <bool WithBoundary>
__global__ void __launch_bounds__(kBlock, PBF_SPH_DENSITY_MIN_BLOCKS) sph_density_kernel(const SphStep st, const uint32_t method, float* density_record,
                                                             float* pressure, float* pressure_term, const float* warm) {
    const Own o = own(st);
    if (!o.p.active) return;
    DensityOp<WithBoundary> op;
    op.pos = st.topology;
    op.boundary = st.g.boundary;
    op.x = o.x;
    op.rest_density = o.pa.x;
    op.k = *o.k;
    op.density = 0.0F;
    replay(op, o.p, st.g, st.list);
    const float rho = op.density;
    const float4 pb = st.g.params_b[o.p.s];
    float p = 0.0F;
    if (method == kWcsph) {
        // p = rho0 c c ((rho / rho0)^gamma - 1) / gamma (sph/wcsph.cu:92-100)
        const float rest = o.pa.x, speed = o.pa.w, exponent = pb.x;
        const float ratio = __fdiv_rn(rho, rest);
        p = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(rest, speed), speed), __fsub_rn(powf(ratio, exponent), 1.0F)), exponent);
        st.aux[o.p.s] = make_float4(rho, o.pa.y, speed, o.pa.z);
    } else {
        st.aux[o.p.s] = make_float4(rho, o.pa.y, 0.0F, 0.0F);
        if (warm) p = warm[st.sorted_index[o.p.s]];
    }
    if (density_record) density_record[o.p.s] = rho;
    if (pressure) pressure[o.p.s] = p;
    if (pressure_term) pressure_term[o.p.s] = __fdiv_rn(p, __fmul_rn(rho, rho));
}

// ------------------------------------------------------------------ WCSPH forces + integrate
struct ForceData {
    float4 q;    // (x, m) or boundary (x, V)
    float4 v;    // (v, -)
    float4 aux;  // (rho, viscosity, speed of sound, -)
    float pt;    // p / rho^2
};

template <bool WithBoundary>
struct WcsphForceOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    const float4* __restrict__ aux;
    const float* __restrict__ pt;
    const float4* __restrict__ boundary;
    const float4* __restrict__ boundary_velocity;
    uint32_t self;
    f3 x, v;
    float mass, rest, density, viscosity, speed, first_term, surface_tension, boundary_tension;
    float boundary_nu;   // viscosity_i h c_i / rho_i (sph/wcsph.cu:167)
    SphConstants k;
    f3 pressure, artificial, surface;

    __device__ __forceinline__ ForceData prefetch(const uint32_t t) const {
        ForceData d;
        if (WithBoundary && (t & kBoundaryBit)) {
            d.q = boundary[t & ~kBoundaryBit];
            d.v = boundary_velocity[t & ~kBoundaryBit];
            d.aux = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
            d.pt = 0.0F;
            return d;
        }
        d.q = pos[t];
        d.v = vel[t];
        d.aux = aux[t];
        d.pt = pt[t];
        return d;
    }
    __device__ __forceinline__ void apply(const uint32_t t, const ForceData& d) {
        const bool is_boundary = WithBoundary && (t & kBoundaryBit);
        if (!is_boundary && t == self) return;
        const f3 disp = sub(x, xyz(d.q));
        const float r2 = sq_xfirst(disp);
        const float distance = __fsqrt_rn(r2);
        if (distance >= k.h) return;
        const bool has_gradient = distance != 0.0F;
        const float s = has_gradient ? cubic_gradient_scale(distance, k) : 0.0F;
        const f3 gradient = scale(disp, s);
        const f3 dv = sub(v, xyz(d.v));
        const float compression = dot_xfirst(dv, disp);
        const float weight = distance > k.diameter ? cubic_inside(distance, k) : k.contact_weight;
        if (is_boundary) {
            const float volume = d.q.w;
            const float rv = __fmul_rn(-rest, volume);
            // pressure: -rho0_i V_b p_i / rho_i^2 grad W (sph/common.cu:183-188)
            if (has_gradient) pressure = fma3(__fmul_rn(rv, first_term), gradient, pressure);
            // artificial viscosity against the boundary (sph/wcsph.cu:162-172)
            if (has_gradient && compression < 0.0F) {
                const float pi = __fdiv_rn(__fmul_rn(-boundary_nu, compression), __fmaf_rn(k.epsilon_factor, k.h, r2));
                artificial = fma3(__fmul_rn(rv, pi), gradient, artificial);
            }
            // boundary adhesion (sph/wcsph.cu:327-335)
            const float factor =
                __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(-boundary_tension, rest), volume), weight), mass);
            surface = fma3(factor, disp, surface);
            return;
        }
        const float mj = d.q.w;
        if (has_gradient) {
            // -m_j (p_i / rho_i^2 + p_j / rho_j^2) grad W (sph/common.cu:180-181)
            pressure = fma3(__fmul_rn(-mj, __fadd_rn(first_term, d.pt)), gradient, pressure);
            if (compression < 0.0F) {
                // Monaghan viscosity (sph/wcsph.cu:149-158)
                const float alpha = __fmul_rn(0.5F, __fadd_rn(viscosity, d.aux.y));
                const float c = __fmul_rn(0.5F, __fadd_rn(speed, d.aux.z));
                const float nu =
                    __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(2.0F, alpha), k.h), c), __fadd_rn(density, d.aux.x));
                // r2 + 0.01 h h with the last product fused into the sum
                const float pi = __fdiv_rn(__fmul_rn(-nu, compression), __fmaf_rn(k.epsilon_factor, k.h, r2));
                artificial = fma3(__fmul_rn(-mj, pi), gradient, artificial);
            }
        }
        // cohesion (sph/wcsph.cu:318-325)
        const float factor = __fdiv_rn(__fmul_rn(__fmul_rn(-surface_tension, mj), weight), mass);
        surface = fma3(factor, disp, surface);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

struct WcsphForceArgs {
    SphStep st;
    const float* pressure_term;
    MutField3 out_positions;
    MutField3 out_velocities;
    float4* record_pressure;
    float4* record_viscosity;
    float4* record_surface;
    float4* record_total;   // the total acceleration (differentiable mode), or null
};

template <bool WithBoundary>
__global__ void __launch_bounds__(kBlock, PBF_WCSPH_FORCE_MIN_BLOCKS) wcsph_force_kernel(const WcsphForceArgs a) {
    const SphStep& st = a.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    WcsphForceOp<WithBoundary> op;
    op.pos = st.topology;
    op.vel = st.velocity;
    op.aux = st.aux;
    op.pt = a.pressure_term;
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
    op.first_term = a.pressure_term[s];
    op.surface_tension = o.pa.z;
    op.boundary_tension = pb.y;
    op.k = *o.k;
    op.boundary_nu = __fdiv_rn(__fmul_rn(__fmul_rn(op.viscosity, op.k.h), op.speed), op.density);
    op.pressure = op.artificial = op.surface = mk(0.0F, 0.0F, 0.0F);
    replay(op, o.p, st.g, st.list);
    // total = (pressure + viscosity) + surface + (gravity + control) (sph/sph.cpp:219-222)
    const uint32_t i = st.sorted_index[s];
    const SceneDesc& sc = *o.p.scene;
    const f3 external = add(mk(sc.gravity_x, sc.gravity_y, sc.gravity_z), mk(st.controls.x[i], st.controls.y[i], st.controls.z[i]));
    const f3 total = add(add(add(op.pressure, op.artificial), op.surface), external);
    f3 xo, vo;
    predict(o.x, op.v, total, sc.time_step, sc.box, op.k, xo, vo);
    a.out_positions.x[i] = xo.x;
    a.out_positions.y[i] = xo.y;
    a.out_positions.z[i] = xo.z;
    a.out_velocities.x[i] = vo.x;
    a.out_velocities.y[i] = vo.y;
    a.out_velocities.z[i] = vo.z;
    if (a.record_pressure) a.record_pressure[s] = make_float4(op.pressure.x, op.pressure.y, op.pressure.z, 0.0F);
    if (a.record_viscosity) a.record_viscosity[s] = make_float4(op.artificial.x, op.artificial.y, op.artificial.z, 0.0F);
    if (a.record_surface) a.record_surface[s] = make_float4(op.surface.x, op.surface.y, op.surface.z, 0.0F);
    if (a.record_total) a.record_total[s] = make_float4(total.x, total.y, total.z, 0.0F);
}

// ------------------------------------------------------------------ non-pressure acceleration
struct ViscosityData {
    float4 q;
    float4 v;
    float4 aux;
};

template <bool WithBoundary>
struct NonPressureOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    const float4* __restrict__ aux;
    const float4* __restrict__ boundary;
    const float4* __restrict__ boundary_velocity;
    uint32_t self;
    f3 x, v;
    float viscosity;
    SphConstants k;
    f3 acceleration;

    __device__ __forceinline__ ViscosityData prefetch(const uint32_t t) const {
        ViscosityData d;
        if (WithBoundary && (t & kBoundaryBit)) {
            d.q = boundary[t & ~kBoundaryBit];
            d.v = boundary_velocity[t & ~kBoundaryBit];
            d.aux = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
            return d;
        }
        d.q = pos[t];
        d.v = vel[t];
        d.aux = aux[t];
        return d;
    }
    __device__ __forceinline__ void apply(const uint32_t t, const ViscosityData& d) {
        const bool is_boundary = WithBoundary && (t & kBoundaryBit);
        if (!is_boundary && t == self) return;
        const float distance = __fsqrt_rn(sq_xfirst(sub(x, xyz(d.q))));
        if (distance >= k.h) return;
        const float laplacian = laplacian_inside(distance, k);
        const f3 dv = sub(xyz(d.v), v);
        if (is_boundary) {
            // viscosity_i V_b lap W (v_b - v_i) (sph/common.cu:38-43)
            acceleration = fma3(__fmul_rn(__fmul_rn(viscosity, d.q.w), laplacian), dv, acceleration);
            return;
        }
        // 0.5 (mu_i + mu_j) m_j lap W / rho_j (v_j - v_i) (sph/common.cu:31-35)
        const float mu = __fmul_rn(0.5F, __fadd_rn(viscosity, d.aux.y));
        const float weight = __fdiv_rn(__fmul_rn(__fmul_rn(mu, d.q.w), laplacian), d.aux.x);
        acceleration = fma3(weight, dv, acceleration);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

template <bool WithBoundary>
__global__ void __launch_bounds__(kBlock, PBF_SPH_NON_PRESSURE_MIN_BLOCKS) non_pressure_kernel(const SphStep st, const int mode, const MutField3 out_positions,
                                                              const MutField3 out_velocities, const uint32_t displacement_slot) {
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    const uint32_t i = st.sorted_index[s];
    const SceneDesc& sc = *o.p.scene;
    NonPressureOp<WithBoundary> op;
    op.pos = st.topology;
    op.vel = st.velocity;
    op.aux = st.aux;
    op.boundary = st.g.boundary;
    op.boundary_velocity = st.boundary_velocity;
    op.self = s;
    op.x = o.x;
    op.v = xyz(st.velocity[s]);
    op.viscosity = o.pa.y;
    op.k = *o.k;
    // starts from gravity + control (sph/common.cu:19)
    op.acceleration = add(mk(sc.gravity_x, sc.gravity_y, sc.gravity_z), mk(st.controls.x[i], st.controls.y[i], st.controls.z[i]));
    replay(op, o.p, st.g, st.list);
    st.non_pressure[s] = make_float4(op.acceleration.x, op.acceleration.y, op.acceleration.z, 0.0F);
    if (mode == 0) return;
    // prediction with the cleared pressure acceleration (sph/sph.cpp:298-303)
    f3 xo, vo;
    predict(o.x, op.v, add(op.acceleration, mk(0.0F, 0.0F, 0.0F)), sc.time_step, sc.box, op.k, xo, vo);
    if (mode == 1) {
        st.predicted[s] = make_float4(xo.x, xo.y, xo.z, o.mass);
        record_displacement(st.displacement + displacement_slot, xo, o.x);
        return;
    }
    out_positions.x[i] = xo.x;
    out_positions.y[i] = xo.y;
    out_positions.z[i] = xo.z;
    out_velocities.x[i] = vo.x;
    out_velocities.y[i] = vo.y;
    out_velocities.z[i] = vo.z;
}

// ------------------------------------------------------------------ predicted density + pressure update
template <bool WithBoundary>
struct PredictedDensityOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ predicted;
    const float4* __restrict__ boundary;
    f3 x;
    float rest_density;
    SphConstants k;
    float density;

    __device__ __forceinline__ float4 prefetch(const uint32_t t) const {
        if (WithBoundary && (t & kBoundaryBit)) return boundary[t & ~kBoundaryBit];
        return predicted[t];
    }
    __device__ __forceinline__ void apply(const uint32_t t, const float4 q) {
        const bool is_boundary = WithBoundary && (t & kBoundaryBit);
        const float distance = __fsqrt_rn(sq_xfirst(sub(x, xyz(q))));
        if (distance >= k.h) return;
        const float w = cubic_inside(distance, k);
        if (is_boundary) density = __fmaf_rn(__fmul_rn(rest_density, q.w), w, density);
        else density = __fmaf_rn(q.w, w, density);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};


template <bool WithBoundary>
__global__ void __launch_bounds__(kBlock, PBF_SPH_DENSITY_MIN_BLOCKS) predicted_density_kernel(const SphStep st, const PressureUpdate update,
                                                                   float* pressure, float* pressure_term, float* record) {
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    PredictedDensityOp<WithBoundary> op;
    op.predicted = st.predicted;
    op.boundary = st.g.boundary;
    op.x = xyz(st.predicted[s]);
    op.rest_density = o.pa.x;
    op.k = *o.k;
    op.density = 0.0F;
    // Every pair within h at the predicted positions lies within h + 2 max|x* - x| at the input
    // positions; when that is inside the list's skin, the list holds all of them in stencil order.
    const float displacement = __uint_as_float(st.displacement[update.displacement_slot]);
    if (__fmul_rn(2.0F, displacement) <= o.k->skin_bound) replay(op, o.p, st.g, st.list);
    else walk(op, o.p, st.g);
    const float predicted_density = op.density;
    if (record) record[s] = predicted_density;
    const float rho = st.aux[s].x;
    const float rest = o.pa.x;
    const float relaxation = update.relaxation == 0u ? o.pa.w : st.g.params_b[s].x;
    // PCISPH uses the rest volume m / rho0 (sph/pcisph.cu:107), IISPH and DFSPH m / rho (sph/iisph.cu:107)
    const float volume = __fdiv_rn(o.mass, update.method == kPcisph ? rest : rho);
    const float dt = o.p.scene->time_step;
    const float delta = __fdiv_rn(1.0F, __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(2.0F, dt), dt), volume), volume),
                                                  o.k->reference_gradient_norm));
    const float target = update.target == 1u ? rho : rest;
    const float p = fmaxf(0.0F, __fmaf_rn(__fmul_rn(relaxation, delta), __fsub_rn(predicted_density, target), pressure[s]));
    pressure[s] = p;
    pressure_term[s] = __fdiv_rn(p, __fmul_rn(rho, rho));
}

// ------------------------------------------------------------------ pressure acceleration + predict
template <bool WithBoundary>
struct PressureOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ pos;
    const float* __restrict__ pt;
    const float4* __restrict__ boundary;
    uint32_t self;
    f3 x;
    float rest, first_term;
    SphConstants k;
    f3 acceleration;

    struct Data {
        float4 q;   // (x, m) or boundary (x, V)
        float pt;   // p_j / rho_j^2
    };
    __device__ __forceinline__ Data prefetch(const uint32_t t) const {
        if (WithBoundary && (t & kBoundaryBit)) return {boundary[t & ~kBoundaryBit], 0.0F};
        return {pos[t], pt[t]};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const Data& d) {
        const bool is_boundary = WithBoundary && (t & kBoundaryBit);
        if (!is_boundary && t == self) return;
        const f3 disp = sub(x, xyz(d.q));
        const float distance = __fsqrt_rn(sq_xfirst(disp));
        if (distance == 0.0F || distance >= k.h) return;
        const f3 gradient = scale(disp, cubic_gradient_scale(distance, k));
        // boundary: -rho0_i V_b p_i / rho_i^2 grad W; fluid: -m_j (p_i / rho_i^2 + p_j / rho_j^2) grad W
        // (sph/common.cu:180-188)
        const float factor = is_boundary ? __fmul_rn(__fmul_rn(-rest, d.q.w), first_term)
                                         : __fmul_rn(-d.q.w, __fadd_rn(first_term, d.pt));
        acceleration = fma3(factor, gradient, acceleration);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

struct PressureKernelArgs {
    SphStep st;
    PressurePassArgs p;
};

template <bool WithBoundary>
__global__ void __launch_bounds__(kBlock, PBF_SPH_PRESSURE_MIN_BLOCKS) pressure_kernel(const PressureKernelArgs a) {
    const SphStep& st = a.st;
    const Own o = own(st);
    if (!o.p.active) return;
    const uint32_t s = o.p.s;
    PressureOp<WithBoundary> op;
    op.pos = st.topology;
    op.pt = a.p.pressure_term;
    op.boundary = st.g.boundary;
    op.self = s;
    op.x = o.x;
    op.rest = o.pa.x;
    op.first_term = a.p.pressure_term[s];
    op.k = *o.k;
    op.acceleration = mk(0.0F, 0.0F, 0.0F);
    replay(op, o.p, st.g, st.list);
    const f3 pressure_acceleration = op.acceleration;
    if (a.p.store_acceleration)
        a.p.store_acceleration[s] = make_float4(pressure_acceleration.x, pressure_acceleration.y, pressure_acceleration.z, 0.0F);
    // DFSPH's density phase predicts with divergence + density pressure accelerations (sph/sph.cpp:596)
    f3 total = pressure_acceleration;
    if (a.p.base) total = add(xyz(a.p.base[s]), pressure_acceleration);
    const float4 np = st.non_pressure[s];
    const SceneDesc& sc = *o.p.scene;
    f3 xo, vo;
    predict(o.x, xyz(st.velocity[s]), add(xyz(np), total), sc.time_step, sc.box, op.k, xo, vo);
    const uint32_t i = st.sorted_index[s];
    if (a.p.warm_out) a.p.warm_out[i] = a.p.pressure[s];
    if (a.p.next_pressure) {
        const float p = a.p.next_warm ? a.p.next_warm[i] : 0.0F;
        const float rho = st.aux[s].x;
        a.p.next_pressure[s] = p;
        a.p.next_pressure_term[s] = __fdiv_rn(p, __fmul_rn(rho, rho));
    }
    if (!a.p.last) {
        st.predicted[s] = make_float4(xo.x, xo.y, xo.z, o.mass);
        record_displacement(st.displacement + a.p.displacement_slot, xo, o.x);
        return;
    }
    a.p.out_positions.x[i] = xo.x;
    a.p.out_positions.y[i] = xo.y;
    a.p.out_positions.z[i] = xo.z;
    a.p.out_velocities.x[i] = vo.x;
    a.p.out_velocities.y[i] = vo.y;
    a.p.out_velocities.z[i] = vo.z;
}

// ------------------------------------------------------------------ constants
__global__ void sph_constants_kernel(const SphSceneInput* __restrict__ inputs, const uint32_t n, SphConstants* __restrict__ out,
                                     KernelConstants* __restrict__ list_constants) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SphSceneInput in = inputs[i];
    const float h = in.h;
    SphConstants k;
    k.h = h;
    k.cubic_coefficient = __fdiv_rn(8.0F, __fmul_rn(__fmul_rn(__fmul_rn(kPi, h), h), h));
    k.cubic_coefficient_2 = __fmul_rn(k.cubic_coefficient, 2.0F);
    // smallest float r2 with sqrtf(r2) >= h; sqrtf is monotone, so bisect on the bit pattern
    uint32_t lo = 0u, hi = 0x7f800000u;
    while (hi - lo > 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (__fsqrt_rn(__uint_as_float(mid)) >= h) hi = mid;
        else lo = mid;
    }
    k.support_threshold = __uint_as_float(hi);
    k.laplacian_denominator = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(kPi, h), h), h), h), h), h);
    k.laplacian_denominator_d = static_cast<double>(kPi) * pow(static_cast<double>(h), 6.0);
    k.support_squared_d = static_cast<double>(h) * static_cast<double>(h);
    k.inverse_h_d = 1.0 / static_cast<double>(h);
    k.inverse_hh_d = 1.0 / static_cast<double>(__fmul_rn(h, h));
    k.cubic_coefficient_d = 8.0 / (static_cast<double>(kPi) * h * h * h);
    k.laplacian_scale_d = -45.0 / k.laplacian_denominator_d;
    k.epsilon_factor = __fmul_rn(0.01F, h);
    k.diameter = __fmul_rn(2.0F, in.particle_radius);
    // cubic({diameter, 0, 0}): its length is sqrtf(fma(0, 0, fma(d, d, 0 * 0)))
    const float contact = __fsqrt_rn(sq_xfirst(mk(k.diameter, 0.0F, 0.0F)));
    k.contact_weight = contact >= h ? 0.0F : cubic_inside(contact, k);
    k.reference_gradient_norm = in.reference_gradient_norm;
    // Skin of the stored lists: they hold the pairs with sqrtf(r2) < h + skin; the predicted
    // density replays them while 2 max|x* - x| <= skin_bound, a bound kept 0.1% inside the skin
    // for the roundings of the distances involved.
    const float skin = __fmul_rn(in.skin, h);
    k.skin_bound = __fmul_rn(skin, 0.999F);
    k.box_vx = in.box_vx;
    k.box_vy = in.box_vy;
    k.box_vz = in.box_vz;
    k.no_slip = in.no_slip;
    out[i] = k;
    // The list lists every candidate whose squared distance, in any of the passes' roundings, can
    // fall below the support threshold: a few ulps of margin above it.
    KernelConstants& lc = list_constants[i];
    if (in.skin > 0.0F) {
        const float outer = __fadd_ru(h, skin);
        lc.list_threshold = __uint_as_float(__float_as_uint(__fmul_ru(outer, outer)) + 8u);
    } else {
        lc.list_threshold = __uint_as_float(hi + 8u);
    }
}

inline unsigned grid_of(const uint32_t n, const unsigned block) { return (n + block - 1u) / block; }

unsigned block_of(const unsigned block) {
    return block >= 32u && block <= static_cast<unsigned>(kBlock) && block % 32u == 0u ? block : static_cast<unsigned>(kBlock);
}

}  // namespace

cudaError_t launch_sph_constants(cudaStream_t stream, const SphSceneInput* inputs, const uint32_t n, SphConstants* out,
                                 KernelConstants* list_constants) {
    sph_constants_kernel<<<grid_of(n, 64), 64, 0, stream>>>(inputs, n, out, list_constants);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_density(cudaStream_t stream, const SphStep& st, const uint32_t method, float* density_record, float* pressure,
                           float* pressure_term, const float* warm, const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    if (st.g.boundary)
        sph_density_kernel<true><<<grid_of(st.g.count, b), b, 0, stream>>>(st, method, density_record, pressure, pressure_term, warm);
    else
        sph_density_kernel<false><<<grid_of(st.g.count, b), b, 0, stream>>>(st, method, density_record, pressure, pressure_term, warm);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_wcsph_forces(cudaStream_t stream, const SphStep& st, const float* pressure_term, const MutField3 out_positions,
                                const MutField3 out_velocities, float4* record_pressure, float4* record_viscosity,
                                float4* record_surface, float4* record_total, const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    const WcsphForceArgs a{st, pressure_term, out_positions, out_velocities, record_pressure, record_viscosity, record_surface,
                           record_total};
    if (st.g.boundary) wcsph_force_kernel<true><<<grid_of(st.g.count, b), b, 0, stream>>>(a);
    else wcsph_force_kernel<false><<<grid_of(st.g.count, b), b, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_non_pressure(cudaStream_t stream, const SphStep& st, const int mode, const MutField3 out_positions,
                                const MutField3 out_velocities, const uint32_t displacement_slot, const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    if (st.g.boundary)
        non_pressure_kernel<true><<<grid_of(st.g.count, b), b, 0, stream>>>(st, mode, out_positions, out_velocities,
                                                                           displacement_slot);
    else
        non_pressure_kernel<false><<<grid_of(st.g.count, b), b, 0, stream>>>(st, mode, out_positions, out_velocities,
                                                                            displacement_slot);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_predicted_density(cudaStream_t stream, const SphStep& st, const PressureUpdate update, float* pressure,
                                     float* pressure_term, float* record, const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    if (st.g.boundary)
        predicted_density_kernel<true><<<grid_of(st.g.count, b), b, 0, stream>>>(st, update, pressure, pressure_term, record);
    else
        predicted_density_kernel<false><<<grid_of(st.g.count, b), b, 0, stream>>>(st, update, pressure, pressure_term, record);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pressure(cudaStream_t stream, const SphStep& st, const PressurePassArgs& p, const unsigned block) {
    if (st.g.count == 0) return cudaSuccess;
    const unsigned b = block_of(block);
    const PressureKernelArgs a{st, p};
    if (st.g.boundary) pressure_kernel<true><<<grid_of(st.g.count, b), b, 0, stream>>>(a);
    else pressure_kernel<false><<<grid_of(st.g.count, b), b, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

// compute_reference_gradient_norm (sph/sph.cpp:36-58): the squared norm of the summed cubic
// gradient plus the sum of squared gradients over a lattice of spacing 2 r inside the support,
// evaluated in float in the reference's loop order (the lattice coordinates are accumulated).  The
// host compiler is told not to contract products into sums (-ffp-contract=off), as the
// reference's host build on x86-64 has no fused multiply-add.
float reference_gradient_norm(const float support_radius, const float particle_radius) {
    const float diameter = 2.0F * particle_radius;
    const float coefficient = 8.0F / (kPi * support_radius * support_radius * support_radius);
    float sum_x = 0.0F, sum_y = 0.0F, sum_z = 0.0F, sum_squares = 0.0F;
    for (float x = -support_radius; x <= support_radius; x += diameter) {
        for (float y = -support_radius; y <= support_radius; y += diameter) {
            for (float z = -support_radius; z <= support_radius; z += diameter) {
                const float r2 = x * x + y * y + z * z;
                const float distance = std::sqrt(r2);
                if (distance == 0.0F || distance >= support_radius) continue;
                const float q = distance / support_radius;
                const float derivative = q <= 0.5F ? 18.0F * q * q - 12.0F * q : -6.0F * (1.0F - q) * (1.0F - q);
                const float s = coefficient * derivative / (support_radius * distance);
                sum_x += s * x;
                sum_y += s * y;
                sum_z += s * z;
                sum_squares += s * s * r2;
            }
        }
    }
    return sum_x * sum_x + sum_y * sum_y + sum_z * sum_z + sum_squares;
}

}  // namespace sph
}  // namespace pbf
