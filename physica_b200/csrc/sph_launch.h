// Launcher declarations and argument blocks of the SPH substep kernels (sph.cu).
//
// The SPH family of the reference (sph/sph.ixx:39-372: WCSPH, PCISPH, IISPH, DFSPH) runs on the
// same cell-sorted particles, stencil order and stored neighbour lists as the PBF substep.  The
// grid is built from the input positions at the input step's time (sph/sph.ixx:351) and every
// gather uses the cubic spline kernel (density/device.cuh:26-43, 72-76).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_launch.h"

namespace pbf {
namespace sph {

enum Method : uint32_t { kWcsph = 0, kPcisph = 1, kIisph = 2, kDfsph = 3 };

// Per-scene constants of the SPH kernels, derived on the device from the domain.
struct SphConstants {
    float h;                        // support radius
    float cubic_coefficient;        // 8 / (pi h h h)                        (density/device.cuh:29)
    float cubic_coefficient_2;      // 2 * cubic_coefficient (exact)         (density/device.cuh:32)
    float support_threshold;        // smallest r2 with sqrtf(r2) >= h: the cubic kernels vanish at r2 >= this
    float laplacian_denominator;    // pi h h h h h h                        (density/device.cuh:75)
    float epsilon_factor;           // 0.01 h: the viscosity denominator is r2 + 0.01 h h (sph/wcsph.cu:157, 169)
    float diameter;                 // 2 r                                   (sph/wcsph.cu:467)
    float contact_weight;           // cubic((2 r, 0, 0))                    (sph/wcsph.cu:326)
    float reference_gradient_norm;  // host value of sph/sph.cpp:36-58
    float box_vx, box_vy, box_vz;   // box velocity, written on collision    (sph/common.cu:313-319)
    uint32_t no_slip;
    float skin_bound;               // the predicted density replays the lists while 2 max|x* - x| <= this
    double laplacian_denominator_d; // pi pow(h, 6) in FP64                  (density/device.cuh:87)
    double support_squared_d;       // h h in FP64 (exact): sqrt(r2) >= h exactly when r2 >= this
    double inverse_h_d;             // 1 / h in FP64
    double inverse_hh_d;            // 1 / (h h), h h rounded to float as in density/device.cuh:59-70
    double cubic_coefficient_d;     // 8 / (pi h h h) in FP64                (density/device.cuh:59-70)
    double laplacian_scale_d;       // -45 / (pi pow(h, 6)) in FP64          (density/device.cuh:84-88)
};

// Sorted per-particle parameters of an SPH step, packed by the grid build:
//   params_a = (rest density, viscosity, surface tension, method parameter 0)
//   params_b = (method parameter 1, method parameter 2, 0, 0)
// Method parameters: WCSPH (speed of sound, Tait exponent, boundary surface tension), PCISPH
// (pressure relaxation), IISPH (Jacobi relaxation), DFSPH (divergence relaxation, density relaxation).

// Buffers of one SPH step in sorted order.
struct SphStep {
    GatherCommon g;
    const SphConstants* constants;   // per scene (SceneDesc::constants indexes it)
    const float4* topology;          // (x, mass): positions of the input state
    const float4* velocity;          // (v, 0)
    StoredList list;                 // in-support neighbours of every particle (fluid and boundary)
    const float4* boundary_velocity; // (velocity, 0) of the cell-sorted boundary particles, or null
    float4* aux;                     // (density, viscosity, speed of sound, surface tension)
    float4* non_pressure;            // non-pressure acceleration (iterative methods)
    float4* predicted;               // (predicted position, mass)
    unsigned int* displacement;      // per prediction: max |x* - x| (float bits), zeroed every step
    const uint32_t* sorted_index;
    Field3 controls;                 // external accelerations, original order
};

// Density (cubic) of every particle over its list; WCSPH also evaluates the Tait equation of state
// (sph/wcsph.cu:92-100) and writes pressure / density^2.  `pressure`, `pressure_term`: sorted
// outputs (pressure_term = p / rho^2 of the first pressure pass).  warm: DFSPH's warm-start
// pressures in original order, or null (pressure 0).
cudaError_t launch_density(cudaStream_t stream, const SphStep& st, uint32_t method, float* density_record, float* pressure,
                           float* pressure_term, const float* warm, unsigned block);

// WCSPH forces (pressure, artificial viscosity, surface), external acceleration and integration
// (sph/sph.cpp:214-225) in one pass; writes the next state in original order.
cudaError_t launch_wcsph_forces(cudaStream_t stream, const SphStep& st, const float* pressure_term, MutField3 out_positions,
                                MutField3 out_velocities, float4* record_pressure, float4* record_viscosity,
                                float4* record_surface, float4* record_total, unsigned block);

// Non-pressure acceleration (sph/common.cu:14-47) and, for PCISPH / IISPH, the first prediction
// with the cleared pressure acceleration (sph/sph.cpp:300-303).
//   mode: 0 acceleration only (DFSPH), 1 also the first predicted positions, 2 the prediction is the
//   next state (no pressure iteration), written in original order.
cudaError_t launch_non_pressure(cudaStream_t stream, const SphStep& st, int mode, MutField3 out_positions,
                                MutField3 out_velocities, uint32_t displacement_slot, unsigned block);

// Predicted density at the predicted positions over the full stencil of the input positions
// (density::sph_forward(topology = x, positions = x*)), then the method's pressure update.
//   target: 0 rest density (PCISPH, IISPH, DFSPH density phase), 1 the step's density (DFSPH divergence)
struct PressureUpdate {
    uint32_t method;       // kPcisph, kIisph, kDfsph
    uint32_t relaxation;   // 0: params_a.w, 1: params_b.x
    uint32_t target;       // 0 rest density, 1 density
    uint32_t displacement_slot;   // the prediction this pass evaluates
};
cudaError_t launch_predicted_density(cudaStream_t stream, const SphStep& st, PressureUpdate update, float* pressure,
                                     float* pressure_term, float* predicted_density_record, unsigned block);

// Pressure acceleration (sph/common.cu:165-194) and the next prediction (sph/pcisph.cu:26-45).
//   base: an acceleration added to the pressure acceleration before prediction (DFSPH density
//   phase: the divergence phase's result), or null.
//   last: write the prediction as the next state (original order) and, when `warm_out` is set,
//   the pressures (original order).  store_acceleration: keep the pressure acceleration.
//   next_pressure / next_pressure_term / next_warm: DFSPH's switch to the density phase: load
//   the density phase's warm-start pressures (original order, or null for 0).
struct PressurePassArgs {
    const float* pressure_term;
    const float* pressure;
    const float4* base;
    int last;
    MutField3 out_positions;
    MutField3 out_velocities;
    float* warm_out;
    float4* store_acceleration;
    float* next_pressure;
    float* next_pressure_term;
    const float* next_warm;
    uint32_t displacement_slot;   // where the prediction's max displacement goes (when not last)
};
cudaError_t launch_pressure(cudaStream_t stream, const SphStep& st, const PressurePassArgs& a, unsigned block);

// Constants of every scene (host inputs: support radius, particle radius, box velocity, no-slip
// flag and the reference gradient norm per scene).
struct SphSceneInput {
    float h, particle_radius, reference_gradient_norm;
    float box_vx, box_vy, box_vz;
    uint32_t no_slip;
    float skin;   // list skin as a fraction of h (0: the lists hold the cubic support only)
};
cudaError_t launch_sph_constants(cudaStream_t stream, const SphSceneInput* inputs, uint32_t n, SphConstants* out,
                                 KernelConstants* list_constants);

// ------------------------------------------------------------------ reverse passes (sph_grad.cu)
// Caller-side parameter adjoints, original order (accumulated).  method0..2 follow the packing of
// params_a.w / params_b.x / params_b.y.
struct SphParameterAdjoints {
    double* masses;
    double* rest_densities;
    double* viscosities;
    double* surface_tensions;
    double* method0;
    double* method1;
    double* method2;
};

// integrate_vjp (sph/common.cu:344-366) of WCSPH; also adds the acceleration adjoint to the control's.
cudaError_t launch_integrate_vjp(cudaStream_t stream, const SphStep& st, const float4* total, ConstAdjField3 next_x,
                                 ConstAdjField3 next_v, AdjField3 x, AdjField3 v, AdjField3 control, double4* acceleration);
// surface, viscosity and pressure VJPs of WCSPH with the equation of state's (sph/sph.cpp:245-248);
// writes the density adjoint (sorted).
cudaError_t launch_wcsph_force_vjp(cudaStream_t stream, const SphStep& st, const float* pressure, const double4* acceleration,
                                   AdjField3 x, AdjField3 v, const SphParameterAdjoints& pa, double* density_adjoint, unsigned block);

// density_vjp (density/density.cu:68-99) at the step's positions or at a prediction; for a
// prediction also the reverse of the prediction (predict_vjp, sph/pcisph.cu:67-103).
struct DensityVjpLaunch {
    SphStep st;
    const float4* positions;
    const double* density_adjoint;
    int walk;                       // 0 list, 1 stencil walk, 2 as the forward decided from the displacement slot
    uint32_t displacement_slot;
    AdjField3 x, v;
    SphParameterAdjoints pa;
    int predicted;
    const float4* acceleration;     // the pressure acceleration of the prediction
    const float4* base;             // DFSPH's divergence acceleration, or null
    double4* non_pressure_adjoint;
    double4* acceleration_adjoint;
    double4* base_adjoint;
};
cudaError_t launch_density_vjp(cudaStream_t stream, const DensityVjpLaunch& d, unsigned block);

// The reverse of the last prediction (the next state) of an iterative method.
cudaError_t launch_predict_vjp(cudaStream_t stream, const SphStep& st, const float4* acceleration, const float4* base,
                               ConstAdjField3 next_x, ConstAdjField3 next_v, AdjField3 x, AdjField3 v, double4* non_pressure_adjoint,
                               double4* acceleration_adjoint, double4* base_adjoint, const double* next_warm,
                               double* pressure_adjoint);

// pressure_vjp (sph/common.cu:239-300) of iterate k and, when it has one, the reverse of the
// pressure update that produced it.
struct PressureVjpLaunch {
    SphStep st;
    const float* pressure;
    const double4* acceleration_adjoint;
    double* pressure_adjoint;
    double* density_adjoint;
    AdjField3 x;
    SphParameterAdjoints pa;
    uint32_t method;                // 0: no update (an iteration-0 pressure)
    uint32_t relaxation;
    uint32_t target;
    const float* previous_pressure;
    const float* predicted_density;
    double* previous_pressure_adjoint;
    double* predicted_density_adjoint;
    double* relaxation_adjoint;
    double* warm_adjoint;
};
cudaError_t launch_pressure_vjp(cudaStream_t stream, const PressureVjpLaunch& d, unsigned block);

// non_pressure_vjp (sph/common.cu:98-163).
cudaError_t launch_non_pressure_vjp(cudaStream_t stream, const SphStep& st, const double4* adjoint, AdjField3 x, AdjField3 v,
                                    AdjField3 control, double* density_adjoint, const SphParameterAdjoints& pa, unsigned block);

// DFSPH's switch from the density to the divergence phase in the reverse sweep.
cudaError_t launch_phase_seed(cudaStream_t stream, uint32_t count, const uint32_t* sorted_index, const double4* from,
                              double4* acceleration_adjoint, const double* next_warm, double* pressure_adjoint);

// ------------------------------------------------------------------ tangent passes (sph_grad.cu)
// Caller-side parameter tangents, original order (null: zero), packed like the adjoints.
struct SphParameterTangents {
    const float* masses;
    const float* rest_densities;
    const float* viscosities;
    const float* surface_tensions;
    const float* method0;
    const float* method1;
    const float* method2;
};

// Sorted tangent workspace of one jvp_step.
struct SphTangentStep {
    SphStep st;
    float4* x;            // (dx, dm)
    float4* v;            // (dv, 0)
    float4* params_a;     // tangents of params_a
    float4* params_b;     // tangents of params_b
    float* density;       // d rho
    float* pressure;      // d p of the current phase
    float4* non_pressure; // d a_np
    float4* predicted;    // d x* of the current iterate
};

cudaError_t launch_tangent_seed(cudaStream_t stream, const SphTangentStep& t, Field3 x, Field3 v, const SphParameterTangents& pt);
// density_jvp at the step's positions (density/density.cu:42-66) with WCSPH's EOS tangent
// (sph/wcsph.cu:102-117); warm: DFSPH's divergence warm-start tangent (original order) or null.
cudaError_t launch_density_jvp(cudaStream_t stream, const SphTangentStep& t, uint32_t method, const float* warm, unsigned block);
// WCSPH force tangents (sph/common.cu:196-237, sph/wcsph.cu:176-240, 341-387) and integrate_jvp
// (sph/common.cu:322-342) into the next tangent (original order).
cudaError_t launch_wcsph_force_jvp(cudaStream_t stream, const SphTangentStep& t, const float* pressure, const float4* total,
                                   Field3 control_tangent, MutField3 out_x, MutField3 out_v, unsigned block);
// non_pressure_jvp (sph/common.cu:49-96); mode as launch_non_pressure.
cudaError_t launch_non_pressure_jvp(cudaStream_t stream, const SphTangentStep& t, Field3 control_tangent, int mode,
                                    MutField3 out_x, MutField3 out_v, unsigned block);
struct PredictedJvp {
    uint32_t method, relaxation, target, displacement_slot;
    const float4* predicted;          // x*_k
    const float* predicted_density;   // rho*_k
    const float* previous_pressure;   // p_(k-1)
};
cudaError_t launch_predicted_density_jvp(cudaStream_t stream, const SphTangentStep& t, const PredictedJvp& u, unsigned block);
struct PressureJvp {
    const float* pressure;            // p_k
    const float4* acceleration;       // a_k
    const float4* base;               // DFSPH density phase: the divergence acceleration, or null
    const float4* base_tangent;
    float4* store;                    // keep d a_k (DFSPH divergence phase), or null
    int last;
    MutField3 out_x, out_v;
    float* warm_out;                  // d p_k to the caller (original order), or null
    float* next_pressure;             // DFSPH: the density phase's tangent buffer, loaded with next_warm
    const float* next_warm;
};
cudaError_t launch_pressure_jvp(cudaStream_t stream, const SphTangentStep& t, const PressureJvp& u, unsigned block);

// compute_reference_gradient_norm (sph/sph.cpp:36-58) on the host.
float reference_gradient_norm(float support_radius, float particle_radius);

}  // namespace sph
}  // namespace pbf
