/*
 * physica_sph.h -- C ABI of the B200 SPH solvers (WCSPH, PCISPH, IISPH, DFSPH).
 *
 * Drop-in boundary for the forward substep of the SPH family of Xayah-Graphics/physica's
 * fluids/liquid/particle module: SPH<Method> (sph/sph.ixx:273-372) with Method one of WCSPH
 * (sph/sph.ixx:39-101), PCISPH (sph/sph.ixx:103-147), IISPH (sph/sph.ixx:149-193) and DFSPH
 * (sph/sph.ixx:195-268).  The reference file:line each entry point replaces is given beside it.
 *
 * The conventions of physica_pbf.h hold: device SoA field pointers owned by the caller, calls
 * asynchronous on the solver's stream, pbf_status returns with pbf_last_error() for the message.
 * The domain description is the PBF one (pbf_domain_configuration: the reference's
 * DomainConfiguration is shared by both families, domain/domain.ixx:12-165).
 *
 * Differentiable mode (PBF_EXECUTION_DIFFERENTIABLE) adds SPH<Method>::jvp_step and ::vjp_step
 * (sph/sph.ixx:356-365): FP32 tangents, and FP64 adjoints accumulated like the PBF ones.
 */
#ifndef PHYSICA_SPH_H
#define PHYSICA_SPH_H

#include "physica_pbf.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* The Method template argument of SPH<Method> (sph/sph.ixx:270-271). */
typedef enum {
    SPH_METHOD_WCSPH = 0,
    SPH_METHOD_PCISPH = 1,
    SPH_METHOD_IISPH = 2,
    SPH_METHOD_DFSPH = 3
} sph_method;

/* Method::Configuration (sph/sph.ixx:40, 104-107, 150-153, 196-201). */
typedef struct {
    sph_method method;
    uint32_t pressure_iterations;     /* PCISPH, IISPH; reference default 6 */
    uint32_t divergence_iterations;   /* DFSPH; reference default 4 */
    uint32_t density_iterations;      /* DFSPH; reference default 6 */
    uint32_t checkpoint_interval;     /* reference default 2; forward mode keeps no checkpoints */
    uint32_t pressure_warm_start;     /* DFSPH; reference default 1 */
} sph_configuration;

/* SPH<Method>::Parameters (sph/sph.ixx:287-290): ParticleParameters (domain/domain.ixx) and
 * Method::Parameters (sph/sph.ixx:45-49, 111, 157, 214-217).  Pointers of the other methods may
 * be NULL. */
typedef struct {
    const float* masses;
    const float* rest_densities;
    const float* viscosities;
    const float* surface_tensions;
    const float* speed_of_sound;             /* WCSPH */
    const float* tait_exponent;              /* WCSPH */
    const float* boundary_surface_tension;   /* WCSPH */
    const float* pressure_relaxation;        /* PCISPH */
    const float* jacobi_relaxation;          /* IISPH */
    const float* divergence_relaxation;      /* DFSPH */
    const float* density_relaxation;         /* DFSPH */
} sph_parameters;

/* Method::State (sph/sph.ixx:202-205, 41, 108, 154): DFSPH's warm-start pressures (original particle order);
 * the other methods have an empty state and ignore it (it may be NULL). */
typedef struct {
    float* warm_divergence_pressure;
    float* warm_density_pressure;
} sph_method_state;

/* SPH<Method>::ParameterAdjoint (sph/sph.ixx:295-298): FP64, one array per parameter, ACCUMULATED.
 * Arrays of the other methods may be NULL. */
typedef struct {
    double* masses;
    double* rest_densities;
    double* viscosities;
    double* surface_tensions;
    double* speed_of_sound;             /* WCSPH */
    double* tait_exponent;              /* WCSPH */
    double* boundary_surface_tension;   /* WCSPH */
    double* pressure_relaxation;        /* PCISPH */
    double* jacobi_relaxation;          /* IISPH */
    double* divergence_relaxation;      /* DFSPH */
    double* density_relaxation;         /* DFSPH */
} sph_parameter_adjoint;

/* Method::StateAdjoint (sph/sph.ixx:210-213): DFSPH's warm-start pressure adjoints (FP64). */
typedef struct {
    double* warm_divergence_pressure;
    double* warm_density_pressure;
} sph_method_state_adjoint;

typedef struct sph_solver sph_solver;           /* SPH<Method> (sph/sph.ixx:273-372) */
typedef struct sph_step_cache sph_step_cache;   /* SPH<Method>::StepCache (sph/sph.ixx:299-303) */

/* Fields of the last forward step, exported in original particle order. */
typedef enum {
    SPH_CACHE_DENSITIES = 0,                /* N: StepCache::densities */
    SPH_CACHE_PRESSURES = 1,                /* N: WCSPH Cache::pressures; iterative: the last iterate's pressures */
    SPH_CACHE_PRESSURE_ACCELERATIONS = 2,   /* 3N: WCSPH Cache::pressure_accelerations; iterative: the last pressure pass */
    SPH_CACHE_VISCOSITY_ACCELERATIONS = 3,  /* 3N: WCSPH Cache::viscosity_accelerations; iterative: non_pressure_accelerations */
    SPH_CACHE_SURFACE_ACCELERATIONS = 4,    /* 3N: WCSPH Cache::surface_accelerations */
    SPH_CACHE_PREDICTED_DENSITIES = 5       /* N: iterative methods, the last iterate's predicted densities */
} sph_cache_field;

/* SPH<Method>::SPH(domain_configuration, method_configuration, mode, stream) (sph/sph.ixx:309-312).
 * cuda_stream: the cudaStream_t every call of the solver runs on (NULL: the default stream). */
int sph_create(const pbf_domain_configuration* domain, const sph_configuration* configuration, pbf_execution_mode mode,
               void* cuda_stream, sph_solver** solver);
int sph_destroy(sph_solver* solver);

/* SPH<Method>::allocate_step_cache (sph/sph.ixx:322) */
int sph_allocate_step_cache(sph_solver* solver, sph_step_cache** cache);
int sph_free_step_cache(sph_solver* solver, sph_step_cache* cache);

/* SPH<Method>::forward_step (sph/sph.ixx:350-354): neighbourhood at the input positions, density,
 * then Method::forward (sph/sph.cpp:214-225, 296-312, 409-425, 572-610).  method_state /
 * next_method_state: DFSPH's warm-start pressures (read / written), else ignored. */
int sph_forward_step(sph_solver* solver, const pbf_particle_state* state, const sph_method_state* method_state,
                     const pbf_control* control, const sph_parameters* parameters, pbf_particle_state* next_state,
                     sph_method_state* next_method_state, sph_step_cache* cache);

/* SPH<Method>::ParameterTangent (sph/sph.ixx:291-294): the layout of sph_parameters, FP32
 * tangents; NULL arrays are zero. */
typedef sph_parameters sph_parameter_tangent;

/* SPH<Method>::jvp_step (sph/sph.ixx:356-359): the tangent of the step recorded in `cache`, FP32,
 * solver in PBF_EXECUTION_DIFFERENTIABLE mode.  method_tangent / next_method_tangent: DFSPH's
 * warm-start pressure tangents (NULL = zero in; the next ones are written when not NULL).
 * next_state is accepted for the reference's signature and not read. */
int sph_jvp_step(sph_solver* solver, const pbf_particle_state* state, const sph_method_state* method_state,
                 const pbf_control* control, const sph_parameters* parameters, const pbf_particle_state* next_state,
                 const sph_step_cache* cache, const pbf_particle_state_tangent* state_tangent,
                 const sph_method_state* method_tangent, const pbf_control* control_tangent,
                 const sph_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_tangent,
                 sph_method_state* next_method_tangent);

/* SPH<Method>::vjp_step (sph/sph.ixx:361-365): the adjoint of the step recorded in `cache` (the
 * forward_step of `state`), solver in PBF_EXECUTION_DIFFERENTIABLE mode.  previous_adjoint,
 * control_adjoint and parameter_adjoint are ACCUMULATED.  DFSPH: next_method_adjoint holds the
 * adjoints of the next warm-start pressures (NULL = zero); previous_method_adjoint receives those of
 * the input warm starts, overwritten when the configuration warm-starts (sph/sph.cpp:714).
 * next_state is accepted for the reference's signature and not read. */
int sph_vjp_step(sph_solver* solver, const pbf_particle_state* state, const sph_method_state* method_state,
                 const pbf_control* control, const sph_parameters* parameters, const pbf_particle_state* next_state,
                 const sph_step_cache* cache, const pbf_particle_state_adjoint* next_adjoint,
                 const sph_method_state_adjoint* next_method_adjoint, pbf_particle_state_adjoint* previous_adjoint,
                 sph_method_state_adjoint* previous_method_adjoint, pbf_control_adjoint* control_adjoint,
                 sph_parameter_adjoint* parameter_adjoint);

/* SPH<Method>::copy_state / copy_state_tangent / copy_state_adjoint / accumulate_state_adjoint
 * (sph/sph.ixx:326-345): the particle fields plus DFSPH's warm-start pressures (the method fields
 * are ignored for the other methods and may be NULL there). */
int sph_copy_state(sph_solver* solver, const pbf_particle_state* source, const sph_method_state* source_method,
                   pbf_particle_state* destination, sph_method_state* destination_method);
int sph_copy_state_tangent(sph_solver* solver, const pbf_particle_state_tangent* source, const sph_method_state* source_method,
                           pbf_particle_state_tangent* destination, sph_method_state* destination_method);
int sph_copy_state_adjoint(sph_solver* solver, const pbf_particle_state_adjoint* source,
                           const sph_method_state_adjoint* source_method, pbf_particle_state_adjoint* destination,
                           sph_method_state_adjoint* destination_method);
int sph_accumulate_state_adjoint(sph_solver* solver, const pbf_particle_state_adjoint* source,
                                 const sph_method_state_adjoint* source_method, pbf_particle_state_adjoint* destination,
                                 sph_method_state_adjoint* destination_method);

/* A field of the step held by `cache`, written to device memory in original particle order
 * (x only for scalar fields). */
int sph_read_cache(sph_solver* solver, const sph_step_cache* cache, sph_cache_field field, float* x, float* y, float* z);

/* The reference gradient norm of PCISPH / IISPH / DFSPH (sph/sph.cpp:36-58, sph/sph.ixx:127). */
int sph_reference_gradient_norm(const sph_solver* solver, float* value);

/* Launch shape of the list scan and the gather passes (the fields of pbf_launch_shape). */
int sph_set_launch_shape(sph_solver* solver, const pbf_launch_shape* shape);
int sph_get_launch_shape(const sph_solver* solver, pbf_launch_shape* shape);

int sph_synchronize(sph_solver* solver);
void* sph_stream(const sph_solver* solver);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* PHYSICA_SPH_H */
