/*
 * physica_pbf.h -- C ABI of the B200 Position Based Fluids solver.
 *
 * Drop-in boundary for the PBF substep of Xayah-Graphics/physica's
 * fluids/liquid/particle module.  Every entry point mirrors one member of the
 * reference's C++23 solver interface (pbf/pbf.ixx:14-141, domain/domain.ixx:12-165);
 * the reference file:line it replaces is given beside each declaration.
 *
 * Conventions
 *  - All field pointers are DEVICE pointers, structure-of-arrays x/y/z, `particle_count`
 *    elements each, owned by the caller (the reference's State/Parameters/adjoint structs
 *    own them as cuda::device_buffer, domain/domain.cpp:35-57).  The solver never frees them.
 *  - Every call is asynchronous on the solver's stream, like the reference
 *    (domain/domain.ixx:313); the only synchronising calls are pbf_create,
 *    pbf_synchronize and the *_host entry points.
 *  - Every call returns a pbf_status and never throws or aborts.  The reference's
 *    launchers return void and check nothing (pbf/kernels.h:12-46); its constructors
 *    throw from CCCL.  Here the failing call returns a non-zero status and
 *    pbf_last_error() gives a message for the calling thread.
 *  - A solver, its caches and its batches are not thread-safe; use one host thread each
 *    (the reference solver is non-copyable, non-movable, pbf/pbf.ixx:74-77).
 *  - vjp_step ACCUMULATES into previous_state_adjoint, control_adjoint and
 *    parameter_adjoint; zero them first (pbf/pbf.cpp:143-160 zero-fills at allocation).
 */
#ifndef PHYSICA_PBF_H
#define PHYSICA_PBF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define PHYSICA_PBF_ABI_VERSION 1

typedef enum {
    PBF_SUCCESS = 0,
    PBF_ERROR_INVALID_ARGUMENT = 1,
    PBF_ERROR_OUT_OF_MEMORY = 2,
    PBF_ERROR_CUDA = 3,
    PBF_ERROR_NOT_DIFFERENTIABLE = 4,   /* adjoint/tangent call on a forward-mode solver */
    PBF_ERROR_UNSUPPORTED = 5,
    PBF_ERROR_DEVICE_TIMEOUT = 6,       /* reserved for a bounded device-side wait that gives up; no kernel
                                           of this library waits on another today */
    PBF_ERROR_CAPACITY = 7              /* a size exceeds a documented maximum */
} pbf_status;

/* domain/domain.ixx:231-234 ExecutionMode */
typedef enum { PBF_EXECUTION_FORWARD = 0, PBF_EXECUTION_DIFFERENTIABLE = 1 } pbf_execution_mode;

/* domain/domain.ixx:202-206 Vector3 */
typedef struct { float x, y, z; } pbf_vector3;

/* domain/domain.ixx:208-213 BoxBoundary */
typedef struct {
    pbf_vector3 minimum;
    pbf_vector3 maximum;
    pbf_vector3 velocity;
    uint32_t no_slip;                    /* accepted and stored; the PBF kernels do not read it */
} pbf_box_boundary;

/* domain/domain.ixx:215-219 BoundaryParticle */
typedef struct {
    pbf_vector3 position;
    pbf_vector3 velocity;
    float volume;
} pbf_boundary_particle;

/* domain/domain.ixx:221-229 DomainConfiguration */
typedef struct {
    uint32_t particle_count;
    float time_step;
    float support_radius;
    float particle_radius;
    pbf_vector3 gravity;
    pbf_box_boundary boundary;
    const pbf_boundary_particle* boundary_particles;   /* host array, copied at creation */
    uint32_t boundary_particle_count;
} pbf_domain_configuration;

/* pbf/pbf.ixx:15-18 PBF::Configuration */
typedef struct {
    uint32_t pressure_iterations;        /* reference default 5 */
    uint32_t checkpoint_interval;        /* reference default 2 */
} pbf_configuration;

/* domain/domain.ixx:244-254 VectorField / VectorAdjointField (device SoA) */
typedef struct { float* x; float* y; float* z; } pbf_vector_field;
typedef struct { double* x; double* y; double* z; } pbf_vector_adjoint_field;

/* domain/domain.ixx:256-260 ParticleState (PBF::State, pbf/pbf.ixx:20) */
typedef struct {
    pbf_vector_field positions;
    pbf_vector_field velocities;
    uint64_t step_index;
} pbf_particle_state;

/* domain/domain.ixx:262-273 Control / ControlTangent */
typedef struct { pbf_vector_field external_accelerations; } pbf_control;

/* domain/domain.ixx:266-269 ParticleStateTangent (PBF::StateTangent, pbf/pbf.ixx:21) */
typedef struct { pbf_vector_field positions; pbf_vector_field velocities; } pbf_particle_state_tangent;

/* domain/domain.ixx:275-282 ParticleStateAdjoint / ControlAdjoint */
typedef struct { pbf_vector_adjoint_field positions; pbf_vector_adjoint_field velocities; } pbf_particle_state_adjoint;
typedef struct { pbf_vector_adjoint_field external_accelerations; } pbf_control_adjoint;

/* pbf/pbf.ixx:24-32 PBF::Parameters (particles = domain/domain.ixx:284-289) */
typedef struct {
    const float* masses;
    const float* rest_densities;
    const float* viscosities;            /* unused by PBF, as in the reference */
    const float* surface_tensions;       /* unused by PBF, as in the reference */
    const float* relaxation;
    const float* artificial_pressure_strength;
    const float* artificial_pressure_exponent;
    const float* artificial_pressure_radius;
    const float* xsph_viscosity;
    const float* vorticity_confinement;
} pbf_parameters;

/* pbf/pbf.ixx:34-42 PBF::ParameterTangent (same layout, tangents) */
typedef pbf_parameters pbf_parameter_tangent;

/* pbf/pbf.ixx:44-52 PBF::ParameterAdjoint (FP64, accumulated) */
typedef struct {
    double* masses;
    double* rest_densities;
    double* viscosities;
    double* surface_tensions;
    double* relaxation;
    double* artificial_pressure_strength;
    double* artificial_pressure_exponent;
    double* artificial_pressure_radius;
    double* xsph_viscosity;
    double* vorticity_confinement;
} pbf_parameter_adjoint;

/* Host-memory state for the *_host entry points (pinned or pageable). */
typedef struct {
    float* positions[3];
    float* velocities[3];
    uint64_t step_index;
} pbf_host_state;

typedef struct pbf_solver pbf_solver;          /* PBF (pbf/pbf.ixx:14-141) */
typedef struct pbf_step_cache pbf_step_cache;  /* PBF::StepCache (pbf/pbf.ixx:54-70) */
typedef struct pbf_batch pbf_batch;            /* many independent scenes in one launch sequence (no reference counterpart) */
typedef struct pbf_launch_shape {
    uint32_t list_scan;         /* 0: per-lane walk, 1: warp-cooperative scan, 2: shared-memory staged walk,
                                   3: per-lane walk with density + lambda in the same kernel,
                                   4: as 3, with hit-mask neighbour lists in forward mode */
    uint32_t scan_block_size;   /* threads per block of the list scan: 32, 64, 96 or 128 */
    uint32_t block_size;        /* threads per block of the gather passes: 32, 64, 96 or 128 */
} pbf_launch_shape;

/* Fields of a step cache that pbf_step_cache_read copies out, in ORIGINAL particle order
 * unless stated otherwise.  Each maps to a StepCache / Neighborhood member. */
typedef enum {
    PBF_CACHE_SORTED_PARTICLE_INDICES = 0, /* uint32[N]   neighborhood/neighborhood.ixx:323 */
    PBF_CACHE_CELL_OFFSETS = 1,            /* uint32[C+1] neighborhood/neighborhood.ixx:324 */
    PBF_CACHE_SORTED_KEYS = 2,             /* uint64[N]   neighborhood/neighborhood.ixx:322 */
    PBF_CACHE_PREDICTED_POSITIONS = 3,     /* float[3N]   pbf/pbf.ixx:61 (x block, y block, z block) */
    PBF_CACHE_CORRECTED_POSITIONS = 4,     /* float[3N]   pbf/pbf.ixx:62 */
    PBF_CACHE_RECONSTRUCTED_VELOCITIES = 5,/* float[3N]   pbf/pbf.ixx:64 */
    PBF_CACHE_VORTICITIES = 6,             /* float[3N]   pbf/pbf.ixx:65 */
    PBF_CACHE_VORTICITY_MAGNITUDES = 7,    /* float[N]    pbf/pbf.ixx:66 */
    PBF_CACHE_VORTICITY_NORMALS = 8,       /* float[3N]   pbf/pbf.ixx:67 */
    PBF_CACHE_VORTICITY_NORMALIZERS = 9,   /* float[N]    pbf/pbf.ixx:68 */
    PBF_CACHE_CONFINED_VELOCITIES = 10,    /* float[3N]   pbf/pbf.ixx:69 */
    PBF_CACHE_FIRST_DENSITIES = 11,        /* float[N]    densities of Jacobi iteration 0 (pbf.cpp:175) */
    PBF_CACHE_FIRST_LAMBDAS = 12,          /* float[N]    lambdas of Jacobi iteration 0 (pbf.cpp:176) */
    PBF_CACHE_NEIGHBOR_COUNTS = 13,        /* uint32[N]   poly6 in-radius neighbours (self excluded) at iteration 0 */
    PBF_CACHE_GRID_RESOLUTION = 14         /* uint32[3]   neighborhood/neighborhood.ixx:328 (host memory) */
} pbf_cache_field;

/* Per-iteration fields of a step cache (the reference's StepCache::IterationCheckpoint positions and
 * the IterationPrimal members, pbf/pbf.ixx:55-58, 98-105), ORIGINAL particle order.  Positions exist for
 * iterations 0..K in every mode (0 = predicted, K = corrected); the others for 0..K-1 and only in
 * PBF_EXECUTION_DIFFERENTIABLE mode, where every iteration is recorded. */
typedef enum {
    PBF_ITERATION_POSITIONS = 0,        /* float[3N] */
    PBF_ITERATION_DENSITIES = 1,        /* float[N]  */
    PBF_ITERATION_LAMBDAS = 2,          /* float[N]  */
    PBF_ITERATION_GRADIENT_SUMS = 3,    /* float[3N] */
    PBF_ITERATION_DENOMINATORS = 4,     /* float[N]  */
    PBF_ITERATION_COLLISION_MASKS = 5   /* uint32[N] */
} pbf_iteration_field;

/* ---- solver lifetime: PBF::PBF (pbf/pbf.cpp:39-72) and the implicit destructor ---- */
int pbf_create(const pbf_domain_configuration* domain, const pbf_configuration* configuration,
               pbf_execution_mode mode, void* cuda_stream, pbf_solver** solver);
int pbf_destroy(pbf_solver* solver);

/* ---- PBF::allocate_step_cache (pbf/pbf.cpp:108-125) ---- */
int pbf_allocate_step_cache(pbf_solver* solver, pbf_step_cache** cache);
int pbf_free_step_cache(pbf_step_cache* cache);

/* ---- PBF::forward_step (pbf/pbf.cpp:167-191) ---- */
int pbf_forward_step(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                     const pbf_parameters* parameters, pbf_particle_state* next_state, pbf_step_cache* cache);

/* ---- PBF::jvp_step (pbf/pbf.cpp:193-215): forward-mode FP32 tangents of the substep that `cache`
 *      holds (pbf_forward_step of `state` on a differentiable solver).  `parameter_tangent` may be
 *      NULL, and so may any of its pointers: a zero tangent.  next_state_tangent is overwritten. ---- */
int pbf_jvp_step(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                 const pbf_parameters* parameters, const pbf_particle_state* next_state, const pbf_step_cache* cache,
                 const pbf_particle_state_tangent* state_tangent, const pbf_control* control_tangent,
                 const pbf_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_state_tangent);

/* ---- PBF::vjp_step (pbf/pbf.cpp:217-258) ---- */
int pbf_vjp_step(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                 const pbf_parameters* parameters, const pbf_particle_state* next_state, const pbf_step_cache* cache,
                 const pbf_particle_state_adjoint* next_state_adjoint, pbf_particle_state_adjoint* previous_state_adjoint,
                 pbf_control_adjoint* control_adjoint, pbf_parameter_adjoint* parameter_adjoint);

/* ---- PBF::copy_state / copy_state_adjoint / accumulate_state_adjoint (pbf/pbf.cpp:162-165,
 *      domain/domain.cpp:129-199) ---- */
int pbf_copy_state(pbf_solver* solver, const pbf_particle_state* source, pbf_particle_state* destination);
/* PBF::copy_state_tangent (pbf/pbf.cpp:163) */
int pbf_copy_state_tangent(pbf_solver* solver, const pbf_particle_state_tangent* source,
                           pbf_particle_state_tangent* destination);
int pbf_copy_state_adjoint(pbf_solver* solver, const pbf_particle_state_adjoint* source,
                           pbf_particle_state_adjoint* destination);
int pbf_accumulate_state_adjoint(pbf_solver* solver, const pbf_particle_state_adjoint* source,
                                 pbf_particle_state_adjoint* destination);

/* ---- forward_step over host buffers: copies in, steps, copies out and waits.  No reference
 *      counterpart; it is the call a C caller without device memory makes (the reference example
 *      uploads with cuda::copy_bytes, examples/fluids/liquid/pbf-dam-break/simulation.ixx:97-105). ---- */
int pbf_forward_step_host(pbf_solver* solver, const pbf_host_state* state, const pbf_control* control,
                          const pbf_parameters* parameters, pbf_host_state* next_state, pbf_step_cache* cache);

/* ---- inspection of a step cache (copies to device memory, or host memory for the grid
 *      resolution).  `bytes` is the capacity of `destination`. ---- */
int pbf_step_cache_read(pbf_solver* solver, const pbf_step_cache* cache, pbf_cache_field field,
                        void* destination, size_t bytes);
int pbf_step_cache_read_iteration(pbf_solver* solver, const pbf_step_cache* cache, pbf_iteration_field field,
                                  uint32_t iteration, void* destination, size_t bytes);
int pbf_grid_cell_count(const pbf_solver* solver, uint64_t* cells);

/* ---- batched scenes: many independent dam breaks advance in one launch sequence per substep,
 *      replayed as one CUDA graph.  No counterpart in the reference (it runs one solver per
 *      scene); each scene behaves exactly as pbf_forward_step / pbf_vjp_step on its own.
 *      Particle arrays are the scenes' arrays concatenated in scene order. ---- */
int pbf_batch_create(const pbf_domain_configuration* scenes, uint32_t scene_count,
                     const pbf_configuration* configuration, pbf_execution_mode mode, void* cuda_stream,
                     pbf_batch** batch);
int pbf_batch_destroy(pbf_batch* batch);
int pbf_batch_particle_offset(const pbf_batch* batch, uint32_t scene, uint32_t* offset, uint32_t* count);
int pbf_batch_forward_step(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                           const pbf_parameters* parameters, pbf_particle_state* next_state, uint32_t cache_slot);
int pbf_batch_vjp_step(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, const pbf_particle_state* next_state, uint32_t cache_slot,
                       const pbf_particle_state_adjoint* next_state_adjoint,
                       pbf_particle_state_adjoint* previous_state_adjoint, pbf_control_adjoint* control_adjoint,
                       pbf_parameter_adjoint* parameter_adjoint);
int pbf_batch_jvp_step(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, const pbf_particle_state* next_state, uint32_t cache_slot,
                       const pbf_particle_state_tangent* state_tangent, const pbf_control* control_tangent,
                       const pbf_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_state_tangent);
int pbf_batch_reserve_caches(pbf_batch* batch, uint32_t cache_slots);

/* ---- compensated FP64 sum of a per-particle adjoint (Neumaier summation in a fixed, deterministic
 *      order), e.g. dL/dc for a scalar parameter shared by all particles: dL/dc = sum_i dL/dc_i.
 *      `values` and `result` are device pointers; `result` receives one double.  No reference
 *      counterpart: the reference keeps only the per-particle parameter adjoints (pbf/pbf.ixx:44-52). ---- */
int pbf_sum_compensated(pbf_solver* solver, const double* values, uint32_t count, double* result);
/* Per-scene compensated sums over a batch's concatenated per-particle values: result[scene_count]. */
int pbf_batch_scene_sums(pbf_batch* batch, const double* values, double* result);

/* ---- per-pass timing: CUDA events recorded on the solver's stream around every kernel group
 *      while enabled (pbf_profile_enable resets the totals); pbf_profile_read synchronises and
 *      returns one entry per pass that ran.  No reference counterpart (the reference has no
 *      timing); bench.py reports per-kernel GB/s from it. ---- */
typedef struct {
    const char* name;          /* static string, e.g. "density_lambda" */
    uint64_t launches;
    double milliseconds;       /* summed over launches */
} pbf_pass_time;
int pbf_profile_enable(pbf_solver* solver, int enable);
int pbf_profile_read(pbf_solver* solver, pbf_pass_time* passes, uint32_t capacity, uint32_t* count);
int pbf_batch_profile_enable(pbf_batch* batch, int enable);
int pbf_batch_profile_read(pbf_batch* batch, pbf_pass_time* passes, uint32_t capacity, uint32_t* count);

/* ---- CUDA-graph replay of the forward substep: the launch sequence is captured once per set of
 *      state / control / parameter / cache buffers and replayed with one graph launch per call
 *      (default off for a solver, on for a batch).  No reference counterpart. ---- */
int pbf_set_graph_mode(pbf_solver* solver, int enable);

/* ---- checkpoint recomputation of the Jacobi iterations (differentiable mode).  The reference's
 *      StepCache keeps the iterate of every checkpoint_interval-th Jacobi iteration and the last one
 *      (pbf/pbf.ixx:54-70, pbf/pbf.cpp:173-182); vjp_step recomputes each segment's lists,
 *      densities, lambdas and iterates from its first iterate before reversing it
 *      (pbf/pbf.cpp:232-245) and jvp_step reruns the iterations (pbf/pbf.cpp:198-212).  Off (the
 *      default): step caches keep every iterate, its fields and its neighbour list, and nothing is
 *      recomputed.  On: step caches allocated afterwards keep the checkpoints only, plus every
 *      iteration's collision mask (1 byte per particle); the solver holds one segment of
 *      recomputed iterations.  Gradients and tangents are bit-identical in both forms.  Returns
 *      PBF_ERROR_NOT_DIFFERENTIABLE for a forward-mode solver. ---- */
int pbf_set_checkpoint_recompute(pbf_solver* solver, int enable);
int pbf_batch_set_checkpoint_recompute(pbf_batch* batch, int enable);
int pbf_batch_set_graph_mode(pbf_batch* batch, int enable);

/* ---- forward substep without any device allocation.  No counterpart in the reference.
 *
 *  For callers that cannot call cudaMalloc where they advance the fluid: hosts with a fixed
 *  device-memory budget that hand out no memory after start-up, and code whose device memory
 *  belongs to another allocator that must not be fragmented.  The caller passes the scene, its inputs and its
 *  outputs (device pointers, as for pbf_forward_step); every intermediate buffer lives in one
 *  library-owned device array of at most PBF_PREALLOCATED_SCRATCH_BYTES that every GPU loading
 *  this library holds until the process exits.  Scenes above PBF_PREALLOCATED_MAX_PARTICLES
 *  particles or PBF_PREALLOCATED_MAX_CELLS grid cells return PBF_ERROR_CAPACITY; boundary
 *  particles return PBF_ERROR_UNSUPPORTED.  Forward mode only; no step cache is kept.
 *  Results are bit-identical to pbf_forward_step on a forward-mode solver of the same scene.
 *  The array exists once per CUDA context (the device's primary context, or a context the caller
 *  created and made current).  The first call in a context looks up the array's device address
 *  there; under lazy module loading (the CUDA default) that call also loads the library's device
 *  code and commits the PBF_PREALLOCATED_SCRATCH_BYTES array, so make it at start-up, inside the
 *  memory budget, and before any stream capture.  A context created later, or the new primary
 *  context after cudaDeviceReset, gets its own first call.  All calls in a context share the array and it keeps the last call's
 *  contents (the call clears what must start at zero): calls whose GPU work overlaps, on different
 *  streams or host threads, race and give undefined results, so order them on one stream.
 *  `cuda_stream` is a cudaStream_t (NULL: the legacy default stream). ---- */
#define PBF_PREALLOCATED_MAX_PARTICLES 32768u
#define PBF_PREALLOCATED_MAX_CELLS 262144u
#define PBF_PREALLOCATED_SCRATCH_BYTES 20971520u   /* 20 MiB */
int pbf_forward_step_preallocated(const pbf_domain_configuration* domain, const pbf_configuration* configuration,
                                  const pbf_particle_state* state, const pbf_control* control,
                                  const pbf_parameters* parameters, pbf_particle_state* next_state, void* cuda_stream);

/* ---- launch shape of the neighbour-list and gather kernels, and its autotuner.  No reference
 *      counterpart.  Every shape gives bit-identical results; only the speed changes.
 *      list_scan: 0 = each lane walks its own stencil, 1 = a warp walks each home cell's
 *      candidates once, 2 = each lane walks its stencil in a shared-memory copy of its warp's
 *      stencil columns, 3 = as 0, and each Jacobi iteration's scan also computes density and lambda
 *      in the same kernel, replaying the list from shared memory (scenes with boundary particles run
 *      3 as 0), 4 = as 3, and a forward-mode step stores each neighbour list as hit masks (one
 *      slot base and 32-bit mask per stencil block with a neighbour) instead of one index per
 *      neighbour (differentiable steps and scenes with boundary particles store index lists);
 *      scan_block_size and block_size: 32, 64, 96 or 128 threads.  pbf_autotune
 *      times the twenty list-scan shapes by their scan and density + lambda time, then the gather block sizes by the
 *      gather passes' time, on `repeats` forward steps from `state` (writing `scratch_state` and
 *      the cache, which then hold that step); it keeps the fastest shape, returns it in `chosen`
 *      (may be NULL) and the substep time with it in `milliseconds_per_step` (may be NULL).  It
 *      synchronises the stream, resets the per-pass profile totals and uses a temporary 256 MiB
 *      device buffer to evict the L2 cache before every timed step. ---- */
int pbf_set_launch_shape(pbf_solver* solver, const pbf_launch_shape* shape);
int pbf_get_launch_shape(pbf_solver* solver, pbf_launch_shape* shape);
int pbf_autotune(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                 const pbf_parameters* parameters, pbf_particle_state* scratch_state, pbf_step_cache* cache,
                 uint32_t repeats, pbf_launch_shape* chosen, float* milliseconds_per_step);
int pbf_batch_set_launch_shape(pbf_batch* batch, const pbf_launch_shape* shape);
int pbf_batch_get_launch_shape(pbf_batch* batch, pbf_launch_shape* shape);
int pbf_batch_autotune(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, pbf_particle_state* scratch_state, uint32_t cache_slot,
                       uint32_t repeats, pbf_launch_shape* chosen, float* milliseconds_per_step);

/* ---- optional input checks.  No reference counterpart (its launchers check nothing,
 *      pbf/kernels.h:12-46).  While enabled, every forward step also tests its inputs on the
 *      device and ORs one bit per kind of invalid input into a device word; reading it
 *      synchronises the stream, returns the bits accumulated since the last read and clears them.
 *      The step itself still runs (the reference's kernels run on whatever they are given). ---- */
#define PBF_INPUT_NONFINITE_POSITION 1u
#define PBF_INPUT_NONFINITE_VELOCITY 2u
#define PBF_INPUT_NONFINITE_CONTROL 4u
#define PBF_INPUT_BAD_MASS 8u   /* a mass that is not finite and positive */
int pbf_set_input_checks(pbf_solver* solver, int enable);
int pbf_read_input_checks(pbf_solver* solver, uint32_t* flags);
int pbf_batch_set_input_checks(pbf_batch* batch, int enable);
int pbf_batch_read_input_checks(pbf_batch* batch, uint32_t* flags);

/* ---- headless frame export.  Replaces the dam-break example's Spectra provider
 *      (examples/fluids/liquid/pbf-dam-break/spectra/provider.ixx:74-96, spectra/kernels.cu:8-13),
 *      which copies every frame's positions and velocities as xyz triples and the step cache's
 *      vorticity magnitudes into viewer buffers: here the buffers are the caller's device memory
 *      (a file dump or any consumer can read them).  `cache` is the step that produced `state`
 *      (it supplies the vorticity magnitudes); `vorticity` may be NULL. ---- */
typedef struct {
    float* positions;    /* 3N floats: x, y, z of particle 0, then particle 1, ... */
    float* velocities;   /* 3N floats, same layout */
    float* vorticity;    /* N floats, |omega| in original particle order, or NULL */
} pbf_frame;
int pbf_export_frame(pbf_solver* solver, const pbf_particle_state* state, const pbf_step_cache* cache, pbf_frame* frame);

/* ---- misc ---- */
int pbf_synchronize(pbf_solver* solver);
int pbf_batch_synchronize(pbf_batch* batch);
const char* pbf_status_string(int status);
const char* pbf_last_error(void);
int pbf_abi_version(void);
/* Number of kernels this library launched since load (all threads). */
uint64_t pbf_launch_count(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* PHYSICA_PBF_H */
