/*
 * FP64 host oracle for the PBF substep -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of the reference Position Based Fluids substep of
 * Xayah-Graphics/physica (fluids/liquid/particle).  It is the checker for the
 * CUDA solver in physica_b200/ and the CPU baseline of bench.py; nothing in
 * the product path links or calls it.
 *
 * Followed reference files (paths inside the reference project):
 *   pbf/pbf.cpp:17-31         collision_box
 *   pbf/pbf.cpp:167-191       PBF::forward_step orchestration
 *   pbf/pbf.cpp:217-258       PBF::vjp_step orchestration
 *   pbf/pbf.cu:18-71          kernel functions (spiky gradient, s_corr)
 *   pbf/pbf.cu:73-794         per-pass formulas (forward and VJP)
 *   density/device.cuh:10-24  poly6 and its gradient
 *   density/density.cu:18-102 density forward / VJP
 *   neighborhood/neighborhood.cu:20-45, neighborhood/device.cuh:28-48  grid
 *
 * Parity pins: tests/golden/ holds outputs of the reference's own CUDA kernels
 * (built from its sources and run on a B200 by tests/golden/make_golden.py);
 * tests/test_oracle.py checks this oracle against them.
 */
#ifndef PHYSICA_PBF_ORACLE_H
#define PHYSICA_PBF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double* x;
    double* y;
    double* z;
} oracle_vec;

typedef struct {
    uint32_t count;
    uint32_t iterations;
    uint64_t step_index;          /* index of the input state; the step produces step_index + 1 */
    float time_step;
    float support_radius;
    float particle_radius;
    float gravity[3];
    float box_min[3];
    float box_max[3];
    float box_velocity[3];
    uint32_t boundary_count;      /* boundary particles (reference BoundaryView) */
    const double* boundary_position[3];
    const double* boundary_velocity[3];
    const double* boundary_volume;
} oracle_scene;

typedef struct {
    const double* masses;
    const double* rest_densities;
    const double* relaxation;
    const double* artificial_pressure_strength;
    const double* artificial_pressure_exponent;
    const double* artificial_pressure_radius;
    const double* xsph_viscosity;
    const double* vorticity_confinement;
} oracle_parameters;

/* Optional per-step outputs for parity checks; every pointer may be NULL. */
typedef struct {
    oracle_vec predicted;          /* x* */
    double* density0;              /* density at iteration 0 */
    double* lambda0;               /* lambda at iteration 0 */
    oracle_vec corrected;          /* x_c after the Jacobi loop */
    oracle_vec vorticity;
    oracle_vec confined_velocity;
    uint32_t* neighbor_count0;     /* poly6 in-radius neighbours (self excluded) at iteration 0 */
} oracle_trace;

/* Adjoint inputs/outputs of one substep (all FP64, accumulated like the reference). */
typedef struct {
    oracle_vec next_position;      /* dL/dx_{n+1} (input) */
    oracle_vec next_velocity;      /* dL/dv_{n+1} (input) */
    oracle_vec position;           /* dL/dx_n (accumulated) */
    oracle_vec velocity;           /* dL/dv_n (accumulated) */
    oracle_vec control;            /* dL/da_n (accumulated) */
    double* masses;                /* per-particle parameter adjoints (accumulated, may be NULL) */
    double* rest_densities;
    double* relaxation;
    double* artificial_pressure_strength;
    double* artificial_pressure_exponent;
    double* artificial_pressure_radius;
    double* xsph_viscosity;
    double* vorticity_confinement;
} oracle_adjoint;

/* One forward substep in FP64.  Returns 0 on success. */
int oracle_forward_step(const oracle_scene* scene, const oracle_parameters* parameters,
                        oracle_vec position, oracle_vec velocity, oracle_vec control,
                        oracle_vec next_position, oracle_vec next_velocity, oracle_trace* trace);

/* Reverse-mode derivative of one substep in FP64 (re-runs the forward internally). */
int oracle_vjp_step(const oracle_scene* scene, const oracle_parameters* parameters,
                    oracle_vec position, oracle_vec velocity, oracle_vec control,
                    oracle_adjoint* adjoint);

/*
 * Uniform-grid build with the reference's FP32 semantics (neighborhood.cu:20-45):
 * key = (z*cy + y)*cx + x of the clamped cell of each point, a stable sort of
 * (key, index) and cell_offsets[c] = first sorted slot with key >= c, c in [0, C].
 * dims receives (cx, cy, cz); cell_offsets must hold C + 1 entries (query C with dims_out first).
 */
int oracle_grid_dims(const float box_min[3], const float box_max[3], float support_radius, uint32_t dims[3]);
int oracle_grid_f32(uint32_t count, const float* x, const float* y, const float* z, float support_radius,
                    const float box_min[3], const float box_max[3], const float box_velocity[3], float time,
                    uint32_t* keys, uint32_t* sorted_indices, uint32_t* cell_offsets);

/*
 * Per-particle count of neighbours j != i in the 27-cell stencil of i's grid cell (cells from
 * `topology`, distances from `position`) with fl32(|x_i - x_j|^2) < fl32(h*h), computed in FP32
 * with the device's contraction of the squared distance.
 */
int oracle_neighbor_counts_f32(uint32_t count, const float* const topology[3], const float* const position[3],
                               float support_radius, const float box_min[3], const float box_max[3],
                               const float box_velocity[3], float time, uint32_t* counts);

/* Kernel functions, exposed for the analytic known-answer tests. */
double oracle_poly6(double dx, double dy, double dz, double h);
void oracle_spiky_gradient(double dx, double dy, double dz, double h, double out[3]);

int oracle_thread_count(void);

#ifdef __cplusplus
}
#endif

#endif
