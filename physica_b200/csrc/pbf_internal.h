// Internal types shared by the PBF CUDA translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_math.cuh"

namespace pbf {

// Uniform grid of one scene (neighborhood/neighborhood.ixx:321-332, neighborhood/device.h:8-24).
struct Grid {
    uint32_t cells_x, cells_y, cells_z;
    uint32_t cell_base;        // first global cell of this scene (0 for a single scene)
    float origin_x, origin_y, origin_z;   // box minimum + t * box velocity (gather side)
    float key_min_x, key_min_y, key_min_z; // box minimum (key side)
    float key_vel_x, key_vel_y, key_vel_z; // box velocity (key side)
    float time;                // (step + 1) * dt
    float cell_size;           // support radius
};

// Linear cell index of the particle sort used here: z fastest, then y, then x.  The cells
// (x, y, z-1), (x, y, z), (x, y, z+1) of a stencil column are then adjacent in the cell-sorted
// particle array, so every column of the 27-cell stencil is one contiguous range, visited in the
// reference's order (neighbour cells x-offset outer, z-offset inner, pbf/pbf.cu:105-110; within a
// cell ascending original index).  Exported grids use the reference's x-fastest index
// (reference_cell_index, neighborhood/neighborhood.cu:20-39).
__host__ __device__ __forceinline__ uint32_t cell_index(const Grid& g, const uint32_t x, const uint32_t y, const uint32_t z) {
    return g.cell_base + (x * g.cells_y + y) * g.cells_z + z;
}

__host__ __device__ __forceinline__ uint32_t reference_cell_index(const Grid& g, const uint32_t x, const uint32_t y,
                                                                   const uint32_t z) {
    return g.cell_base + (z * g.cells_y + y) * g.cells_x + x;
}

// Collision box of one scene at the step being computed (pbf/pbf.cpp:17-31).
struct Box {
    float min_x, min_y, min_z, max_x, max_y, max_z;
};

// Per-scene description used by the batched kernels; a single scene is a batch of one.
struct SceneDesc {
    Grid grid;
    Box box;
    uint32_t first;            // first particle (original order) of the scene
    uint32_t count;
    float time_step;
    float inverse_time_step;   // 1 / dt computed on the host in float, as pbf/pbf.cpp:184
    float gravity_x, gravity_y, gravity_z;
    uint32_t constants;        // index into the KernelConstants table
};

// Time-independent box data of one scene, from which the device derives the per-step fields.
struct SceneStatic {
    float min_x, min_y, min_z, max_x, max_y, max_z;
    float vel_x, vel_y, vel_z;
    float particle_radius;
    uint32_t grid_at_input_step;   // 0: the step's time is (step + 1) dt (PBF); 1: step dt (SPH)
};

// Per-particle parameters gathered into sorted order once per substep.
//   a = (rest density, relaxation, xsph viscosity, vorticity confinement)
//   b = (artificial pressure strength, exponent, radius, unused)
struct SortedParameters {
    float4* a;
    float4* b;
};

// Caller-side (original order) SoA views.
struct Field3 { const float* x; const float* y; const float* z; };
struct MutField3 { float* x; float* y; float* z; };
struct AdjField3 { double* x; double* y; double* z; };
struct ConstAdjField3 { const double* x; const double* y; const double* z; };

struct ParamPointers {
    const float* masses;
    const float* rest_densities;
    const float* relaxation;
    const float* strength;
    const float* exponent;
    const float* radius;
    const float* xsph;
    const float* vorticity;
};

// Device data of one step cache: everything lives in SORTED particle order except
// the neighbourhood permutation itself.
struct SortedState {
    uint32_t count;
    uint64_t cells;               // total cells (all scenes)
    uint32_t* cell_offsets;       // cells + 1
    uint32_t* sorted_index;       // sorted slot -> original particle
    uint32_t* slot_of;            // original particle -> sorted slot
    uint32_t* scene_of;           // sorted slot -> scene (batched only; null for one scene)
    int4* cell;                   // gather cell (x, y, z, scene) of each sorted particle
    float4* topology;             // predicted positions x* and mass
    SortedParameters params;
};

constexpr uint32_t kMaxIterations = 64;
// Stored neighbour-list capacity per particle (a longer list is rebuilt by scanning).
constexpr uint32_t kListCapacity = 96;

}  // namespace pbf
