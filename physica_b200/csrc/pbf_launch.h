// Launcher declarations and argument blocks of the PBF kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_internal.h"

namespace pbf {

void count_launch(unsigned n = 1);
uint64_t launch_count();

// Iterate positions in sorted order as three arrays (x, y, z) for the packed list scan.  Each
// array starts 16-byte aligned and has at least three readable floats past its last slot.
struct PackedPositions {
    float* x = nullptr;
    float* y = nullptr;
    float* z = nullptr;
};

struct GridBuildArgs {
    uint32_t count;
    uint64_t cells;
    const SceneDesc* scenes;
    const uint32_t* scene_of;      // original particle -> scene (null: one scene)
    Field3 positions, velocities, controls;
    ParamPointers params;
    float4* predicted;             // original order, x* and mass
    uint32_t* keys;                // original order
    uint32_t* arrival;             // original order
    uint32_t* cell_offsets;        // cells + 1
    uint32_t* tile_sums;
    uint32_t* unordered;
    uint32_t* sorted_index;
    uint32_t* slot_of;
    int4* cell;
    float4* topology;
    float4* params_a;
    float4* params_b;
    uint32_t* input_flags = nullptr;   // optional input checks (PBF_INPUT_* bits), null when off
    int key_current = 0;               // key the input positions instead of the predicted ones (SPH)
    float4* sorted_velocity = nullptr; // optional (v, 0) in sorted order
    PackedPositions packed{};          // optional x* as three arrays in sorted order
};

size_t scan_tile_count(uint64_t n);
cudaError_t launch_grid_build(cudaStream_t stream, const GridBuildArgs& args);
cudaError_t launch_exclusive_scan(cudaStream_t stream, uint32_t* data, uint64_t n, uint32_t* tile_sums);
// Cell offsets in the reference's grid layout (x-fastest cell index) from this layout's offsets.
cudaError_t launch_reference_offsets(cudaStream_t stream, const SceneDesc* host_scenes, uint32_t scene_count, uint64_t cells,
                                     const uint32_t* cell_offsets, uint32_t* reference_offsets, uint32_t* tile_sums);
// The reference's sorted order: original indices and uint64 reference keys by reference slot.
cudaError_t launch_reference_order(cudaStream_t stream, uint32_t count, const SceneDesc* scenes, const int4* cell,
                                   const uint32_t* sorted_index, const uint32_t* keys, const uint32_t* cell_offsets,
                                   const uint32_t* reference_offsets, uint32_t* out_index, unsigned long long* out_keys);

// A stored neighbour list (warp-interleaved entries + per-particle counts).  Two formats share the
// buffer of `capacity` 32-bit words per particle:
// - index lists (masks = 0): one sorted slot per in-support neighbour, counts = entries;
// - hit-mask lists (masks = 1): one (slot of bit 0, 32-bit hit mask) pair per 32-slot block of a
//   stencil column that holds a neighbour, capacity / 2 pairs per particle, counts = neighbours.
// Either lists the same neighbours in the same order; kOverflow marks a particle whose list did not
// fit (it walks its stencil instead).
struct StoredList {
    uint32_t* entries;
    uint32_t* counts;
    uint32_t capacity;
    int masks = 0;
};

// Common inputs of every neighbour-gather pass.
struct GatherCommon {
    uint32_t count;
    const SceneDesc* scenes;
    const KernelConstants* constants;
    const uint32_t* cell_offsets;
    const int4* cell;
    const float4* params_a;
    const float4* params_b;
    // Boundary particles of the step (null when the scenes have none): cell offsets into the
    // cell-sorted boundary array and its entries (position at the step's time, volume).
    const uint32_t* boundary_offsets = nullptr;
    const float4* boundary = nullptr;
    // Hand the blocks out last particles first.  A pass that replays the list the previous pass wrote
    // (or read) front to back then starts on the entries still in L2.  Results do not depend on it.
    int reverse = 0;
};

// Boundary particles (neighborhood/neighborhood.cu:63-69): keyed and sorted into the same cells
// as the fluid at every step, at their position p + t v (neighborhood/device.cuh:16-22).
struct BoundaryBuildArgs {
    uint32_t count;
    uint64_t cells;
    const SceneDesc* scenes;
    const uint32_t* scene_of;      // boundary particle -> scene (null: one scene)
    const float4* rest;            // (position at t = 0, volume), original order
    const float4* velocity;        // (velocity, 0), original order
    uint32_t* keys;
    uint32_t* arrival;
    uint32_t* unordered;
    uint32_t* tile_sums;
    uint32_t* cell_offsets;        // cells + 1
    float4* sorted;                // (position at the step's time, volume), cell-sorted
    float4* sorted_velocity = nullptr;   // optional (velocity, 0), cell-sorted
};
cudaError_t launch_boundary_build(cudaStream_t stream, const BoundaryBuildArgs& args);

struct DensityLambdaArgs {
    GatherCommon g;
    const float4* pos;         // current iterate x_k (and mass)
    float* lambda;
    float* density;            // optional record
    float4* gsum_denom;        // optional record: gradient sum S and denominator D
    uint32_t* neighbor_count;  // optional: poly6 in-radius neighbours, self excluded
    StoredList list;
};

struct CorrectionArgs {
    GatherCommon g;
    const float4* pos;
    const float* lambda;
    float4* pos_next;
    uint8_t* mask;             // optional record of the collision mask
    int last;                  // last iteration: reconstruct velocities and write positions out
    Field3 previous_positions; // original order (state.positions)
    const uint32_t* sorted_index;
    MutField3 out_positions;   // original order (next_state.positions)
    float4* velocity;          // reconstructed velocity (sorted)
    StoredList list;
    PackedPositions packed{};  // optional copy of pos_next as three arrays
};

struct VorticityArgs {
    GatherCommon g;
    const float4* pos;
    const float4* velocity;
    float4* vorticity;         // (omega, |omega|)
    StoredList list;
};

struct NormalArgs {
    GatherCommon g;
    const float4* pos;
    const float4* velocity;
    const float4* vorticity;
    float4* normal;            // (N, normalizer)
    float4* confined;          // confined velocity
    StoredList list;
};

struct XsphArgs {
    GatherCommon g;
    const float4* pos;
    const float4* confined;
    const uint32_t* sorted_index;
    MutField3 out_velocities;  // original order (next_state.velocities)
    StoredList list;
};

struct ListScanArgs {
    GatherCommon g;
    const float4* pos;
    StoredList list;
    int boundary = 0;   // also list boundary particles (density, lambda and correction lists)
    // optional: the same positions as three arrays; the per-lane scan then tests candidates in
    // pairs with packed FP32 arithmetic (ignored for lists with boundary particles)
    PackedPositions packed{};
};

// Launch shape of the neighbour-list and gather kernels.  Every shape gives bit-identical results
// (the per-particle arithmetic and its order do not depend on it); the autotuner picks the fastest.
enum ListScanVariant : uint32_t {
    kScanPerLane = 0,       // every lane walks its own 27 cells (run-mates share each load)
    kScanCooperative = 1,   // a warp walks each home-cell run's candidates once, 32 at a time
    kScanStaged = 2,        // a warp stages its column group's candidates in shared memory
    kScanFusedDensity = 3,  // per lane, and the Jacobi iterations' scans also run density + lambda
                            // in the same kernel (scenes without boundary particles)
    kScanFusedMasks = 4,    // as 3, and forward-mode steps store hit-mask lists (scenes without
                            // boundary particles; differentiable steps store index lists)
};
struct LaunchShape {
    uint32_t scan = kScanPerLane;
    uint32_t scan_block = 128;   // threads per block of the list scan: 32, 64, 96 or 128
    uint32_t block = 128;        // threads per block of the gather passes: 32, 64, 96 or 128
};
bool valid_shape(const LaunchShape& shape);

cudaError_t launch_list_scan(cudaStream_t stream, const ListScanArgs& a, const LaunchShape& shape = LaunchShape{});
// Whether `shape` runs the scan of `a` fused with density + lambda (launch_scan_density_lambda).
bool fuses_density(const LaunchShape& shape, const ListScanArgs& a);
// Whether a forward-mode step with `shape` stores hit-mask lists (no boundary particles).
bool stores_masks(const LaunchShape& shape, bool differentiable, bool boundary);
// The list scan of a Jacobi iteration and its density + lambda pass in one kernel (same list and
// results as launch_list_scan followed by launch_density_lambda).
cudaError_t launch_scan_density_lambda(cudaStream_t stream, const ListScanArgs& a, const DensityLambdaArgs& d,
                                       const LaunchShape& shape);
// Device step counter and the per-step scene fields derived from it (time, grid origin, collision box).
cudaError_t launch_set_step(cudaStream_t stream, unsigned long long* step, uint64_t value);
cudaError_t launch_advance_step(cudaStream_t stream, unsigned long long* step);
cudaError_t launch_scene_time(cudaStream_t stream, const SceneStatic* statics, SceneDesc* scenes, const unsigned long long* step,
                              uint32_t count);
cudaError_t launch_constants(cudaStream_t stream, const float* support_radii, uint32_t n, KernelConstants* out);
cudaError_t launch_density_lambda(cudaStream_t stream, const DensityLambdaArgs& a, unsigned block);
cudaError_t launch_correction(cudaStream_t stream, const CorrectionArgs& a, unsigned block);
cudaError_t launch_vorticity(cudaStream_t stream, const VorticityArgs& a, unsigned block);
cudaError_t launch_normal(cudaStream_t stream, const NormalArgs& a, unsigned block);
cudaError_t launch_xsph(cudaStream_t stream, const XsphArgs& a, unsigned block);
// Reconstruct velocities and write positions when no Jacobi iteration runs (K = 0).
cudaError_t launch_reconstruct(cudaStream_t stream, uint32_t count, const SceneDesc* scenes, const int4* cell,
                               const float4* positions, Field3 previous_positions, const uint32_t* sorted_index,
                               MutField3 out_positions, float4* velocity);

// FP64 dst[f][i] += src[f][i] for up to six fields.
cudaError_t launch_accumulate(cudaStream_t stream, size_t count, const double* const* src, double* const* dst, int fields);

// Neumaier-compensated FP64 sums of `segments` ranges (first/count device arrays; null: one range
// [0, single_count)).
cudaError_t launch_segment_sums(cudaStream_t stream, const double* values, const uint32_t* first, const uint32_t* count,
                                uint32_t segments, uint32_t single_count, double* out);

// Inspection helpers: scatter sorted arrays back to original order.
cudaError_t launch_export_frame(cudaStream_t stream, uint32_t count, Field3 positions, Field3 velocities, const uint32_t* slot_of,
                                const float4* vorticity, float* out_positions, float* out_velocities, float* out_vorticity);
cudaError_t launch_unsort_float4(cudaStream_t stream, uint32_t count, const uint32_t* sorted_index, const float4* in,
                                 int components, float* out_x, float* out_y, float* out_z, float* out_w);
cudaError_t launch_unsort_mask(cudaStream_t stream, uint32_t count, const uint32_t* sorted_index, const uint8_t* in,
                               uint32_t* out);
cudaError_t launch_unsort_scalar(cudaStream_t stream, uint32_t count, const uint32_t* sorted_index, const void* in,
                                 uint32_t element_bytes, void* out);

}  // namespace pbf
