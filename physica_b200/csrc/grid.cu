// Uniform-grid build of one substep: predict + cell key, a stable counting sort by cell,
// and the reorder of every per-particle input into cell-sorted float4 arrays.
//
// Reference behaviour (neighborhood/neighborhood.cu:20-70, pbf/pbf.cu:73-78):
//   key  = (z * cells_y + y) * cells_x + x of the clamped cell of x*,
//   order = stable sort of (key, original index)  [CUB radix sort in the reference],
//   cell_offsets[c] = first sorted slot with key >= c, c in [0, C].
// Here the same order comes from a counting sort: an atomic histogram, an exclusive
// scan over cells, a scatter, and a per-cell ranking by original index that restores
// the stable order, so sorted_index / cell_offsets equal the reference's bit for bit.
// Keys are global across the scenes of a batch (scene cell ranges are disjoint and
// ordered), so one sort serves one scene or many.
#include "pbf_internal.h"
#include "../../include/physica_pbf.h"
#include "pbf_launch.h"

namespace pbf {

namespace {

__device__ __forceinline__ int clamp_cell(const float q, const uint32_t cells) {
    return min(static_cast<int>(cells) - 1, max(0, __float2int_rd(q)));
}

// x* = x + dt (v + dt (g + a)) and the cell key of x*; histogram of keys.
__global__ void predict_key_kernel(const uint32_t count, const SceneDesc* __restrict__ scenes,
                                   const uint32_t* __restrict__ scene_of, const Field3 positions,
                                   const Field3 velocities, const Field3 controls,
                                   const float* __restrict__ masses, float4* __restrict__ predicted,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ arrival,
                                   uint32_t* __restrict__ histogram, uint32_t* __restrict__ input_flags,
                                   const int key_current) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const SceneDesc& sc = scenes[scene_of ? scene_of[i] : 0u];
    const f3 gravity = mk(sc.gravity_x, sc.gravity_y, sc.gravity_z);
    const f3 v = mk(velocities.x[i], velocities.y[i], velocities.z[i]);
    const f3 a = mk(controls.x[i], controls.y[i], controls.z[i]);
    if (input_flags) {   // optional input checks: one bit per kind of invalid input
        const float px = positions.x[i], py = positions.y[i], pz = positions.z[i], m = masses[i];
        uint32_t bad = 0u;
        if (!isfinite(px) || !isfinite(py) || !isfinite(pz)) bad |= PBF_INPUT_NONFINITE_POSITION;
        if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) bad |= PBF_INPUT_NONFINITE_VELOCITY;
        if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) bad |= PBF_INPUT_NONFINITE_CONTROL;
        if (!(isfinite(m) && m > 0.0F)) bad |= PBF_INPUT_BAD_MASS;
        if (bad) atomicOr(input_flags, bad);
    }
    const f3 x = mk(positions.x[i], positions.y[i], positions.z[i]);
    const float dt = sc.time_step;
    // PBF keys the predicted positions (pbf/pbf.cpp:168-170); SPH keys the input positions (sph/sph.ixx:351)
    const f3 xs = key_current ? x : fma3(dt, fma3(dt, add(gravity, a), v), x);
    predicted[i] = make_float4(xs.x, xs.y, xs.z, masses[i]);
    const Grid& g = sc.grid;
    // (x - minimum - time * velocity) / h, the product fused into the subtraction
    const int cx = clamp_cell(__fdiv_rn(__fmaf_rn(-g.time, g.key_vel_x, __fsub_rn(xs.x, g.key_min_x)), g.cell_size), g.cells_x);
    const int cy = clamp_cell(__fdiv_rn(__fmaf_rn(-g.time, g.key_vel_y, __fsub_rn(xs.y, g.key_min_y)), g.cell_size), g.cells_y);
    const int cz = clamp_cell(__fdiv_rn(__fmaf_rn(-g.time, g.key_vel_z, __fsub_rn(xs.z, g.key_min_z)), g.cell_size), g.cells_z);
    const uint32_t key = cell_index(g, static_cast<uint32_t>(cx), static_cast<uint32_t>(cy), static_cast<uint32_t>(cz));
    keys[i] = key;
    arrival[i] = atomicAdd(histogram + key, 1u);
}

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

__global__ void scan_reduce_kernel(const uint32_t* __restrict__ data, const uint64_t n, uint32_t* __restrict__ tile_sums) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint64_t idx = base + static_cast<uint64_t>(k) * kScanThreads + threadIdx.x;
        if (idx < n) s += data[idx];
    }
    // warp + block reduction
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ uint32_t partial[kScanThreads / 32];
    if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t t = threadIdx.x < kScanThreads / 32 ? partial[threadIdx.x] : 0u;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) tile_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile sums by one block, in chunks.
__global__ void scan_tiles_kernel(uint32_t* __restrict__ tile_sums, const uint32_t tiles) {
    __shared__ uint32_t carry_s;
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += kScanThreads) {
        const uint32_t idx = base + threadIdx.x;
        const uint32_t v = idx < tiles ? tile_sums[idx] : 0u;
        const uint32_t inc = warp_inclusive(v);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        uint32_t warp_prefix = 0, chunk_total = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) {
            if (w < warp) warp_prefix += warp_tot[w];
            chunk_total += warp_tot[w];
        }
        const uint32_t carry = carry_s;
        if (idx < tiles) tile_sums[idx] = carry + warp_prefix + inc - v;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + chunk_total;
        __syncthreads();
    }
}

// In-place exclusive scan of each tile plus its tile prefix: histogram -> cell offsets.
__global__ void scan_apply_kernel(uint32_t* __restrict__ data, const uint64_t n, const uint32_t* __restrict__ tile_sums) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
    // each thread owns kScanItems consecutive elements
    uint32_t vals[kScanItems];
    uint32_t local = 0;
    const uint64_t first = base + static_cast<uint64_t>(threadIdx.x) * kScanItems;
    // a whole tile of a 16-byte aligned array moves as uint4 (four loads and stores per thread
    // instead of sixteen); the last tile and unaligned arrays take the element loop
    const bool vector = base + kScanTile <= n && (reinterpret_cast<uintptr_t>(data) & 15u) == 0u;
    if (vector) {
        const uint4* const src = reinterpret_cast<const uint4*>(data + first);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const uint4 v = src[q];
            vals[4 * q] = v.x;
            vals[4 * q + 1] = v.y;
            vals[4 * q + 2] = v.z;
            vals[4 * q + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const uint64_t idx = first + k;
            vals[k] = idx < n ? data[idx] : 0u;
        }
    }
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) local += vals[k];
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    const uint32_t inc = warp_inclusive(local);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t warp_prefix = 0;
    for (int w = 0; w < warp; ++w) warp_prefix += warp_tot[w];
    uint32_t running = tile_sums[blockIdx.x] + warp_prefix + inc - local;
    if (vector) {
        uint4* const dst = reinterpret_cast<uint4*>(data + first);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            uint4 v;
            v.x = running;
            running += vals[4 * q];
            v.y = running;
            running += vals[4 * q + 1];
            v.z = running;
            running += vals[4 * q + 2];
            v.w = running;
            running += vals[4 * q + 3];
            dst[q] = v;
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint64_t idx = first + k;
        if (idx < n) data[idx] = running;
        running += vals[k];
    }
}

__global__ void scatter_kernel(const uint32_t count, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ arrival,
                               const uint32_t* __restrict__ cell_offsets, uint32_t* __restrict__ unordered) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    unordered[cell_offsets[keys[i]] + arrival[i]] = i;
}

// Restore ascending original index inside each cell and gather the sorted arrays.
__global__ void reorder_kernel(const uint32_t count, const SceneDesc* __restrict__ scenes,
                               const uint32_t* __restrict__ scene_of, const uint32_t* __restrict__ keys,
                               const uint32_t* __restrict__ cell_offsets, const uint32_t* __restrict__ unordered,
                               const float4* __restrict__ predicted, const ParamPointers params,
                               uint32_t* __restrict__ sorted_index, uint32_t* __restrict__ slot_of,
                               int4* __restrict__ cell, float4* __restrict__ topology, float4* __restrict__ params_a,
                               float4* __restrict__ params_b, const Field3 velocities, float4* __restrict__ sorted_velocity,
                               const PackedPositions packed) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t i = unordered[t];
    const uint32_t key = keys[i];
    const uint32_t first = cell_offsets[key], last = cell_offsets[key + 1u];
    uint32_t rank = 0;
    for (uint32_t u = first; u < last; ++u) rank += unordered[u] < i ? 1u : 0u;
    const uint32_t s = first + rank;
    sorted_index[s] = i;
    slot_of[i] = s;
    const float4 xs = predicted[i];
    topology[s] = xs;
    if (packed.x) {
        packed.x[s] = xs.x;
        packed.y[s] = xs.y;
        packed.z[s] = xs.z;
    }
    const uint32_t scene = scene_of ? scene_of[i] : 0u;
    const Grid& g = scenes[scene].grid;
    // gather-side cell of x* (neighborhood/device.cuh:44-48)
    const int cx = clamp_cell(__fdiv_rn(__fsub_rn(xs.x, g.origin_x), g.cell_size), g.cells_x);
    const int cy = clamp_cell(__fdiv_rn(__fsub_rn(xs.y, g.origin_y), g.cell_size), g.cells_y);
    const int cz = clamp_cell(__fdiv_rn(__fsub_rn(xs.z, g.origin_z), g.cell_size), g.cells_z);
    cell[s] = make_int4(cx, cy, cz, static_cast<int>(scene));
    params_a[s] = make_float4(params.rest_densities[i], params.relaxation[i], params.xsph[i], params.vorticity[i]);
    params_b[s] = make_float4(params.strength[i], params.exponent[i], params.radius[i], 0.0F);
    if (sorted_velocity) sorted_velocity[s] = make_float4(velocities.x[i], velocities.y[i], velocities.z[i], 0.0F);
}

// ---- boundary particles (neighborhood/neighborhood.cu:63-69, key_kernel with moving positions) ----
// Key of a boundary particle at the step's time: x = p + t v (fused as the reference compiles
// `x += time * velocity`), then the fluid's cell formula; histogram of keys.
__global__ void boundary_key_kernel(const uint32_t count, const SceneDesc* __restrict__ scenes,
                                    const uint32_t* __restrict__ scene_of, const float4* __restrict__ rest,
                                    const float4* __restrict__ velocity, uint32_t* __restrict__ keys,
                                    uint32_t* __restrict__ arrival, uint32_t* __restrict__ histogram) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    const Grid& g = scenes[scene_of ? scene_of[b] : 0u].grid;
    const float4 p = rest[b], v = velocity[b];
    const f3 xs = mk(__fmaf_rn(g.time, v.x, p.x), __fmaf_rn(g.time, v.y, p.y), __fmaf_rn(g.time, v.z, p.z));
    const int cx = clamp_cell(__fdiv_rn(__fmaf_rn(-g.time, g.key_vel_x, __fsub_rn(xs.x, g.key_min_x)), g.cell_size), g.cells_x);
    const int cy = clamp_cell(__fdiv_rn(__fmaf_rn(-g.time, g.key_vel_y, __fsub_rn(xs.y, g.key_min_y)), g.cell_size), g.cells_y);
    const int cz = clamp_cell(__fdiv_rn(__fmaf_rn(-g.time, g.key_vel_z, __fsub_rn(xs.z, g.key_min_z)), g.cell_size), g.cells_z);
    const uint32_t key = cell_index(g, static_cast<uint32_t>(cx), static_cast<uint32_t>(cy), static_cast<uint32_t>(cz));
    keys[b] = key;
    arrival[b] = atomicAdd(histogram + key, 1u);
}

// Stable order inside each cell (ascending boundary index) and the sorted (position at t, volume).
__global__ void boundary_reorder_kernel(const uint32_t count, const SceneDesc* __restrict__ scenes,
                                        const uint32_t* __restrict__ scene_of, const uint32_t* __restrict__ keys,
                                        const uint32_t* __restrict__ cell_offsets, const uint32_t* __restrict__ unordered,
                                        const float4* __restrict__ rest, const float4* __restrict__ velocity,
                                        float4* __restrict__ sorted, float4* __restrict__ sorted_velocity) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    const uint32_t key = keys[b];
    const uint32_t first = cell_offsets[key], last = cell_offsets[key + 1u];
    uint32_t rank = 0;
    for (uint32_t u = first; u < last; ++u) rank += unordered[u] < b ? 1u : 0u;
    const float t = scenes[scene_of ? scene_of[b] : 0u].grid.time;
    const float4 p = rest[b], v = velocity[b];
    // boundary_position (neighborhood/device.cuh:16-22)
    sorted[first + rank] = make_float4(__fmaf_rn(t, v.x, p.x), __fmaf_rn(t, v.y, p.y), __fmaf_rn(t, v.z, p.z), p.w);
    if (sorted_velocity) sorted_velocity[first + rank] = v;
}

// ---- export in the reference's grid layout (cell index x fastest) ----
// Particle count of every cell of one scene, stored at the cell's reference index.
__global__ void reference_counts_kernel(const Grid g, const uint32_t* __restrict__ cell_offsets, uint32_t* __restrict__ out) {
    const uint32_t local = blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= g.cells_x * g.cells_y * g.cells_z) return;
    const uint32_t z = local % g.cells_z, y = (local / g.cells_z) % g.cells_y, x = local / (g.cells_z * g.cells_y);
    const uint32_t c = g.cell_base + local;
    out[reference_cell_index(g, x, y, z)] = cell_offsets[c + 1u] - cell_offsets[c];
}

// Slot of every particle in the reference's sorted order (cells by reference index, ascending
// original index within a cell), with its original index and its reference key.
__global__ void reference_order_kernel(const uint32_t count, const SceneDesc* __restrict__ scenes, const int4* __restrict__ cell,
                                       const uint32_t* __restrict__ sorted_index, const uint32_t* __restrict__ keys,
                                       const uint32_t* __restrict__ cell_offsets, const uint32_t* __restrict__ reference_offsets,
                                       uint32_t* __restrict__ out_index, unsigned long long* __restrict__ out_keys) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint32_t i = sorted_index[s];
    const uint32_t key = keys[i];
    const Grid& g = scenes[cell[s].w].grid;
    const uint32_t local = key - g.cell_base;
    const uint32_t z = local % g.cells_z, y = (local / g.cells_z) % g.cells_y, x = local / (g.cells_z * g.cells_y);
    const uint32_t reference = reference_cell_index(g, x, y, z);
    const uint32_t slot = reference_offsets[reference] + (s - cell_offsets[key]);
    if (out_index) out_index[slot] = i;
    if (out_keys) out_keys[slot] = reference;
}

__global__ void set_step_kernel(unsigned long long* step, const unsigned long long value) { *step = value; }
__global__ void advance_step_kernel(unsigned long long* step) { *step += 1ull; }

// Per-step scene fields from the device step counter (the step advances state `step` to `step + 1`):
// time = float(step + 1) * dt (pbf/pbf.cpp:18, neighborhood/neighborhood.cu:55), or float(step) * dt
// for a grid built at the input step (SPH, sph/sph.ixx:351, sph/sph.cpp:21-35), the gather origin
// (neighborhood/neighborhood.cpp:83-88) and the collision box (pbf/pbf.cpp:17-31), each with the
// float operation order of the reference's host code.
__global__ void scene_time_kernel(const SceneStatic* __restrict__ statics, SceneDesc* __restrict__ scenes,
                                  const unsigned long long* __restrict__ step, const uint32_t count) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const SceneStatic st = statics[s];
    SceneDesc& d = scenes[s];
    const float time = __fmul_rn(__ull2float_rn(*step + (st.grid_at_input_step ? 0ull : 1ull)), d.time_step);
    const float ox = __fadd_rn(st.min_x, __fmul_rn(time, st.vel_x));
    const float oy = __fadd_rn(st.min_y, __fmul_rn(time, st.vel_y));
    const float oz = __fadd_rn(st.min_z, __fmul_rn(time, st.vel_z));
    d.grid.time = time;
    d.grid.origin_x = ox;
    d.grid.origin_y = oy;
    d.grid.origin_z = oz;
    d.box.min_x = __fadd_rn(ox, st.particle_radius);
    d.box.min_y = __fadd_rn(oy, st.particle_radius);
    d.box.min_z = __fadd_rn(oz, st.particle_radius);
    d.box.max_x = __fsub_rn(__fadd_rn(st.max_x, __fmul_rn(time, st.vel_x)), st.particle_radius);
    d.box.max_y = __fsub_rn(__fadd_rn(st.max_y, __fmul_rn(time, st.vel_y)), st.particle_radius);
    d.box.max_z = __fsub_rn(__fadd_rn(st.max_z, __fmul_rn(time, st.vel_z)), st.particle_radius);
}

inline unsigned blocks_for(const uint64_t n, const unsigned threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

}  // namespace

cudaError_t launch_set_step(cudaStream_t stream, unsigned long long* step, const uint64_t value) {
    set_step_kernel<<<1, 1, 0, stream>>>(step, value);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_advance_step(cudaStream_t stream, unsigned long long* step) {
    advance_step_kernel<<<1, 1, 0, stream>>>(step);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scene_time(cudaStream_t stream, const SceneStatic* statics, SceneDesc* scenes, const unsigned long long* step,
                              const uint32_t count) {
    scene_time_kernel<<<blocks_for(count, 128), 128, 0, stream>>>(statics, scenes, step, count);
    count_launch();
    return cudaGetLastError();
}

size_t scan_tile_count(const uint64_t n) { return static_cast<size_t>((n + kScanTile - 1) / kScanTile); }

cudaError_t launch_grid_build(cudaStream_t stream, const GridBuildArgs& a) {
    const unsigned tpb = 256;
    cudaError_t e = cudaMemsetAsync(a.cell_offsets, 0, (a.cells + 1) * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    if (a.count > 0) {
        predict_key_kernel<<<blocks_for(a.count, tpb), tpb, 0, stream>>>(a.count, a.scenes, a.scene_of, a.positions,
                                                                         a.velocities, a.controls, a.params.masses,
                                                                         a.predicted, a.keys, a.arrival, a.cell_offsets,
                                                                         a.input_flags, a.key_current);
        count_launch();
    }
    const uint64_t n = a.cells + 1;
    const unsigned tiles = static_cast<unsigned>(scan_tile_count(n));
    scan_reduce_kernel<<<tiles, kScanThreads, 0, stream>>>(a.cell_offsets, n, a.tile_sums);
    scan_tiles_kernel<<<1, kScanThreads, 0, stream>>>(a.tile_sums, tiles);
    scan_apply_kernel<<<tiles, kScanThreads, 0, stream>>>(a.cell_offsets, n, a.tile_sums);
    count_launch(3);
    if (a.count > 0) {
        scatter_kernel<<<blocks_for(a.count, tpb), tpb, 0, stream>>>(a.count, a.keys, a.arrival, a.cell_offsets, a.unordered);
        reorder_kernel<<<blocks_for(a.count, tpb), tpb, 0, stream>>>(
            a.count, a.scenes, a.scene_of, a.keys, a.cell_offsets, a.unordered, a.predicted, a.params, a.sorted_index,
            a.slot_of, a.cell, a.topology, a.params_a, a.params_b, a.velocities, a.sorted_velocity, a.packed);
        count_launch(2);
    }
    return cudaGetLastError();
}

cudaError_t launch_boundary_build(cudaStream_t stream, const BoundaryBuildArgs& a) {
    cudaError_t e = cudaMemsetAsync(a.cell_offsets, 0, (a.cells + 1) * sizeof(uint32_t), stream);
    if (e != cudaSuccess || a.count == 0) return e;
    const unsigned tpb = 256;
    boundary_key_kernel<<<blocks_for(a.count, tpb), tpb, 0, stream>>>(a.count, a.scenes, a.scene_of, a.rest, a.velocity, a.keys,
                                                                      a.arrival, a.cell_offsets);
    count_launch();
    if ((e = launch_exclusive_scan(stream, a.cell_offsets, a.cells + 1, a.tile_sums)) != cudaSuccess) return e;
    scatter_kernel<<<blocks_for(a.count, tpb), tpb, 0, stream>>>(a.count, a.keys, a.arrival, a.cell_offsets, a.unordered);
    boundary_reorder_kernel<<<blocks_for(a.count, tpb), tpb, 0, stream>>>(a.count, a.scenes, a.scene_of, a.keys, a.cell_offsets,
                                                                          a.unordered, a.rest, a.velocity, a.sorted,
                                                                          a.sorted_velocity);
    count_launch(2);
    return cudaGetLastError();
}

cudaError_t launch_exclusive_scan(cudaStream_t stream, uint32_t* data, const uint64_t n, uint32_t* tile_sums) {
    const unsigned tiles = static_cast<unsigned>(scan_tile_count(n));
    scan_reduce_kernel<<<tiles, kScanThreads, 0, stream>>>(data, n, tile_sums);
    scan_tiles_kernel<<<1, kScanThreads, 0, stream>>>(tile_sums, tiles);
    scan_apply_kernel<<<tiles, kScanThreads, 0, stream>>>(data, n, tile_sums);
    count_launch(3);
    return cudaGetLastError();
}

cudaError_t launch_reference_offsets(cudaStream_t stream, const SceneDesc* host_scenes, const uint32_t scene_count,
                                     const uint64_t cells, const uint32_t* cell_offsets, uint32_t* reference_offsets,
                                     uint32_t* tile_sums) {
    cudaError_t e = cudaMemsetAsync(reference_offsets, 0, (cells + 1) * sizeof(uint32_t), stream);
    for (uint32_t s = 0; s < scene_count && e == cudaSuccess; ++s) {
        const Grid& g = host_scenes[s].grid;
        const uint32_t n = g.cells_x * g.cells_y * g.cells_z;
        reference_counts_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(g, cell_offsets, reference_offsets);
        count_launch();
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    return launch_exclusive_scan(stream, reference_offsets, cells + 1, tile_sums);
}

cudaError_t launch_reference_order(cudaStream_t stream, const uint32_t count, const SceneDesc* scenes, const int4* cell,
                                   const uint32_t* sorted_index, const uint32_t* keys, const uint32_t* cell_offsets,
                                   const uint32_t* reference_offsets, uint32_t* out_index, unsigned long long* out_keys) {
    if (count == 0) return cudaSuccess;
    reference_order_kernel<<<blocks_for(count, 256), 256, 0, stream>>>(count, scenes, cell, sorted_index, keys, cell_offsets,
                                                                       reference_offsets, out_index, out_keys);
    count_launch();
    return cudaGetLastError();
}

}  // namespace pbf
