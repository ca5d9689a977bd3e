// pbf_forward_step_preallocated: one forward substep of one scene that allocates no device memory.
//
// Some callers cannot call cudaMalloc on the path where they advance the fluid: a host that
// enforces a fixed device-memory budget and hands out no memory after start-up (game and
// visual-effects engines, embedded simulators), or code whose device memory belongs to another
// allocator that must not be fragmented.  For them this
// entry point takes the caller's inputs and outputs only and keeps every intermediate buffer of
// the substep (scene table, kernel constants, cell-sorted copies, cell offsets, iterates, neighbour
// lists) in one file-scope device array, `g_scratch`, of kScratchBytes, sized for scenes of at most
// kMaxParticles particles and kMaxCells grid cells.  Every GPU that loads this library holds the
// array until the process exits.
//
// Set-up: the array exists once per CUDA context (the device's primary context, or a context the
// caller created with the driver API and made current).  The first call in a context asks the
// runtime for the array's device address there with cudaGetSymbolAddress and keeps it, keyed by
// the context's process-unique ID, so a later context on the same device (one created by the
// caller, or the new primary context after cudaDeviceReset) gets its own look-up.  Under lazy
// module loading, the CUDA default, that first call also loads this library's device code into the
// context and commits the array: make it at start-up, inside the caller's memory budget, and before
// any stream capture.  Every later call in the context reuses the address.
//
// Sharing: every call on a device uses the same array, and the array keeps the last call's
// contents.  The substep clears what must start at zero (the cell histogram) and writes every
// other buffer before reading it.  Calls whose GPU work overlaps (two streams, two host threads,
// or a call issued before the previous call's kernels finished on another stream) race on the
// array and give undefined results; order them on one stream.
//
// The launch sequence is the one of a forward-mode solver (pbf_forward_step) with these buffers
// in place of the solver's, so the outputs are bit-identical to pbf_forward_step on the same inputs.
#include <algorithm>
#include <exception>
#include <cmath>
#include <mutex>
#include <string>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "../../include/physica_pbf.h"
#include "engine.h"
#include "pbf_internal.h"
#include "pbf_launch.h"

namespace pbf {
namespace {

constexpr uint32_t kMaxParticles = PBF_PREALLOCATED_MAX_PARTICLES;
constexpr uint64_t kMaxCells = PBF_PREALLOCATED_MAX_CELLS;
constexpr size_t kAlign = 256;

constexpr size_t align_up(const size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Byte offsets of every buffer inside the scratch array for n particles and `cells` grid cells.
struct Layout {
    size_t scenes, statics, constants, radius, step;
    size_t predicted, arrival, unordered, tile_sums;
    size_t cell_offsets, sorted_index, slot_of, keys, cell, topology, params_a, params_b;
    size_t positions0, positions1, lambda, first_lambda, first_density, neighbor_count;
    size_t velocity, vorticity, normal, confined, list_entries, list_counts;
    size_t total;
};

constexpr Layout layout(const uint64_t n, const uint64_t cells, const uint64_t tiles) {
    Layout l{};
    size_t at = 0;
    auto take = [&at](const size_t bytes) {
        const size_t here = at;
        at += align_up(bytes ? bytes : 1);
        return here;
    };
    const size_t padded = (n + 31u) / 32u * 32u;
    l.scenes = take(sizeof(SceneDesc));
    l.statics = take(sizeof(SceneStatic));
    l.constants = take(sizeof(KernelConstants));
    l.radius = take(sizeof(float));
    l.step = take(sizeof(unsigned long long));
    l.predicted = take(n * sizeof(float4));
    l.arrival = take(n * sizeof(uint32_t));
    l.unordered = take(n * sizeof(uint32_t));
    l.tile_sums = take(tiles * sizeof(uint32_t));
    l.cell_offsets = take((cells + 1) * sizeof(uint32_t));
    l.sorted_index = take(n * sizeof(uint32_t));
    l.slot_of = take(n * sizeof(uint32_t));
    l.keys = take(n * sizeof(uint32_t));
    l.cell = take(n * sizeof(int4));
    l.topology = take(n * sizeof(float4));
    l.params_a = take(n * sizeof(float4));
    l.params_b = take(n * sizeof(float4));
    l.positions0 = take(n * sizeof(float4));
    l.positions1 = take(n * sizeof(float4));
    l.lambda = take(n * sizeof(float));
    l.first_lambda = take(n * sizeof(float));
    l.first_density = take(n * sizeof(float));
    l.neighbor_count = take(n * sizeof(uint32_t));
    l.velocity = take(n * sizeof(float4));
    l.vorticity = take(n * sizeof(float4));
    l.normal = take(n * sizeof(float4));
    l.confined = take(n * sizeof(float4));
    l.list_entries = take(padded * kListCapacity * sizeof(uint32_t));
    l.list_counts = take(n * sizeof(uint32_t));
    l.total = at;
    return l;
}

// The cell-offset scan uses one partial sum per tile of at least 256 cells.
constexpr uint64_t kMaxTiles = (kMaxCells + 1 + 255) / 256;
constexpr size_t kScratchBytes = layout(kMaxParticles, kMaxCells, kMaxTiles).total;
static_assert(kScratchBytes <= PBF_PREALLOCATED_SCRATCH_BYTES, "the documented scratch size is an upper bound");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// One set-up per CUDA context, keyed by the context's process-unique ID (cuCtxGetId).
struct ScratchSlot {
    unsigned long long context;
    unsigned char* address;
};
constexpr size_t kMaxSlots = 64;
std::mutex g_setup_mutex;
ScratchSlot g_slots[kMaxSlots] = {};
size_t g_slot_count = 0, g_slot_next = 0;
PFN_cuCtxGetCurrent g_ctx_get_current = nullptr;
PFN_cuCtxGetId g_ctx_get_id = nullptr;

// The process-unique ID of the current context, 0 when none is current.  Called with the mutex held.
int current_context(unsigned long long* id) {
    *id = 0;
    if (!g_ctx_get_current || !g_ctx_get_id) {
        cudaDriverEntryPointQueryResult found{};
        void* fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &found);
        if (e != cudaSuccess || found != cudaDriverEntryPointSuccess || !fn) {
            set_error("driver entry point cuCtxGetCurrent not found");
            return PBF_ERROR_CUDA;
        }
        g_ctx_get_current = reinterpret_cast<PFN_cuCtxGetCurrent>(fn);
        fn = nullptr;
        e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &found);
        if (e != cudaSuccess || found != cudaDriverEntryPointSuccess || !fn) {
            set_error("driver entry point cuCtxGetId not found");
            return PBF_ERROR_CUDA;
        }
        g_ctx_get_id = reinterpret_cast<PFN_cuCtxGetId>(fn);
    }
    CUcontext context = nullptr;
    if (g_ctx_get_current(&context) != CUDA_SUCCESS) {
        set_error("cuCtxGetCurrent failed");
        return PBF_ERROR_CUDA;
    }
    if (context && g_ctx_get_id(context, id) != CUDA_SUCCESS) {
        set_error("cuCtxGetId failed");
        return PBF_ERROR_CUDA;
    }
    return PBF_SUCCESS;
}

// The device address of g_scratch in the current context (looked up once per context).
int scratch_address(unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long context = 0;
    if (int rc = current_context(&context)) return rc;
    if (context)
        for (size_t k = 0; k < g_slot_count; ++k)
            if (g_slots[k].context == context) {
                *out = g_slots[k].address;
                return PBF_SUCCESS;
            }
    // Set-up.  With no context current, the runtime makes the device's primary context current here.
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess || !ptr) {
        set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        return PBF_ERROR_CUDA;
    }
    if (int rc = current_context(&context)) return rc;
    if (!context) {
        set_error("no CUDA context is current after the scratch look-up");
        return PBF_ERROR_CUDA;
    }
    // Slots of contexts that no longer exist (after cudaDeviceReset) are never matched again; the
    // table overwrites its oldest slot once full.
    g_slots[g_slot_next] = {context, static_cast<unsigned char*>(ptr)};
    g_slot_next = (g_slot_next + 1) % kMaxSlots;
    if (g_slot_count < kMaxSlots) ++g_slot_count;
    *out = static_cast<unsigned char*>(ptr);
    return PBF_SUCCESS;
}

// Writes the scene's static tables into scratch (kernel arguments, so no host copy is needed).
__global__ void scene_tables_kernel(const SceneDesc desc, const SceneStatic statics, const float radius,
                                    const unsigned long long step, SceneDesc* __restrict__ desc_out,
                                    SceneStatic* __restrict__ statics_out, float* __restrict__ radius_out,
                                    unsigned long long* __restrict__ step_out) {
    *desc_out = desc;
    *statics_out = statics;
    *radius_out = radius;
    *step_out = step;
}

bool has3(const pbf_vector_field& f) { return f.x && f.y && f.z; }

int fail(const int code, const char* message) {
    set_error(message);
    return code;
}

int cuda(const cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PBF_SUCCESS;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return PBF_ERROR_CUDA;
}

int forward_preallocated(const pbf_domain_configuration* domain, const pbf_configuration* configuration,
                         const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                         pbf_particle_state* next_state, cudaStream_t stream) {
    if (!domain || !configuration || !state || !control || !parameters || !next_state)
        return fail(PBF_ERROR_INVALID_ARGUMENT, "null argument");
    const pbf_domain_configuration& c = *domain;
    if (!(std::isfinite(c.time_step) && c.time_step > 0.0F) || !(std::isfinite(c.support_radius) && c.support_radius > 0.0F) ||
        !std::isfinite(c.particle_radius))
        return fail(PBF_ERROR_INVALID_ARGUMENT, "time_step and support_radius must be finite and positive");
    if (c.boundary_particle_count > 0) return fail(PBF_ERROR_UNSUPPORTED, "boundary particles are not supported by this build");
    if (configuration->pressure_iterations > kMaxIterations)
        return fail(PBF_ERROR_CAPACITY, "pressure_iterations exceeds the supported maximum");
    if (c.particle_count > kMaxParticles)
        return fail(PBF_ERROR_CAPACITY, "particle_count exceeds PBF_PREALLOCATED_MAX_PARTICLES of the preallocated entry point");
    // neighborhood/neighborhood.cpp:28-32: ceil((max - min) / h) in float, as the solver does
    const float mins[3] = {c.boundary.minimum.x, c.boundary.minimum.y, c.boundary.minimum.z};
    const float maxs[3] = {c.boundary.maximum.x, c.boundary.maximum.y, c.boundary.maximum.z};
    uint32_t dims[3];
    uint64_t cells = 1;
    for (int a = 0; a < 3; ++a) {
        const float n = std::ceil((maxs[a] - mins[a]) / c.support_radius);
        if (!(n >= 1.0F) || n > 1048576.0F)
            return fail(PBF_ERROR_INVALID_ARGUMENT, "box extent / support_radius must be in [1, 2^20] per axis");
        dims[a] = static_cast<uint32_t>(n);
        cells *= dims[a];
    }
    if (cells > kMaxCells) return fail(PBF_ERROR_CAPACITY, "grid cells exceed PBF_PREALLOCATED_MAX_CELLS of the preallocated entry point");
    const uint32_t n = c.particle_count;
    if (n > 0) {
        if (!has3(state->positions) || !has3(state->velocities) || !has3(control->external_accelerations) ||
            !has3(next_state->positions) || !has3(next_state->velocities))
            return fail(PBF_ERROR_INVALID_ARGUMENT, "null field pointer");
        const pbf_parameters& p = *parameters;
        if (!p.masses || !p.rest_densities || !p.relaxation || !p.artificial_pressure_strength ||
            !p.artificial_pressure_exponent || !p.artificial_pressure_radius || !p.xsph_viscosity || !p.vorticity_confinement)
            return fail(PBF_ERROR_INVALID_ARGUMENT, "null parameter pointer");
    }
    const uint64_t tiles = scan_tile_count(cells + 1);
    const Layout L = layout(n, cells, tiles);
    if (tiles > kMaxTiles || L.total > kScratchBytes) return fail(PBF_ERROR_CAPACITY, "scene does not fit the preallocated scratch");

    unsigned char* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    auto at = [base](const size_t offset) { return static_cast<void*>(base + offset); };

    // Scene table, as the solver builds it at creation (time-dependent fields follow on the device).
    SceneDesc d{};
    d.grid.cells_x = dims[0];
    d.grid.cells_y = dims[1];
    d.grid.cells_z = dims[2];
    d.grid.cell_base = 0;
    d.grid.key_min_x = c.boundary.minimum.x;
    d.grid.key_min_y = c.boundary.minimum.y;
    d.grid.key_min_z = c.boundary.minimum.z;
    d.grid.key_vel_x = c.boundary.velocity.x;
    d.grid.key_vel_y = c.boundary.velocity.y;
    d.grid.key_vel_z = c.boundary.velocity.z;
    d.grid.cell_size = c.support_radius;
    d.first = 0;
    d.count = n;
    d.time_step = c.time_step;
    d.inverse_time_step = 1.0F / c.time_step;   // pbf/pbf.cpp:184, evaluated on the host in float
    d.gravity_x = c.gravity.x;
    d.gravity_y = c.gravity.y;
    d.gravity_z = c.gravity.z;
    d.constants = 0;
    const SceneStatic st{c.boundary.minimum.x, c.boundary.minimum.y, c.boundary.minimum.z, c.boundary.maximum.x,
                         c.boundary.maximum.y, c.boundary.maximum.z, c.boundary.velocity.x, c.boundary.velocity.y,
                         c.boundary.velocity.z, c.particle_radius};
    auto* scenes = static_cast<SceneDesc*>(at(L.scenes));
    auto* statics = static_cast<SceneStatic*>(at(L.statics));
    auto* constants = static_cast<KernelConstants*>(at(L.constants));
    auto* radius = static_cast<float*>(at(L.radius));
    auto* step = static_cast<unsigned long long*>(at(L.step));
    scene_tables_kernel<<<1, 1, 0, stream>>>(d, st, c.support_radius, state->step_index, scenes, statics, radius, step);
    count_launch();
    if (int rc = cuda(cudaGetLastError(), "scene table")) return rc;
    if (int rc = cuda(launch_constants(stream, radius, 1, constants), "kernel constants")) return rc;
    if (int rc = cuda(launch_scene_time(stream, statics, scenes, step, 1), "scene time")) return rc;

    GridBuildArgs g{};
    g.count = n;
    g.cells = cells;
    g.scenes = scenes;
    g.scene_of = nullptr;
    g.positions = {state->positions.x, state->positions.y, state->positions.z};
    g.velocities = {state->velocities.x, state->velocities.y, state->velocities.z};
    g.controls = {control->external_accelerations.x, control->external_accelerations.y, control->external_accelerations.z};
    g.params = {parameters->masses, parameters->rest_densities, parameters->relaxation,
                parameters->artificial_pressure_strength, parameters->artificial_pressure_exponent,
                parameters->artificial_pressure_radius, parameters->xsph_viscosity, parameters->vorticity_confinement};
    g.predicted = static_cast<float4*>(at(L.predicted));
    g.keys = static_cast<uint32_t*>(at(L.keys));
    g.arrival = static_cast<uint32_t*>(at(L.arrival));
    g.cell_offsets = static_cast<uint32_t*>(at(L.cell_offsets));
    g.tile_sums = static_cast<uint32_t*>(at(L.tile_sums));
    g.unordered = static_cast<uint32_t*>(at(L.unordered));
    g.sorted_index = static_cast<uint32_t*>(at(L.sorted_index));
    g.slot_of = static_cast<uint32_t*>(at(L.slot_of));
    g.cell = static_cast<int4*>(at(L.cell));
    g.topology = static_cast<float4*>(at(L.topology));
    g.params_a = static_cast<float4*>(at(L.params_a));
    g.params_b = static_cast<float4*>(at(L.params_b));
    // the grid build clears the cell histogram (cell_offsets) before counting into it
    if (int rc = cuda(launch_grid_build(stream, g), "grid build")) return rc;

    const uint32_t K = configuration->pressure_iterations;
    const unsigned block = 128;
    const GatherCommon gc{n, scenes, constants, g.cell_offsets, g.cell, g.params_a, g.params_b};
    float4* positions[2] = {static_cast<float4*>(at(L.positions0)), static_cast<float4*>(at(L.positions1))};
    auto iterate = [&](const uint32_t k) -> float4* { return k == 0 ? g.topology : positions[(k - 1) & 1u]; };
    auto* lambda = static_cast<float*>(at(L.lambda));
    auto* first_lambda = static_cast<float*>(at(L.first_lambda));
    auto* first_density = static_cast<float*>(at(L.first_density));
    auto* neighbor_count = static_cast<uint32_t*>(at(L.neighbor_count));
    auto* velocity = static_cast<float4*>(at(L.velocity));
    auto* vorticity = static_cast<float4*>(at(L.vorticity));
    auto* normal = static_cast<float4*>(at(L.normal));
    auto* confined = static_cast<float4*>(at(L.confined));
    const StoredList list{static_cast<uint32_t*>(at(L.list_entries)), static_cast<uint32_t*>(at(L.list_counts)), kListCapacity};
    const Field3 previous{state->positions.x, state->positions.y, state->positions.z};
    const MutField3 out_positions{next_state->positions.x, next_state->positions.y, next_state->positions.z};
    for (uint32_t k = 0; k < K; ++k) {
        const float4* xk = iterate(k);
        float4* xk1 = iterate(k + 1);
        float* lam = k == 0 ? first_lambda : lambda;
        if (int rc = cuda(launch_list_scan(stream, ListScanArgs{gc, xk, list}), "neighbour list scan")) return rc;
        const DensityLambdaArgs dl{gc, xk, lam, k == 0 ? first_density : nullptr, nullptr, k == 0 ? neighbor_count : nullptr,
                                   list};
        if (int rc = cuda(launch_density_lambda(stream, dl, block), "density/lambda")) return rc;
        const CorrectionArgs cr{gc, xk, lam, xk1, nullptr, k + 1 == K ? 1 : 0, previous, g.sorted_index, out_positions,
                                velocity, list};
        if (int rc = cuda(launch_correction(stream, cr, block), "correction/project")) return rc;
    }
    const float4* xK = iterate(K);
    if (K == 0) {
        if (int rc = cuda(launch_reconstruct(stream, n, scenes, g.cell, g.topology, previous, g.sorted_index, out_positions,
                                             velocity),
                          "reconstruct"))
            return rc;
    }
    if (int rc = cuda(launch_list_scan(stream, ListScanArgs{gc, xK, list}), "neighbour list scan")) return rc;
    if (int rc = cuda(launch_vorticity(stream, VorticityArgs{gc, xK, velocity, vorticity, list}, block), "vorticity")) return rc;
    if (int rc = cuda(launch_normal(stream, NormalArgs{gc, xK, velocity, vorticity, normal, confined, list}, block),
                      "normal/confinement"))
        return rc;
    const XsphArgs x{gc, xK, confined, g.sorted_index,
                     {next_state->velocities.x, next_state->velocities.y, next_state->velocities.z}, list};
    if (int rc = cuda(launch_xsph(stream, x, block), "xsph")) return rc;
    next_state->step_index = state->step_index + 1u;
    return PBF_SUCCESS;
}

}  // namespace
}  // namespace pbf

extern "C" {

int pbf_forward_step_preallocated(const pbf_domain_configuration* domain, const pbf_configuration* configuration,
                                  const pbf_particle_state* state, const pbf_control* control,
                                  const pbf_parameters* parameters, pbf_particle_state* next_state, void* cuda_stream) {
    try {
        return pbf::forward_preallocated(domain, configuration, state, control, parameters, next_state,
                                         static_cast<cudaStream_t>(cuda_stream));
    } catch (const std::exception& e) {
        pbf::set_error(std::string("internal exception: ") + e.what());
        return PBF_ERROR_CUDA;
    } catch (...) {
        pbf::set_error("internal exception");
        return PBF_ERROR_CUDA;
    }
}

}  // extern "C"
