// Host side of the SPH solvers (include/physica_sph.h): the scene table, the step cache and the
// launch sequence of SPH<Method>::forward_step (sph/sph.ixx:350-354) for the four methods, over
// the grid build, boundary build and list scan shared with the PBF substep.
#include <cmath>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/physica_sph.h"
#include "engine.h"
#include "sph_launch.h"

namespace pbf {
namespace sph {

// SPH<Method>::StepCache (sph/sph.ixx:299-303) in sorted order, plus the method's cache fields
// that the API exports.
struct SphRecord {
    DeviceArena arena;
    bool valid = false;
    uint64_t step_index = 0;
    uint32_t* cell_offsets = nullptr;
    uint32_t* sorted_index = nullptr;
    uint32_t* slot_of = nullptr;
    uint32_t* keys = nullptr;
    int4* cell = nullptr;
    float4* topology = nullptr;
    float4* params_a = nullptr;
    float4* params_b = nullptr;
    float4* velocity = nullptr;
    uint32_t* list_entries = nullptr;
    uint32_t* list_counts = nullptr;
    uint32_t list_capacity = 0;
    uint32_t* boundary_offsets = nullptr;
    float4* boundary = nullptr;
    float4* boundary_velocity = nullptr;
    float* density = nullptr;
    float4* aux = nullptr;
    float4* non_pressure = nullptr;
    float4* divergence_acceleration = nullptr;   // DFSPH, forward mode
    float4* pressure_acceleration = nullptr;     // the last pressure pass (WCSPH: pressure term)
    float4* viscosity_acceleration = nullptr;    // WCSPH
    float4* surface_acceleration = nullptr;      // WCSPH
    unsigned int* displacement = nullptr;   // max |x* - x| of every prediction of the step
    // The pressure-iteration phases of the iterative methods (PCISPH / IISPH: one; DFSPH: the
    // divergence and the density phase).  Differentiable mode keeps every iterate k = 0..K
    // (pressures, predictions, predicted densities, pressure accelerations) for the tangent and
    // the reverse passes; forward mode reuses one buffer of each.
    struct Phase {
        uint32_t iterations = 0;
        uint32_t first_slot = 0;                // displacement slot of the phase's first prediction
        std::vector<float*> pressure;           // p_k
        std::vector<float4*> predicted;         // x*_k (index k; K + 1 is scratch)
        std::vector<float*> predicted_density;  // rho*_k
        std::vector<float4*> acceleration;      // pressure acceleration of iterate k
        float* pressure_term = nullptr;         // p / rho^2 of the current iterate
        float* P(uint32_t k) const { return pressure[pressure.size() > 1 ? k : 0]; }
        float4* X(uint32_t k) const { return predicted[predicted.size() > 1 ? k : 0]; }
        float* R(uint32_t k) const { return predicted_density[predicted_density.size() > 1 ? k : 0]; }
        float4* A(uint32_t k) const { return acceleration.empty() ? nullptr : acceleration[k]; }
    };
    Phase phase[2];
    float4* total_acceleration = nullptr;   // WCSPH, differentiable mode
    const float* final_pressure = nullptr;
    const float* final_predicted_density = nullptr;
    float4* final_acceleration = nullptr;
    bool differentiable = false;
};

// List skin of the iterative methods, as a fraction of h: their predicted densities replay the
// stored lists instead of walking the stencil while twice the largest predicted displacement
// stays inside it (always exact: otherwise they walk).
constexpr float kIterativeSkin = 0.1F;
constexpr uint32_t kDisplacementSlots = 2u * kMaxIterations + 4u;

using Phase = SphRecord::Phase;

class SphEngine {
public:
    SphEngine() = default;
    SphEngine(const SphEngine&) = delete;
    SphEngine& operator=(const SphEngine&) = delete;
    ~SphEngine() {
        if (stream_) cudaStreamSynchronize(stream_);
    }

    int init(const pbf_domain_configuration* domain, const sph_configuration* configuration, pbf_execution_mode mode,
             cudaStream_t stream);
    int allocate(SphRecord& r);
    int forward(const pbf_particle_state* state, const sph_method_state* method_state, const pbf_control* control,
                const sph_parameters* parameters, pbf_particle_state* next_state, sph_method_state* next_method_state,
                SphRecord& r);
    int read(const SphRecord& r, sph_cache_field field, float* x, float* y, float* z);
    int reverse(const pbf_particle_state* state, const sph_method_state* method_state, const sph_parameters* parameters,
                const SphRecord& r, const pbf_particle_state_adjoint* next_adjoint,
                const sph_method_state_adjoint* next_method_adjoint, pbf_particle_state_adjoint* previous_adjoint,
                sph_method_state_adjoint* previous_method_adjoint, pbf_control_adjoint* control_adjoint,
                sph_parameter_adjoint* parameter_adjoint);
    bool differentiable() const { return differentiable_; }
    int tangent(const pbf_particle_state* state, const SphRecord& r, const pbf_particle_state_tangent* state_tangent,
                const sph_method_state* method_tangent, const pbf_control* control_tangent,
                const sph_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_tangent,
                sph_method_state* next_method_tangent);
    int check(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return PBF_SUCCESS;
        cudaGetLastError();
        set_error(std::string(what) + ": " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PBF_ERROR_OUT_OF_MEMORY : PBF_ERROR_CUDA;
    }
    cudaStream_t stream() const { return stream_; }
    uint32_t count() const { return count_; }
    bool dfsph() const { return config_.method == SPH_METHOD_DFSPH; }
    float reference_gradient_norm() const { return reference_gradient_norm_; }
    LaunchShape shape{};

private:
    int launch(cudaStream_t s, const pbf_particle_state* state, const sph_method_state* method_state, const pbf_control* control,
               const sph_parameters* parameters, pbf_particle_state* next_state, sph_method_state* next_method_state,
               SphRecord& r);

    sph_configuration config_{};
    bool differentiable_ = false;
    pbf_domain_configuration domain_{};
    std::vector<pbf_boundary_particle> boundary_host_;
    uint32_t count_ = 0;
    uint64_t cells_ = 0;
    uint32_t dims_[3] = {0, 0, 0};
    float reference_gradient_norm_ = 0.0F;
    cudaStream_t stream_ = nullptr;
    DeviceArena arena_;
    SceneDesc* d_scenes_ = nullptr;
    SceneStatic* d_static_ = nullptr;
    KernelConstants* d_list_constants_ = nullptr;
    SphConstants* d_constants_ = nullptr;
    unsigned long long* d_step_ = nullptr;
    uint64_t host_step_ = ~0ull;
    float4* scratch_ = nullptr;      // grid build: (x, m) in original order
    PackedPositions packed_{};       // the sorted positions again as x, y, z arrays (packed list scan)
    uint32_t* arrival_ = nullptr;
    uint32_t* unordered_ = nullptr;
    uint32_t* tile_sums_ = nullptr;
    uint32_t boundary_count_ = 0;
    float4* boundary_rest_ = nullptr;
    float4* boundary_velocity_ = nullptr;
    uint32_t* boundary_keys_ = nullptr;
    uint32_t* boundary_arrival_ = nullptr;
    uint32_t* boundary_unordered_ = nullptr;
    // reverse-pass workspace (sorted order), allocated on first use
    int reverse_workspace();
    SphStep step_of(const SphRecord& r) const;
    DeviceArena reverse_arena_;
    double4* acceleration_adjoint_[2] = {nullptr, nullptr};
    double4* non_pressure_adjoint_ = nullptr;
    double4* divergence_adjoint_ = nullptr;
    double* density_adjoint_ = nullptr;
    double* pressure_adjoint_[2] = {nullptr, nullptr};
    double* predicted_density_adjoint_ = nullptr;
    // tangent workspace (sorted order), allocated on first use
    DeviceArena tangent_arena_;
    float4* tangent_x_ = nullptr;
    float4* tangent_v_ = nullptr;
    float4* tangent_a_ = nullptr;
    float4* tangent_b_ = nullptr;
    float* tangent_density_ = nullptr;
    float* tangent_pressure_[2] = {nullptr, nullptr};
    float4* tangent_non_pressure_ = nullptr;
    float4* tangent_predicted_ = nullptr;
    float4* tangent_divergence_ = nullptr;
};

namespace {
bool finite_positive(const float v) { return std::isfinite(v) && v > 0.0F; }
bool has3(const pbf_vector_field& f) { return f.x && f.y && f.z; }
}  // namespace

int SphEngine::init(const pbf_domain_configuration* domain, const sph_configuration* configuration, const pbf_execution_mode mode,
                    cudaStream_t stream) {
    if (mode != PBF_EXECUTION_FORWARD && mode != PBF_EXECUTION_DIFFERENTIABLE) {
        set_error("unknown execution mode");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (configuration->method > SPH_METHOD_DFSPH) {
        set_error("unknown SPH method");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (configuration->checkpoint_interval == 0) {
        set_error("checkpoint_interval must be at least 1");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (configuration->pressure_iterations > kMaxIterations || configuration->divergence_iterations > kMaxIterations ||
        configuration->density_iterations > kMaxIterations) {
        set_error("iteration counts must not exceed " + std::to_string(kMaxIterations));
        return PBF_ERROR_CAPACITY;
    }
    const pbf_domain_configuration& c = *domain;
    if (!finite_positive(c.time_step) || !finite_positive(c.support_radius) || !std::isfinite(c.particle_radius)) {
        set_error("time_step and support_radius must be finite and positive");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (c.boundary_particle_count > 0 && !c.boundary_particles) {
        set_error("boundary_particles is null but boundary_particle_count > 0");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    config_ = *configuration;
    differentiable_ = mode == PBF_EXECUTION_DIFFERENTIABLE;
    domain_ = c;
    domain_.boundary_particles = nullptr;
    if (c.boundary_particle_count > 0) boundary_host_.assign(c.boundary_particles, c.boundary_particles + c.boundary_particle_count);
    const float mins[3] = {c.boundary.minimum.x, c.boundary.minimum.y, c.boundary.minimum.z};
    const float maxs[3] = {c.boundary.maximum.x, c.boundary.maximum.y, c.boundary.maximum.z};
    cells_ = 1;
    for (int a = 0; a < 3; ++a) {
        // neighborhood/neighborhood.cpp:28-32: ceil((max - min) / h) in float
        const float n = std::ceil((maxs[a] - mins[a]) / c.support_radius);
        if (!(n >= 1.0F) || n > 1048576.0F) {
            set_error("box extent / support_radius must be in [1, 2^20] per axis");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        dims_[a] = static_cast<uint32_t>(n);
        cells_ *= dims_[a];
    }
    if (cells_ >= (1ull << 31) || c.particle_count >= (1u << 31) || c.boundary_particle_count >= (1u << 31)) {
        set_error("cells and particles must each stay below 2^31");
        return PBF_ERROR_CAPACITY;
    }
    count_ = c.particle_count;
    boundary_count_ = c.boundary_particle_count;
    stream_ = stream;
    arena_.set_stream(stream);
    reference_gradient_norm_ = sph::reference_gradient_norm(c.support_radius, c.particle_radius);

    cudaError_t e = cudaSuccess;
    d_scenes_ = arena_.alloc<SceneDesc>(1, e);
    d_static_ = arena_.alloc<SceneStatic>(1, e);
    d_list_constants_ = arena_.alloc<KernelConstants>(1, e);
    d_constants_ = arena_.alloc<SphConstants>(1, e);
    d_step_ = arena_.alloc<unsigned long long>(1, e);
    float* d_radius = arena_.alloc<float>(1, e);
    SphSceneInput* d_input = arena_.alloc<SphSceneInput>(1, e);
    scratch_ = arena_.alloc<float4>(count_, e);
    packed_ = alloc_packed(arena_, count_, e);
    arrival_ = arena_.alloc<uint32_t>(count_, e);
    unordered_ = arena_.alloc<uint32_t>(count_, e);
    tile_sums_ = arena_.alloc<uint32_t>(scan_tile_count(cells_ + 1), e);
    if (boundary_count_ > 0) {
        boundary_rest_ = arena_.alloc<float4>(boundary_count_, e);
        boundary_velocity_ = arena_.alloc<float4>(boundary_count_, e);
        boundary_keys_ = arena_.alloc<uint32_t>(boundary_count_, e);
        boundary_arrival_ = arena_.alloc<uint32_t>(boundary_count_, e);
        boundary_unordered_ = arena_.alloc<uint32_t>(boundary_count_, e);
    }
    if (int rc = check(e, "device allocation")) return rc;

    SceneDesc d{};
    d.grid.cells_x = dims_[0];
    d.grid.cells_y = dims_[1];
    d.grid.cells_z = dims_[2];
    d.grid.cell_base = 0;
    d.grid.key_min_x = c.boundary.minimum.x;
    d.grid.key_min_y = c.boundary.minimum.y;
    d.grid.key_min_z = c.boundary.minimum.z;
    d.grid.key_vel_x = c.boundary.velocity.x;
    d.grid.key_vel_y = c.boundary.velocity.y;
    d.grid.key_vel_z = c.boundary.velocity.z;
    d.grid.cell_size = c.support_radius;
    d.first = 0;
    d.count = count_;
    d.time_step = c.time_step;
    d.inverse_time_step = 1.0F / c.time_step;
    d.gravity_x = c.gravity.x;
    d.gravity_y = c.gravity.y;
    d.gravity_z = c.gravity.z;
    d.constants = 0;
    const SceneStatic st{c.boundary.minimum.x, c.boundary.minimum.y, c.boundary.minimum.z, c.boundary.maximum.x,
                         c.boundary.maximum.y, c.boundary.maximum.z, c.boundary.velocity.x, c.boundary.velocity.y,
                         c.boundary.velocity.z, c.particle_radius, 1u};
    const SphSceneInput in{c.support_radius, c.particle_radius, reference_gradient_norm_, c.boundary.velocity.x,
                           c.boundary.velocity.y, c.boundary.velocity.z, c.boundary.no_slip ? 1u : 0u,
                           configuration->method == SPH_METHOD_WCSPH ? 0.0F : kIterativeSkin};
    e = cudaMemcpyAsync(d_scenes_, &d, sizeof(d), cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_static_, &st, sizeof(st), cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_input, &in, sizeof(in), cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_radius, &c.support_radius, sizeof(float), cudaMemcpyHostToDevice, stream_);
    if (int rc = check(e, "upload scene table")) return rc;
    // PBF's constants give the list kernels their fields; the SPH constants then set the list threshold.
    if (int rc = check(launch_constants(stream_, d_radius, 1, d_list_constants_), "kernel constants")) return rc;
    if (int rc = check(launch_sph_constants(stream_, d_input, 1, d_constants_, d_list_constants_), "SPH constants")) return rc;
    if (boundary_count_ > 0) {
        std::vector<float4> rest, velocity;
        rest.reserve(boundary_count_);
        velocity.reserve(boundary_count_);
        for (const pbf_boundary_particle& b : boundary_host_) {
            rest.push_back(make_float4(b.position.x, b.position.y, b.position.z, b.volume));
            velocity.push_back(make_float4(b.velocity.x, b.velocity.y, b.velocity.z, 0.0F));
        }
        e = cudaMemcpyAsync(boundary_rest_, rest.data(), rest.size() * sizeof(float4), cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(boundary_velocity_, velocity.data(), velocity.size() * sizeof(float4), cudaMemcpyHostToDevice,
                                stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);   // the host vectors go out of scope
        if (int rc = check(e, "upload boundary particles")) return rc;
    }
    host_step_ = ~0ull;
    return check(cudaStreamSynchronize(stream_), "SPH solver initialisation");
}

int SphEngine::allocate(SphRecord& r) {
    r.arena.set_stream(stream_);
    cudaError_t e = cudaSuccess;
    const uint32_t n = count_;
    r.cell_offsets = r.arena.alloc<uint32_t>(cells_ + 1, e);
    r.sorted_index = r.arena.alloc<uint32_t>(n, e);
    r.slot_of = r.arena.alloc<uint32_t>(n, e);
    r.keys = r.arena.alloc<uint32_t>(n, e);
    r.cell = r.arena.alloc<int4>(n, e);
    r.topology = r.arena.alloc<float4>(n, e);
    r.params_a = r.arena.alloc<float4>(n, e);
    r.params_b = r.arena.alloc<float4>(n, e);
    r.velocity = r.arena.alloc<float4>(n, e);
    r.list_capacity = kListCapacity;
    const size_t padded = (static_cast<size_t>(n) + 31u) / 32u * 32u;
    r.list_entries = r.arena.alloc<uint32_t>(padded * r.list_capacity, e);
    r.list_counts = r.arena.alloc<uint32_t>(n, e);
    if (boundary_count_ > 0) {
        r.boundary_offsets = r.arena.alloc<uint32_t>(cells_ + 1, e);
        r.boundary = r.arena.alloc<float4>(boundary_count_, e);
        r.boundary_velocity = r.arena.alloc<float4>(boundary_count_, e);
    }
    r.density = r.arena.alloc<float>(n, e);
    r.aux = r.arena.alloc<float4>(n, e);
    r.pressure_acceleration = r.arena.alloc<float4>(n, e);
    r.differentiable = differentiable_;
    if (config_.method == SPH_METHOD_WCSPH) {
        Phase& ph = r.phase[0];
        ph.pressure.push_back(r.arena.alloc<float>(n, e));
        ph.pressure_term = r.arena.alloc<float>(n, e);
        r.viscosity_acceleration = r.arena.alloc<float4>(n, e);
        r.surface_acceleration = r.arena.alloc<float4>(n, e);
        if (differentiable_) r.total_acceleration = r.arena.alloc<float4>(n, e);
    } else {
        r.non_pressure = r.arena.alloc<float4>(n, e);
        r.displacement = r.arena.alloc<unsigned int>(kDisplacementSlots, e);
        const bool dfsph = config_.method == SPH_METHOD_DFSPH;
        const uint32_t phases = dfsph ? 2u : 1u;
        for (uint32_t q = 0; q < phases; ++q) {
            Phase& ph = r.phase[q];
            ph.iterations = dfsph ? (q == 0 ? config_.divergence_iterations : config_.density_iterations) : config_.pressure_iterations;
            ph.first_slot = q == 0 ? 0u : config_.divergence_iterations + 1u;
            const uint32_t K = ph.iterations;
            const uint32_t copies = differentiable_ ? K + 1u : 1u;
            for (uint32_t k = 0; k < copies; ++k) ph.pressure.push_back(r.arena.alloc<float>(n, e));
            for (uint32_t k = 0; k < (differentiable_ ? K + 2u : 1u); ++k) ph.predicted.push_back(r.arena.alloc<float4>(n, e));
            for (uint32_t k = 0; k < copies; ++k) ph.predicted_density.push_back(r.arena.alloc<float>(n, e));
            if (differentiable_)
                for (uint32_t k = 0; k <= K; ++k) ph.acceleration.push_back(r.arena.alloc<float4>(n, e));
            ph.pressure_term = r.arena.alloc<float>(n, e);
        }
        if (dfsph && !differentiable_) r.divergence_acceleration = r.arena.alloc<float4>(n, e);
    }
    r.valid = false;
    if (int rc = check(e, "step cache allocation")) return rc;
    for (uint32_t q = 0; q < 2; ++q) {
        for (float* d : r.phase[q].predicted_density)
            if (int rc = check(cudaMemsetAsync(d, 0, static_cast<size_t>(n) * sizeof(float), stream_), "clear")) return rc;
        for (float4* a : r.phase[q].acceleration)
            if (int rc = check(cudaMemsetAsync(a, 0, static_cast<size_t>(n) * sizeof(float4), stream_), "clear")) return rc;
    }
    return check(cudaStreamSynchronize(stream_), "step cache allocation");
}

int SphEngine::forward(const pbf_particle_state* state, const sph_method_state* method_state, const pbf_control* control,
                       const sph_parameters* parameters, pbf_particle_state* next_state, sph_method_state* next_method_state,
                       SphRecord& r) {
    if (!state || !control || !parameters || !next_state) {
        set_error("null argument");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    const uint32_t method = config_.method;
    if (count_ > 0) {
        if (!has3(state->positions) || !has3(state->velocities) || !has3(control->external_accelerations) ||
            !has3(next_state->positions) || !has3(next_state->velocities)) {
            set_error("null field pointer");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        const sph_parameters& p = *parameters;
        bool ok = p.masses && p.rest_densities && p.viscosities && p.surface_tensions;
        if (method == SPH_METHOD_WCSPH) ok = ok && p.speed_of_sound && p.tait_exponent && p.boundary_surface_tension;
        if (method == SPH_METHOD_PCISPH) ok = ok && p.pressure_relaxation;
        if (method == SPH_METHOD_IISPH) ok = ok && p.jacobi_relaxation;
        if (method == SPH_METHOD_DFSPH) ok = ok && p.divergence_relaxation && p.density_relaxation;
        if (!ok) {
            set_error("null parameter pointer for this method");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        if (method == SPH_METHOD_DFSPH) {
            if (!next_method_state || !next_method_state->warm_divergence_pressure || !next_method_state->warm_density_pressure ||
                (config_.pressure_warm_start &&
                 (!method_state || !method_state->warm_divergence_pressure || !method_state->warm_density_pressure))) {
                set_error("DFSPH needs its method state (warm-start pressures)");
                return PBF_ERROR_INVALID_ARGUMENT;
            }
        }
    }
    if (host_step_ != state->step_index) {
        if (int rc = check(launch_set_step(stream_, d_step_, state->step_index), "step counter")) return rc;
        host_step_ = state->step_index;
    }
    if (int rc = launch(stream_, state, method_state, control, parameters, next_state, next_method_state, r)) return rc;
    // the device counter then holds the index of the next state, as the host counter does
    if (int rc = check(launch_advance_step(stream_, d_step_), "step counter")) return rc;
    host_step_ = state->step_index + 1u;
    next_state->step_index = state->step_index + 1u;
    r.valid = true;
    r.step_index = state->step_index;
    return PBF_SUCCESS;
}

int SphEngine::launch(cudaStream_t s, const pbf_particle_state* state, const sph_method_state* method_state,
                      const pbf_control* control, const sph_parameters* parameters, pbf_particle_state* next_state,
                      sph_method_state* next_method_state, SphRecord& r) {
    if (int rc = check(launch_scene_time(s, d_static_, d_scenes_, d_step_, 1), "scene table")) return rc;
    const sph_parameters& p = *parameters;
    const uint32_t method = config_.method;
    // params_a = (rest density, viscosity, surface tension, method 0), params_b = (method 1, method 2, 0)
    const float* method0 = method == SPH_METHOD_WCSPH    ? p.speed_of_sound
                           : method == SPH_METHOD_PCISPH ? p.pressure_relaxation
                           : method == SPH_METHOD_IISPH  ? p.jacobi_relaxation
                                                         : p.divergence_relaxation;
    const float* method1 = method == SPH_METHOD_WCSPH ? p.tait_exponent : method == SPH_METHOD_DFSPH ? p.density_relaxation : method0;
    const float* method2 = method == SPH_METHOD_WCSPH ? p.boundary_surface_tension : method0;
    GridBuildArgs g{};
    g.count = count_;
    g.cells = cells_;
    g.scenes = d_scenes_;
    g.scene_of = nullptr;
    g.positions = {state->positions.x, state->positions.y, state->positions.z};
    g.velocities = {state->velocities.x, state->velocities.y, state->velocities.z};
    g.controls = {control->external_accelerations.x, control->external_accelerations.y, control->external_accelerations.z};
    // ParamPointers slots: (masses, rest densities, relaxation -> viscosities, strength -> method 1,
    // exponent -> method 2, radius -> method 2, xsph -> surface tensions, vorticity -> method 0)
    g.params = {p.masses, p.rest_densities, p.viscosities, method1, method2, method2, p.surface_tensions, method0};
    g.predicted = scratch_;
    g.keys = r.keys;
    g.arrival = arrival_;
    g.cell_offsets = r.cell_offsets;
    g.tile_sums = tile_sums_;
    g.unordered = unordered_;
    g.sorted_index = r.sorted_index;
    g.slot_of = r.slot_of;
    g.cell = r.cell;
    g.topology = r.topology;
    g.params_a = r.params_a;
    g.params_b = r.params_b;
    g.key_current = 1;
    g.sorted_velocity = r.velocity;
    g.packed = packed_;
    if (int rc = check(launch_grid_build(s, g), "grid build")) return rc;
    if (boundary_count_ > 0) {
        BoundaryBuildArgs b{boundary_count_, cells_, d_scenes_, nullptr, boundary_rest_, boundary_velocity_, boundary_keys_,
                            boundary_arrival_, boundary_unordered_, tile_sums_, r.boundary_offsets, r.boundary};
        b.sorted_velocity = r.boundary_velocity;
        if (int rc = check(launch_boundary_build(s, b), "boundary grid build")) return rc;
    }
    GatherCommon gc{count_, d_scenes_, d_list_constants_, r.cell_offsets, r.cell, r.params_a, r.params_b};
    if (boundary_count_ > 0) {
        gc.boundary_offsets = r.boundary_offsets;
        gc.boundary = r.boundary;
    }
    const StoredList list{r.list_entries, r.list_counts, r.list_capacity};
    ListScanArgs scan{gc, r.topology, list, 1};
    scan.packed = packed_;
    if (int rc = check(launch_list_scan(s, scan, shape), "neighbour list scan")) return rc;
    SphStep st{gc,
               d_constants_,
               r.topology,
               r.velocity,
               list,
               r.boundary_velocity,
               r.aux,
               r.non_pressure,
               nullptr,
               r.displacement,
               r.sorted_index,
               {control->external_accelerations.x, control->external_accelerations.y, control->external_accelerations.z}};
    const unsigned block = shape.block;
    const MutField3 out_x{next_state->positions.x, next_state->positions.y, next_state->positions.z};
    const MutField3 out_v{next_state->velocities.x, next_state->velocities.y, next_state->velocities.z};
    const bool warm = method == SPH_METHOD_DFSPH && config_.pressure_warm_start != 0;
    const bool diff = differentiable_;
    Phase& p0 = r.phase[0];
    if (int rc = check(launch_density(s, st, method, r.density, p0.P(0), p0.pressure_term,
                                      warm ? method_state->warm_divergence_pressure : nullptr, block),
                       "density"))
        return rc;
    if (method == SPH_METHOD_WCSPH) {
        r.final_pressure = p0.P(0);
        r.final_acceleration = r.pressure_acceleration;
        return check(launch_wcsph_forces(s, st, p0.pressure_term, out_x, out_v, r.pressure_acceleration,
                                         r.viscosity_acceleration, r.surface_acceleration, r.total_acceleration, block),
                     "WCSPH forces");
    }
    // Prediction p of the step records its largest displacement in slot p; the predicted density
    // that evaluates it reads that slot.
    if (int rc = check(cudaMemsetAsync(r.displacement, 0, kDisplacementSlots * sizeof(unsigned int), s), "clear")) return rc;
    const size_t scalar_bytes = static_cast<size_t>(count_) * sizeof(float);
    // One pressure iteration k of a phase: predicted density at x*_k with the pressure update, then
    // the pressure acceleration with the next prediction (sph/sph.cpp:301-306).
    auto iterate = [&](Phase& ph, const uint32_t k, const PressureUpdate update) -> int {
        if (diff && count_ > 0) {   // p_k starts from p_(k-1); the update runs in place
            if (int rc = check(cudaMemcpyAsync(ph.P(k), ph.P(k - 1), scalar_bytes, cudaMemcpyDeviceToDevice, s), "copy")) return rc;
        }
        SphStep sk = st;
        sk.predicted = ph.X(k);
        return check(launch_predicted_density(s, sk, update, ph.P(k), ph.pressure_term, ph.R(k), block), "predicted density");
    };
    auto pressure_pass = [&](Phase& ph, const uint32_t k, PressurePassArgs a) -> int {
        SphStep sk = st;
        sk.predicted = ph.X(k + 1);   // the next prediction (index K + 1: scratch)
        a.pressure_term = ph.pressure_term;
        a.pressure = ph.P(k);
        a.out_positions = out_x;
        a.out_velocities = out_v;
        a.displacement_slot = ph.first_slot + k;
        if (diff) a.store_acceleration = ph.A(k);
        return check(launch_pressure(s, sk, a, block), "pressure acceleration");
    };
    if (method == SPH_METHOD_PCISPH || method == SPH_METHOD_IISPH) {
        const uint32_t K = p0.iterations;
        if (K == 0 && !diff) {   // the cleared primal iterate's acceleration (sph/sph.cpp:298)
            if (int rc = check(cudaMemsetAsync(r.pressure_acceleration, 0, static_cast<size_t>(count_) * sizeof(float4), s),
                               "clear"))
                return rc;
        }
        SphStep s1 = st;
        s1.predicted = p0.X(1 <= K ? 1 : 0);
        if (int rc = check(launch_non_pressure(s, s1, K > 0 ? 1 : 2, out_x, out_v, 0u, block), "non-pressure acceleration"))
            return rc;
        for (uint32_t it = 1; it <= K; ++it) {
            if (int rc = iterate(p0, it, PressureUpdate{method, 0u, 0u, it - 1u})) return rc;
            PressurePassArgs a{};
            a.last = it == K ? 1 : 0;
            a.store_acceleration = it == K ? r.pressure_acceleration : nullptr;
            if (int rc = pressure_pass(p0, it, a)) return rc;
        }
        r.final_pressure = p0.P(K);
        r.final_predicted_density = p0.R(K);
        r.final_acceleration = diff ? p0.A(K) : r.pressure_acceleration;
        return PBF_SUCCESS;
    }
    // DFSPH::forward (sph/sph.cpp:572-610): the divergence phase, then the density phase, whose
    // warm start the divergence phase's last pressure pass loads (its neighbours still read the
    // divergence pressures, so the phases use separate buffers).
    if (int rc = check(launch_non_pressure(s, st, 0, out_x, out_v, 0u, block), "non-pressure acceleration")) return rc;
    Phase& p1 = r.phase[1];
    const uint32_t Kd = p0.iterations, Kr = p1.iterations;
    float4* divergence_acceleration = diff ? p0.A(Kd) : r.divergence_acceleration;
    for (uint32_t it = 0; it <= Kd; ++it) {
        if (it > 0) {
            if (int rc = iterate(p0, it, PressureUpdate{SPH_METHOD_DFSPH, 0u, 1u, it - 1u})) return rc;
        }
        PressurePassArgs a{};
        if (it == Kd) {
            a.store_acceleration = divergence_acceleration;
            a.warm_out = next_method_state->warm_divergence_pressure;
            a.next_pressure = p1.P(0);
            a.next_pressure_term = p1.pressure_term;
            a.next_warm = warm ? method_state->warm_density_pressure : nullptr;
        }
        if (int rc = pressure_pass(p0, it, a)) return rc;
    }
    for (uint32_t it = 0; it <= Kr; ++it) {
        if (it > 0) {
            if (int rc = iterate(p1, it, PressureUpdate{SPH_METHOD_DFSPH, 1u, 0u, p1.first_slot + it - 1u})) return rc;
        }
        PressurePassArgs a{};
        a.base = divergence_acceleration;
        if (it == Kr) {
            a.last = 1;
            a.warm_out = next_method_state->warm_density_pressure;
            a.store_acceleration = r.pressure_acceleration;
        }
        if (int rc = pressure_pass(p1, it, a)) return rc;
    }
    r.final_pressure = p1.P(Kr);
    r.final_predicted_density = p1.R(Kr);   // the density phase's primal (cleared when it has no iteration)
    r.final_acceleration = diff ? p1.A(Kr) : r.pressure_acceleration;
    return PBF_SUCCESS;
}

SphStep SphEngine::step_of(const SphRecord& r) const {
    GatherCommon gc{count_, d_scenes_, d_list_constants_, r.cell_offsets, r.cell, r.params_a, r.params_b};
    if (boundary_count_ > 0) {
        gc.boundary_offsets = r.boundary_offsets;
        gc.boundary = r.boundary;
    }
    return SphStep{gc,
                   d_constants_,
                   r.topology,
                   r.velocity,
                   StoredList{r.list_entries, r.list_counts, r.list_capacity},
                   r.boundary_velocity,
                   r.aux,
                   r.non_pressure,
                   nullptr,
                   r.displacement,
                   r.sorted_index,
                   {nullptr, nullptr, nullptr}};
}

int SphEngine::reverse_workspace() {
    if (density_adjoint_) return PBF_SUCCESS;
    reverse_arena_.set_stream(stream_);
    cudaError_t e = cudaSuccess;
    const size_t n = count_;
    for (auto& a : acceleration_adjoint_) a = reverse_arena_.alloc<double4>(n, e);
    non_pressure_adjoint_ = reverse_arena_.alloc<double4>(n, e);
    divergence_adjoint_ = reverse_arena_.alloc<double4>(n, e);
    for (auto& p : pressure_adjoint_) p = reverse_arena_.alloc<double>(n, e);
    predicted_density_adjoint_ = reverse_arena_.alloc<double>(n, e);
    density_adjoint_ = reverse_arena_.alloc<double>(n, e);
    if (int rc = check(e, "reverse workspace")) {
        reverse_arena_.release();
        density_adjoint_ = nullptr;
        return rc;
    }
    return PBF_SUCCESS;
}

// SPH<Method>::vjp_step (sph/sph.ixx:361-365): Method::vjp (sph/sph.cpp:239-250, 332-373,
// 445-486, 661-722) from the iterates the forward kept, newest first, then the density's reverse.
int SphEngine::reverse(const pbf_particle_state* state, const sph_method_state* method_state, const sph_parameters* parameters,
                       const SphRecord& r, const pbf_particle_state_adjoint* next_adjoint,
                       const sph_method_state_adjoint* next_method_adjoint, pbf_particle_state_adjoint* previous_adjoint,
                       sph_method_state_adjoint* previous_method_adjoint, pbf_control_adjoint* control_adjoint,
                       sph_parameter_adjoint* parameter_adjoint) {
    if (!differentiable_) {
        set_error("vjp_step needs a solver created in PBF_EXECUTION_DIFFERENTIABLE mode");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    if (!state || !parameters || !next_adjoint || !previous_adjoint || !control_adjoint || !parameter_adjoint) {
        set_error("null argument");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    (void)method_state;
    if (!r.valid || !r.differentiable || r.step_index != state->step_index) {
        set_error("the step cache does not hold the forward step of this state");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (count_ == 0) return PBF_SUCCESS;
    auto has = [](const pbf_vector_adjoint_field& f) { return f.x && f.y && f.z; };
    if (!has(next_adjoint->positions) || !has(next_adjoint->velocities) || !has(previous_adjoint->positions) ||
        !has(previous_adjoint->velocities) || !has(control_adjoint->external_accelerations)) {
        set_error("null adjoint field pointer");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (int rc = reverse_workspace()) return rc;
    const uint32_t method = config_.method;
    const sph_parameter_adjoint& q = *parameter_adjoint;
    SphParameterAdjoints pa{q.masses, q.rest_densities, q.viscosities, q.surface_tensions, nullptr, nullptr, nullptr};
    if (method == SPH_METHOD_WCSPH) {
        pa.method0 = q.speed_of_sound;
        pa.method1 = q.tait_exponent;
        pa.method2 = q.boundary_surface_tension;
    } else if (method == SPH_METHOD_PCISPH) {
        pa.method0 = q.pressure_relaxation;
    } else if (method == SPH_METHOD_IISPH) {
        pa.method0 = q.jacobi_relaxation;
    } else {
        pa.method0 = q.divergence_relaxation;
        pa.method1 = q.density_relaxation;
    }
    const SphStep st = step_of(r);
    const cudaStream_t s = stream_;
    const unsigned block = shape.block;
    const ConstAdjField3 nx{next_adjoint->positions.x, next_adjoint->positions.y, next_adjoint->positions.z};
    const ConstAdjField3 nv{next_adjoint->velocities.x, next_adjoint->velocities.y, next_adjoint->velocities.z};
    const AdjField3 X{previous_adjoint->positions.x, previous_adjoint->positions.y, previous_adjoint->positions.z};
    const AdjField3 V{previous_adjoint->velocities.x, previous_adjoint->velocities.y, previous_adjoint->velocities.z};
    const AdjField3 C{control_adjoint->external_accelerations.x, control_adjoint->external_accelerations.y,
                      control_adjoint->external_accelerations.z};
    const size_t n = count_;
    auto zero = [&](void* p, const size_t bytes) { return check(cudaMemsetAsync(p, 0, bytes, s), "clear"); };
    if (int rc = zero(density_adjoint_, n * sizeof(double))) return rc;
    auto density_step = [&]() {   // density_vjp at the step's positions (sph/sph.ixx:364)
        DensityVjpLaunch d{};
        d.st = st;
        d.positions = r.topology;
        d.density_adjoint = density_adjoint_;
        d.x = X;
        d.v = V;
        d.pa = pa;
        return check(launch_density_vjp(s, d, block), "density reverse");
    };
    if (method == SPH_METHOD_WCSPH) {
        if (int rc = check(launch_integrate_vjp(s, st, r.total_acceleration, nx, nv, X, V, C, acceleration_adjoint_[0]),
                           "integrate reverse"))
            return rc;
        if (int rc = check(launch_wcsph_force_vjp(s, st, r.phase[0].P(0), acceleration_adjoint_[0], X, V, pa, density_adjoint_, block),
                           "force reverse"))
            return rc;
        return density_step();
    }
    for (double4* a : {acceleration_adjoint_[0], acceleration_adjoint_[1], non_pressure_adjoint_, divergence_adjoint_})
        if (int rc = zero(a, n * sizeof(double4))) return rc;
    for (double* a : {pressure_adjoint_[0], pressure_adjoint_[1]})
        if (int rc = zero(a, n * sizeof(double))) return rc;
    uint32_t cur = 0;
    // One reverse iteration k of a phase: the pressure pass with the update that produced p_k, then
    // the predicted density of x*_k with the prediction that produced it.
    auto reverse_iteration = [&](const Phase& ph, const uint32_t k, const uint32_t relaxation, const uint32_t target,
                                 double* relaxation_adjoint, const float4* base, double4* base_adjoint) -> int {
        const uint32_t prev = cur ^ 1u;
        if (int rc = zero(acceleration_adjoint_[prev], n * sizeof(double4))) return rc;
        if (int rc = zero(pressure_adjoint_[prev], n * sizeof(double))) return rc;
        PressureVjpLaunch p{};
        p.st = st;
        p.pressure = ph.P(k);
        p.acceleration_adjoint = acceleration_adjoint_[cur];
        p.pressure_adjoint = pressure_adjoint_[cur];
        p.density_adjoint = density_adjoint_;
        p.x = X;
        p.pa = pa;
        p.method = method;
        p.relaxation = relaxation;
        p.target = target;
        p.previous_pressure = ph.P(k - 1);
        p.predicted_density = ph.R(k);
        p.previous_pressure_adjoint = pressure_adjoint_[prev];
        p.predicted_density_adjoint = predicted_density_adjoint_;
        p.relaxation_adjoint = relaxation_adjoint;
        if (int rc = check(launch_pressure_vjp(s, p, block), "pressure reverse")) return rc;
        DensityVjpLaunch d{};
        d.st = st;
        d.positions = ph.X(k);
        d.density_adjoint = predicted_density_adjoint_;
        d.walk = 2;
        d.displacement_slot = ph.first_slot + k - 1u;
        d.x = X;
        d.v = V;
        d.pa = pa;
        d.predicted = 1;
        d.acceleration = ph.A(k - 1);
        d.base = base;
        d.non_pressure_adjoint = non_pressure_adjoint_;
        d.acceleration_adjoint = acceleration_adjoint_[prev];
        d.base_adjoint = base_adjoint;
        if (int rc = check(launch_density_vjp(s, d, block), "predicted density reverse")) return rc;
        cur = prev;
        return PBF_SUCCESS;
    };
    // The pressure pass of an iteration-0 pressure (DFSPH's warm starts): no update before it.
    auto reverse_warm_pressure = [&](const Phase& ph, double* warm_adjoint) -> int {
        PressureVjpLaunch p{};
        p.st = st;
        p.pressure = ph.P(0);
        p.acceleration_adjoint = acceleration_adjoint_[cur];
        p.pressure_adjoint = pressure_adjoint_[cur];
        p.density_adjoint = density_adjoint_;
        p.x = X;
        p.pa = pa;
        p.method = 0u;
        p.warm_adjoint = warm_adjoint;
        return check(launch_pressure_vjp(s, p, block), "pressure reverse");
    };
    const Phase& p0 = r.phase[0];
    if (method == SPH_METHOD_PCISPH || method == SPH_METHOD_IISPH) {
        const uint32_t K = p0.iterations;
        if (int rc = check(launch_predict_vjp(s, st, p0.A(K), nullptr, nx, nv, X, V, non_pressure_adjoint_, acceleration_adjoint_[cur],
                                              nullptr, nullptr, pressure_adjoint_[cur]),
                           "prediction reverse"))
            return rc;
        for (uint32_t k = K; k >= 1u; --k)
            if (int rc = reverse_iteration(p0, k, 0u, 0u, pa.method0, nullptr, nullptr)) return rc;
    } else {
        const Phase& p1 = r.phase[1];
        const uint32_t Kd = p0.iterations, Kr = p1.iterations;
        const bool warm = config_.pressure_warm_start != 0;
        const float4* divergence = p0.A(Kd);
        const double* next_warm_density = next_method_adjoint ? next_method_adjoint->warm_density_pressure : nullptr;
        const double* next_warm_divergence = next_method_adjoint ? next_method_adjoint->warm_divergence_pressure : nullptr;
        if (warm && (!previous_method_adjoint || !previous_method_adjoint->warm_divergence_pressure ||
                     !previous_method_adjoint->warm_density_pressure)) {
            set_error("DFSPH with warm starts needs previous_method_adjoint");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        if (int rc = check(launch_predict_vjp(s, st, p1.A(Kr), divergence, nx, nv, X, V, non_pressure_adjoint_, acceleration_adjoint_[cur],
                                              divergence_adjoint_, next_warm_density, pressure_adjoint_[cur]),
                           "prediction reverse"))
            return rc;
        for (uint32_t k = Kr; k >= 1u; --k)
            if (int rc = reverse_iteration(p1, k, 1u, 0u, pa.method1, divergence, divergence_adjoint_)) return rc;
        if (int rc = reverse_warm_pressure(p1, warm ? previous_method_adjoint->warm_density_pressure : nullptr)) return rc;
        if (int rc = check(launch_phase_seed(s, count_, r.sorted_index, divergence_adjoint_, acceleration_adjoint_[cur],
                                             next_warm_divergence, pressure_adjoint_[cur]),
                           "phase switch"))
            return rc;
        for (uint32_t k = Kd; k >= 1u; --k)
            if (int rc = reverse_iteration(p0, k, 0u, 1u, pa.method0, nullptr, nullptr)) return rc;
        if (int rc = reverse_warm_pressure(p0, warm ? previous_method_adjoint->warm_divergence_pressure : nullptr)) return rc;
    }
    if (int rc = check(launch_non_pressure_vjp(s, st, non_pressure_adjoint_, X, V, C, density_adjoint_, pa, block),
                       "non-pressure reverse"))
        return rc;
    return density_step();
}

// SPH<Method>::jvp_step (sph/sph.ixx:356-359): the density's tangent, then Method::jvp
// (sph/sph.cpp:227-237, 314-330, 427-443, 612-659) over the iterates the forward kept.
int SphEngine::tangent(const pbf_particle_state* state, const SphRecord& r, const pbf_particle_state_tangent* state_tangent,
                       const sph_method_state* method_tangent, const pbf_control* control_tangent,
                       const sph_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_tangent,
                       sph_method_state* next_method_tangent) {
    if (!differentiable_) {
        set_error("jvp_step needs a solver created in PBF_EXECUTION_DIFFERENTIABLE mode");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    if (!state || !state_tangent || !control_tangent || !next_tangent) {
        set_error("null argument");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!r.valid || !r.differentiable || r.step_index != state->step_index) {
        set_error("the step cache does not hold the forward step of this state");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (count_ == 0) return PBF_SUCCESS;
    auto has = [](const pbf_vector_field& f) { return f.x && f.y && f.z; };
    if (!has(state_tangent->positions) || !has(state_tangent->velocities) || !has(control_tangent->external_accelerations) ||
        !has(next_tangent->positions) || !has(next_tangent->velocities)) {
        set_error("null tangent field pointer");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!tangent_x_) {
        tangent_arena_.set_stream(stream_);
        cudaError_t e = cudaSuccess;
        const size_t n = count_;
        tangent_x_ = tangent_arena_.alloc<float4>(n, e);
        tangent_v_ = tangent_arena_.alloc<float4>(n, e);
        tangent_a_ = tangent_arena_.alloc<float4>(n, e);
        tangent_b_ = tangent_arena_.alloc<float4>(n, e);
        tangent_density_ = tangent_arena_.alloc<float>(n, e);
        for (auto& p : tangent_pressure_) p = tangent_arena_.alloc<float>(n, e);
        tangent_non_pressure_ = tangent_arena_.alloc<float4>(n, e);
        tangent_predicted_ = tangent_arena_.alloc<float4>(n, e);
        tangent_divergence_ = tangent_arena_.alloc<float4>(n, e);
        if (int rc = check(e, "tangent workspace")) {
            tangent_arena_.release();
            tangent_x_ = nullptr;
            return rc;
        }
    }
    const uint32_t method = config_.method;
    SphParameterTangents pt{};
    if (parameter_tangent) {
        const sph_parameter_tangent& q = *parameter_tangent;
        pt = {q.masses, q.rest_densities, q.viscosities, q.surface_tensions, nullptr, nullptr, nullptr};
        if (method == SPH_METHOD_WCSPH) {
            pt.method0 = q.speed_of_sound;
            pt.method1 = q.tait_exponent;
            pt.method2 = q.boundary_surface_tension;
        } else if (method == SPH_METHOD_PCISPH) {
            pt.method0 = q.pressure_relaxation;
        } else if (method == SPH_METHOD_IISPH) {
            pt.method0 = q.jacobi_relaxation;
        } else {
            pt.method0 = q.divergence_relaxation;
            pt.method1 = q.density_relaxation;
        }
    }
    const cudaStream_t s = stream_;
    const unsigned block = shape.block;
    SphTangentStep t{step_of(r), tangent_x_, tangent_v_, tangent_a_, tangent_b_, tangent_density_, tangent_pressure_[0],
                     tangent_non_pressure_, tangent_predicted_};
    const Field3 tx{state_tangent->positions.x, state_tangent->positions.y, state_tangent->positions.z};
    const Field3 tv{state_tangent->velocities.x, state_tangent->velocities.y, state_tangent->velocities.z};
    const Field3 tc{control_tangent->external_accelerations.x, control_tangent->external_accelerations.y,
                    control_tangent->external_accelerations.z};
    const MutField3 out_x{next_tangent->positions.x, next_tangent->positions.y, next_tangent->positions.z};
    const MutField3 out_v{next_tangent->velocities.x, next_tangent->velocities.y, next_tangent->velocities.z};
    if (int rc = check(launch_tangent_seed(s, t, tx, tv, pt), "tangent seed")) return rc;
    const bool warm = method == SPH_METHOD_DFSPH && config_.pressure_warm_start != 0;
    const float* warm_divergence = warm && method_tangent ? method_tangent->warm_divergence_pressure : nullptr;
    const float* warm_density = warm && method_tangent ? method_tangent->warm_density_pressure : nullptr;
    if (int rc = check(launch_density_jvp(s, t, method, warm_divergence, block), "density tangent")) return rc;
    const Phase& p0 = r.phase[0];
    if (method == SPH_METHOD_WCSPH)
        return check(launch_wcsph_force_jvp(s, t, p0.P(0), r.total_acceleration, tc, out_x, out_v, block), "force tangent");
    auto iterate = [&](const SphTangentStep& tp, const Phase& ph, const uint32_t k, const uint32_t relaxation,
                       const uint32_t target) {
        const PredictedJvp u{method, relaxation, target, ph.first_slot + k - 1u, ph.X(k), ph.R(k), ph.P(k - 1u)};
        return check(launch_predicted_density_jvp(s, tp, u, block), "predicted density tangent");
    };
    if (method == SPH_METHOD_PCISPH || method == SPH_METHOD_IISPH) {
        const uint32_t K = p0.iterations;
        if (int rc = check(launch_non_pressure_jvp(s, t, tc, K > 0 ? 1 : 2, out_x, out_v, block), "non-pressure tangent"))
            return rc;
        for (uint32_t k = 1; k <= K; ++k) {
            if (int rc = iterate(t, p0, k, 0u, 0u)) return rc;
            PressureJvp u{};
            u.pressure = p0.P(k);
            u.acceleration = p0.A(k);
            u.last = k == K ? 1 : 0;
            u.out_x = out_x;
            u.out_v = out_v;
            if (int rc = check(launch_pressure_jvp(s, t, u, block), "pressure tangent")) return rc;
        }
        return PBF_SUCCESS;
    }
    // DFSPH: the divergence phase on tangent buffer 0, the density phase on buffer 1
    if (int rc = check(launch_non_pressure_jvp(s, t, tc, 0, out_x, out_v, block), "non-pressure tangent")) return rc;
    const Phase& p1 = r.phase[1];
    const uint32_t Kd = p0.iterations, Kr = p1.iterations;
    SphTangentStep t1 = t;
    t1.pressure = tangent_pressure_[1];
    for (uint32_t k = 0; k <= Kd; ++k) {
        if (k > 0) {
            if (int rc = iterate(t, p0, k, 0u, 1u)) return rc;
        }
        PressureJvp u{};
        u.pressure = p0.P(k);
        u.acceleration = p0.A(k);
        if (k == Kd) {
            u.store = tangent_divergence_;
            u.warm_out = next_method_tangent ? next_method_tangent->warm_divergence_pressure : nullptr;
            u.next_pressure = tangent_pressure_[1];
            u.next_warm = warm_density;
        }
        if (int rc = check(launch_pressure_jvp(s, t, u, block), "pressure tangent")) return rc;
    }
    for (uint32_t k = 0; k <= Kr; ++k) {
        if (k > 0) {
            if (int rc = iterate(t1, p1, k, 1u, 0u)) return rc;
        }
        PressureJvp u{};
        u.pressure = p1.P(k);
        u.acceleration = p1.A(k);
        u.base = p0.A(Kd);
        u.base_tangent = tangent_divergence_;
        if (k == Kr) {
            u.last = 1;
            u.out_x = out_x;
            u.out_v = out_v;
            u.warm_out = next_method_tangent ? next_method_tangent->warm_density_pressure : nullptr;
        }
        if (int rc = check(launch_pressure_jvp(s, t1, u, block), "pressure tangent")) return rc;
    }
    return PBF_SUCCESS;
}

int SphEngine::read(const SphRecord& r, const sph_cache_field field, float* x, float* y, float* z) {
    if (!r.valid) {
        set_error("the step cache holds no forward step");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    auto vec = [&](const float4* v) -> int {
        if (!v) {
            set_error("this field is not part of this method's cache");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        if (!x || !y || !z) {
            set_error("null destination");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        return check(launch_unsort_float4(stream_, count_, r.sorted_index, v, 3, x, y, z, nullptr), "read cache");
    };
    auto scalar = [&](const float* v) -> int {
        if (!v) {
            set_error("this field is not part of this method's cache");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        if (!x) {
            set_error("null destination");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        return check(launch_unsort_scalar(stream_, count_, r.sorted_index, v, sizeof(float), x), "read cache");
    };
    const bool w = config_.method == SPH_METHOD_WCSPH;
    switch (field) {
        case SPH_CACHE_DENSITIES: return scalar(r.density);
        case SPH_CACHE_PRESSURES: return scalar(r.final_pressure);
        case SPH_CACHE_PRESSURE_ACCELERATIONS: return vec(r.final_acceleration);
        case SPH_CACHE_VISCOSITY_ACCELERATIONS: return vec(w ? r.viscosity_acceleration : r.non_pressure);
        case SPH_CACHE_SURFACE_ACCELERATIONS: return vec(r.surface_acceleration);
        case SPH_CACHE_PREDICTED_DENSITIES: return scalar(r.final_predicted_density);
        default: break;
    }
    set_error("unknown cache field");
    return PBF_ERROR_INVALID_ARGUMENT;
}

}  // namespace sph
}  // namespace pbf

struct sph_solver {
    pbf::sph::SphEngine engine;
};

struct sph_step_cache {
    sph_solver* solver = nullptr;
    pbf::sph::SphRecord record;
};

namespace {

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        pbf::set_error("host allocation failed");
        return PBF_ERROR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        pbf::set_error(e.what());
        return PBF_ERROR_CUDA;
    } catch (...) {
        pbf::set_error("unknown failure");
        return PBF_ERROR_CUDA;
    }
}

int null_arg(const char* what) {
    pbf::set_error(std::string("null argument: ") + what);
    return PBF_ERROR_INVALID_ARGUMENT;
}

}  // namespace

extern "C" {

int sph_create(const pbf_domain_configuration* domain, const sph_configuration* configuration, const pbf_execution_mode mode,
               void* cuda_stream, sph_solver** solver) {
    if (!solver) return null_arg("solver");
    *solver = nullptr;
    if (!domain) return null_arg("domain");
    if (!configuration) return null_arg("configuration");
    return guarded([&] {
        auto s = std::make_unique<sph_solver>();
        const int rc = s->engine.init(domain, configuration, mode, static_cast<cudaStream_t>(cuda_stream));
        if (rc) return rc;
        *solver = s.release();
        return static_cast<int>(PBF_SUCCESS);
    });
}

int sph_destroy(sph_solver* solver) {
    if (!solver) return PBF_SUCCESS;
    return guarded([&] {
        delete solver;
        return static_cast<int>(PBF_SUCCESS);
    });
}

int sph_allocate_step_cache(sph_solver* solver, sph_step_cache** cache) {
    if (!cache) return null_arg("cache");
    *cache = nullptr;
    if (!solver) return null_arg("solver");
    return guarded([&] {
        auto c = std::make_unique<sph_step_cache>();
        c->solver = solver;
        const int rc = solver->engine.allocate(c->record);
        if (rc) return rc;
        *cache = c.release();
        return static_cast<int>(PBF_SUCCESS);
    });
}

int sph_free_step_cache(sph_solver* solver, sph_step_cache* cache) {
    if (!cache) return PBF_SUCCESS;
    if (!solver || cache->solver != solver) {
        pbf::set_error("the step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] {
        cudaStreamSynchronize(solver->engine.stream());
        delete cache;
        return static_cast<int>(PBF_SUCCESS);
    });
}

int sph_forward_step(sph_solver* solver, const pbf_particle_state* state, const sph_method_state* method_state,
                     const pbf_control* control, const sph_parameters* parameters, pbf_particle_state* next_state,
                     sph_method_state* next_method_state, sph_step_cache* cache) {
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    if (cache->solver != solver) {
        pbf::set_error("the step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] {
        return solver->engine.forward(state, method_state, control, parameters, next_state, next_method_state, cache->record);
    });
}

int sph_jvp_step(sph_solver* solver, const pbf_particle_state* state, const sph_method_state* method_state,
                 const pbf_control* control, const sph_parameters* parameters, const pbf_particle_state* next_state,
                 const sph_step_cache* cache, const pbf_particle_state_tangent* state_tangent,
                 const sph_method_state* method_tangent, const pbf_control* control_tangent,
                 const sph_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_tangent,
                 sph_method_state* next_method_tangent) {
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    (void)method_state;
    (void)control;
    (void)parameters;
    (void)next_state;
    if (cache->solver != solver) {
        pbf::set_error("the step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] {
        return solver->engine.tangent(state, cache->record, state_tangent, method_tangent, control_tangent, parameter_tangent,
                                      next_tangent, next_method_tangent);
    });
}

int sph_vjp_step(sph_solver* solver, const pbf_particle_state* state, const sph_method_state* method_state,
                 const pbf_control* control, const sph_parameters* parameters, const pbf_particle_state* next_state,
                 const sph_step_cache* cache, const pbf_particle_state_adjoint* next_adjoint,
                 const sph_method_state_adjoint* next_method_adjoint, pbf_particle_state_adjoint* previous_adjoint,
                 sph_method_state_adjoint* previous_method_adjoint, pbf_control_adjoint* control_adjoint,
                 sph_parameter_adjoint* parameter_adjoint) {
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    (void)control;
    (void)next_state;
    if (cache->solver != solver) {
        pbf::set_error("the step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] {
        return solver->engine.reverse(state, method_state, parameters, cache->record, next_adjoint, next_method_adjoint,
                                      previous_adjoint, previous_method_adjoint, control_adjoint, parameter_adjoint);
    });
}

}  // extern "C"

namespace {

// Copies (or FP64 accumulations) of the six particle fields and, for DFSPH, the two warm-start
// pressure fields.
template <class T>
int copy_fields(sph_solver* solver, const T* const* src, T* const* dst, const int fields, const bool accumulate) {
    pbf::sph::SphEngine& en = solver->engine;
    const size_t n = en.count();
    if (n == 0) return PBF_SUCCESS;
    for (int k = 0; k < fields; ++k)
        if (!src[k] || !dst[k]) return null_arg("field");
    if (!accumulate) {
        for (int k = 0; k < fields; ++k)
            if (int rc = en.check(cudaMemcpyAsync(dst[k], src[k], n * sizeof(T), cudaMemcpyDeviceToDevice, en.stream()), "copy"))
                return rc;
        return PBF_SUCCESS;
    }
    if constexpr (std::is_same_v<T, double>) {
        for (int k = 0; k < fields; k += 6) {
            const int count = fields - k < 6 ? fields - k : 6;
            if (int rc = en.check(pbf::launch_accumulate(en.stream(), n, src + k, dst + k, count), "accumulate")) return rc;
        }
    }
    return PBF_SUCCESS;
}

template <class State, class Method, class T>
int copy_state_like(sph_solver* solver, const State* source, const Method* source_method, State* destination,
                    Method* destination_method, const bool accumulate) {
    if (!solver || !source || !destination) return null_arg("solver/source/destination");
    const bool dfsph = solver->engine.dfsph();
    if (dfsph && (!source_method || !destination_method)) return null_arg("DFSPH method state");
    const T* src[8] = {source->positions.x, source->positions.y, source->positions.z,
                       source->velocities.x, source->velocities.y, source->velocities.z,
                       dfsph ? source_method->warm_divergence_pressure : nullptr,
                       dfsph ? source_method->warm_density_pressure : nullptr};
    T* dst[8] = {destination->positions.x, destination->positions.y, destination->positions.z,
                 destination->velocities.x, destination->velocities.y, destination->velocities.z,
                 dfsph ? destination_method->warm_divergence_pressure : nullptr,
                 dfsph ? destination_method->warm_density_pressure : nullptr};
    return guarded([&] { return copy_fields<T>(solver, src, dst, dfsph ? 8 : 6, accumulate); });
}

}  // namespace

extern "C" {

int sph_copy_state(sph_solver* solver, const pbf_particle_state* source, const sph_method_state* source_method,
                   pbf_particle_state* destination, sph_method_state* destination_method) {
    const int rc = copy_state_like<pbf_particle_state, sph_method_state, float>(solver, source, source_method, destination,
                                                                               destination_method, false);
    if (rc == PBF_SUCCESS) destination->step_index = source->step_index;
    return rc;
}

int sph_copy_state_tangent(sph_solver* solver, const pbf_particle_state_tangent* source, const sph_method_state* source_method,
                           pbf_particle_state_tangent* destination, sph_method_state* destination_method) {
    return copy_state_like<pbf_particle_state_tangent, sph_method_state, float>(solver, source, source_method, destination,
                                                                               destination_method, false);
}

int sph_copy_state_adjoint(sph_solver* solver, const pbf_particle_state_adjoint* source,
                           const sph_method_state_adjoint* source_method, pbf_particle_state_adjoint* destination,
                           sph_method_state_adjoint* destination_method) {
    return copy_state_like<pbf_particle_state_adjoint, sph_method_state_adjoint, double>(solver, source, source_method,
                                                                                        destination, destination_method, false);
}

int sph_accumulate_state_adjoint(sph_solver* solver, const pbf_particle_state_adjoint* source,
                                 const sph_method_state_adjoint* source_method, pbf_particle_state_adjoint* destination,
                                 sph_method_state_adjoint* destination_method) {
    return copy_state_like<pbf_particle_state_adjoint, sph_method_state_adjoint, double>(solver, source, source_method,
                                                                                        destination, destination_method, true);
}

int sph_read_cache(sph_solver* solver, const sph_step_cache* cache, const sph_cache_field field, float* x, float* y, float* z) {
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    if (cache->solver != solver) {
        pbf::set_error("the step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] { return solver->engine.read(cache->record, field, x, y, z); });
}

int sph_reference_gradient_norm(const sph_solver* solver, float* value) {
    if (!solver) return null_arg("solver");
    if (!value) return null_arg("value");
    *value = solver->engine.reference_gradient_norm();
    return PBF_SUCCESS;
}

int sph_set_launch_shape(sph_solver* solver, const pbf_launch_shape* shape) {
    if (!solver) return null_arg("solver");
    if (!shape) return null_arg("shape");
    const pbf::LaunchShape s{shape->list_scan, shape->scan_block_size, shape->block_size};
    if (!pbf::valid_shape(s)) {
        pbf::set_error("invalid launch shape");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    solver->engine.shape = s;
    return PBF_SUCCESS;
}

int sph_get_launch_shape(const sph_solver* solver, pbf_launch_shape* shape) {
    if (!solver) return null_arg("solver");
    if (!shape) return null_arg("shape");
    shape->list_scan = solver->engine.shape.scan;
    shape->scan_block_size = solver->engine.shape.scan_block;
    shape->block_size = solver->engine.shape.block;
    return PBF_SUCCESS;
}

int sph_synchronize(sph_solver* solver) {
    if (!solver) return null_arg("solver");
    return guarded([&] { return solver->engine.check(cudaStreamSynchronize(solver->engine.stream()), "synchronize"); });
}

void* sph_stream(const sph_solver* solver) { return solver ? static_cast<void*>(solver->engine.stream()) : nullptr; }

}  // extern "C"
