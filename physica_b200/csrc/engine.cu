// Engine: scene table, buffers and the forward launch sequence of one substep.
//
// Forward substep (reference orchestration pbf/pbf.cpp:167-191):
//   grid build (predict + key + stable counting sort + reorder)      5 kernels + memset
//   K x [density+lambda, correction+project(+reconstruct on the last)]  2K kernels
//   vorticity(+magnitude), normal(+confinement), XSPH(+write-back)      3 kernels
// All launches are asynchronous on the engine's stream; nothing synchronises.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "engine.h"

namespace pbf {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
}  // namespace

void set_error(const std::string& message) { g_last_error = message; }
const char* last_error_cstr() { return g_last_error.c_str(); }
void count_launch(const unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

const char* pass_name(const int pass) {
    static const char* names[kPassCount] = {"grid_build", "list_scan", "density_lambda", "correction_project", "vorticity",
                                            "normal_confinement", "xsph", "adjoint_seed", "xsph_vjp", "normal_vjp",
                                            "vorticity_vjp", "correction_vjp", "lambda_vjp", "density_vjp",
                                            "tangent_seed", "density_lambda_jvp", "correction_jvp", "vorticity_jvp",
                                            "normal_jvp", "xsph_jvp", "list_scan_density_lambda", "host_upload",
                                            "host_download"};
    return pass >= 0 && pass < kPassCount ? names[pass] : "unknown";
}

PassTimer::~PassTimer() {
    for (auto& m : pending_) {
        cudaEventDestroy(m.start);
        cudaEventDestroy(m.end);
    }
    for (cudaEvent_t ev : pool_) cudaEventDestroy(ev);
    if (open_) cudaEventDestroy(open_);
}

void PassTimer::enable(const bool on) {
    enabled_ = on;
    for (int p = 0; p < kPassCount; ++p) {
        ms_[p] = 0.0;
        launches_[p] = 0;
    }
}

cudaEvent_t PassTimer::take() {
    if (!pool_.empty()) {
        cudaEvent_t ev = pool_.back();
        pool_.pop_back();
        return ev;
    }
    cudaEvent_t ev = nullptr;
    cudaEventCreate(&ev);
    return ev;
}

// Every pass is also an NVTX range named after it (a no-op unless a profiler is attached).
void PassTimer::begin(cudaStream_t stream, const int pass) {
    nvtxRangePushA(pass_name(pass));
    if (!enabled_) return;
    open_ = take();
    cudaEventRecord(open_, stream);
}

void PassTimer::end(cudaStream_t stream, const int pass) {
    nvtxRangePop();
    if (!enabled_ || !open_) return;
    cudaEvent_t stop = take();
    cudaEventRecord(stop, stream);
    pending_.push_back({pass, open_, stop});
    open_ = nullptr;
}

int PassTimer::collect(cudaStream_t stream) {
    const cudaError_t e = cudaStreamSynchronize(stream);
    for (auto& m : pending_) {
        float ms = 0.0F;
        if (cudaEventElapsedTime(&ms, m.start, m.end) == cudaSuccess) {
            ms_[m.pass] += ms;
            launches_[m.pass] += 1;
        }
        pool_.push_back(m.start);
        pool_.push_back(m.end);
    }
    pending_.clear();
    return e == cudaSuccess ? PBF_SUCCESS : PBF_ERROR_CUDA;
}

int read_profile(Engine& engine, pbf_pass_time* passes, const uint32_t capacity, uint32_t* count) {
    if (int rc = engine.timer().collect(engine.stream())) {
        set_error("synchronise for profile");
        return rc;
    }
    uint32_t k = 0;
    for (int p = 0; p < kPassCount; ++p) {
        if (engine.timer().launches(p) == 0) continue;
        if (passes && k < capacity) passes[k] = {pass_name(p), engine.timer().launches(p), engine.timer().milliseconds(p)};
        ++k;
    }
    *count = k;
    return PBF_SUCCESS;
}

int Engine::check(const cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PBF_SUCCESS;
    cudaGetLastError();   // a non-sticky error becomes this call's status; later calls start clean
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PBF_ERROR_OUT_OF_MEMORY : PBF_ERROR_CUDA;
}

void destroy_adjoint_workspace(void* workspace);
void destroy_tangent_workspace(void* workspace);

Engine::~Engine() {
    if (stream_) cudaStreamSynchronize(stream_);
    drop_graphs();
    if (capture_stream_) cudaStreamDestroy(capture_stream_);
    destroy_adjoint_workspace(adjoint_);
    adjoint_ = nullptr;
    destroy_tangent_workspace(tangent_);
    tangent_ = nullptr;
    delete segment_;
    segment_ = nullptr;
    arena_.release();
}

static bool finite_positive(const float v) { return std::isfinite(v) && v > 0.0F; }

int Engine::init(const pbf_domain_configuration* scenes, const uint32_t scene_count, const pbf_configuration* configuration,
                 const pbf_execution_mode mode, cudaStream_t stream) {
    if (!scenes || scene_count == 0 || !configuration) {
        set_error("null configuration or zero scenes");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (mode != PBF_EXECUTION_FORWARD && mode != PBF_EXECUTION_DIFFERENTIABLE) {
        set_error("unknown execution mode");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (configuration->pressure_iterations > kMaxIterations) {
        set_error("pressure_iterations exceeds " + std::to_string(kMaxIterations));
        return PBF_ERROR_CAPACITY;
    }
    if (configuration->checkpoint_interval == 0) {
        set_error("checkpoint_interval must be at least 1");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    iterations_ = configuration->pressure_iterations;
    checkpoint_interval_ = configuration->checkpoint_interval;
    mode_ = mode;
    stream_ = stream;
    arena_.set_stream(stream);
    uint64_t total_cells = 0, total_particles = 0;
    scenes_.resize(scene_count);
    for (uint32_t s = 0; s < scene_count; ++s) {
        const pbf_domain_configuration& c = scenes[s];
        SceneHost& h = scenes_[s];
        h.config = c;
        h.config.boundary_particles = nullptr;
        if (!finite_positive(c.time_step) || !finite_positive(c.support_radius) || !std::isfinite(c.particle_radius)) {
            set_error("scene " + std::to_string(s) + ": time_step and support_radius must be finite and positive");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        if (c.boundary_particle_count > 0) {
            if (!c.boundary_particles) {
                set_error("boundary_particles is null but boundary_particle_count > 0");
                return PBF_ERROR_INVALID_ARGUMENT;
            }
            // domain/domain.cpp: the boundary set is copied at construction
            h.boundary.assign(c.boundary_particles, c.boundary_particles + c.boundary_particle_count);
        }
        const float mins[3] = {c.boundary.minimum.x, c.boundary.minimum.y, c.boundary.minimum.z};
        const float maxs[3] = {c.boundary.maximum.x, c.boundary.maximum.y, c.boundary.maximum.z};
        uint64_t cells = 1;
        for (int a = 0; a < 3; ++a) {
            // neighborhood/neighborhood.cpp:28-32: ceil((max - min) / h) in float
            const float extent = maxs[a] - mins[a];
            const float n = std::ceil(extent / c.support_radius);
            if (!(n >= 1.0F) || n > 1048576.0F) {
                set_error("scene " + std::to_string(s) + ": box extent / support_radius must be in [1, 2^20] per axis");
                return PBF_ERROR_INVALID_ARGUMENT;
            }
            h.dims[a] = static_cast<uint32_t>(n);
            cells *= h.dims[a];
        }
        h.cells = cells;
        h.cell_base = static_cast<uint32_t>(total_cells);
        h.first = static_cast<uint32_t>(total_particles);
        total_cells += cells;
        total_particles += c.particle_count;
        if (total_cells >= (1ull << 31) || total_particles >= (1ull << 31)) {
            set_error("total cells and particles must each stay below 2^31");
            return PBF_ERROR_CAPACITY;
        }
    }
    count_ = static_cast<uint32_t>(total_particles);
    cells_ = total_cells;
    cudaError_t e = cudaSuccess;
    scene_table_.resize(scene_count);
    d_scenes_ = arena_.alloc<SceneDesc>(scene_count, e);
    d_constants_ = arena_.alloc<KernelConstants>(scene_count, e);
    float* d_radii = arena_.alloc<float>(scene_count, e);
    predicted_ = arena_.alloc<float4>(count_, e);
    packed_ = alloc_packed(arena_, count_, e);
    arrival_ = arena_.alloc<uint32_t>(count_, e);
    unordered_ = arena_.alloc<uint32_t>(count_, e);
    tile_sums_ = arena_.alloc<uint32_t>(scan_tile_count(cells_ + 1), e);
    if (scene_count > 1) d_scene_of_ = arena_.alloc<uint32_t>(count_, e);
    if (int rc = check(e, "device allocation")) return rc;
    std::vector<float> radii(scene_count);
    for (uint32_t s = 0; s < scene_count; ++s) radii[s] = scenes_[s].config.support_radius;
    e = cudaMemcpyAsync(d_radii, radii.data(), radii.size() * sizeof(float), cudaMemcpyHostToDevice, stream_);
    if (int rc = check(e, "upload support radii")) return rc;
    if (int rc = check(launch_constants(stream_, d_radii, scene_count, d_constants_), "kernel constants")) return rc;
    if (scene_count > 1) {
        std::vector<uint32_t> scene_of(count_);
        for (uint32_t s = 0; s < scene_count; ++s)
            for (uint32_t i = 0; i < scenes_[s].config.particle_count; ++i) scene_of[scenes_[s].first + i] = s;
        e = cudaMemcpyAsync(d_scene_of_, scene_of.data(), scene_of.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_);
        if (int rc = check(e, "upload scene table")) return rc;
        e = cudaStreamSynchronize(stream_);
        if (int rc = check(e, "synchronise")) return rc;
    }
    // Boundary particles of every scene, concatenated.
    uint64_t boundary_total = 0;
    for (const SceneHost& h : scenes_) boundary_total += h.boundary.size();
    if (boundary_total >= (1ull << 31)) {
        set_error("boundary particles must stay below 2^31");
        return PBF_ERROR_CAPACITY;
    }
    boundary_count_ = static_cast<uint32_t>(boundary_total);
    if (boundary_count_ > 0) {
        std::vector<float4> rest, velocity;
        std::vector<uint32_t> scene_of;
        for (uint32_t s = 0; s < scene_count; ++s)
            for (const pbf_boundary_particle& b : scenes_[s].boundary) {
                rest.push_back(make_float4(b.position.x, b.position.y, b.position.z, b.volume));
                velocity.push_back(make_float4(b.velocity.x, b.velocity.y, b.velocity.z, 0.0F));
                scene_of.push_back(s);
            }
        boundary_rest_ = arena_.alloc<float4>(boundary_count_, e);
        boundary_velocity_ = arena_.alloc<float4>(boundary_count_, e);
        boundary_keys_ = arena_.alloc<uint32_t>(boundary_count_, e);
        boundary_arrival_ = arena_.alloc<uint32_t>(boundary_count_, e);
        boundary_unordered_ = arena_.alloc<uint32_t>(boundary_count_, e);
        if (scene_count > 1) boundary_scene_ = arena_.alloc<uint32_t>(boundary_count_, e);
        if (int rc = check(e, "device allocation")) return rc;
        e = cudaMemcpyAsync(boundary_rest_, rest.data(), rest.size() * sizeof(float4), cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(boundary_velocity_, velocity.data(), velocity.size() * sizeof(float4), cudaMemcpyHostToDevice,
                                stream_);
        if (e == cudaSuccess && boundary_scene_)
            e = cudaMemcpyAsync(boundary_scene_, scene_of.data(), scene_of.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);   // the host vectors go out of scope
        if (int rc = check(e, "upload boundary particles")) return rc;
    }
    // Time-independent scene table; the per-step fields are derived on the device from a step counter.
    std::vector<SceneStatic> statics(scene_count);
    for (uint32_t s = 0; s < scene_count; ++s) {
        const SceneHost& h = scenes_[s];
        const pbf_domain_configuration& c = h.config;
        SceneDesc& d = scene_table_[s];
        d = SceneDesc{};
        d.grid.cells_x = h.dims[0];
        d.grid.cells_y = h.dims[1];
        d.grid.cells_z = h.dims[2];
        d.grid.cell_base = h.cell_base;
        d.grid.key_min_x = c.boundary.minimum.x;
        d.grid.key_min_y = c.boundary.minimum.y;
        d.grid.key_min_z = c.boundary.minimum.z;
        d.grid.key_vel_x = c.boundary.velocity.x;
        d.grid.key_vel_y = c.boundary.velocity.y;
        d.grid.key_vel_z = c.boundary.velocity.z;
        d.grid.cell_size = c.support_radius;
        d.first = h.first;
        d.count = c.particle_count;
        d.time_step = c.time_step;
        d.inverse_time_step = 1.0F / c.time_step;   // pbf/pbf.cpp:184, evaluated on the host in float
        d.gravity_x = c.gravity.x;
        d.gravity_y = c.gravity.y;
        d.gravity_z = c.gravity.z;
        d.constants = s;
        statics[s] = {c.boundary.minimum.x, c.boundary.minimum.y, c.boundary.minimum.z, c.boundary.maximum.x,
                      c.boundary.maximum.y, c.boundary.maximum.z, c.boundary.velocity.x, c.boundary.velocity.y,
                      c.boundary.velocity.z, c.particle_radius};
    }
    d_static_ = arena_.alloc<SceneStatic>(scene_count, e);
    d_step_ = arena_.alloc<unsigned long long>(1, e);
    d_input_flags_ = arena_.alloc<uint32_t>(1, e);
    if (int rc = check(e, "device allocation")) return rc;
    e = cudaMemcpyAsync(d_scenes_, scene_table_.data(), scene_count * sizeof(SceneDesc), cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_static_, statics.data(), scene_count * sizeof(SceneStatic), cudaMemcpyHostToDevice, stream_);
    if (int rc = check(e, "upload scene table")) return rc;
    if (int rc = check(cudaMemsetAsync(d_input_flags_, 0, sizeof(uint32_t), stream_), "input flags")) return rc;
    host_step_ = ~0ull;
    if (int rc = check(cudaStreamCreateWithFlags(&capture_stream_, cudaStreamNonBlocking), "capture stream")) return rc;
    return check(cudaStreamSynchronize(stream_), "engine initialisation");
}

bool Engine::GraphKey::operator==(const GraphKey& o) const {
    if (record != o.record || positions_ready != o.positions_ready) return false;
    for (int k = 0; k < 16; ++k)
        if (p[k] != o.p[k]) return false;
    return true;
}

void Engine::drop_graphs() {
    for (auto& g : graph_cache_) cudaGraphExecDestroy(g.exec);
    graph_cache_.clear();
}

void Engine::forget(const StepRecord* record) {
    for (size_t k = 0; k < graph_cache_.size();) {
        if (graph_cache_[k].key.record == record) {
            cudaGraphExecDestroy(graph_cache_[k].exec);
            graph_cache_.erase(graph_cache_.begin() + static_cast<long>(k));
        } else {
            ++k;
        }
    }
}

int Engine::allocate_record(StepRecord& r) {
    r.arena.set_stream(stream_);
    cudaError_t e = cudaSuccess;
    const uint32_t n = count_, K = iterations_;
    const bool diff = differentiable();
    r.recompute = diff && recompute_;
    r.checkpoint_interval = checkpoint_interval_;
    const bool keep = r.keeps_all(diff);
    r.cell_offsets = r.arena.alloc<uint32_t>(cells_ + 1, e);
    r.sorted_index = r.arena.alloc<uint32_t>(n, e);
    r.slot_of = r.arena.alloc<uint32_t>(n, e);
    r.keys = r.arena.alloc<uint32_t>(n, e);
    r.cell = r.arena.alloc<int4>(n, e);
    r.topology = r.arena.alloc<float4>(n, e);
    r.params_a = r.arena.alloc<float4>(n, e);
    r.params_b = r.arena.alloc<float4>(n, e);
    const uint32_t npos = keep ? K : (K < 2 ? K : 2);
    r.positions.assign(npos, nullptr);
    for (auto& p : r.positions) p = r.arena.alloc<float4>(n, e);
    if (r.recompute) {
        r.checkpoints.assign(K ? (K + r.checkpoint_interval - 1) / r.checkpoint_interval : 0, nullptr);
        for (auto& p : r.checkpoints) p = r.arena.alloc<float4>(n, e);
    }
    r.lambda.assign(keep ? K : (K ? 1 : 0), nullptr);
    for (auto& p : r.lambda) p = r.arena.alloc<float>(n, e);
    if (keep) {
        r.density.assign(K, nullptr);
        r.gsum.assign(K, nullptr);
        for (uint32_t k = 0; k < K; ++k) {
            r.density[k] = r.arena.alloc<float>(n, e);
            r.gsum[k] = r.arena.alloc<float4>(n, e);
        }
    }
    if (diff) {
        r.mask.assign(K, nullptr);
        for (uint32_t k = 0; k < K; ++k) r.mask[k] = r.arena.alloc<uint8_t>(n, e);
    }
    r.first_density = r.arena.alloc<float>(n, e);
    r.first_lambda = r.arena.alloc<float>(n, e);
    r.neighbor_count = r.arena.alloc<uint32_t>(n, e);
    r.velocity = r.arena.alloc<float4>(n, e);
    r.vorticity = r.arena.alloc<float4>(n, e);
    r.normal = r.arena.alloc<float4>(n, e);
    r.confined = r.arena.alloc<float4>(n, e);
    // Neighbour lists: kListCapacity entries per particle, warp-interleaved.
    r.list_capacity = kListCapacity;
    const size_t padded = (static_cast<size_t>(n) + 31u) / 32u * 32u;
    const uint32_t lists = keep ? K + 1 : 1;
    r.list_entries.assign(lists, nullptr);
    r.list_counts.assign(lists, nullptr);
    for (uint32_t l = 0; l < lists; ++l) {
        r.list_entries[l] = r.arena.alloc<uint32_t>(padded * r.list_capacity, e);
        r.list_counts[l] = r.arena.alloc<uint32_t>(n, e);
    }
    if (boundary_count_ > 0) {
        r.boundary_offsets = r.arena.alloc<uint32_t>(cells_ + 1, e);
        r.boundary = r.arena.alloc<float4>(boundary_count_, e);
    }
    r.valid = false;
    if (int rc = check(e, "step cache allocation")) return rc;
    return check(cudaStreamSynchronize(stream_), "step cache allocation");
}

static bool has3(const pbf_vector_field& f) { return f.x && f.y && f.z; }

int Engine::forward(const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                    pbf_particle_state* next_state, StepRecord& r) {
    if (!state || !control || !parameters || !next_state) {
        set_error("null argument");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (count_ > 0) {
        if (!has3(state->positions) || !has3(state->velocities) || !has3(control->external_accelerations) ||
            !has3(next_state->positions) || !has3(next_state->velocities)) {
            set_error("null field pointer");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        const pbf_parameters& p = *parameters;
        if (!p.masses || !p.rest_densities || !p.relaxation || !p.artificial_pressure_strength ||
            !p.artificial_pressure_exponent || !p.artificial_pressure_radius || !p.xsph_viscosity || !p.vorticity_confinement) {
            set_error("null parameter pointer");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
    }
    // The device step counter holds the index of the state being advanced.
    if (host_step_ != state->step_index) {
        if (int rc = check(launch_set_step(stream_, d_step_, state->step_index), "step counter")) return rc;
        host_step_ = state->step_index;
    }
    int rc = PBF_SUCCESS;
    if (graphs_ && !timer_.enabled()) {
        GraphKey key{};
        const void* ptrs[16] = {state->positions.x, state->positions.y, state->positions.z, state->velocities.x,
                                state->velocities.y, state->velocities.z, control->external_accelerations.x,
                                control->external_accelerations.y, control->external_accelerations.z, parameters->masses,
                                parameters->rest_densities, parameters->relaxation, parameters->xsph_viscosity,
                                next_state->positions.x, next_state->velocities.x, parameters->vorticity_confinement};
        for (int k = 0; k < 16; ++k) key.p[k] = ptrs[k];
        key.record = &r;
        key.positions_ready = positions_ready_;
        cudaGraphExec_t exec = nullptr;
        unsigned captured_launches = 0;
        for (size_t k = 0; k < graph_cache_.size(); ++k) {
            const GraphEntry& g = graph_cache_[k];
            if (g.key == key && g.extra[0] == parameters->artificial_pressure_strength &&
                g.extra[1] == parameters->artificial_pressure_exponent && g.extra[2] == parameters->artificial_pressure_radius &&
                g.extra[3] == next_state->positions.y && g.extra[4] == next_state->positions.z &&
                g.extra[5] == next_state->velocities.y && g.extra[6] == next_state->velocities.z) {
                exec = g.exec;
                captured_launches = g.launches;
                // least recently used entries sit at the front
                std::rotate(graph_cache_.begin() + static_cast<long>(k), graph_cache_.begin() + static_cast<long>(k) + 1,
                            graph_cache_.end());
                break;
            }
        }
        if (!exec) {
            cudaGraph_t graph = nullptr;
            if ((rc = check(cudaStreamBeginCapture(capture_stream_, cudaStreamCaptureModeThreadLocal), "begin capture")))
                return rc;
            const uint64_t before = launch_count();
            rc = launch_forward(capture_stream_, state, control, parameters, next_state, r);
            captured_launches = static_cast<unsigned>(launch_count() - before);
            const cudaError_t ce = cudaStreamEndCapture(capture_stream_, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if ((rc = check(ce, "end capture"))) return rc;
            rc = check(cudaGraphInstantiate(&exec, graph, 0), "instantiate graph");
            cudaGraphDestroy(graph);
            if (rc) return rc;
            if (graph_cache_.size() >= kGraphCacheEntries) {
                cudaGraphExecDestroy(graph_cache_.front().exec);
                graph_cache_.erase(graph_cache_.begin());
            }
            GraphEntry entry{key, exec, {parameters->artificial_pressure_strength, parameters->artificial_pressure_exponent,
                                         parameters->artificial_pressure_radius, next_state->positions.y,
                                         next_state->positions.z, next_state->velocities.y, next_state->velocities.z},
                             captured_launches};
            graph_cache_.push_back(entry);
        } else {
            count_launch(captured_launches);   // the replayed kernels (capture counted them the first time)
        }
        rc = check(cudaGraphLaunch(exec, stream_), "graph launch");
    } else {
        rc = launch_forward(stream_, state, control, parameters, next_state, r);
    }
    if (rc) return rc;
    host_step_ = state->step_index + 1u;
    next_state->step_index = state->step_index + 1u;
    r.valid = true;
    r.step_index = state->step_index;
    return PBF_SUCCESS;
}

int Engine::read_input_checks(uint32_t* flags) {
    uint32_t value = 0;
    cudaError_t e = cudaMemcpyAsync(&value, d_input_flags_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_input_flags_, 0, sizeof(uint32_t), stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (int rc = check(e, "read input checks")) return rc;
    *flags = value;
    return PBF_SUCCESS;
}

GatherCommon Engine::gather_common(const StepRecord& r) const {
    GatherCommon gc{count_, d_scenes_, d_constants_, r.cell_offsets, r.cell, r.params_a, r.params_b};
    if (boundary_count_ > 0) {
        gc.boundary_offsets = r.boundary_offsets;
        gc.boundary = r.boundary;
    }
    return gc;
}

int Engine::launch_forward(cudaStream_t stream, const pbf_particle_state* state, const pbf_control* control,
                           const pbf_parameters* parameters, pbf_particle_state* next_state, StepRecord& r) {
    if (int rc = check(launch_scene_time(stream, d_static_, d_scenes_, d_step_, static_cast<uint32_t>(scenes_.size())),
                       "scene table"))
        return rc;
    const bool diff = differentiable();
    const bool keep = r.keeps_all(diff);
    const uint32_t K = iterations_;
    GridBuildArgs g{};
    g.count = count_;
    g.cells = cells_;
    g.scenes = d_scenes_;
    g.scene_of = d_scene_of_;
    g.positions = {state->positions.x, state->positions.y, state->positions.z};
    g.velocities = {state->velocities.x, state->velocities.y, state->velocities.z};
    g.controls = {control->external_accelerations.x, control->external_accelerations.y, control->external_accelerations.z};
    g.params = {parameters->masses, parameters->rest_densities, parameters->relaxation,
                parameters->artificial_pressure_strength, parameters->artificial_pressure_exponent,
                parameters->artificial_pressure_radius, parameters->xsph_viscosity, parameters->vorticity_confinement};
    g.predicted = predicted_;
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
    g.input_flags = input_checks_ ? d_input_flags_ : nullptr;
    g.packed = packed_;
    timer_.begin(stream, kPassGrid);
    if (int rc = check(launch_grid_build(stream, g), "grid build")) return rc;
    if (boundary_count_ > 0) {
        BoundaryBuildArgs b{boundary_count_, cells_, d_scenes_, boundary_scene_, boundary_rest_, boundary_velocity_,
                            boundary_keys_, boundary_arrival_, boundary_unordered_, tile_sums_, r.boundary_offsets, r.boundary};
        if (int rc = check(launch_boundary_build(stream, b), "boundary grid build")) return rc;
    }
    timer_.end(stream, kPassGrid);

    const GatherCommon gc = gather_common(r);
    const Field3 previous{state->positions.x, state->positions.y, state->positions.z};
    const MutField3 out_positions{next_state->positions.x, next_state->positions.y, next_state->positions.z};
    // Forward-mode steps of scenes without boundary particles may store hit-mask lists (launch shape).
    const int masks = stores_masks(shape_, diff, boundary_count_ > 0) ? 1 : 0;
    for (uint32_t k = 0; k < K; ++k) {
        const float4* xk = r.iterate(k, K, diff);
        float4* xk1 = const_cast<float4*>(r.iterate(k + 1, K, diff));
        float* lam = keep ? r.lambda[k] : (k == 0 ? r.first_lambda : r.lambda[0]);
        const uint32_t l = keep ? k : 0u;
        const StoredList list{r.list_entries[l], r.list_counts[l], r.list_capacity, masks};
        ListScanArgs scan{gc, xk, list, 1};
        scan.packed = packed_;
        DensityLambdaArgs d{gc, xk, lam, keep ? r.density[k] : (k == 0 ? r.first_density : nullptr),
                            keep ? r.gsum[k] : nullptr, k == 0 ? r.neighbor_count : nullptr, list};
        if (fuses_density(shape_, scan)) {
            timer_.begin(stream, kPassScanDensityLambda);
            if (int rc = check(launch_scan_density_lambda(stream, scan, d, shape_), "neighbour list scan + density/lambda"))
                return rc;
            timer_.end(stream, kPassScanDensityLambda);
        } else {
            timer_.begin(stream, kPassListScan);
            if (int rc = check(launch_list_scan(stream, scan, shape_), "neighbour list scan")) return rc;
            timer_.end(stream, kPassListScan);
            timer_.begin(stream, kPassDensityLambda);
            if (int rc = check(launch_density_lambda(stream, d, shape_.block), "density/lambda")) return rc;
            timer_.end(stream, kPassDensityLambda);
        }
        // The correction replays the list the scan has just written, last particles first (their
        // entries are the ones still in L2).
        GatherCommon gc_reverse = gc;
        gc_reverse.reverse = 1;
        CorrectionArgs c{gc_reverse, xk, lam, xk1, diff ? r.mask[k] : nullptr, k + 1 == K ? 1 : 0, previous, r.sorted_index,
                         out_positions, r.velocity, list};
        c.packed = packed_;
        timer_.begin(stream, kPassCorrection);
        if (int rc = check(launch_correction(stream, c, shape_.block), "correction/project")) return rc;
        timer_.end(stream, kPassCorrection);
    }
    const float4* xK = r.iterate(K, K, diff);
    if (K == 0) {
        if (int rc = check(launch_reconstruct(stream, count_, d_scenes_, r.cell, r.topology, previous, r.sorted_index,
                                              out_positions, r.velocity),
                           "reconstruct"))
            return rc;
    }
    // next_state.positions are final here.  Under capture the record must be external to become an
    // event node of the graph; outside a capture it is a plain record.
    if (positions_ready_) {
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        if (int rc = check(cudaStreamIsCapturing(stream, &capture), "capture status")) return rc;
        const unsigned flags = capture == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
        if (int rc = check(cudaEventRecordWithFlags(positions_ready_, stream, flags), "positions event")) return rc;
    }
    const uint32_t lp = keep ? K : 0u;
    const StoredList post{r.list_entries[lp], r.list_counts[lp], r.list_capacity, masks};
    timer_.begin(stream, kPassListScan);
    ListScanArgs post_scan{gc, xK, post};
    post_scan.packed = packed_;
    if (int rc = check(launch_list_scan(stream, post_scan, shape_), "neighbour list scan")) return rc;
    timer_.end(stream, kPassListScan);
    // The three post-loop passes replay one list in alternating directions, each starting where the
    // previous one ended.
    GatherCommon gc_reverse = gc;
    gc_reverse.reverse = 1;
    VorticityArgs v{gc_reverse, xK, r.velocity, r.vorticity, post};
    timer_.begin(stream, kPassVorticity);
    if (int rc = check(launch_vorticity(stream, v, shape_.block), "vorticity")) return rc;
    timer_.end(stream, kPassVorticity);
    NormalArgs nm{gc, xK, r.velocity, r.vorticity, r.normal, r.confined, post};
    timer_.begin(stream, kPassNormal);
    if (int rc = check(launch_normal(stream, nm, shape_.block), "normal/confinement")) return rc;
    timer_.end(stream, kPassNormal);
    XsphArgs x{gc_reverse, xK, r.confined, r.sorted_index,
               {next_state->velocities.x, next_state->velocities.y, next_state->velocities.z}, post};
    timer_.begin(stream, kPassXsph);
    if (int rc = check(launch_xsph(stream, x, shape_.block), "xsph")) return rc;
    timer_.end(stream, kPassXsph);
    return check(launch_advance_step(stream, d_step_), "step counter");
}

int Engine::segment_workspace(Segment** out) {
    if (!segment_) {
        auto* sg = new Segment();
        sg->arena.set_stream(stream_);
        const uint32_t n = count_;
        const uint32_t L = std::max(1u, std::min(checkpoint_interval_, iterations_));
        sg->length = L;
        cudaError_t e = cudaSuccess;
        sg->positions.assign(std::max(L - 1u, 2u), nullptr);
        for (auto& p : sg->positions) p = sg->arena.alloc<float4>(n, e);
        sg->lambda.assign(L, nullptr);
        sg->density.assign(L, nullptr);
        sg->gsum.assign(L, nullptr);
        sg->list_entries.assign(L, nullptr);
        sg->list_counts.assign(L, nullptr);
        const size_t padded = (static_cast<size_t>(n) + 31u) / 32u * 32u;
        for (uint32_t j = 0; j < L; ++j) {
            sg->lambda[j] = sg->arena.alloc<float>(n, e);
            sg->density[j] = sg->arena.alloc<float>(n, e);
            sg->gsum[j] = sg->arena.alloc<float4>(n, e);
            sg->list_entries[j] = sg->arena.alloc<uint32_t>(padded * kListCapacity, e);
            sg->list_counts[j] = sg->arena.alloc<uint32_t>(n, e);
        }
        if (e != cudaSuccess) {
            delete sg;
            return check(e, "recomputation workspace");
        }
        segment_ = sg;
    }
    *out = segment_;
    return PBF_SUCCESS;
}

int Engine::recompute_segment(const StepRecord& r, const uint32_t first, const uint32_t length) {
    Segment* sg = nullptr;
    if (int rc = segment_workspace(&sg)) return rc;
    const GatherCommon gc = gather_common(r);
    for (uint32_t j = 0; j < length; ++j) {
        const float4* xk = segment_iterate(r, first, j);
        const StoredList list{sg->list_entries[j], sg->list_counts[j], kListCapacity};
        // The packed copy holds the iterate written by the previous correction; the segment's first
        // iterate comes from a checkpoint, so its scan tests the float4 positions (same list).
        ListScanArgs scan{gc, xk, list, 1};
        if (j > 0) scan.packed = packed_;
        DensityLambdaArgs d{gc, xk, sg->lambda[j], sg->density[j], sg->gsum[j], nullptr, list};
        if (fuses_density(shape_, scan)) {
            if (int rc = check(launch_scan_density_lambda(stream_, scan, d, shape_), "recompute: scan + density/lambda"))
                return rc;
        } else {
            if (int rc = check(launch_list_scan(stream_, scan, shape_), "recompute: neighbour list scan")) return rc;
            if (int rc = check(launch_density_lambda(stream_, d, shape_.block), "recompute: density/lambda")) return rc;
        }
        if (j + 1 < length) {
            CorrectionArgs c{gc, xk, sg->lambda[j], sg->positions[j], nullptr, 0, Field3{}, r.sorted_index, MutField3{},
                             nullptr, list};
            c.packed = packed_;
            if (int rc = check(launch_correction(stream_, c, shape_.block), "recompute: correction/project")) return rc;
        }
    }
    return PBF_SUCCESS;
}

int Engine::autotune(const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                     pbf_particle_state* next_state, StepRecord& record, const uint32_t repeats, float* best_ms) {
    const uint32_t reps = repeats ? repeats : 1u;
    const LaunchShape previous = shape_;
    const bool graphs = graphs_;
    graphs_ = false;
    // A temporary buffer larger than the 126 MB L2, rewritten before every timed step so that each
    // step starts from cold caches as consecutive substeps of a large scene do.
    constexpr size_t kFlushBytes = size_t{256} << 20;
    DeviceArena scratch(stream_);
    cudaError_t fe = cudaSuccess;
    unsigned char* flush = scratch.alloc<unsigned char>(kFlushBytes, fe);
    if (int rc = check(fe, "autotune scratch")) {
        graphs_ = graphs;
        return rc;
    }
    // Per-pass times of `reps` steps with the current shape (after one warm-up step).
    auto measure = [&](double* pass_ms) -> int {
        pbf_particle_state out = *next_state;
        if (int rc = forward(state, control, parameters, &out, record)) return rc;
        timer_.enable(true);
        for (uint32_t k = 0; k < reps; ++k) {
            if (int rc = check(cudaMemsetAsync(flush, static_cast<int>(k + 1u), kFlushBytes, stream_), "autotune flush")) {
                timer_.enable(false);
                return rc;
            }
            out = *next_state;
            if (int rc = forward(state, control, parameters, &out, record)) {
                timer_.enable(false);
                return rc;
            }
        }
        const int rc = timer_.collect(stream_);
        for (int p = 0; p < kPassCount; ++p) pass_ms[p] = timer_.milliseconds(p) / reps;
        timer_.enable(false);
        return rc;
    };
    const uint32_t scans[5] = {kScanPerLane, kScanCooperative, kScanStaged, kScanFusedDensity, kScanFusedMasks};
    const uint32_t blocks[4] = {32u, 64u, 96u, 128u};
    double ms[kPassCount];
    int rc = PBF_SUCCESS;
    // 1. the list scan: variant x block size, by the time of the scans and the density + lambda
    //    passes (one kernel in the fused variant)
    LaunchShape best = previous;
    best.block = 128u;
    double best_scan = -1.0;
    for (int v = 0; v < 5 && !rc; ++v)
        for (int b = 0; b < 4 && !rc; ++b) {
            shape_ = best;
            shape_.scan = scans[v];
            shape_.scan_block = blocks[b];
            if ((rc = measure(ms))) break;
            const double scan_ms = ms[kPassListScan] + ms[kPassDensityLambda] + ms[kPassScanDensityLambda];
            if (best_scan < 0.0 || scan_ms < best_scan) {
                best_scan = scan_ms;
                best.scan = scans[v];
                best.scan_block = blocks[b];
            }
        }
    // 2. the gather passes' block size, by their summed time
    double best_gather = -1.0, best_total = 0.0;
    for (int b = 0; b < 4 && !rc; ++b) {
        shape_ = best;
        shape_.block = blocks[b];
        if ((rc = measure(ms))) break;
        double gather = 0.0, total = 0.0;
        for (int p = 0; p < kPassCount; ++p) total += ms[p];
        for (const int p : {kPassDensityLambda, kPassCorrection, kPassVorticity, kPassNormal, kPassXsph}) gather += ms[p];
        if (best_gather < 0.0 || gather < best_gather) {
            best_gather = gather;
            best_total = total;
            best.block = blocks[b];
        }
    }
    graphs_ = graphs;
    shape_ = rc ? previous : best;
    drop_graphs();
    if (!rc && best_ms) *best_ms = static_cast<float>(best_total);
    if (!rc) next_state->step_index = state->step_index + 1u;
    return rc;
}

int Engine::read(const StepRecord& r, const pbf_cache_field field, void* destination, const size_t bytes) {
    const uint32_t n = count_;
    const bool diff = differentiable();
    if (field == PBF_CACHE_GRID_RESOLUTION) {
        if (!destination || bytes < 3 * sizeof(uint32_t)) {
            set_error("destination too small");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        std::memcpy(destination, scenes_[0].dims, 3 * sizeof(uint32_t));
        return PBF_SUCCESS;
    }
    if (!r.valid) {
        set_error("step cache holds no step yet");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    size_t need = 0;
    switch (field) {
        case PBF_CACHE_SORTED_PARTICLE_INDICES: need = n * sizeof(uint32_t); break;
        case PBF_CACHE_CELL_OFFSETS: need = (cells_ + 1) * sizeof(uint32_t); break;
        case PBF_CACHE_SORTED_KEYS: need = n * sizeof(uint64_t); break;
        case PBF_CACHE_VORTICITY_MAGNITUDES:
        case PBF_CACHE_VORTICITY_NORMALIZERS:
        case PBF_CACHE_FIRST_DENSITIES:
        case PBF_CACHE_FIRST_LAMBDAS:
        case PBF_CACHE_NEIGHBOR_COUNTS: need = n * sizeof(float); break;
        case PBF_CACHE_PREDICTED_POSITIONS:
        case PBF_CACHE_CORRECTED_POSITIONS:
        case PBF_CACHE_RECONSTRUCTED_VELOCITIES:
        case PBF_CACHE_VORTICITIES:
        case PBF_CACHE_VORTICITY_NORMALS:
        case PBF_CACHE_CONFINED_VELOCITIES: need = 3ull * n * sizeof(float); break;
        default: set_error("unknown cache field"); return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!destination || bytes < need) {
        set_error("destination too small for the requested field");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (n == 0 && field != PBF_CACHE_CELL_OFFSETS) return PBF_SUCCESS;
    float* f = static_cast<float*>(destination);
    auto vec = [&](const float4* src) {
        return launch_unsort_float4(stream_, n, r.sorted_index, src, 3, f, f + n, f + 2ull * n, nullptr);
    };
    auto w = [&](const float4* src) { return launch_unsort_float4(stream_, n, r.sorted_index, src, 0, nullptr, nullptr, nullptr, f); };
    cudaError_t e = cudaSuccess;
    switch (field) {
        // the grid is exported in the reference's layout (x-fastest cell index), converted from the
        // z-fastest layout the solver sorts by
        case PBF_CACHE_CELL_OFFSETS:
            e = launch_reference_offsets(stream_, scene_table_.data(), static_cast<uint32_t>(scene_table_.size()), cells_,
                                         r.cell_offsets, static_cast<uint32_t*>(destination), tile_sums_);
            break;
        case PBF_CACHE_SORTED_PARTICLE_INDICES:
        case PBF_CACHE_SORTED_KEYS: {
            if (!export_offsets_) export_offsets_ = arena_.alloc<uint32_t>(cells_ + 1, e);
            if (e == cudaSuccess)
                e = launch_reference_offsets(stream_, scene_table_.data(), static_cast<uint32_t>(scene_table_.size()), cells_,
                                             r.cell_offsets, export_offsets_, tile_sums_);
            if (e == cudaSuccess)
                e = launch_reference_order(stream_, n, d_scenes_, r.cell, r.sorted_index, r.keys, r.cell_offsets, export_offsets_,
                                           field == PBF_CACHE_SORTED_PARTICLE_INDICES ? static_cast<uint32_t*>(destination) : nullptr,
                                           field == PBF_CACHE_SORTED_KEYS ? static_cast<unsigned long long*>(destination) : nullptr);
            break;
        }
        case PBF_CACHE_PREDICTED_POSITIONS: e = vec(r.topology); break;
        case PBF_CACHE_CORRECTED_POSITIONS: e = vec(r.iterate(iterations_, iterations_, diff)); break;
        case PBF_CACHE_RECONSTRUCTED_VELOCITIES: e = vec(r.velocity); break;
        case PBF_CACHE_VORTICITIES: e = vec(r.vorticity); break;
        case PBF_CACHE_VORTICITY_MAGNITUDES: e = w(r.vorticity); break;
        case PBF_CACHE_VORTICITY_NORMALS: e = vec(r.normal); break;
        case PBF_CACHE_VORTICITY_NORMALIZERS: e = w(r.normal); break;
        case PBF_CACHE_CONFINED_VELOCITIES: e = vec(r.confined); break;
        case PBF_CACHE_FIRST_DENSITIES:
            if (iterations_ == 0) { set_error("no Jacobi iteration ran"); return PBF_ERROR_INVALID_ARGUMENT; }
            e = launch_unsort_scalar(stream_, n, r.sorted_index, r.keeps_all(diff) ? r.density[0] : r.first_density, 4,
                                     destination);
            break;
        case PBF_CACHE_FIRST_LAMBDAS:
            if (iterations_ == 0) { set_error("no Jacobi iteration ran"); return PBF_ERROR_INVALID_ARGUMENT; }
            e = launch_unsort_scalar(stream_, n, r.sorted_index, r.keeps_all(diff) ? r.lambda[0] : r.first_lambda, 4,
                                     destination);
            break;
        case PBF_CACHE_NEIGHBOR_COUNTS:
            if (iterations_ == 0) { set_error("no Jacobi iteration ran"); return PBF_ERROR_INVALID_ARGUMENT; }
            e = launch_unsort_scalar(stream_, n, r.sorted_index, r.neighbor_count, 4, destination);
            break;
        default: break;
    }
    return check(e, "read step cache");
}

int Engine::read_iteration(const StepRecord& r, const pbf_iteration_field field, const uint32_t k, void* destination,
                           const size_t bytes) {
    const uint32_t n = count_, K = iterations_;
    const bool diff = differentiable();
    if (!r.valid) {
        set_error("step cache holds no step yet");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    const bool vec = field == PBF_ITERATION_POSITIONS || field == PBF_ITERATION_GRADIENT_SUMS;
    const size_t need = (vec ? 3ull : 1ull) * n * 4ull;
    if (!destination || bytes < need) {
        set_error("destination too small for the requested field");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (field == PBF_ITERATION_POSITIONS) {
        const bool kept = k == 0 || k == K || r.keeps_all(diff) || (r.recompute && r.is_checkpoint(k, K));
        if (k > K || !kept) {
            set_error("iteration positions exist for 0..K (every k only in differentiable mode; checkpoint recomputation "
                      "keeps 0, the checkpoints and K)");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
    } else if (field == PBF_ITERATION_COLLISION_MASKS ? (!diff || k >= K) : (!r.keeps_all(diff) || k >= K)) {
        set_error("per-iteration fields need differentiable mode with every iterate kept (collision masks: either form) "
                  "and iteration < K");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (n == 0) return PBF_SUCCESS;
    float* f = static_cast<float*>(destination);
    cudaError_t e = cudaSuccess;
    switch (field) {
        case PBF_ITERATION_POSITIONS:
            e = launch_unsort_float4(stream_, n, r.sorted_index, r.iterate(k, K, diff), 3, f, f + n, f + 2ull * n, nullptr);
            break;
        case PBF_ITERATION_DENSITIES: e = launch_unsort_scalar(stream_, n, r.sorted_index, r.density[k], 4, destination); break;
        case PBF_ITERATION_LAMBDAS: e = launch_unsort_scalar(stream_, n, r.sorted_index, r.lambda[k], 4, destination); break;
        case PBF_ITERATION_GRADIENT_SUMS:
            e = launch_unsort_float4(stream_, n, r.sorted_index, r.gsum[k], 3, f, f + n, f + 2ull * n, nullptr);
            break;
        case PBF_ITERATION_DENOMINATORS:
            e = launch_unsort_float4(stream_, n, r.sorted_index, r.gsum[k], 0, nullptr, nullptr, nullptr, f);
            break;
        case PBF_ITERATION_COLLISION_MASKS:
            e = launch_unsort_mask(stream_, n, r.sorted_index, r.mask[k], static_cast<uint32_t*>(destination));
            break;
        default: set_error("unknown iteration field"); return PBF_ERROR_INVALID_ARGUMENT;
    }
    return check(e, "read iteration field");
}

}  // namespace pbf
