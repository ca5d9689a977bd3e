// C ABI (include/physica_pbf.h) over the Engine.  No exception crosses this boundary:
// every entry point returns a pbf_status and records a message for pbf_last_error().
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "engine.h"

namespace pbf {
const char* last_error_cstr();
}

struct pbf_solver {
    pbf::Engine engine;
    // staging buffers of the *_host entry points (device), allocated on first use
    pbf::DeviceArena staging;
    float* in = nullptr;
    float* out = nullptr;
    // download stream of the *_host entry points: the positions are read back on it while the
    // post-loop passes still run on the engine's stream
    cudaStream_t download = nullptr;
    cudaEvent_t positions_ready = nullptr;
    ~pbf_solver() {
        if (positions_ready) cudaEventDestroy(positions_ready);
        if (download) cudaStreamDestroy(download);
    }
};

struct pbf_step_cache {
    pbf_solver* solver = nullptr;
    pbf::StepRecord record;
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

int pbf_abi_version(void) { return PHYSICA_PBF_ABI_VERSION; }

uint64_t pbf_launch_count(void) { return pbf::launch_count(); }

const char* pbf_last_error(void) { return pbf::last_error_cstr(); }

const char* pbf_status_string(const int status) {
    switch (status) {
        case PBF_SUCCESS: return "success";
        case PBF_ERROR_INVALID_ARGUMENT: return "invalid argument";
        case PBF_ERROR_OUT_OF_MEMORY: return "out of memory";
        case PBF_ERROR_CUDA: return "CUDA error";
        case PBF_ERROR_NOT_DIFFERENTIABLE: return "solver was created in forward mode";
        case PBF_ERROR_UNSUPPORTED: return "unsupported";
        case PBF_ERROR_DEVICE_TIMEOUT: return "device wait timed out";
        case PBF_ERROR_CAPACITY: return "capacity exceeded";
        default: return "unknown status";
    }
}

int pbf_create(const pbf_domain_configuration* domain, const pbf_configuration* configuration, const pbf_execution_mode mode,
               void* cuda_stream, pbf_solver** solver) {
    if (!solver) return null_arg("solver");
    *solver = nullptr;
    if (!domain) return null_arg("domain");
    if (!configuration) return null_arg("configuration");
    return guarded([&] {
        auto s = std::make_unique<pbf_solver>();
        const int rc = s->engine.init(domain, 1, configuration, mode, static_cast<cudaStream_t>(cuda_stream));
        if (rc) return rc;
        s->staging.set_stream(static_cast<cudaStream_t>(cuda_stream));
        *solver = s.release();
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_destroy(pbf_solver* solver) {
    if (!solver) return PBF_SUCCESS;
    return guarded([&] {
        cudaStreamSynchronize(solver->engine.stream());
        delete solver;
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_allocate_step_cache(pbf_solver* solver, pbf_step_cache** cache) {
    if (!cache) return null_arg("cache");
    *cache = nullptr;
    if (!solver) return null_arg("solver");
    return guarded([&] {
        auto c = std::make_unique<pbf_step_cache>();
        c->solver = solver;
        const int rc = solver->engine.allocate_record(c->record);
        if (rc) return rc;
        *cache = c.release();
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_free_step_cache(pbf_step_cache* cache) {
    if (!cache) return PBF_SUCCESS;
    return guarded([&] {
        cudaStreamSynchronize(cache->solver->engine.stream());
        cache->solver->engine.forget(&cache->record);
        delete cache;
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_forward_step(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                     const pbf_parameters* parameters, pbf_particle_state* next_state, pbf_step_cache* cache) {
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    if (cache->solver != solver) {
        pbf::set_error("step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] { return solver->engine.forward(state, control, parameters, next_state, cache->record); });
}

int pbf_jvp_step(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                 const pbf_parameters* parameters, const pbf_particle_state* next_state, const pbf_step_cache* cache,
                 const pbf_particle_state_tangent* state_tangent, const pbf_control* control_tangent,
                 const pbf_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_state_tangent) {
    (void)control;
    (void)parameters;
    (void)next_state;
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    if (cache->solver != solver) {
        pbf::set_error("step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    return guarded([&] {
        return solver->engine.tangent(state, cache->record, state_tangent, control_tangent, parameter_tangent, next_state_tangent);
    });
}

int pbf_vjp_step(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                 const pbf_parameters* parameters, const pbf_particle_state* next_state, const pbf_step_cache* cache,
                 const pbf_particle_state_adjoint* next_state_adjoint, pbf_particle_state_adjoint* previous_state_adjoint,
                 pbf_control_adjoint* control_adjoint, pbf_parameter_adjoint* parameter_adjoint) {
    (void)next_state;
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    if (cache->solver != solver) {
        pbf::set_error("step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!solver->engine.differentiable()) {
        pbf::set_error("vjp_step needs a solver created in PBF_EXECUTION_DIFFERENTIABLE mode");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    return guarded([&] {
        return solver->engine.reverse(state, control, parameters, cache->record, next_state_adjoint, previous_state_adjoint,
                                      control_adjoint, parameter_adjoint);
    });
}

int pbf_copy_state(pbf_solver* solver, const pbf_particle_state* source, pbf_particle_state* destination) {
    if (!solver || !source || !destination) return null_arg("solver/source/destination");
    return guarded([&] {
        const size_t bytes = static_cast<size_t>(solver->engine.count()) * sizeof(float);
        cudaStream_t st = solver->engine.stream();
        const float* src[6] = {source->positions.x, source->positions.y, source->positions.z,
                               source->velocities.x, source->velocities.y, source->velocities.z};
        float* dst[6] = {destination->positions.x, destination->positions.y, destination->positions.z,
                         destination->velocities.x, destination->velocities.y, destination->velocities.z};
        for (int k = 0; k < 6; ++k) {
            if (bytes && (!src[k] || !dst[k])) return null_arg("field");
            if (int rc = solver->engine.check(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToDevice, st), "copy_state"))
                return rc;
        }
        destination->step_index = source->step_index;
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_copy_state_tangent(pbf_solver* solver, const pbf_particle_state_tangent* source,
                           pbf_particle_state_tangent* destination) {
    if (!solver || !source || !destination) return null_arg("solver/source/destination");
    return guarded([&] {
        const size_t bytes = static_cast<size_t>(solver->engine.count()) * sizeof(float);
        cudaStream_t st = solver->engine.stream();
        const float* src[6] = {source->positions.x, source->positions.y, source->positions.z,
                               source->velocities.x, source->velocities.y, source->velocities.z};
        float* dst[6] = {destination->positions.x, destination->positions.y, destination->positions.z,
                         destination->velocities.x, destination->velocities.y, destination->velocities.z};
        for (int k = 0; k < 6; ++k) {
            if (bytes && (!src[k] || !dst[k])) return null_arg("field");
            if (int rc = solver->engine.check(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToDevice, st),
                                              "copy_state_tangent"))
                return rc;
        }
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_copy_state_adjoint(pbf_solver* solver, const pbf_particle_state_adjoint* source, pbf_particle_state_adjoint* destination) {
    if (!solver || !source || !destination) return null_arg("solver/source/destination");
    return guarded([&] {
        const size_t bytes = static_cast<size_t>(solver->engine.count()) * sizeof(double);
        cudaStream_t st = solver->engine.stream();
        const double* src[6] = {source->positions.x, source->positions.y, source->positions.z,
                                source->velocities.x, source->velocities.y, source->velocities.z};
        double* dst[6] = {destination->positions.x, destination->positions.y, destination->positions.z,
                          destination->velocities.x, destination->velocities.y, destination->velocities.z};
        for (int k = 0; k < 6; ++k) {
            if (bytes && (!src[k] || !dst[k])) return null_arg("field");
            if (int rc = solver->engine.check(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToDevice, st),
                                              "copy_state_adjoint"))
                return rc;
        }
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_accumulate_state_adjoint(pbf_solver* solver, const pbf_particle_state_adjoint* source,
                                 pbf_particle_state_adjoint* destination) {
    if (!solver || !source || !destination) return null_arg("solver/source/destination");
    return guarded([&] {
        const double* src[6] = {source->positions.x, source->positions.y, source->positions.z,
                                source->velocities.x, source->velocities.y, source->velocities.z};
        double* dst[6] = {destination->positions.x, destination->positions.y, destination->positions.z,
                          destination->velocities.x, destination->velocities.y, destination->velocities.z};
        if (solver->engine.count() > 0)
            for (int k = 0; k < 6; ++k)
                if (!src[k] || !dst[k]) return null_arg("field");
        return solver->engine.check(pbf::launch_accumulate(solver->engine.stream(), solver->engine.count(), src, dst, 6),
                                    "accumulate_state_adjoint");
    });
}

int pbf_forward_step_host(pbf_solver* solver, const pbf_host_state* state, const pbf_control* control,
                          const pbf_parameters* parameters, pbf_host_state* next_state, pbf_step_cache* cache) {
    if (!solver || !state || !next_state || !cache) return null_arg("solver/state/next_state/cache");
    return guarded([&] {
        pbf::Engine& en = solver->engine;
        const size_t n = en.count();
        cudaStream_t st = en.stream();
        if (!solver->in) {
            cudaError_t e = cudaSuccess;
            solver->in = solver->staging.alloc<float>(6 * n, e);
            solver->out = solver->staging.alloc<float>(6 * n, e);
            if (int rc = en.check(e, "staging allocation")) return rc;
        }
        if (!solver->download) {
            if (int rc = en.check(cudaStreamCreateWithFlags(&solver->download, cudaStreamNonBlocking), "download stream"))
                return rc;
            if (int rc = en.check(cudaEventCreateWithFlags(&solver->positions_ready, cudaEventDisableTiming), "download event"))
                return rc;
        }
        for (int k = 0; k < 3; ++k) {
            if (n && (!state->positions[k] || !state->velocities[k] || !next_state->positions[k] || !next_state->velocities[k]))
                return null_arg("host field");
        }
        en.timer().begin(st, pbf::kPassHostUpload);
        for (int k = 0; k < 3; ++k) {
            if (int rc = en.check(cudaMemcpyAsync(solver->in + k * n, state->positions[k], n * sizeof(float),
                                                  cudaMemcpyHostToDevice, st), "upload"))
                return rc;
            if (int rc = en.check(cudaMemcpyAsync(solver->in + (3 + k) * n, state->velocities[k], n * sizeof(float),
                                                  cudaMemcpyHostToDevice, st), "upload"))
                return rc;
        }
        en.timer().end(st, pbf::kPassHostUpload);
        pbf_particle_state in{{solver->in, solver->in + n, solver->in + 2 * n},
                              {solver->in + 3 * n, solver->in + 4 * n, solver->in + 5 * n}, state->step_index};
        pbf_particle_state out{{solver->out, solver->out + n, solver->out + 2 * n},
                               {solver->out + 3 * n, solver->out + 4 * n, solver->out + 5 * n}, 0};
        // The positions are final after the last correction: their download on the second stream
        // overlaps the post-loop passes; the velocities follow XSPH on the engine's stream.
        en.set_positions_ready_event(solver->positions_ready);
        const int frc = en.forward(&in, control, parameters, &out, cache->record);
        en.set_positions_ready_event(nullptr);
        if (frc) return frc;
        cudaStream_t dl = solver->download;
        if (int rc = en.check(cudaStreamWaitEvent(dl, solver->positions_ready, 0), "download wait")) return rc;
        int rc = PBF_SUCCESS;
        // profiled: the two downloads are timed on their own streams and summed under host_download
        en.timer().begin(dl, pbf::kPassHostDownload);
        for (int k = 0; k < 3 && !rc; ++k)
            rc = en.check(cudaMemcpyAsync(next_state->positions[k], solver->out + k * n, n * sizeof(float),
                                          cudaMemcpyDeviceToHost, dl), "download");
        en.timer().end(dl, pbf::kPassHostDownload);
        en.timer().begin(st, pbf::kPassHostDownload);
        for (int k = 0; k < 3 && !rc; ++k)
            rc = en.check(cudaMemcpyAsync(next_state->velocities[k], solver->out + (3 + k) * n, n * sizeof(float),
                                          cudaMemcpyDeviceToHost, st), "download");
        en.timer().end(st, pbf::kPassHostDownload);
        // both streams drain before returning, so the next call may reuse the staging buffers
        const int src = en.check(cudaStreamSynchronize(st), "forward_step_host");
        const int drc = en.check(cudaStreamSynchronize(dl), "forward_step_host download");
        if (rc) return rc;
        if (src) return src;
        if (drc) return drc;
        next_state->step_index = out.step_index;
        return static_cast<int>(PBF_SUCCESS);
    });
}

int pbf_step_cache_read(pbf_solver* solver, const pbf_step_cache* cache, const pbf_cache_field field, void* destination,
                        const size_t bytes) {
    if (!solver || !cache) return null_arg("solver/cache");
    return guarded([&] { return solver->engine.read(cache->record, field, destination, bytes); });
}

int pbf_step_cache_read_iteration(pbf_solver* solver, const pbf_step_cache* cache, const pbf_iteration_field field,
                                  const uint32_t iteration, void* destination, const size_t bytes) {
    if (!solver || !cache) return null_arg("solver/cache");
    return guarded([&] { return solver->engine.read_iteration(cache->record, field, iteration, destination, bytes); });
}

int pbf_grid_cell_count(const pbf_solver* solver, uint64_t* cells) {
    if (!solver || !cells) return null_arg("solver/cells");
    *cells = solver->engine.cells();
    return PBF_SUCCESS;
}

int pbf_sum_compensated(pbf_solver* solver, const double* values, const uint32_t count, double* result) {
    if (!solver || !result || (count && !values)) return null_arg("solver/values/result");
    return solver->engine.check(pbf::launch_segment_sums(solver->engine.stream(), values, nullptr, nullptr, 1, count, result),
                                "sum_compensated");
}

int pbf_set_checkpoint_recompute(pbf_solver* solver, const int enable) {
    if (!solver) return null_arg("solver");
    if (!solver->engine.differentiable()) {
        pbf::set_error("checkpoint recomputation needs PBF_EXECUTION_DIFFERENTIABLE");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    solver->engine.set_recompute(enable != 0);
    return PBF_SUCCESS;
}

int pbf_set_graph_mode(pbf_solver* solver, const int enable) {
    if (!solver) return null_arg("solver");
    solver->engine.set_graphs(enable != 0);
    return PBF_SUCCESS;
}

int pbf_set_launch_shape(pbf_solver* solver, const pbf_launch_shape* shape) {
    if (!solver) return null_arg("solver");
    if (!shape) return null_arg("shape");
    const pbf::LaunchShape s{shape->list_scan, shape->scan_block_size, shape->block_size};
    if (!pbf::valid_shape(s)) {
        pbf::set_error("launch shape: list_scan must be 0 to 4 and the block sizes one of 32, 64, 96, 128");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    solver->engine.set_shape(s);
    return PBF_SUCCESS;
}

int pbf_get_launch_shape(pbf_solver* solver, pbf_launch_shape* shape) {
    if (!solver) return null_arg("solver");
    if (!shape) return null_arg("shape");
    shape->list_scan = solver->engine.shape().scan;
    shape->scan_block_size = solver->engine.shape().scan_block;
    shape->block_size = solver->engine.shape().block;
    return PBF_SUCCESS;
}

int pbf_autotune(pbf_solver* solver, const pbf_particle_state* state, const pbf_control* control,
                 const pbf_parameters* parameters, pbf_particle_state* scratch_state, pbf_step_cache* cache,
                 const uint32_t repeats, pbf_launch_shape* chosen, float* milliseconds_per_step) {
    if (!solver) return null_arg("solver");
    if (!cache) return null_arg("cache");
    if (cache->solver != solver) {
        pbf::set_error("step cache belongs to another solver");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    if (!state || !control || !parameters || !scratch_state) return null_arg("state/control/parameters/scratch_state");
    const int rc = guarded([&] {
        return solver->engine.autotune(state, control, parameters, scratch_state, cache->record, repeats, milliseconds_per_step);
    });
    if (rc) return rc;
    return chosen ? pbf_get_launch_shape(solver, chosen) : PBF_SUCCESS;
}

int pbf_export_frame(pbf_solver* solver, const pbf_particle_state* state, const pbf_step_cache* cache, pbf_frame* frame) {
    if (!solver) return null_arg("solver");
    if (!state || !frame || !frame->positions || !frame->velocities) return null_arg("state/frame");
    if (frame->vorticity) {
        if (!cache) return null_arg("cache (needed for the vorticity magnitudes)");
        if (cache->solver != solver) {
            pbf::set_error("step cache belongs to another solver");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
        if (!cache->record.valid || cache->record.step_index + 1u != state->step_index) {
            pbf::set_error("the step cache does not hold the step that produced this state");
            return PBF_ERROR_INVALID_ARGUMENT;
        }
    }
    const pbf::Field3 x{state->positions.x, state->positions.y, state->positions.z};
    const pbf::Field3 v{state->velocities.x, state->velocities.y, state->velocities.z};
    if (solver->engine.count() > 0 && (!x.x || !x.y || !x.z || !v.x || !v.y || !v.z)) return null_arg("state field");
    const pbf::StepRecord* r = frame->vorticity ? &cache->record : nullptr;
    return solver->engine.check(pbf::launch_export_frame(solver->engine.stream(), solver->engine.count(), x, v,
                                                         r ? r->slot_of : nullptr, r ? r->vorticity : nullptr,
                                                         frame->positions, frame->velocities, frame->vorticity),
                                "export frame");
}

int pbf_set_input_checks(pbf_solver* solver, const int enable) {
    if (!solver) return null_arg("solver");
    solver->engine.set_input_checks(enable != 0);
    return PBF_SUCCESS;
}

int pbf_read_input_checks(pbf_solver* solver, uint32_t* flags) {
    if (!solver) return null_arg("solver");
    if (!flags) return null_arg("flags");
    return guarded([&] { return solver->engine.read_input_checks(flags); });
}

int pbf_profile_enable(pbf_solver* solver, const int enable) {
    if (!solver) return null_arg("solver");
    solver->engine.timer().enable(enable != 0);
    return PBF_SUCCESS;
}

int pbf_profile_read(pbf_solver* solver, pbf_pass_time* passes, const uint32_t capacity, uint32_t* count) {
    if (!solver || !count) return null_arg("solver/count");
    return pbf::read_profile(solver->engine, passes, capacity, count);
}

int pbf_synchronize(pbf_solver* solver) {
    if (!solver) return null_arg("solver");
    return solver->engine.check(cudaStreamSynchronize(solver->engine.stream()), "synchronize");
}

}  // extern "C"
