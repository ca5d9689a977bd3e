// Batched scenes (pbf_batch_*): many independent dam breaks in one launch sequence.
#include <memory>
#include <vector>

#include "engine.h"

struct pbf_batch {
    pbf::Engine engine;
    std::vector<std::unique_ptr<pbf::StepRecord>> caches;
    pbf::DeviceArena arena;
    uint32_t* scene_first = nullptr;
    uint32_t* scene_count = nullptr;
};

extern "C" {

int pbf_batch_create(const pbf_domain_configuration* scenes, const uint32_t scene_count, const pbf_configuration* configuration,
                     const pbf_execution_mode mode, void* cuda_stream, pbf_batch** batch) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    *batch = nullptr;
    try {
        auto b = std::make_unique<pbf_batch>();
        const int rc = b->engine.init(scenes, scene_count, configuration, mode, static_cast<cudaStream_t>(cuda_stream));
        if (rc) return rc;
        b->engine.set_graphs(true);   // one graph launch per substep
        *batch = b.release();
        return PBF_SUCCESS;
    } catch (...) {
        pbf::set_error("batch creation failed");
        return PBF_ERROR_OUT_OF_MEMORY;
    }
}

int pbf_batch_destroy(pbf_batch* batch) {
    if (!batch) return PBF_SUCCESS;
    cudaStreamSynchronize(batch->engine.stream());
    delete batch;
    return PBF_SUCCESS;
}

int pbf_batch_particle_offset(const pbf_batch* batch, const uint32_t scene, uint32_t* offset, uint32_t* count) {
    if (!batch || !offset || !count) return PBF_ERROR_INVALID_ARGUMENT;
    const auto& sc = batch->engine.scenes();
    if (scene >= sc.size()) {
        pbf::set_error("scene index out of range");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    *offset = sc[scene].first;
    *count = sc[scene].config.particle_count;
    return PBF_SUCCESS;
}

int pbf_batch_reserve_caches(pbf_batch* batch, const uint32_t cache_slots) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    try {
        while (batch->caches.size() < cache_slots) {
            auto r = std::make_unique<pbf::StepRecord>();
            if (int rc = batch->engine.allocate_record(*r)) return rc;
            batch->caches.push_back(std::move(r));
        }
        return PBF_SUCCESS;
    } catch (...) {
        pbf::set_error("cache reservation failed");
        return PBF_ERROR_OUT_OF_MEMORY;
    }
}

int pbf_batch_forward_step(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                           const pbf_parameters* parameters, pbf_particle_state* next_state, const uint32_t cache_slot) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    if (int rc = pbf_batch_reserve_caches(batch, cache_slot + 1)) return rc;
    return batch->engine.forward(state, control, parameters, next_state, *batch->caches[cache_slot]);
}

int pbf_batch_vjp_step(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, const pbf_particle_state* next_state, const uint32_t cache_slot,
                       const pbf_particle_state_adjoint* next_state_adjoint, pbf_particle_state_adjoint* previous_state_adjoint,
                       pbf_control_adjoint* control_adjoint, pbf_parameter_adjoint* parameter_adjoint) {
    (void)next_state;
    if (!batch || cache_slot >= batch->caches.size()) return PBF_ERROR_INVALID_ARGUMENT;
    if (!batch->engine.differentiable()) return PBF_ERROR_NOT_DIFFERENTIABLE;
    return batch->engine.reverse(state, control, parameters, *batch->caches[cache_slot], next_state_adjoint,
                                 previous_state_adjoint, control_adjoint, parameter_adjoint);
}

int pbf_batch_jvp_step(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, const pbf_particle_state* next_state, const uint32_t cache_slot,
                       const pbf_particle_state_tangent* state_tangent, const pbf_control* control_tangent,
                       const pbf_parameter_tangent* parameter_tangent, pbf_particle_state_tangent* next_state_tangent) {
    (void)control;
    (void)parameters;
    (void)next_state;
    if (!batch || cache_slot >= batch->caches.size()) return PBF_ERROR_INVALID_ARGUMENT;
    if (!batch->engine.differentiable()) return PBF_ERROR_NOT_DIFFERENTIABLE;
    return batch->engine.tangent(state, *batch->caches[cache_slot], state_tangent, control_tangent, parameter_tangent,
                                 next_state_tangent);
}

int pbf_batch_set_input_checks(pbf_batch* batch, const int enable) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    batch->engine.set_input_checks(enable != 0);
    return PBF_SUCCESS;
}

int pbf_batch_read_input_checks(pbf_batch* batch, uint32_t* flags) {
    if (!batch || !flags) return PBF_ERROR_INVALID_ARGUMENT;
    return batch->engine.read_input_checks(flags);
}

int pbf_batch_set_launch_shape(pbf_batch* batch, const pbf_launch_shape* shape) {
    if (!batch || !shape) return PBF_ERROR_INVALID_ARGUMENT;
    const pbf::LaunchShape s{shape->list_scan, shape->scan_block_size, shape->block_size};
    if (!pbf::valid_shape(s)) {
        pbf::set_error("launch shape: list_scan must be 0 to 4 and the block sizes one of 32, 64, 96, 128");
        return PBF_ERROR_INVALID_ARGUMENT;
    }
    batch->engine.set_shape(s);
    return PBF_SUCCESS;
}

int pbf_batch_get_launch_shape(pbf_batch* batch, pbf_launch_shape* shape) {
    if (!batch || !shape) return PBF_ERROR_INVALID_ARGUMENT;
    shape->list_scan = batch->engine.shape().scan;
    shape->scan_block_size = batch->engine.shape().scan_block;
    shape->block_size = batch->engine.shape().block;
    return PBF_SUCCESS;
}

int pbf_batch_autotune(pbf_batch* batch, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, pbf_particle_state* scratch_state, const uint32_t cache_slot,
                       const uint32_t repeats, pbf_launch_shape* chosen, float* milliseconds_per_step) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    if (int rc = pbf_batch_reserve_caches(batch, cache_slot + 1)) return rc;
    if (!state || !control || !parameters || !scratch_state) return PBF_ERROR_INVALID_ARGUMENT;
    const int rc = batch->engine.autotune(state, control, parameters, scratch_state, *batch->caches[cache_slot], repeats,
                                          milliseconds_per_step);
    if (rc) return rc;
    return chosen ? pbf_batch_get_launch_shape(batch, chosen) : PBF_SUCCESS;
}

int pbf_batch_scene_sums(pbf_batch* batch, const double* values, double* result) {
    if (!batch || !values || !result) return PBF_ERROR_INVALID_ARGUMENT;
    const auto& sc = batch->engine.scenes();
    const uint32_t n = static_cast<uint32_t>(sc.size());
    if (!batch->scene_first) {
        cudaError_t e = cudaSuccess;
        batch->arena.set_stream(batch->engine.stream());
        batch->scene_first = batch->arena.alloc<uint32_t>(n, e);
        batch->scene_count = batch->arena.alloc<uint32_t>(n, e);
        if (int rc = batch->engine.check(e, "scene table")) return rc;
        std::vector<uint32_t> f(n), c(n);
        for (uint32_t s = 0; s < n; ++s) {
            f[s] = sc[s].first;
            c[s] = sc[s].config.particle_count;
        }
        e = cudaMemcpyAsync(batch->scene_first, f.data(), n * 4, cudaMemcpyHostToDevice, batch->engine.stream());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(batch->scene_count, c.data(), n * 4, cudaMemcpyHostToDevice, batch->engine.stream());
        if (e == cudaSuccess) e = cudaStreamSynchronize(batch->engine.stream());
        if (int rc = batch->engine.check(e, "scene table upload")) return rc;
    }
    return batch->engine.check(pbf::launch_segment_sums(batch->engine.stream(), values, batch->scene_first, batch->scene_count, n, 0,
                                                        result),
                               "batch scene sums");
}

int pbf_batch_set_checkpoint_recompute(pbf_batch* batch, const int enable) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    if (!batch->engine.differentiable()) {
        pbf::set_error("checkpoint recomputation needs PBF_EXECUTION_DIFFERENTIABLE");
        return PBF_ERROR_NOT_DIFFERENTIABLE;
    }
    batch->engine.set_recompute(enable != 0);
    return PBF_SUCCESS;
}

int pbf_batch_set_graph_mode(pbf_batch* batch, const int enable) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    batch->engine.set_graphs(enable != 0);
    return PBF_SUCCESS;
}

int pbf_batch_profile_enable(pbf_batch* batch, const int enable) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    batch->engine.timer().enable(enable != 0);
    return PBF_SUCCESS;
}

int pbf_batch_profile_read(pbf_batch* batch, pbf_pass_time* passes, const uint32_t capacity, uint32_t* count) {
    if (!batch || !count) return PBF_ERROR_INVALID_ARGUMENT;
    return pbf::read_profile(batch->engine, passes, capacity, count);
}

int pbf_batch_synchronize(pbf_batch* batch) {
    if (!batch) return PBF_ERROR_INVALID_ARGUMENT;
    return batch->engine.check(cudaStreamSynchronize(batch->engine.stream()), "synchronize");
}

}  // extern "C"
