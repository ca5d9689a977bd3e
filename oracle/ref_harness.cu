// Replay harness of the reference PBF and SPH -- TEST INFRASTRUCTURE ONLY.
//
// Linked with the reference's own kernel translation units (pbf/pbf.cu, density/density.cu,
// neighborhood/neighborhood.cu, domain/domain.cu of fluids/liquid/particle, compiled from the
// reference sources by oracle/build.py into oracle/_ref/libpbf_ref.so).  The reference's host
// layer is a set of C++23 module units (import std) that this toolchain cannot build, so this
// file replays PBF::forward_step (pbf/pbf.cpp:167-191) and PBF::vjp_step (pbf/pbf.cpp:217-258)
// call for call over the reference's launch_* functions, with plain cudaMalloc buffers in place
// of cuda::device_buffer.  It exists to produce golden outputs of the reference on a GPU and to
// time the reference as the baseline arm of bench.py; the product never links it.
// The SPH section at the end replays SPH<Method>::forward_step (sph/sph.ixx:350-354) and the four
// methods' forward() (sph/sph.cpp:214-225, 296-312, 409-425, 572-610) over the reference's
// sph/*.cu launchers in the same way.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <cuda/stream>

#include "density/kernels.h"
#include "domain/kernels.h"
#include "neighborhood/device.cuh"
#include "neighborhood/kernels.h"
#include "pbf/kernels.h"
#include "sph/dfsph.h"
#include "sph/iisph.h"
#include "sph/kernels.h"
#include "sph/pcisph.h"
#include "sph/wcsph.h"

namespace cd = physica::fluids::liquid::particle::cuda_detail;

namespace {

struct Vec { float* x = nullptr; float* y = nullptr; float* z = nullptr; };
struct DVec { double* x = nullptr; double* y = nullptr; double* z = nullptr; };

struct Iteration {
    float* densities;
    Vec gradient_sums;
    float* denominators;
    float* lambdas;
    Vec corrections;
    uint32_t* masks;
};

}  // namespace

extern "C" {

typedef struct {
    uint32_t particle_count;
    float time_step, support_radius, particle_radius;
    float gravity[3];
    float box_min[3], box_max[3], box_velocity[3];
    uint32_t no_slip;
    uint32_t pressure_iterations, checkpoint_interval;
    int differentiable;
} ref_config;

typedef struct {
    const float* px; const float* py; const float* pz;
    const float* vx; const float* vy; const float* vz;
} ref_state_in;

typedef struct {
    float* px; float* py; float* pz;
    float* vx; float* vy; float* vz;
} ref_state_out;

typedef struct {
    const float* masses; const float* rest_densities; const float* relaxation;
    const float* strength; const float* exponent; const float* radius;
    const float* xsph; const float* vorticity;
} ref_params;

typedef struct {
    double* px; double* py; double* pz;
    double* vx; double* vy; double* vz;
} ref_adjoint_state;

typedef struct {
    double* masses; double* rest_densities; double* relaxation;
    double* strength; double* exponent; double* radius;
    double* xsph; double* vorticity;
} ref_param_adjoint;

}  // extern "C"

namespace {

struct Harness {
    ref_config cfg{};
    cudaStream_t stream = nullptr;
    std::vector<void*> allocations;
    uint32_t cells_x = 0, cells_y = 0, cells_z = 0, cells = 0;
    // neighbourhood (neighborhood/neighborhood.ixx:321-332, neighborhood.cpp:14-42)
    uint64_t *unsorted_keys, *sorted_keys, *sorted_boundary_keys, *unsorted_boundary_keys;
    uint32_t *unsorted_indices, *sorted_indices, *cell_offsets, *sorted_boundary_indices, *unsorted_boundary_indices,
        *boundary_cell_offsets;
    void* sort_scratch = nullptr;
    size_t sort_scratch_bytes = 0;
    void* boundary_scratch = nullptr;
    size_t boundary_scratch_bytes = 0;
    float origin[3] = {0, 0, 0};
    float boundary_time = 0.0F;
    // step cache (pbf/pbf.ixx:54-70)
    Vec predicted, corrected, reconstructed, vorticities, normals, confined;
    float *magnitudes, *normalizers;
    std::vector<std::pair<uint32_t, Vec>> checkpoints;
    Iteration forward_iteration{};
    float* first_densities;
    float* first_lambdas;
    uint64_t step_index = 0;
    // differentiation workspace (pbf/pbf.ixx:107-132)
    std::vector<Vec> segment_positions;
    std::vector<Iteration> segment_iterations;
    DVec current_position_adjoint, next_position_adjoint, correction_adjoint, reconstructed_velocity_adjoint,
        vorticity_adjoint, vorticity_normal_adjoint, confined_velocity_adjoint;
    double *lambda_adjoint, *density_adjoint;
    // tangent workspace of PBF::jvp_step (allocated on first use)
    bool tangents_ready = false;
    Vec current_position_tangent, next_position_tangent, gradient_sum_tangent, correction_tangent,
        reconstructed_velocity_tangent, vorticity_tangent, vorticity_normal_tangent, confined_velocity_tangent, jvp_positions;
    float *density_tangent, *denominator_tangent, *lambda_tangent, *vorticity_magnitude_tangent;
    // boundary particles (empty unless ref_set_boundary was called)
    float* empty_f = nullptr;
    uint32_t boundary_count = 0;
    Vec boundary_positions, boundary_velocities;
    float* boundary_volumes = nullptr;

    template <class T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        allocations.push_back(p);
        return static_cast<T*>(p);
    }
    Vec vec() { const size_t n = cfg.particle_count; return {alloc<float>(n), alloc<float>(n), alloc<float>(n)}; }
    DVec dvec() { const size_t n = cfg.particle_count; return {alloc<double>(n), alloc<double>(n), alloc<double>(n)}; }
    Iteration iteration() {
        const size_t n = cfg.particle_count;
        return {alloc<float>(n), vec(), alloc<float>(n), alloc<float>(n), vec(), alloc<uint32_t>(n)};
    }
    ~Harness() {
        cudaStreamSynchronize(stream);
        for (void* p : allocations) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    cd::ConstVectorView<float> cv(const Vec& v) const { return {v.x, v.y, v.z}; }
    cd::VectorView<float> mv(const Vec& v) const { return {v.x, v.y, v.z}; }
    cd::ConstVectorView<double> cdv(const DVec& v) const { return {v.x, v.y, v.z}; }
    cd::VectorView<double> mdv(const DVec& v) const { return {v.x, v.y, v.z}; }

    cd::NeighborhoodView neighborhood() const {
        return {sorted_keys, sorted_indices, cell_offsets, sorted_boundary_keys, sorted_boundary_indices, boundary_cell_offsets,
                cfg.particle_count, boundary_count, cells_x, cells_y, cells_z, origin[0], origin[1], origin[2], cfg.support_radius};
    }
    cd::BoundaryView boundary() const {
        if (boundary_count == 0) return {empty_f, empty_f, empty_f, empty_f, empty_f, empty_f, empty_f, 0u, boundary_time};
        return {boundary_positions.x, boundary_positions.y, boundary_positions.z, boundary_velocities.x, boundary_velocities.y,
                boundary_velocities.z, boundary_volumes, boundary_count, boundary_time};
    }

    // pbf/pbf.cpp:17-31
    cd::Box collision_box(const uint64_t step) const {
        const float time = static_cast<float>(step) * cfg.time_step;
        return {cfg.box_min[0] + time * cfg.box_velocity[0] + cfg.particle_radius,
                cfg.box_min[1] + time * cfg.box_velocity[1] + cfg.particle_radius,
                cfg.box_min[2] + time * cfg.box_velocity[2] + cfg.particle_radius,
                cfg.box_max[0] + time * cfg.box_velocity[0] - cfg.particle_radius,
                cfg.box_max[1] + time * cfg.box_velocity[1] - cfg.particle_radius,
                cfg.box_max[2] + time * cfg.box_velocity[2] - cfg.particle_radius,
                cfg.box_velocity[0], cfg.box_velocity[1], cfg.box_velocity[2], cfg.no_slip};
    }

    void copy(const Vec& src, const Vec& dst) const {
        const size_t b = cfg.particle_count * sizeof(float);
        cudaMemcpyAsync(dst.x, src.x, b, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(dst.y, src.y, b, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(dst.z, src.z, b, cudaMemcpyDeviceToDevice, stream);
    }
    void clear(const DVec& v) const {
        const size_t b = cfg.particle_count * sizeof(double);
        cudaMemsetAsync(v.x, 0, b, stream);
        cudaMemsetAsync(v.y, 0, b, stream);
        cudaMemsetAsync(v.z, 0, b, stream);
    }
    void clear(double* v) const { cudaMemsetAsync(v, 0, cfg.particle_count * sizeof(double), stream); }
    void copy(const DVec& src, const DVec& dst) const {
        const size_t b = cfg.particle_count * sizeof(double);
        cudaMemcpyAsync(dst.x, src.x, b, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(dst.y, src.y, b, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(dst.z, src.z, b, cudaMemcpyDeviceToDevice, stream);
    }

    // NeighborhoodSearch::build (neighborhood/neighborhood.cpp:44-89)
    void build(const uint64_t step, const Vec& positions) {
        const cd::Box box{cfg.box_min[0], cfg.box_min[1], cfg.box_min[2], cfg.box_max[0], cfg.box_max[1], cfg.box_max[2],
                          cfg.box_velocity[0], cfg.box_velocity[1], cfg.box_velocity[2], cfg.no_slip};
        const bool b = boundary_count > 0;
        cd::build_neighborhood(::cuda::stream_ref{stream}, cfg.particle_count, boundary_count, cfg.support_radius, cfg.time_step,
                               step, box, cv(positions),
                               b ? cv(boundary_positions) : cd::ConstVectorView<float>{empty_f, empty_f, empty_f},
                               b ? cv(boundary_velocities) : cd::ConstVectorView<float>{empty_f, empty_f, empty_f},
                               unsorted_keys, unsorted_indices,
                               unsorted_boundary_keys, unsorted_boundary_indices, sort_scratch, sort_scratch_bytes,
                               boundary_scratch, boundary_scratch_bytes, sorted_keys, sorted_indices, cell_offsets,
                               sorted_boundary_keys, sorted_boundary_indices, boundary_cell_offsets);
        boundary_time = static_cast<float>(step) * cfg.time_step;
        for (int a = 0; a < 3; ++a) origin[a] = cfg.box_min[a] + boundary_time * cfg.box_velocity[a];
    }

    void iterate(const ref_params& p, const cd::ParticleParameterView& pv, const Vec& positions, Iteration& it,
                 const Vec& output, const uint64_t step) {
        const ::cuda::stream_ref s{stream};
        const uint32_t n = cfg.particle_count;
        cd::density_forward(s, n, cfg.support_radius, true, cv(predicted), cv(positions), pv, neighborhood(), boundary(),
                            it.densities);
        cd::pbf::launch_lambda_forward(s, n, cfg.support_radius, cv(predicted), cv(positions), pv, neighborhood(), boundary(),
                                       it.densities, p.relaxation, mv(it.gradient_sums), it.denominators, it.lambdas);
        cd::pbf::launch_correction_forward(s, n, cfg.support_radius, cv(predicted), cv(positions), pv, neighborhood(), boundary(),
                                           it.lambdas, p.strength, p.exponent, p.radius, mv(it.corrections));
        cd::pbf::launch_project_forward(s, n, collision_box(step), cv(positions), cv(it.corrections), it.masks, mv(output));
    }
};

cd::ParticleParameterView param_view(const ref_params& p) {
    return {p.masses, p.rest_densities, nullptr, nullptr};
}

}  // namespace

extern "C" {

int ref_create(const ref_config* cfg, void** handle) {
    if (!cfg || !handle) return 1;
    auto* h = new Harness();
    h->cfg = *cfg;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return 3; }
    const uint32_t n = cfg->particle_count;
    h->cells_x = static_cast<uint32_t>(std::ceil((cfg->box_max[0] - cfg->box_min[0]) / cfg->support_radius));
    h->cells_y = static_cast<uint32_t>(std::ceil((cfg->box_max[1] - cfg->box_min[1]) / cfg->support_radius));
    h->cells_z = static_cast<uint32_t>(std::ceil((cfg->box_max[2] - cfg->box_min[2]) / cfg->support_radius));
    h->cells = h->cells_x * h->cells_y * h->cells_z;
    h->unsorted_keys = h->alloc<uint64_t>(n);
    h->sorted_keys = h->alloc<uint64_t>(n);
    h->unsorted_indices = h->alloc<uint32_t>(n);
    h->sorted_indices = h->alloc<uint32_t>(n);
    h->cell_offsets = h->alloc<uint32_t>(h->cells + 1);
    h->unsorted_boundary_keys = h->alloc<uint64_t>(0);
    h->sorted_boundary_keys = h->alloc<uint64_t>(0);
    h->unsorted_boundary_indices = h->alloc<uint32_t>(0);
    h->sorted_boundary_indices = h->alloc<uint32_t>(0);
    h->boundary_cell_offsets = h->alloc<uint32_t>(h->cells + 1);
    h->sort_scratch_bytes = cd::radix_sort_storage_size(n);
    h->sort_scratch = h->alloc<uint8_t>(h->sort_scratch_bytes);
    h->boundary_scratch_bytes = cd::radix_sort_storage_size(0u);
    h->boundary_scratch = h->alloc<uint8_t>(h->boundary_scratch_bytes);
    h->empty_f = h->alloc<float>(1);
    h->predicted = h->vec();
    h->corrected = h->vec();
    h->reconstructed = h->vec();
    h->vorticities = h->vec();
    h->normals = h->vec();
    h->confined = h->vec();
    h->magnitudes = h->alloc<float>(n);
    h->normalizers = h->alloc<float>(n);
    h->first_densities = h->alloc<float>(n);
    h->first_lambdas = h->alloc<float>(n);
    h->forward_iteration = h->iteration();
    // PBF::allocate_step_cache (pbf/pbf.cpp:108-125): checkpoints at 0, ci, 2ci, ... and K.
    const uint32_t K = cfg->pressure_iterations, ci = cfg->checkpoint_interval ? cfg->checkpoint_interval : 1u;
    h->checkpoints.push_back({0u, h->vec()});
    for (uint32_t it = ci; it < K; it += ci) h->checkpoints.push_back({it, h->vec()});
    if (K != 0u) h->checkpoints.push_back({K, h->vec()});
    if (cfg->differentiable) {
        for (uint32_t k = 0; k <= ci; ++k) h->segment_positions.push_back(h->vec());
        for (uint32_t k = 0; k < ci; ++k) h->segment_iterations.push_back(h->iteration());
        h->current_position_adjoint = h->dvec();
        h->next_position_adjoint = h->dvec();
        h->correction_adjoint = h->dvec();
        h->reconstructed_velocity_adjoint = h->dvec();
        h->vorticity_adjoint = h->dvec();
        h->vorticity_normal_adjoint = h->dvec();
        h->confined_velocity_adjoint = h->dvec();
        h->lambda_adjoint = h->alloc<double>(n);
        h->density_adjoint = h->alloc<double>(n);
    }
    for (void* p : h->allocations)
        if (!p) { delete h; return 2; }
    cudaMemsetAsync(h->magnitudes, 0, n * sizeof(float), h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) { delete h; return 3; }
    *handle = h;
    return 0;
}

// Boundary particles (host arrays; copied): positions, velocities (x, y, z) and volumes.
int ref_set_boundary(void* handle, const float* const* positions, const float* const* velocities, const float* volumes,
                     const uint32_t count) {
    auto* h = static_cast<Harness*>(handle);
    h->boundary_count = count;
    if (count == 0) return 0;
    h->boundary_positions = {h->alloc<float>(count), h->alloc<float>(count), h->alloc<float>(count)};
    h->boundary_velocities = {h->alloc<float>(count), h->alloc<float>(count), h->alloc<float>(count)};
    h->boundary_volumes = h->alloc<float>(count);
    h->unsorted_boundary_keys = h->alloc<uint64_t>(count);
    h->sorted_boundary_keys = h->alloc<uint64_t>(count);
    h->unsorted_boundary_indices = h->alloc<uint32_t>(count);
    h->sorted_boundary_indices = h->alloc<uint32_t>(count);
    h->boundary_scratch_bytes = cd::radix_sort_storage_size(count);
    h->boundary_scratch = h->alloc<uint8_t>(h->boundary_scratch_bytes);
    for (void* q : h->allocations)
        if (!q) return 2;
    const size_t b = count * sizeof(float);
    float* const dp[3] = {h->boundary_positions.x, h->boundary_positions.y, h->boundary_positions.z};
    float* const dv[3] = {h->boundary_velocities.x, h->boundary_velocities.y, h->boundary_velocities.z};
    for (int a = 0; a < 3; ++a) {
        cudaMemcpy(dp[a], positions[a], b, cudaMemcpyHostToDevice);
        cudaMemcpy(dv[a], velocities[a], b, cudaMemcpyHostToDevice);
    }
    cudaMemcpy(h->boundary_volumes, volumes, b, cudaMemcpyHostToDevice);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3;
}

int ref_destroy(void* handle) {
    delete static_cast<Harness*>(handle);
    return 0;
}

// PBF::forward_step (pbf/pbf.cpp:167-191).
int ref_forward_step(void* handle, const ref_state_in* state, const float* const* controls, const ref_params* p,
                     const ref_state_out* next, const uint64_t step_index) {
    auto* h = static_cast<Harness*>(handle);
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float h_radius = h->cfg.support_radius;
    const cd::ConstVectorView<float> x{state->px, state->py, state->pz}, v{state->vx, state->vy, state->vz},
        a{controls[0], controls[1], controls[2]};
    const cd::ParticleParameterView pv = param_view(*p);
    cd::pbf::launch_predict_forward(s, n, h->cfg.time_step, h->cfg.gravity[0], h->cfg.gravity[1], h->cfg.gravity[2], x, v, a,
                                    h->mv(h->predicted));
    h->build(step_index + 1u, h->predicted);
    h->copy(h->predicted, h->corrected);
    h->copy(h->corrected, h->checkpoints[0].second);
    size_t checkpoint = 1;
    for (uint32_t it = 0; it < h->cfg.pressure_iterations; ++it) {
        h->iterate(*p, pv, h->corrected, h->forward_iteration, h->corrected, step_index + 1u);
        if (it == 0) {
            cudaMemcpyAsync(h->first_densities, h->forward_iteration.densities, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
            cudaMemcpyAsync(h->first_lambdas, h->forward_iteration.lambdas, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
        }
        if (checkpoint < h->checkpoints.size() && h->checkpoints[checkpoint].first == it + 1u) {
            h->copy(h->corrected, h->checkpoints[checkpoint].second);
            ++checkpoint;
        }
    }
    cd::pbf::launch_reconstruct_forward(s, n, 1.0F / h->cfg.time_step, x, h->cv(h->corrected), h->mv(h->reconstructed));
    cd::pbf::launch_vorticity_forward(s, n, h_radius, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->reconstructed),
                                      h->neighborhood(), h->mv(h->vorticities));
    cd::pbf::launch_normal_forward(s, n, h_radius, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->vorticities),
                                   h->neighborhood(), h->magnitudes, h->mv(h->normals), h->normalizers);
    cd::pbf::launch_confinement_forward(s, n, h->cfg.time_step, h->cv(h->reconstructed), h->cv(h->vorticities),
                                        h->cv(h->normals), p->vorticity, h->mv(h->confined));
    cd::pbf::launch_xsph_forward(s, n, h_radius, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->confined),
                                 h->neighborhood(), p->xsph, cd::VectorView<float>{next->vx, next->vy, next->vz});
    h->copy(h->corrected, Vec{next->px, next->py, next->pz});
    h->step_index = step_index;
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// PBF::vjp_step (pbf/pbf.cpp:217-258).  Adjoint outputs are accumulated.
int ref_vjp_step(void* handle, const ref_state_in* state, const ref_params* p, const ref_adjoint_state* next_adjoint,
                 const ref_adjoint_state* previous_adjoint, double* const* control_adjoint, const ref_param_adjoint* pa) {
    auto* h = static_cast<Harness*>(handle);
    if (!h->cfg.differentiable) return 4;
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float hr = h->cfg.support_radius;
    const cd::ParticleParameterView pv = param_view(*p);
    const cd::ParticleParameterAdjointView pav{pa->masses, pa->rest_densities, nullptr, nullptr};
    const cd::VectorView<double> prev_x{previous_adjoint->px, previous_adjoint->py, previous_adjoint->pz};
    const cd::VectorView<double> prev_v{previous_adjoint->vx, previous_adjoint->vy, previous_adjoint->vz};
    const cd::ConstVectorView<double> next_x{next_adjoint->px, next_adjoint->py, next_adjoint->pz};
    const cd::ConstVectorView<double> next_v{next_adjoint->vx, next_adjoint->vy, next_adjoint->vz};
    const cd::ConstVectorView<float> x{state->px, state->py, state->pz};
    (void)x;
    const size_t db = n * sizeof(double);
    cudaMemcpyAsync(h->current_position_adjoint.x, next_x.x, db, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->current_position_adjoint.y, next_x.y, db, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->current_position_adjoint.z, next_x.z, db, cudaMemcpyDeviceToDevice, h->stream);
    h->clear(h->confined_velocity_adjoint);
    cd::pbf::launch_xsph_vjp(s, n, hr, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->confined), h->neighborhood(), p->xsph,
                             next_v, h->mdv(h->current_position_adjoint), h->mdv(h->confined_velocity_adjoint), pa->xsph);
    h->clear(h->reconstructed_velocity_adjoint);
    h->clear(h->vorticity_adjoint);
    h->clear(h->vorticity_normal_adjoint);
    cd::pbf::launch_confinement_vjp(s, n, h->cfg.time_step, h->cv(h->vorticities), h->cv(h->normals), p->vorticity,
                                    h->cdv(h->confined_velocity_adjoint), h->mdv(h->reconstructed_velocity_adjoint),
                                    h->mdv(h->vorticity_adjoint), h->mdv(h->vorticity_normal_adjoint), pa->vorticity);
    cd::pbf::launch_normal_vjp(s, n, hr, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->vorticities), h->neighborhood(),
                               h->magnitudes, h->cv(h->normals), h->normalizers, h->cdv(h->vorticity_normal_adjoint),
                               h->mdv(h->current_position_adjoint), h->mdv(h->vorticity_adjoint));
    cd::pbf::launch_vorticity_vjp(s, n, hr, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->reconstructed), h->neighborhood(),
                                  h->cdv(h->vorticity_adjoint), h->mdv(h->current_position_adjoint),
                                  h->mdv(h->reconstructed_velocity_adjoint));
    cd::pbf::launch_reconstruct_vjp(s, n, 1.0F / h->cfg.time_step, h->cdv(h->reconstructed_velocity_adjoint), prev_x,
                                    h->mdv(h->current_position_adjoint));
    for (size_t segment = h->checkpoints.size(); segment-- > 1;) {
        const auto& start = h->checkpoints[segment - 1];
        const auto& end = h->checkpoints[segment];
        const uint32_t length = end.first - start.first;
        h->copy(start.second, h->segment_positions[0]);
        for (uint32_t k = 0; k < length; ++k)
            h->iterate(*p, pv, h->segment_positions[k], h->segment_iterations[k], h->segment_positions[k + 1], h->step_index + 1u);
        for (uint32_t k = length; k-- > 0;) {
            Iteration& it = h->segment_iterations[k];
            h->clear(h->next_position_adjoint);
            h->clear(h->correction_adjoint);
            h->clear(h->lambda_adjoint);
            h->clear(h->density_adjoint);
            cd::pbf::launch_project_vjp(s, n, it.masks, h->cdv(h->current_position_adjoint), h->mdv(h->next_position_adjoint),
                                        h->mdv(h->correction_adjoint));
            cd::pbf::launch_correction_vjp(s, n, hr, h->cv(h->predicted), h->cv(h->segment_positions[k]), pv, h->neighborhood(),
                                           h->boundary(), it.lambdas, p->strength, p->exponent, p->radius,
                                           h->cdv(h->correction_adjoint), h->mdv(h->next_position_adjoint), h->lambda_adjoint,
                                           pav, pa->strength, pa->exponent, pa->radius);
            cd::pbf::launch_lambda_vjp(s, n, hr, h->cv(h->predicted), h->cv(h->segment_positions[k]), pv, h->neighborhood(),
                                       h->boundary(), it.densities, h->cv(it.gradient_sums), it.denominators, h->lambda_adjoint,
                                       h->mdv(h->next_position_adjoint), h->density_adjoint, pav, pa->relaxation);
            cd::density_vjp(s, n, hr, true, h->cv(h->predicted), h->cv(h->segment_positions[k]), pv, h->neighborhood(),
                            h->boundary(), h->density_adjoint, h->mdv(h->next_position_adjoint), pav);
            std::swap(h->current_position_adjoint, h->next_position_adjoint);
        }
    }
    cd::pbf::launch_predict_vjp(s, n, h->cfg.time_step, h->cdv(h->current_position_adjoint), prev_x, prev_v,
                                cd::VectorView<double>{control_adjoint[0], control_adjoint[1], control_adjoint[2]});
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// PBF::jvp_step (pbf/pbf.cpp:193-215), after ref_forward_step of the same state.  Tangents are
// FP32 device SoA; `pt` holds the parameter tangents in the ref_params layout.
int ref_jvp_step(void* handle, const ref_state_in* state, const ref_params* p, const ref_state_in* tangent,
                 const float* const* control_tangent, const ref_params* pt, const ref_state_out* next_tangent) {
    auto* h = static_cast<Harness*>(handle);
    if (!h->cfg.differentiable) return 4;
    (void)state;
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float hr = h->cfg.support_radius;
    if (!h->tangents_ready) {
        h->current_position_tangent = h->vec();
        h->next_position_tangent = h->vec();
        h->gradient_sum_tangent = h->vec();
        h->correction_tangent = h->vec();
        h->reconstructed_velocity_tangent = h->vec();
        h->vorticity_tangent = h->vec();
        h->vorticity_normal_tangent = h->vec();
        h->confined_velocity_tangent = h->vec();
        h->jvp_positions = h->vec();
        h->density_tangent = h->alloc<float>(n);
        h->denominator_tangent = h->alloc<float>(n);
        h->lambda_tangent = h->alloc<float>(n);
        h->vorticity_magnitude_tangent = h->alloc<float>(n);
        for (void* q : h->allocations)
            if (!q) return 2;
        h->tangents_ready = true;
    }
    const cd::ParticleParameterView pv = param_view(*p);
    const cd::ParticleParameterTangentView ptv{pt->masses, pt->rest_densities, nullptr, nullptr};
    const cd::ConstVectorView<float> xd{tangent->px, tangent->py, tangent->pz}, vd{tangent->vx, tangent->vy, tangent->vz},
        ad{control_tangent[0], control_tangent[1], control_tangent[2]};
    Iteration& it = h->forward_iteration;
    cd::pbf::launch_predict_jvp(s, n, h->cfg.time_step, xd, vd, ad, h->mv(h->current_position_tangent));
    h->copy(h->predicted, h->jvp_positions);
    for (uint32_t k = 0; k < h->cfg.pressure_iterations; ++k) {
        cd::density_forward(s, n, hr, true, h->cv(h->predicted), h->cv(h->jvp_positions), pv, h->neighborhood(), h->boundary(),
                            it.densities);
        cd::density_jvp(s, n, hr, true, h->cv(h->predicted), h->cv(h->jvp_positions), h->cv(h->current_position_tangent), pv, ptv,
                        h->neighborhood(), h->boundary(), h->density_tangent);
        cd::pbf::launch_lambda_forward(s, n, hr, h->cv(h->predicted), h->cv(h->jvp_positions), pv, h->neighborhood(),
                                       h->boundary(), it.densities, p->relaxation, h->mv(it.gradient_sums), it.denominators,
                                       it.lambdas);
        cd::pbf::launch_lambda_jvp(s, n, hr, h->cv(h->predicted), h->cv(h->jvp_positions), h->cv(h->current_position_tangent), pv,
                                   ptv, h->neighborhood(), h->boundary(), it.densities, h->density_tangent, p->relaxation,
                                   pt->relaxation, h->mv(h->gradient_sum_tangent), h->denominator_tangent, h->lambda_tangent);
        cd::pbf::launch_correction_forward(s, n, hr, h->cv(h->predicted), h->cv(h->jvp_positions), pv, h->neighborhood(),
                                           h->boundary(), it.lambdas, p->strength, p->exponent, p->radius, h->mv(it.corrections));
        cd::pbf::launch_correction_jvp(s, n, hr, h->cv(h->predicted), h->cv(h->jvp_positions), h->cv(h->current_position_tangent),
                                       pv, ptv, h->neighborhood(), h->boundary(), it.lambdas, h->lambda_tangent, p->strength,
                                       pt->strength, p->exponent, pt->exponent, p->radius, pt->radius,
                                       h->mv(h->correction_tangent));
        cd::pbf::launch_project_forward(s, n, h->collision_box(h->step_index + 1u), h->cv(h->jvp_positions),
                                        h->cv(it.corrections), it.masks, h->mv(h->jvp_positions));
        cd::pbf::launch_project_jvp(s, n, it.masks, h->cv(h->current_position_tangent), h->cv(h->correction_tangent),
                                    h->mv(h->next_position_tangent));
        std::swap(h->current_position_tangent, h->next_position_tangent);
    }
    cd::pbf::launch_reconstruct_jvp(s, n, 1.0F / h->cfg.time_step, xd, h->cv(h->current_position_tangent),
                                    h->mv(h->reconstructed_velocity_tangent));
    cd::pbf::launch_vorticity_jvp(s, n, hr, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->reconstructed),
                                  h->cv(h->current_position_tangent), h->cv(h->reconstructed_velocity_tangent), h->neighborhood(),
                                  h->mv(h->vorticity_tangent));
    cd::pbf::launch_normal_jvp(s, n, hr, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->vorticities),
                               h->cv(h->current_position_tangent), h->cv(h->vorticity_tangent), h->neighborhood(), h->magnitudes,
                               h->cv(h->normals), h->normalizers, h->vorticity_magnitude_tangent,
                               h->mv(h->vorticity_normal_tangent));
    cd::pbf::launch_confinement_jvp(s, n, h->cfg.time_step, h->cv(h->vorticities), h->cv(h->normals), p->vorticity,
                                    h->cv(h->reconstructed_velocity_tangent), h->cv(h->vorticity_tangent),
                                    h->cv(h->vorticity_normal_tangent), pt->vorticity, h->mv(h->confined_velocity_tangent));
    cd::pbf::launch_xsph_jvp(s, n, hr, h->cv(h->predicted), h->cv(h->corrected), h->cv(h->confined),
                             h->cv(h->current_position_tangent), h->cv(h->confined_velocity_tangent), h->neighborhood(), p->xsph,
                             pt->xsph, cd::VectorView<float>{next_tangent->vx, next_tangent->vy, next_tangent->vz});
    h->copy(h->current_position_tangent, Vec{next_tangent->px, next_tangent->py, next_tangent->pz});
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Copy a step-cache field of the last forward step to device memory `dst`.
//   0 sorted_keys (u64 N)  1 sorted indices (u32 N)  2 cell offsets (u32 C+1)  3 predicted (3N)
//   4 corrected (3N)  5 reconstructed (3N)  6 vorticities (3N)  7 magnitudes (N)  8 normals (3N)
//   9 normalizers (N)  10 confined (3N)  11 first densities (N)  12 first lambdas (N)
int ref_read(void* handle, const int field, void* dst) {
    auto* h = static_cast<Harness*>(handle);
    const size_t n = h->cfg.particle_count;
    auto vec3 = [&](const Vec& v) {
        float* d = static_cast<float*>(dst);
        cudaMemcpyAsync(d, v.x, n * 4, cudaMemcpyDeviceToDevice, h->stream);
        cudaMemcpyAsync(d + n, v.y, n * 4, cudaMemcpyDeviceToDevice, h->stream);
        cudaMemcpyAsync(d + 2 * n, v.z, n * 4, cudaMemcpyDeviceToDevice, h->stream);
    };
    switch (field) {
        case 0: cudaMemcpyAsync(dst, h->sorted_keys, n * 8, cudaMemcpyDeviceToDevice, h->stream); break;
        case 1: cudaMemcpyAsync(dst, h->sorted_indices, n * 4, cudaMemcpyDeviceToDevice, h->stream); break;
        case 2: cudaMemcpyAsync(dst, h->cell_offsets, (h->cells + 1ull) * 4, cudaMemcpyDeviceToDevice, h->stream); break;
        case 3: vec3(h->predicted); break;
        case 4: vec3(h->corrected); break;
        case 5: vec3(h->reconstructed); break;
        case 6: vec3(h->vorticities); break;
        case 7: cudaMemcpyAsync(dst, h->magnitudes, n * 4, cudaMemcpyDeviceToDevice, h->stream); break;
        case 8: vec3(h->normals); break;
        case 9: cudaMemcpyAsync(dst, h->normalizers, n * 4, cudaMemcpyDeviceToDevice, h->stream); break;
        case 10: vec3(h->confined); break;
        case 11: cudaMemcpyAsync(dst, h->first_densities, n * 4, cudaMemcpyDeviceToDevice, h->stream); break;
        case 12: cudaMemcpyAsync(dst, h->first_lambdas, n * 4, cudaMemcpyDeviceToDevice, h->stream); break;
        default: return 1;
    }
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : 3;
}

// ---- single passes of the reference on caller-chosen inputs (all pointers: device SoA) ----
// Build the neighbourhood from topology positions `x*` for the step `step` (= state step + 1).
int ref_pass_topology(void* handle, const float* const* topology, const uint64_t step) {
    auto* h = static_cast<Harness*>(handle);
    const size_t b = h->cfg.particle_count * sizeof(float);
    cudaMemcpyAsync(h->predicted.x, topology[0], b, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->predicted.y, topology[1], b, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->predicted.z, topology[2], b, cudaMemcpyDeviceToDevice, h->stream);
    h->build(step, h->predicted);
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : 3;
}

// pass: 0 density, 1 lambda, 2 correction, 3 project, 4 vorticity, 5 normal (+magnitude), 6 confinement, 7 xsph
//   in3[0..2] : vector inputs (positions, velocities/vorticities/..., normals) as SoA triples
//   sin[0..1] : scalar inputs (densities, lambdas / magnitudes)
//   out3[0..1]: vector outputs; sout[0..1]: scalar outputs; mask: uint32 masks
int ref_pass(void* handle, const int pass, const float* const* in3, const float* const* sin, const ref_params* p,
             float* const* out3, float* const* sout, uint32_t* mask, const uint64_t step) {
    auto* h = static_cast<Harness*>(handle);
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float hr = h->cfg.support_radius;
    const cd::ParticleParameterView pv = param_view(*p);
    auto cin = [&](int k) { return cd::ConstVectorView<float>{in3[3 * k], in3[3 * k + 1], in3[3 * k + 2]}; };
    auto vout = [&](int k) { return cd::VectorView<float>{out3[3 * k], out3[3 * k + 1], out3[3 * k + 2]}; };
    switch (pass) {
        case 0: cd::density_forward(s, n, hr, true, h->cv(h->predicted), cin(0), pv, h->neighborhood(), h->boundary(), sout[0]); break;
        case 1: cd::pbf::launch_lambda_forward(s, n, hr, h->cv(h->predicted), cin(0), pv, h->neighborhood(), h->boundary(), sin[0],
                                               p->relaxation, vout(0), sout[0], sout[1]); break;
        case 2: cd::pbf::launch_correction_forward(s, n, hr, h->cv(h->predicted), cin(0), pv, h->neighborhood(), h->boundary(), sin[0],
                                                   p->strength, p->exponent, p->radius, vout(0)); break;
        case 3: cd::pbf::launch_project_forward(s, n, h->collision_box(step), cin(0), cin(1), mask, vout(0)); break;
        case 4: cd::pbf::launch_vorticity_forward(s, n, hr, h->cv(h->predicted), cin(0), cin(1), h->neighborhood(), vout(0)); break;
        case 5: cd::pbf::launch_normal_forward(s, n, hr, h->cv(h->predicted), cin(0), cin(1), h->neighborhood(), sout[0], vout(0), sout[1]); break;
        case 6: cd::pbf::launch_confinement_forward(s, n, h->cfg.time_step, cin(0), cin(1), cin(2), p->vorticity, vout(0)); break;
        case 7: cd::pbf::launch_xsph_forward(s, n, hr, h->cv(h->predicted), cin(0), cin(1), h->neighborhood(), p->xsph, vout(0)); break;
        case 8: cd::pbf::launch_reconstruct_forward(s, n, 1.0F / h->cfg.time_step, cin(0), cin(1), vout(0)); break;
        default: return 1;
    }
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : 3;
}

int ref_cells(void* handle, uint32_t* dims) {
    auto* h = static_cast<Harness*>(handle);
    dims[0] = h->cells_x; dims[1] = h->cells_y; dims[2] = h->cells_z;
    return 0;
}

int ref_synchronize(void* handle) {
    return cudaStreamSynchronize(static_cast<Harness*>(handle)->stream) == cudaSuccess ? 0 : 3;
}

// Stream of the harness (to time it with events on that stream).
void* ref_stream(void* handle) { return static_cast<Harness*>(handle)->stream; }

}  // extern "C"

// ================================================================================ SPH
namespace {

// compute_reference_gradient_norm (sph/sph.cpp:36-58): host float arithmetic over a lattice of
// spacing 2 r inside the support, evaluated here in the same order and precision.
float sph_reference_gradient_norm(const float support_radius, const float particle_radius) {
    const float pi = 3.14159265358979323846F;
    const float diameter = 2.0F * particle_radius;
    const float coefficient = 8.0F / (pi * support_radius * support_radius * support_radius);
    float gx = 0.0F, gy = 0.0F, gz = 0.0F, squared = 0.0F;
    for (float x = -support_radius; x <= support_radius; x += diameter)
        for (float y = -support_radius; y <= support_radius; y += diameter)
            for (float z = -support_radius; z <= support_radius; z += diameter) {
                const float xx = x * x, yy = y * y, zz = z * z;
                const float distance = std::sqrt(xx + yy + zz);
                if (distance == 0.0F || distance >= support_radius) continue;
                const float q = distance / support_radius;
                const float derivative = q <= 0.5F ? 18.0F * q * q - 12.0F * q : -6.0F * (1.0F - q) * (1.0F - q);
                const float scale = coefficient * derivative / (support_radius * distance);
                gx += scale * x;
                gy += scale * y;
                gz += scale * z;
                squared += scale * scale * (xx + yy + zz);
            }
    return gx * gx + gy * gy + gz * gz + squared;
}

// PressureIterationCache / Tangent / Adjoint (sph/sph.ixx:14-37)
struct IterCache {
    uint32_t iteration = 0;
    float* pressures = nullptr;
    float* predicted_densities = nullptr;
    Vec pressure_acc, predicted_positions, predicted_velocities;
};
struct IterTangent {
    float* pressures = nullptr;
    float* predicted_densities = nullptr;
    Vec pressure_acc, predicted_positions, predicted_velocities;
};
struct IterAdjoint {
    double* pressures = nullptr;
    double* predicted_densities = nullptr;
    DVec pressure_acc, predicted_positions, predicted_velocities;
};

struct SphReplay {
    Harness* h = nullptr;
    int method = 0;   // 0 WCSPH, 1 PCISPH, 2 IISPH, 3 DFSPH
    uint32_t pressure_iterations = 6, divergence_iterations = 4, density_iterations = 6, checkpoint_interval = 2;
    int warm_start = 1;
    bool differentiable = false;
    float reference_gradient_norm = 0.0F;
    std::vector<void*> allocations;
    float* densities = nullptr;
    // WCSPH::Cache (sph/sph.ixx:63-70)
    float* pressures = nullptr;
    Vec pressure_acc, viscosity_acc, surface_acc, external_acc, total_acc;
    // the iterative methods' caches (sph/sph.ixx:114-117, 160-163, 226-232) and members
    Vec non_pressure_acc, divergence_pressure_acc, total_pressure_acc, total_pressure_acceleration;
    IterCache primal;
    std::vector<IterCache> checkpoints, divergence_checkpoints, density_checkpoints, recomputed;
    // differentiation workspaces (sph/sph.ixx:71-79, 119-125, 235-246, 306-308)
    float* density_tangent = nullptr;
    double* density_adjoint = nullptr;
    float* pressure_tangent = nullptr;
    Vec pressure_acc_tangent, viscosity_acc_tangent, surface_acc_tangent, total_acc_tangent;
    double* pressure_adjoint = nullptr;
    DVec total_acc_adjoint;
    IterTangent tangent;
    IterAdjoint adjoint, previous_adjoint;
    Vec non_pressure_acc_tangent, divergence_pressure_acc_tangent, total_pressure_acc_tangent;
    DVec non_pressure_acc_adjoint, divergence_pressure_acc_adjoint, total_pressure_acc_adjoint;
    double* target_density_adjoint = nullptr;

    template <class T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
            allocations.push_back(nullptr);
            return nullptr;
        }
        allocations.push_back(p);
        return static_cast<T*>(p);
    }
    size_t n() const { return h->cfg.particle_count; }
    Vec vec() { return {alloc<float>(n()), alloc<float>(n()), alloc<float>(n())}; }
    DVec dvec() { return {alloc<double>(n()), alloc<double>(n()), alloc<double>(n())}; }
    IterCache iter() { return {0u, alloc<float>(n()), alloc<float>(n()), vec(), vec(), vec()}; }
    IterTangent iter_tangent() { return {alloc<float>(n()), alloc<float>(n()), vec(), vec(), vec()}; }
    IterAdjoint iter_adjoint() { return {alloc<double>(n()), alloc<double>(n()), dvec(), dvec(), dvec()}; }
    ~SphReplay() {
        if (h) cudaStreamSynchronize(h->stream);
        for (void* p : allocations)
            if (p) cudaFree(p);
    }
    void clear(float* p) const { cudaMemsetAsync(p, 0, n() * sizeof(float), h->stream); }
    void clear(double* p) const { cudaMemsetAsync(p, 0, n() * sizeof(double), h->stream); }
    void clear(const Vec& v) const { clear(v.x); clear(v.y); clear(v.z); }
    void clear(const DVec& v) const { clear(v.x); clear(v.y); clear(v.z); }
    void copy(const float* src, float* dst) const {
        cudaMemcpyAsync(dst, src, n() * sizeof(float), cudaMemcpyDeviceToDevice, h->stream);
    }
    void copy(const double* src, double* dst) const {
        cudaMemcpyAsync(dst, src, n() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
    }
    void copy(const Vec& a, const Vec& b) const { copy(a.x, b.x); copy(a.y, b.y); copy(a.z, b.z); }
    void copy(const DVec& a, const DVec& b) const { copy(a.x, b.x); copy(a.y, b.y); copy(a.z, b.z); }
    // clear_iteration / copy_iteration (sph/sph.cpp:91-126)
    void clear(IterCache& c) const {
        clear(c.pressures); clear(c.predicted_densities); clear(c.pressure_acc); clear(c.predicted_positions);
        clear(c.predicted_velocities);
    }
    void clear(IterTangent& c) const {
        clear(c.pressures); clear(c.predicted_densities); clear(c.pressure_acc); clear(c.predicted_positions);
        clear(c.predicted_velocities);
    }
    void clear(IterAdjoint& c) const {
        clear(c.pressures); clear(c.predicted_densities); clear(c.pressure_acc); clear(c.predicted_positions);
        clear(c.predicted_velocities);
    }
    void copy(const IterCache& a, IterCache& b) const {
        b.iteration = a.iteration;
        copy(a.pressures, b.pressures); copy(a.predicted_densities, b.predicted_densities); copy(a.pressure_acc, b.pressure_acc);
        copy(a.predicted_positions, b.predicted_positions); copy(a.predicted_velocities, b.predicted_velocities);
    }
    // Method::allocate_cache: checkpoints at 0, every interval and the last iteration (sph/sph.cpp:282-288)
    std::vector<IterCache> checkpoint_set(const uint32_t iterations) {
        const uint32_t ci = checkpoint_interval;
        const uint32_t count = 1u + iterations / ci + (iterations % ci == 0u ? 0u : 1u);
        std::vector<IterCache> out;
        for (uint32_t k = 0; k < count; ++k) out.push_back(iter());
        return out;
    }
};

cd::ParticleParameterTangentView tangent_view(const float* const* p) { return {p[0], p[1], p[2], p[3]}; }
cd::ParticleParameterAdjointView adjoint_view(double* const* p) { return {p[0], p[1], p[2], p[3]}; }

}  // namespace

extern "C" {

typedef struct {
    int method;                       // 0 WCSPH, 1 PCISPH, 2 IISPH, 3 DFSPH
    uint32_t pressure_iterations;     // PCISPH / IISPH
    uint32_t divergence_iterations;   // DFSPH
    uint32_t density_iterations;      // DFSPH
    int pressure_warm_start;          // DFSPH
    uint32_t checkpoint_interval;     // differentiable mode
    int differentiable;
} ref_sph_config;

// ParticleParameters (masses, rest densities, viscosities, surface tensions) and the method's
// Parameters: WCSPH (speed of sound, Tait exponent, boundary surface tension), PCISPH (pressure
// relaxation), IISPH (Jacobi relaxation), DFSPH (divergence relaxation, density relaxation).
typedef struct {
    const float* masses; const float* rest_densities; const float* viscosities; const float* surface_tensions;
    const float* method0; const float* method1; const float* method2;
} ref_sph_params;

int ref_sph_create(void* harness, const ref_sph_config* c, void** out) {
    if (!harness || !c || !out || c->method < 0 || c->method > 3) return 1;
    auto* r = new SphReplay();
    r->h = static_cast<Harness*>(harness);
    r->method = c->method;
    r->pressure_iterations = c->pressure_iterations;
    r->divergence_iterations = c->divergence_iterations;
    r->density_iterations = c->density_iterations;
    r->warm_start = c->pressure_warm_start;
    r->checkpoint_interval = c->checkpoint_interval ? c->checkpoint_interval : 2u;
    r->differentiable = c->differentiable != 0;
    r->reference_gradient_norm = sph_reference_gradient_norm(r->h->cfg.support_radius, r->h->cfg.particle_radius);
    const size_t n = r->n();
    r->densities = r->alloc<float>(n);
    if (r->method == 0) {
        r->pressures = r->alloc<float>(n);
        r->pressure_acc = r->vec();
        r->viscosity_acc = r->vec();
        r->surface_acc = r->vec();
        r->external_acc = r->vec();
        r->total_acc = r->vec();
    } else {
        r->non_pressure_acc = r->vec();
        r->primal = r->iter();
        if (r->method == 3) {
            r->divergence_pressure_acc = r->vec();
            r->total_pressure_acc = r->vec();
            r->total_pressure_acceleration = r->vec();
            r->divergence_checkpoints = r->checkpoint_set(r->divergence_iterations);
            r->density_checkpoints = r->checkpoint_set(r->density_iterations);
        } else {
            r->checkpoints = r->checkpoint_set(r->pressure_iterations);
        }
    }
    if (r->differentiable) {
        r->density_tangent = r->alloc<float>(n);
        r->density_adjoint = r->alloc<double>(n);
        if (r->method == 0) {
            r->pressure_tangent = r->alloc<float>(n);
            r->pressure_acc_tangent = r->vec();
            r->viscosity_acc_tangent = r->vec();
            r->surface_acc_tangent = r->vec();
            r->total_acc_tangent = r->vec();
            r->pressure_adjoint = r->alloc<double>(n);
            r->total_acc_adjoint = r->dvec();
        } else {
            for (uint32_t k = 0; k <= r->checkpoint_interval; ++k) r->recomputed.push_back(r->iter());
            r->tangent = r->iter_tangent();
            r->adjoint = r->iter_adjoint();
            r->previous_adjoint = r->iter_adjoint();
            r->non_pressure_acc_tangent = r->vec();
            r->non_pressure_acc_adjoint = r->dvec();
            if (r->method == 3) {
                r->divergence_pressure_acc_tangent = r->vec();
                r->total_pressure_acc_tangent = r->vec();
                r->target_density_adjoint = r->alloc<double>(n);
                r->divergence_pressure_acc_adjoint = r->dvec();
                r->total_pressure_acc_adjoint = r->dvec();
            }
        }
    }
    for (void* p : r->allocations)
        if (!p) { delete r; return 2; }
    *out = r;
    return 0;
}

int ref_sph_destroy(void* sph) {
    delete static_cast<SphReplay*>(sph);
    return 0;
}

float ref_sph_reference_gradient_norm(void* sph) { return static_cast<SphReplay*>(sph)->reference_gradient_norm; }

// SPH<Method>::forward_step (sph/sph.ixx:350-354).  warm_* / next_warm_*: DFSPH's method state
// (sph/sph.ixx:202-205), ignored by the other methods.
int ref_sph_forward_step(void* sph, const ref_state_in* state, const float* const* controls, const ref_sph_params* p,
                         const float* warm_divergence, const float* warm_density, const ref_state_out* next,
                         float* next_warm_divergence, float* next_warm_density, const uint64_t step_index) {
    auto* r = static_cast<SphReplay*>(sph);
    Harness* h = r->h;
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float hr = h->cfg.support_radius;
    const float dt = h->cfg.time_step;
    const Vec positions{const_cast<float*>(state->px), const_cast<float*>(state->py), const_cast<float*>(state->pz)};
    const cd::ConstVectorView<float> x{state->px, state->py, state->pz}, v{state->vx, state->vy, state->vz},
        a{controls[0], controls[1], controls[2]};
    const cd::VectorView<float> xo{next->px, next->py, next->pz}, vo{next->vx, next->vy, next->vz};
    const cd::ParticleParameterView pv{p->masses, p->rest_densities, p->viscosities, p->surface_tensions};
    const cd::Box box = h->collision_box(step_index);
    h->build(step_index, positions);
    cd::density_forward(s, n, hr, false, x, x, pv, h->neighborhood(), h->boundary(), r->densities);
    if (r->method == 0) {   // WCSPH::forward (sph/sph.cpp:214-225)
        namespace w = cd::wcsph;
        w::launch_eos_forward(s, n, r->densities, pv, p->method0, p->method1, r->pressures);
        cd::sph::pressure_forward(s, n, hr, x, pv, h->neighborhood(), h->boundary(), r->densities, r->pressures,
                                  h->mv(r->pressure_acc));
        w::launch_artificial_viscosity_forward(s, n, hr, x, v, pv, p->method0, h->neighborhood(), h->boundary(), r->densities,
                                               h->mv(r->viscosity_acc));
        w::launch_surface_forward(s, n, hr, h->cfg.particle_radius, x, pv, p->method2, h->neighborhood(), h->boundary(),
                                  h->mv(r->surface_acc));
        cd::sph::add(s, n, h->cv(r->pressure_acc), h->cv(r->viscosity_acc), h->mv(r->total_acc));
        cd::sph::add(s, n, h->cv(r->total_acc), h->cv(r->surface_acc), h->mv(r->total_acc));
        w::launch_external_forward(s, n, h->cfg.gravity[0], h->cfg.gravity[1], h->cfg.gravity[2], a, h->mv(r->external_acc));
        cd::sph::add(s, n, h->cv(r->total_acc), h->cv(r->external_acc), h->mv(r->total_acc));
        cd::sph::integrate_forward(s, n, dt, box, x, v, h->cv(r->total_acc), xo, vo);
        return cudaGetLastError() == cudaSuccess ? 0 : 3;
    }
    cd::sph::non_pressure_forward(s, n, hr, h->cfg.gravity[0], h->cfg.gravity[1], h->cfg.gravity[2], x, v, a, pv,
                                  h->neighborhood(), h->boundary(), r->densities, h->mv(r->non_pressure_acc));
    const float rgn = r->reference_gradient_norm;
    IterCache& pr = r->primal;
    auto predict = [&](const Vec& pressure_acc, const cd::VectorView<float> px, const cd::VectorView<float> pvv) {
        if (r->method == 1)
            cd::pcisph::launch_predict_forward(s, n, dt, box, x, v, h->cv(r->non_pressure_acc), h->cv(pressure_acc), px, pvv);
        else if (r->method == 2)
            cd::iisph::launch_predict_forward(s, n, dt, box, x, v, h->cv(r->non_pressure_acc), h->cv(pressure_acc), px, pvv);
        else
            cd::dfsph::launch_predict_forward(s, n, dt, box, x, v, h->cv(r->non_pressure_acc), h->cv(pressure_acc), px, pvv);
    };
    auto pressure = [&]() {
        cd::sph::pressure_forward(s, n, hr, x, pv, h->neighborhood(), h->boundary(), r->densities, pr.pressures,
                                  h->mv(pr.pressure_acc));
    };
    auto predicted_density = [&]() {
        cd::density_forward(s, n, hr, false, x, h->cv(pr.predicted_positions), pv, h->neighborhood(), h->boundary(),
                            pr.predicted_densities);
    };
    auto checkpoint = [&](std::vector<IterCache>& set, size_t& next_checkpoint, const uint32_t it, const uint32_t last) {
        if (it == 0u || it % r->checkpoint_interval == 0u || it == last) r->copy(pr, set[next_checkpoint++]);
    };
    if (r->method == 1 || r->method == 2) {   // PCISPH::forward / IISPH::forward (sph/sph.cpp:296-312, 409-425)
        r->clear(pr);
        pr.iteration = 0u;
        size_t c = 0;
        checkpoint(r->checkpoints, c, 0u, r->pressure_iterations);
        for (uint32_t it = 1; it <= r->pressure_iterations; ++it) {
            predict(pr.pressure_acc, h->mv(pr.predicted_positions), h->mv(pr.predicted_velocities));
            predicted_density();
            if (r->method == 1)
                cd::pcisph::launch_pressure_update_forward(s, n, dt, rgn, pv, pr.pressures, pr.predicted_densities, p->method0,
                                                           pr.pressures);
            else
                cd::iisph::launch_jacobi_update_forward(s, n, dt, rgn, pv, r->densities, pr.pressures, pr.predicted_densities,
                                                        p->method0, pr.pressures);
            pressure();
            pr.iteration = it;
            checkpoint(r->checkpoints, c, it, r->pressure_iterations);
        }
        predict(pr.pressure_acc, xo, vo);
        return cudaGetLastError() == cudaSuccess ? 0 : 3;
    }
    // DFSPH::forward (sph/sph.cpp:572-610)
    r->clear(pr);
    if (r->warm_start) r->copy(warm_divergence, pr.pressures);
    pressure();
    pr.iteration = 0u;
    size_t c = 0;
    checkpoint(r->divergence_checkpoints, c, 0u, r->divergence_iterations);
    for (uint32_t it = 1; it <= r->divergence_iterations; ++it) {
        predict(pr.pressure_acc, h->mv(pr.predicted_positions), h->mv(pr.predicted_velocities));
        predicted_density();
        cd::dfsph::launch_projection_update_forward(s, n, dt, rgn, pv, r->densities, r->densities, pr.pressures,
                                                    pr.predicted_densities, p->method0, pr.pressures);
        pressure();
        pr.iteration = it;
        checkpoint(r->divergence_checkpoints, c, it, r->divergence_iterations);
    }
    r->copy(pr.pressure_acc, r->divergence_pressure_acc);
    r->copy(pr.pressures, next_warm_divergence);
    r->clear(pr);
    if (r->warm_start) r->copy(warm_density, pr.pressures);
    pressure();
    pr.iteration = 0u;
    c = 0;
    checkpoint(r->density_checkpoints, c, 0u, r->density_iterations);
    for (uint32_t it = 1; it <= r->density_iterations; ++it) {
        cd::sph::add(s, n, h->cv(r->divergence_pressure_acc), h->cv(pr.pressure_acc), h->mv(r->total_pressure_acceleration));
        predict(r->total_pressure_acceleration, h->mv(pr.predicted_positions), h->mv(pr.predicted_velocities));
        predicted_density();
        cd::dfsph::launch_projection_update_forward(s, n, dt, rgn, pv, r->densities, p->rest_densities, pr.pressures,
                                                    pr.predicted_densities, p->method1, pr.pressures);
        pressure();
        pr.iteration = it;
        checkpoint(r->density_checkpoints, c, it, r->density_iterations);
    }
    cd::sph::add(s, n, h->cv(r->divergence_pressure_acc), h->cv(pr.pressure_acc), h->mv(r->total_pressure_acc));
    r->copy(pr.pressures, next_warm_density);
    predict(r->total_pressure_acc, xo, vo);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// SPH<Method>::jvp_step (sph/sph.ixx:356-359) after ref_sph_forward_step of the same state.
//   tangent: state tangent (SoA); control_tangent[3]; particle_tangent[4] (masses, rest densities,
//   viscosities, surface tensions); method_tangent[3] (the method's parameters, as in ref_sph_params);
//   warm_tangent[2] / next_warm_tangent[2]: DFSPH's method-state tangents.
int ref_sph_jvp_step(void* sph, const ref_state_in* state, const ref_sph_params* p, const ref_state_in* tangent,
                     const float* const* control_tangent, const float* const* particle_tangent,
                     const float* const* method_tangent, const float* const* warm_tangent, const ref_state_out* next_tangent,
                     float* const* next_warm_tangent, const uint64_t step_index, const float* warm_divergence,
                     const float* warm_density) {
    auto* r = static_cast<SphReplay*>(sph);
    if (!r->differentiable) return 1;
    Harness* h = r->h;
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float hr = h->cfg.support_radius;
    const float dt = h->cfg.time_step;
    const cd::ConstVectorView<float> x{state->px, state->py, state->pz}, v{state->vx, state->vy, state->vz};
    const cd::ConstVectorView<float> xt{tangent->px, tangent->py, tangent->pz}, vt{tangent->vx, tangent->vy, tangent->vz};
    const cd::ConstVectorView<float> at{control_tangent[0], control_tangent[1], control_tangent[2]};
    const cd::VectorView<float> xo{next_tangent->px, next_tangent->py, next_tangent->pz},
        vo{next_tangent->vx, next_tangent->vy, next_tangent->vz};
    const cd::ParticleParameterView pv{p->masses, p->rest_densities, p->viscosities, p->surface_tensions};
    const cd::ParticleParameterTangentView pt = tangent_view(particle_tangent);
    const cd::Box box = h->collision_box(step_index);
    const auto nb = h->neighborhood();
    const auto bd = h->boundary();
    cd::density_jvp(s, n, hr, false, x, x, xt, pv, pt, nb, bd, r->density_tangent);
    const float* rho = r->densities;
    const float* rho_t = r->density_tangent;
    if (r->method == 0) {   // WCSPH::jvp (sph/sph.cpp:227-237)
        namespace w = cd::wcsph;
        w::launch_eos_jvp(s, n, rho, rho_t, pv, pt, p->method0, method_tangent[0], p->method1, method_tangent[1], r->pressure_tangent);
        cd::sph::pressure_jvp(s, n, hr, x, xt, pv, pt, nb, bd, rho, rho_t, r->pressures, r->pressure_tangent,
                              h->mv(r->pressure_acc_tangent));
        w::launch_artificial_viscosity_jvp(s, n, hr, x, v, xt, vt, pv, pt, p->method0, method_tangent[0], nb, bd, rho, rho_t,
                                           h->mv(r->viscosity_acc_tangent));
        w::launch_surface_jvp(s, n, hr, h->cfg.particle_radius, x, xt, pv, pt, p->method2, method_tangent[2], nb, bd,
                              h->mv(r->surface_acc_tangent));
        cd::sph::add(s, n, h->cv(r->pressure_acc_tangent), h->cv(r->viscosity_acc_tangent), h->mv(r->total_acc_tangent));
        cd::sph::add(s, n, h->cv(r->total_acc_tangent), h->cv(r->surface_acc_tangent), h->mv(r->total_acc_tangent));
        cd::sph::add(s, n, h->cv(r->total_acc_tangent), at, h->mv(r->total_acc_tangent));
        cd::sph::integrate_jvp(s, n, dt, box, x, v, h->cv(r->total_acc), xt, vt, h->cv(r->total_acc_tangent), xo, vo);
        return cudaGetLastError() == cudaSuccess ? 0 : 3;
    }
    const float rgn = r->reference_gradient_norm;
    IterCache& pr = r->primal;
    IterTangent& tg = r->tangent;
    cd::sph::non_pressure_jvp(s, n, hr, x, v, at, xt, vt, pv, pt, nb, bd, rho, rho_t, h->mv(r->non_pressure_acc_tangent));
    auto predict = [&](const Vec& pressure_acc, const cd::VectorView<float> px, const cd::VectorView<float> pvv) {
        if (r->method == 1)
            cd::pcisph::launch_predict_forward(s, n, dt, box, x, v, h->cv(r->non_pressure_acc), h->cv(pressure_acc), px, pvv);
        else if (r->method == 2)
            cd::iisph::launch_predict_forward(s, n, dt, box, x, v, h->cv(r->non_pressure_acc), h->cv(pressure_acc), px, pvv);
        else
            cd::dfsph::launch_predict_forward(s, n, dt, box, x, v, h->cv(r->non_pressure_acc), h->cv(pressure_acc), px, pvv);
    };
    auto predict_jvp = [&](const Vec& pressure_acc, const Vec& pressure_acc_tangent, const cd::VectorView<float> px,
                           const cd::VectorView<float> pvv) {
        const auto anp = h->cv(r->non_pressure_acc);
        const auto anpt = h->cv(r->non_pressure_acc_tangent);
        if (r->method == 1)
            cd::pcisph::launch_predict_jvp(s, n, dt, box, x, v, anp, h->cv(pressure_acc), xt, vt, anpt, h->cv(pressure_acc_tangent), px, pvv);
        else if (r->method == 2)
            cd::iisph::launch_predict_jvp(s, n, dt, box, x, v, anp, h->cv(pressure_acc), xt, vt, anpt, h->cv(pressure_acc_tangent), px, pvv);
        else
            cd::dfsph::launch_predict_jvp(s, n, dt, box, x, v, anp, h->cv(pressure_acc), xt, vt, anpt, h->cv(pressure_acc_tangent), px, pvv);
    };
    auto pressure = [&]() {
        cd::sph::pressure_forward(s, n, hr, x, pv, nb, bd, rho, pr.pressures, h->mv(pr.pressure_acc));
    };
    auto pressure_jvp = [&]() {
        cd::sph::pressure_jvp(s, n, hr, x, xt, pv, pt, nb, bd, rho, rho_t, pr.pressures, tg.pressures, h->mv(tg.pressure_acc));
    };
    auto densities_at_prediction = [&]() {
        cd::density_forward(s, n, hr, false, x, h->cv(pr.predicted_positions), pv, nb, bd, pr.predicted_densities);
        cd::density_jvp(s, n, hr, false, x, h->cv(pr.predicted_positions), h->cv(tg.predicted_positions), pv, pt, nb, bd,
                        tg.predicted_densities);
    };
    if (r->method == 1 || r->method == 2) {   // PCISPH::jvp / IISPH::jvp (sph/sph.cpp:314-330, 427-443)
        r->clear(pr);
        r->clear(tg);
        for (uint32_t it = 1; it <= r->pressure_iterations; ++it) {
            predict(pr.pressure_acc, h->mv(pr.predicted_positions), h->mv(pr.predicted_velocities));
            predict_jvp(pr.pressure_acc, tg.pressure_acc, h->mv(tg.predicted_positions), h->mv(tg.predicted_velocities));
            densities_at_prediction();
            if (r->method == 1) {
                cd::pcisph::launch_pressure_update_jvp(s, n, dt, rgn, pv, pt, pr.pressures, pr.predicted_densities, p->method0,
                                                       tg.pressures, tg.predicted_densities, method_tangent[0], tg.pressures);
                cd::pcisph::launch_pressure_update_forward(s, n, dt, rgn, pv, pr.pressures, pr.predicted_densities, p->method0,
                                                           pr.pressures);
            } else {
                cd::iisph::launch_jacobi_update_jvp(s, n, dt, rgn, pv, pt, rho, rho_t, pr.pressures, pr.predicted_densities,
                                                    p->method0, tg.pressures, tg.predicted_densities, method_tangent[0],
                                                    tg.pressures);
                cd::iisph::launch_jacobi_update_forward(s, n, dt, rgn, pv, rho, pr.pressures, pr.predicted_densities, p->method0,
                                                        pr.pressures);
            }
            pressure_jvp();
            pressure();
        }
        predict_jvp(pr.pressure_acc, tg.pressure_acc, xo, vo);
        return cudaGetLastError() == cudaSuccess ? 0 : 3;
    }
    // DFSPH::jvp (sph/sph.cpp:612-659)
    r->clear(pr);
    r->clear(tg);
    if (r->warm_start) {
        r->copy(warm_divergence, pr.pressures);
        r->copy(warm_tangent[0], tg.pressures);
    }
    pressure();
    pressure_jvp();
    for (uint32_t it = 1; it <= r->divergence_iterations; ++it) {
        predict(pr.pressure_acc, h->mv(pr.predicted_positions), h->mv(pr.predicted_velocities));
        predict_jvp(pr.pressure_acc, tg.pressure_acc, h->mv(tg.predicted_positions), h->mv(tg.predicted_velocities));
        densities_at_prediction();
        cd::dfsph::launch_projection_update_jvp(s, n, dt, rgn, pv, pt, rho, rho_t, rho, rho_t, pr.pressures, pr.predicted_densities,
                                                p->method0, tg.pressures, tg.predicted_densities, method_tangent[0], tg.pressures);
        cd::dfsph::launch_projection_update_forward(s, n, dt, rgn, pv, rho, rho, pr.pressures, pr.predicted_densities, p->method0,
                                                    pr.pressures);
        pressure_jvp();
        pressure();
    }
    r->copy(tg.pressure_acc, r->divergence_pressure_acc_tangent);
    r->copy(tg.pressures, next_warm_tangent[0]);
    r->clear(pr);
    r->clear(tg);
    if (r->warm_start) {
        r->copy(warm_density, pr.pressures);
        r->copy(warm_tangent[1], tg.pressures);
    }
    pressure();
    pressure_jvp();
    for (uint32_t it = 1; it <= r->density_iterations; ++it) {
        cd::sph::add(s, n, h->cv(r->divergence_pressure_acc), h->cv(pr.pressure_acc), h->mv(r->total_pressure_acceleration));
        cd::sph::add(s, n, h->cv(r->divergence_pressure_acc_tangent), h->cv(tg.pressure_acc), h->mv(r->total_pressure_acc_tangent));
        predict(r->total_pressure_acceleration, h->mv(pr.predicted_positions), h->mv(pr.predicted_velocities));
        predict_jvp(r->total_pressure_acceleration, r->total_pressure_acc_tangent, h->mv(tg.predicted_positions),
                    h->mv(tg.predicted_velocities));
        densities_at_prediction();
        cd::dfsph::launch_projection_update_jvp(s, n, dt, rgn, pv, pt, rho, rho_t, p->rest_densities, pt.rest_densities,
                                                pr.pressures, pr.predicted_densities, p->method1, tg.pressures,
                                                tg.predicted_densities, method_tangent[1], tg.pressures);
        cd::dfsph::launch_projection_update_forward(s, n, dt, rgn, pv, rho, p->rest_densities, pr.pressures, pr.predicted_densities,
                                                    p->method1, pr.pressures);
        pressure_jvp();
        pressure();
    }
    cd::sph::add(s, n, h->cv(r->divergence_pressure_acc_tangent), h->cv(tg.pressure_acc), h->mv(r->total_pressure_acc_tangent));
    r->copy(tg.pressures, next_warm_tangent[1]);
    predict_jvp(r->total_pressure_acc, r->total_pressure_acc_tangent, xo, vo);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// SPH<Method>::vjp_step (sph/sph.ixx:361-365) after ref_sph_forward_step of the same state.  All
// outputs are accumulated (FP64, SoA): previous[6] (positions, velocities), control[3], particle[4]
// (masses, rest densities, viscosities, surface tensions), method[3] (the method's parameters);
// next_warm[2] / previous_warm[2]: DFSPH's method-state adjoints (the reference copies into
// previous_warm, sph/sph.cpp:714).
int ref_sph_vjp_step(void* sph, const ref_state_in* state, const ref_sph_params* p, const double* const* next_adjoint,
                     const double* const* next_warm, double* const* previous, double* const* control, double* const* particle,
                     double* const* method_adjoint, double* const* previous_warm, const uint64_t step_index) {
    auto* r = static_cast<SphReplay*>(sph);
    if (!r->differentiable) return 1;
    Harness* h = r->h;
    const ::cuda::stream_ref s{h->stream};
    const uint32_t n = h->cfg.particle_count;
    const float hr = h->cfg.support_radius;
    const float dt = h->cfg.time_step;
    const cd::ConstVectorView<float> x{state->px, state->py, state->pz}, v{state->vx, state->vy, state->vz};
    const cd::ConstVectorView<double> nx{next_adjoint[0], next_adjoint[1], next_adjoint[2]},
        nv{next_adjoint[3], next_adjoint[4], next_adjoint[5]};
    const cd::VectorView<double> px{previous[0], previous[1], previous[2]}, pvv{previous[3], previous[4], previous[5]};
    const DVec control_adjoint{control[0], control[1], control[2]};
    const cd::ParticleParameterView pv{p->masses, p->rest_densities, p->viscosities, p->surface_tensions};
    const cd::ParticleParameterAdjointView pa = adjoint_view(particle);
    const cd::Box box = h->collision_box(step_index);
    const auto nb = h->neighborhood();
    const auto bd = h->boundary();
    const float* rho = r->densities;
    double* rho_a = r->density_adjoint;
    r->clear(rho_a);
    auto accumulate = [&](const DVec& from, const DVec& to) {   // domain.accumulate (domain/domain.cu)
        cd::accumulate(s, h->cdv(from), h->mdv(to), n);
    };
    if (r->method == 0) {   // WCSPH::vjp (sph/sph.cpp:239-250)
        namespace w = cd::wcsph;
        r->clear(r->pressure_adjoint);
        r->clear(r->total_acc_adjoint);
        cd::sph::integrate_vjp(s, n, dt, box, x, v, h->cv(r->total_acc), nx, nv, px, pvv, h->mdv(r->total_acc_adjoint));
        accumulate(r->total_acc_adjoint, control_adjoint);
        w::launch_surface_vjp(s, n, hr, h->cfg.particle_radius, x, pv, p->method2, nb, bd, h->cdv(r->total_acc_adjoint), px, pa,
                              method_adjoint[2]);
        w::launch_artificial_viscosity_vjp(s, n, hr, x, v, pv, p->method0, nb, bd, rho, h->cdv(r->total_acc_adjoint), px, pvv,
                                           rho_a, pa, method_adjoint[0]);
        cd::sph::pressure_vjp(s, n, hr, x, pv, nb, bd, rho, r->pressures, h->cdv(r->total_acc_adjoint), px, rho_a,
                              r->pressure_adjoint, pa);
        w::launch_eos_vjp(s, n, rho, pv, p->method0, p->method1, r->pressure_adjoint, rho_a, pa, method_adjoint[0],
                          method_adjoint[1]);
        cd::density_vjp(s, n, hr, false, x, x, pv, nb, bd, rho_a, px, pa);
        return cudaGetLastError() == cudaSuccess ? 0 : 3;
    }
    const float rgn = r->reference_gradient_norm;
    const auto anp = h->cv(r->non_pressure_acc);
    auto predict_forward = [&](const Vec& pressure_acc, const Vec& pos, const Vec& vel) {
        if (r->method == 1) cd::pcisph::launch_predict_forward(s, n, dt, box, x, v, anp, h->cv(pressure_acc), h->mv(pos), h->mv(vel));
        else if (r->method == 2) cd::iisph::launch_predict_forward(s, n, dt, box, x, v, anp, h->cv(pressure_acc), h->mv(pos), h->mv(vel));
        else cd::dfsph::launch_predict_forward(s, n, dt, box, x, v, anp, h->cv(pressure_acc), h->mv(pos), h->mv(vel));
    };
    auto predict_vjp = [&](const Vec& pressure_acc, const cd::ConstVectorView<double> pos_a, const cd::ConstVectorView<double> vel_a,
                           const DVec& pressure_acc_adjoint) {
        const auto npa = h->mdv(r->non_pressure_acc_adjoint);
        if (r->method == 1)
            cd::pcisph::launch_predict_vjp(s, n, dt, box, x, v, anp, h->cv(pressure_acc), pos_a, vel_a, px, pvv, npa, h->mdv(pressure_acc_adjoint));
        else if (r->method == 2)
            cd::iisph::launch_predict_vjp(s, n, dt, box, x, v, anp, h->cv(pressure_acc), pos_a, vel_a, px, pvv, npa, h->mdv(pressure_acc_adjoint));
        else
            cd::dfsph::launch_predict_vjp(s, n, dt, box, x, v, anp, h->cv(pressure_acc), pos_a, vel_a, px, pvv, npa, h->mdv(pressure_acc_adjoint));
    };
    auto pressure_forward = [&](IterCache& c) {
        cd::sph::pressure_forward(s, n, hr, x, pv, nb, bd, rho, c.pressures, h->mv(c.pressure_acc));
    };
    auto pressure_vjp = [&](const float* pressures) {
        cd::sph::pressure_vjp(s, n, hr, x, pv, nb, bd, rho, pressures, h->cdv(r->adjoint.pressure_acc), px, rho_a,
                              r->adjoint.pressures, pa);
    };
    r->clear(r->non_pressure_acc_adjoint);
    r->clear(r->adjoint);
    r->clear(r->previous_adjoint);
    if (r->method == 1 || r->method == 2) {   // PCISPH::vjp / IISPH::vjp (sph/sph.cpp:332-373, 445-486)
        predict_vjp(r->checkpoints.back().pressure_acc, nx, nv, r->adjoint.pressure_acc);
        for (size_t c = r->checkpoints.size() - 1; c > 0; --c) {
            const IterCache& first = r->checkpoints[c - 1];
            const IterCache& last = r->checkpoints[c];
            r->copy(first, r->recomputed[0]);
            for (uint32_t it = first.iteration + 1u; it <= last.iteration; ++it) {
                IterCache& prev = r->recomputed[it - first.iteration - 1u];
                IterCache& cur = r->recomputed[it - first.iteration];
                cur.iteration = it;
                predict_forward(prev.pressure_acc, cur.predicted_positions, cur.predicted_velocities);
                cd::density_forward(s, n, hr, false, x, h->cv(cur.predicted_positions), pv, nb, bd, cur.predicted_densities);
                if (r->method == 1)
                    cd::pcisph::launch_pressure_update_forward(s, n, dt, rgn, pv, prev.pressures, cur.predicted_densities,
                                                               p->method0, cur.pressures);
                else
                    cd::iisph::launch_jacobi_update_forward(s, n, dt, rgn, pv, rho, prev.pressures, cur.predicted_densities,
                                                            p->method0, cur.pressures);
                pressure_forward(cur);
            }
            for (uint32_t it = last.iteration; it > first.iteration; --it) {
                IterCache& prev = r->recomputed[it - first.iteration - 1u];
                IterCache& cur = r->recomputed[it - first.iteration];
                r->clear(r->previous_adjoint);
                pressure_vjp(cur.pressures);
                if (r->method == 1)
                    cd::pcisph::launch_pressure_update_vjp(s, n, dt, rgn, pv, prev.pressures, cur.predicted_densities, p->method0,
                                                           r->adjoint.pressures, pa, r->previous_adjoint.pressures,
                                                           r->adjoint.predicted_densities, method_adjoint[0]);
                else
                    cd::iisph::launch_jacobi_update_vjp(s, n, dt, rgn, pv, rho, prev.pressures, cur.predicted_densities,
                                                        p->method0, r->adjoint.pressures, pa, rho_a, r->previous_adjoint.pressures,
                                                        r->adjoint.predicted_densities, method_adjoint[0]);
                cd::density_vjp(s, n, hr, false, x, h->cv(cur.predicted_positions), pv, nb, bd, r->adjoint.predicted_densities,
                                h->mdv(r->adjoint.predicted_positions), pa);
                predict_vjp(prev.pressure_acc, h->cdv(r->adjoint.predicted_positions), h->cdv(r->adjoint.predicted_velocities),
                            r->previous_adjoint.pressure_acc);
                std::swap(r->adjoint, r->previous_adjoint);
            }
        }
    } else {   // DFSPH::vjp (sph/sph.cpp:661-722)
        r->clear(r->target_density_adjoint);
        r->clear(r->divergence_pressure_acc_adjoint);
        r->clear(r->total_pressure_acc_adjoint);
        predict_vjp(r->total_pressure_acc, nx, nv, r->total_pressure_acc_adjoint);
        r->copy(r->total_pressure_acc_adjoint, r->divergence_pressure_acc_adjoint);
        r->copy(r->total_pressure_acc_adjoint, r->adjoint.pressure_acc);
        r->copy(next_warm[1], r->adjoint.pressures);
        auto reverse_phase = [&](std::vector<IterCache>& checkpoints, const float* relaxation, double* relaxation_adjoint,
                                 const float* target, double* target_adjoint, const Vec* base, const DVec* base_adjoint,
                                 double* warm_adjoint) {
            for (size_t c = checkpoints.size(); c-- > 1;) {
                const IterCache& first = checkpoints[c - 1];
                const IterCache& last = checkpoints[c];
                r->copy(first, r->recomputed[0]);
                for (uint32_t it = first.iteration + 1u; it <= last.iteration; ++it) {
                    IterCache& prev = r->recomputed[it - first.iteration - 1u];
                    IterCache& cur = r->recomputed[it - first.iteration];
                    cur.iteration = it;
                    const Vec* prediction = &prev.pressure_acc;
                    if (base) {
                        cd::sph::add(s, n, h->cv(*base), h->cv(prev.pressure_acc), h->mv(r->total_pressure_acceleration));
                        prediction = &r->total_pressure_acceleration;
                    }
                    predict_forward(*prediction, cur.predicted_positions, cur.predicted_velocities);
                    cd::density_forward(s, n, hr, false, x, h->cv(cur.predicted_positions), pv, nb, bd, cur.predicted_densities);
                    cd::dfsph::launch_projection_update_forward(s, n, dt, rgn, pv, rho, target, prev.pressures,
                                                                cur.predicted_densities, relaxation, cur.pressures);
                    pressure_forward(cur);
                }
                for (uint32_t it = last.iteration; it > first.iteration; --it) {
                    IterCache& prev = r->recomputed[it - first.iteration - 1u];
                    IterCache& cur = r->recomputed[it - first.iteration];
                    r->clear(r->previous_adjoint);
                    pressure_vjp(cur.pressures);
                    cd::dfsph::launch_projection_update_vjp(s, n, dt, rgn, pv, rho, target, prev.pressures, cur.predicted_densities,
                                                            relaxation, r->adjoint.pressures, pa, rho_a, target_adjoint,
                                                            r->previous_adjoint.pressures, r->adjoint.predicted_densities,
                                                            relaxation_adjoint);
                    cd::density_vjp(s, n, hr, false, x, h->cv(cur.predicted_positions), pv, nb, bd,
                                    r->adjoint.predicted_densities, h->mdv(r->adjoint.predicted_positions), pa);
                    if (!base) {
                        predict_vjp(prev.pressure_acc, h->cdv(r->adjoint.predicted_positions),
                                    h->cdv(r->adjoint.predicted_velocities), r->previous_adjoint.pressure_acc);
                    } else {
                        r->clear(r->total_pressure_acc_adjoint);
                        cd::sph::add(s, n, h->cv(*base), h->cv(prev.pressure_acc), h->mv(r->total_pressure_acceleration));
                        predict_vjp(r->total_pressure_acceleration, h->cdv(r->adjoint.predicted_positions),
                                    h->cdv(r->adjoint.predicted_velocities), r->total_pressure_acc_adjoint);
                        cd::sph::add_adjoint(s, n, h->cdv(r->total_pressure_acc_adjoint), h->mdv(*base_adjoint),
                                             h->mdv(r->previous_adjoint.pressure_acc));
                    }
                    std::swap(r->adjoint, r->previous_adjoint);
                }
            }
            pressure_vjp(checkpoints.front().pressures);
            if (r->warm_start) r->copy(r->adjoint.pressures, warm_adjoint);
        };
        reverse_phase(r->density_checkpoints, p->method1, method_adjoint[1], p->rest_densities, pa.rest_densities,
                      &r->divergence_pressure_acc, &r->divergence_pressure_acc_adjoint, previous_warm[1]);
        r->clear(r->adjoint);
        r->copy(r->divergence_pressure_acc_adjoint, r->adjoint.pressure_acc);
        r->copy(next_warm[0], r->adjoint.pressures);
        reverse_phase(r->divergence_checkpoints, p->method0, method_adjoint[0], rho, r->target_density_adjoint, nullptr, nullptr,
                      previous_warm[0]);
        cd::accumulate(s, r->target_density_adjoint, rho_a, n);
    }
    cd::sph::non_pressure_vjp(s, n, hr, x, v, pv, nb, bd, rho, h->cdv(r->non_pressure_acc_adjoint), px, pvv,
                              h->mdv(control_adjoint), rho_a, pa);
    cd::density_vjp(s, n, hr, false, x, x, pv, nb, bd, rho_a, px, pa);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Copy a field of the last SPH step to device memory (x, y, z: SoA destinations; scalars use x).
//   0 densities  1 pressures (WCSPH) / last iterate's pressures  2 pressure acceleration
//   3 viscosity acceleration (WCSPH) / non-pressure acceleration  4 surface acceleration (WCSPH)
//   5 predicted densities (last iterate)  6 total acceleration (WCSPH) / total pressure acceleration (DFSPH)
int ref_sph_read(void* sph, const int field, float* x, float* y, float* z) {
    auto* r = static_cast<SphReplay*>(sph);
    auto vec3 = [&](const Vec& v) {
        if (!v.x) return 1;
        r->copy(v.x, x);
        r->copy(v.y, y);
        r->copy(v.z, z);
        return 0;
    };
    auto scalar = [&](const float* f) {
        if (!f) return 1;
        r->copy(f, x);
        return 0;
    };
    const bool w = r->method == 0;
    int rc = 1;
    switch (field) {
        case 0: rc = scalar(r->densities); break;
        case 1: rc = scalar(w ? r->pressures : r->primal.pressures); break;
        case 2: rc = vec3(w ? r->pressure_acc : r->primal.pressure_acc); break;
        case 3: rc = vec3(w ? r->viscosity_acc : r->non_pressure_acc); break;
        case 4: rc = w ? vec3(r->surface_acc) : 1; break;
        case 5: rc = scalar(r->primal.predicted_densities); break;
        case 6: rc = vec3(w ? r->total_acc : r->total_pressure_acc); break;
        default: break;
    }
    if (rc) return rc;
    return cudaStreamSynchronize(r->h->stream) == cudaSuccess ? 0 : 3;
}

}  // extern "C"
