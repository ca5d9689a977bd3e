// physica_pbf.hpp -- C++17 front end of the B200 Position Based Fluids solver.
//
// Mirrors the reference's C++ interface, physica::fluids::liquid::particle::PBF
// (pbf/pbf.ixx:14-141), and the domain types it takes (domain/domain.ixx:12-165), over the C ABI
// of physica_pbf.h.  A caller written against the reference's PBF compiles against this header
// with the same names, members and argument meaning; it links libphysica_pbf.so and the CUDA
// runtime.
//
// Differences a caller can see:
//  - `::cuda::device_buffer<T>` and `::cuda::stream_ref` (CCCL) become `device_buffer<T>` below and
//    `cudaStream_t`: the reference's module build needs C++23 `import std`, which this header does
//    not.  The device_buffer here is move-only, zero-filled at allocation and freed with cudaFree.
//  - PBF::StepCache is opaque: the solver keeps the neighbourhood, the Jacobi iterates and the
//    post-loop fields in its own cell-sorted layout.  `StepCache::handle()` reads them with
//    pbf_step_cache_read / pbf_step_cache_read_iteration, in the reference's original order.
//  - Failures throw physica::fluids::liquid::particle::Error (a std::runtime_error carrying the
//    pbf_status); the reference throws from CCCL on allocation failures and checks no launch.
//  - Like the reference, every call is asynchronous on the solver's stream, vjp_step accumulates
//    into its outputs, and PBF is neither copyable nor movable.
#ifndef PHYSICA_PBF_HPP
#define PHYSICA_PBF_HPP

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "physica_pbf.h"

namespace physica::fluids::liquid::particle {

// A failed call: `status` is the pbf_status (or PBF_ERROR_CUDA for a CUDA runtime error here).
struct Error : std::runtime_error {
    int status;
    Error(const int s, const std::string& message) : std::runtime_error(message), status(s) {}
};

namespace detail {
inline void check(const int status) {
    if (status != PBF_SUCCESS) throw Error(status, std::string(pbf_status_string(status)) + ": " + pbf_last_error());
}
inline void check_cuda(const cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(PBF_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace detail

// Device array of `count` elements (the reference's ::cuda::device_buffer<T>).
template <class T>
class device_buffer {
public:
    device_buffer() = default;
    device_buffer(const std::size_t count, cudaStream_t stream) : size_(count) {
        if (count == 0) return;
        detail::check_cuda(cudaMalloc(reinterpret_cast<void**>(&data_), count * sizeof(T)), "device_buffer allocation");
        detail::check_cuda(cudaMemsetAsync(data_, 0, count * sizeof(T), stream), "device_buffer fill");
    }
    ~device_buffer() { release(); }
    device_buffer(const device_buffer&) = delete;
    device_buffer& operator=(const device_buffer&) = delete;
    device_buffer(device_buffer&& o) noexcept : data_(std::exchange(o.data_, nullptr)), size_(std::exchange(o.size_, 0)) {}
    device_buffer& operator=(device_buffer&& o) noexcept {
        if (this != &o) {
            release();
            data_ = std::exchange(o.data_, nullptr);
            size_ = std::exchange(o.size_, 0);
        }
        return *this;
    }
    T* data() { return data_; }
    const T* data() const { return data_; }
    std::size_t size() const { return size_; }

private:
    void release() {
        if (data_) cudaFree(data_);
        data_ = nullptr;
        size_ = 0;
    }
    T* data_ = nullptr;
    std::size_t size_ = 0;
};

// ---------------------------------------------------------------- domain/domain.ixx:12-119
struct Vector3 {
    float x;
    float y;
    float z;
};

struct BoxBoundary {
    Vector3 minimum;
    Vector3 maximum;
    Vector3 velocity;
    bool no_slip{true};
};

struct BoundaryParticle {
    Vector3 position;
    Vector3 velocity;
    float volume;
};

struct DomainConfiguration {
    std::uint32_t particle_count;
    float time_step;
    float support_radius;
    float particle_radius;
    Vector3 gravity;
    BoxBoundary boundary;
    std::vector<BoundaryParticle> boundary_particles;
};

enum class ExecutionMode : std::uint32_t {
    forward,
    differentiable,
};

struct ScalarField {
    device_buffer<float> values;
};
struct ScalarAdjointField {
    device_buffer<double> values;
};
struct VectorField {
    device_buffer<float> x;
    device_buffer<float> y;
    device_buffer<float> z;
};
struct VectorAdjointField {
    device_buffer<double> x;
    device_buffer<double> y;
    device_buffer<double> z;
};

struct ParticleState {
    VectorField positions;
    VectorField velocities;
    std::uint64_t step_index{};
};
struct Control {
    VectorField external_accelerations;
};
struct ParticleStateTangent {
    VectorField positions;
    VectorField velocities;
};
struct ControlTangent {
    VectorField external_accelerations;
};
struct ParticleStateAdjoint {
    VectorAdjointField positions;
    VectorAdjointField velocities;
};
struct ControlAdjoint {
    VectorAdjointField external_accelerations;
};

struct ParticleParameters {
    device_buffer<float> masses;
    device_buffer<float> rest_densities;
    device_buffer<float> viscosities;
    device_buffer<float> surface_tensions;
};
struct ParticleParameterTangent {
    device_buffer<float> masses;
    device_buffer<float> rest_densities;
    device_buffer<float> viscosities;
    device_buffer<float> surface_tensions;
};
struct ParticleParameterAdjoint {
    device_buffer<double> masses;
    device_buffer<double> rest_densities;
    device_buffer<double> viscosities;
    device_buffer<double> surface_tensions;
};

namespace detail {
inline pbf_vector_field view(const VectorField& f) {
    return {const_cast<float*>(f.x.data()), const_cast<float*>(f.y.data()), const_cast<float*>(f.z.data())};
}
inline pbf_vector_adjoint_field view(const VectorAdjointField& f) {
    return {const_cast<double*>(f.x.data()), const_cast<double*>(f.y.data()), const_cast<double*>(f.z.data())};
}
inline VectorField vector_field(const std::size_t n, cudaStream_t s) { return {{n, s}, {n, s}, {n, s}}; }
inline VectorAdjointField vector_adjoint_field(const std::size_t n, cudaStream_t s) { return {{n, s}, {n, s}, {n, s}}; }
// The C description of a domain; `storage` holds the boundary particles it points to.
inline pbf_domain_configuration domain_view(const DomainConfiguration& d, std::vector<pbf_boundary_particle>& storage) {
    storage.clear();
    storage.reserve(d.boundary_particles.size());
    for (const BoundaryParticle& b : d.boundary_particles)
        storage.push_back({{b.position.x, b.position.y, b.position.z}, {b.velocity.x, b.velocity.y, b.velocity.z}, b.volume});
    return {d.particle_count,
            d.time_step,
            d.support_radius,
            d.particle_radius,
            {d.gravity.x, d.gravity.y, d.gravity.z},
            {{d.boundary.minimum.x, d.boundary.minimum.y, d.boundary.minimum.z},
             {d.boundary.maximum.x, d.boundary.maximum.y, d.boundary.maximum.z},
             {d.boundary.velocity.x, d.boundary.velocity.y, d.boundary.velocity.z},
             d.boundary.no_slip ? 1u : 0u},
            storage.empty() ? nullptr : storage.data(),
            static_cast<std::uint32_t>(storage.size())};
}
}  // namespace detail

// ---------------------------------------------------------------- pbf/pbf.ixx:14-141
struct PBF final {
    struct Configuration {
        std::uint32_t pressure_iterations{5u};
        std::uint32_t checkpoint_interval{2u};
    };

    struct State {
        ParticleState particles;
    };
    struct StateTangent {
        ParticleStateTangent particles;
    };
    struct StateAdjoint {
        ParticleStateAdjoint particles;
    };

    struct Parameters {
        ParticleParameters particles;
        device_buffer<float> relaxation;
        device_buffer<float> artificial_pressure_strength;
        device_buffer<float> artificial_pressure_exponent;
        device_buffer<float> artificial_pressure_radius;
        device_buffer<float> xsph_viscosity;
        device_buffer<float> vorticity_confinement;
    };
    struct ParameterTangent {
        ParticleParameterTangent particles;
        device_buffer<float> relaxation;
        device_buffer<float> artificial_pressure_strength;
        device_buffer<float> artificial_pressure_exponent;
        device_buffer<float> artificial_pressure_radius;
        device_buffer<float> xsph_viscosity;
        device_buffer<float> vorticity_confinement;
    };
    struct ParameterAdjoint {
        ParticleParameterAdjoint particles;
        device_buffer<double> relaxation;
        device_buffer<double> artificial_pressure_strength;
        device_buffer<double> artificial_pressure_exponent;
        device_buffer<double> artificial_pressure_radius;
        device_buffer<double> xsph_viscosity;
        device_buffer<double> vorticity_confinement;
    };

    // Opaque: the library's step cache (pbf_step_cache), freed with the object.
    class StepCache {
    public:
        StepCache() = default;
        explicit StepCache(pbf_step_cache* handle) : handle_(handle) {}
        ~StepCache() {
            if (handle_) pbf_free_step_cache(handle_);
        }
        StepCache(const StepCache&) = delete;
        StepCache& operator=(const StepCache&) = delete;
        StepCache(StepCache&& o) noexcept : handle_(std::exchange(o.handle_, nullptr)) {}
        StepCache& operator=(StepCache&& o) noexcept {
            if (this != &o) {
                if (handle_) pbf_free_step_cache(handle_);
                handle_ = std::exchange(o.handle_, nullptr);
            }
            return *this;
        }
        pbf_step_cache* handle() const { return handle_; }

    private:
        pbf_step_cache* handle_ = nullptr;
    };

    PBF(DomainConfiguration domain_configuration, Configuration configuration, ExecutionMode mode, cudaStream_t stream)
        : configuration_(configuration), count_(domain_configuration.particle_count), stream_(stream) {
        std::vector<pbf_boundary_particle> boundary;
        const pbf_domain_configuration dc = detail::domain_view(domain_configuration, boundary);
        const pbf_configuration cc{configuration.pressure_iterations, configuration.checkpoint_interval};
        detail::check(pbf_create(&dc, &cc,
                                 mode == ExecutionMode::differentiable ? PBF_EXECUTION_DIFFERENTIABLE : PBF_EXECUTION_FORWARD,
                                 stream, &handle_));
    }
    ~PBF() {
        if (handle_) pbf_destroy(handle_);
    }
    PBF(const PBF&) = delete;
    PBF& operator=(const PBF&) = delete;
    PBF(PBF&&) = delete;
    PBF& operator=(PBF&&) = delete;

    // Step caches allocated afterwards keep every checkpoint_interval-th Jacobi iterate only, as the
    // reference's StepCache does, and vjp_step / jvp_step recompute the iterations in between
    // (differentiable mode; off by default: every iterate kept).
    void set_checkpoint_recompute(bool enable) { detail::check(pbf_set_checkpoint_recompute(handle_, enable ? 1 : 0)); }

    [[nodiscard]] State allocate_state() const {
        return {{detail::vector_field(count_, stream_), detail::vector_field(count_, stream_), 0u}};
    }
    [[nodiscard]] Control allocate_control() const { return {detail::vector_field(count_, stream_)}; }
    [[nodiscard]] Parameters allocate_parameters() const {
        return {{f(), f(), f(), f()}, f(), f(), f(), f(), f(), f()};
    }
    [[nodiscard]] StepCache allocate_step_cache() const {
        pbf_step_cache* cache = nullptr;
        detail::check(pbf_allocate_step_cache(handle_, &cache));
        return StepCache(cache);
    }
    [[nodiscard]] StateTangent allocate_state_tangent() const {
        return {{detail::vector_field(count_, stream_), detail::vector_field(count_, stream_)}};
    }
    [[nodiscard]] ControlTangent allocate_control_tangent() const { return {detail::vector_field(count_, stream_)}; }
    [[nodiscard]] ParameterTangent allocate_parameter_tangent() const {
        return {{f(), f(), f(), f()}, f(), f(), f(), f(), f(), f()};
    }
    [[nodiscard]] StateAdjoint allocate_state_adjoint() const {
        return {{detail::vector_adjoint_field(count_, stream_), detail::vector_adjoint_field(count_, stream_)}};
    }
    [[nodiscard]] ControlAdjoint allocate_control_adjoint() const { return {detail::vector_adjoint_field(count_, stream_)}; }
    [[nodiscard]] ParameterAdjoint allocate_parameter_adjoint() const {
        return {{d(), d(), d(), d()}, d(), d(), d(), d(), d(), d()};
    }

    void copy_state(const State& source, State& destination) const {
        const pbf_particle_state s = state(source);
        pbf_particle_state t = state(destination);
        detail::check(pbf_copy_state(handle_, &s, &t));
        destination.particles.step_index = source.particles.step_index;
    }
    void copy_state_tangent(const StateTangent& source, StateTangent& destination) const {
        const pbf_particle_state_tangent s = tangent(source);
        pbf_particle_state_tangent t = tangent(destination);
        detail::check(pbf_copy_state_tangent(handle_, &s, &t));
    }
    void copy_state_adjoint(const StateAdjoint& source, StateAdjoint& destination) const {
        const pbf_particle_state_adjoint s = adjoint(source);
        pbf_particle_state_adjoint t = adjoint(destination);
        detail::check(pbf_copy_state_adjoint(handle_, &s, &t));
    }
    void accumulate_state_adjoint(const StateAdjoint& source, StateAdjoint& destination) const {
        const pbf_particle_state_adjoint s = adjoint(source);
        pbf_particle_state_adjoint t = adjoint(destination);
        detail::check(pbf_accumulate_state_adjoint(handle_, &s, &t));
    }

    void forward_step(const State& state_in, const Control& control, const Parameters& parameters, State& next_state,
                      StepCache& cache) {
        const pbf_particle_state s = state(state_in);
        pbf_particle_state n = state(next_state);
        const pbf_control c{detail::view(control.external_accelerations)};
        const pbf_parameters p = params(parameters);
        detail::check(pbf_forward_step(handle_, &s, &c, &p, &n, cache.handle()));
        next_state.particles.step_index = n.step_index;
    }
    void jvp_step(const State& state_in, const Control& control, const Parameters& parameters, const State& next_state,
                  const StepCache& cache, const StateTangent& state_tangent, const ControlTangent& control_tangent,
                  const ParameterTangent& parameter_tangent, StateTangent& next_state_tangent) {
        const pbf_particle_state s = state(state_in), n = state(next_state);
        const pbf_control c{detail::view(control.external_accelerations)};
        const pbf_parameters p = params(parameters);
        const pbf_particle_state_tangent st = tangent(state_tangent);
        pbf_particle_state_tangent nt = tangent(next_state_tangent);
        const pbf_control ct{detail::view(control_tangent.external_accelerations)};
        const pbf_parameter_tangent pt = params(parameter_tangent);
        detail::check(pbf_jvp_step(handle_, &s, &c, &p, &n, cache.handle(), &st, &ct, &pt, &nt));
    }
    void vjp_step(const State& state_in, const Control& control, const Parameters& parameters, const State& next_state,
                  const StepCache& cache, const StateAdjoint& next_state_adjoint, StateAdjoint& previous_state_adjoint,
                  ControlAdjoint& control_adjoint, ParameterAdjoint& parameter_adjoint) {
        const pbf_particle_state s = state(state_in), n = state(next_state);
        const pbf_control c{detail::view(control.external_accelerations)};
        const pbf_parameters p = params(parameters);
        const pbf_particle_state_adjoint na = adjoint(next_state_adjoint);
        pbf_particle_state_adjoint pa = adjoint(previous_state_adjoint);
        pbf_control_adjoint ca{detail::view(control_adjoint.external_accelerations)};
        pbf_parameter_adjoint qa = params(parameter_adjoint);
        detail::check(pbf_vjp_step(handle_, &s, &c, &p, &n, cache.handle(), &na, &pa, &ca, &qa));
    }

    // Not in the reference's interface: the C ABI handle, the stream, and a wait for queued work.
    pbf_solver* handle() const { return handle_; }
    cudaStream_t stream() const { return stream_; }
    void synchronize() const { detail::check(pbf_synchronize(handle_)); }

private:
    device_buffer<float> f() const { return device_buffer<float>(count_, stream_); }
    device_buffer<double> d() const { return device_buffer<double>(count_, stream_); }
    static pbf_particle_state state(const State& s) {
        return {detail::view(s.particles.positions), detail::view(s.particles.velocities), s.particles.step_index};
    }
    static pbf_particle_state_tangent tangent(const StateTangent& s) {
        return {detail::view(s.particles.positions), detail::view(s.particles.velocities)};
    }
    static pbf_particle_state_adjoint adjoint(const StateAdjoint& s) {
        return {detail::view(s.particles.positions), detail::view(s.particles.velocities)};
    }
    template <class P>
    static pbf_parameters params(const P& p) {
        return {p.particles.masses.data(),       p.particles.rest_densities.data(),
                p.particles.viscosities.data(),  p.particles.surface_tensions.data(),
                p.relaxation.data(),             p.artificial_pressure_strength.data(),
                p.artificial_pressure_exponent.data(), p.artificial_pressure_radius.data(),
                p.xsph_viscosity.data(),         p.vorticity_confinement.data()};
    }
    static pbf_parameter_adjoint params(ParameterAdjoint& p) {
        return {p.particles.masses.data(),       p.particles.rest_densities.data(),
                p.particles.viscosities.data(),  p.particles.surface_tensions.data(),
                p.relaxation.data(),             p.artificial_pressure_strength.data(),
                p.artificial_pressure_exponent.data(), p.artificial_pressure_radius.data(),
                p.xsph_viscosity.data(),         p.vorticity_confinement.data()};
    }

    Configuration configuration_;
    std::size_t count_;
    cudaStream_t stream_;
    pbf_solver* handle_ = nullptr;
};

// ---------------------------------------------------------------- host transfers
// The reference's Domain::upload (domain/domain.ixx:163-164), stream-ordered; the host data must
// stay alive until the stream reaches the copy (pageable memory: the call returns after it).
inline void upload(const std::vector<float>& source, device_buffer<float>& destination, cudaStream_t stream) {
    if (source.size() != destination.size()) throw Error(PBF_ERROR_INVALID_ARGUMENT, "upload: size mismatch");
    detail::check_cuda(cudaMemcpyAsync(destination.data(), source.data(), source.size() * sizeof(float),
                                       cudaMemcpyHostToDevice, stream),
                       "upload");
}
inline void upload(const std::vector<Vector3>& source, VectorField& destination, cudaStream_t stream) {
    std::vector<float> x(source.size()), y(source.size()), z(source.size());
    for (std::size_t i = 0; i < source.size(); ++i) {
        x[i] = source[i].x;
        y[i] = source[i].y;
        z[i] = source[i].z;
    }
    upload(x, destination.x, stream);
    upload(y, destination.y, stream);
    upload(z, destination.z, stream);
    detail::check_cuda(cudaStreamSynchronize(stream), "upload");   // x, y, z are about to go out of scope
}
// Reads a field back to the host (waits for the stream).
inline std::vector<float> download(const device_buffer<float>& source, cudaStream_t stream) {
    std::vector<float> out(source.size());
    detail::check_cuda(cudaMemcpyAsync(out.data(), source.data(), out.size() * sizeof(float), cudaMemcpyDeviceToHost, stream),
                       "download");
    detail::check_cuda(cudaStreamSynchronize(stream), "download");
    return out;
}
inline std::vector<double> download(const device_buffer<double>& source, cudaStream_t stream) {
    std::vector<double> out(source.size());
    detail::check_cuda(cudaMemcpyAsync(out.data(), source.data(), out.size() * sizeof(double), cudaMemcpyDeviceToHost, stream),
                       "download");
    detail::check_cuda(cudaStreamSynchronize(stream), "download");
    return out;
}

}  // namespace physica::fluids::liquid::particle

#endif  // PHYSICA_PBF_HPP
