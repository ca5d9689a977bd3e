// physica_sph.hpp -- C++17 front end of the B200 SPH solvers.
//
// Mirrors the reference's SPH<Method> (sph/sph.ixx:273-372) with Method one of WCSPH
// (sph/sph.ixx:39-101), PCISPH (:103-147), IISPH (:149-193) and DFSPH (:195-268), over the C ABI
// of physica_sph.h.  The domain types, device_buffer and Error come from physica_pbf.hpp, with the
// same differences from the reference noted there.  SPH<Method>::StepCache is opaque (read it
// with sph_read_cache through `cache.handle()`).  The methods' Cache / Differentiation members and
// their forward / jvp / vjp members, which SPH<Method> calls internally, are not part of this
// front end: the library runs them.
#ifndef PHYSICA_SPH_HPP
#define PHYSICA_SPH_HPP

#include <type_traits>

#include "physica_pbf.hpp"
#include "physica_sph.h"

namespace physica::fluids::liquid::particle {

namespace detail {
// A method's configuration as the C ABI takes it.
inline sph_configuration sph_config(const sph_method m, const std::uint32_t pressure, const std::uint32_t divergence,
                                    const std::uint32_t density, const std::uint32_t checkpoint, const bool warm) {
    return {m, pressure, divergence, density, checkpoint, warm ? 1u : 0u};
}
}  // namespace detail

// ---------------------------------------------------------------- sph/sph.ixx:39-101
struct WCSPH final {
    struct Configuration {};
    struct State {};
    struct StateTangent {};
    struct StateAdjoint {};
    struct Parameters {
        device_buffer<float> speed_of_sound;
        device_buffer<float> tait_exponent;
        device_buffer<float> boundary_surface_tension;
    };
    struct ParameterTangent {
        device_buffer<float> speed_of_sound;
        device_buffer<float> tait_exponent;
        device_buffer<float> boundary_surface_tension;
    };
    struct ParameterAdjoint {
        device_buffer<double> speed_of_sound;
        device_buffer<double> tait_exponent;
        device_buffer<double> boundary_surface_tension;
    };

    static sph_configuration configure(const Configuration&) { return detail::sph_config(SPH_METHOD_WCSPH, 6u, 4u, 6u, 2u, true); }
    static State state(std::size_t, cudaStream_t) { return {}; }
    static StateAdjoint state_adjoint(std::size_t, cudaStream_t) { return {}; }
    template <class P>
    static P parameters(const std::size_t n, cudaStream_t s) {
        return {{n, s}, {n, s}, {n, s}};
    }
    template <class C, class P>
    static void bind(C& c, const P& p) {
        c.speed_of_sound = const_cast<decltype(c.speed_of_sound)>(p.speed_of_sound.data());
        c.tait_exponent = const_cast<decltype(c.tait_exponent)>(p.tait_exponent.data());
        c.boundary_surface_tension = const_cast<decltype(c.boundary_surface_tension)>(p.boundary_surface_tension.data());
    }
};

// ---------------------------------------------------------------- sph/sph.ixx:103-147
struct PCISPH final {
    struct Configuration {
        std::uint32_t pressure_iterations{6u};
        std::uint32_t checkpoint_interval{2u};
    };
    struct State {};
    struct StateTangent {};
    struct StateAdjoint {};
    struct Parameters {
        device_buffer<float> pressure_relaxation;
    };
    struct ParameterTangent {
        device_buffer<float> pressure_relaxation;
    };
    struct ParameterAdjoint {
        device_buffer<double> pressure_relaxation;
    };

    static sph_configuration configure(const Configuration& c) {
        return detail::sph_config(SPH_METHOD_PCISPH, c.pressure_iterations, 4u, 6u, c.checkpoint_interval, true);
    }
    static State state(std::size_t, cudaStream_t) { return {}; }
    static StateAdjoint state_adjoint(std::size_t, cudaStream_t) { return {}; }
    template <class P>
    static P parameters(const std::size_t n, cudaStream_t s) {
        return {{n, s}};
    }
    template <class C, class P>
    static void bind(C& c, const P& p) {
        c.pressure_relaxation = const_cast<decltype(c.pressure_relaxation)>(p.pressure_relaxation.data());
    }
};

// ---------------------------------------------------------------- sph/sph.ixx:149-193
struct IISPH final {
    struct Configuration {
        std::uint32_t pressure_iterations{6u};
        std::uint32_t checkpoint_interval{2u};
    };
    struct State {};
    struct StateTangent {};
    struct StateAdjoint {};
    struct Parameters {
        device_buffer<float> jacobi_relaxation;
    };
    struct ParameterTangent {
        device_buffer<float> jacobi_relaxation;
    };
    struct ParameterAdjoint {
        device_buffer<double> jacobi_relaxation;
    };

    static sph_configuration configure(const Configuration& c) {
        return detail::sph_config(SPH_METHOD_IISPH, c.pressure_iterations, 4u, 6u, c.checkpoint_interval, true);
    }
    static State state(std::size_t, cudaStream_t) { return {}; }
    static StateAdjoint state_adjoint(std::size_t, cudaStream_t) { return {}; }
    template <class P>
    static P parameters(const std::size_t n, cudaStream_t s) {
        return {{n, s}};
    }
    template <class C, class P>
    static void bind(C& c, const P& p) {
        c.jacobi_relaxation = const_cast<decltype(c.jacobi_relaxation)>(p.jacobi_relaxation.data());
    }
};

// ---------------------------------------------------------------- sph/sph.ixx:195-268
struct DFSPH final {
    struct Configuration {
        std::uint32_t divergence_iterations{4u};
        std::uint32_t density_iterations{6u};
        std::uint32_t checkpoint_interval{2u};
        bool pressure_warm_start{true};
    };
    struct State {
        ScalarField warm_divergence_pressure;
        ScalarField warm_density_pressure;
    };
    struct StateTangent {
        ScalarField warm_divergence_pressure;
        ScalarField warm_density_pressure;
    };
    struct StateAdjoint {
        ScalarAdjointField warm_divergence_pressure;
        ScalarAdjointField warm_density_pressure;
    };
    struct Parameters {
        device_buffer<float> divergence_relaxation;
        device_buffer<float> density_relaxation;
    };
    struct ParameterTangent {
        device_buffer<float> divergence_relaxation;
        device_buffer<float> density_relaxation;
    };
    struct ParameterAdjoint {
        device_buffer<double> divergence_relaxation;
        device_buffer<double> density_relaxation;
    };

    static sph_configuration configure(const Configuration& c) {
        return detail::sph_config(SPH_METHOD_DFSPH, 6u, c.divergence_iterations, c.density_iterations, c.checkpoint_interval,
                                  c.pressure_warm_start);
    }
    static State state(const std::size_t n, cudaStream_t s) { return {{{n, s}}, {{n, s}}}; }
    static StateAdjoint state_adjoint(const std::size_t n, cudaStream_t s) { return {{{n, s}}, {{n, s}}}; }
    template <class P>
    static P parameters(const std::size_t n, cudaStream_t s) {
        return {{n, s}, {n, s}};
    }
    template <class C, class P>
    static void bind(C& c, const P& p) {
        c.divergence_relaxation = const_cast<decltype(c.divergence_relaxation)>(p.divergence_relaxation.data());
        c.density_relaxation = const_cast<decltype(c.density_relaxation)>(p.density_relaxation.data());
    }
};

namespace detail {
// Method::State / StateTangent as the C ABI's sph_method_state (the warm starts of DFSPH, else null).
template <class S>
sph_method_state method_state(const S& s) {
    if constexpr (std::is_same_v<S, DFSPH::State> || std::is_same_v<S, DFSPH::StateTangent>)
        return {const_cast<float*>(s.warm_divergence_pressure.values.data()),
                const_cast<float*>(s.warm_density_pressure.values.data())};
    else
        return {nullptr, nullptr};
}
template <class S>
sph_method_state_adjoint method_adjoint(const S& s) {
    if constexpr (std::is_same_v<S, DFSPH::StateAdjoint>)
        return {const_cast<double*>(s.warm_divergence_pressure.values.data()),
                const_cast<double*>(s.warm_density_pressure.values.data())};
    else
        return {nullptr, nullptr};
}
}  // namespace detail

// ---------------------------------------------------------------- sph/sph.ixx:270-372
template <class Method>
struct SPH final {
    static_assert(std::is_same_v<Method, WCSPH> || std::is_same_v<Method, PCISPH> || std::is_same_v<Method, IISPH> ||
                      std::is_same_v<Method, DFSPH>,
                  "SPH<Method>: Method is WCSPH, PCISPH, IISPH or DFSPH");

    struct State {
        ParticleState particles;
        typename Method::State method;
    };
    struct StateTangent {
        ParticleStateTangent particles;
        typename Method::StateTangent method;
    };
    struct StateAdjoint {
        ParticleStateAdjoint particles;
        typename Method::StateAdjoint method;
    };
    struct Parameters {
        ParticleParameters particles;
        typename Method::Parameters method;
    };
    struct ParameterTangent {
        ParticleParameterTangent particles;
        typename Method::ParameterTangent method;
    };
    struct ParameterAdjoint {
        ParticleParameterAdjoint particles;
        typename Method::ParameterAdjoint method;
    };

    // Opaque: the library's step cache (sph_step_cache), freed with the object.
    class StepCache {
    public:
        StepCache() = default;
        StepCache(sph_solver* solver, sph_step_cache* handle) : solver_(solver), handle_(handle) {}
        ~StepCache() { release(); }
        StepCache(const StepCache&) = delete;
        StepCache& operator=(const StepCache&) = delete;
        StepCache(StepCache&& o) noexcept : solver_(o.solver_), handle_(std::exchange(o.handle_, nullptr)) {}
        StepCache& operator=(StepCache&& o) noexcept {
            if (this != &o) {
                release();
                solver_ = o.solver_;
                handle_ = std::exchange(o.handle_, nullptr);
            }
            return *this;
        }
        sph_step_cache* handle() const { return handle_; }

    private:
        void release() {
            if (handle_) sph_free_step_cache(solver_, handle_);
            handle_ = nullptr;
        }
        sph_solver* solver_ = nullptr;
        sph_step_cache* handle_ = nullptr;
    };

    SPH(DomainConfiguration domain_configuration, typename Method::Configuration method_configuration,
        const ExecutionMode mode, cudaStream_t stream)
        : count_(domain_configuration.particle_count), stream_(stream) {
        std::vector<pbf_boundary_particle> boundary;
        const pbf_domain_configuration dc = detail::domain_view(domain_configuration, boundary);
        const sph_configuration cc = Method::configure(method_configuration);
        detail::check(sph_create(&dc, &cc,
                                 mode == ExecutionMode::differentiable ? PBF_EXECUTION_DIFFERENTIABLE : PBF_EXECUTION_FORWARD,
                                 stream, &handle_));
    }
    ~SPH() {
        if (handle_) sph_destroy(handle_);
    }
    SPH(const SPH&) = delete;
    SPH& operator=(const SPH&) = delete;
    SPH(SPH&&) = delete;
    SPH& operator=(SPH&&) = delete;

    [[nodiscard]] State allocate_state() const {
        return {{detail::vector_field(count_, stream_), detail::vector_field(count_, stream_), 0u}, Method::state(count_, stream_)};
    }
    [[nodiscard]] Control allocate_control() const { return {detail::vector_field(count_, stream_)}; }
    [[nodiscard]] Parameters allocate_parameters() const {
        return {particle_parameters<ParticleParameters>(), Method::template parameters<typename Method::Parameters>(count_, stream_)};
    }
    [[nodiscard]] StepCache allocate_step_cache() const {
        sph_step_cache* cache = nullptr;
        detail::check(sph_allocate_step_cache(handle_, &cache));
        return StepCache(handle_, cache);
    }
    [[nodiscard]] StateTangent allocate_state_tangent() const {
        typename Method::StateTangent method{};
        if constexpr (std::is_same_v<Method, DFSPH>) method = {{{count_, stream_}}, {{count_, stream_}}};
        return {{detail::vector_field(count_, stream_), detail::vector_field(count_, stream_)}, std::move(method)};
    }
    [[nodiscard]] ControlTangent allocate_control_tangent() const { return {detail::vector_field(count_, stream_)}; }
    [[nodiscard]] ParameterTangent allocate_parameter_tangent() const {
        return {particle_parameters<ParticleParameterTangent>(),
                Method::template parameters<typename Method::ParameterTangent>(count_, stream_)};
    }
    [[nodiscard]] StateAdjoint allocate_state_adjoint() const {
        return {{detail::vector_adjoint_field(count_, stream_), detail::vector_adjoint_field(count_, stream_)},
                Method::state_adjoint(count_, stream_)};
    }
    [[nodiscard]] ControlAdjoint allocate_control_adjoint() const { return {detail::vector_adjoint_field(count_, stream_)}; }
    [[nodiscard]] ParameterAdjoint allocate_parameter_adjoint() const {
        return {particle_parameters<ParticleParameterAdjoint>(),
                Method::template parameters<typename Method::ParameterAdjoint>(count_, stream_)};
    }

    void copy_state(const State& source, State& destination) const {
        const pbf_particle_state s = particles(source);
        pbf_particle_state d = particles(destination);
        const sph_method_state sm = detail::method_state(source.method);
        sph_method_state dm = detail::method_state(destination.method);
        detail::check(sph_copy_state(handle_, &s, &sm, &d, &dm));
        destination.particles.step_index = source.particles.step_index;
    }
    void copy_state_tangent(const StateTangent& source, StateTangent& destination) const {
        const pbf_particle_state_tangent s = particles(source);
        pbf_particle_state_tangent d = particles(destination);
        const sph_method_state sm = detail::method_state(source.method);
        sph_method_state dm = detail::method_state(destination.method);
        detail::check(sph_copy_state_tangent(handle_, &s, &sm, &d, &dm));
    }
    void copy_state_adjoint(const StateAdjoint& source, StateAdjoint& destination) const {
        const pbf_particle_state_adjoint s = particles(source);
        pbf_particle_state_adjoint d = particles(destination);
        const sph_method_state_adjoint sm = detail::method_adjoint(source.method);
        sph_method_state_adjoint dm = detail::method_adjoint(destination.method);
        detail::check(sph_copy_state_adjoint(handle_, &s, &sm, &d, &dm));
    }
    void accumulate_state_adjoint(const StateAdjoint& source, StateAdjoint& destination) const {
        const pbf_particle_state_adjoint s = particles(source);
        pbf_particle_state_adjoint d = particles(destination);
        const sph_method_state_adjoint sm = detail::method_adjoint(source.method);
        sph_method_state_adjoint dm = detail::method_adjoint(destination.method);
        detail::check(sph_accumulate_state_adjoint(handle_, &s, &sm, &d, &dm));
    }

    void forward_step(const State& state, const Control& control, const Parameters& parameters, State& next_state,
                      StepCache& cache) {
        const pbf_particle_state s = particles(state);
        pbf_particle_state n = particles(next_state);
        const sph_method_state sm = detail::method_state(state.method);
        sph_method_state nm = detail::method_state(next_state.method);
        const pbf_control c{detail::view(control.external_accelerations)};
        const sph_parameters p = c_parameters<sph_parameters>(parameters);
        detail::check(sph_forward_step(handle_, &s, &sm, &c, &p, &n, &nm, cache.handle()));
        next_state.particles.step_index = n.step_index;
    }
    void jvp_step(const State& state, const Control& control, const Parameters& parameters, const State& next_state,
                  const StepCache& cache, const StateTangent& state_tangent, const ControlTangent& control_tangent,
                  const ParameterTangent& parameter_tangent, StateTangent& next_state_tangent) {
        const pbf_particle_state s = particles(state), n = particles(next_state);
        const sph_method_state sm = detail::method_state(state.method);
        const pbf_control c{detail::view(control.external_accelerations)};
        const sph_parameters p = c_parameters<sph_parameters>(parameters);
        const pbf_particle_state_tangent st = particles(state_tangent);
        const sph_method_state smt = detail::method_state(state_tangent.method);
        const pbf_control ct{detail::view(control_tangent.external_accelerations)};
        const sph_parameter_tangent pt = c_parameters<sph_parameter_tangent>(parameter_tangent);
        pbf_particle_state_tangent nt = particles(next_state_tangent);
        sph_method_state nmt = detail::method_state(next_state_tangent.method);
        detail::check(sph_jvp_step(handle_, &s, &sm, &c, &p, &n, cache.handle(), &st, &smt, &ct, &pt, &nt, &nmt));
    }
    void vjp_step(const State& state, const Control& control, const Parameters& parameters, const State& next_state,
                  const StepCache& cache, const StateAdjoint& next_state_adjoint, StateAdjoint& previous_state_adjoint,
                  ControlAdjoint& control_adjoint, ParameterAdjoint& parameter_adjoint) {
        const pbf_particle_state s = particles(state), n = particles(next_state);
        const sph_method_state sm = detail::method_state(state.method);
        const pbf_control c{detail::view(control.external_accelerations)};
        const sph_parameters p = c_parameters<sph_parameters>(parameters);
        const pbf_particle_state_adjoint na = particles(next_state_adjoint);
        const sph_method_state_adjoint nma = detail::method_adjoint(next_state_adjoint.method);
        pbf_particle_state_adjoint pa = particles(previous_state_adjoint);
        sph_method_state_adjoint pma = detail::method_adjoint(previous_state_adjoint.method);
        pbf_control_adjoint ca{detail::view(control_adjoint.external_accelerations)};
        sph_parameter_adjoint qa = c_parameters<sph_parameter_adjoint>(parameter_adjoint);
        detail::check(sph_vjp_step(handle_, &s, &sm, &c, &p, &n, cache.handle(), &na, &nma, &pa, &pma, &ca, &qa));
    }

    // Not in the reference's interface: the C ABI handle, the stream, and a wait for queued work.
    sph_solver* handle() const { return handle_; }
    cudaStream_t stream() const { return stream_; }
    void synchronize() const { detail::check(sph_synchronize(handle_)); }

private:
    template <class P>
    P particle_parameters() const {
        return {{count_, stream_}, {count_, stream_}, {count_, stream_}, {count_, stream_}};
    }
    static pbf_particle_state particles(const State& s) {
        return {detail::view(s.particles.positions), detail::view(s.particles.velocities), s.particles.step_index};
    }
    static pbf_particle_state_tangent particles(const StateTangent& s) {
        return {detail::view(s.particles.positions), detail::view(s.particles.velocities)};
    }
    static pbf_particle_state_adjoint particles(const StateAdjoint& s) {
        return {detail::view(s.particles.positions), detail::view(s.particles.velocities)};
    }
    // sph_parameters / sph_parameter_adjoint from SPH<Method>::Parameters / ParameterTangent / ParameterAdjoint:
    // the particle arrays, this method's arrays, null for the other methods'.
    template <class C, class P>
    static C c_parameters(const P& p) {
        C c{};
        using Pointer = decltype(c.masses);
        c.masses = const_cast<Pointer>(p.particles.masses.data());
        c.rest_densities = const_cast<Pointer>(p.particles.rest_densities.data());
        c.viscosities = const_cast<Pointer>(p.particles.viscosities.data());
        c.surface_tensions = const_cast<Pointer>(p.particles.surface_tensions.data());
        Method::bind(c, p.method);
        return c;
    }

    std::size_t count_;
    cudaStream_t stream_;
    sph_solver* handle_ = nullptr;
};

}  // namespace physica::fluids::liquid::particle

#endif  // PHYSICA_SPH_HPP
