// Drives the SPH solvers through the C++ front end (include/physica_sph.hpp) the way a caller of the
// reference's SPH<Method> does: allocate_* buffers, forward_step rollouts, then one jvp_step and one
// vjp_step of the last substep.  tests/test_cpp_front_end.py writes the scene, runs this program and
// compares its outputs with the same calls made through the Python binding.
//
// Input (binary, little endian): u32 method (0 WCSPH, 1 PCISPH, 2 IISPH, 3 DFSPH), particle_count,
// steps, pressure_iterations, divergence_iterations, density_iterations; f32 time_step,
// support_radius, particle_radius, gravity[3], box minimum[3], maximum[3], velocity[3]; u32 no_slip;
// f32 positions x[n] y[n] z[n], velocities x[n] y[n] z[n]; the eleven parameter arrays of n floats
// (masses, rest_densities, viscosities, surface_tensions, speed_of_sound, tait_exponent,
// boundary_surface_tension, pressure_relaxation, jacobi_relaxation, divergence_relaxation,
// density_relaxation); DFSPH's warm divergence and density pressures (n floats each).
// Output: f32 positions[3n], velocities[3n] after `steps` substeps; f32 next-state position tangent
// [3n] of the last substep for a unit position tangent; f64 previous-state position and velocity
// adjoints [6n] and the mass adjoint [n] for a unit next-position adjoint.
#include <cstdio>
#include <exception>
#include <vector>

#include "physica_sph.hpp"

namespace pp = physica::fluids::liquid::particle;

namespace {

struct Input {
    std::uint32_t method, n, steps, pressure_iterations, divergence_iterations, density_iterations;
    pp::DomainConfiguration domain;
    std::vector<std::vector<float>> fields;   // 6 state arrays, 11 parameter arrays, 2 warm starts
};

template <class T>
T read_one(std::FILE* f) {
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::runtime_error("short input");
    return v;
}

Input read_input(const char* path) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error("cannot open input");
    Input in{};
    in.method = read_one<std::uint32_t>(f);
    in.n = read_one<std::uint32_t>(f);
    in.steps = read_one<std::uint32_t>(f);
    in.pressure_iterations = read_one<std::uint32_t>(f);
    in.divergence_iterations = read_one<std::uint32_t>(f);
    in.density_iterations = read_one<std::uint32_t>(f);
    pp::DomainConfiguration& d = in.domain;
    d.particle_count = in.n;
    d.time_step = read_one<float>(f);
    d.support_radius = read_one<float>(f);
    d.particle_radius = read_one<float>(f);
    auto vec = [&] {
        pp::Vector3 v;
        v.x = read_one<float>(f);
        v.y = read_one<float>(f);
        v.z = read_one<float>(f);
        return v;
    };
    d.gravity = vec();
    d.boundary.minimum = vec();
    d.boundary.maximum = vec();
    d.boundary.velocity = vec();
    d.boundary.no_slip = read_one<std::uint32_t>(f) != 0u;
    for (int k = 0; k < 6 + 11 + 2; ++k) {
        std::vector<float> v(in.n);
        if (in.n && std::fread(v.data(), sizeof(float), in.n, f) != in.n) throw std::runtime_error("short input");
        in.fields.push_back(std::move(v));
    }
    std::fclose(f);
    return in;
}

void write(std::FILE* f, const std::vector<float>& v) { std::fwrite(v.data(), sizeof(float), v.size(), f); }
void write(std::FILE* f, const std::vector<double>& v) { std::fwrite(v.data(), sizeof(double), v.size(), f); }

template <class Field>
void write_field(std::FILE* f, const Field& v, cudaStream_t s) {
    write(f, pp::download(v.x, s));
    write(f, pp::download(v.y, s));
    write(f, pp::download(v.z, s));
}

void fill(pp::device_buffer<double>& b, const double value, cudaStream_t s) {
    std::vector<double> h(b.size(), value);
    pp::detail::check_cuda(cudaMemcpyAsync(b.data(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s), "fill");
    pp::detail::check_cuda(cudaStreamSynchronize(s), "fill");
}

void fill(pp::device_buffer<float>& b, const float value, cudaStream_t s) {
    pp::upload(std::vector<float>(b.size(), value), b, s);
    pp::detail::check_cuda(cudaStreamSynchronize(s), "fill");
}

// The method's own parameter arrays, by position in the input's eleven.
void upload_method(const Input& in, pp::WCSPH::Parameters& p, cudaStream_t s) {
    pp::upload(in.fields[6 + 4], p.speed_of_sound, s);
    pp::upload(in.fields[6 + 5], p.tait_exponent, s);
    pp::upload(in.fields[6 + 6], p.boundary_surface_tension, s);
}
void upload_method(const Input& in, pp::PCISPH::Parameters& p, cudaStream_t s) { pp::upload(in.fields[6 + 7], p.pressure_relaxation, s); }
void upload_method(const Input& in, pp::IISPH::Parameters& p, cudaStream_t s) { pp::upload(in.fields[6 + 8], p.jacobi_relaxation, s); }
void upload_method(const Input& in, pp::DFSPH::Parameters& p, cudaStream_t s) {
    pp::upload(in.fields[6 + 9], p.divergence_relaxation, s);
    pp::upload(in.fields[6 + 10], p.density_relaxation, s);
}

template <class Method>
typename Method::Configuration configuration(const Input& in) {
    typename Method::Configuration c{};
    if constexpr (std::is_same_v<Method, pp::PCISPH> || std::is_same_v<Method, pp::IISPH>) c.pressure_iterations = in.pressure_iterations;
    if constexpr (std::is_same_v<Method, pp::DFSPH>) {
        c.divergence_iterations = in.divergence_iterations;
        c.density_iterations = in.density_iterations;
    }
    return c;
}

template <class Method>
void run(const Input& in, const char* output, cudaStream_t stream) {
    using Solver = pp::SPH<Method>;
    Solver solver(in.domain, configuration<Method>(in), pp::ExecutionMode::differentiable, stream);
    typename Solver::State current = solver.allocate_state(), next = solver.allocate_state();
    pp::upload(in.fields[0], current.particles.positions.x, stream);
    pp::upload(in.fields[1], current.particles.positions.y, stream);
    pp::upload(in.fields[2], current.particles.positions.z, stream);
    pp::upload(in.fields[3], current.particles.velocities.x, stream);
    pp::upload(in.fields[4], current.particles.velocities.y, stream);
    pp::upload(in.fields[5], current.particles.velocities.z, stream);
    if constexpr (std::is_same_v<Method, pp::DFSPH>) {
        pp::upload(in.fields[17], current.method.warm_divergence_pressure.values, stream);
        pp::upload(in.fields[18], current.method.warm_density_pressure.values, stream);
    }
    const pp::Control control = solver.allocate_control();
    typename Solver::Parameters parameters = solver.allocate_parameters();
    pp::upload(in.fields[6], parameters.particles.masses, stream);
    pp::upload(in.fields[7], parameters.particles.rest_densities, stream);
    pp::upload(in.fields[8], parameters.particles.viscosities, stream);
    pp::upload(in.fields[9], parameters.particles.surface_tensions, stream);
    upload_method(in, parameters.method, stream);
    pp::detail::check_cuda(cudaStreamSynchronize(stream), "upload");

    typename Solver::StepCache cache = solver.allocate_step_cache();
    for (std::uint32_t k = 0; k + 1 < in.steps; ++k) {
        solver.forward_step(current, control, parameters, next, cache);
        std::swap(current, next);
    }
    typename Solver::State last = solver.allocate_state();
    solver.copy_state(current, last);
    solver.forward_step(last, control, parameters, next, cache);
    if (next.particles.step_index != in.steps) throw std::runtime_error("step index");

    typename Solver::StateTangent tangent = solver.allocate_state_tangent(), copied = solver.allocate_state_tangent();
    typename Solver::StateTangent next_tangent = solver.allocate_state_tangent();
    fill(tangent.particles.positions.x, 1.0F, stream);
    fill(tangent.particles.positions.y, 1.0F, stream);
    fill(tangent.particles.positions.z, 1.0F, stream);
    solver.copy_state_tangent(tangent, copied);
    solver.jvp_step(last, control, parameters, next, cache, copied, solver.allocate_control_tangent(),
                    solver.allocate_parameter_tangent(), next_tangent);

    typename Solver::StateAdjoint next_adjoint = solver.allocate_state_adjoint(), previous = solver.allocate_state_adjoint();
    fill(next_adjoint.particles.positions.x, 1.0, stream);
    fill(next_adjoint.particles.positions.y, 1.0, stream);
    fill(next_adjoint.particles.positions.z, 1.0, stream);
    pp::ControlAdjoint control_adjoint = solver.allocate_control_adjoint();
    typename Solver::ParameterAdjoint parameter_adjoint = solver.allocate_parameter_adjoint();
    solver.vjp_step(last, control, parameters, next, cache, next_adjoint, previous, control_adjoint, parameter_adjoint);
    solver.synchronize();

    std::FILE* out = std::fopen(output, "wb");
    if (!out) throw std::runtime_error("cannot open output");
    write_field(out, next.particles.positions, stream);
    write_field(out, next.particles.velocities, stream);
    write_field(out, next_tangent.particles.positions, stream);
    write_field(out, previous.particles.positions, stream);
    write_field(out, previous.particles.velocities, stream);
    write(out, pp::download(parameter_adjoint.particles.masses, stream));
    std::fclose(out);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    try {
        const Input in = read_input(argv[1]);
        cudaStream_t stream = nullptr;
        pp::detail::check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        switch (in.method) {
            case 0: run<pp::WCSPH>(in, argv[2], stream); break;
            case 1: run<pp::PCISPH>(in, argv[2], stream); break;
            case 2: run<pp::IISPH>(in, argv[2], stream); break;
            case 3: run<pp::DFSPH>(in, argv[2], stream); break;
            default: throw std::runtime_error("unknown method");
        }
        cudaStreamDestroy(stream);
        return 0;
    } catch (const pp::Error& e) {
        std::fprintf(stderr, "solver error (status %d): %s\n", e.status, e.what());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
    }
    return 1;
}
