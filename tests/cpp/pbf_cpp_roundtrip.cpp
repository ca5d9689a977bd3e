// Drives the solver through the C++ front end (include/physica_pbf.hpp) the way a caller of the
// reference's PBF class does: allocate_* buffers, forward_step rollouts, then one jvp_step and one
// vjp_step of the last substep.  tests/test_cpp_front_end.py writes the scene, runs this program and
// compares its outputs with the same calls made through the Python binding.
//
// Input (binary, little endian): u32 particle_count, u32 pressure_iterations, u32 steps,
// f32 time_step, support_radius, particle_radius, gravity[3], box minimum[3], maximum[3],
// velocity[3], u32 no_slip; then f32 positions x[n] y[n] z[n], velocities x[n] y[n] z[n], and the
// ten PBF parameter arrays of n floats (masses, rest_densities, viscosities, surface_tensions,
// relaxation, s_corr strength, exponent, radius, xsph_viscosity, vorticity_confinement).
// Output: f32 positions[3n], velocities[3n] after `steps` substeps; f32 next-state position
// tangent[3n] of the last substep for a unit position tangent; f64 previous-state position and
// velocity adjoints[6n] and the mass adjoint[n] for a unit next-position adjoint.
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "physica_pbf.hpp"

namespace pp = physica::fluids::liquid::particle;

namespace {

template <class T>
T read_one(std::FILE* f) {
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::runtime_error("short input");
    return v;
}

std::vector<float> read_floats(std::FILE* f, const std::size_t n) {
    std::vector<float> v(n);
    if (n && std::fread(v.data(), sizeof(float), n, f) != n) throw std::runtime_error("short input");
    return v;
}

void write(std::FILE* f, const std::vector<float>& v) { std::fwrite(v.data(), sizeof(float), v.size(), f); }
void write(std::FILE* f, const std::vector<double>& v) { std::fwrite(v.data(), sizeof(double), v.size(), f); }

void write_field(std::FILE* f, const pp::VectorField& v, cudaStream_t s) {
    write(f, pp::download(v.x, s));
    write(f, pp::download(v.y, s));
    write(f, pp::download(v.z, s));
}

void write_field(std::FILE* f, const pp::VectorAdjointField& v, cudaStream_t s) {
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

int run(const char* input, const char* output) {
    std::FILE* in = std::fopen(input, "rb");
    if (!in) throw std::runtime_error("cannot open input");
    const auto n = read_one<std::uint32_t>(in);
    const auto iterations = read_one<std::uint32_t>(in);
    const auto steps = read_one<std::uint32_t>(in);
    const bool recompute = read_one<std::uint32_t>(in) != 0u;   // keep checkpoints only (interval 2)
    pp::DomainConfiguration domain{};
    domain.particle_count = n;
    domain.time_step = read_one<float>(in);
    domain.support_radius = read_one<float>(in);
    domain.particle_radius = read_one<float>(in);
    auto vec = [&] { pp::Vector3 v; v.x = read_one<float>(in); v.y = read_one<float>(in); v.z = read_one<float>(in); return v; };
    domain.gravity = vec();
    domain.boundary.minimum = vec();
    domain.boundary.maximum = vec();
    domain.boundary.velocity = vec();
    domain.boundary.no_slip = read_one<std::uint32_t>(in) != 0u;
    std::vector<std::vector<float>> fields;
    for (int k = 0; k < 6 + 10; ++k) fields.push_back(read_floats(in, n));
    std::fclose(in);

    cudaStream_t stream = nullptr;
    pp::detail::check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    {
        pp::PBF::Configuration configuration;
        configuration.pressure_iterations = iterations;
        configuration.checkpoint_interval = 2u;
        pp::PBF solver(domain, configuration, pp::ExecutionMode::differentiable, stream);
        solver.set_checkpoint_recompute(recompute);
        pp::PBF::State current = solver.allocate_state(), next = solver.allocate_state();
        pp::upload(fields[0], current.particles.positions.x, stream);
        pp::upload(fields[1], current.particles.positions.y, stream);
        pp::upload(fields[2], current.particles.positions.z, stream);
        pp::upload(fields[3], current.particles.velocities.x, stream);
        pp::upload(fields[4], current.particles.velocities.y, stream);
        pp::upload(fields[5], current.particles.velocities.z, stream);
        const pp::Control control = solver.allocate_control();
        pp::PBF::Parameters parameters = solver.allocate_parameters();
        pp::device_buffer<float>* slots[10] = {&parameters.particles.masses, &parameters.particles.rest_densities,
                                               &parameters.particles.viscosities, &parameters.particles.surface_tensions,
                                               &parameters.relaxation, &parameters.artificial_pressure_strength,
                                               &parameters.artificial_pressure_exponent, &parameters.artificial_pressure_radius,
                                               &parameters.xsph_viscosity, &parameters.vorticity_confinement};
        for (int k = 0; k < 10; ++k) pp::upload(fields[6 + k], *slots[k], stream);
        pp::detail::check_cuda(cudaStreamSynchronize(stream), "upload");

        pp::PBF::StepCache cache = solver.allocate_step_cache();
        for (std::uint32_t k = 0; k + 1 < steps; ++k) {
            solver.forward_step(current, control, parameters, next, cache);
            std::swap(current, next);
        }
        // the last substep keeps its cache for the tangent and the adjoint
        pp::PBF::State last = solver.allocate_state();
        solver.copy_state(current, last);
        solver.forward_step(last, control, parameters, next, cache);
        if (next.particles.step_index != steps) throw std::runtime_error("step index");

        pp::PBF::StateTangent tangent = solver.allocate_state_tangent(), copied = solver.allocate_state_tangent();
        pp::PBF::StateTangent next_tangent = solver.allocate_state_tangent();
        fill(tangent.particles.positions.x, 1.0F, stream);
        fill(tangent.particles.positions.y, 1.0F, stream);
        fill(tangent.particles.positions.z, 1.0F, stream);
        solver.copy_state_tangent(tangent, copied);
        solver.jvp_step(last, control, parameters, next, cache, copied, solver.allocate_control_tangent(),
                        solver.allocate_parameter_tangent(), next_tangent);

        pp::PBF::StateAdjoint next_adjoint = solver.allocate_state_adjoint(), previous = solver.allocate_state_adjoint();
        fill(next_adjoint.particles.positions.x, 1.0, stream);
        fill(next_adjoint.particles.positions.y, 1.0, stream);
        fill(next_adjoint.particles.positions.z, 1.0, stream);
        pp::ControlAdjoint control_adjoint = solver.allocate_control_adjoint();
        pp::PBF::ParameterAdjoint parameter_adjoint = solver.allocate_parameter_adjoint();
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
    cudaStreamDestroy(stream);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    try {
        return run(argv[1], argv[2]);
    } catch (const pp::Error& e) {
        std::fprintf(stderr, "solver error (status %d): %s\n", e.status, e.what());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
    }
    return 1;
}
