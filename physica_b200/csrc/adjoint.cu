// Reverse-mode substep (PBF::vjp_step, pbf/pbf.cpp:217-258) over cell-sorted particles.
#include "engine.h"

namespace pbf {

namespace {

__global__ void accumulate_kernel(const size_t count, const double* const* __restrict__ src, double* const* __restrict__ dst,
                                  const int fields) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    for (int f = 0; f < fields; ++f) dst[f][i] += src[f][i];
}

struct PointerBlock {
    const double* src[6];
    double* dst[6];
};

__global__ void accumulate6_kernel(const size_t count, const PointerBlock p, const int fields) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    for (int f = 0; f < fields; ++f) p.dst[f][i] += p.src[f][i];
}

}  // namespace

// domain/domain.cu:8-29: FP64 dst += src over up to six fields.
cudaError_t launch_accumulate(cudaStream_t stream, const size_t count, const double* const* src, double* const* dst,
                              const int fields) {
    if (count == 0) return cudaSuccess;
    PointerBlock p{};
    for (int f = 0; f < fields && f < 6; ++f) {
        p.src[f] = src[f];
        p.dst[f] = dst[f];
    }
    accumulate6_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(count, p, fields < 6 ? fields : 6);
    count_launch();
    (void)accumulate_kernel;
    return cudaGetLastError();
}

void destroy_adjoint_workspace(void* workspace) { (void)workspace; }

int Engine::reverse(const pbf_particle_state*, const pbf_control*, const pbf_parameters*, const StepRecord&,
                    const pbf_particle_state_adjoint*, pbf_particle_state_adjoint*, pbf_control_adjoint*,
                    pbf_parameter_adjoint*) {
    set_error("vjp_step is not available in this build yet");
    return PBF_ERROR_UNSUPPORTED;
}

}  // namespace pbf
