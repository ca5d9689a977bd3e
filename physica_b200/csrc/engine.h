// Host-side engine of the PBF substep: device buffers, the scene table and the launch
// sequence of one forward / reverse substep.  One scene is a pbf_solver; many scenes
// advancing together are a pbf_batch.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/physica_pbf.h"
#include "pbf_internal.h"
#include "pbf_launch.h"

namespace pbf {

void set_error(const std::string& message);

// Stream-ordered device allocations released together.
class DeviceArena {
public:
    explicit DeviceArena(cudaStream_t stream = nullptr) : stream_(stream) {}
    DeviceArena(const DeviceArena&) = delete;
    DeviceArena& operator=(const DeviceArena&) = delete;
    ~DeviceArena() { release(); }
    void set_stream(cudaStream_t s) { stream_ = s; }
    template <class T>
    T* alloc(size_t count, cudaError_t& err) {
        void* p = nullptr;
        if (err != cudaSuccess) return nullptr;
        const size_t bytes = count ? count * sizeof(T) : sizeof(T);
        err = cudaMallocAsync(&p, bytes, stream_);
        if (err == cudaSuccess) ptrs_.push_back(p);
        else cudaGetLastError();   // the status is reported by the caller; clear the runtime's last error
        return static_cast<T*>(p);
    }
    void release() {
        for (void* p : ptrs_) cudaFreeAsync(p, stream_);
        ptrs_.clear();
    }
    size_t size() const { return ptrs_.size(); }

private:
    cudaStream_t stream_;
    std::vector<void*> ptrs_;
};

// Three arrays of count + 4 floats or more, each 16-byte aligned, for the packed list scan.
inline PackedPositions alloc_packed(DeviceArena& arena, const uint32_t count, cudaError_t& err) {
    const size_t stride = (static_cast<size_t>(count) + 4u + 31u) / 32u * 32u;
    float* base = arena.alloc<float>(3 * stride + 4, err);
    if (!base) return PackedPositions{};
    base = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(base) + 15u) & ~uintptr_t{15});
    return PackedPositions{base, base + stride, base + 2 * stride};
}

struct SceneHost {
    pbf_domain_configuration config;     // boundary pointer cleared
    std::vector<pbf_boundary_particle> boundary;
    uint32_t dims[3];
    uint64_t cells;
    uint32_t cell_base;
    uint32_t first;
};

// Everything one forward substep leaves behind for export and for the reverse pass.
struct StepRecord {
    DeviceArena arena;
    bool valid = false;
    uint64_t step_index = 0;         // index of the input state
    uint32_t* cell_offsets = nullptr;
    uint32_t* sorted_index = nullptr;
    uint32_t* slot_of = nullptr;
    uint32_t* keys = nullptr;        // original order
    int4* cell = nullptr;
    float4* topology = nullptr;      // x* and mass (iterate 0)
    float4* params_a = nullptr;
    float4* params_b = nullptr;
    // Iterates 1..K.  Differentiable records keep all of them; forward-mode records pass them
    // through 2 ping-pong buffers.  A checkpoint-recompute record (differentiable, `recompute`)
    // keeps every checkpoint_interval-th iterate and the last one in `checkpoints`, as the
    // reference's StepCache::checkpoints (pbf/pbf.ixx:54-70, pbf/pbf.cpp:173-182), and passes the
    // others through the 2 ping-pong buffers.
    std::vector<float4*> positions;
    bool recompute = false;
    uint32_t checkpoint_interval = 1;
    std::vector<float4*> checkpoints;   // iterates c, 2c, ... below K, then K
    std::vector<float*> lambda;      // per iteration (forward mode and checkpoint-recompute: 1)
    std::vector<float*> density;     // per iteration (differentiable mode, all iterates kept)
    std::vector<float4*> gsum;       // per iteration (differentiable mode, all iterates kept)
    std::vector<uint8_t*> mask;      // per iteration (differentiable mode, both storage forms)
    float* first_density = nullptr;
    float* first_lambda = nullptr;
    uint32_t* neighbor_count = nullptr;
    float4* velocity = nullptr;
    float4* vorticity = nullptr;
    float4* normal = nullptr;
    float4* confined = nullptr;
    // Stored neighbour lists: one per iterate when all iterates are kept (0..K), else one reused
    // (it holds the post-loop list after the step).
    std::vector<uint32_t*> list_entries;
    std::vector<uint32_t*> list_counts;
    uint32_t list_capacity = 0;
    // Boundary particles of the step (only when the scenes have some).
    uint32_t* boundary_offsets = nullptr;   // cells + 1
    float4* boundary = nullptr;             // (position at the step's time, volume), cell-sorted

    // Whether every iterate and its per-iteration fields and list are kept.
    bool keeps_all(bool differentiable) const { return differentiable && !recompute; }
    bool is_checkpoint(uint32_t k, uint32_t K) const { return k == K || k % checkpoint_interval == 0; }
    const float4* iterate(uint32_t k, uint32_t K, bool differentiable) const {
        if (k == 0) return topology;
        if (recompute) {
            if (is_checkpoint(k, K)) return checkpoints[k == K ? (K - 1) / checkpoint_interval : k / checkpoint_interval - 1];
            return positions[(k - 1) & 1u];
        }
        if (differentiable) return positions[k - 1];
        return positions[(k - 1) & 1u];
    }
};

enum PassId : int {
    kPassGrid = 0,
    kPassListScan,
    kPassDensityLambda,
    kPassCorrection,
    kPassVorticity,
    kPassNormal,
    kPassXsph,
    kPassSeed,
    kPassXsphVjp,
    kPassNormalVjp,
    kPassVorticityVjp,
    kPassCorrectionVjp,
    kPassLambdaVjp,
    kPassDensityVjp,
    kPassTangentSeed,
    kPassDensityLambdaJvp,
    kPassCorrectionJvp,
    kPassVorticityJvp,
    kPassNormalJvp,
    kPassXsphJvp,
    kPassScanDensityLambda,
    kPassHostUpload,
    kPassHostDownload,
    kPassCount
};

const char* pass_name(int pass);

// CUDA-event timing of kernel groups on the engine's stream.
class PassTimer {
public:
    ~PassTimer();
    void enable(bool on);
    bool enabled() const { return enabled_; }
    void begin(cudaStream_t stream, int pass);
    void end(cudaStream_t stream, int pass);
    int collect(cudaStream_t stream);   // synchronises; folds pending intervals into the totals
    double milliseconds(int pass) const { return ms_[pass]; }
    uint64_t launches(int pass) const { return launches_[pass]; }

private:
    cudaEvent_t take();
    struct Mark { int pass; cudaEvent_t start, end; };
    bool enabled_ = false;
    std::vector<Mark> pending_;
    std::vector<cudaEvent_t> pool_;
    cudaEvent_t open_ = nullptr;
    double ms_[kPassCount] = {};
    uint64_t launches_[kPassCount] = {};
};

class Engine {
public:
    Engine() = default;
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;
    ~Engine();

    int init(const pbf_domain_configuration* scenes, uint32_t scene_count, const pbf_configuration* configuration,
             pbf_execution_mode mode, cudaStream_t stream);
    int allocate_record(StepRecord& r);
    int forward(const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                pbf_particle_state* next_state, StepRecord& record);
    // Forward-mode tangent of the substep recorded in `record` (jvp.cu).
    int tangent(const pbf_particle_state* state, const StepRecord& record, const pbf_particle_state_tangent* state_tangent,
                const pbf_control* control_tangent, const pbf_parameter_tangent* parameter_tangent,
                pbf_particle_state_tangent* next_state_tangent);
    int reverse(const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                const StepRecord& record, const pbf_particle_state_adjoint* next_adjoint,
                pbf_particle_state_adjoint* previous_adjoint, pbf_control_adjoint* control_adjoint,
                pbf_parameter_adjoint* parameter_adjoint);
    int read(const StepRecord& record, pbf_cache_field field, void* destination, size_t bytes);
    int read_iteration(const StepRecord& record, pbf_iteration_field field, uint32_t iteration, void* destination,
                       size_t bytes);

    uint32_t count() const { return count_; }
    uint64_t cells() const { return cells_; }
    uint32_t iterations() const { return iterations_; }
    bool differentiable() const { return mode_ == PBF_EXECUTION_DIFFERENTIABLE; }
    cudaStream_t stream() const { return stream_; }
    const std::vector<SceneHost>& scenes() const { return scenes_; }
    // Launch shape of the list and gather kernels (bit-identical results for every shape).
    void set_shape(const LaunchShape& shape) {
        shape_ = shape;
        drop_graphs();
    }
    const LaunchShape& shape() const { return shape_; }
    // Optional device-side input checks (PBF_INPUT_* bits accumulated until read).
    void set_input_checks(bool on) {
        input_checks_ = on;
        drop_graphs();
    }
    int read_input_checks(uint32_t* flags);
    // Checkpoint recomputation (differentiable mode): step caches allocated while it is on keep only
    // every checkpoint_interval-th Jacobi iterate, and the adjoint and tangent recompute the rest.
    void set_recompute(bool on) { recompute_ = on; }
    bool recompute() const { return recompute_; }
    // Times every candidate shape on `repeats` forward steps from `state` (writing `next_state` and
    // the record) and keeps the fastest; returns its per-step milliseconds in `best_ms`.
    int autotune(const pbf_particle_state* state, const pbf_control* control, const pbf_parameters* parameters,
                 pbf_particle_state* next_state, StepRecord& record, uint32_t repeats, float* best_ms);

    int check(cudaError_t e, const char* what);
    PassTimer& timer() { return timer_; }
    // Replay the forward launch sequence as a CUDA graph, captured once per buffer set.
    void set_graphs(bool on) { graphs_ = on; }
    bool graphs() const { return graphs_; }
    // Optional event recorded on the step's stream as soon as next_state.positions are final (after
    // the last correction, before the post-loop passes), so that a caller can start reading them
    // while vorticity, confinement and XSPH run.  Null: no event.  Part of the graph key.
    void set_positions_ready_event(cudaEvent_t event) { positions_ready_ = event; }
    void forget(const StepRecord* record);

private:
    struct GraphKey {
        const void* p[16];
        const StepRecord* record;
        cudaEvent_t positions_ready;
        bool operator==(const GraphKey& o) const;
    };
    struct GraphEntry {
        GraphKey key;
        cudaGraphExec_t exec;
        const void* extra[7];   // the remaining parameter / next-state pointers
        unsigned launches;      // kernels in the captured sequence
    };
    int launch_forward(cudaStream_t s, const pbf_particle_state* state, const pbf_control* control,
                       const pbf_parameters* parameters, pbf_particle_state* next_state, StepRecord& record);
    void drop_graphs();
    // Instantiated forward graphs kept per solver (one per buffer set; least recently used dropped).
    static constexpr size_t kGraphCacheEntries = 32;

    PassTimer timer_;
    bool graphs_ = false;
    cudaEvent_t positions_ready_ = nullptr;
    cudaStream_t capture_stream_ = nullptr;
    std::vector<GraphEntry> graph_cache_;
    SceneStatic* d_static_ = nullptr;
    uint32_t* export_offsets_ = nullptr;   // reference-layout cell offsets for exports (allocated on first use)
    // Boundary particles of all scenes, concatenated in scene order (original order).
    uint32_t boundary_count_ = 0;
    float4* boundary_rest_ = nullptr;       // (position at t = 0, volume)
    float4* boundary_velocity_ = nullptr;
    uint32_t* boundary_scene_ = nullptr;    // boundary particle -> scene (several scenes only)
    uint32_t* boundary_keys_ = nullptr;
    uint32_t* boundary_arrival_ = nullptr;
    uint32_t* boundary_unordered_ = nullptr;
    // The gather inputs shared by every pass of a step recorded in `r`.
    GatherCommon gather_common(const StepRecord& r) const;
    unsigned long long* d_step_ = nullptr;
    uint64_t host_step_ = ~0ull;   // step index the device counter holds

    uint32_t count_ = 0;
    uint64_t cells_ = 0;
    uint32_t iterations_ = 0;
    uint32_t checkpoint_interval_ = 1;
    pbf_execution_mode mode_ = PBF_EXECUTION_FORWARD;
    cudaStream_t stream_ = nullptr;
    LaunchShape shape_{};
    bool input_checks_ = false;
    uint32_t* d_input_flags_ = nullptr;
    std::vector<SceneHost> scenes_;
    std::vector<SceneDesc> scene_table_;
    DeviceArena arena_;
    SceneDesc* d_scenes_ = nullptr;
    KernelConstants* d_constants_ = nullptr;
    uint32_t* d_scene_of_ = nullptr;
    // grid-build scratch
    float4* predicted_ = nullptr;
    // The current iterate as three arrays in sorted order (x, y, z), written by the grid build and
    // every correction, read by the per-lane list scan.
    PackedPositions packed_{};
    uint32_t* arrival_ = nullptr;
    uint32_t* unordered_ = nullptr;
    uint32_t* tile_sums_ = nullptr;
    friend struct AdjointWorkspace;
    void* adjoint_ = nullptr;  // AdjointWorkspace*, differentiable mode
    void* tangent_ = nullptr;  // TangentWorkspace*, differentiable mode
    bool recompute_ = false;
    // One segment of recomputed Jacobi iterations (checkpoint-recompute records): its iterates, their
    // per-iteration fields and lists, allocated on first use (pbf/pbf.ixx:107-110).
    struct Segment {
        DeviceArena arena;
        uint32_t length = 0;                 // iterations per segment: min(checkpoint interval, K)
        std::vector<float4*> positions;      // local iterates 1.. (at least 2, the tangent's ping-pong)
        std::vector<float*> lambda, density;
        std::vector<float4*> gsum;
        std::vector<uint32_t*> list_entries, list_counts;
    };
    Segment* segment_ = nullptr;
    int segment_workspace(Segment** out);
    // Recomputes iterations first .. first + length - 1 of the step in `r` into the segment
    // workspace: their lists, densities, gradient sums, denominators and lambdas, and the iterates
    // first + 1 .. first + length - 1 (the last iterate of a segment is a stored checkpoint).
    int recompute_segment(const StepRecord& r, uint32_t first, uint32_t length);
    // Iterate first + j of the segment being recomputed.
    const float4* segment_iterate(const StepRecord& r, uint32_t first, uint32_t j) const {
        return j == 0 ? r.iterate(first, iterations_, true) : segment_->positions[j - 1];
    }
};

int read_profile(Engine& engine, pbf_pass_time* passes, uint32_t capacity, uint32_t* count);

}  // namespace pbf
