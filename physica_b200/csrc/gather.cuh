// Ordered neighbour gathers shared by the forward and adjoint kernels.
//
// A warp owns 32 consecutive cell-sorted particles (lane = particle).  Their neighbour
// candidates are the particles of the 27 stencil cells of each particle's home cell, in the
// reference order: stencil cells x offset outer, z offset inner (pbf/pbf.cu:105-110), and
// within a cell ascending original index, which is the sorted order.
//
// Scan (build a list): consecutive lanes that share a home cell form a run; for each run the
// warp lays the run's 27 cell ranges end to end and walks them 32 candidates at a time, one
// candidate per lane.  Every home particle of the run tests all 32 candidates against its own
// position (a broadcast from shared memory); a ballot and a prefix popcount append the hits to
// that particle's list in candidate order.  A candidate is loaded once per run instead of once
// per home particle, and no lane diverges while walking the stencil.
//
// Process: each lane then drains its own list in order with the pass's per-pair arithmetic, so
// per-particle sums accumulate in exactly the reference's order.  Candidates left out of a list
// contribute an exact zero in the reference (their kernel terms vanish), so the sums are equal
// bit for bit.
//
// Reuse: a list can be written to device memory (warp-interleaved, so that every later read of
// entry k by the 32 lanes is one coalesced transaction) and consumed by later passes over the
// same positions without scanning again.  A particle whose list exceeds the stored capacity is
// marked as overflowed, and warps holding one fall back to scanning.
#pragma once

#include "pbf_internal.h"
#include "pbf_launch.h"

namespace pbf {
namespace gather_detail {

constexpr int kWarpsPerBlock = 4;
constexpr int kBlock = 32 * kWarpsPerBlock;
constexpr int kListCap = 64;                 // per-lane list held in shared memory between drains
constexpr int kListStride = kListCap + 1;    // padded row: conflict-free appends and drains
constexpr unsigned kFull = 0xffffffffu;

struct WarpScratch {
    uint32_t list[32 * kListStride];
    uint32_t first[32];
    uint32_t base[32];
    float4 home[32];
};

struct Particle {
    uint32_t s;
    bool active;
    int4 c;
    const SceneDesc* scene;
    KernelConstants k;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ Particle locate(const GatherCommon& g) {
    Particle p;
    p.s = blockIdx.x * blockDim.x + threadIdx.x;
    p.active = p.s < g.count;
    p.c = p.active ? g.cell[p.s] : make_int4(0, 0, 0, 0);
    p.scene = g.scenes + p.c.w;
    p.k = g.constants[p.scene->constants];
    return p;
}

// Where a scan's list goes for later passes.
struct ListWriter {
    uint32_t* entries;    // stored lists (null: do not store)
    uint32_t* counts;
    uint32_t capacity;
};

// Drain this lane's shared list in order.  `op.process(t)` returns whether the pair is kept
// in the stored list.
template <class Op>
__device__ __forceinline__ void drain(Op& op, WarpScratch& ws, int& n, const ListWriter& w, const uint32_t s, uint32_t& stored) {
    __syncwarp();
    const uint32_t lane = lane_id();
    const size_t row = (static_cast<size_t>(s >> 5) * w.capacity) * 32u + lane;
    for (int k = 0; k < n; ++k) {
        const uint32_t t = ws.list[lane * kListStride + k];
        op.process(t);
        if (w.entries) {
            if (stored < w.capacity) w.entries[row + static_cast<size_t>(stored) * 32u] = t;
            ++stored;
        }
    }
    __syncwarp();
    n = 0;
}

// Scan the stencils of the warp's particles and process every particle's candidates in
// reference order.  Candidates enter a list when their squared distance to the home particle is
// below `threshold` (the home particle itself too when kSelf).
template <bool kSelf, class Op>
__device__ void scan(Op& op, const Particle& p, const GatherCommon& g, const float4* __restrict__ pos,
                     const float threshold, WarpScratch& ws, const ListWriter& w) {
    const uint32_t lane = lane_id();
    const uint32_t warp_first = p.s - lane;
    const int nact = __popc(__ballot_sync(kFull, p.active));
    ws.home[lane] = p.active ? pos[p.s] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    const int px = __shfl_up_sync(kFull, p.c.x, 1), py = __shfl_up_sync(kFull, p.c.y, 1);
    const int pz = __shfl_up_sync(kFull, p.c.z, 1), pw = __shfl_up_sync(kFull, p.c.w, 1);
    const bool start = p.active && (lane == 0 || px != p.c.x || py != p.c.y || pz != p.c.z || pw != p.c.w);
    uint32_t starts = __ballot_sync(kFull, start);
    const unsigned lower = (1u << lane) - 1u;
    int n = 0;
    uint32_t stored = 0;
    __syncwarp();
    while (starts) {
        const int a = __ffs(starts) - 1;
        starts &= starts - 1u;
        const int b = starts ? __ffs(starts) - 1 : nact;
        const int hx = __shfl_sync(kFull, p.c.x, a), hy = __shfl_sync(kFull, p.c.y, a);
        const int hz = __shfl_sync(kFull, p.c.z, a), hw = __shfl_sync(kFull, p.c.w, a);
        const float thr = __shfl_sync(kFull, threshold, a);
        const Grid& grid = g.scenes[hw].grid;
        uint32_t first = 0, cnt = 0;
        if (lane < 27u) {
            const int x = hx + static_cast<int>(lane) / 9 - 1;
            const int y = hy + (static_cast<int>(lane) / 3) % 3 - 1;
            const int z = hz + static_cast<int>(lane) % 3 - 1;
            if (x >= 0 && y >= 0 && z >= 0 && x < static_cast<int>(grid.cells_x) && y < static_cast<int>(grid.cells_y) &&
                z < static_cast<int>(grid.cells_z)) {
                const uint32_t c = grid.cell_base +
                                   (static_cast<uint32_t>(z) * grid.cells_y + static_cast<uint32_t>(y)) * grid.cells_x +
                                   static_cast<uint32_t>(x);
                first = g.cell_offsets[c];
                cnt = g.cell_offsets[c + 1u] - first;
            }
        }
        uint32_t inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, inc, o);
            if (lane >= static_cast<uint32_t>(o)) inc += v;
        }
        const uint32_t total = __shfl_sync(kFull, inc, 31);
        __syncwarp();
        ws.first[lane] = first;
        ws.base[lane] = lane < 27u ? inc - cnt : total;
        __syncwarp();
        for (uint32_t u0 = 0; u0 < total; u0 += 32u) {
            if (__any_sync(kFull, n > kListCap - 32)) drain(op, ws, n, w, p.s, stored);
            const uint32_t u = u0 + lane;
            const bool valid = u < total;
            uint32_t o = 0;
#pragma unroll
            for (uint32_t step = 16; step > 0; step >>= 1)
                if (ws.base[o + step] <= u) o += step;
            const uint32_t t = ws.first[o] + (u - ws.base[o]);
            const float4 q = valid ? pos[t] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
            for (int h = a; h < b; ++h) {
                const float4 xh = ws.home[h];
                const float r2 = squared(mk(__fsub_rn(xh.x, q.x), __fsub_rn(xh.y, q.y), __fsub_rn(xh.z, q.z)));
                const bool in = valid && r2 < thr && (kSelf || t != warp_first + static_cast<uint32_t>(h));
                const unsigned m = __ballot_sync(kFull, in);
                if (m) {
                    const int nh = __shfl_sync(kFull, n, h);
                    if (in) ws.list[h * kListStride + nh + __popc(m & lower)] = t;
                    if (static_cast<int>(lane) == h) n += __popc(m);
                }
            }
        }
        __syncwarp();
    }
    drain(op, ws, n, w, p.s, stored);
    if (w.entries && p.active) w.counts[p.s] = stored <= w.capacity ? stored : 0xffffffffu;
}

// Process a list stored by an earlier scan over the same positions; warps holding an
// overflowed list scan instead.
template <bool kSelf, class Op>
__device__ void replay(Op& op, const Particle& p, const GatherCommon& g, const float4* __restrict__ pos,
                       const float threshold, WarpScratch& ws, const uint32_t* __restrict__ entries,
                       const uint32_t* __restrict__ counts, const uint32_t capacity) {
    const uint32_t n = p.active ? counts[p.s] : 0u;
    if (__any_sync(kFull, n == 0xffffffffu)) {
        scan<kSelf>(op, p, g, pos, threshold, ws, ListWriter{nullptr, nullptr, 0});
        return;
    }
    const uint32_t nmax = __reduce_max_sync(kFull, n);
    const size_t row = (static_cast<size_t>(p.s >> 5) * capacity) * 32u + lane_id();
    for (uint32_t k = 0; k < nmax; ++k) {
        if (k < n) op.process(entries[row + static_cast<size_t>(k) * 32u]);
    }
}

}  // namespace gather_detail
}  // namespace pbf
