// Ordered neighbour lists shared by the forward and adjoint kernels.
//
// Every per-particle sum of the reference runs over the particles of the 27 stencil cells of the
// particle's home cell in a fixed order: stencil cells x offset outer, z offset inner
// (pbf/pbf.cu:105-110), and within a cell ascending original index, which is the sorted order.
// Cells are sorted z fastest (cell_index), so the three cells of each (x, y) stencil column are
// one contiguous range of the sorted array and the stencil is nine ranges.
// Candidates whose squared distance is at or beyond the list threshold contribute exact zeros to
// every sum of every pass, so each particle only needs its in-support candidates, in that order.
//
// Scan, per lane (list_walk_kernel): each lane walks its own nine column ranges and appends its
// hits.  Scan, cooperative (list_scan_kernel): a warp owns 32 consecutive sorted particles.
// Lanes that share a home cell form a run; for each run the warp lays the run's nine column
// ranges end to end (an exclusive warp scan of their lengths) and walks them 32 candidates at a
// time, one candidate per lane, so a candidate is loaded once per run.  Each home particle of the run tests the 32 candidates against
// its position (a shared-memory broadcast); a ballot and a prefix popcount give every hit its slot
// in the home particle's list, written straight to device memory.  Lists are warp-interleaved:
// entry k of the warp's 32 particles is one 128-byte line, so a later read of entry k by the 32
// lanes is one coalesced transaction.  A list longer than the capacity is marked overflowed.
//
// Replay (replay): each lane drains its own list in order with a pass's per-pair arithmetic, the
// next entry's loads (and the index after it) issued before the current entry is processed.  An overflowed particle walks
// its stencil directly (same order, every candidate offered to the pass), which gives the same sums.
#pragma once

#include <type_traits>

#include "pbf_internal.h"
#include "pbf_launch.h"

namespace pbf {
namespace gather_detail {

constexpr int kWarpsPerBlock = 4;
constexpr int kBlock = 32 * kWarpsPerBlock;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kOverflow = 0xffffffffu;
// A list entry with this bit set is a boundary particle (slot in the cell-sorted boundary array).
constexpr uint32_t kBoundaryBit = 0x80000000u;

// Passes with boundary terms (density, lambda, correction and their derivatives) declare
// `static constexpr bool kBoundary = true`; their overflow walk then visits each cell's boundary
// particles after its fluid particles, as the reference's cell loops do (pbf/pbf.cu:111-121).
template <class T, class = void>
struct takes_boundary : std::false_type {};
template <class T>
struct takes_boundary<T, std::void_t<decltype(T::kBoundary)>> : std::integral_constant<bool, T::kBoundary> {};

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
    const uint32_t block = g.reverse ? gridDim.x - 1u - blockIdx.x : blockIdx.x;
    p.s = block * blockDim.x + threadIdx.x;
    p.active = p.s < g.count;
    p.c = p.active ? g.cell[p.s] : make_int4(0, 0, 0, 0);
    p.scene = g.scenes + p.c.w;
    p.k = g.constants[p.scene->constants];
    return p;
}

__device__ __forceinline__ size_t list_row(const uint32_t s, const uint32_t capacity) {
    return (static_cast<size_t>(s >> 5) * capacity) * 32u + (s & 31u);
}

// Order-preserving direct walk of one particle's stencil (overflow fallback).
template <class Op>
__device__ void walk(Op& op, const Particle& p, const GatherCommon& g) {
    const Grid& grid = p.scene->grid;
    if constexpr (takes_boundary<Op>::value) {
        if (g.boundary_offsets) {   // cell by cell: fluid particles, then boundary particles
            for (int o = 0; o < 27; ++o) {
                const int x = p.c.x + o / 9 - 1, y = p.c.y + (o / 3) % 3 - 1, z = p.c.z + o % 3 - 1;
                if (x < 0 || y < 0 || z < 0 || x >= static_cast<int>(grid.cells_x) || y >= static_cast<int>(grid.cells_y) ||
                    z >= static_cast<int>(grid.cells_z))
                    continue;
                const uint32_t c = cell_index(grid, x, y, z);
                const uint32_t end = g.cell_offsets[c + 1u];
                for (uint32_t t = g.cell_offsets[c]; t < end; ++t) op.process(t);
                const uint32_t bend = g.boundary_offsets[c + 1u];
                for (uint32_t b = g.boundary_offsets[c]; b < bend; ++b) op.process(b | kBoundaryBit);
            }
            return;
        }
    }
    const int cz = static_cast<int>(grid.cells_z);
    const uint32_t z_lo = static_cast<uint32_t>(p.c.z > 0 ? p.c.z - 1 : 0);
    const uint32_t z_hi = static_cast<uint32_t>(p.c.z + 1 < cz ? p.c.z + 1 : cz - 1);
    for (int o = 0; o < 9; ++o) {   // stencil columns, x-offset outer; cells z-1..z+1 are contiguous
        const int x = p.c.x + o / 3 - 1, y = p.c.y + o % 3 - 1;
        if (x < 0 || y < 0 || x >= static_cast<int>(grid.cells_x) || y >= static_cast<int>(grid.cells_y)) continue;
        const uint32_t end = g.cell_offsets[cell_index(grid, x, y, z_hi) + 1u];
        for (uint32_t t = g.cell_offsets[cell_index(grid, x, y, z_lo)]; t < end; ++t) op.process(t);
    }
}

// Drain this lane's stored list in order.  Op::prefetch(t) starts the loads of entry t and
// returns them; Op::apply(t, data) consumes them.  IndexLead: how many list indices ahead of the
// applied entry are loaded (1 or 2).
template <int IndexLead = 1, class Op>
__device__ __forceinline__ void replay(Op& op, const Particle& p, const GatherCommon& g, const StoredList& list) {
    if (!p.active) return;
    const uint32_t n = list.counts[p.s];
    if (n == kOverflow) {
        walk(op, p, g);
        return;
    }
    const uint32_t* __restrict__ entries = list.entries + list_row(p.s, list.capacity);
    if (n == 0) return;
    if constexpr (IndexLead >= 2) {
        // Pipeline: the indices of entries k+1 and k+2 and the data of entry k are in flight while
        // entry k-1 is applied.  The indices come from the stored list, which a replay after another
        // pass reads from DRAM; two entries of lead cover that latency.
        uint32_t t = entries[0];
        uint32_t tn = n > 1u ? entries[32] : 0u;
        uint32_t tnn = n > 2u ? entries[64] : 0u;
        auto data = op.prefetch(t);
        for (uint32_t k = 1; k < n; ++k) {
            const uint32_t t3 = k + 2u < n ? entries[static_cast<size_t>(k + 2u) * 32u] : 0u;
            const auto next = op.prefetch(tn);
            op.apply(t, data);
            t = tn;
            tn = tnn;
            tnn = t3;
            data = next;
        }
        op.apply(t, data);
    } else {
        // Two-stage pipeline: the index of entry k+1 and the data of entry k are in flight while
        // entry k-1 is applied.
        uint32_t t = entries[0];
        uint32_t tn = n > 1u ? entries[32] : 0u;
        auto data = op.prefetch(t);
        for (uint32_t k = 1; k < n; ++k) {
            const uint32_t tnn = k + 1u < n ? entries[static_cast<size_t>(k + 1u) * 32u] : 0u;
            const auto next = op.prefetch(tn);
            op.apply(t, data);
            t = tn;
            tn = tnn;
            data = next;
        }
        op.apply(t, data);
    }
}

// Two lanes per particle (the FP64 reverse passes, whose sums carry a tolerance rather than the
// forward's bit-exact order).  Threads 2q and 2q + 1 of the grid share particle q; lane `half` (0 or
// 1) takes the list entries half, half + 2, ... (or every other candidate of the stencil walk), and
// pair_sum() then adds the two partial sums, giving both lanes the same total.  A particle's
// result depends only on its own list, never on which particles share its warp.
__device__ __forceinline__ Particle locate_pair(const GatherCommon& g, uint32_t& half) {
    Particle p;
    const uint32_t block = g.reverse ? gridDim.x - 1u - blockIdx.x : blockIdx.x;
    const uint32_t thread = block * blockDim.x + threadIdx.x;
    half = thread & 1u;
    p.s = thread >> 1;
    p.active = p.s < g.count;
    p.c = p.active ? g.cell[p.s] : make_int4(0, 0, 0, 0);
    p.scene = g.scenes + p.c.w;
    p.k = g.constants[p.scene->constants];
    return p;
}

// walk() with the candidates dealt alternately to the two lanes of a particle.
template <class Op>
struct Alternate {
    static constexpr bool kBoundary = takes_boundary<Op>::value;
    Op& op;
    uint32_t turn;
    __device__ __forceinline__ void process(const uint32_t t) {
        if ((turn & 1u) == 0u) op.process(t);
        ++turn;
    }
};

template <class Op>
__device__ void walk_pair(Op& op, const Particle& p, const GatherCommon& g, const uint32_t half) {
    Alternate<Op> alternate{op, half};
    walk(alternate, p, g);
}

// replay() over this lane's half of the list: entries half, half + 2, ...
template <class Op>
__device__ __forceinline__ void replay_pair(Op& op, const Particle& p, const GatherCommon& g, const StoredList& list,
                                            const uint32_t half) {
    if (!p.active) return;
    const uint32_t n = list.counts[p.s];
    if (n == kOverflow) {
        walk_pair(op, p, g, half);
        return;
    }
    if (half >= n) return;
    const uint32_t* __restrict__ entries = list.entries + list_row(p.s, list.capacity);
    uint32_t t = entries[static_cast<size_t>(half) * 32u];
    uint32_t k = half + 2u;
    uint32_t tn = k < n ? entries[static_cast<size_t>(k) * 32u] : 0u;
    auto data = op.prefetch(t);
    for (; k < n; k += 2u) {
        const uint32_t tnn = k + 2u < n ? entries[static_cast<size_t>(k + 2u) * 32u] : 0u;
        const auto next = op.prefetch(tn);
        op.apply(t, data);
        t = tn;
        tn = tnn;
        data = next;
    }
    op.apply(t, data);
}

// The sum of a value over the two lanes of a particle (every lane of the warp must call it).
__device__ __forceinline__ double pair_sum(const double v) { return v + __shfl_xor_sync(kFull, v, 1); }
__device__ __forceinline__ d3 pair_sum(const d3 v) { return {pair_sum(v.x), pair_sum(v.y), pair_sum(v.z)}; }

// Hit-mask lists: pair j of particle s is one 8-byte word of its warp's interleaved row.
__device__ __forceinline__ size_t mask_row(const uint32_t s, const uint32_t capacity_pairs) {
    return (static_cast<size_t>(s >> 5) * capacity_pairs) * 32u + (s & 31u);
}

// Yields the slots of a hit-mask list in order: the set bits of each (base, mask) pair, ascending.
// The next pair is loaded while the current one is drained.
struct MaskCursor {
    const uint2* __restrict__ pairs;   // the particle's row (stride 32 pairs)
    uint32_t capacity;
    uint32_t next_index;
    uint2 current, upcoming;
    __device__ __forceinline__ void start(const uint2* row, const uint32_t capacity_pairs) {
        pairs = row;
        capacity = capacity_pairs;
        current = row[0];
        upcoming = capacity_pairs > 1u ? row[32] : make_uint2(0u, 0u);
        next_index = 2u;
    }
    // The next slot; call at most as many times as the list has neighbours.
    __device__ __forceinline__ uint32_t take() {
        if (current.y == 0u) {
            current = upcoming;
            upcoming = next_index < capacity ? pairs[static_cast<size_t>(next_index) * 32u] : make_uint2(0u, 0u);
            ++next_index;
        }
        const uint32_t k = static_cast<uint32_t>(__ffs(current.y)) - 1u;
        current.y &= current.y - 1u;
        return current.x + k;
    }
};

// replay over a hit-mask list: the same entries in the same order as the index list.
template <class Op>
__device__ __forceinline__ void replay_masks(Op& op, const Particle& p, const GatherCommon& g, const StoredList& list) {
    if (!p.active) return;
    const uint32_t n = list.counts[p.s];
    if (n == kOverflow) {
        walk(op, p, g);
        return;
    }
    if (n == 0) return;
    MaskCursor cursor;
    const uint32_t capacity = list.capacity / 2u;
    cursor.start(reinterpret_cast<const uint2*>(list.entries) + mask_row(p.s, capacity), capacity);
    uint32_t t = cursor.take();
    auto data = op.prefetch(t);
    for (uint32_t k = 1; k < n; ++k) {
        const uint32_t tn = cursor.take();
        const auto next = op.prefetch(tn);
        op.apply(t, data);
        t = tn;
        data = next;
    }
    op.apply(t, data);
}

// The replay of either list format (Masks: a hit-mask list).  Expanding the masks into a
// shared-memory index list before the replay was slower at 1M particles (0.32-0.45 ms per pass
// against 0.17-0.20 ms): the stage cost occupancy and its decode loop serialised the pair loads.
template <bool Masks, class Op>
__device__ __forceinline__ void replay_list(Op& op, const Particle& p, const GatherCommon& g, const StoredList& list) {
    if constexpr (Masks) replay_masks(op, p, g, list);
    else replay<2>(op, p, g, list);
}

}  // namespace gather_detail
}  // namespace pbf
