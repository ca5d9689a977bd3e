// Forward neighbour-gather passes of the PBF substep over cell-sorted particles.
//
// Reference passes and the fused kernels that replace them:
//   density (density/density.cu:18-40) + lambda (pbf/pbf.cu:95-127)    -> density_lambda_kernel
//   correction (pbf/pbf.cu:254-288) + project (pbf/pbf.cu:417-431)
//     [+ reconstruct (pbf/pbf.cu:456-460) on the last iteration]        -> correction_kernel
//   vorticity (pbf/pbf.cu:476-497) + magnitude (pbf/pbf.cu:565-569)    -> vorticity_kernel
//   normal (pbf/pbf.cu:571-593) + confinement (pbf/pbf.cu:674-678)     -> normal_kernel
//   XSPH (pbf/pbf.cu:700-721) + write-back of next_state               -> xsph_kernel
//
// A list-scan kernel first writes, for every particle, the sorted slots of its neighbours inside
// the union of all supports, in the reference's stencil order (gather.cuh); each gather pass then
// replays the list with the reference's per-pair expressions, so every per-particle sum is
// accumulated in the reference's order and equals it bit for bit (skipped candidates contribute
// an exact zero in the reference).  Separating the cheap candidate tests from the costly per-pair
// math (sqrt, divisions) keeps that math convergent across the warp.
#include <climits>

#include "gather.cuh"

namespace pbf {

namespace {

using namespace gather_detail;

// --------------------------------------------------------------- list scan
// Builds the ordered neighbour list of every particle over the positions `pos` (gather.cuh).
// Per-lane list scan: every lane walks its own nine stencil columns in the reference's order and
// appends its hits; lanes of one home cell read the same candidates at the same time (one
// broadcast load).  Same lists as list_scan_kernel.
//
// A range is tested 32 candidates at a time: four loads are issued together, each test sets one
// bit of a hit mask, and the hits are then appended in ascending order from the mask.  The
// per-candidate work is the distance test alone, with no branch; only hits pay for a store.
struct RangeScan {
    f3 x;
    float threshold;
    uint32_t capacity;
    uint32_t* __restrict__ entries;
    uint32_t n;

    __device__ __forceinline__ uint32_t hit(const float4 q) const {
        return squared(mk(__fsub_rn(x.x, q.x), __fsub_rn(x.y, q.y), __fsub_rn(x.z, q.z))) < threshold ? 1u : 0u;
    }
    __device__ __forceinline__ uint32_t hits4(const float4 q0, const float4 q1, const float4 q2, const float4 q3) const {
        return hit(q0) | (hit(q1) << 1) | (hit(q2) << 2) | (hit(q3) << 3);
    }
    // Appends slot base + k (with `tag`) for every set bit k of `mask`, in ascending k.
    __device__ __forceinline__ void append(uint32_t mask, const uint32_t base, const uint32_t tag) {
        while (mask) {
            const uint32_t k = static_cast<uint32_t>(__ffs(mask)) - 1u;
            if (n < capacity) entries[static_cast<size_t>(n) * 32u] = (base + k) | tag;
            ++n;
            mask &= mask - 1u;
        }
    }
    // Tests the candidates pos[first, end) in order.  The last group of a 32-candidate block
    // repeats slot end - 1 in place of the slots past the range and drops their bits.
    __device__ __forceinline__ void run(const float4* __restrict__ pos, const uint32_t first, const uint32_t end,
                                        const uint32_t tag = 0u) {
        for (uint32_t base = first; base < end; base += 32u) {
            const uint32_t span = min(end - base, 32u);
            uint32_t mask = 0u, k = 0u;
            for (; k + 4u <= span; k += 4u) {
                const uint32_t t = base + k;
                mask |= hits4(pos[t], pos[t + 1u], pos[t + 2u], pos[t + 3u]) << k;
            }
            if (k < span) {
                const uint32_t t = base + k, l = end - 1u;
                const uint32_t m = hits4(pos[t], pos[min(t + 1u, l)], pos[min(t + 2u, l)], pos[min(t + 3u, l)]);
                mask |= (m & ((1u << (span - k)) - 1u)) << k;
            }
            append(mask, base, tag);
        }
    }
};

// The same test over positions stored as three arrays, two candidates per packed FP32 instruction
// (__fadd2_rn, __fmul2_rn, __ffma2_rn round each half exactly as the scalar intrinsics do).  The
// difference is taken as candidate minus particle; it is the exact negation of the scalar form's
// particle minus candidate, so the squared distance has the same bits.  Groups of four slots are
// loaded as one aligned float4 per axis: a range is widened down to a multiple of four and the
// slots outside it are dropped from the mask.
struct PackedScan {
    float2 nx, ny, nz;   // the particle's negated coordinates, in both halves
    float threshold;
    uint32_t capacity;
    uint32_t* __restrict__ entries;
    uint32_t n;

    __device__ __forceinline__ uint32_t hits2(const float2 x, const float2 y, const float2 z) const {
        const float2 dx = __fadd2_rn(x, nx), dy = __fadd2_rn(y, ny), dz = __fadd2_rn(z, nz);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
        return (r2.x < threshold ? 1u : 0u) | (r2.y < threshold ? 2u : 0u);
    }
    __device__ __forceinline__ uint32_t hits4(const float4 x, const float4 y, const float4 z) const {
        return hits2(make_float2(x.x, x.y), make_float2(y.x, y.y), make_float2(z.x, z.y)) |
               (hits2(make_float2(x.z, x.w), make_float2(y.z, y.w), make_float2(z.z, z.w)) << 2);
    }
    __device__ __forceinline__ void append(uint32_t mask, const uint32_t base) {
        while (mask) {
            const uint32_t k = static_cast<uint32_t>(__ffs(mask)) - 1u;
            if (n < capacity) entries[static_cast<size_t>(n) * 32u] = base + k;
            ++n;
            mask &= mask - 1u;
        }
    }
    // Hit mask of the 32-slot block at `base` (4-aligned) of the range [first, end).
    __device__ __forceinline__ uint32_t block_mask(const PackedPositions p, const uint32_t base, const uint32_t first,
                                                   const uint32_t end) const {
        const uint32_t stop = min(end, base + 32u);
        uint32_t mask = 0u;
        for (uint32_t k = 0u; base + k < stop; k += 4u) {
            const uint32_t t = base + k;
            mask |= hits4(*reinterpret_cast<const float4*>(p.x + t), *reinterpret_cast<const float4*>(p.y + t),
                          *reinterpret_cast<const float4*>(p.z + t))
                    << k;
        }
        if (base < first) mask &= ~0u << (first - base);
        if (end - base < 32u) mask &= (1u << (end - base)) - 1u;
        return mask;
    }
    __device__ __forceinline__ void run(const PackedPositions p, const uint32_t first, const uint32_t end) {
        if (first >= end) return;
        for (uint32_t base = first & ~3u; base < end; base += 32u) append(block_mask(p, base, first, end), base);
    }
    // The same blocks stored as a hit-mask list: one (base, mask) pair per block with a hit, `pairs`
    // of them so far (at most `pair_capacity` are written), `n` neighbours.
    __device__ __forceinline__ void run_masks(const PackedPositions p, const uint32_t first, const uint32_t end,
                                              uint2* __restrict__ row, const uint32_t pair_capacity, uint32_t& pairs) {
        if (first >= end) return;
        for (uint32_t base = first & ~3u; base < end; base += 32u) {
            const uint32_t mask = block_mask(p, base, first, end);
            if (mask) {
                if (pairs < pair_capacity) row[static_cast<size_t>(pairs) * 32u] = make_uint2(base, mask);
                ++pairs;
                n += static_cast<uint32_t>(__popc(mask));
            }
        }
    }
};

template <bool Masks>
__global__ void __launch_bounds__(kBlock, 12) list_walk_kernel(const ListScanArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.g.count) return;
    const int4 c = a.g.cell[s];
    const SceneDesc* scene = a.g.scenes + c.w;
    const Grid grid = scene->grid;
    const int cx = static_cast<int>(grid.cells_x), cy = static_cast<int>(grid.cells_y), cz = static_cast<int>(grid.cells_z);
    const uint32_t z_lo = static_cast<uint32_t>(c.z > 0 ? c.z - 1 : 0);
    const uint32_t z_hi = static_cast<uint32_t>(c.z + 1 < cz ? c.z + 1 : cz - 1);
    RangeScan scan;
    scan.x = xyz(a.pos[s]);
    scan.threshold = a.g.constants[scene->constants].list_threshold;
    scan.capacity = a.list.capacity;
    scan.entries = a.list.entries + list_row(s, scan.capacity);
    scan.n = 0;
    const uint32_t* __restrict__ offsets = a.g.cell_offsets;
    if (a.boundary && a.g.boundary_offsets) {
        // cell by cell: each cell's fluid particles, then its boundary particles (pbf/pbf.cu:111-121)
        const uint32_t* __restrict__ boffsets = a.g.boundary_offsets;
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = c.x + dx;
            if (x < 0 || x >= cx) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = c.y + dy;
                if (y < 0 || y >= cy) continue;
                for (uint32_t z = z_lo; z <= z_hi; ++z) {
                    const uint32_t cell = cell_index(grid, x, y, z);
                    scan.run(a.pos, offsets[cell], offsets[cell + 1u]);
                    scan.run(a.g.boundary, boffsets[cell], boffsets[cell + 1u], kBoundaryBit);
                }
            }
        }
    } else if (a.packed.x) {
        // At 1M particles the packed test cut a scan from 0.233 to 0.200 ms.  A budget of 40
        // registers (12 blocks of 128 per SM) measured fastest; 45 and 52 were within 1 %.
        PackedScan packed;
        packed.nx = make_float2(-scan.x.x, -scan.x.x);
        packed.ny = make_float2(-scan.x.y, -scan.x.y);
        packed.nz = make_float2(-scan.x.z, -scan.x.z);
        packed.threshold = scan.threshold;
        packed.capacity = scan.capacity;
        packed.entries = scan.entries;
        packed.n = 0;
        if constexpr (Masks) {
            const uint32_t pair_capacity = scan.capacity / 2u;
            uint2* row = reinterpret_cast<uint2*>(a.list.entries) + mask_row(s, pair_capacity);
            uint32_t pairs = 0;
#pragma unroll 1
            for (int o = 0; o < 9; ++o) {
                const int x = c.x + o / 3 - 1, y = c.y + o % 3 - 1;
                if (x < 0 || x >= cx || y < 0 || y >= cy) continue;
                packed.run_masks(a.packed, offsets[cell_index(grid, x, y, z_lo)], offsets[cell_index(grid, x, y, z_hi) + 1u],
                                 row, pair_capacity, pairs);
            }
            a.list.counts[s] = pairs <= pair_capacity ? packed.n : kOverflow;
            return;
        }
#pragma unroll 1
        for (int o = 0; o < 9; ++o) {
            const int x = c.x + o / 3 - 1, y = c.y + o % 3 - 1;
            if (x < 0 || x >= cx || y < 0 || y >= cy) continue;
            packed.run(a.packed, offsets[cell_index(grid, x, y, z_lo)], offsets[cell_index(grid, x, y, z_hi) + 1u]);
        }
        scan.n = packed.n;
    } else {
        // Nine stencil columns, x-offset outer; each column's three cells are one contiguous range.
#pragma unroll 1
        for (int o = 0; o < 9; ++o) {
            const int x = c.x + o / 3 - 1, y = c.y + o % 3 - 1;
            if (x < 0 || x >= cx || y < 0 || y >= cy) continue;
            scan.run(a.pos, offsets[cell_index(grid, x, y, z_lo)], offsets[cell_index(grid, x, y, z_hi) + 1u]);
        }
    }
    a.list.counts[s] = scan.n <= scan.capacity ? scan.n : kOverflow;
}

// Staged list scan: the lanes of a warp that share a stencil column (same x, y and scene) stage
// the union of their nine column ranges (cells z_min-1 .. z_max+1 of the group) in shared memory
// with coalesced loads, then each lane tests its own nine ranges there.  A group whose union
// exceeds the stage walks global memory instead.  Same lists as the other scans.
constexpr uint32_t kStageCapacity = 704;   // float4 per warp (44 KB per 128-thread block)

__global__ void __launch_bounds__(kBlock) list_staged_kernel(const ListScanArgs a) {
    __shared__ float4 stage[kWarpsPerBlock][kStageCapacity];
    __shared__ uint32_t column_first[kWarpsPerBlock][9];
    __shared__ uint32_t column_base[kWarpsPerBlock][9];
    const uint32_t w = threadIdx.x >> 5, lane = lane_id();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = s < a.g.count;
    const int4 c = active ? a.g.cell[s] : make_int4(0, 0, 0, 0);
    const float4 xi = active ? a.pos[s] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    const uint32_t cap = a.list.capacity;
    uint32_t* __restrict__ entries = a.list.entries + list_row(s, cap);
    const uint32_t* __restrict__ offsets = a.g.cell_offsets;
    const float4* __restrict__ pos = a.pos;
    uint32_t n = 0;
    uint32_t pending = __ballot_sync(kFull, active);
    while (pending) {
        const int leader = __ffs(static_cast<int>(pending)) - 1;
        const int gx = __shfl_sync(kFull, c.x, leader), gy = __shfl_sync(kFull, c.y, leader);
        const int gw = __shfl_sync(kFull, c.w, leader);
        const bool mine = ((pending >> lane) & 1u) != 0u && c.x == gx && c.y == gy && c.w == gw;
        pending &= ~__ballot_sync(kFull, mine);
        const SceneDesc* scene = a.g.scenes + gw;
        const Grid grid = scene->grid;
        const float thr = a.g.constants[scene->constants].list_threshold;
        const int cx = static_cast<int>(grid.cells_x), cy = static_cast<int>(grid.cells_y), cz = static_cast<int>(grid.cells_z);
        const int zmin = __reduce_min_sync(kFull, mine ? c.z : INT_MAX);
        const int zmax = __reduce_max_sync(kFull, mine ? c.z : INT_MIN);
        const uint32_t zlo = static_cast<uint32_t>(zmin > 0 ? zmin - 1 : 0);
        const uint32_t zhi = static_cast<uint32_t>(zmax + 1 < cz ? zmax + 1 : cz - 1);
        // lane o < 9: the group's union range of stencil column o
        uint32_t first = 0u, length = 0u;
        if (lane < 9u) {
            const int x = gx + static_cast<int>(lane) / 3 - 1, y = gy + static_cast<int>(lane) % 3 - 1;
            if (x >= 0 && x < cx && y >= 0 && y < cy) {
                first = offsets[cell_index(grid, x, y, zlo)];
                length = offsets[cell_index(grid, x, y, zhi) + 1u] - first;
            }
        }
        uint32_t inclusive = length;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, inclusive, o);
            if (lane >= static_cast<uint32_t>(o)) inclusive += v;
        }
        const uint32_t total = __shfl_sync(kFull, inclusive, 8);
        if (lane < 9u) {
            column_first[w][lane] = first;
            column_base[w][lane] = inclusive - length;
        }
        __syncwarp();
        const bool staged = total <= kStageCapacity;
        if (staged) {
            for (uint32_t u = lane; u < total; u += 32u) {
                uint32_t o = 0;   // the column holding staged slot u: last o with base <= u
#pragma unroll
                for (uint32_t step = 8; step > 0; step >>= 1)
                    if (o + step <= 8u && column_base[w][o + step] <= u) o += step;
                stage[w][u] = pos[column_first[w][o] + (u - column_base[w][o])];
            }
        }
        __syncwarp();
        if (mine) {
            const uint32_t z_lo = static_cast<uint32_t>(c.z > 0 ? c.z - 1 : 0);
            const uint32_t z_hi = static_cast<uint32_t>(c.z + 1 < cz ? c.z + 1 : cz - 1);
            auto test = [&](const float4 q, const uint32_t t) {
                const float r2 = squared(mk(__fsub_rn(xi.x, q.x), __fsub_rn(xi.y, q.y), __fsub_rn(xi.z, q.z)));
                if (r2 < thr) {
                    if (n < cap) entries[static_cast<size_t>(n) * 32u] = t;
                    ++n;
                }
            };
#pragma unroll
            for (int o = 0; o < 9; ++o) {
                const int x = c.x + o / 3 - 1, y = c.y + o % 3 - 1;
                if (x < 0 || x >= cx || y < 0 || y >= cy) continue;
                const uint32_t lo = offsets[cell_index(grid, x, y, z_lo)];
                const uint32_t hi = offsets[cell_index(grid, x, y, z_hi) + 1u];
                if (staged) {
                    // slot t of this column sits at stage index t - first + base
                    const uint32_t shift = column_base[w][o] - column_first[w][o];
                    for (uint32_t t = lo; t < hi; ++t) test(stage[w][t + shift], t);
                } else {
                    for (uint32_t t = lo; t < hi; ++t) test(pos[t], t);
                }
            }
        }
        __syncwarp();
    }
    if (active) a.list.counts[s] = n <= cap ? n : kOverflow;
}

__global__ void __launch_bounds__(kBlock) list_scan_kernel(const ListScanArgs a) {
    __shared__ float4 home_s[kWarpsPerBlock][32];
    __shared__ uint32_t first_s[kWarpsPerBlock][32];
    __shared__ uint32_t base_s[kWarpsPerBlock][32];
    const uint32_t w = threadIdx.x >> 5, lane = lane_id();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = s < a.g.count;
    const int4 c = active ? a.g.cell[s] : make_int4(0, 0, 0, 0);
    const float threshold = active ? a.g.constants[a.g.scenes[c.w].constants].list_threshold : 0.0F;
    const int nact = __popc(__ballot_sync(kFull, active));
    home_s[w][lane] = active ? a.pos[s] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    const int px = __shfl_up_sync(kFull, c.x, 1), py = __shfl_up_sync(kFull, c.y, 1);
    const int pz = __shfl_up_sync(kFull, c.z, 1), pw = __shfl_up_sync(kFull, c.w, 1);
    const bool start = active && (lane == 0 || px != c.x || py != c.y || pz != c.z || pw != c.w);
    uint32_t starts = __ballot_sync(kFull, start);
    const unsigned lower = (1u << lane) - 1u;
    const uint32_t cap = a.list.capacity;
    uint32_t* __restrict__ entries = a.list.entries + static_cast<size_t>(s >> 5) * cap * 32u;
    uint32_t n = 0;
    __syncwarp();
    while (starts) {
        const int ra = __ffs(starts) - 1;
        starts &= starts - 1u;
        const int rb = starts ? __ffs(starts) - 1 : nact;
        const int hx = __shfl_sync(kFull, c.x, ra), hy = __shfl_sync(kFull, c.y, ra);
        const int hz = __shfl_sync(kFull, c.z, ra), hw = __shfl_sync(kFull, c.w, ra);
        const float thr = __shfl_sync(kFull, threshold, ra);
        const Grid& grid = a.g.scenes[hw].grid;
        // lane o < 9 holds stencil column o (x-offset outer): cells z-1..z+1, one contiguous range
        uint32_t first = 0, cnt = 0;
        if (lane < 9u) {
            const int x = hx + static_cast<int>(lane) / 3 - 1;
            const int y = hy + static_cast<int>(lane) % 3 - 1;
            const int cz = static_cast<int>(grid.cells_z);
            if (x >= 0 && y >= 0 && x < static_cast<int>(grid.cells_x) && y < static_cast<int>(grid.cells_y)) {
                const uint32_t z_lo = static_cast<uint32_t>(hz > 0 ? hz - 1 : 0);
                const uint32_t z_hi = static_cast<uint32_t>(hz + 1 < cz ? hz + 1 : cz - 1);
                first = a.g.cell_offsets[cell_index(grid, x, y, z_lo)];
                cnt = a.g.cell_offsets[cell_index(grid, x, y, z_hi) + 1u] - first;
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
        first_s[w][lane] = first;
        base_s[w][lane] = lane < 9u ? inc - cnt : total;
        __syncwarp();
        for (uint32_t u0 = 0; u0 < total; u0 += 32u) {
            const uint32_t u = u0 + lane;
            const bool valid = u < total;
            uint32_t o = 0;
#pragma unroll
            for (uint32_t step = 8; step > 0; step >>= 1)
                if (base_s[w][o + step] <= u) o += step;
            const uint32_t t = first_s[w][o] + (u - base_s[w][o]);
            const float4 q = valid ? a.pos[t] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
            for (int h = ra; h < rb; ++h) {
                const float4 xh = home_s[w][h];
                const float r2 = squared(mk(__fsub_rn(xh.x, q.x), __fsub_rn(xh.y, q.y), __fsub_rn(xh.z, q.z)));
                const bool in = valid && r2 < thr;
                const unsigned m = __ballot_sync(kFull, in);
                if (m) {
                    const uint32_t nh = __shfl_sync(kFull, n, h);
                    const uint32_t k = nh + __popc(m & lower);
                    if (in && k < cap) entries[static_cast<size_t>(k) * 32u + static_cast<uint32_t>(h)] = t;
                    if (static_cast<int>(lane) == h) n += __popc(m);
                }
            }
        }
        __syncwarp();
    }
    if (active) a.list.counts[s] = n <= cap ? n : kOverflow;
}

// ------------------------------------------------------------------ density + lambda
// density (density/density.cu:18-40) and lambda (pbf/pbf.cu:95-127) of one particle in one walk.
// m_j / rho0_i for a run of neighbours: most neighbours share a mass, so the last quotient is
// kept and reused while the mass bits repeat (same operands, same correctly rounded quotient).
struct MassRatio {
    uint32_t mass_bits;
    float quotient;
    __device__ __forceinline__ void reset(const float mass, const float rest_density) {
        mass_bits = __float_as_uint(mass);
        quotient = __fdiv_rn(mass, rest_density);
    }
    __device__ __forceinline__ float operator()(const float mass, const float rest_density) {
        const uint32_t bits = __float_as_uint(mass);
        if (bits != mass_bits) reset(mass, rest_density);
        return quotient;
    }
};

// WithBoundary: the scene has boundary particles (their entries carry kBoundaryBit); the plain
// instantiation, launched otherwise, carries no boundary test.
template <bool WithBoundary>
struct DensityLambdaOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    f3 x;
    uint32_t self;
    float rest_density;
    KernelConstants k;
    float density;
    f3 gradient_sum;
    float denominator;
    uint32_t neighbors;
    MassRatio ratio;

    __device__ __forceinline__ float4 prefetch(const uint32_t t) const {
        if constexpr (WithBoundary) return (t & kBoundaryBit) ? boundary[t & ~kBoundaryBit] : pos[t];
        return pos[t];
    }
    __device__ __forceinline__ void apply(const uint32_t t, const float4 q) {
        const f3 d = sub(x, xyz(q));
        const float r2 = squared(d);
        if (WithBoundary && (t & kBoundaryBit)) {
            // boundary particle b: density += rho0_i V_b W (density/density.cu:34-37),
            // S += V_b grad W (pbf/pbf.cu:118-121); no denominator term
            if (r2 < k.h2) density = __fmaf_rn(__fmul_rn(rest_density, q.w), poly6_inside(r2, k), density);
            const float distance = __fsqrt_rn(r2);
            if (distance == 0.0F || distance >= k.h) return;
            gradient_sum = fma3(q.w, spiky_gradient_at(d, distance, k), gradient_sum);
            return;
        }
        if (r2 < k.h2) density = __fmaf_rn(q.w, poly6_inside(r2, k), density);
        if (t == self) return;
        if (r2 < k.h2) ++neighbors;
        const float distance = __fsqrt_rn(r2);
        if (distance == 0.0F || distance >= k.h) return;
        const f3 gradient = spiky_gradient_at(d, distance, k);
        const float coefficient = ratio(q.w, rest_density);
        gradient_sum = fma3(coefficient, gradient, gradient_sum);
        denominator = __fmaf_rn(__fmul_rn(coefficient, coefficient), sq_xfirst(gradient), denominator);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

template <bool WithBoundary>
__global__ void __launch_bounds__(kBlock) density_lambda_kernel(const DensityLambdaArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    DensityLambdaOp<WithBoundary> op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    op.self = p.s;
    op.k = p.k;
    const float4 xi = a.pos[p.s];
    const float4 pa = a.g.params_a[p.s];
    op.x = xyz(xi);
    op.rest_density = pa.x;
    op.density = 0.0F;
    op.gradient_sum = mk(0.0F, 0.0F, 0.0F);
    op.denominator = pa.y;  // relaxation
    op.neighbors = 0;
    op.ratio.reset(xi.w, op.rest_density);
    replay<2>(op, p, a.g, a.list);
    const float denominator = __fadd_rn(op.denominator, sq_yfirst(op.gradient_sum));
    a.lambda[p.s] = __fdiv_rn(-__fsub_rn(__fdiv_rn(op.density, op.rest_density), 1.0F), denominator);
    if (a.density) a.density[p.s] = op.density;
    if (a.gsum_denom) a.gsum_denom[p.s] = make_float4(op.gradient_sum.x, op.gradient_sum.y, op.gradient_sum.z, denominator);
    if (a.neighbor_count) a.neighbor_count[p.s] = op.neighbors;
}

// ------------------------------------------- list scan fused with density + lambda
// One kernel per Jacobi iteration in place of list_walk_kernel + density_lambda_kernel: each lane
// runs the per-lane packed scan of its particle, writing the stored list (which the correction pass
// replays) and, for its first kStagedEntries entries, a copy in shared memory; it then replays its
// own list with the density and lambda arithmetic, reading the staged entries from shared memory
// (the rest, if any, from the stored list).  The list, its order and every sum are those of the
// two-kernel path, so the results are bit-identical.  Scenes with boundary particles use the two
// kernels.
// Staged entries per lane and the blocks per SM the register budget is sized for (compile-time
// tuning knobs; the defaults measured fastest at 1M particles).
// At 1M particles (steps 3-13 of the dam break, ms per launch): 9 blocks and 40 entries 0.336;
// 8 and 32 0.341; 8 and 48 0.360; 10 and 40 (spilling) 0.400; 8 and 64 0.410; 12 and 32 0.513.
#ifndef PBF_FUSED_STAGED_ENTRIES
#define PBF_FUSED_STAGED_ENTRIES 40
#endif
#ifndef PBF_FUSED_MIN_BLOCKS
#define PBF_FUSED_MIN_BLOCKS 9
#endif
constexpr uint32_t kStagedEntries = PBF_FUSED_STAGED_ENTRIES;   // 40: 20 KB of shared memory per 128-thread block

// Masks: the list is stored as a hit-mask list (one (base, mask) pair per block with a hit), the
// first kStagedEntries / 2 pairs staged in the same shared memory.
template <bool Masks>
__global__ void __launch_bounds__(kBlock, PBF_FUSED_MIN_BLOCKS) scan_density_lambda_kernel(const ListScanArgs a,
                                                                                          const DensityLambdaArgs d) {
    __shared__ __align__(8) uint32_t staged[kStagedEntries * kBlock];
    constexpr uint32_t kStagedPairs = kStagedEntries / 2u;
    uint2* const staged_pairs = reinterpret_cast<uint2*>(staged);
    const Particle p = locate(a.g);
    if (!p.active) return;
    const uint32_t s = p.s, lane_slot = threadIdx.x;
    const Grid& grid = p.scene->grid;
    const int cx = static_cast<int>(grid.cells_x), cy = static_cast<int>(grid.cells_y), cz = static_cast<int>(grid.cells_z);
    const uint32_t z_lo = static_cast<uint32_t>(p.c.z > 0 ? p.c.z - 1 : 0);
    const uint32_t z_hi = static_cast<uint32_t>(p.c.z + 1 < cz ? p.c.z + 1 : cz - 1);
    const float4 xi = a.pos[s];
    const uint32_t capacity = a.list.capacity;
    const uint32_t pair_capacity = capacity / 2u;
    uint32_t* __restrict__ entries = a.list.entries + list_row(s, capacity);
    uint2* __restrict__ pairs_row = reinterpret_cast<uint2*>(a.list.entries) + mask_row(s, pair_capacity);
    const uint32_t* __restrict__ offsets = a.g.cell_offsets;
    // 1. the per-lane packed scan (PackedScan), appending to the stored list and the stage
    uint32_t n = 0, pairs = 0;
    {
        PackedScan scan;
        scan.nx = make_float2(-xi.x, -xi.x);
        scan.ny = make_float2(-xi.y, -xi.y);
        scan.nz = make_float2(-xi.z, -xi.z);
        scan.threshold = p.k.list_threshold;
        const PackedPositions pk = a.packed;
#pragma unroll 1
        for (int o = 0; o < 9; ++o) {
            const int x = p.c.x + o / 3 - 1, y = p.c.y + o % 3 - 1;
            if (x < 0 || x >= cx || y < 0 || y >= cy) continue;
            const uint32_t first = offsets[cell_index(grid, x, y, z_lo)];
            const uint32_t end = offsets[cell_index(grid, x, y, z_hi) + 1u];
            if (first >= end) continue;
            for (uint32_t base = first & ~3u; base < end; base += 32u) {
                uint32_t mask = scan.block_mask(pk, base, first, end);
                if constexpr (Masks) {
                    if (mask) {
                        const uint2 pair = make_uint2(base, mask);
                        if (pairs < pair_capacity) pairs_row[static_cast<size_t>(pairs) * 32u] = pair;
                        if (pairs < kStagedPairs) staged_pairs[pairs * kBlock + lane_slot] = pair;
                        ++pairs;
                        n += static_cast<uint32_t>(__popc(mask));
                    }
                } else {
                    while (mask) {
                        const uint32_t k = static_cast<uint32_t>(__ffs(mask)) - 1u;
                        if (n < capacity) entries[static_cast<size_t>(n) * 32u] = base + k;
                        if (n < kStagedEntries) staged[n * kBlock + lane_slot] = base + k;
                        ++n;
                        mask &= mask - 1u;
                    }
                }
            }
        }
        const bool overflow = Masks ? pairs > pair_capacity : n > capacity;
        a.list.counts[s] = overflow ? kOverflow : n;
        if (overflow) n = kOverflow;
    }
    // 2. density (density/density.cu:18-40) and lambda (pbf/pbf.cu:95-127) over the same list
    DensityLambdaOp<false> op;
    op.pos = a.pos;
    op.boundary = nullptr;
    op.self = s;
    op.k = p.k;
    const float4 pa = a.g.params_a[s];
    op.x = xyz(xi);
    op.rest_density = pa.x;
    op.density = 0.0F;
    op.gradient_sum = mk(0.0F, 0.0F, 0.0F);
    op.denominator = pa.y;  // relaxation
    op.neighbors = 0;
    op.ratio.reset(xi.w, op.rest_density);
    if (n == kOverflow) {
        walk(op, p, a.g);
    } else if (n > 0) {
        uint2 current{}, upcoming{};
        uint32_t next_pair = 2u;
        auto pair_at = [&](const uint32_t j) -> uint2 {
            return j < kStagedPairs ? staged_pairs[j * kBlock + lane_slot] : pairs_row[static_cast<size_t>(j) * 32u];
        };
        if constexpr (Masks) {
            current = pair_at(0);
            upcoming = pairs > 1u ? pair_at(1) : make_uint2(0u, 0u);
        }
        auto entry = [&](const uint32_t k) -> uint32_t {
            if constexpr (Masks) {
                (void)k;
                if (current.y == 0u) {
                    current = upcoming;
                    upcoming = next_pair < pairs ? pair_at(next_pair) : make_uint2(0u, 0u);
                    ++next_pair;
                }
                const uint32_t bit = static_cast<uint32_t>(__ffs(current.y)) - 1u;
                current.y &= current.y - 1u;
                return current.x + bit;
            } else {
                return k < kStagedEntries ? staged[k * kBlock + lane_slot] : entries[static_cast<size_t>(k) * 32u];
            }
        };
        uint32_t t = entry(0);
        uint32_t tn = n > 1u ? entry(1) : 0u;
        float4 data = op.prefetch(t);
        for (uint32_t k = 1; k < n; ++k) {
            const uint32_t tnn = k + 1u < n ? entry(k + 1u) : 0u;
            const float4 next = op.prefetch(tn);
            op.apply(t, data);
            t = tn;
            tn = tnn;
            data = next;
        }
        op.apply(t, data);
    }
    const float denominator = __fadd_rn(op.denominator, sq_yfirst(op.gradient_sum));
    d.lambda[s] = __fdiv_rn(-__fsub_rn(__fdiv_rn(op.density, op.rest_density), 1.0F), denominator);
    if (d.density) d.density[s] = op.density;
    if (d.gsum_denom) d.gsum_denom[s] = make_float4(op.gradient_sum.x, op.gradient_sum.y, op.gradient_sum.z, denominator);
    if (d.neighbor_count) d.neighbor_count[s] = op.neighbors;
}

// ------------------------------------------------------- correction + project
// correction (pbf/pbf.cu:254-288) and project (pbf/pbf.cu:417-431); on the last iteration
// also reconstruct (pbf/pbf.cu:456-460) and the write-back of next_state.positions.
struct PositionLambda {
    float4 q;
    float lambda;
};

template <bool WithBoundary>
struct CorrectionOp {
    static constexpr bool kBoundary = WithBoundary;
    const float4* __restrict__ pos;
    const float4* __restrict__ boundary;
    const float* __restrict__ lambda;
    f3 x;
    uint32_t self;
    float rest_density;
    float lambda_i;
    float strength, exponent, reference_weight;
    bool artificial_full;
    KernelConstants k;
    f3 correction;
    MassRatio ratio;

    __device__ __forceinline__ PositionLambda prefetch(const uint32_t t) const {
        if (WithBoundary && (t & kBoundaryBit)) return {boundary[t & ~kBoundaryBit], 0.0F};
        return {pos[t], lambda[t]};
    }
    __device__ __forceinline__ void apply(const uint32_t t, const PositionLambda in) {
        if (t == self) return;
        const f3 d = sub(x, xyz(in.q));
        const float r2 = squared(d);
        const float distance = __fsqrt_rn(r2);
        if (distance == 0.0F || distance >= k.h) return;
        // s_corr (pbf/pbf.cu:56-71).  With zero strength it is -strength * ratio^n, i.e. -0 inside
        // the poly6 support and 0 outside, which the fast branch yields without powf.
        float artificial;
        if (artificial_full) {
            const float weight = r2 >= k.h2 ? 0.0F : poly6_inside(r2, k);
            artificial = weight == 0.0F ? 0.0F : __fmul_rn(-strength, powf(__fdiv_rn(weight, reference_weight), exponent));
        } else {
            artificial = r2 < k.h2 ? -strength : 0.0F;
        }
        if (WithBoundary && (t & kBoundaryBit)) {
            // boundary particle b: V_b (lambda_i + s_corr) grad W (pbf/pbf.cu:278-285)
            const float factor = __fmul_rn(in.q.w, __fadd_rn(lambda_i, artificial));
            correction = fma3(factor, spiky_gradient_at(d, distance, k), correction);
            return;
        }
        const float coefficient = ratio(in.q.w, rest_density);
        const float factor = __fmul_rn(coefficient, __fadd_rn(__fadd_rn(lambda_i, in.lambda), artificial));
        correction = fma3(factor, spiky_gradient_at(d, distance, k), correction);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

// Resident 128-thread blocks per SM the register budget of the correction and of the post-loop
// passes is sized for (compile-time tuning knobs; 0 leaves the register count to the compiler).
// At 1M particles (substeps 25-28, ms per launch): the correction at 9 (56 registers instead of
// 58, 36 resident warps instead of 32) 0.193 against 0.203, at 10 (48, spilling) 0.286; the
// vorticity / normal / XSPH passes at 10 (48 registers) 0.192 / 0.176 / 0.188 against 0.207 /
// 0.183 / 0.196 unbounded.
#ifndef PBF_CORRECTION_MIN_BLOCKS
#define PBF_CORRECTION_MIN_BLOCKS 9
#endif
#ifndef PBF_POST_MIN_BLOCKS
#define PBF_POST_MIN_BLOCKS 10
#endif

template <bool WithBoundary, bool Masks>
__global__ void __launch_bounds__(kBlock, PBF_CORRECTION_MIN_BLOCKS) correction_kernel(const CorrectionArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    CorrectionOp<WithBoundary> op;
    op.pos = a.pos;
    op.boundary = a.g.boundary;
    op.lambda = a.lambda;
    op.self = p.s;
    op.k = p.k;
    const float4 xi = a.pos[p.s];
    const float4 pa = a.g.params_a[p.s];
    const float4 pb = a.g.params_b[p.s];
    op.x = xyz(xi);
    op.rest_density = pa.x;
    op.ratio.reset(xi.w, op.rest_density);
    op.lambda_i = a.lambda[p.s];
    op.strength = pb.x;
    op.exponent = pb.y;
    op.artificial_full = pb.x != 0.0F;
    op.reference_weight = op.artificial_full ? poly6(mk(pb.z, 0.0F, 0.0F), p.k) : 1.0F;
    op.correction = mk(0.0F, 0.0F, 0.0F);
    replay_list<Masks>(op, p, a.g, a.list);
    const Box& box = p.scene->box;
    const f3 candidate = add(op.x, op.correction);
    uint32_t mask = 0u;
    if (candidate.x < box.min_x || candidate.x > box.max_x) mask |= 1u;
    if (candidate.y < box.min_y || candidate.y > box.max_y) mask |= 2u;
    if (candidate.z < box.min_z || candidate.z > box.max_z) mask |= 4u;
    const f3 projected = mk(fminf(box.max_x, fmaxf(box.min_x, candidate.x)), fminf(box.max_y, fmaxf(box.min_y, candidate.y)),
                            fminf(box.max_z, fmaxf(box.min_z, candidate.z)));
    a.pos_next[p.s] = make_float4(projected.x, projected.y, projected.z, xi.w);
    if (a.packed.x) {
        a.packed.x[p.s] = projected.x;
        a.packed.y[p.s] = projected.y;
        a.packed.z[p.s] = projected.z;
    }
    if (a.mask) a.mask[p.s] = static_cast<uint8_t>(mask);
    if (a.last) {
        const uint32_t i = a.sorted_index[p.s];
        const f3 previous = mk(a.previous_positions.x[i], a.previous_positions.y[i], a.previous_positions.z[i]);
        const f3 velocity = scale(sub(projected, previous), p.scene->inverse_time_step);
        a.velocity[p.s] = make_float4(velocity.x, velocity.y, velocity.z, 0.0F);
        a.out_positions.x[i] = projected.x;
        a.out_positions.y[i] = projected.y;
        a.out_positions.z[i] = projected.z;
    }
}

// ---------------------------------------------------------------- vorticity
// vorticity (pbf/pbf.cu:476-497) and its magnitude (pbf/pbf.cu:565-569).
struct PositionVector {
    float4 q;
    float4 v;
};

struct VorticityOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ velocity;
    f3 x, v;
    uint32_t self;
    KernelConstants k;
    f3 vorticity;

    __device__ __forceinline__ PositionVector prefetch(const uint32_t t) const { return {pos[t], velocity[t]}; }
    __device__ __forceinline__ void apply(const uint32_t t, const PositionVector in) {
        if (t == self) return;
        const f3 d = sub(x, xyz(in.q));
        const float distance = __fsqrt_rn(squared(d));
        if (distance == 0.0F || distance >= k.h) return;
        vorticity = add(vorticity, cross_f(sub(xyz(in.v), v), spiky_gradient_at(d, distance, k)));
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

template <bool Masks>
__global__ void __launch_bounds__(kBlock, PBF_POST_MIN_BLOCKS) vorticity_kernel(const VorticityArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    VorticityOp op;
    op.pos = a.pos;
    op.velocity = a.velocity;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.v = xyz(a.velocity[p.s]);
    op.vorticity = mk(0.0F, 0.0F, 0.0F);
    replay_list<Masks>(op, p, a.g, a.list);
    a.vorticity[p.s] = make_float4(op.vorticity.x, op.vorticity.y, op.vorticity.z, __fsqrt_rn(sq_xfirst(op.vorticity)));
}

// ------------------------------------------------------- normal + confinement
// normal (pbf/pbf.cu:571-593) and confinement (pbf/pbf.cu:674-678).
struct PositionScalar {
    float4 q;
    float w;
};

struct NormalOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ vorticity;
    f3 x;
    float magnitude;
    uint32_t self;
    KernelConstants k;
    f3 gradient;

    __device__ __forceinline__ PositionScalar prefetch(const uint32_t t) const { return {pos[t], vorticity[t].w}; }
    __device__ __forceinline__ void apply(const uint32_t t, const PositionScalar in) {
        if (t == self) return;
        const f3 d = sub(x, xyz(in.q));
        const float distance = __fsqrt_rn(squared(d));
        if (distance == 0.0F || distance >= k.h) return;
        gradient = fma3(__fsub_rn(in.w, magnitude), spiky_gradient_at(d, distance, k), gradient);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

template <bool Masks>
__global__ void __launch_bounds__(kBlock, PBF_POST_MIN_BLOCKS) normal_kernel(const NormalArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    NormalOp op;
    op.pos = a.pos;
    op.vorticity = a.vorticity;
    op.self = p.s;
    op.k = p.k;
    const float4 wi = a.vorticity[p.s];
    op.x = xyz(a.pos[p.s]);
    op.magnitude = wi.w;
    op.gradient = mk(0.0F, 0.0F, 0.0F);
    replay_list<Masks>(op, p, a.g, a.list);
    const float normalizer = __fsqrt_rn(sq_yfirst(op.gradient));
    const f3 normal = normalizer > 0.0F ? scale(op.gradient, __fdiv_rn(1.0F, normalizer)) : mk(0.0F, 0.0F, 0.0F);
    a.normal[p.s] = make_float4(normal.x, normal.y, normal.z, normalizer);
    const float4 pa = a.g.params_a[p.s];
    const f3 v = xyz(a.velocity[p.s]);
    const f3 confined = fma3(__fmul_rn(p.scene->time_step, pa.w), cross_f(normal, xyz(wi)), v);
    a.confined[p.s] = make_float4(confined.x, confined.y, confined.z, 0.0F);
}

// ---------------------------------------------------------------------- XSPH
// XSPH (pbf/pbf.cu:700-721) and the write-back of next_state.velocities.
struct XsphOp {
    const float4* __restrict__ pos;
    const float4* __restrict__ confined;
    f3 x, v;
    uint32_t self;
    KernelConstants k;
    f3 smoothing;

    __device__ __forceinline__ PositionVector prefetch(const uint32_t t) const { return {pos[t], confined[t]}; }
    __device__ __forceinline__ void apply(const uint32_t t, const PositionVector in) {
        if (t == self) return;
        const f3 d = sub(x, xyz(in.q));
        const float r2 = squared(d);
        if (r2 >= k.h2) return;
        smoothing = fma3(poly6_inside(r2, k), sub(xyz(in.v), v), smoothing);
    }
    __device__ __forceinline__ void process(const uint32_t t) { apply(t, prefetch(t)); }
};

template <bool Masks>
__global__ void __launch_bounds__(kBlock, PBF_POST_MIN_BLOCKS) xsph_kernel(const XsphArgs a) {
    const Particle p = locate(a.g);
    if (!p.active) return;
    XsphOp op;
    op.pos = a.pos;
    op.confined = a.confined;
    op.self = p.s;
    op.k = p.k;
    op.x = xyz(a.pos[p.s]);
    op.v = xyz(a.confined[p.s]);
    op.smoothing = mk(0.0F, 0.0F, 0.0F);
    replay_list<Masks>(op, p, a.g, a.list);
    const float viscosity = a.g.params_a[p.s].z;
    const f3 out = fma3(viscosity, op.smoothing, op.v);
    const uint32_t i = a.sorted_index[p.s];
    a.out_velocities.x[i] = out.x;
    a.out_velocities.y[i] = out.y;
    a.out_velocities.z[i] = out.z;
}

// ------------------------------------------------------------------ constants
__global__ void constants_kernel(const float* __restrict__ radii, const uint32_t n, KernelConstants* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float h = radii[i];
    const float squared_radius = __fmul_rn(h, h);
    KernelConstants k;
    k.h = h;
    k.h2 = squared_radius;
    k.poly6_denominator = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(64.0F * kPi, squared_radius), squared_radius),
                                                                     squared_radius), h), h), h);
    k.poly6_grad_denominator = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(32.0F * kPi, squared_radius), squared_radius),
                                                                          squared_radius), h), h), h);
    k.spiky_coefficient = __fdiv_rn(-45.0F, __fmul_rn(kPi, powf(h, 6.0F)));
    // Smallest float r2 with sqrtf(r2) >= h; sqrtf is monotone, so bisect on the bit pattern.
    uint32_t lo = 0u, hi = 0x7f800000u;
    while (hi - lo > 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (sqrtf(__uint_as_float(mid)) >= h) hi = mid;
        else lo = mid;
    }
    k.spiky_threshold = __uint_as_float(hi);
    k.union_threshold = fmaxf(k.h2, k.spiky_threshold);
    // Smallest float r2 with sqrt((double)r2) >= h (the FP64 Hessian's support test).
    lo = 0u;
    hi = 0x7f800000u;
    while (hi - lo > 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (sqrt(static_cast<double>(__uint_as_float(mid))) >= static_cast<double>(h)) hi = mid;
        else lo = mid;
    }
    k.hessian_threshold = __uint_as_float(hi);
    k.adjoint_threshold = fmaxf(k.spiky_threshold, k.hessian_threshold);
    k.list_threshold = fmaxf(k.union_threshold, k.hessian_threshold);
    k.poly6_radial_coefficient = __fdiv_rn(315.0F, __fmul_rn(64.0F * kPi, powf(h, 9.0F)));
    k.spiky_coefficient_d = -45.0 / (static_cast<double>(kPi) * pow(static_cast<double>(h), 6.0));
    out[i] = k;
}

__global__ void unsort_float4_kernel(const uint32_t count, const uint32_t* __restrict__ sorted_index,
                                     const float4* __restrict__ in, const int components, float* out_x, float* out_y,
                                     float* out_z, float* out_w) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint32_t i = sorted_index[s];
    const float4 v = in[s];
    if (out_x) out_x[i] = v.x;
    if (components > 1 && out_y) out_y[i] = v.y;
    if (components > 2 && out_z) out_z[i] = v.z;
    if (out_w) out_w[i] = v.w;
}

__global__ void unsort_mask_kernel(const uint32_t count, const uint32_t* __restrict__ sorted_index,
                                   const uint8_t* __restrict__ in, uint32_t* __restrict__ out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    out[sorted_index[s]] = in[s];
}

__global__ void unsort_scalar_kernel(const uint32_t count, const uint32_t* __restrict__ sorted_index, const uint8_t* in,
                                     const uint32_t bytes, uint8_t* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint32_t i = sorted_index[s];
    for (uint32_t b = 0; b < bytes; ++b) out[static_cast<size_t>(i) * bytes + b] = in[static_cast<size_t>(s) * bytes + b];
}

__global__ void reconstruct_kernel(const uint32_t count, const SceneDesc* __restrict__ scenes, const int4* __restrict__ cell,
                                   const float4* __restrict__ positions, const Field3 previous,
                                   const uint32_t* __restrict__ sorted_index, const MutField3 out, float4* __restrict__ velocity) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const SceneDesc& sc = scenes[cell[s].w];
    const uint32_t i = sorted_index[s];
    const f3 x = xyz(positions[s]);
    const f3 v = scale(sub(x, mk(previous.x[i], previous.y[i], previous.z[i])), sc.inverse_time_step);
    velocity[s] = make_float4(v.x, v.y, v.z, 0.0F);
    out.x[i] = x.x;
    out.y[i] = x.y;
    out.z[i] = x.z;
}

inline unsigned grid_of(const uint32_t n, const unsigned block) { return (n + block - 1) / block; }

// Headless frame export (the example's Spectra write_vectors kernel and vorticity copy): xyz
// triples of the state and the step's vorticity magnitudes in original particle order.
__global__ void export_frame_kernel(const uint32_t count, const Field3 positions, const Field3 velocities,
                                    const uint32_t* __restrict__ slot_of, const float4* __restrict__ vorticity,
                                    float* __restrict__ out_positions, float* __restrict__ out_velocities,
                                    float* __restrict__ out_vorticity) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    out_positions[3u * i] = positions.x[i];
    out_positions[3u * i + 1u] = positions.y[i];
    out_positions[3u * i + 2u] = positions.z[i];
    out_velocities[3u * i] = velocities.x[i];
    out_velocities[3u * i + 1u] = velocities.y[i];
    out_velocities[3u * i + 2u] = velocities.z[i];
    if (out_vorticity) out_vorticity[i] = vorticity[slot_of[i]].w;
}

}  // namespace

cudaError_t launch_export_frame(cudaStream_t stream, const uint32_t count, const Field3 positions, const Field3 velocities,
                                const uint32_t* slot_of, const float4* vorticity, float* out_positions, float* out_velocities,
                                float* out_vorticity) {
    if (count == 0) return cudaSuccess;
    export_frame_kernel<<<grid_of(count, 256), 256, 0, stream>>>(count, positions, velocities, slot_of, vorticity, out_positions,
                                                                  out_velocities, out_vorticity);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_constants(cudaStream_t stream, const float* radii, const uint32_t n, KernelConstants* out) {
    constants_kernel<<<grid_of(n, 64), 64, 0, stream>>>(radii, n, out);
    count_launch();
    return cudaGetLastError();
}

bool valid_shape(const LaunchShape& shape) {
    auto ok = [](const uint32_t b) { return b >= 32u && b <= static_cast<uint32_t>(kBlock) && b % 32u == 0u; };
    return (shape.scan == kScanPerLane || shape.scan == kScanCooperative || shape.scan == kScanStaged ||
            shape.scan == kScanFusedDensity || shape.scan == kScanFusedMasks) &&
           ok(shape.scan_block) && ok(shape.block);
}

bool fuses_density(const LaunchShape& shape, const ListScanArgs& a) {
    return (shape.scan == kScanFusedDensity || shape.scan == kScanFusedMasks) && a.packed.x && !a.g.boundary &&
           !a.g.boundary_offsets;
}

bool stores_masks(const LaunchShape& shape, const bool differentiable, const bool boundary) {
    return shape.scan == kScanFusedMasks && !differentiable && !boundary;
}

namespace {
unsigned block_of(const unsigned block) {
    return block >= 32u && block <= static_cast<unsigned>(kBlock) && block % 32u == 0u ? block : static_cast<unsigned>(kBlock);
}
}  // namespace

cudaError_t launch_list_scan(cudaStream_t stream, const ListScanArgs& a, const LaunchShape& shape) {
    if (a.g.count == 0) return cudaSuccess;
    const unsigned block = block_of(shape.scan_block);
    // the cooperative and staged scans list fluid particles only; lists with boundary particles
    // use the per-lane walk
    const bool fluid_only = !(a.boundary && a.g.boundary_offsets);
    if (a.list.masks) {   // hit-mask lists: the per-lane packed walk, scenes without boundary particles
        if (!fluid_only || !a.packed.x) return cudaErrorInvalidValue;
        list_walk_kernel<true><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    } else if (shape.scan == kScanCooperative && fluid_only)
        list_scan_kernel<<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    else if (shape.scan == kScanStaged && fluid_only)
        list_staged_kernel<<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    else
        list_walk_kernel<false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scan_density_lambda(cudaStream_t stream, const ListScanArgs& a, const DensityLambdaArgs& d,
                                       const LaunchShape& shape) {
    if (a.g.count == 0) return cudaSuccess;
    const unsigned block = block_of(shape.scan_block);
    if (a.list.masks)
        scan_density_lambda_kernel<true><<<grid_of(a.g.count, block), block, 0, stream>>>(a, d);
    else
        scan_density_lambda_kernel<false><<<grid_of(a.g.count, block), block, 0, stream>>>(a, d);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_density_lambda(cudaStream_t stream, const DensityLambdaArgs& a, const unsigned block_size) {
    if (a.g.count == 0) return cudaSuccess;
    if (a.list.masks) return cudaErrorInvalidValue;   // hit-mask lists are read by the fused scan only
    const unsigned block = block_of(block_size);
    if (a.g.boundary)
        density_lambda_kernel<true><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    else
        density_lambda_kernel<false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_correction(cudaStream_t stream, const CorrectionArgs& a, const unsigned block_size) {
    if (a.g.count == 0) return cudaSuccess;
    const unsigned block = block_of(block_size);
    if (a.g.boundary) {
        if (a.list.masks) return cudaErrorInvalidValue;
        correction_kernel<true, false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    } else if (a.list.masks) {
        correction_kernel<false, true><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    } else {
        correction_kernel<false, false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_vorticity(cudaStream_t stream, const VorticityArgs& a, const unsigned block_size) {
    if (a.g.count == 0) return cudaSuccess;
    const unsigned block = block_of(block_size);
    if (a.list.masks)
        vorticity_kernel<true><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    else
        vorticity_kernel<false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_normal(cudaStream_t stream, const NormalArgs& a, const unsigned block_size) {
    if (a.g.count == 0) return cudaSuccess;
    const unsigned block = block_of(block_size);
    if (a.list.masks)
        normal_kernel<true><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    else
        normal_kernel<false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_xsph(cudaStream_t stream, const XsphArgs& a, const unsigned block_size) {
    if (a.g.count == 0) return cudaSuccess;
    const unsigned block = block_of(block_size);
    if (a.list.masks)
        xsph_kernel<true><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    else
        xsph_kernel<false><<<grid_of(a.g.count, block), block, 0, stream>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_reconstruct(cudaStream_t stream, const uint32_t count, const SceneDesc* scenes, const int4* cell,
                               const float4* positions, const Field3 previous_positions, const uint32_t* sorted_index,
                               const MutField3 out_positions, float4* velocity) {
    if (count == 0) return cudaSuccess;
    reconstruct_kernel<<<grid_of(count, 256), 256, 0, stream>>>(count, scenes, cell, positions, previous_positions, sorted_index,
                                                               out_positions, velocity);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_unsort_float4(cudaStream_t stream, const uint32_t count, const uint32_t* sorted_index, const float4* in,
                                 const int components, float* out_x, float* out_y, float* out_z, float* out_w) {
    if (count == 0) return cudaSuccess;
    unsort_float4_kernel<<<grid_of(count, 256), 256, 0, stream>>>(count, sorted_index, in, components, out_x, out_y, out_z, out_w);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_unsort_mask(cudaStream_t stream, const uint32_t count, const uint32_t* sorted_index, const uint8_t* in,
                               uint32_t* out) {
    if (count == 0) return cudaSuccess;
    unsort_mask_kernel<<<grid_of(count, 256), 256, 0, stream>>>(count, sorted_index, in, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_unsort_scalar(cudaStream_t stream, const uint32_t count, const uint32_t* sorted_index, const void* in,
                                 const uint32_t bytes, void* out) {
    if (count == 0) return cudaSuccess;
    unsort_scalar_kernel<<<grid_of(count, 256), 256, 0, stream>>>(count, sorted_index, static_cast<const uint8_t*>(in), bytes,
                                                                 static_cast<uint8_t*>(out));
    count_launch();
    return cudaGetLastError();
}

}  // namespace pbf
