/*
 * FP64 host oracle for the PBF substep -- TEST INFRASTRUCTURE ONLY (see pbf_oracle.h).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
 * library, and only as the checker / baseline; the CUDA solver never calls it.
 *
 * Everything here is double precision except the two functions that restate the
 * reference's FP32 integer work (grid keys and neighbour counts).  Passes loop over
 * particles with OpenMP; neighbours are visited in the reference order: stencil
 * cells x-outer, y, z-inner (pbf/pbf.cu:105-110), particles of a cell in ascending
 * original index (stable sort, neighborhood/neighborhood.cu:57).
 */
#include "pbf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The reference's pi is a float constant (density/device.cuh:8); its value is kept here. */
static const double PI_REF = (double)3.14159265358979323846f;

typedef struct { double x, y, z; } d3;

static inline d3 v3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 add3(d3 a, d3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 sub3(d3 a, d3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 mul3(d3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross3(d3 a, d3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double len3(d3 a) { return sqrt(dot3(a, a)); }
static inline d3 ld(oracle_vec v, uint32_t i) { return v3(v.x[i], v.y[i], v.z[i]); }
static inline void st(oracle_vec v, uint32_t i, d3 a) { v.x[i] = a.x; v.y[i] = a.y; v.z[i] = a.z; }
static inline void acc(oracle_vec v, uint32_t i, d3 a) { v.x[i] += a.x; v.y[i] += a.y; v.z[i] += a.z; }

int oracle_thread_count(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------- kernels */
/* poly6 and its gradient: density/device.cuh:10-24. */
double oracle_poly6(double dx, double dy, double dz, double h) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double h2 = h * h;
    if (r2 >= h2) return 0.0;
    const double d = h2 - r2;
    return 315.0 * d * d * d / (64.0 * PI_REF * h2 * h2 * h2 * h * h * h);
}

static d3 poly6_gradient(d3 d, double h) {
    const double r2 = dot3(d, d);
    const double h2 = h * h;
    if (r2 >= h2) return v3(0, 0, 0);
    const double q = h2 - r2;
    return mul3(d, -945.0 * q * q / (32.0 * PI_REF * h2 * h2 * h2 * h * h * h));
}

/* d/dr of poly6 along a radius: pbf/pbf.cu:18-24. */
static double poly6_radial_derivative(double r, double h) {
    if (r >= h) return 0.0;
    const double q = h * h - r * r;
    return -6.0 * (315.0 / (64.0 * PI_REF * pow(h, 9.0))) * r * q * q;
}

/* Spiky gradient and its Hessian-vector product: pbf/pbf.cu:26-54. */
static d3 spiky_gradient(d3 d, double h) {
    const double r = len3(d);
    if (r == 0.0 || r >= h) return v3(0, 0, 0);
    const double q = h - r;
    return mul3(d, (-45.0 / (PI_REF * pow(h, 6.0))) * q * q / r);
}

void oracle_spiky_gradient(double dx, double dy, double dz, double h, double out[3]) {
    d3 g = spiky_gradient(v3(dx, dy, dz), h);
    out[0] = g.x; out[1] = g.y; out[2] = g.z;
}

static d3 spiky_hessian_product(d3 d, d3 v, double h) {
    const double r = len3(d);
    if (r == 0.0 || r >= h) return v3(0, 0, 0);
    const d3 u = mul3(d, 1.0 / r);
    const double p = dot3(u, v);
    const d3 ut = mul3(sub3(v, mul3(u, p)), 1.0 / r);
    const double q = h - r;
    const double k = -45.0 / (PI_REF * pow(h, 6.0));
    return mul3(add3(mul3(u, -2.0 * q * p), mul3(ut, q * q)), k);
}

/* s_corr = -k (W(d)/W(dq))^n and its derivatives: pbf/pbf.cu:56-71. */
typedef struct { double value; d3 gradient; double d_strength, d_exponent, d_radius; } scorr;

static scorr artificial_pressure(d3 d, double h, double k, double n, double dq) {
    scorr s; memset(&s, 0, sizeof s);
    const double ref = oracle_poly6(dq, 0.0, 0.0, h);
    const double w = oracle_poly6(d.x, d.y, d.z, h);
    if (w == 0.0) return s;
    const double ratio = w / ref;
    const double power = pow(ratio, n);
    s.value = -k * power;
    s.d_strength = -power;
    s.d_exponent = s.value * log(ratio);
    s.d_radius = -s.value * n * poly6_radial_derivative(dq, h) / ref;
    s.gradient = mul3(poly6_gradient(d, h), -k * n * pow(ratio, n - 1.0) / ref);
    return s;
}

/* ------------------------------------------------------------------- grid */
int oracle_grid_dims(const float box_min[3], const float box_max[3], float h, uint32_t dims[3]) {
    for (int a = 0; a < 3; ++a) {
        const float extent = box_max[a] - box_min[a];
        const float cells = ceilf(extent / h);
        if (!(cells >= 1.0f) || cells > 4294967295.0f) return 1;
        dims[a] = (uint32_t)cells;
    }
    return 0;
}

/* Device __float2int_rd: round toward -inf, saturating, NaN -> 0. */
static int f2i_rd(float q) {
    if (q != q) return 0;
    const float f = floorf(q);
    if (f >= 2147483648.0f) return 2147483647;
    if (f < -2147483648.0f) return (-2147483647 - 1);
    return (int)f;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

typedef struct {
    uint32_t dims[3];
    uint64_t cells;
    uint32_t* offsets;   /* cells + 1 */
    uint32_t* sorted;    /* count */
    int* cell_of;        /* 3 * count: gather cell of each particle */
} grid;

static void grid_free(grid* g) { free(g->offsets); free(g->sorted); free(g->cell_of); memset(g, 0, sizeof *g); }

/* Stable counting sort of particle indices by cell key. */
static int grid_sort(grid* g, uint32_t count, const uint64_t* keys) {
    g->offsets = (uint32_t*)calloc(g->cells + 1, sizeof(uint32_t));
    g->sorted = (uint32_t*)malloc((size_t)(count ? count : 1) * sizeof(uint32_t));
    if (!g->offsets || !g->sorted) return 2;
    for (uint32_t i = 0; i < count; ++i) g->offsets[keys[i] + 1]++;
    for (uint64_t c = 0; c < g->cells; ++c) g->offsets[c + 1] += g->offsets[c];
    uint32_t* fill = (uint32_t*)malloc((size_t)(g->cells ? g->cells : 1) * sizeof(uint32_t));
    if (!fill) return 2;
    memcpy(fill, g->offsets, (size_t)g->cells * sizeof(uint32_t));
    for (uint32_t i = 0; i < count; ++i) g->sorted[fill[keys[i]]++] = i;
    free(fill);
    return 0;
}

int oracle_grid_f32(uint32_t count, const float* x, const float* y, const float* z, float h,
                    const float box_min[3], const float box_max[3], const float box_velocity[3], float time,
                    uint32_t* keys, uint32_t* sorted_indices, uint32_t* cell_offsets) {
    uint32_t dims[3];
    if (oracle_grid_dims(box_min, box_max, h, dims)) return 1;
    const uint64_t cells = (uint64_t)dims[0] * dims[1] * dims[2];
    uint64_t* k64 = (uint64_t*)malloc((size_t)(count ? count : 1) * sizeof(uint64_t));
    if (!k64) return 2;
    const float* p[3] = {x, y, z};
    for (uint32_t i = 0; i < count; ++i) {
        int c[3];
        for (int a = 0; a < 3; ++a) {
            /* (p - min - time*vel)/h with the device's fused multiply-add of time*vel */
            const float shifted = fmaf(-time, box_velocity[a], p[a][i] - box_min[a]);
            c[a] = clampi(f2i_rd(shifted / h), 0, (int)dims[a] - 1);
            if (c[a] < 0) c[a] = 0;
        }
        k64[i] = ((uint64_t)c[2] * dims[1] + (uint64_t)c[1]) * dims[0] + (uint64_t)c[0];
        if (keys) keys[i] = (uint32_t)k64[i];
    }
    grid g; memset(&g, 0, sizeof g);
    g.cells = cells;
    int rc = grid_sort(&g, count, k64);
    if (!rc) {
        if (sorted_indices) memcpy(sorted_indices, g.sorted, (size_t)count * sizeof(uint32_t));
        if (cell_offsets) memcpy(cell_offsets, g.offsets, (size_t)(cells + 1) * sizeof(uint32_t));
    }
    grid_free(&g);
    free(k64);
    return rc;
}

/* FP32 squared distance with the device's contraction: fma(z,z, fma(x,x, y*y)). */
static inline float r2_f32(float dx, float dy, float dz) { return fmaf(dz, dz, fmaf(dx, dx, dy * dy)); }

int oracle_neighbor_counts_f32(uint32_t count, const float* const topology[3], const float* const position[3],
                               float h, const float box_min[3], const float box_max[3],
                               const float box_velocity[3], float time, uint32_t* counts) {
    uint32_t dims[3];
    if (oracle_grid_dims(box_min, box_max, h, dims)) return 1;
    const uint64_t cells = (uint64_t)dims[0] * dims[1] * dims[2];
    uint32_t* offsets = (uint32_t*)malloc((size_t)(cells + 1) * sizeof(uint32_t));
    uint32_t* sorted = (uint32_t*)malloc((size_t)(count ? count : 1) * sizeof(uint32_t));
    if (!offsets || !sorted) { free(offsets); free(sorted); return 2; }
    int rc = oracle_grid_f32(count, topology[0], topology[1], topology[2], h, box_min, box_max, box_velocity, time,
                             NULL, sorted, offsets);
    const float h2 = h * h;
    float origin[3];
    for (int a = 0; a < 3; ++a) origin[a] = box_min[a] + time * box_velocity[a];
    if (!rc) {
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)count; ++ii) {
            const uint32_t i = (uint32_t)ii;
            int c[3];
            for (int a = 0; a < 3; ++a) c[a] = clampi(f2i_rd((topology[a][i] - origin[a]) / h), 0, (int)dims[a] - 1);
            uint32_t n = 0;
            for (int ox = -1; ox <= 1; ++ox)
                for (int oy = -1; oy <= 1; ++oy)
                    for (int oz = -1; oz <= 1; ++oz) {
                        const int cx = c[0] + ox, cy = c[1] + oy, cz = c[2] + oz;
                        if (cx < 0 || cy < 0 || cz < 0 || cx >= (int)dims[0] || cy >= (int)dims[1] || cz >= (int)dims[2]) continue;
                        const uint64_t cell = ((uint64_t)cz * dims[1] + (uint64_t)cy) * dims[0] + (uint64_t)cx;
                        for (uint32_t s = offsets[cell]; s < offsets[cell + 1]; ++s) {
                            const uint32_t j = sorted[s];
                            if (j == i) continue;
                            const float dx = position[0][i] - position[0][j];
                            const float dy = position[1][i] - position[1][j];
                            const float dz = position[2][i] - position[2][j];
                            if (r2_f32(dx, dy, dz) < h2) ++n;
                        }
                    }
            counts[i] = n;
        }
    }
    free(offsets);
    free(sorted);
    return rc;
}

/* ------------------------------------------------------- the FP64 substep */
typedef struct {
    const oracle_scene* sc;
    const oracle_parameters* p;
    uint32_t n;
    double h, dt;
    float time;                 /* (step_index + 1) * dt, in float as the reference */
    double box_lo[3], box_hi[3];
    grid g;
    /* boundary particles */
    grid bg;
    double* bx[3];              /* boundary positions at `time` */
    /* per-particle gather cell */
} context;

static int context_init(context* ctx, const oracle_scene* sc, const oracle_parameters* p, oracle_vec topology) {
    memset(ctx, 0, sizeof *ctx);
    ctx->sc = sc; ctx->p = p; ctx->n = sc->count;
    ctx->h = sc->support_radius; ctx->dt = sc->time_step;
    ctx->time = (float)(sc->step_index + 1u) * sc->time_step;
    /* collision box: pbf/pbf.cpp:17-31 (float arithmetic) */
    for (int a = 0; a < 3; ++a) {
        ctx->box_lo[a] = (double)(sc->box_min[a] + ctx->time * sc->box_velocity[a] + sc->particle_radius);
        ctx->box_hi[a] = (double)(sc->box_max[a] + ctx->time * sc->box_velocity[a] - sc->particle_radius);
    }
    if (oracle_grid_dims(sc->box_min, sc->box_max, sc->support_radius, ctx->g.dims)) return 1;
    ctx->g.cells = (uint64_t)ctx->g.dims[0] * ctx->g.dims[1] * ctx->g.dims[2];
    const uint32_t n = ctx->n;
    uint64_t* keys = (uint64_t*)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    ctx->g.cell_of = (int*)malloc((size_t)(n ? n : 1) * 3 * sizeof(int));
    if (!keys || !ctx->g.cell_of) return 2;
    double origin[3];
    for (int a = 0; a < 3; ++a) origin[a] = (double)(sc->box_min[a] + ctx->time * sc->box_velocity[a]);
    const double* tp[3] = {topology.x, topology.y, topology.z};
    for (uint32_t i = 0; i < n; ++i) {
        int kc[3];
        for (int a = 0; a < 3; ++a) {
            const double q = (tp[a][i] - sc->box_min[a] - (double)ctx->time * sc->box_velocity[a]) / ctx->h;
            kc[a] = clampi(q >= 2147483647.0 ? 2147483647 : (q < -2147483648.0 ? (-2147483647 - 1) : (int)floor(q)), 0, (int)ctx->g.dims[a] - 1);
            const double qg = (tp[a][i] - origin[a]) / ctx->h;
            ctx->g.cell_of[3 * i + a] = clampi(qg >= 2147483647.0 ? 2147483647 : (qg < -2147483648.0 ? (-2147483647 - 1) : (int)floor(qg)), 0, (int)ctx->g.dims[a] - 1);
        }
        keys[i] = ((uint64_t)kc[2] * ctx->g.dims[1] + (uint64_t)kc[1]) * ctx->g.dims[0] + (uint64_t)kc[0];
    }
    int rc = grid_sort(&ctx->g, n, keys);
    free(keys);
    if (rc) return rc;
    /* boundary particles: moving positions p + time * v, sorted on the same grid */
    const uint32_t nb = sc->boundary_count;
    ctx->bg.dims[0] = ctx->g.dims[0]; ctx->bg.dims[1] = ctx->g.dims[1]; ctx->bg.dims[2] = ctx->g.dims[2];
    ctx->bg.cells = ctx->g.cells;
    uint64_t* bkeys = (uint64_t*)malloc((size_t)(nb ? nb : 1) * sizeof(uint64_t));
    for (int a = 0; a < 3; ++a) ctx->bx[a] = (double*)malloc((size_t)(nb ? nb : 1) * sizeof(double));
    if (!bkeys || !ctx->bx[0] || !ctx->bx[1] || !ctx->bx[2]) return 2;
    for (uint32_t b = 0; b < nb; ++b) {
        int kc[3];
        for (int a = 0; a < 3; ++a) {
            const double pa = sc->boundary_position[a][b] + (double)ctx->time * sc->boundary_velocity[a][b];
            ctx->bx[a][b] = pa;
            const double q = (pa - sc->box_min[a] - (double)ctx->time * sc->box_velocity[a]) / ctx->h;
            kc[a] = clampi(q >= 2147483647.0 ? 2147483647 : (q < -2147483648.0 ? (-2147483647 - 1) : (int)floor(q)), 0, (int)ctx->g.dims[a] - 1);
        }
        bkeys[b] = ((uint64_t)kc[2] * ctx->g.dims[1] + (uint64_t)kc[1]) * ctx->g.dims[0] + (uint64_t)kc[0];
    }
    rc = grid_sort(&ctx->bg, nb, bkeys);
    free(bkeys);
    return rc;
}

static void context_free(context* ctx) {
    grid_free(&ctx->g);
    grid_free(&ctx->bg);
    for (int a = 0; a < 3; ++a) free(ctx->bx[a]);
}

/* Visit the 27 stencil cells of particle i in reference order: x offset outer, z inner.
   The macro opens a block that the caller closes. */
#define STENCIL_BEGIN(ctx, i, CELLVAR)                                                                   \
    for (int o_ = 0; o_ < 27; ++o_) {                                                                    \
        uint64_t CELLVAR;                                                                                \
        if (!stencil_cell(ctx, i, o_ / 9 - 1, (o_ / 3) % 3 - 1, o_ % 3 - 1, &CELLVAR)) continue;

static inline int stencil_cell(const context* ctx, uint32_t i, int ox, int oy, int oz, uint64_t* cell) {
    const int cx = ctx->g.cell_of[3 * i] + ox, cy = ctx->g.cell_of[3 * i + 1] + oy, cz = ctx->g.cell_of[3 * i + 2] + oz;
    if (cx < 0 || cy < 0 || cz < 0 || cx >= (int)ctx->g.dims[0] || cy >= (int)ctx->g.dims[1] || cz >= (int)ctx->g.dims[2]) return 0;
    *cell = ((uint64_t)cz * ctx->g.dims[1] + (uint64_t)cy) * ctx->g.dims[0] + (uint64_t)cx;
    return 1;
}

static inline d3 bpos(const context* ctx, uint32_t b) { return v3(ctx->bx[0][b], ctx->bx[1][b], ctx->bx[2][b]); }

/* One Jacobi iteration's primal fields. */
typedef struct {
    double* density;
    d3* gsum;
    double* denom;
    double* lambda;
    d3* corr;
    uint32_t* mask;
} iteration;

static int iteration_alloc(iteration* it, uint32_t n) {
    const size_t m = n ? n : 1;
    it->density = (double*)malloc(m * sizeof(double));
    it->gsum = (d3*)malloc(m * sizeof(d3));
    it->denom = (double*)malloc(m * sizeof(double));
    it->lambda = (double*)malloc(m * sizeof(double));
    it->corr = (d3*)malloc(m * sizeof(d3));
    it->mask = (uint32_t*)malloc(m * sizeof(uint32_t));
    return (it->density && it->gsum && it->denom && it->lambda && it->corr && it->mask) ? 0 : 2;
}

static void iteration_free(iteration* it) {
    free(it->density); free(it->gsum); free(it->denom); free(it->lambda); free(it->corr); free(it->mask);
}

/* density (density/density.cu:18-40), lambda (pbf.cu:95-127), correction (pbf.cu:254-288),
   project (pbf.cu:417-431) of one iteration: x -> x_next. */
static void jacobi_iteration(const context* ctx, const d3* x, d3* x_next, iteration* it, uint32_t* ncount) {
    const oracle_parameters* p = ctx->p;
    const double h = ctx->h;
    const uint32_t n = ctx->n;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const double rho0 = p->rest_densities[i];
        double rho = 0.0;
        d3 s = v3(0, 0, 0);
        double denom = p->relaxation[i];
        uint32_t cnt = 0;
        STENCIL_BEGIN(ctx, i, cell)
            for (uint32_t q = ctx->g.offsets[cell]; q < ctx->g.offsets[cell + 1]; ++q) {
                const uint32_t j = ctx->g.sorted[q];
                const d3 d = sub3(x[i], x[j]);
                rho += p->masses[j] * oracle_poly6(d.x, d.y, d.z, h);
                if (j == i) continue;
                if (dot3(d, d) < h * h) ++cnt;
                const d3 g = spiky_gradient(d, h);
                const double c = p->masses[j] / rho0;
                s = add3(s, mul3(g, c));
                denom += c * c * dot3(g, g);
            }
            for (uint32_t q = ctx->bg.offsets[cell]; q < ctx->bg.offsets[cell + 1]; ++q) {
                const uint32_t b = ctx->bg.sorted[q];
                const d3 d = sub3(x[i], bpos(ctx, b));
                rho += rho0 * ctx->sc->boundary_volume[b] * oracle_poly6(d.x, d.y, d.z, h);
                s = add3(s, mul3(spiky_gradient(d, h), ctx->sc->boundary_volume[b]));
            }
        }
        denom += dot3(s, s);
        it->density[i] = rho;
        it->gsum[i] = s;
        it->denom[i] = denom;
        it->lambda[i] = -(rho / rho0 - 1.0) / denom;
        if (ncount) ncount[i] = cnt;
    }
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const double rho0 = p->rest_densities[i];
        const double k = p->artificial_pressure_strength[i], ex = p->artificial_pressure_exponent[i], dq = p->artificial_pressure_radius[i];
        d3 corr = v3(0, 0, 0);
        STENCIL_BEGIN(ctx, i, cell)
            for (uint32_t q = ctx->g.offsets[cell]; q < ctx->g.offsets[cell + 1]; ++q) {
                const uint32_t j = ctx->g.sorted[q];
                if (j == i) continue;
                const d3 d = sub3(x[i], x[j]);
                const scorr sc = artificial_pressure(d, h, k, ex, dq);
                const double c = p->masses[j] / rho0;
                corr = add3(corr, mul3(spiky_gradient(d, h), c * (it->lambda[i] + it->lambda[j] + sc.value)));
            }
            for (uint32_t q = ctx->bg.offsets[cell]; q < ctx->bg.offsets[cell + 1]; ++q) {
                const uint32_t b = ctx->bg.sorted[q];
                const d3 d = sub3(x[i], bpos(ctx, b));
                const scorr sc = artificial_pressure(d, h, k, ex, dq);
                corr = add3(corr, mul3(spiky_gradient(d, h), ctx->sc->boundary_volume[b] * (it->lambda[i] + sc.value)));
            }
        }
        it->corr[i] = corr;
        const d3 cand = add3(x[i], corr);
        const double cv[3] = {cand.x, cand.y, cand.z};
        double out[3];
        uint32_t mask = 0;
        for (int a = 0; a < 3; ++a) {
            if (cv[a] < ctx->box_lo[a] || cv[a] > ctx->box_hi[a]) mask |= 1u << a;
            out[a] = fmin(ctx->box_hi[a], fmax(ctx->box_lo[a], cv[a]));
        }
        it->mask[i] = mask;
        x_next[i] = v3(out[0], out[1], out[2]);
    }
}

typedef struct {
    d3* xs;          /* predicted */
    d3** xk;         /* K + 1 position iterates */
    iteration* it;   /* K iterations */
    d3* vr;          /* reconstructed velocities */
    d3* w;           /* vorticities */
    double* wm;      /* |w| */
    d3* nrm;         /* normals */
    double* nz;      /* normalizers */
    d3* vc;          /* confined velocities */
    d3* vout;
} forward_record;

static void record_free(forward_record* r, uint32_t K) {
    free(r->xs);
    if (r->xk) for (uint32_t k = 0; k <= K; ++k) free(r->xk[k]);
    free(r->xk);
    if (r->it) for (uint32_t k = 0; k < K; ++k) iteration_free(&r->it[k]);
    free(r->it);
    free(r->vr); free(r->w); free(r->wm); free(r->nrm); free(r->nz); free(r->vc); free(r->vout);
}

static int forward(const oracle_scene* sc, const oracle_parameters* p, oracle_vec x0, oracle_vec v0, oracle_vec a0,
                   context* ctx, forward_record* r, oracle_trace* trace) {
    const uint32_t n = sc->count, K = sc->iterations;
    const size_t m = n ? n : 1;
    memset(r, 0, sizeof *r);
    r->xs = (d3*)malloc(m * sizeof(d3));
    r->xk = (d3**)calloc(K + 1, sizeof(d3*));
    r->it = (iteration*)calloc(K ? K : 1, sizeof(iteration));
    r->vr = (d3*)malloc(m * sizeof(d3)); r->w = (d3*)malloc(m * sizeof(d3)); r->wm = (double*)malloc(m * sizeof(double));
    r->nrm = (d3*)malloc(m * sizeof(d3)); r->nz = (double*)malloc(m * sizeof(double)); r->vc = (d3*)malloc(m * sizeof(d3));
    r->vout = (d3*)malloc(m * sizeof(d3));
    if (!r->xs || !r->xk || !r->it || !r->vr || !r->w || !r->wm || !r->nrm || !r->nz || !r->vc || !r->vout) return 2;
    for (uint32_t k = 0; k <= K; ++k) { r->xk[k] = (d3*)malloc(m * sizeof(d3)); if (!r->xk[k]) return 2; }
    for (uint32_t k = 0; k < K; ++k) if (iteration_alloc(&r->it[k], n)) return 2;
    const double dt = sc->time_step;
    const d3 g = v3(sc->gravity[0], sc->gravity[1], sc->gravity[2]);
    /* predict: pbf.cu:73-78 */
    for (uint32_t i = 0; i < n; ++i) {
        const d3 vp = add3(ld(v0, i), mul3(add3(g, ld(a0, i)), dt));
        r->xs[i] = add3(ld(x0, i), mul3(vp, dt));
    }
    oracle_vec topo;
    double* tp = (double*)malloc(3 * m * sizeof(double));
    if (!tp) return 2;
    topo.x = tp; topo.y = tp + m; topo.z = tp + 2 * m;
    for (uint32_t i = 0; i < n; ++i) st(topo, i, r->xs[i]);
    int rc = context_init(ctx, sc, p, topo);
    free(tp);
    if (rc) return rc;
    memcpy(r->xk[0], r->xs, n * sizeof(d3));
    for (uint32_t k = 0; k < K; ++k)
        jacobi_iteration(ctx, r->xk[k], r->xk[k + 1], &r->it[k], (k == 0 && trace) ? trace->neighbor_count0 : NULL);
    const d3* xc = r->xk[K];
    const double h = ctx->h;
    /* reconstruct: pbf.cu:456-460 */
    for (uint32_t i = 0; i < n; ++i) r->vr[i] = mul3(sub3(xc[i], ld(x0, i)), 1.0 / dt);
    /* vorticity: pbf.cu:476-497 */
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        d3 w = v3(0, 0, 0);
        STENCIL_BEGIN(ctx, i, cell)
            for (uint32_t q = ctx->g.offsets[cell]; q < ctx->g.offsets[cell + 1]; ++q) {
                const uint32_t j = ctx->g.sorted[q];
                if (j == i) continue;
                w = add3(w, cross3(sub3(r->vr[j], r->vr[i]), spiky_gradient(sub3(xc[i], xc[j]), h)));
            }
        }
        r->w[i] = w;
        r->wm[i] = len3(w);
    }
    /* normal + confinement: pbf.cu:565-593, 674-678 */
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        d3 eta = v3(0, 0, 0);
        STENCIL_BEGIN(ctx, i, cell)
            for (uint32_t q = ctx->g.offsets[cell]; q < ctx->g.offsets[cell + 1]; ++q) {
                const uint32_t j = ctx->g.sorted[q];
                if (j == i) continue;
                eta = add3(eta, mul3(spiky_gradient(sub3(xc[i], xc[j]), h), r->wm[j] - r->wm[i]));
            }
        }
        const double nz = len3(eta);
        r->nz[i] = nz;
        r->nrm[i] = nz > 0.0 ? mul3(eta, 1.0 / nz) : v3(0, 0, 0);
        r->vc[i] = add3(r->vr[i], mul3(cross3(r->nrm[i], r->w[i]), dt * p->vorticity_confinement[i]));
    }
    /* XSPH: pbf.cu:700-721 */
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        d3 sm = v3(0, 0, 0);
        STENCIL_BEGIN(ctx, i, cell)
            for (uint32_t q = ctx->g.offsets[cell]; q < ctx->g.offsets[cell + 1]; ++q) {
                const uint32_t j = ctx->g.sorted[q];
                if (j == i) continue;
                const d3 d = sub3(xc[i], xc[j]);
                sm = add3(sm, mul3(sub3(r->vc[j], r->vc[i]), oracle_poly6(d.x, d.y, d.z, h)));
            }
        }
        r->vout[i] = add3(r->vc[i], mul3(sm, p->xsph_viscosity[i]));
    }
    if (trace) {
        for (uint32_t i = 0; i < n; ++i) {
            if (trace->predicted.x) st(trace->predicted, i, r->xs[i]);
            if (trace->density0 && K) trace->density0[i] = r->it[0].density[i];
            if (trace->lambda0 && K) trace->lambda0[i] = r->it[0].lambda[i];
            if (trace->corrected.x) st(trace->corrected, i, xc[i]);
            if (trace->vorticity.x) st(trace->vorticity, i, r->w[i]);
            if (trace->confined_velocity.x) st(trace->confined_velocity, i, r->vc[i]);
        }
    }
    return 0;
}

int oracle_forward_step(const oracle_scene* sc, const oracle_parameters* p, oracle_vec x0, oracle_vec v0, oracle_vec a0,
                        oracle_vec x1, oracle_vec v1, oracle_trace* trace) {
    if (!sc || !p) return 1;
    context ctx;
    forward_record r;
    int rc = forward(sc, p, x0, v0, a0, &ctx, &r, trace);
    if (!rc) {
        const d3* xc = r.xk[sc->iterations];
        for (uint32_t i = 0; i < sc->count; ++i) { st(x1, i, xc[i]); st(v1, i, r.vout[i]); }
    }
    context_free(&ctx);
    record_free(&r, sc->iterations);
    return rc;
}

/* ----------------------------------------------------------- the adjoint */
static inline d3 nrm_adj(d3 nrm, double nz, d3 nbar) {
    if (nz == 0.0) return v3(0, 0, 0);
    return mul3(add3(nbar, mul3(nrm, -dot3(nbar, nrm))), 1.0 / nz);
}

#define PADJ(ptr, i, val) do { if (ptr) (ptr)[i] += (val); } while (0)

int oracle_vjp_step(const oracle_scene* sc, const oracle_parameters* p, oracle_vec x0, oracle_vec v0, oracle_vec a0,
                    oracle_adjoint* adj) {
    if (!sc || !p || !adj) return 1;
    const uint32_t n = sc->count, K = sc->iterations;
    const size_t m = n ? n : 1;
    context ctx;
    forward_record r;
    int rc = forward(sc, p, x0, v0, a0, &ctx, &r, NULL);
    if (rc) { context_free(&ctx); record_free(&r, K); return rc; }
    const double h = ctx.h, dt = sc->time_step;
    d3* xbar = (d3*)calloc(m, sizeof(d3));       /* adjoint of the current position iterate */
    d3* xbar_next = (d3*)calloc(m, sizeof(d3));
    d3* vcbar = (d3*)calloc(m, sizeof(d3));      /* confined velocity */
    d3* vrbar = (d3*)calloc(m, sizeof(d3));      /* reconstructed velocity */
    d3* wbar = (d3*)calloc(m, sizeof(d3));
    d3* nbar = (d3*)calloc(m, sizeof(d3));
    d3* cbar = (d3*)calloc(m, sizeof(d3));       /* correction */
    double* lbar = (double*)calloc(m, sizeof(double));
    double* rbar = (double*)calloc(m, sizeof(double));
    d3* etabar = (d3*)calloc(m, sizeof(d3));
    if (!xbar || !xbar_next || !vcbar || !vrbar || !wbar || !nbar || !cbar || !lbar || !rbar || !etabar) rc = 2;
    const d3* xc = r.xk[K];
    if (!rc) {
        for (uint32_t i = 0; i < n; ++i) xbar[i] = ld(adj->next_position, i);
        /* XSPH VJP: pbf.cu:756-790 */
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            const d3 ob = ld(adj->next_velocity, i);
            const double ci = p->xsph_viscosity[i];
            d3 px = v3(0, 0, 0), pv = ob;
            double pc = 0.0;
            STENCIL_BEGIN(&ctx, i, cell)
                for (uint32_t q = ctx.g.offsets[cell]; q < ctx.g.offsets[cell + 1]; ++q) {
                    const uint32_t j = ctx.g.sorted[q];
                    if (j == i) continue;
                    const d3 d = sub3(xc[i], xc[j]);
                    const d3 diff = sub3(r.vc[j], r.vc[i]);
                    const double wgt = oracle_poly6(d.x, d.y, d.z, h);
                    pv = add3(pv, mul3(ob, -ci * wgt));
                    px = add3(px, mul3(poly6_gradient(d, h), ci * dot3(ob, diff)));
                    pc += wgt * dot3(ob, diff);
                    const d3 obj = ld(adj->next_velocity, j);
                    const double cj = p->xsph_viscosity[j];
                    pv = add3(pv, mul3(obj, cj * wgt));
                    px = add3(px, mul3(poly6_gradient(mul3(d, -1.0), h), -cj * dot3(obj, mul3(diff, -1.0))));
                }
            }
            xbar[i] = add3(xbar[i], px);
            vcbar[i] = pv;
            PADJ(adj->xsph_viscosity, i, pc);
        }
        /* confinement VJP: pbf.cu:688-698 */
        for (uint32_t i = 0; i < n; ++i) {
            const double e = dt * p->vorticity_confinement[i];
            vrbar[i] = vcbar[i];
            wbar[i] = mul3(cross3(vcbar[i], r.nrm[i]), e);
            nbar[i] = mul3(cross3(r.w[i], vcbar[i]), e);
            PADJ(adj->vorticity_confinement, i, dt * dot3(vcbar[i], cross3(r.nrm[i], r.w[i])));
        }
        /* normal VJP: pbf.cu:633-672 */
        for (uint32_t i = 0; i < n; ++i) etabar[i] = nrm_adj(r.nrm[i], r.nz[i], nbar[i]);
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            d3 px = v3(0, 0, 0);
            double mbar = 0.0;
            STENCIL_BEGIN(&ctx, i, cell)
                for (uint32_t q = ctx.g.offsets[cell]; q < ctx.g.offsets[cell + 1]; ++q) {
                    const uint32_t j = ctx.g.sorted[q];
                    if (j == i) continue;
                    const d3 d = sub3(xc[i], xc[j]);
                    const d3 gr = spiky_gradient(d, h);
                    px = add3(px, spiky_hessian_product(d, mul3(etabar[i], r.wm[j] - r.wm[i]), h));
                    mbar -= dot3(etabar[i], gr);
                    const d3 rd = mul3(d, -1.0);
                    px = add3(px, mul3(spiky_hessian_product(rd, mul3(etabar[j], r.wm[i] - r.wm[j]), h), -1.0));
                    mbar += dot3(etabar[j], spiky_gradient(rd, h));
                }
            }
            xbar[i] = add3(xbar[i], px);
            if (r.wm[i] > 0.0) wbar[i] = add3(wbar[i], mul3(r.w[i], mbar / r.wm[i]));
        }
        /* vorticity VJP: pbf.cu:528-563 */
#pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            d3 px = v3(0, 0, 0), pv = v3(0, 0, 0);
            STENCIL_BEGIN(&ctx, i, cell)
                for (uint32_t q = ctx.g.offsets[cell]; q < ctx.g.offsets[cell + 1]; ++q) {
                    const uint32_t j = ctx.g.sorted[q];
                    if (j == i) continue;
                    const d3 d = sub3(xc[i], xc[j]);
                    const d3 gr = spiky_gradient(d, h);
                    const d3 diff = sub3(r.vr[j], r.vr[i]);
                    pv = add3(pv, cross3(wbar[i], gr));
                    px = add3(px, spiky_hessian_product(d, cross3(wbar[i], diff), h));
                    const d3 rd = mul3(d, -1.0);
                    pv = add3(pv, cross3(spiky_gradient(rd, h), wbar[j]));
                    px = add3(px, mul3(spiky_hessian_product(rd, cross3(wbar[j], mul3(diff, -1.0)), h), -1.0));
                }
            }
            xbar[i] = add3(xbar[i], px);
            vrbar[i] = add3(vrbar[i], pv);
        }
        /* reconstruct VJP: pbf.cu:468-474 */
        for (uint32_t i = 0; i < n; ++i) {
            const d3 c = mul3(vrbar[i], 1.0 / dt);
            acc(adj->position, i, mul3(c, -1.0));
            xbar[i] = add3(xbar[i], c);
        }
        /* Jacobi iterations in reverse */
        for (uint32_t kk = K; kk-- > 0;) {
            const d3* x = r.xk[kk];
            const iteration* it = &r.it[kk];
            /* project VJP: pbf.cu:444-454 */
            for (uint32_t i = 0; i < n; ++i) {
                d3 a = xbar[i];
                if (it->mask[i] & 1u) a.x = 0.0;
                if (it->mask[i] & 2u) a.y = 0.0;
                if (it->mask[i] & 4u) a.z = 0.0;
                xbar_next[i] = a;
                cbar[i] = a;
                lbar[i] = 0.0;
                rbar[i] = 0.0;
            }
            /* correction VJP: pbf.cu:335-415 */
#pragma omp parallel for schedule(static)
            for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
                const uint32_t i = (uint32_t)ii;
                const double rho0 = p->rest_densities[i];
                const d3 ob = cbar[i];
                d3 px = v3(0, 0, 0);
                double pl = 0, pm = 0, pr = 0, pk = 0, pe = 0, pq = 0;
                STENCIL_BEGIN(&ctx, i, cell)
                    for (uint32_t q = ctx.g.offsets[cell]; q < ctx.g.offsets[cell + 1]; ++q) {
                        const uint32_t j = ctx.g.sorted[q];
                        if (j == i) continue;
                        const d3 d = sub3(x[i], x[j]);
                        const d3 gr = spiky_gradient(d, h);
                        const scorr s = artificial_pressure(d, h, p->artificial_pressure_strength[i], p->artificial_pressure_exponent[i], p->artificial_pressure_radius[i]);
                        const double c = p->masses[j] / rho0;
                        const double mu = it->lambda[i] + it->lambda[j] + s.value;
                        const double sa = c * dot3(ob, gr);
                        px = add3(px, spiky_hessian_product(d, mul3(ob, c * mu), h));
                        px = add3(px, mul3(s.gradient, sa));
                        pl += sa;
                        pr -= dot3(ob, mul3(gr, c * mu)) / rho0;
                        pk += sa * s.d_strength; pe += sa * s.d_exponent; pq += sa * s.d_radius;
                        const d3 rd = mul3(d, -1.0);
                        const d3 rg = spiky_gradient(rd, h);
                        const scorr rs = artificial_pressure(rd, h, p->artificial_pressure_strength[j], p->artificial_pressure_exponent[j], p->artificial_pressure_radius[j]);
                        const double rrho0 = p->rest_densities[j];
                        const double rc_ = p->masses[i] / rrho0;
                        const double rmu = it->lambda[j] + it->lambda[i] + rs.value;
                        const d3 rob = cbar[j];
                        const double rsa = rc_ * dot3(rob, rg);
                        px = add3(px, mul3(spiky_hessian_product(rd, mul3(rob, rc_ * rmu), h), -1.0));
                        px = add3(px, mul3(rs.gradient, -rsa));
                        pl += rsa;
                        pm += dot3(rob, mul3(rg, rmu / rrho0));
                    }
                    for (uint32_t q = ctx.bg.offsets[cell]; q < ctx.bg.offsets[cell + 1]; ++q) {
                        const uint32_t b = ctx.bg.sorted[q];
                        const d3 d = sub3(x[i], bpos(&ctx, b));
                        const d3 gr = spiky_gradient(d, h);
                        const scorr s = artificial_pressure(d, h, p->artificial_pressure_strength[i], p->artificial_pressure_exponent[i], p->artificial_pressure_radius[i]);
                        const double vol = sc->boundary_volume[b];
                        const double mu = it->lambda[i] + s.value;
                        const double sa = vol * dot3(ob, gr);
                        px = add3(px, spiky_hessian_product(d, mul3(ob, vol * mu), h));
                        px = add3(px, mul3(s.gradient, sa));
                        pl += sa;
                        pk += sa * s.d_strength; pe += sa * s.d_exponent; pq += sa * s.d_radius;
                    }
                }
                xbar_next[i] = add3(xbar_next[i], px);
                lbar[i] += pl;
                PADJ(adj->masses, i, pm);
                PADJ(adj->rest_densities, i, pr);
                PADJ(adj->artificial_pressure_strength, i, pk);
                PADJ(adj->artificial_pressure_exponent, i, pe);
                PADJ(adj->artificial_pressure_radius, i, pq);
            }
            /* lambda VJP: pbf.cu:180-252 */
#pragma omp parallel for schedule(static)
            for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
                const uint32_t i = (uint32_t)ii;
                const double rho0 = p->rest_densities[i];
                const double lb = lbar[i];
                const double C = it->density[i] / rho0 - 1.0;
                const double Db = lb * C / (it->denom[i] * it->denom[i]);
                const d3 Sb = mul3(it->gsum[i], 2.0 * Db);
                d3 px = v3(0, 0, 0);
                double pm = 0.0;
                double pr = lb * it->density[i] / (it->denom[i] * rho0 * rho0);
                STENCIL_BEGIN(&ctx, i, cell)
                    for (uint32_t q = ctx.g.offsets[cell]; q < ctx.g.offsets[cell + 1]; ++q) {
                        const uint32_t j = ctx.g.sorted[q];
                        if (j == i) continue;
                        const d3 d = sub3(x[i], x[j]);
                        const d3 gr = spiky_gradient(d, h);
                        const double c = p->masses[j] / rho0;
                        const d3 gij = mul3(gr, c);
                        const d3 gbar = add3(Sb, mul3(gij, 2.0 * Db));
                        px = add3(px, spiky_hessian_product(d, mul3(gbar, c), h));
                        pr -= dot3(gbar, gij) / rho0;
                        const double rrho0 = p->rest_densities[j];
                        const double rC = it->density[j] / rrho0 - 1.0;
                        const double rDb = lbar[j] * rC / (it->denom[j] * it->denom[j]);
                        const d3 rSb = mul3(it->gsum[j], 2.0 * rDb);
                        const d3 rd = mul3(d, -1.0);
                        const d3 rg = spiky_gradient(rd, h);
                        const double rcf = p->masses[i] / rrho0;
                        const d3 rgbar = add3(rSb, mul3(rg, 2.0 * rDb * rcf));
                        px = add3(px, mul3(spiky_hessian_product(rd, mul3(rgbar, rcf), h), -1.0));
                        pm += dot3(rgbar, rg) / rrho0;
                    }
                    for (uint32_t q = ctx.bg.offsets[cell]; q < ctx.bg.offsets[cell + 1]; ++q) {
                        const uint32_t b = ctx.bg.sorted[q];
                        const d3 d = sub3(x[i], bpos(&ctx, b));
                        px = add3(px, spiky_hessian_product(d, mul3(Sb, sc->boundary_volume[b]), h));
                    }
                }
                xbar_next[i] = add3(xbar_next[i], px);
                rbar[i] -= lb / (it->denom[i] * rho0);
                PADJ(adj->masses, i, pm);
                PADJ(adj->rest_densities, i, pr);
                PADJ(adj->relaxation, i, Db);
            }
            /* density VJP: density/density.cu:69-102 */
#pragma omp parallel for schedule(static)
            for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
                const uint32_t i = (uint32_t)ii;
                const double ob = rbar[i];
                d3 px = v3(0, 0, 0);
                double pm = 0.0, pr = 0.0;
                STENCIL_BEGIN(&ctx, i, cell)
                    for (uint32_t q = ctx.g.offsets[cell]; q < ctx.g.offsets[cell + 1]; ++q) {
                        const uint32_t j = ctx.g.sorted[q];
                        const d3 d = sub3(x[i], x[j]);
                        px = add3(px, mul3(poly6_gradient(d, h), ob * p->masses[j] + rbar[j] * p->masses[i]));
                        pm += rbar[j] * oracle_poly6(d.x, d.y, d.z, h);
                    }
                    for (uint32_t q = ctx.bg.offsets[cell]; q < ctx.bg.offsets[cell + 1]; ++q) {
                        const uint32_t b = ctx.bg.sorted[q];
                        const d3 d = sub3(x[i], bpos(&ctx, b));
                        const double vol = sc->boundary_volume[b];
                        px = add3(px, mul3(poly6_gradient(d, h), ob * p->rest_densities[i] * vol));
                        pr += ob * vol * oracle_poly6(d.x, d.y, d.z, h);
                    }
                }
                xbar_next[i] = add3(xbar_next[i], px);
                PADJ(adj->masses, i, pm);
                PADJ(adj->rest_densities, i, pr);
            }
            d3* t = xbar; xbar = xbar_next; xbar_next = t;
        }
        /* predict VJP: pbf.cu:86-93 */
        for (uint32_t i = 0; i < n; ++i) {
            acc(adj->position, i, xbar[i]);
            acc(adj->velocity, i, mul3(xbar[i], dt));
            acc(adj->control, i, mul3(xbar[i], dt * dt));
        }
    }
    free(xbar); free(xbar_next); free(vcbar); free(vrbar); free(wbar); free(nbar); free(cbar); free(lbar); free(rbar); free(etabar);
    context_free(&ctx);
    record_free(&r, K);
    return rc;
}
