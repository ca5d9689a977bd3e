"""FP64 host restatement of the SPH family's forward substep -- TEST INFRASTRUCTURE ONLY.

SPH<Method>::forward_step (fluids/liquid/particle/sph/sph.ixx:350-354) for WCSPH, PCISPH, IISPH and
DFSPH (sph/sph.cpp:214-225, 296-312, 409-425, 572-610), restated in numpy for small scenes: pairs
are enumerated by brute force and filtered exactly as the reference's grid does (a candidate is
stored in the cell of its key, neighborhood/neighborhood.cu:20-34, and a particle gathers over
the 27 cells around its own cell, neighborhood/device.cuh:44-48; both cell formulas in float32,
as the reference evaluates them).  Kernel values, sums and updates are FP64:
  cubic spline, gradient, viscosity Laplacian   density/device.cuh:26-43, 72-76
  density (cubic)                               density/density.cu:18-40
  Tait equation of state                        sph/wcsph.cu:92-100
  pressure acceleration                         sph/common.cu:165-194
  artificial viscosity                          sph/wcsph.cu:136-174
  cohesion / adhesion                           sph/wcsph.cu:306-339
  non-pressure acceleration                     sph/common.cu:14-47
  prediction / integration with the box         sph/pcisph.cu:26-45, sph/common.cu:302-320
  pressure updates                              sph/pcisph.cu:104-110, sph/iisph.cu:104-110,
                                                sph/dfsph.cu:104-110
  reference gradient norm                       sph/sph.cpp:36-58 (float32 loop, as the reference)
Only tests/ and bench.py's CPU baseline use this module; the product never does.  It is pinned
against the reference's own kernels by tests/golden/sph_reference_small.npz
(tests/golden/make_sph_golden.py).
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32
PI32 = F32(3.14159265358979323846)


def reference_gradient_norm(support_radius: float, particle_radius: float) -> float:
    """sph/sph.cpp:36-58 in float32, one rounding per operation."""
    h, d = F32(support_radius), F32(2.0) * F32(particle_radius)
    coefficient = F32(8.0) / (PI32 * h * h * h)
    sx = sy = sz = ss = F32(0.0)
    x = -h
    while x <= h:
        y = -h
        while y <= h:
            z = -h
            while z <= h:
                r2 = x * x + y * y + z * z
                dist = F32(np.sqrt(r2))
                if dist != 0.0 and dist < h:
                    q = dist / h
                    der = F32(18.0) * q * q - F32(12.0) * q if q <= 0.5 else F32(-6.0) * (F32(1.0) - q) * (F32(1.0) - q)
                    s = coefficient * der / (h * dist)
                    sx, sy, sz = sx + s * x, sy + s * y, sz + s * z
                    ss = ss + s * s * r2
                z = F32(z + d)
            y = F32(y + d)
        x = F32(x + d)
    return float(sx * sx + sy * sy + sz * sz + ss)


# ------------------------------------------------------------------ kernels (FP64)
def cubic(r, h):
    q = r / h
    c = 8.0 / (math.pi * h ** 3)
    w = np.where(q <= 0.5, c * (6.0 * q ** 3 - 6.0 * q ** 2 + 1.0), 2.0 * c * (1.0 - q) ** 3)
    return np.where(r < h, w, 0.0)


def cubic_gradient(d, r, h):
    """d: (3, P) displacements, r: (P,) distances."""
    q = r / h
    c = 8.0 / (math.pi * h ** 3)
    der = np.where(q <= 0.5, 18.0 * q * q - 12.0 * q, -6.0 * (1.0 - q) ** 2)
    safe = np.where(r > 0.0, r, 1.0)
    s = np.where((r > 0.0) & (r < h), c * der / (h * safe), 0.0)
    return d * s


def laplacian(r, h):
    return np.where(r < h, 45.0 * (h - r) / (math.pi * h ** 6), 0.0)


# ------------------------------------------------------------------ grid
class Grid:
    """The reference's uniform grid of cell size h (neighborhood/neighborhood.cpp:28-32, 83-88)."""

    def __init__(self, scene, step: int):
        self.h = F32(scene.support_radius)
        lo, hi = np.asarray(scene.box_min, F32), np.asarray(scene.box_max, F32)
        self.dims = np.array([int(np.ceil(F32(hi[a] - lo[a]) / self.h)) for a in range(3)])
        self.time = F32(step) * F32(scene.time_step)
        self.min = lo
        self.vel = np.asarray(scene.box_velocity, F32)
        self.origin = (lo + self.time * self.vel).astype(F32)

    def _clamp(self, q):
        return np.clip(np.floor(q).astype(np.int64), 0, (self.dims - 1)[:, None])

    def key_cells(self, x):
        """Storage cell: (x - min - t v) / h (neighborhood/neighborhood.cu:30-32)."""
        x = np.asarray(x, F32)
        q = ((x - self.min[:, None]) - self.time * self.vel[:, None]) / self.h
        return self._clamp(q.astype(F32))

    def gather_cells(self, x):
        """Home cell of a gather: (x - origin) / h (neighborhood/device.cuh:44-48)."""
        x = np.asarray(x, F32)
        q = (x - self.origin[:, None]) / self.h
        return self._clamp(q.astype(F32))


def stencil_pairs(home, stored):
    """All (i, j) with cell j within one cell of the home cell of i (i == j included)."""
    diff = np.abs(home[:, :, None] - stored[:, None, :]).max(axis=0)
    i, j = np.nonzero(diff <= 1)
    return i, j


class Step:
    """One substep's neighbourhood: fluid pairs (home cell of x, stored cell of x) and boundary
    pairs (boundary particles at p + t v, keyed like the fluid)."""

    def __init__(self, scene, x, step):
        self.grid = Grid(scene, step)
        self.x = np.asarray(x, np.float64)
        home = self.grid.gather_cells(x)
        self.i, self.j = stencil_pairs(home, self.grid.key_cells(x))
        b = getattr(scene, "boundary", None)
        if b is not None and len(b["volumes"]):
            t = self.grid.time
            bp = (np.asarray(b["positions"], F32) + t * np.asarray(b["velocities"], F32)).astype(F32)
            self.bx = bp.astype(np.float64)
            self.bv = np.asarray(b["velocities"], np.float64)
            self.bvol = np.asarray(b["volumes"], np.float64)
            self.bi, self.bj = stencil_pairs(home, self.grid.key_cells(bp))
        else:
            self.bx = np.zeros((3, 0))
            self.bv = np.zeros((3, 0))
            self.bvol = np.zeros(0)
            self.bi = self.bj = np.zeros(0, np.int64)


def _sum(i, values, n):
    """Per-particle sums of pair values (scalar or (3, P))."""
    if values.ndim == 1:
        return np.bincount(i, weights=values, minlength=n)
    return np.stack([np.bincount(i, weights=values[a], minlength=n) for a in range(3)])


def density(st, positions, mass, rest, h):
    """density_forward at `positions` over the stencil of the step's positions."""
    n = positions.shape[1]
    d = positions[:, st.i] - positions[:, st.j]
    rho = _sum(st.i, mass[st.j] * cubic(np.linalg.norm(d, axis=0), h), n)
    if len(st.bi):
        db = positions[:, st.bi] - st.bx[:, st.bj]
        rho += _sum(st.bi, rest[st.bi] * st.bvol[st.bj] * cubic(np.linalg.norm(db, axis=0), h), n)
    return rho


def pressure_acceleration(st, mass, rest, rho, p, h):
    n = st.x.shape[1]
    ft = p / (rho * rho)
    keep = st.i != st.j
    i, j = st.i[keep], st.j[keep]
    d = st.x[:, i] - st.x[:, j]
    g = cubic_gradient(d, np.linalg.norm(d, axis=0), h)
    a = _sum(i, g * (-mass[j] * (ft[i] + ft[j])), n)
    if len(st.bi):
        db = st.x[:, st.bi] - st.bx[:, st.bj]
        gb = cubic_gradient(db, np.linalg.norm(db, axis=0), h)
        a += _sum(st.bi, gb * (-rest[st.bi] * st.bvol[st.bj] * ft[st.bi]), n)
    return a


def box_of(scene, step):
    t = F32(step) * F32(scene.time_step)
    r = F32(scene.particle_radius)
    lo = np.array([F32(scene.box_min[a]) + t * F32(scene.box_velocity[a]) + r for a in range(3)], np.float64)
    hi = np.array([F32(scene.box_max[a]) + t * F32(scene.box_velocity[a]) - r for a in range(3)], np.float64)
    return lo, hi


def predict(scene, step, x, v, a):
    """v' = v + dt a, x' = x + dt v', clamped to the box; colliding axes take the box velocity
    (all axes when no_slip)."""
    dt = float(F32(scene.time_step))
    lo, hi = box_of(scene, step)
    vel = v + dt * a
    pos = x + dt * vel
    hit = (pos < lo[:, None]) | (pos > hi[:, None])
    pos = np.minimum(hi[:, None], np.maximum(lo[:, None], pos))
    box_v = np.asarray(scene.box_velocity, np.float64)[:, None]
    if getattr(scene, "no_slip", True):
        any_hit = hit.any(axis=0)
        vel = np.where(any_hit[None, :], box_v, vel)
    else:
        vel = np.where(hit, box_v, vel)
    return pos, vel


def forward_step(scene, method: str, x, v, step_index=0, iterations=(6, 4, 6), warm=None, warm_start=True):
    """One SPH substep in FP64 from float32 inputs.  iterations: (pressure, divergence, density).
    Returns (next positions, next velocities, fields) where fields holds densities, pressures and
    DFSPH's next warm pressures."""
    p_sph = scene.sph
    mass = np.asarray(p_sph["masses"], np.float64)
    rest = np.asarray(p_sph["rest_densities"], np.float64)
    visc = np.asarray(p_sph["viscosities"], np.float64)
    h = float(F32(scene.support_radius))
    dt = float(F32(scene.time_step))
    x64, v64 = np.asarray(x, np.float64), np.asarray(v, np.float64)
    n = x64.shape[1]
    st = Step(scene, x, step_index)
    rho = density(st, x64, mass, rest, h)
    gravity = np.asarray(scene.gravity, np.float64)[:, None]
    control = np.asarray(scene.controls, np.float64)
    fields = {"densities": rho}
    keep = st.i != st.j
    i, j = st.i[keep], st.j[keep]
    d = x64[:, i] - x64[:, j]
    r = np.linalg.norm(d, axis=0)
    if method == "wcsph":
        c = np.asarray(p_sph["speed_of_sound"], np.float64)
        gamma = np.asarray(p_sph["tait_exponent"], np.float64)
        p = rest * c * c * ((rho / rest) ** gamma - 1.0) / gamma
        fields["pressures"] = p
        a_p = pressure_acceleration(st, mass, rest, rho, p, h)
        # artificial viscosity (sph/wcsph.cu:149-171)
        vd = v64[:, i] - v64[:, j]
        comp = (vd * d).sum(axis=0)
        nu = 2.0 * (0.5 * (visc[i] + visc[j])) * h * (0.5 * (c[i] + c[j])) / (rho[i] + rho[j])
        pi = np.where(comp < 0.0, -nu * comp / (r * r + 0.01 * h * h), 0.0)
        a_v = _sum(i, cubic_gradient(d, r, h) * (-mass[j] * pi), n)
        # cohesion (sph/wcsph.cu:318-325)
        diam = 2.0 * float(F32(scene.particle_radius))
        contact = float(cubic(np.array([diam]), h)[0])
        st_i = np.asarray(p_sph["surface_tensions"], np.float64)
        weight = np.where(r > diam, cubic(r, h), contact)
        factor = np.where(r < h, -st_i[i] * mass[j] * weight / mass[i], 0.0)
        a_s = _sum(i, d * factor, n)
        if len(st.bi):
            db = x64[:, st.bi] - st.bx[:, st.bj]
            rb = np.linalg.norm(db, axis=0)
            vdb = v64[:, st.bi] - st.bv[:, st.bj]
            compb = (vdb * db).sum(axis=0)
            nub = visc[st.bi] * h * c[st.bi] / rho[st.bi]
            pib = np.where(compb < 0.0, -nub * compb / (rb * rb + 0.01 * h * h), 0.0)
            a_v += _sum(st.bi, cubic_gradient(db, rb, h) * (-rest[st.bi] * st.bvol[st.bj] * pib), n)
            bst = np.asarray(p_sph["boundary_surface_tension"], np.float64)
            wb = np.where(rb > diam, cubic(rb, h), contact)
            fb = np.where(rb < h, -bst[st.bi] * rest[st.bi] * st.bvol[st.bj] * wb / mass[st.bi], 0.0)
            a_s += _sum(st.bi, db * fb, n)
        total = a_p + a_v + a_s + gravity + control
        xo, vo = predict(scene, step_index, x64, v64, total)
        return xo, vo, fields
    # non-pressure acceleration (sph/common.cu:14-47)
    lap = laplacian(r, h)
    mu = 0.5 * (visc[i] + visc[j])
    a_np = gravity + control + _sum(i, (v64[:, j] - v64[:, i]) * (mu * mass[j] * lap / rho[j]), n)
    if len(st.bi):
        db = x64[:, st.bi] - st.bx[:, st.bj]
        lb = laplacian(np.linalg.norm(db, axis=0), h)
        a_np += _sum(st.bi, (st.bv[:, st.bj] - v64[:, st.bi]) * (visc[st.bi] * st.bvol[st.bj] * lb), n)
    rgn = reference_gradient_norm(scene.support_radius, scene.particle_radius)

    def update(p_prev, rho_star, relaxation, volume, target):
        delta = 1.0 / (2.0 * dt * dt * volume * volume * rgn)
        return np.maximum(0.0, p_prev + relaxation * delta * (rho_star - target))

    def iterate(p, a_p, count, base, relaxation, volume, target):
        for _ in range(count):
            total = a_p if base is None else base + a_p
            xs, _vs = predict(scene, step_index, x64, v64, a_np + total)
            rho_star = density(st, xs, mass, rest, h)
            p = update(p, rho_star, relaxation, volume, target)
            a_p = pressure_acceleration(st, mass, rest, rho, p, h)
        return p, a_p

    if method in ("pcisph", "iisph"):
        relax = np.asarray(p_sph["pressure_relaxation" if method == "pcisph" else "jacobi_relaxation"], np.float64)
        volume = mass / (rest if method == "pcisph" else rho)
        p, a_p = iterate(np.zeros(n), np.zeros((3, n)), iterations[0], None, relax, volume, rest)
        fields["pressures"] = p
        xo, vo = predict(scene, step_index, x64, v64, a_np + a_p)
        return xo, vo, fields
    # DFSPH
    volume = mass / rho
    w0 = np.asarray(warm[0], np.float64) if (warm is not None and warm_start) else np.zeros(n)
    w1 = np.asarray(warm[1], np.float64) if (warm is not None and warm_start) else np.zeros(n)
    p_d, a_d = iterate(w0, pressure_acceleration(st, mass, rest, rho, w0, h), iterations[1], None,
                       np.asarray(p_sph["divergence_relaxation"], np.float64), volume, rho)
    p_r, a_r = iterate(w1, pressure_acceleration(st, mass, rest, rho, w1, h), iterations[2], a_d,
                       np.asarray(p_sph["density_relaxation"], np.float64), volume, rest)
    fields["pressures"] = p_r
    fields["warm"] = (p_d, p_r)
    xo, vo = predict(scene, step_index, x64, v64, a_np + a_d + a_r)
    return xo, vo, fields
