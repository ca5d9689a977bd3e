"""Seeded synthetic dam-break scenes for the PBF substep.

Every scene is generated on the host from one counter-based SplitMix64 stream,
so the same seed gives byte-identical float32 inputs to the CUDA solver, the
reference kernels and the FP64 host oracle.

The workloads follow the particle module's dam-break example
(examples/fluids/liquid/pbf-dam-break/simulation.ixx:16-21,62-79,83-112):
mass = rest_density * spacing^3, relaxation 1000, artificial pressure
strength 0 / exponent 4 / radius 0.3 h, a static box with no boundary
particles.  Lattice point (i, j, k) sits at box_min + (i+1, j+1, k+1) * spacing
plus a uniform jitter of +-0.01 h per axis.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """Counter-based SplitMix64: element i is the mix of seed + (stream, i)."""
    with np.errstate(over="ignore"):
        base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
        z = base + (np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """Float64 uniforms in [0, 1) with 53 random bits."""
    return (splitmix64(seed, count, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """Standard normals by Box-Muller from two uniform streams."""
    u1 = uniform01(seed, count, 2 * stream + 1)
    u2 = uniform01(seed, count, 2 * stream + 2)
    u1 = np.maximum(u1, 1e-300)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


@dataclasses.dataclass
class Scene:
    """One dam-break scene: float32 SoA state plus the domain description."""

    positions: np.ndarray          # (3, N) float32
    velocities: np.ndarray         # (3, N) float32
    controls: np.ndarray           # (3, N) float32 external accelerations
    masses: np.ndarray             # (N,) float32
    rest_densities: np.ndarray
    relaxation: np.ndarray
    artificial_pressure_strength: np.ndarray
    artificial_pressure_exponent: np.ndarray
    artificial_pressure_radius: np.ndarray
    xsph_viscosity: np.ndarray
    vorticity_confinement: np.ndarray
    time_step: float
    support_radius: float
    particle_radius: float
    gravity: tuple
    box_min: tuple
    box_max: tuple
    box_velocity: tuple
    pressure_iterations: int
    name: str = ""
    targets: np.ndarray | None = None  # (3, N) float32 target cloud for the loss
    # boundary particles: {"positions": (3, B), "velocities": (3, B), "volumes": (B,)} float32
    boundary: dict | None = None
    # SPH parameters (sph_dam_break): one (N,) float32 array per SPH<Method>::Parameters field
    sph: dict | None = None
    # BoxBoundary::no_slip: a colliding particle takes the box velocity on every axis (SPH reads it)
    no_slip: bool = True

    @property
    def count(self) -> int:
        return int(self.positions.shape[1])

    def grid_dims(self) -> tuple:
        h = np.float32(self.support_radius)
        return tuple(int(np.ceil(np.float32(np.float32(self.box_max[a]) - np.float32(self.box_min[a])) / h)) for a in range(3))

    def parameter_arrays(self) -> dict:
        return {
            "masses": self.masses,
            "rest_densities": self.rest_densities,
            "relaxation": self.relaxation,
            "artificial_pressure_strength": self.artificial_pressure_strength,
            "artificial_pressure_exponent": self.artificial_pressure_exponent,
            "artificial_pressure_radius": self.artificial_pressure_radius,
            "xsph_viscosity": self.xsph_viscosity,
            "vorticity_confinement": self.vorticity_confinement,
        }


H = 0.025
SPACING = 0.5 * H


def dam_break(lattice, box_min, box_max, seed, iterations, *, h=H, dt=1.0 / 120.0,
              velocity_sigma=0.0, xsph=0.01, vorticity=1e-4, gravity=(0.0, -9.8, 0.0),
              fill_order="zyx", count=None, name="") -> Scene:
    """Jittered lattice in the low corner of a box.

    fill_order "zyx" fills x fastest, then y, then z (the example's order);
    "yzx" fills x fastest, then z, then y (used by the batched scenes, which
    truncate the lattice at an exact particle count).
    """
    nx, ny, nz = lattice
    spacing = np.float64(0.5 * h)
    if fill_order == "zyx":
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    else:
        j, k, i = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    if count is not None:
        i, j, k = i[:count], j[:count], k[:count]
    n = i.size
    jitter = (uniform01(seed, 3 * n, 0).reshape(3, n) * 2.0 - 1.0) * (0.01 * h)
    pos = np.empty((3, n), dtype=np.float32)
    pos[0] = (box_min[0] + (i + 1) * spacing + jitter[0]).astype(np.float32)
    pos[1] = (box_min[1] + (j + 1) * spacing + jitter[1]).astype(np.float32)
    pos[2] = (box_min[2] + (k + 1) * spacing + jitter[2]).astype(np.float32)
    if velocity_sigma > 0.0:
        vel = (normal(seed, 3 * n, 1).reshape(3, n) * velocity_sigma).astype(np.float32)
    else:
        vel = np.zeros((3, n), dtype=np.float32)
    f32 = np.float32
    full = lambda value: np.full(n, value, dtype=np.float32)
    return Scene(
        positions=pos,
        velocities=vel,
        controls=np.zeros((3, n), dtype=np.float32),
        masses=full(f32(1000.0) * f32(spacing) * f32(spacing) * f32(spacing)),
        rest_densities=full(1000.0),
        relaxation=full(1000.0),
        artificial_pressure_strength=full(0.0),
        artificial_pressure_exponent=full(4.0),
        artificial_pressure_radius=full(f32(0.3) * f32(h)),
        # The reference's XSPH and confinement sums (pbf/pbf.cu:476-497, 674-678, 700-721)
        # carry no particle volume m_j/rho_j, so the physical coefficients c and eps are
        # stored premultiplied by the particle volume V = m/rho0 = spacing^3.
        xsph_viscosity=full(f32(xsph) * f32(spacing) ** 3),
        vorticity_confinement=full(f32(vorticity) * f32(spacing) ** 3),
        time_step=float(f32(dt)),
        support_radius=float(f32(h)),
        particle_radius=float(f32(0.2) * f32(h)),
        gravity=tuple(float(f32(g)) for g in gravity),
        box_min=tuple(float(f32(b)) for b in box_min),
        box_max=tuple(float(f32(b)) for b in box_max),
        box_velocity=(0.0, 0.0, 0.0),
        pressure_iterations=iterations,
        name=name,
    )


def target_cloud(seed: int, n: int, lo=(0.25, 0.0, 0.25), hi=(0.75, 0.5, 0.75)) -> np.ndarray:
    u = uniform01(seed ^ 0x7A7A7A7A, 3 * n, 7).reshape(3, n)
    out = np.empty((3, n), dtype=np.float32)
    for a in range(3):
        out[a] = (lo[a] + (hi[a] - lo[a]) * u[a]).astype(np.float32)
    return out


def plain_small(seed=1, lattice=(32, 32, 32), iterations=4) -> Scene:
    """32,768-particle dam break in a [0,1]x[0,2]x[0,1] box (4 iterations, 100 steps)."""
    return dam_break(lattice, (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), seed, iterations, name="dam_break_32k")


def plain_large(seed=2, lattice=(128, 64, 128), iterations=8) -> Scene:
    """1,048,576-particle dam break (128x64x128 lattice) in a [0,4]^3 box, 8 iterations."""
    return dam_break(lattice, (0.0, 0.0, 0.0), (4.0, 4.0, 4.0), seed, iterations, name="dam_break_1m")


def differentiable(seed=3, lattice=(32, 64, 32), iterations=4) -> Scene:
    """65,536 particles with v0 ~ N(0, 0.1) and a uniform target cloud in a 0.5^3 box."""
    scene = dam_break(lattice, (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), seed, iterations,
                      velocity_sigma=0.1, name="differentiable_64k")
    scene.targets = target_cloud(seed, scene.count)
    return scene


def batched_counts(seed: int, scenes: int, lo: int, hi: int, log_uniform: bool) -> list:
    u = uniform01(seed, scenes, 11)
    if log_uniform:
        counts = np.round(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo))))
    else:
        counts = np.floor(lo + u * (hi - lo + 1))
    return [int(min(max(c, lo), hi)) for c in counts]


def batched_scene(count: int, seed: int, iterations: int, velocity_sigma=0.0, name="") -> Scene:
    """A dam break of exactly `count` particles in a box whose side scales with the count.

    Lattice nx = nz = ceil((count/2)^(1/3)), filled x fastest, then z, then y,
    truncated at `count`; box [0,L]x[0,2L]x[0,L] with L = 2.5 nx spacing.
    """
    nx = int(math.ceil((count / 2.0) ** (1.0 / 3.0)))
    ny = int(math.ceil(count / float(nx * nx)))
    side = 2.5 * nx * SPACING
    return dam_break((nx, ny, nx), (0.0, 0.0, 0.0), (side, 2.0 * side, side), seed, iterations,
                     velocity_sigma=velocity_sigma, fill_order="yzx", count=count, name=name)


def batched_forward(seed=4, scenes=256, iterations=4) -> list:
    """256 scenes with counts log-uniform in [2048, 65536]."""
    counts = batched_counts(seed, scenes, 2048, 65536, True)
    return [batched_scene(c, seed * 1000003 + s, iterations, name=f"scene{s}") for s, c in enumerate(counts)]


def batched_adjoint(seed=5, scenes=32, iterations=4) -> list:
    """32 scenes with counts uniform in [16384, 131072], each with its own target cloud."""
    counts = batched_counts(seed, scenes, 16384, 131072, False)
    out = []
    for s, c in enumerate(counts):
        sc = batched_scene(c, seed * 1000003 + s, iterations, name=f"scene{s}")
        side = sc.box_max[0]
        sc.targets = target_cloud(seed * 7919 + s, c, (0.25 * side, 0.0, 0.25 * side), (0.75 * side, 0.5 * side, 0.75 * side))
        out.append(sc)
    return out


def with_boundary(scene: Scene, seed: int, floor_velocity=(0.05, 0.0, 0.0)) -> Scene:
    """The scene plus boundary particles: a moving floor plate under the fluid column (a 0.5h
    lattice at y = 0.6 spacing, sliding with `floor_velocity`) and a static wall plate at
    x = 0.4 in front of it, each particle with volume spacing^3 (jittered by +-1%)."""
    spacing = 0.5 * scene.support_radius
    lo = np.asarray(scene.positions.min(axis=1), dtype=np.float64)
    hi = np.asarray(scene.positions.max(axis=1), dtype=np.float64)
    xs = np.arange(lo[0] - 2 * spacing, hi[0] + 2 * spacing, spacing)
    zs = np.arange(lo[2] - 2 * spacing, hi[2] + 2 * spacing, spacing)
    fx, fz = np.meshgrid(xs, zs, indexing="ij")
    floor = np.stack([fx.ravel(), np.full(fx.size, 0.6 * spacing), fz.ravel()])
    ys = np.arange(0.5 * spacing, hi[1] + 2 * spacing, spacing)
    wy, wz = np.meshgrid(ys, zs, indexing="ij")
    wall = np.stack([np.full(wy.size, hi[0] + 1.5 * spacing), wy.ravel(), wz.ravel()])
    positions = np.concatenate([floor, wall], axis=1)
    velocities = np.zeros_like(positions)
    velocities[:, :floor.shape[1]] = np.asarray(floor_velocity, dtype=np.float64)[:, None]
    volumes = spacing ** 3 * (1.0 + 0.02 * (uniform01(seed, positions.shape[1], 17) - 0.5))
    scene.boundary = {"positions": positions.astype(np.float32), "velocities": velocities.astype(np.float32),
                      "volumes": volumes.astype(np.float32)}
    return scene


def example_dam_break() -> Scene:
    """The reference's own dam-break example (examples/fluids/liquid/pbf-dam-break/simulation.ixx):
    a 16 x 28 x 12 lattice at spacing 0.025 starting at 0.08 (x fastest, then y, then z), h = 0.05,
    dt = 1/240, particle radius 0.01, gravity -9.81, box [0,0.8] x [0,1.1] x [0,0.5], 5 Jacobi
    iterations, relaxation 1000, s_corr strength 0 / exponent 4 / radius 0.3h, no XSPH and no
    vorticity confinement, zero velocities and controls.  No jitter: the example has none."""
    f32 = np.float32
    nx, ny, nz = 16, 28, 12
    spacing, h = f32(0.025), f32(0.050)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pos = np.stack([f32(0.08) + i.ravel().astype(f32) * spacing, f32(0.08) + j.ravel().astype(f32) * spacing,
                    f32(0.08) + k.ravel().astype(f32) * spacing]).astype(np.float32)
    n = pos.shape[1]
    full = lambda value: np.full(n, value, dtype=np.float32)
    return Scene(
        positions=pos,
        velocities=np.zeros((3, n), dtype=np.float32),
        controls=np.zeros((3, n), dtype=np.float32),
        masses=full(f32(1000.0) * spacing * spacing * spacing),
        rest_densities=full(1000.0),
        relaxation=full(1000.0),
        artificial_pressure_strength=full(0.0),
        artificial_pressure_exponent=full(4.0),
        artificial_pressure_radius=full(f32(0.3) * h),
        xsph_viscosity=full(0.0),
        vorticity_confinement=full(0.0),
        time_step=float(f32(1.0) / f32(240.0)),
        support_radius=float(h),
        particle_radius=float(f32(0.010)),
        gravity=(0.0, float(f32(-9.81)), 0.0),
        box_min=(0.0, 0.0, 0.0),
        box_max=(float(f32(0.8)), float(f32(1.1)), float(f32(0.5))),
        box_velocity=(0.0, 0.0, 0.0),
        pressure_iterations=5,
        name="example_dam_break",
    )


SPH_DT = 4.0e-4


def sph_parameter_arrays(scene: Scene, *, viscosity=None, surface_tension=0.05, speed_of_sound=20.0,
                         tait_exponent=7.0, boundary_surface_tension=0.02, relaxation=0.5, method="wcsph") -> dict:
    """SPH particle and method parameters for a dam-break scene (sph/sph.ixx:45-49, 111, 157,
    214-217): the scene's masses and rest densities; viscosity 0.05 (Monaghan alpha of WCSPH) or
    0.001 (kinematic viscosity of the others' Laplacian term); cohesion 0.05; c = 20 m/s and
    gamma = 7 in the Tait equation; adhesion 0.02; every pressure relaxation 0.5."""
    n = scene.count
    full = lambda value: np.full(n, value, dtype=np.float32)
    if viscosity is None:
        viscosity = 0.05 if method == "wcsph" else 0.001
    return {
        "masses": scene.masses.copy(),
        "rest_densities": scene.rest_densities.copy(),
        "viscosities": full(viscosity),
        "surface_tensions": full(surface_tension),
        "speed_of_sound": full(speed_of_sound),
        "tait_exponent": full(tait_exponent),
        "boundary_surface_tension": full(boundary_surface_tension),
        "pressure_relaxation": full(relaxation),
        "jacobi_relaxation": full(relaxation),
        "divergence_relaxation": full(relaxation),
        "density_relaxation": full(relaxation),
    }


def sph_dam_break(lattice, box_min, box_max, seed, *, method="wcsph", dt=SPH_DT, velocity_sigma=0.0, name="",
                  **parameters) -> Scene:
    """The dam-break lattice of `dam_break` (spacing 0.5 h, particle radius 0.2 h) with SPH
    parameters and an SPH time step (CFL 0.4 h / c at c = 20 m/s is 5e-4 s)."""
    scene = dam_break(lattice, box_min, box_max, seed, 0, dt=dt, velocity_sigma=velocity_sigma, name=name)
    scene.sph = sph_parameter_arrays(scene, method=method, **parameters)
    return scene


def sph_large(seed=6, method="wcsph") -> Scene:
    """1,048,576-particle SPH dam break (128x64x128 lattice) in a [0,4]^3 box."""
    return sph_dam_break((128, 64, 128), (0.0, 0.0, 0.0), (4.0, 4.0, 4.0), seed, method=method, name="sph_dam_break_1m")
