"""CPU tests of the FP64 host oracle: analytic known answers, grid semantics, and the pins
against outputs of the reference's own CUDA kernels (tests/golden/*.npz, made on a B200 by
tests/golden/make_golden.py)."""
import math
import pathlib

import numpy as np
import pytest

from physica_b200 import scenes

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def test_poly6_normalisation(oracle_lib):
    """The poly6 kernel integrates to 1 over its support (density/device.cuh:10-16)."""
    h = 0.025
    r = np.linspace(0.0, h, 20001)
    w = np.array([oracle_lib.poly6((x, 0.0, 0.0), h) for x in r])
    integral = np.trapezoid(4.0 * math.pi * r * r * w, r)
    # the reference's float pi differs from pi by 2.8e-8 relative
    assert abs(integral - 1.0) < 1e-6


def test_spiky_gradient_antisymmetric_and_analytic(oracle_lib):
    h = 0.025
    rng = np.random.default_rng(0)
    for _ in range(50):
        d = rng.uniform(-h, h, 3)
        g = oracle_lib.spiky_gradient(d, h)
        gm = oracle_lib.spiky_gradient(-d, h)
        assert np.allclose(g, -gm, rtol=0, atol=1e-12 * max(1.0, np.abs(g).max()))
        r = np.linalg.norm(d)
        expect = np.zeros(3) if r >= h else d * (-45.0 / (math.pi * h ** 6)) * (h - r) ** 2 / r
        assert np.allclose(g, expect, rtol=1e-6, atol=0)
    assert np.all(oracle_lib.spiky_gradient((0.0, 0.0, 0.0), h) == 0.0)
    assert np.all(oracle_lib.spiky_gradient((h, 0.0, 0.0), h) == 0.0)


def _single(position, velocity=(0.0, 0.0, 0.0), iterations=3):
    sc = scenes.dam_break((1, 1, 1), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), 5, iterations)
    sc.positions[:, 0] = position
    sc.velocities[:, 0] = velocity
    return sc


def test_single_particle_free_fall(oracle_lib):
    """A lone particle follows symplectic Euler exactly: x_n = x0 + dt^2 g n(n+1)/2."""
    sc = _single((0.5, 1.5, 0.5))
    x, v = sc.positions.astype(np.float64), sc.velocities.astype(np.float64)
    dt = sc.time_step
    g = sc.gravity[1]
    for n in range(1, 21):
        x, v = oracle_lib.forward_step(sc, x, v, step_index=n - 1)
        expect_y = 1.5 + dt * dt * g * n * (n + 1) / 2.0
        assert abs(x[1, 0] - expect_y) < 1e-12
        assert abs(v[1, 0] - dt * g * n) < 1e-10
        assert x[0, 0] == pytest.approx(0.5) and x[2, 0] == pytest.approx(0.5)


def test_particle_at_rest_on_floor(oracle_lib):
    """A particle resting on the floor is projected back onto the collision box each step."""
    sc = _single((0.5, 0.0, 0.5))
    floor = sc.box_min[1] + np.float32(sc.particle_radius)
    x, v = sc.positions.astype(np.float64), sc.velocities.astype(np.float64)
    x[1, 0] = floor
    for n in range(5):
        x, v = oracle_lib.forward_step(sc, x, v, step_index=n)
        assert x[1, 0] == pytest.approx(float(floor), abs=1e-7)
        assert abs(v[1, 0]) < 1e-6


def test_grid_f32_stable_and_clamped(oracle_lib):
    """Keys clamp out-of-grid points; the order is stable by original index; offsets bracket cells."""
    sc = scenes.plain_small(lattice=(6, 6, 6))
    pts = sc.positions.copy()
    pts[:, 0] = (-5.0, 9.0, 0.5)        # outside the box: clamped into edge cells
    pts[:, 1] = pts[:, 2]               # duplicate point: same cell, order by index
    keys, srt, off, dims = oracle_lib.grid_f32(sc, pts, 0.0)
    assert dims == (40, 80, 40)
    assert keys[0] == (int(0.5 / 0.025) * 80 + 79) * 40 + 0
    assert np.all(np.diff(keys[srt].astype(np.int64)) >= 0)
    for c in np.unique(keys):
        members = srt[off[c]:off[c + 1]]
        assert np.all(keys[members] == c)
        assert np.all(np.diff(members.astype(np.int64)) > 0)
    assert off[-1] == sc.count and off[0] == 0


def test_neighbor_counts_match_bruteforce(oracle_lib):
    sc = scenes.plain_small(lattice=(10, 10, 10))
    pts = sc.positions
    counts = oracle_lib.neighbor_counts_f32(sc, pts, pts, 0.0)
    h = np.float32(sc.support_radius)
    h2 = h * h
    brute = []
    for i in range(sc.count):
        d = (pts - pts[:, i:i + 1]).astype(np.float32)
        r2 = (d[0] * d[0] + d[1] * d[1]).astype(np.float32) + d[2] * d[2]
        brute.append(int((r2 < h2).sum()) - 1)
    # contraction differences can only flip pairs within one ulp of h^2
    assert np.abs(counts.astype(np.int64) - np.array(brute)).max() <= 1
    assert (counts == np.array(brute)).mean() > 0.999


def test_oracle_vjp_matches_central_differences(oracle_lib):
    """FP64 adjoint of one substep against central differences of the FP64 forward."""
    sc = scenes.dam_break((5, 5, 5), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), 21, 3, velocity_sigma=0.1)
    x0, v0 = sc.positions.astype(np.float64), sc.velocities.astype(np.float64)
    rng = np.random.default_rng(1)
    wx, wv = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))

    def loss(x, v, params=None):
        x1, v1 = oracle_lib.forward_step(sc, x, v, params=params)
        return float((wx * x1).sum() + (wv * v1).sum())

    adj = oracle_lib.vjp_step(sc, x0, v0, wx, wv)
    eps = 1e-7
    for (arr, grad, name) in ((v0, adj["velocity"], "v"), (x0, adj["position"], "x")):
        for (a, i) in ((0, 3), (1, 60), (2, 100)):
            p = arr.copy(); m = arr.copy()
            p[a, i] += eps; m[a, i] -= eps
            if name == "v":
                fd = (loss(x0, p) - loss(x0, m)) / (2 * eps)
            else:
                fd = (loss(p, v0) - loss(m, v0)) / (2 * eps)
            assert grad[a, i] == pytest.approx(fd, rel=1e-4, abs=1e-6)
    # scalar XSPH viscosity shared by all particles: dL/dc = sum_i dL/dc_i
    c = float(sc.xsph_viscosity[0])
    dc = c * 1e-4
    fd = (loss(x0, v0, oracle_lib.Parameters(sc, c + dc)) - loss(x0, v0, oracle_lib.Parameters(sc, c - dc))) / (2 * dc)
    assert adj["xsph_viscosity"].sum() == pytest.approx(fd, rel=1e-4)


def _golden(name):
    path = GOLDEN / f"{name}.npz"
    if not path.exists():
        pytest.skip(f"golden fixture {path.name} not generated yet")
    return np.load(path)


def test_oracle_grid_matches_reference_golden(oracle_lib):
    """Integer grid of the reference kernels (keys, stable order, offsets) is reproduced exactly."""
    g = _golden("reference_step_small")
    sc = scenes.dam_break(tuple(g["lattice"]), tuple(g["box_min"]), tuple(g["box_max"]), int(g["seed"]),
                          int(g["iterations"]))
    keys, srt, off, _ = oracle_lib.grid_f32(sc, g["predicted"], float(np.float32(1) * np.float32(sc.time_step)))
    assert np.array_equal(srt, g["sorted_indices"].astype(np.uint32))
    assert np.array_equal(off, g["cell_offsets"].astype(np.uint32))
    assert np.array_equal(keys[srt].astype(np.uint64), g["sorted_keys"].astype(np.uint64))


def test_oracle_step_matches_reference_golden(oracle_lib):
    """One FP64 substep agrees with the reference's FP32 kernels on the same inputs."""
    g = _golden("reference_step_small")
    sc = scenes.dam_break(tuple(g["lattice"]), tuple(g["box_min"]), tuple(g["box_max"]), int(g["seed"]),
                          int(g["iterations"]))
    assert np.array_equal(sc.positions, g["x0"]) and np.array_equal(sc.velocities, g["v0"])
    x1, v1, tr = oracle_lib.forward_step(sc, g["x0"], g["v0"], trace=True)
    h = sc.support_radius
    assert np.abs(tr["predicted"] - g["predicted"]).max() < 1e-6 * h
    assert np.abs(tr["density0"] - g["first_densities"]).max() / 1000.0 < 1e-5
    assert np.abs(x1 - g["x1"]).max() < 1e-4 * h
    assert np.abs(v1 - g["v1"]).max() < 1e-4 * h / sc.time_step
    counts = oracle_lib.neighbor_counts_f32(sc, g["predicted"], g["predicted"], float(np.float32(sc.time_step)))
    assert np.array_equal(counts, tr["neighbor_count0"])


def test_oracle_vjp_matches_reference_golden(oracle_lib):
    """FP64 VJP of one substep agrees with the reference's VJP kernels (FP32 primal, FP64 adjoint)."""
    g = _golden("reference_vjp_small")
    sc = scenes.dam_break(tuple(g["lattice"]), tuple(g["box_min"]), tuple(g["box_max"]), int(g["seed"]),
                          int(g["iterations"]), velocity_sigma=float(g["velocity_sigma"]))
    adj = oracle_lib.vjp_step(sc, g["x0"], g["v0"], g["next_position_adjoint"], g["next_velocity_adjoint"])
    for key in ("position", "velocity", "control"):
        ref = g[f"adj_{key}"]
        scale = np.abs(ref).max()
        assert np.abs(adj[key] - ref).max() <= 1e-3 * scale, key
    ref = g["adj_xsph_viscosity"]
    assert adj["xsph_viscosity"].sum() == pytest.approx(ref.sum(), rel=1e-3)
