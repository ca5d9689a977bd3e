"""GPU parity tests of the SPH solvers (WCSPH, PCISPH, IISPH, DFSPH) against the reference's own
sph/*.cu kernels replayed by the harness (SPH<Method>::forward_step, sph/sph.ixx:350-354) on the
same inputs: every substep bit for bit, and the step cache's fields (densities, pressures,
accelerations) bit for bit after one step."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes, sph

pytestmark = pytest.mark.gpu

METHODS = ("wcsph", "pcisph", "iisph", "dfsph")


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def reference_or_skip():
    from oracle import reference
    if not reference.available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    return reference


def bits(a, b):
    a = a.detach().cpu().contiguous()
    b = b.detach().cpu().contiguous()
    return int((a.view(torch.int32) != b.view(torch.int32)).sum())


def _scene(method, seed=91, lattice=(10, 10, 10), boundary=False, box_velocity=(0.0, 0.0, 0.0), velocity_sigma=0.2):
    sc = scenes.sph_dam_break(lattice, (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), seed, method=method, velocity_sigma=velocity_sigma)
    if boundary:
        sc = scenes.with_boundary(sc, seed + 1)
    sc.box_velocity = box_velocity
    return sc


def _configuration(method, **overrides):
    values = dict(method=sph.Method[method], pressure_iterations=4, divergence_iterations=3, density_iterations=4)
    values.update(overrides)
    return sph.Configuration(**values)


def _run_pair(sc, method, steps, check_fields=False, **overrides):
    reference = reference_or_skip()
    cfg = _configuration(method, **overrides)
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[method], configuration=cfg)
    cache = solver.allocate_step_cache()
    ref = reference.ReferenceSPH(sc, int(sph.Method[method]), cfg.pressure_iterations, cfg.divergence_iterations,
                                 cfg.density_iterations, pressure_warm_start=cfg.pressure_warm_start)
    dfsph = method == "dfsph"
    rng = np.random.default_rng(5)
    if dfsph:   # non-zero warm starts
        for t in (state.warm_divergence_pressure, state.warm_density_pressure):
            t.copy_(torch.from_numpy(rng.uniform(0, 50, sc.count).astype(np.float32)))
    cur, nxt = state, solver.allocate_state()
    xr, vr = state.positions.clone(), state.velocities.clone()
    xr2, vr2 = torch.zeros_like(xr), torch.zeros_like(vr)
    wr = (state.warm_divergence_pressure.clone(), state.warm_density_pressure.clone()) if dfsph else None
    wr2 = (torch.zeros_like(wr[0]), torch.zeros_like(wr[1])) if dfsph else None
    for k in range(steps):
        solver.forward_step(cur, control, params, nxt, cache)
        ref.forward_step(xr, vr, xr2, vr2, k, warm=wr, warm_out=wr2)
        torch.cuda.synchronize()
        if check_fields:
            _compare_fields(method, cache, ref, k)
        cur, nxt = nxt, cur
        xr, xr2, vr, vr2 = xr2, xr, vr2, vr
        if dfsph:
            wr, wr2 = wr2, wr
        assert bits(cur.positions, xr) == 0, (method, k, float((cur.positions - xr).abs().max()))
        assert bits(cur.velocities, vr) == 0, (method, k, float((cur.velocities - vr).abs().max()))
        if dfsph:
            assert bits(cur.warm_divergence_pressure, wr[0]) == 0, (k, "warm divergence pressure")
            assert bits(cur.warm_density_pressure, wr[1]) == 0, (k, "warm density pressure")
        assert cur.step_index == k + 1
    assert torch.isfinite(cur.positions).all()
    return cur


def _compare_fields(method, cache, ref, step=0):
    F = sph.CacheField
    pairs = [(F.DENSITIES, "densities"), (F.PRESSURES, "pressures"), (F.PRESSURE_ACCELERATIONS, "pressure_accelerations"),
             (F.VISCOSITY_ACCELERATIONS, "viscosity_accelerations")]
    if method == "wcsph":
        pairs.append((F.SURFACE_ACCELERATIONS, "surface_accelerations"))
    else:
        pairs.append((F.PREDICTED_DENSITIES, "predicted_densities"))
    bad = {}
    for field, name in pairs:
        mine, theirs = cache.read(field), ref.read(name)
        torch.cuda.synchronize()
        n = bits(mine, theirs)
        if n:
            bad[name] = (n, float((mine - theirs).abs().max()))
    assert not bad, (method, step, bad)


@pytest.mark.parametrize("method", METHODS)
def test_forward_matches_reference_bit_for_bit(method):
    sc = _scene(method)
    _run_pair(sc, method, 12, check_fields=True)


@pytest.mark.parametrize("method", METHODS)
def test_forward_with_boundary_particles_matches_reference(method):
    sc = _scene(method, seed=92, boundary=True)
    assert len(sc.boundary["volumes"]) > 0
    _run_pair(sc, method, 8, check_fields=True)


@pytest.mark.parametrize("method", ("wcsph", "dfsph"))
def test_moving_box_matches_reference(method):
    """A box translating at (0.2, 0, -0.1) m/s: the grid origin and collision box at t = step dt
    (sph/sph.cpp:21-35, neighborhood/neighborhood.cpp:83-88)."""
    sc = _scene(method, seed=93, boundary=True, box_velocity=(0.2, 0.0, -0.1))
    _run_pair(sc, method, 8, check_fields=True)


@pytest.mark.parametrize("method", ("pcisph", "dfsph"))
def test_large_displacements_walk_the_stencil(method):
    """Velocities of 20 m/s move the predictions 0.3 h, beyond the lists' skin: the predicted
    densities walk the full stencil instead of replaying the lists, with the same results."""
    sc = _scene(method, seed=96, boundary=True, velocity_sigma=20.0)
    _run_pair(sc, method, 4, check_fields=True)


@pytest.mark.parametrize("method,overrides", [("pcisph", {"pressure_iterations": 0}), ("iisph", {"pressure_iterations": 1}),
                                              ("dfsph", {"divergence_iterations": 0, "density_iterations": 2}),
                                              ("dfsph", {"divergence_iterations": 2, "density_iterations": 0}),
                                              ("dfsph", {"pressure_warm_start": False})])
def test_iteration_counts_and_warm_start(method, overrides):
    """Zero and one pressure iterations, empty DFSPH phases and DFSPH without warm starts."""
    _run_pair(_scene(method, seed=97, boundary=True), method, 4, check_fields=True, **overrides)


@pytest.mark.parametrize("method", ("wcsph", "pcisph"))
def test_slip_box_matches_reference(method):
    """A box without no-slip: colliding particles keep their tangential velocities (sph/common.cu:313-319);
    a fast scene drives many of them into the walls."""
    sc = _scene(method, seed=98, velocity_sigma=3.0)
    sc.no_slip = False
    _run_pair(sc, method, 6)


def test_crowded_cells_overflow_the_lists():
    """216 particles packed into one corner overflow the stored lists; the walk fallback gives the
    same sums in the same order."""
    sc = scenes.sph_dam_break((6, 6, 6), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), 94, method="pcisph")
    rng = np.random.default_rng(12)
    sc.positions[:] = (np.array([[0.5], [0.02], [0.5]]) + rng.uniform(0, 0.02, sc.positions.shape)).astype(np.float32)
    _run_pair(sc, "pcisph", 3)


def test_reference_gradient_norm_matches_the_reference_host_value():
    reference = reference_or_skip()
    sc = _scene("pcisph")
    solver, _, _, _ = sph.solver_for_scene(sc, sph.Method.pcisph)
    ref = reference.ReferenceSPH(sc, 1)
    a, b = np.float32(solver.reference_gradient_norm), np.float32(ref.reference_gradient_norm)
    assert a.view(np.int32) == b.view(np.int32), (a, b)
    assert a > 0


@pytest.mark.parametrize("shape", [(0, 128, 128), (1, 64, 96), (2, 128, 32)])
def test_launch_shapes_give_identical_results(shape):
    sc = _scene("wcsph", seed=95)
    outs = []
    for s in ((0, 128, 128), shape):
        solver, state, control, params = sph.solver_for_scene(sc, sph.Method.wcsph)
        solver.launch_shape = pbf.LaunchShape(*s)
        cache = solver.allocate_step_cache()
        nxt = solver.allocate_state()
        solver.forward_step(state, control, params, nxt, cache)
        torch.cuda.synchronize()
        outs.append((nxt.positions.clone(), nxt.velocities.clone()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


def test_vjp_needs_a_differentiable_solver():
    sc = _scene("wcsph")
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method.wcsph)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    with pytest.raises(pbf.PBFError) as err:
        solver.vjp_step(state, control, params, nxt, cache, solver.allocate_state_adjoint(), solver.allocate_state_adjoint(),
                        solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint())
    assert err.value.status == 4   # PBF_ERROR_NOT_DIFFERENTIABLE


def test_empty_scene_steps():
    dc = pbf.DomainConfiguration(particle_count=0, time_step=4e-4, support_radius=0.025, particle_radius=0.005,
                                 boundary=pbf.BoxBoundary((0, 0, 0), (1, 2, 1), (0, 0, 0), True))
    for method in sph.Method:
        solver = sph.SPH(dc, sph.Configuration(method=method))
        state, nxt = solver.allocate_state(), solver.allocate_state()
        solver.forward_step(state, solver.allocate_control(), solver.allocate_parameters(), nxt, solver.allocate_step_cache())
        solver.synchronize()
        assert nxt.step_index == 1


@pytest.mark.parametrize("method", METHODS)
def test_benchmark_workload_matches_reference_bit_for_bit(method):
    """The 1,048,576-particle SPH benchmark dam break with the reference's default iteration counts:
    ten substeps equal the reference kernels' bit for bit."""
    reference = reference_or_skip()
    sc = scenes.sph_large(method=method)
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[method])
    cache = solver.allocate_step_cache()
    ref = reference.ReferenceSPH(sc, int(sph.Method[method]))
    n = sc.count
    cur, nxt = state, solver.allocate_state()
    xr, vr = state.positions.clone(), state.velocities.clone()
    xr2, vr2 = torch.zeros_like(xr), torch.zeros_like(vr)
    dfsph = method == "dfsph"
    wr = (torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")) if dfsph else None
    wr2 = (torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")) if dfsph else None
    for k in range(10):
        solver.forward_step(cur, control, params, nxt, cache)
        ref.forward_step(xr, vr, xr2, vr2, k, warm=wr, warm_out=wr2)
        torch.cuda.synchronize()
        cur, nxt = nxt, cur
        xr, xr2, vr, vr2 = xr2, xr, vr2, vr
        if dfsph:
            wr, wr2 = wr2, wr
        assert bits(cur.positions, xr) == 0 and bits(cur.velocities, vr) == 0, (method, k)
        if dfsph:
            assert bits(cur.warm_density_pressure, wr[1]) == 0, (method, k)
    ref.close()
