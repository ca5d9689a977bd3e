"""GPU tests of the SPH adjoint (SPH<Method>::vjp_step, sph/sph.ixx:361-365) against the
reference's own vjp kernels replayed by the harness (sph/sph.cpp:239-250, 332-373, 445-486,
661-722, with its checkpoint recomputation) after the same forward step: every adjoint output to
FP64 rounding."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes, sph

pytestmark = pytest.mark.gpu

METHODS = ("wcsph", "pcisph", "iisph", "dfsph")
PARTICLE = ("masses", "rest_densities", "viscosities", "surface_tensions")


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def reference_or_skip():
    from oracle import reference
    if not reference.available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    return reference


def rel(a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    s = float(b.abs().max())
    d = float((a - b).abs().max())
    return d / s if s > 0 else d


def _scene(method, seed, boundary=False, box_velocity=(0.0, 0.0, 0.0)):
    sc = scenes.sph_dam_break((8, 8, 8), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), seed, method=method, velocity_sigma=0.2)
    if boundary:
        sc = scenes.with_boundary(sc, seed + 1)
    sc.box_velocity = box_velocity
    return sc


def _compare_vjp(method, sc, tolerance=1e-9, steps_before=1, **overrides):
    reference = reference_or_skip()
    values = dict(method=sph.Method[method], pressure_iterations=3, divergence_iterations=2, density_iterations=3)
    values.update(overrides)
    cfg = sph.Configuration(**values)
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[method], configuration=cfg,
                                                          mode=pbf.ExecutionMode.differentiable)
    ref = reference.ReferenceSPH(sc, int(sph.Method[method]), cfg.pressure_iterations, cfg.divergence_iterations,
                                 cfg.density_iterations, pressure_warm_start=cfg.pressure_warm_start, checkpoint_interval=2,
                                 differentiable=True)
    dfsph = method == "dfsph"
    n = sc.count
    rng = np.random.default_rng(17)
    if dfsph:
        for t in (state.warm_divergence_pressure, state.warm_density_pressure):
            t.copy_(torch.from_numpy(rng.uniform(0, 50, n).astype(np.float32)))
    cache = solver.allocate_step_cache()
    # advance a few steps first (same inputs on both sides), then differentiate one step
    cur, nxt = state, solver.allocate_state()
    for _ in range(steps_before):
        solver.forward_step(cur, control, params, nxt, cache)
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    k = cur.step_index
    x, v = cur.positions.clone(), cur.velocities.clone()
    warm = (cur.warm_divergence_pressure.clone(), cur.warm_density_pressure.clone()) if dfsph else None
    solver.forward_step(cur, control, params, nxt, cache)
    ref.forward_step(x, v, torch.zeros_like(x), torch.zeros_like(v), k, warm=warm,
                     warm_out=(torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")) if dfsph else None)
    torch.cuda.synchronize()
    na = sph.StateAdjoint(torch.from_numpy(rng.normal(size=(3, n))).cuda(), torch.from_numpy(rng.normal(size=(3, n))).cuda(),
                          torch.from_numpy(rng.normal(size=n) * 1e-3).cuda() if dfsph else None,
                          torch.from_numpy(rng.normal(size=n) * 1e-3).cuda() if dfsph else None)
    pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
    solver.vjp_step(cur, control, params, nxt, cache, na, pa, ca, qa)
    z3 = lambda: torch.zeros((3, n), dtype=torch.float64, device="cuda")
    rprev = {"positions": z3(), "velocities": z3()}
    rctrl = z3()
    rq = {k2: torch.zeros(n, dtype=torch.float64, device="cuda") for k2 in sph.PARAMETER_NAMES}
    rwarm = (torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.float64, device="cuda"))
    ref.vjp_step(x, v, {"positions": na.positions, "velocities": na.velocities}, rprev, rctrl, rq, k,
                 next_warm=(na.warm_divergence_pressure, na.warm_density_pressure) if dfsph else None, previous_warm=rwarm)
    torch.cuda.synchronize()
    errors = {"positions": rel(pa.positions, rprev["positions"]), "velocities": rel(pa.velocities, rprev["velocities"]),
              "control": rel(ca.external_accelerations, rctrl)}
    for name in PARTICLE + sph.METHOD_PARAMETERS[method]:
        errors[name] = rel(qa.tensors[name], rq[name])
    if dfsph and cfg.pressure_warm_start:
        errors["warm_divergence"] = rel(pa.warm_divergence_pressure, rwarm[0])
        errors["warm_density"] = rel(pa.warm_density_pressure, rwarm[1])
    bad = {key: value for key, value in errors.items() if not value < tolerance}
    assert not bad, (method, bad, errors)
    assert float(pa.positions.abs().max()) > 0


@pytest.mark.parametrize("method", METHODS)
def test_vjp_matches_reference(method):
    _compare_vjp(method, _scene(method, 101))


@pytest.mark.parametrize("method,overrides", [("pcisph", {"pressure_iterations": 0}), ("iisph", {"pressure_iterations": 5}),
                                              ("dfsph", {"divergence_iterations": 0, "density_iterations": 1}),
                                              ("dfsph", {"pressure_warm_start": False})])
def test_vjp_iteration_counts_and_warm_start(method, overrides):
    """Zero iterations, odd counts across the reference's checkpoint interval, DFSPH without warm starts."""
    _compare_vjp(method, _scene(method, 109, boundary=True), **overrides)


@pytest.mark.parametrize("method", METHODS)
def test_vjp_with_boundary_particles_matches_reference(method):
    _compare_vjp(method, _scene(method, 103, boundary=True, box_velocity=(0.1, 0.0, 0.0)), steps_before=2)


def _compare_jvp(method, sc, tolerance=1e-4):
    reference = reference_or_skip()
    cfg = sph.Configuration(method=sph.Method[method], pressure_iterations=3, divergence_iterations=2, density_iterations=3)
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[method], configuration=cfg,
                                                          mode=pbf.ExecutionMode.differentiable)
    ref = reference.ReferenceSPH(sc, int(sph.Method[method]), cfg.pressure_iterations, cfg.divergence_iterations,
                                 cfg.density_iterations, checkpoint_interval=2, differentiable=True)
    dfsph = method == "dfsph"
    n = sc.count
    rng = np.random.default_rng(23)
    if dfsph:
        for t in (state.warm_divergence_pressure, state.warm_density_pressure):
            t.copy_(torch.from_numpy(rng.uniform(0, 50, n).astype(np.float32)))
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    x, v = state.positions.clone(), state.velocities.clone()
    warm = (state.warm_divergence_pressure.clone(), state.warm_density_pressure.clone()) if dfsph else None
    solver.forward_step(state, control, params, nxt, cache)
    ref.forward_step(x, v, torch.zeros_like(x), torch.zeros_like(v), 0, warm=warm,
                     warm_out=(torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")) if dfsph else None)
    f32 = lambda a: torch.from_numpy(np.asarray(a, dtype=np.float32)).cuda()
    st = sph.StateTangent(f32(rng.normal(size=(3, n)) * 1e-3), f32(rng.normal(size=(3, n)) * 1e-2),
                          f32(rng.normal(size=n)) if dfsph else None, f32(rng.normal(size=n)) if dfsph else None)
    ct = pbf.Control(f32(rng.normal(size=(3, n))))
    pt = solver.allocate_parameter_tangent()
    pt.tensors["rest_densities"].copy_(f32(rng.normal(size=n)))
    pt.tensors["masses"].copy_(f32(rng.normal(size=n) * 1e-7))
    pt.tensors["viscosities"].copy_(f32(rng.normal(size=n) * 1e-3))
    pt.tensors["surface_tensions"].copy_(f32(rng.normal(size=n) * 1e-3))
    for name in sph.METHOD_PARAMETERS[method]:
        pt.tensors[name].copy_(f32(rng.normal(size=n) * 1e-2))
    out = solver.allocate_state_tangent()
    solver.jvp_step(state, control, params, nxt, cache, st, ct, pt, out)
    tout = {"positions": torch.zeros_like(x), "velocities": torch.zeros_like(v)}
    nwt = (torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda"))
    ref.jvp_step(x, v, {"positions": st.positions, "velocities": st.velocities}, ct.external_accelerations, pt.tensors, tout, 0,
                 warm=warm, warm_tangent=(st.warm_divergence_pressure, st.warm_density_pressure) if dfsph else None,
                 next_warm_tangent=nwt)
    torch.cuda.synchronize()
    errors = {"positions": rel(out.positions, tout["positions"]), "velocities": rel(out.velocities, tout["velocities"])}
    if dfsph:
        errors["warm_divergence"] = rel(out.warm_divergence_pressure, nwt[0])
        errors["warm_density"] = rel(out.warm_density_pressure, nwt[1])
    bad = {key: value for key, value in errors.items() if not value < tolerance}
    assert not bad, (method, bad, errors)
    assert float(out.velocities.abs().max()) > 0


@pytest.mark.parametrize("method", METHODS)
def test_jvp_matches_reference(method):
    _compare_jvp(method, _scene(method, 105))


@pytest.mark.parametrize("method", METHODS)
def test_jvp_with_boundary_particles_matches_reference(method):
    _compare_jvp(method, _scene(method, 107, boundary=True))


@pytest.mark.parametrize("method", ("wcsph", "dfsph"))
def test_state_copies_and_adjoint_accumulation(method):
    """copy_state / copy_state_tangent / copy_state_adjoint / accumulate_state_adjoint
    (sph/sph.ixx:326-345), DFSPH's warm-start fields included."""
    sc = _scene(method, 111)
    solver, state, _, _ = sph.solver_for_scene(sc, sph.Method[method], mode=pbf.ExecutionMode.differentiable)
    dfsph = method == "dfsph"
    if dfsph:
        state.warm_divergence_pressure.uniform_(0, 5)
        state.warm_density_pressure.uniform_(0, 5)
    state.step_index = 7
    copy = solver.allocate_state()
    solver.copy_state(state, copy)
    assert copy.step_index == 7 and torch.equal(copy.positions, state.positions) and torch.equal(copy.velocities, state.velocities)
    if dfsph:
        assert torch.equal(copy.warm_density_pressure, state.warm_density_pressure)
    t = solver.allocate_state_tangent()
    t.positions.normal_()
    if dfsph:
        t.warm_divergence_pressure.normal_()
    t2 = solver.allocate_state_tangent()
    solver.copy_state_tangent(t, t2)
    assert torch.equal(t2.positions, t.positions)
    if dfsph:
        assert torch.equal(t2.warm_divergence_pressure, t.warm_divergence_pressure)
    a, b = solver.allocate_state_adjoint(), solver.allocate_state_adjoint()
    a.positions.normal_()
    a.velocities.normal_()
    b.positions.normal_()
    if dfsph:
        a.warm_density_pressure.normal_()
        b.warm_density_pressure.normal_()
    expected = b.positions + a.positions
    expected_warm = (b.warm_density_pressure + a.warm_density_pressure) if dfsph else None
    solver.accumulate_state_adjoint(a, b)
    torch.cuda.synchronize()
    assert torch.equal(b.positions, expected)
    if dfsph:
        assert torch.equal(b.warm_density_pressure, expected_warm)
    c = solver.allocate_state_adjoint()
    solver.copy_state_adjoint(a, c)
    torch.cuda.synchronize()
    assert torch.equal(c.velocities, a.velocities)
