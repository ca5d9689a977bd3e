"""GPU tests of boundary particles (the reference's BoundaryView terms of density, lambda and
correction, pbf/pbf.cu:118-121,278-285, density/density.cu:34-37) against the reference's own
kernels run through the harness on the same inputs: the forward substep bit for bit, the adjoint
to FP64 rounding, the tangent to FP32 rounding; a moving floor plate checks the time terms."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes

pytestmark = pytest.mark.gpu

NAMES = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
         "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")


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


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def _scene(seed=61, lattice=(10, 10, 10), strength=0.0):
    sc = scenes.dam_break(lattice, (0, 0, 0), (1, 2, 1), seed, 3, velocity_sigma=0.1)
    sc.artificial_pressure_strength[:] = strength
    return scenes.with_boundary(sc, seed + 1)


@pytest.mark.parametrize("strength", [0.0, 0.1])
def test_forward_with_boundary_particles_matches_reference_bit_for_bit(strength):
    """20 substeps with a sliding floor plate and a static wall (with and without s_corr)."""
    reference = reference_or_skip()
    sc = _scene(strength=strength)
    assert len(sc.boundary["volumes"]) > 0
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    ref = reference.ReferencePBF(sc)
    cur, nxt = state, solver.allocate_state()
    xr, vr = state.positions.clone(), state.velocities.clone()
    xr2, vr2 = torch.zeros_like(xr), torch.zeros_like(vr)
    for k in range(20):
        solver.forward_step(cur, control, params, nxt, cache)
        ref.forward_step(xr, vr, xr2, vr2, k)
        torch.cuda.synchronize()
        cur, nxt = nxt, cur
        xr, xr2, vr, vr2 = xr2, xr, vr2, vr
        assert bits(cur.positions, xr) == 0, (k, float((cur.positions - xr).abs().max()))
        assert bits(cur.velocities, vr) == 0, (k, float((cur.velocities - vr).abs().max()))


def test_boundary_particles_change_the_substep():
    """The boundary terms are active: the same scene without its boundary particles differs."""
    sc = _scene(62)
    with_b = pbf.solver_for_scene(sc)
    bare = scenes.dam_break((10, 10, 10), (0, 0, 0), (1, 2, 1), 62, 3, velocity_sigma=0.1)
    without = pbf.solver_for_scene(bare)
    outs = []
    for solver, state, control, params in (with_b, without):
        nxt = solver.allocate_state()
        solver.forward_step(state, control, params, nxt, solver.allocate_step_cache())
        outs.append(nxt.positions.cpu())
    assert not torch.equal(outs[0], outs[1])


def test_vjp_with_boundary_particles_matches_reference():
    reference = reference_or_skip()
    sc = _scene(63)
    rng = np.random.default_rng(9)
    nxa, nva = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    na = pbf.StateAdjoint(torch.from_numpy(nxa).cuda(), torch.from_numpy(nva).cuda())
    pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
    solver.vjp_step(state, control, params, nxt, cache, na, pa, ca, qa)
    ref = reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    ref.forward_step(x, v, torch.zeros_like(x), torch.zeros_like(v), 0)
    z3 = lambda: torch.zeros((3, sc.count), dtype=torch.float64, device="cuda")
    prev = {"positions": z3(), "velocities": z3()}
    ctrl = z3()
    rpa = {k: torch.zeros(sc.count, dtype=torch.float64, device="cuda") for k in NAMES}
    ref.vjp_step(x, v, {"positions": torch.from_numpy(nxa).cuda(), "velocities": torch.from_numpy(nva).cuda()},
                 prev, ctrl, rpa)
    torch.cuda.synchronize()
    assert rel(pa.positions.cpu(), prev["positions"].cpu()) < 1e-9
    assert rel(pa.velocities.cpu(), prev["velocities"].cpu()) < 1e-9
    assert rel(ca.external_accelerations.cpu(), ctrl.cpu()) < 1e-9
    for k in ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "xsph_viscosity"):
        assert rel(qa.tensors[k].cpu(), rpa[k].cpu()) < 1e-9, k


def test_jvp_with_boundary_particles_matches_reference():
    reference = reference_or_skip()
    sc = _scene(64)
    rng = np.random.default_rng(10)
    n = sc.count
    t = {"positions": (rng.normal(size=(3, n)) * 1e-3).astype(np.float32),
         "velocities": (rng.normal(size=(3, n)) * 1e-2).astype(np.float32),
         "control": rng.normal(size=(3, n)).astype(np.float32)}
    pt = {k: np.zeros(n, dtype=np.float32) for k in NAMES}
    pt["rest_densities"] = rng.normal(size=n).astype(np.float32)
    pt["artificial_pressure_strength"] = (rng.normal(size=n) * 1e-3).astype(np.float32)
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    st = pbf.StateTangent(torch.from_numpy(t["positions"]).cuda(), torch.from_numpy(t["velocities"]).cuda())
    ptt = solver.allocate_parameter_tangent()
    for k in NAMES:
        ptt.tensors[k].copy_(torch.from_numpy(pt[k]))
    out = solver.allocate_state_tangent()
    solver.jvp_step(state, control, params, nxt, cache, st, pbf.Control(torch.from_numpy(t["control"]).cuda()), ptt, out)
    ref = reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    ref.forward_step(x, v, torch.zeros_like(x), torch.zeros_like(v), 0)
    tout = {"positions": torch.zeros_like(x), "velocities": torch.zeros_like(v)}
    ref.jvp_step(x, v, {"positions": st.positions, "velocities": st.velocities}, torch.from_numpy(t["control"]).cuda(),
                 {k: torch.from_numpy(pt[k]).cuda() for k in NAMES}, tout)
    torch.cuda.synchronize()
    assert rel(out.positions.cpu(), tout["positions"].cpu()) < 1e-4
    assert rel(out.velocities.cpu(), tout["velocities"].cpu()) < 1e-4


def test_batched_scenes_with_boundary_particles_equal_per_scene_solvers():
    scs = [scenes.with_boundary(scenes.batched_scene(c, 600 + k, 3, velocity_sigma=0.1), 700 + k)
           for k, c in enumerate((800, 1500))]
    scs.append(scenes.batched_scene(900, 602, 3))   # one scene without boundary particles
    batch, state, control, params = pbf.batch_for_scenes(scs)
    cur, nxt = state, batch.allocate_state()
    for _ in range(5):
        batch.forward_step(cur, control, params, nxt)
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    for s, sc in enumerate(scs):
        solver, st, ctl, prm = pbf.solver_for_scene(sc)
        cache = solver.allocate_step_cache()
        a, b = st, solver.allocate_state()
        for _ in range(5):
            solver.forward_step(a, ctl, prm, b, cache)
            a, b = b, a
        sl = batch.particle_range(s)
        assert torch.equal(cur.positions[:, sl], a.positions), s
        assert torch.equal(cur.velocities[:, sl], a.velocities), s


def test_crowded_cells_with_boundary_particles_walk_in_order():
    """125 fluid particles packed just above the floor plate overflow the stored lists; the
    overflow walk visits each cell's boundary particles after its fluid ones, like the reference."""
    reference = reference_or_skip()
    sc = scenes.dam_break((5, 5, 5), (0, 0, 0), (1, 2, 1), 65, 3)
    rng = np.random.default_rng(11)
    sc.positions[:] = (np.array([[0.5], [0.01], [0.5]]) + rng.uniform(0, 0.02, sc.positions.shape)).astype(np.float32)
    sc = scenes.with_boundary(sc, 66)
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    ref = reference.ReferencePBF(sc)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    ref.forward_step(x, v, xo, vo, 0)
    torch.cuda.synchronize()
    assert bits(nxt.positions, xo) == 0
    assert bits(nxt.velocities, vo) == 0


def test_moving_box_matches_reference_bit_for_bit():
    """A box translating at (0.2, 0, -0.1) m/s with boundary particles: the time terms of the key,
    the gather origin and the collision box (pbf/pbf.cpp:17-31, neighborhood.cpp:83-88)."""
    reference = reference_or_skip()
    sc = _scene(67)
    sc.box_velocity = (0.2, 0.0, -0.1)
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    ref = reference.ReferencePBF(sc)
    cur, nxt = state, solver.allocate_state()
    xr, vr = state.positions.clone(), state.velocities.clone()
    xr2, vr2 = torch.zeros_like(xr), torch.zeros_like(vr)
    for k in range(15):
        solver.forward_step(cur, control, params, nxt, cache)
        ref.forward_step(xr, vr, xr2, vr2, k)
        torch.cuda.synchronize()
        cur, nxt = nxt, cur
        xr, xr2, vr, vr2 = xr2, xr, vr2, vr
        assert bits(cur.positions, xr) == 0, k
        assert bits(cur.velocities, vr) == 0, k
