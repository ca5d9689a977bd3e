"""GPU tests of the adjoint: one substep against the reference's VJP kernels and the FP64 oracle,
central finite differences of the FP64 forward, and a checkpointed multi-step rollout."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes, trajectory

pytestmark = pytest.mark.gpu

NAMES = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
         "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def my_vjp(sc, nxa, nva, checkpoint_interval=1):
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable,
                                                          checkpoint_interval=checkpoint_interval)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    na = pbf.StateAdjoint(torch.from_numpy(nxa).cuda(), torch.from_numpy(nva).cuda())
    pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
    solver.vjp_step(state, control, params, nxt, cache, na, pa, ca, qa)
    torch.cuda.synchronize()
    return {"position": pa.positions.cpu().numpy(), "velocity": pa.velocities.cpu().numpy(),
            "control": ca.external_accelerations.cpu().numpy(), **{k: qa.tensors[k].cpu().numpy() for k in NAMES}}


def _scene(lattice=(10, 10, 10), seed=12):
    return scenes.dam_break(lattice, (0, 0, 0), (1, 2, 1), seed, 4, velocity_sigma=0.1)


def reference_vjp(sc, nxa, nva):
    """The reference's forward_step and vjp_step (its own kernels) on the same scene and adjoints."""
    from oracle import reference
    if not reference.available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    ref = reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    ref.forward_step(x, v, xo, vo, 0)
    z3 = lambda: torch.zeros((3, sc.count), dtype=torch.float64, device="cuda")
    prev = {"positions": z3(), "velocities": z3()}
    ctrl = z3()
    pa = {k: torch.zeros(sc.count, dtype=torch.float64, device="cuda") for k in NAMES}
    ref.vjp_step(x, v, {"positions": torch.from_numpy(nxa).cuda(), "velocities": torch.from_numpy(nva).cuda()},
                 prev, ctrl, pa)
    return {"position": prev["positions"].cpu().numpy(), "velocity": prev["velocities"].cpu().numpy(),
            "control": ctrl.cpu().numpy(), **{k: pa[k].cpu().numpy() for k in NAMES}}


COMPARED = ("position", "velocity", "control", "masses", "rest_densities", "relaxation", "artificial_pressure_strength",
            "xsph_viscosity", "vorticity_confinement")


def test_vjp_matches_reference_vjp():
    """The adjoint of one substep equals the reference's vjp_step to FP64 rounding."""
    sc = _scene()
    rng = np.random.default_rng(5)
    nxa, nva = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    mine = my_vjp(sc, nxa, nva)
    theirs = reference_vjp(sc, nxa, nva)
    for k in COMPARED:
        assert rel(mine[k], theirs[k]) < 1e-9, (k, rel(mine[k], theirs[k]))


def test_vjp_of_overflowing_lists_matches_reference_vjp():
    """125 particles packed into a 0.02 m cube: every particle has more neighbours than its stored
    list holds, so each pass walks its stencil (in the reverse passes split between two lanes); the
    adjoint still equals the reference's vjp_step to FP64 rounding."""
    sc = scenes.dam_break((5, 5, 5), (0, 0, 0), (1, 2, 1), 68, 3, velocity_sigma=0.1)
    rng = np.random.default_rng(13)
    sc.positions[:] = (np.array([[0.5], [0.3], [0.5]]) + rng.uniform(0, 0.02, sc.positions.shape)).astype(np.float32)
    p = sc.positions.T.astype(np.float64)
    in_support = (np.sqrt(((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)) < sc.support_radius).sum(1)
    assert in_support.min() > 96   # more than a stored list holds
    nxa, nva = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    mine = my_vjp(sc, nxa, nva)
    theirs = reference_vjp(sc, nxa, nva)
    for k in COMPARED:
        assert rel(mine[k], theirs[k]) < 1e-9, (k, rel(mine[k], theirs[k]))


def test_vjp_matches_fp64_oracle():
    from oracle import oracle
    sc = _scene()
    rng = np.random.default_rng(6)
    nxa, nva = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    mine = my_vjp(sc, nxa, nva)
    o = oracle.vjp_step(sc, sc.positions, sc.velocities, nxa, nva)
    for k in ("position", "velocity", "control", "xsph_viscosity", "vorticity_confinement", "relaxation"):
        assert rel(mine[k], o[k]) < 1e-3, (k, rel(mine[k], o[k]))


def test_vjp_directional_derivative_matches_central_differences():
    """<dL/dv0, dv> of the CUDA adjoint equals the central difference of the FP64 forward (1e-3 relative)."""
    from oracle import oracle
    sc = _scene((8, 8, 8), 13)
    rng = np.random.default_rng(7)
    wx, wv = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    mine = my_vjp(sc, wx, wv)
    x0, v0 = sc.positions.astype(np.float64), sc.velocities.astype(np.float64)

    def loss(x, v):
        x1, v1 = oracle.forward_step(sc, x, v)
        return float((wx * x1).sum() + (wv * v1).sum())

    for target, grad in (("v", mine["velocity"]), ("x", mine["position"])):
        dirn = rng.normal(size=(3, sc.count))
        eps = 1e-6
        if target == "v":
            fd = (loss(x0, v0 + eps * dirn) - loss(x0, v0 - eps * dirn)) / (2 * eps)
        else:
            fd = (loss(x0 + eps * dirn, v0) - loss(x0 - eps * dirn, v0)) / (2 * eps)
        ad = float((grad * dirn).sum())
        assert ad == pytest.approx(fd, rel=1e-3), (target, ad, fd)


def test_vjp_independent_of_checkpoint_interval():
    sc = _scene((8, 8, 8), 14)
    rng = np.random.default_rng(8)
    nxa, nva = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    a = my_vjp(sc, nxa, nva, 1)
    b = my_vjp(sc, nxa, nva, 3)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_rollout_gradient_matches_oracle_chain_along_the_same_trajectory():
    """Checkpointed 8-step rollout: the driver's dL/dv0 and dL/dc equal the FP64 oracle's VJPs chained
    along the GPU's own FP32 trajectory (the dam break is chaotic, so FP32 and FP64 trajectories
    diverge and each has its own gradient; this checks the rollout and checkpoint logic)."""
    from oracle import oracle
    sc = scenes.dam_break((8, 8, 8), (0, 0, 0), (1, 2, 1), 15, 3, velocity_sigma=0.1)
    targets = scenes.target_cloud(15, sc.count)
    steps, every = 8, 3
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
    g = trajectory.loss_and_gradients(solver, state, control, params, torch.from_numpy(targets).cuda(), steps, every)
    # the FP32 trajectory of the GPU
    cache = solver.allocate_step_cache()
    states = [(sc.positions.copy(), sc.velocities.copy())]
    cur = state
    for k in range(steps):
        nxt = solver.allocate_state()
        solver.forward_step(cur, control, params, nxt, cache)
        states.append((nxt.positions.cpu().numpy(), nxt.velocities.cpu().numpy()))
        cur = nxt
    xT = states[-1][0].astype(np.float64)
    ax = 2.0 * (xT - targets) / sc.count
    av = np.zeros_like(ax)
    dc = 0.0
    for k in reversed(range(steps)):
        out = oracle.vjp_step(sc, states[k][0], states[k][1], ax, av, step_index=k)
        ax, av = out["position"], out["velocity"]
        dc += out["xsph_viscosity"].sum()
    assert rel(g.initial_velocities.cpu().numpy(), av) < 1e-3
    assert rel(g.initial_positions.cpu().numpy(), ax) < 1e-3
    assert g.scalar["xsph_viscosity"] == pytest.approx(dc, rel=1e-3)


def test_short_rollout_gradient_matches_fp64_finite_differences():
    """3-step rollout: directional dL/dv0 against converged central differences of the FP64 forward."""
    from oracle import oracle
    sc = scenes.dam_break((8, 8, 8), (0, 0, 0), (1, 2, 1), 16, 3, velocity_sigma=0.1)
    targets = scenes.target_cloud(16, sc.count)
    steps = 3
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
    g = trajectory.loss_and_gradients(solver, state, control, params, torch.from_numpy(targets).cuda(), steps, 2)

    def rollout_loss(v0):
        x, v = sc.positions.astype(np.float64), v0
        for k in range(steps):
            x, v = oracle.forward_step(sc, x, v, step_index=k)
        d = x - targets.astype(np.float64)
        return float((d * d).sum() / sc.count)

    rng = np.random.default_rng(19)
    dirn = rng.normal(size=(3, sc.count))
    v0 = sc.velocities.astype(np.float64)
    eps = 1e-7
    fd = (rollout_loss(v0 + eps * dirn) - rollout_loss(v0 - eps * dirn)) / (2 * eps)
    ad = float((g.initial_velocities.cpu().numpy() * dirn).sum())
    assert ad == pytest.approx(fd, rel=1e-3)


def test_viscosity_gradient_matches_fp64_finite_differences():
    """3-step rollout: the scalar XSPH viscosity gradient dL/dc (c shared by every particle; the
    per-particle adjoints of xsph_vjp_kernel, pbf/pbf.cu:756-794, summed with Neumaier compensation
    in FP64) against central differences of the FP64 forward in c, at two step sizes that agree."""
    from oracle import oracle
    sc = scenes.dam_break((8, 8, 8), (0, 0, 0), (1, 2, 1), 18, 3, velocity_sigma=0.1)
    targets = scenes.target_cloud(18, sc.count)
    steps = 3
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
    g = trajectory.loss_and_gradients(solver, state, control, params, torch.from_numpy(targets).cuda(), steps, 2)
    c = float(sc.xsph_viscosity[0])

    def rollout_loss(cv):
        prm = oracle.Parameters(sc, xsph_override=cv)
        x, v = sc.positions.astype(np.float64), sc.velocities.astype(np.float64)
        for k in range(steps):
            x, v = oracle.forward_step(sc, x, v, step_index=k, params=prm)
        d = x - targets.astype(np.float64)
        return float((d * d).sum() / sc.count)

    fd = [(rollout_loss(c * (1 + r)) - rollout_loss(c * (1 - r))) / (2 * c * r) for r in (1e-2, 1e-3)]
    assert fd[1] == pytest.approx(fd[0], rel=1e-3)   # converged
    assert g.scalar["xsph_viscosity"] == pytest.approx(fd[1], rel=1e-3)


def test_compensated_sum_is_exact_for_a_hard_case():
    solver, state, control, params = pbf.solver_for_scene(scenes.dam_break((2, 2, 2), (0, 0, 0), (1, 2, 1), 1, 1))
    vals = torch.tensor([1e16, 1.0, -1e16, 3.0] * 1000, dtype=torch.float64, device="cuda")
    assert trajectory.compensated_sum(solver, vals).item() == 4000.0


def test_rollout_reuse_and_graph_mode_give_identical_gradients():
    """A reused Rollout, with and without CUDA graph replay of the forward steps, gives bit-identical
    gradients (the graphs replay exactly the launches of the direct path)."""
    sc = scenes.dam_break((8, 8, 8), (0, 0, 0), (1, 2, 1), 17, 3, velocity_sigma=0.1)
    targets = torch.from_numpy(scenes.target_cloud(17, sc.count)).cuda()
    results = []
    for graphs in (False, True):
        solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
        solver.set_graph_mode(graphs)
        r = trajectory.Rollout(solver, control, params, 7, 3)
        for _ in range(2):
            g = trajectory.loss_and_gradients(solver, state, control, params, targets, 7, rollout=r)
            results.append((g.loss, g.initial_velocities.cpu().numpy().copy(), g.initial_positions.cpu().numpy().copy(),
                            g.scalar["xsph_viscosity"]))
    for other in results[1:]:
        assert other[0] == results[0][0]
        assert np.array_equal(other[1], results[0][1])
        assert np.array_equal(other[2], results[0][2])
        assert other[3] == results[0][3]


def test_benchmark_rollout_gradient_matches_reference_rollout():
    """The 65,536-particle differentiable configuration at its full length (60 steps, 4 iterations,
    trajectory checkpoints every 10): the checkpointed rollout gradient equals the one chained
    through the reference's own forward_step / vjp_step to FP64 rounding."""
    from oracle import reference
    if not reference.available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    sc = scenes.differentiable()
    steps, every = 60, 10
    n = sc.count
    targets = torch.from_numpy(sc.targets).cuda()
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
    mine = trajectory.loss_and_gradients(solver, state, control, params, targets, steps, every)
    torch.cuda.synchronize()

    refs = [reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True) for _ in range(every)]
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    checkpoints = []
    for k in range(steps):
        if k % every == 0:
            checkpoints.append((x.clone(), v.clone()))
        xo, vo = torch.empty_like(x), torch.empty_like(v)
        refs[k % every].forward_step(x, v, xo, vo, k)
        x, v = xo, vo
    diff = x.double() - targets.double()
    assert abs(float((diff * diff).sum() / n) - mine.loss) <= 1e-12 * abs(mine.loss)   # bit-identical trajectory
    adj = {"positions": diff * (2.0 / n), "velocities": torch.zeros((3, n), dtype=torch.float64, device="cuda")}
    pa = {k: torch.zeros(n, dtype=torch.float64, device="cuda") for k in NAMES}
    ctrl = torch.zeros((3, n), dtype=torch.float64, device="cuda")
    for seg in reversed(range(len(checkpoints))):
        xs, vs = [checkpoints[seg][0]], [checkpoints[seg][1]]
        begin = seg * every
        for k in range(begin, min(begin + every, steps)):
            xo, vo = torch.empty_like(xs[-1]), torch.empty_like(vs[-1])
            refs[k - begin].forward_step(xs[-1], vs[-1], xo, vo, k)
            xs.append(xo)
            vs.append(vo)
        for k in reversed(range(begin, min(begin + every, steps))):
            j = k - begin
            prev = {"positions": torch.zeros((3, n), dtype=torch.float64, device="cuda"),
                    "velocities": torch.zeros((3, n), dtype=torch.float64, device="cuda")}
            refs[j].vjp_step(xs[j], vs[j], adj, prev, ctrl, pa)
            adj = prev
    torch.cuda.synchronize()
    print("relative differences:", rel(mine.initial_positions.cpu().numpy(), adj["positions"].cpu().numpy()),
          rel(mine.initial_velocities.cpu().numpy(), adj["velocities"].cpu().numpy()))
    assert rel(mine.initial_positions.cpu().numpy(), adj["positions"].cpu().numpy()) < 1e-7
    assert rel(mine.initial_velocities.cpu().numpy(), adj["velocities"].cpu().numpy()) < 1e-7
    assert rel(mine.controls.cpu().numpy(), ctrl.cpu().numpy()) < 1e-7
    for k in ("masses", "rest_densities", "relaxation", "xsph_viscosity", "vorticity_confinement"):
        assert rel(mine.parameters.tensors[k].cpu().numpy(), pa[k].cpu().numpy()) < 1e-7, k
    for r in refs:
        r.close()
