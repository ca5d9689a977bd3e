"""GPU tests of the batched form: every scene of a batch evolves exactly as its own solver, forward
and adjoint, with or without CUDA-graph replay."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def _scenes(velocity_sigma=0.0):
    counts = [2048, 3001, 777, 5000, 1]
    return [scenes.batched_scene(c, 100 + k, 3, velocity_sigma=velocity_sigma) for k, c in enumerate(counts)]


@pytest.mark.parametrize("graphs", [False, True])
def test_batched_forward_equals_per_scene_solvers(graphs):
    scs = _scenes()
    batch, state, control, params = pbf.batch_for_scenes(scs)
    batch.set_graph_mode(graphs)
    nxt = batch.allocate_state()
    cur = state
    for k in range(6):
        batch.forward_step(cur, control, params, nxt)
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    for s, sc in enumerate(scs):
        solver, st, ctl, prm = pbf.solver_for_scene(sc)
        cache = solver.allocate_step_cache()
        a, b = st, solver.allocate_state()
        for k in range(6):
            solver.forward_step(a, ctl, prm, b, cache)
            a, b = b, a
        sl = batch.particle_range(s)
        assert torch.equal(cur.positions[:, sl], a.positions), s
        assert torch.equal(cur.velocities[:, sl], a.velocities), s
    assert cur.step_index == 6


def test_graph_replay_equals_direct_launches():
    sc = scenes.plain_small(lattice=(12, 12, 12))
    out = []
    for graphs in (False, True):
        solver, state, control, params = pbf.solver_for_scene(sc)
        solver.set_graph_mode(graphs)
        cache = solver.allocate_step_cache()
        cur, nxt = state, solver.allocate_state()
        for k in range(8):
            solver.forward_step(cur, control, params, nxt, cache)
            cur, nxt = nxt, cur
        out.append((cur.positions.clone(), cur.velocities.clone()))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])


def test_batched_vjp_equals_per_scene_vjp():
    scs = _scenes(0.1)[:3]
    batch, state, control, params = pbf.batch_for_scenes(scs, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
    nxt = batch.allocate_state()
    batch.forward_step(state, control, params, nxt, 0)
    rng = np.random.default_rng(4)
    nxa = torch.from_numpy(rng.normal(size=(3, batch.count))).cuda()
    nva = torch.from_numpy(rng.normal(size=(3, batch.count))).cuda()
    na = pbf.StateAdjoint(nxa, nva)
    pa, ca, qa = batch.allocate_state_adjoint(), batch.allocate_control_adjoint(), batch.allocate_parameter_adjoint()
    batch.vjp_step(state, control, params, nxt, 0, na, pa, ca, qa)
    sums = batch.scene_sums(qa.tensors["xsph_viscosity"]).cpu().numpy()
    for s, sc in enumerate(scs):
        sl = batch.particle_range(s)
        solver, st, ctl, prm = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable, checkpoint_interval=1)
        cache = solver.allocate_step_cache()
        b = solver.allocate_state()
        solver.forward_step(st, ctl, prm, b, cache)
        a1 = pbf.StateAdjoint(nxa[:, sl].contiguous(), nva[:, sl].contiguous())
        p1, c1, q1 = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
        solver.vjp_step(st, ctl, prm, b, cache, a1, p1, c1, q1)
        assert torch.equal(pa.positions[:, sl], p1.positions), s
        assert torch.equal(pa.velocities[:, sl], p1.velocities), s
        assert torch.equal(qa.tensors["xsph_viscosity"][sl], q1.tensors["xsph_viscosity"]), s
        assert sums[s] == pytest.approx(float(q1.tensors["xsph_viscosity"].sum()), rel=1e-12)


def test_batched_rollout_gradients_equal_per_scene_rollouts():
    """A checkpointed rollout of a differentiable batch gives every scene exactly the loss, dL/dv0
    and dL/dc of that scene's own rollout."""
    from physica_b200 import trajectory
    scs = [scenes.batched_scene(c, 400 + k, 3, velocity_sigma=0.1) for k, c in enumerate((900, 2100, 1500))]
    targets = [scenes.target_cloud(500 + k, sc.count) for k, sc in enumerate(scs)]
    batch, state, control, params = pbf.batch_for_scenes(scs, mode=pbf.ExecutionMode.differentiable)
    t_all = torch.from_numpy(np.concatenate(targets, axis=1)).cuda()
    g = trajectory.loss_and_gradients(batch, state, control, params, t_all, 5, 2)
    torch.cuda.synchronize()
    for s, sc in enumerate(scs):
        solver, st, ctl, prm = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
        gs = trajectory.loss_and_gradients(solver, st, ctl, prm, torch.from_numpy(targets[s]).cuda(), 5, 2)
        sl = batch.particle_range(s)
        assert g.loss[s] == gs.loss
        assert torch.equal(g.initial_velocities[:, sl], gs.initial_velocities), s
        assert g.scalar["xsph_viscosity"][s] == gs.scalar["xsph_viscosity"], s


def test_benchmark_batch_equals_per_scene_solvers():
    """The 256-scene batched benchmark (2,048-65,536 particles per scene, 4 iterations), autotuned
    and graph-replayed as bench.py runs it, for its full 100 substeps: every scene equals its own
    solver bit for bit, and eight of them (every 32nd) equal the reference's kernels bit for bit."""
    from oracle import reference
    scs = scenes.batched_forward()
    steps = 100
    batch, state, control, params = pbf.batch_for_scenes(scs)
    batch.autotune(state, control, params, repeats=1)
    batch.set_graph_mode(True)
    cur, nxt = pbf.State(state.positions.clone(), state.velocities.clone(), 0), batch.allocate_state()
    for _ in range(steps):
        batch.forward_step(cur, control, params, nxt)
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    for s, sc in enumerate(scs):
        solver, st, ctl, prm = pbf.solver_for_scene(sc)
        solver.set_graph_mode(True)
        cache = solver.allocate_step_cache()
        a, b = st, solver.allocate_state()
        for _ in range(steps):
            solver.forward_step(a, ctl, prm, b, cache)
            a, b = b, a
        sl = batch.particle_range(s)
        assert torch.equal(cur.positions[:, sl], a.positions), s
        assert torch.equal(cur.velocities[:, sl], a.velocities), s
        del solver, cache
    if not reference.available():
        return
    for s in range(0, len(scs), 32):
        ref = reference.ReferencePBF(scs[s])
        x = torch.from_numpy(scs[s].positions).cuda().contiguous()
        v = torch.from_numpy(scs[s].velocities).cuda().contiguous()
        xo, vo = torch.zeros_like(x), torch.zeros_like(v)
        for k in range(steps):
            ref.forward_step(x, v, xo, vo, k)
            x, xo, v, vo = xo, x, vo, v
        torch.cuda.synchronize()
        sl = batch.particle_range(s)
        assert torch.equal(cur.positions[:, sl], x), s
        assert torch.equal(cur.velocities[:, sl], v), s
        ref.close()


def test_batched_adjoint_benchmark_equals_per_scene_rollouts():
    """The 32-scene batched adjoint configuration (16,384-131,072 particles per scene, 4 iterations)
    at its full length: a 100-step rollout with trajectory checkpoints every 10 gives every scene
    exactly the loss, dL/dv0 and dL/dc of that scene's own rollout."""
    import gc
    from physica_b200 import trajectory
    scs = scenes.batched_adjoint()
    steps, every = 100, 10
    diff = pbf.ExecutionMode.differentiable
    batch, state, control, params = pbf.batch_for_scenes(scs, mode=diff)
    targets = torch.from_numpy(np.concatenate([sc.targets for sc in scs], axis=1)).cuda()
    g = trajectory.loss_and_gradients(batch, state, control, params, targets, steps, every)
    torch.cuda.synchronize()
    ranges = [batch.particle_range(s) for s in range(len(scs))]
    velocities = g.initial_velocities.clone()
    losses, viscosity = list(g.loss), list(g.scalar["xsph_viscosity"])
    del g, batch, state, control, params, targets
    gc.collect()
    for s, sc in enumerate(scs):
        solver, st, ctl, prm = pbf.solver_for_scene(sc, mode=diff)
        gs = trajectory.loss_and_gradients(solver, st, ctl, prm, torch.from_numpy(sc.targets).cuda(), steps, every)
        assert losses[s] == gs.loss, s
        assert torch.equal(velocities[:, ranges[s]], gs.initial_velocities), s
        assert viscosity[s] == gs.scalar["xsph_viscosity"], s
        del solver, gs
        gc.collect()
