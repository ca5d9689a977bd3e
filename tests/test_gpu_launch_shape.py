"""GPU tests of the launch shapes and the autotuner: every shape of the list and gather kernels
gives bit-identical substeps, for one scene and for a batch, and the autotuner keeps a valid shape."""
import itertools

import pytest
import torch

from physica_b200 import pbf, scenes

pytestmark = pytest.mark.gpu

SHAPES = [pbf.LaunchShape(v, b, g) for v, b, g in itertools.product((0, 1, 2, 3, 4), (32, 64, 96, 128), (32, 64, 96, 128))]


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def _run(solver, state, control, params, steps):
    cache = solver.allocate_step_cache()
    cur = pbf.State(state.positions.clone(), state.velocities.clone(), state.step_index)
    nxt = solver.allocate_state()
    for _ in range(steps):
        solver.forward_step(cur, control, params, nxt, cache)
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    return cur.positions.clone(), cur.velocities.clone()


def test_every_shape_gives_identical_substeps():
    sc = scenes.dam_break((14, 14, 14), (0, 0, 0), (1, 2, 1), 31, 3, velocity_sigma=0.1)
    solver, state, control, params = pbf.solver_for_scene(sc)
    results = []
    for shape in SHAPES[::3]:
        solver.launch_shape = shape
        assert solver.launch_shape == shape
        results.append(_run(solver, state, control, params, 5))
    for shape, (x, v) in zip(SHAPES[::3][1:], results[1:]):
        assert torch.equal(x, results[0][0]), shape
        assert torch.equal(v, results[0][1]), shape


def test_invalid_shapes_are_rejected():
    solver, _, _, _ = pbf.solver_for_scene(scenes.dam_break((4, 4, 4), (0, 0, 0), (1, 2, 1), 32, 2))
    for bad in (pbf.LaunchShape(5, 128, 128), pbf.LaunchShape(0, 48, 128), pbf.LaunchShape(0, 128, 256),
                pbf.LaunchShape(1, 0, 64)):
        with pytest.raises(pbf.PBFError):
            solver.launch_shape = bad


def test_autotune_keeps_a_valid_shape_and_identical_results():
    sc = scenes.dam_break((16, 16, 16), (0, 0, 0), (1, 2, 1), 33, 3)
    solver, state, control, params = pbf.solver_for_scene(sc)
    before = _run(solver, state, control, params, 3)
    shape, ms = solver.autotune(state, control, params, repeats=1)
    assert shape in SHAPES and ms > 0.0
    assert solver.launch_shape == shape
    after = _run(solver, state, control, params, 3)
    assert torch.equal(before[0], after[0]) and torch.equal(before[1], after[1])


def test_batch_autotune_and_shapes_give_identical_substeps():
    scs = [scenes.batched_scene(c, 200 + k, 3) for k, c in enumerate((1500, 4000, 257))]
    batch, state, control, params = pbf.batch_for_scenes(scs)
    out = []
    for shape in (pbf.LaunchShape(0, 128, 128), pbf.LaunchShape(1, 64, 96), pbf.LaunchShape(2, 128, 64),
                  pbf.LaunchShape(3, 96, 128), pbf.LaunchShape(4, 64, 32)):
        batch.launch_shape = shape
        cur = pbf.State(state.positions.clone(), state.velocities.clone(), 0)
        nxt = batch.allocate_state()
        for _ in range(4):
            batch.forward_step(cur, control, params, nxt)
            cur, nxt = nxt, cur
        torch.cuda.synchronize()
        out.append((cur.positions.clone(), cur.velocities.clone()))
    for other in out[1:]:
        assert torch.equal(out[0][0], other[0]) and torch.equal(out[0][1], other[1])
    shape, ms = batch.autotune(state, control, params, repeats=1)
    assert shape in SHAPES and ms > 0.0


def test_fused_density_records_the_same_iterates_for_the_adjoint():
    """Differentiable mode: the fused scan + density/lambda kernel records the same densities,
    gradient sums and lambdas as the two-kernel path, so the adjoint is bit-identical."""
    import numpy as np
    sc = scenes.dam_break((12, 12, 12), (0, 0, 0), (1, 2, 1), 34, 3, velocity_sigma=0.2)
    rng = np.random.default_rng(7)
    wx = torch.from_numpy(rng.normal(size=(3, sc.count))).cuda()
    wv = torch.from_numpy(rng.normal(size=(3, sc.count))).cuda()
    out = []
    for shape in (pbf.LaunchShape(0, 128, 128), pbf.LaunchShape(3, 64, 128)):
        solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
        solver.launch_shape = shape
        cache = solver.allocate_step_cache()
        nxt = solver.allocate_state()
        solver.forward_step(state, control, params, nxt, cache)
        pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
        solver.vjp_step(state, control, params, nxt, cache, pbf.StateAdjoint(wx, wv), pa, ca, qa)
        torch.cuda.synchronize()
        fields = [cache.read_iteration(pbf.IterationField.DENSITIES, k) for k in range(3)]
        fields += [cache.read_iteration(pbf.IterationField.LAMBDAS, k) for k in range(3)]
        fields += [cache.read_iteration(pbf.IterationField.GRADIENT_SUMS, k) for k in range(3)]
        out.append((nxt.positions.clone(), nxt.velocities.clone(), pa.positions.clone(), pa.velocities.clone(), fields))
    a, b = out
    for x, y in zip(a[:4], b[:4]):
        assert torch.equal(x, y)
    for x, y in zip(a[4], b[4]):
        assert torch.equal(x, y)


def test_hit_mask_lists_equal_index_lists_over_a_long_run_and_when_crowded():
    """Launch-shape variant 4 stores each neighbour list as (slot base, 32-bit hit mask) pairs: 60
    steps of a 3,375-particle dam break, and 3 steps of a clump eight times denser than the lattice
    (its hit-mask lists overflow and walk the stencil), equal the index-list solver bit for bit."""
    sc = scenes.dam_break((15, 15, 15), (0, 0, 0), (1, 2, 1), 35, 4, velocity_sigma=0.2)
    crowded = scenes.dam_break((16, 16, 16), (0, 0, 0), (1, 2, 1), 36, 3)
    crowded.positions = (crowded.positions * 0.5 + 0.1).astype(crowded.positions.dtype)
    for scene, steps in ((sc, 60), (crowded, 3)):
        out = []
        for shape in (pbf.LaunchShape(3, 128, 128), pbf.LaunchShape(4, 128, 128), pbf.LaunchShape(4, 32, 64)):
            solver, state, control, params = pbf.solver_for_scene(scene)
            solver.launch_shape = shape
            out.append(_run(solver, state, control, params, steps))
        for x, v in out[1:]:
            assert torch.equal(x, out[0][0]) and torch.equal(v, out[0][1])


def test_hit_mask_lists_with_no_particles_and_no_iterations():
    """An empty scene and a scene with zero Jacobi iterations (only the post-loop list) step with
    hit-mask lists, the latter equal to index lists bit for bit."""
    dc = pbf.DomainConfiguration(particle_count=0, time_step=1.0 / 120.0, support_radius=0.025, particle_radius=0.005,
                                 boundary=pbf.BoxBoundary((0, 0, 0), (1, 2, 1), (0, 0, 0), True))
    solver = pbf.PBF(dc, pbf.Configuration(4, 2))
    solver.launch_shape = pbf.LaunchShape(4, 128, 128)
    state, nxt = solver.allocate_state(), solver.allocate_state()
    solver.forward_step(state, solver.allocate_control(), solver.allocate_parameters(), nxt, solver.allocate_step_cache())
    solver.synchronize()
    assert nxt.step_index == 1
    sc = scenes.dam_break((10, 10, 10), (0, 0, 0), (1, 2, 1), 37, 0, velocity_sigma=0.3)
    out = []
    for shape in (pbf.LaunchShape(0, 128, 128), pbf.LaunchShape(4, 128, 128)):
        solver, state, control, params = pbf.solver_for_scene(sc)
        solver.launch_shape = shape
        out.append(_run(solver, state, control, params, 3))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
