"""GPU tests of checkpoint recomputation (pbf_set_checkpoint_recompute): step caches that keep every
checkpoint_interval-th Jacobi iterate only, as the reference's StepCache::checkpoints
(pbf/pbf.ixx:54-70, pbf/pbf.cpp:173-182), with vjp_step recomputing each segment before reversing
it (pbf/pbf.cpp:232-245) and jvp_step rerunning the iterations (pbf/pbf.cpp:198-212).  Every
gradient and tangent is bit-identical to the store-everything form."""
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


def _derivatives(sc, interval, recompute, shape=None, s_corr=0.0):
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable,
                                                          checkpoint_interval=interval)
    if s_corr:
        params.tensors["artificial_pressure_strength"].fill_(s_corr)
    if shape is not None:
        solver.launch_shape = shape
    solver.set_checkpoint_recompute(recompute)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    rng = np.random.default_rng(11)
    n = sc.count
    na = pbf.StateAdjoint(torch.from_numpy(rng.normal(size=(3, n))).cuda(), torch.from_numpy(rng.normal(size=(3, n))).cuda())
    pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
    solver.vjp_step(state, control, params, nxt, cache, na, pa, ca, qa)
    st = solver.allocate_state_tangent()
    st.positions.copy_(torch.from_numpy(rng.normal(size=(3, n)).astype(np.float32)))
    st.velocities.copy_(torch.from_numpy(rng.normal(size=(3, n)).astype(np.float32)))
    ct = solver.allocate_control()
    pt = solver.allocate_parameter_tangent()
    for t in pt.tensors.values():
        t.copy_(torch.from_numpy(rng.normal(size=n).astype(np.float32)) * 1e-3)
    nt = solver.allocate_state_tangent()
    solver.jvp_step(state, control, params, nxt, cache, st, ct, pt, nt)
    torch.cuda.synchronize()
    out = {"x": nxt.positions, "v": nxt.velocities, "ax": pa.positions, "av": pa.velocities,
           "actrl": ca.external_accelerations, "tx": nt.positions, "tv": nt.velocities}
    out.update({k: qa.tensors[k] for k in NAMES})
    return {k: t.clone() for k, t in out.items()}


@pytest.mark.parametrize("interval", [1, 2, 3, 5, 7])
def test_recomputed_derivatives_equal_stored_ones(interval):
    """5 Jacobi iterations: segments of 1, 2, 3, 5 and 7 (one segment) iterations."""
    sc = scenes.dam_break((12, 12, 12), (0, 0, 0), (1, 2, 1), 41, 5, velocity_sigma=0.2)
    a = _derivatives(sc, interval, False)
    b = _derivatives(sc, interval, True)
    for k in a:
        assert torch.equal(a[k], b[k]), k


@pytest.mark.parametrize("list_scan", [0, 1, 3])
def test_recomputation_with_every_scan_variant_and_s_corr(list_scan):
    sc = scenes.dam_break((10, 10, 10), (0, 0, 0), (1, 2, 1), 42, 4, velocity_sigma=0.2)
    shape = pbf.LaunchShape(list_scan, 64, 96)
    a = _derivatives(sc, 2, False, shape, s_corr=1e-4)
    b = _derivatives(sc, 2, True, shape, s_corr=1e-4)
    for k in a:
        assert torch.equal(a[k], b[k]), k


def test_recomputation_with_boundary_particles():
    sc = scenes.with_boundary(scenes.dam_break((9, 9, 9), (0, 0, 0), (1, 2, 1), 43, 4, velocity_sigma=0.2), 44)
    a = _derivatives(sc, 3, False)
    b = _derivatives(sc, 3, True)
    for k in a:
        assert torch.equal(a[k], b[k]), k


def test_recompute_cache_is_smaller_and_keeps_only_checkpoints():
    sc = scenes.dam_break((24, 24, 24), (0, 0, 0), (1, 2, 1), 45, 8)
    sizes = {}
    for recompute in (False, True):
        solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable,
                                                              checkpoint_interval=2)
        solver.set_checkpoint_recompute(recompute)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        cache = solver.allocate_step_cache()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        sizes[recompute] = free0 - free1
        nxt = solver.allocate_state()
        solver.forward_step(state, control, params, nxt, cache)
        if recompute:
            for k in (0, 2, 4, 6, 8):
                cache.read_iteration(pbf.IterationField.POSITIONS, k)
            cache.read_iteration(pbf.IterationField.COLLISION_MASKS, 3)
            with pytest.raises(pbf.PBFError):
                cache.read_iteration(pbf.IterationField.POSITIONS, 3)
            with pytest.raises(pbf.PBFError):
                cache.read_iteration(pbf.IterationField.LAMBDAS, 2)
        del cache
    assert sizes[True] * 3 < sizes[False], sizes


def test_forward_mode_solver_rejects_recomputation():
    solver, _, _, _ = pbf.solver_for_scene(scenes.dam_break((4, 4, 4), (0, 0, 0), (1, 2, 1), 46, 2))
    with pytest.raises(pbf.PBFError) as e:
        solver.set_checkpoint_recompute(True)
    assert e.value.status == 4


def test_batched_rollout_gradients_equal_with_recomputation():
    """A two-scene batch, 6-step rollout with trajectory checkpoints every 3 steps: the per-scene
    loss, dL/dv0 and dL/dc are bit-identical with and without in-step recomputation."""
    scs = [scenes.batched_scene(c, 300 + k, 4, velocity_sigma=0.1) for k, c in enumerate((1800, 2600))]
    for k, s in enumerate(scs):
        s.targets = scenes.target_cloud(310 + k, s.count)
    targets = torch.from_numpy(np.concatenate([s.targets for s in scs], axis=1)).cuda()
    out = []
    for recompute in (False, True):
        batch, state, control, params = pbf.batch_for_scenes(scs, mode=pbf.ExecutionMode.differentiable,
                                                             checkpoint_interval=3)
        batch.set_checkpoint_recompute(recompute)
        g = trajectory.loss_and_gradients(batch, state, control, params, targets, 6, 3)
        torch.cuda.synchronize()
        out.append((g.loss, g.initial_velocities.clone(), g.scalar["xsph_viscosity"]))
    assert np.array_equal(np.asarray(out[0][0]), np.asarray(out[1][0]))
    assert torch.equal(out[0][1], out[1][1])
    assert np.array_equal(np.asarray(out[0][2]), np.asarray(out[1][2]))
