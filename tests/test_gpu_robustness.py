"""GPU tests of determinism and of the host-visible failure paths (no GPU fault is provoked):
repeated runs are bit-identical, an empty scene steps, an allocation that cannot fit is reported
as PBF_ERROR_OUT_OF_MEMORY and the solver stays usable, and a step cache is tied to its solver."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def _run(sc, steps, graphs=False):
    solver, state, control, params = pbf.solver_for_scene(sc)
    solver.set_graph_mode(graphs)
    cache = solver.allocate_step_cache()
    cur, nxt = state, solver.allocate_state()
    for _ in range(steps):
        solver.forward_step(cur, control, params, nxt, cache)
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    return cur.positions.clone(), cur.velocities.clone()


def test_repeated_runs_are_bit_identical():
    """The stable counting sort and the fixed summation order make every run reproducible, with
    and without graph replay (atomics only count particles per cell; slots are re-ranked)."""
    sc = scenes.dam_break((14, 14, 14), (0, 0, 0), (1, 2, 1), 81, 4, velocity_sigma=0.2)
    a = _run(sc, 12)
    b = _run(sc, 12)
    c = _run(sc, 12, graphs=True)
    for other in (b, c):
        assert torch.equal(a[0], other[0]) and torch.equal(a[1], other[1])


def test_same_step_twice_from_the_same_state():
    sc = scenes.dam_break((10, 10, 10), (0, 0, 0), (1, 2, 1), 82, 3, velocity_sigma=0.1)
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    outs = []
    for _ in range(2):
        nxt = solver.allocate_state()
        solver.forward_step(state, control, params, nxt, cache)
        torch.cuda.synchronize()
        outs.append((nxt.positions.clone(), nxt.velocities.clone()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


def test_empty_scene_steps():
    dc = pbf.DomainConfiguration(particle_count=0, time_step=1.0 / 120.0, support_radius=0.025, particle_radius=0.005,
                                 boundary=pbf.BoxBoundary((0, 0, 0), (1, 2, 1), (0, 0, 0), True))
    solver = pbf.PBF(dc, pbf.Configuration(4, 2))
    state, nxt = solver.allocate_state(), solver.allocate_state()
    cache = solver.allocate_step_cache()
    solver.forward_step(state, solver.allocate_control(), solver.allocate_parameters(), nxt, cache)
    solver.synchronize()
    assert nxt.step_index == 1


def test_allocation_failure_is_reported_and_the_solver_stays_usable():
    """400M particles: the step cache (about 240 GB) cannot fit in the GPU's memory; the call
    returns PBF_ERROR_OUT_OF_MEMORY and frees what it had allocated."""
    free_before, _ = torch.cuda.mem_get_info()
    n = 400_000_000
    dc = pbf.DomainConfiguration(particle_count=n, time_step=1.0 / 120.0, support_radius=0.025, particle_radius=0.005,
                                 boundary=pbf.BoxBoundary((0, 0, 0), (1, 2, 1), (0, 0, 0), True))
    try:
        solver = pbf.PBF(dc, pbf.Configuration(4, 2))
    except pbf.PBFError as e:            # a smaller GPU already fails at creation
        assert e.status == 2
        return
    with pytest.raises(pbf.PBFError) as err:
        solver.allocate_step_cache()
    assert err.value.status == 2         # PBF_ERROR_OUT_OF_MEMORY
    solver.close()
    torch.cuda.synchronize()
    # the device keeps working: a small scene still steps exactly as before
    sc = scenes.dam_break((6, 6, 6), (0, 0, 0), (1, 2, 1), 83, 2)
    a = _run(sc, 3)
    b = _run(sc, 3)
    assert torch.equal(a[0], b[0])
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after > free_before - (1 << 30)


def test_step_cache_of_another_solver_is_rejected():
    sc = scenes.dam_break((4, 4, 4), (0, 0, 0), (1, 2, 1), 84, 2)
    s1, state, control, params = pbf.solver_for_scene(sc)
    s2, _, _, _ = pbf.solver_for_scene(sc)
    foreign = s2.allocate_step_cache()
    with pytest.raises(pbf.PBFError) as err:
        s1.forward_step(state, control, params, s1.allocate_state(), foreign)
    assert err.value.status == 1         # PBF_ERROR_INVALID_ARGUMENT


def test_vjp_with_a_cache_of_another_step_is_rejected():
    sc = scenes.dam_break((4, 4, 4), (0, 0, 0), (1, 2, 1), 85, 2)
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    later = solver.allocate_state()
    solver.forward_step(nxt, control, params, later, solver.allocate_step_cache())
    na = solver.allocate_state_adjoint()
    with pytest.raises(pbf.PBFError):
        # `cache` holds the step of `state`, not of `nxt`
        solver.vjp_step(nxt, control, params, later, cache, na, solver.allocate_state_adjoint(),
                        solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint())


def test_input_checks_flag_invalid_inputs():
    sc = scenes.dam_break((6, 6, 6), (0, 0, 0), (1, 2, 1), 86, 2)
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.set_input_checks(True)
    solver.forward_step(state, control, params, nxt, cache)
    assert solver.read_input_checks() == 0
    bad = pbf.State(state.positions.clone(), state.velocities.clone(), 0)
    bad.velocities[1, 7] = float("nan")
    bad.positions[0, 3] = float("inf")
    solver.forward_step(bad, control, params, nxt, cache)
    flags = solver.read_input_checks()
    assert flags == pbf.INPUT_NONFINITE_VELOCITY | pbf.INPUT_NONFINITE_POSITION
    assert solver.read_input_checks() == 0          # cleared by the read
    params.tensors["masses"][5] = -1.0
    control.external_accelerations[2, 0] = float("nan")
    solver.forward_step(state, control, params, nxt, cache)
    assert solver.read_input_checks() == pbf.INPUT_BAD_MASS | pbf.INPUT_NONFINITE_CONTROL
    solver.set_input_checks(False)
    solver.forward_step(bad, control, params, nxt, cache)
    assert solver.read_input_checks() == 0          # nothing is tested while disabled
