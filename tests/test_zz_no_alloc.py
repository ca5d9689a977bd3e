"""GPU tests of pbf_forward_step_preallocated, the forward substep that allocates no device memory.

Called through the C ABI (ctypes on the library) and compared with pbf_forward_step of a
forward-mode solver on the same inputs: bit-identical positions and velocities, the tolerance of
every forward parity test here, on two calls in a row.  This file runs last so that the first call
on the device may come either from a fresh process or after every other GPU test.
"""
import ctypes

import pytest
import torch

from physica_b200 import pbf, scenes

pytestmark = pytest.mark.gpu

PBF_ERROR_CAPACITY = 7


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def _entry():
    lib = pbf.library()
    fn = lib.pbf_forward_step_preallocated
    P = ctypes.POINTER
    fn.argtypes = [P(pbf.DomainConfigurationC), P(pbf.ConfigurationC), P(pbf.ParticleStateC), P(pbf.ControlC),
                   P(pbf.ParametersC), P(pbf.ParticleStateC), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _preallocated_step(fn, dc, cc, state, control, params, nxt, stream):
    nc = nxt.c()
    rc = fn(ctypes.byref(dc), ctypes.byref(cc), ctypes.byref(state.c()), ctypes.byref(control.c()),
            ctypes.byref(params.c()), ctypes.byref(nc), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, (rc, pbf.library().pbf_last_error())
    nxt.step_index = int(nc.step_index)


def _run_both(sc, calls=2):
    """`calls` chained substeps through both entry points; returns the per-call states of each."""
    fn = _entry()
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    dc = pbf.DomainConfiguration.from_scene(sc).to_c()
    cc = pbf.ConfigurationC(sc.pressure_iterations, 1)
    mine, theirs = [], []
    a = pbf.State(state.positions.clone(), state.velocities.clone(), state.step_index)
    b = pbf.State(state.positions.clone(), state.velocities.clone(), state.step_index)
    for _ in range(calls):
        a_next = solver.allocate_state()
        _preallocated_step(fn, dc, cc, a, control, params, a_next, solver.stream)
        b_next = solver.allocate_state()
        solver.forward_step(b, control, params, b_next, cache)
        torch.cuda.synchronize()
        mine.append(a_next)
        theirs.append(b_next)
        a, b = a_next, b_next
    return mine, theirs


def test_two_calls_in_a_row_equal_the_solver_at_the_maximum_size():
    """32,768 particles (the documented maximum) and 128,000 cells, 4 Jacobi iterations."""
    sc = scenes.plain_small()
    assert sc.count == 32768
    mine, theirs = _run_both(sc)
    for k, (m, t) in enumerate(zip(mine, theirs)):
        assert torch.equal(m.positions, t.positions), k
        assert torch.equal(m.velocities, t.velocities), k
        assert m.step_index == t.step_index == k + 1


def test_smaller_scene_after_a_larger_one_reuses_the_scratch_cleanly():
    """A 1,000-particle scene after the 32k scene: nothing of the previous call's scratch contents
    (cell histogram, lists, iterates) leaks into the result."""
    sc = scenes.dam_break((10, 10, 10), (0, 0, 0), (1, 2, 1), 21, 3, velocity_sigma=0.1)
    mine, theirs = _run_both(sc)
    for k, (m, t) in enumerate(zip(mine, theirs)):
        assert torch.equal(m.positions, t.positions), k
        assert torch.equal(m.velocities, t.velocities), k


def test_repeated_calls_allocate_no_device_memory():
    """At the maximum size: after the first call in this context (the set-up, which may load the
    library's device code), further calls leave the device's free memory unchanged."""
    sc = scenes.plain_small(seed=22)
    fn = _entry()
    solver, state, control, params = pbf.solver_for_scene(sc)
    dc = pbf.DomainConfiguration.from_scene(sc).to_c()
    cc = pbf.ConfigurationC(sc.pressure_iterations, 1)
    nxt = solver.allocate_state()
    _preallocated_step(fn, dc, cc, state, control, params, nxt, solver.stream)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        _preallocated_step(fn, dc, cc, state, control, params, nxt, solver.stream)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_a_call_records_into_a_cuda_graph_under_global_capture():
    """After the set-up call, a call records into a CUDA graph in global capture mode, where
    cudaMalloc and every synchronising call fail the capture; the replayed graph gives the direct
    call's bits.  This also catches an allocation freed again before the call returns."""
    sc = scenes.plain_small(seed=24)
    fn = _entry()
    solver, state, control, params = pbf.solver_for_scene(sc)
    dc = pbf.DomainConfiguration.from_scene(sc).to_c()
    cc = pbf.ConfigurationC(sc.pressure_iterations, 1)
    direct = solver.allocate_state()
    _preallocated_step(fn, dc, cc, state, control, params, direct, solver.stream)
    torch.cuda.synchronize()
    replayed = solver.allocate_state()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream, capture_error_mode="global"):
        _preallocated_step(fn, dc, cc, state, control, params, replayed, stream)
    replayed.positions.fill_(float("nan"))
    replayed.velocities.fill_(float("nan"))
    graph.replay()
    torch.cuda.synchronize()
    assert replayed.step_index == direct.step_index
    assert torch.equal(replayed.positions, direct.positions)
    assert torch.equal(replayed.velocities, direct.velocities)


def test_sizes_beyond_the_maximum_are_rejected():
    fn = _entry()
    sc = scenes.dam_break((4, 4, 4), (0, 0, 0), (1, 2, 1), 23, 2)
    state = pbf.State(torch.zeros(3, 1, device="cuda"), torch.zeros(3, 1, device="cuda"), 0)
    control = pbf.Control(torch.zeros(3, 1, device="cuda"))
    params = pbf.Parameters({n: None for n in pbf.PARAMETER_NAMES})
    cc = pbf.ConfigurationC(2, 1)
    stream = torch.cuda.current_stream()
    too_many = pbf.DomainConfiguration.from_scene(sc).to_c()
    too_many.particle_count = 32769
    nc = state.c()
    rc = fn(ctypes.byref(too_many), ctypes.byref(cc), ctypes.byref(state.c()), ctypes.byref(control.c()),
            ctypes.byref(params.c()), ctypes.byref(nc), ctypes.c_void_p(stream.cuda_stream))
    assert rc == PBF_ERROR_CAPACITY
    assert b"PBF_PREALLOCATED_MAX_PARTICLES" in pbf.library().pbf_last_error()
    too_many_cells = pbf.DomainConfiguration.from_scene(sc).to_c()
    too_many_cells.boundary.maximum.x = 100.0   # 4000 x 80 x 40 cells at h = 0.025
    rc = fn(ctypes.byref(too_many_cells), ctypes.byref(cc), ctypes.byref(state.c()), ctypes.byref(control.c()),
            ctypes.byref(params.c()), ctypes.byref(nc), ctypes.c_void_p(stream.cuda_stream))
    assert rc == PBF_ERROR_CAPACITY
    assert b"PBF_PREALLOCATED_MAX_CELLS" in pbf.library().pbf_last_error()
