"""GPU test of the headless frame export (the dam-break example's Spectra provider fields)."""
import numpy as np
import pytest
import torch

from physica_b200 import export, pbf, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def test_frame_export_and_dump(tmp_path):
    sc = scenes.dam_break((8, 8, 8), (0, 0, 0), (1, 2, 1), 91, 3, velocity_sigma=0.1)
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    writer = export.FrameWriter(tmp_path, solver, sc.time_step)
    cur, nxt = state, solver.allocate_state()
    for _ in range(3):
        solver.forward_step(cur, control, params, nxt, cache)
        cur, nxt = nxt, cur
        path = writer.write(cur, cache)
    frame = solver.export_frame(cur, cache)
    torch.cuda.synchronize()
    assert torch.equal(frame["positions"], cur.positions.t())
    assert torch.equal(frame["velocities"], cur.velocities.t())
    assert torch.equal(frame["vorticity"], cache.read(pbf.CacheField.VORTICITY_MAGNITUDES))
    saved = np.load(path)
    assert int(saved["step"]) == 3
    assert saved["time"] == pytest.approx(3 * sc.time_step)
    assert np.array_equal(saved["positions"], cur.positions.t().cpu().numpy())
    assert np.array_equal(saved["vorticity"], frame["vorticity"].cpu().numpy())
    # a cache of another step is rejected for the vorticity field
    with pytest.raises(pbf.PBFError):
        solver.export_frame(state, cache)
    assert solver.export_frame(state)["positions"].shape == (sc.count, 3)
