"""GPU test of the reference's own dam-break example (examples/fluids/liquid/pbf-dam-break):
its 5,376-particle scene stepped 240 times by the example driver here and by the reference's
kernels through the harness, compared bit for bit every 60 steps, plus the driver's output."""
import numpy as np
import pytest
import torch

from physica_b200 import scenes, simulation

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def test_example_scene_matches_reference_for_240_steps():
    from oracle import reference
    if not reference.available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    sim = simulation.Simulation()
    sc = scenes.example_dam_break()
    assert sim.particle_count == 16 * 28 * 12
    ref = reference.ReferencePBF(sc, checkpoint_interval=2)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    x2, v2 = torch.zeros_like(x), torch.zeros_like(v)
    for k in range(240):
        sim.step()
        ref.forward_step(x, v, x2, v2, k)
        x, x2, v, v2 = x2, x, v2, v
        if sim.step_index % 60 == 0:
            torch.cuda.synchronize()
            assert torch.equal(sim.current_state.positions, x), sim.step_index
            assert torch.equal(sim.current_state.velocities, v), sim.step_index
    assert sim.step_index == 240
    assert sim.physical_time == pytest.approx(1.0)


def test_example_driver_prints_and_dumps_frames(tmp_path, capsys):
    assert simulation.main(["--steps", "120", "--frames", str(tmp_path)]) == 0
    out = capsys.readouterr().out.splitlines()
    assert out[0] == "PBF dam break with 5376 particles"
    assert out[1].startswith("step  60  time 0.250 s") and out[2].startswith("step 120  time 0.500 s")
    frames = sorted(tmp_path.glob("frame_*.npz"))
    assert len(frames) == 120
    last = np.load(frames[-1])
    assert last["positions"].shape == (5376, 3) and np.all(np.isfinite(last["positions"]))
