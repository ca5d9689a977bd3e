"""The reference's dam-break example driver on this solver.

Mirrors examples/fluids/liquid/pbf-dam-break/simulation.ixx (the Simulation struct: a solver in
forward mode with 5 Jacobi iterations, the current and next state, one step cache, step_index
and physical_time; reset() lays out the lattice, step() advances and swaps) and main.cpp (240
steps, a line every 60).  `--frames DIR` dumps every frame (positions, velocities, vorticity
magnitudes) where the example publishes to its Spectra viewer.

    python -m physica_b200.simulation [--steps 240] [--frames DIR]
"""
from __future__ import annotations

import argparse
import sys

import torch

from . import export, pbf, scenes


class Simulation:
    """simulation.ixx:17-52 on the B200 solver."""

    def __init__(self, device: str = "cuda"):
        self.scene = scenes.example_dam_break()
        self.particle_count = self.scene.count
        self.time_step = self.scene.time_step
        self.solver, self._initial, self.control, self.parameters = pbf.solver_for_scene(self.scene, device=device)
        self.step_cache = self.solver.allocate_step_cache()
        self.current_state = self.solver.allocate_state()
        self.next_state = self.solver.allocate_state()
        self.reset()

    def reset(self):
        """simulation.ixx:84-112: the lattice at rest, step 0."""
        self.solver.copy_state(self._initial, self.current_state)
        self.current_state.step_index = 0
        self.solver.copy_state(self.current_state, self.next_state)
        self.control.external_accelerations.zero_()
        self.solver.synchronize()
        self.step_index = 0
        self.physical_time = 0.0

    def step(self):
        """simulation.ixx:114-119."""
        self.solver.forward_step(self.current_state, self.control, self.parameters, self.next_state, self.step_cache)
        self.current_state, self.next_state = self.next_state, self.current_state
        self.step_index = self.current_state.step_index
        self.physical_time = float(self.step_index) * self.time_step


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="PBF dam break (the reference example) on the B200 solver")
    ap.add_argument("--steps", type=int, default=240)
    ap.add_argument("--frames", default="", help="directory for one .npz per frame")
    args = ap.parse_args(argv)
    try:
        simulation = Simulation()
        writer = export.FrameWriter(args.frames, simulation.solver, simulation.time_step) if args.frames else None
        print(f"PBF dam break with {simulation.particle_count} particles")
        for _ in range(args.steps):
            simulation.step()
            if writer is not None:
                writer.write(simulation.current_state, simulation.step_cache)
            if simulation.step_index % 60 == 0:
                print(f"step {simulation.step_index:3d}  time {simulation.physical_time:.3f} s")
        torch.cuda.synchronize()
        return 0
    except Exception as error:   # main.cpp:18-21 reports and exits 1
        print(f"PBF dam-break example failed: {error}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
