"""Headless frame dump of a PBF run.

The reference's dam-break example publishes every frame to the Spectra viewer
(examples/fluids/liquid/pbf-dam-break/spectra/provider.ixx:74-96): particle positions and
velocities as xyz triples, the step cache's vorticity magnitudes, and the step index and
simulated time.  There is no viewer here; pbf_export_frame writes the same fields into device
buffers and FrameWriter stores one .npz file per frame.
"""
from __future__ import annotations

import pathlib

import numpy as np

from . import pbf


class FrameWriter:
    """Writes frame_<step>.npz files (positions (N, 3), velocities (N, 3), vorticity (N,),
    step, time) into `directory`."""

    def __init__(self, directory, solver: pbf.PBF, time_step: float):
        self.directory = pathlib.Path(directory)
        self.directory.mkdir(parents=True, exist_ok=True)
        self.solver = solver
        self.time_step = float(time_step)

    def write(self, state: pbf.State, cache: pbf.StepCache | None = None) -> pathlib.Path:
        frame = self.solver.export_frame(state, cache)
        path = self.directory / f"frame_{state.step_index:06d}.npz"
        arrays = {k: v.cpu().numpy() for k, v in frame.items() if k != "step"}
        np.savez(path, step=np.uint64(state.step_index), time=np.float64(state.step_index * self.time_step), **arrays)
        return path
