"""Differentiable rollouts of the PBF solver with trajectory checkpointing.

The reference differentiates one substep at a time (PBF::vjp_step, pbf/pbf.cpp:217-258) and
leaves the rollout to its caller; this module is that caller.  A rollout of `steps` substeps
keeps the state every `checkpoint_every` steps; the reverse sweep recomputes one segment at a
time (forward steps whose step caches it keeps) and runs vjp_step backwards through it, so the
memory held is one segment of step caches plus the checkpoints.

Loss: the mean squared distance of the final positions to a target cloud,
    L = (1/N) sum_i |x_i(T) - t_i|^2,
its gradient w.r.t. the initial velocities, and the gradient w.r.t. a scalar parameter shared
by all particles (dL/dc = sum_i dL/dc_i, a compensated FP64 sum on the device).
"""
from __future__ import annotations

import ctypes
import dataclasses

import torch

from . import pbf


def _new_like(state: pbf.State) -> pbf.State:
    return pbf.State(torch.empty_like(state.positions), torch.empty_like(state.velocities), state.step_index)


def compensated_sum(solver: pbf.PBF, values: torch.Tensor) -> torch.Tensor:
    """Neumaier-compensated FP64 sum of a device vector (deterministic)."""
    out = torch.empty(1, dtype=torch.float64, device=values.device)
    pbf.check(pbf.library().pbf_sum_compensated(solver.handle, ctypes.c_void_p(values.data_ptr()), values.numel(),
                                                ctypes.c_void_p(out.data_ptr())))
    return out


@dataclasses.dataclass
class Gradients:
    loss: float
    initial_positions: torch.Tensor      # (3, N) float64
    initial_velocities: torch.Tensor     # (3, N) float64
    controls: torch.Tensor               # (3, N) float64, summed over steps
    parameters: pbf.Parameters           # per-particle FP64 adjoints
    scalar: dict                         # name -> dL/dc for a parameter shared by all particles


class Rollout:
    """Forward `steps` substeps from `state0`, then the reverse sweep with recompute."""

    def __init__(self, solver: pbf.PBF, control: pbf.Control, parameters: pbf.Parameters, steps: int,
                 checkpoint_every: int = 10):
        if solver.mode != pbf.ExecutionMode.differentiable:
            raise ValueError("a differentiable rollout needs a solver in ExecutionMode.differentiable")
        if steps < 1 or checkpoint_every < 1:
            raise ValueError("steps and checkpoint_every must be positive")
        self.solver = solver
        self.control = control
        self.parameters = parameters
        self.steps = steps
        self.every = checkpoint_every
        self.caches = [solver.allocate_step_cache() for _ in range(min(checkpoint_every, steps))]
        self.checkpoints: list[pbf.State] = []
        self.final: pbf.State | None = None

    def forward(self, state0: pbf.State) -> pbf.State:
        """Run the rollout, keeping a state every `checkpoint_every` steps."""
        s = self.solver
        self.checkpoints = []
        cur = _new_like(state0)
        s.copy_state(state0, cur)
        nxt = _new_like(state0)
        for k in range(self.steps):
            if k % self.every == 0:
                cp = _new_like(cur)
                s.copy_state(cur, cp)
                self.checkpoints.append(cp)
            s.forward_step(cur, self.control, self.parameters, nxt, self.caches[k % self.every])
            cur, nxt = nxt, cur
        self.final = cur
        return cur

    def backward(self, final_position_adjoint: torch.Tensor, final_velocity_adjoint: torch.Tensor | None = None,
                 scalar_parameters=("xsph_viscosity",)) -> Gradients:
        """Reverse sweep: dL/d(initial state), dL/d(control), per-particle and scalar parameter adjoints."""
        s = self.solver
        adj = s.allocate_state_adjoint()
        adj.positions.copy_(final_position_adjoint)
        if final_velocity_adjoint is not None:
            adj.velocities.copy_(final_velocity_adjoint)
        control_adj = s.allocate_control_adjoint()
        param_adj = s.allocate_parameter_adjoint()
        prev = s.allocate_state_adjoint()
        segments = len(self.checkpoints)
        for seg in reversed(range(segments)):
            begin = seg * self.every
            end = min(begin + self.every, self.steps)
            states = [self.checkpoints[seg]]
            for k in range(begin, end):
                nxt = _new_like(states[-1])
                s.forward_step(states[-1], self.control, self.parameters, nxt, self.caches[k - begin])
                states.append(nxt)
            for k in reversed(range(begin, end)):
                j = k - begin
                prev.positions.zero_()
                prev.velocities.zero_()
                s.vjp_step(states[j], self.control, self.parameters, states[j + 1], self.caches[j], adj, prev,
                           control_adj, param_adj)
                adj, prev = prev, adj
        scalar = {name: compensated_sum(s, param_adj.tensors[name]) for name in scalar_parameters}
        return Gradients(loss=float("nan"), initial_positions=adj.positions, initial_velocities=adj.velocities,
                         controls=control_adj.external_accelerations, parameters=param_adj,
                         scalar={k: float(v.item()) for k, v in scalar.items()})


def target_loss(positions: torch.Tensor, targets: torch.Tensor):
    """L = (1/N) sum |x - t|^2 in FP64 and dL/dx = (2/N)(x - t)."""
    diff = positions.double() - targets.double()
    n = positions.shape[1]
    loss = float((diff * diff).sum() / n)
    return loss, diff * (2.0 / n)


def loss_and_gradients(solver: pbf.PBF, state0: pbf.State, control: pbf.Control, parameters: pbf.Parameters,
                       targets: torch.Tensor, steps: int, checkpoint_every: int = 10) -> Gradients:
    """Rollout, target loss and its gradients in one call."""
    r = Rollout(solver, control, parameters, steps, checkpoint_every)
    final = r.forward(state0)
    loss, dx = target_loss(final.positions, targets)
    g = r.backward(dx)
    g.loss = loss
    return g
