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


def compensated_sum(solver: pbf.PBF, values: torch.Tensor) -> torch.Tensor:
    """Neumaier-compensated FP64 sum of a device vector (deterministic)."""
    out = torch.empty(1, dtype=torch.float64, device=values.device)
    pbf.check(pbf.library().pbf_sum_compensated(solver.handle, ctypes.c_void_p(values.data_ptr()), values.numel(),
                                                ctypes.c_void_p(out.data_ptr())))
    return out


@dataclasses.dataclass
class Gradients:
    loss: float                          # a list of per-scene losses for a batch
    initial_positions: torch.Tensor      # (3, N) float64
    initial_velocities: torch.Tensor     # (3, N) float64
    controls: torch.Tensor               # (3, N) float64, summed over steps
    parameters: pbf.Parameters           # per-particle FP64 adjoints
    scalar: dict                         # name -> dL/dc of a parameter shared by all particles (per scene for a batch)


class _Stepper:
    """The calls a rollout makes, for a single-scene solver (PBF) or a batch of scenes (Batch)."""

    def __init__(self, solver, cache_count: int):
        self.solver = solver
        self.batched = isinstance(solver, pbf.Batch)
        if self.batched:
            solver.reserve_caches(cache_count)
            self.caches = list(range(cache_count))
        else:
            self.caches = [solver.allocate_step_cache() for _ in range(cache_count)]

    def copy_state(self, source: pbf.State, destination: pbf.State):
        if self.batched:
            destination.positions.copy_(source.positions)
            destination.velocities.copy_(source.velocities)
            destination.step_index = source.step_index
        else:
            self.solver.copy_state(source, destination)

    def forward(self, state, control, parameters, next_state, j):
        self.solver.forward_step(state, control, parameters, next_state, self.caches[j])

    def vjp(self, state, control, parameters, next_state, j, next_adjoint, previous_adjoint, control_adjoint,
            parameter_adjoint):
        self.solver.vjp_step(state, control, parameters, next_state, self.caches[j], next_adjoint, previous_adjoint,
                             control_adjoint, parameter_adjoint)

    def scalar(self, values: torch.Tensor):
        """dL/dc of a parameter shared by all particles (a batch: one per scene)."""
        if self.batched:
            return self.solver.scene_sums(values).cpu().tolist()
        return float(compensated_sum(self.solver, values).item())


class Rollout:
    """Forward `steps` substeps from `state0`, then the reverse sweep with recompute.

    `solver` is a differentiable PBF or a differentiable Batch (every scene rolls out together;
    scalar parameter gradients are then per scene).  Every buffer (step caches, checkpoints,
    segment states, adjoints) is allocated once here and reused by later calls, so the tensors of
    a returned `Gradients` are overwritten by the next backward sweep of the same rollout; copy
    them to keep them."""

    def __init__(self, solver, control: pbf.Control, parameters: pbf.Parameters, steps: int,
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
        self.stepper = _Stepper(solver, min(checkpoint_every, steps))
        segments = (steps + checkpoint_every - 1) // checkpoint_every
        self.checkpoints: list[pbf.State] = [solver.allocate_state() for _ in range(segments)]
        # segment states are reused by every segment, so their buffers (and any CUDA graph keyed on
        # them) repeat from call to call
        self.segment = [solver.allocate_state() for _ in range(min(checkpoint_every, steps) + 1)]
        self.adjoints = [solver.allocate_state_adjoint() for _ in range(2)]
        self.control_adjoint = solver.allocate_control_adjoint()
        self.parameter_adjoint = solver.allocate_parameter_adjoint()
        self.final: pbf.State | None = None

    def forward(self, state0: pbf.State) -> pbf.State:
        """Run the rollout, keeping a state every `checkpoint_every` steps."""
        s = self.stepper
        for k in range(self.steps):
            j = k % self.every
            if j == 0:
                # a new segment starts from the previous segment's last state
                source = state0 if k == 0 else self.segment[self.every]
                s.copy_state(source, self.checkpoints[k // self.every])
                s.copy_state(source, self.segment[0])
            s.forward(self.segment[j], self.control, self.parameters, self.segment[j + 1], j)
        last = (self.steps - 1) % self.every + 1
        self.final = self.segment[last]
        return self.final

    def backward(self, final_position_adjoint: torch.Tensor, final_velocity_adjoint: torch.Tensor | None = None,
                 scalar_parameters=("xsph_viscosity",)) -> Gradients:
        """Reverse sweep: dL/d(initial state), dL/d(control), per-particle and scalar parameter adjoints."""
        s = self.stepper
        adj, prev = self.adjoints
        adj.positions.copy_(final_position_adjoint)
        if final_velocity_adjoint is not None:
            adj.velocities.copy_(final_velocity_adjoint)
        else:
            adj.velocities.zero_()
        control_adj = self.control_adjoint
        param_adj = self.parameter_adjoint
        control_adj.external_accelerations.zero_()
        for t in param_adj.tensors.values():
            t.zero_()
        segments = len(self.checkpoints)
        for seg in reversed(range(segments)):
            begin = seg * self.every
            end = min(begin + self.every, self.steps)
            states = self.segment
            s.copy_state(self.checkpoints[seg], states[0])
            # the last segment's step caches still hold its forward steps
            if seg != segments - 1:
                for k in range(begin, end):
                    s.forward(states[k - begin], self.control, self.parameters, states[k - begin + 1], k - begin)
            for k in reversed(range(begin, end)):
                j = k - begin
                prev.positions.zero_()
                prev.velocities.zero_()
                s.vjp(states[j], self.control, self.parameters, states[j + 1], j, adj, prev, control_adj, param_adj)
                adj, prev = prev, adj
        scalar = {name: s.scalar(param_adj.tensors[name]) for name in scalar_parameters}
        self.adjoints = [adj, prev]
        return Gradients(loss=float("nan"), initial_positions=adj.positions, initial_velocities=adj.velocities,
                         controls=control_adj.external_accelerations, parameters=param_adj, scalar=scalar)


def target_loss(positions: torch.Tensor, targets: torch.Tensor, ranges=None):
    """L = (1/N) sum |x - t|^2 in FP64 and dL/dx = (2/N)(x - t).  With `ranges` (a batch's
    per-scene particle slices) every scene has its own loss L_s over its N_s particles; the losses
    are returned as a list and dL/dx holds each scene's own gradient."""
    diff = positions.double() - targets.double()
    if ranges is None:
        n = positions.shape[1]
        return float((diff * diff).sum() / n), diff * (2.0 / n)
    losses, grad = [], torch.empty_like(diff)
    for sl in ranges:
        d = diff[:, sl]
        n = d.shape[1]
        losses.append(float((d * d).sum() / n) if n else 0.0)
        grad[:, sl] = d * (2.0 / n) if n else d
    return losses, grad


def loss_and_gradients(solver, state0: pbf.State, control: pbf.Control, parameters: pbf.Parameters,
                       targets: torch.Tensor, steps: int, checkpoint_every: int = 10, rollout: Rollout | None = None) -> Gradients:
    """Rollout, target loss and its gradients in one call (pass `rollout` to reuse its buffers).
    For a Batch the loss and the scalar parameter gradients are per scene (lists)."""
    r = rollout or Rollout(solver, control, parameters, steps, checkpoint_every)
    final = r.forward(state0)
    ranges = [solver.particle_range(s) for s in range(solver.scene_count)] if isinstance(solver, pbf.Batch) else None
    loss, dx = target_loss(final.positions, targets, ranges)
    g = r.backward(dx)
    g.loss = loss
    return g
