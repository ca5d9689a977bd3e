"""Python front end of the B200 SPH solvers over the C ABI of include/physica_sph.h.

Mirrors the reference's SPH<Method> (fluids/liquid/particle/sph/sph.ixx:273-372) with Method one
of WCSPH, PCISPH, IISPH and DFSPH: `SPH(domain_configuration, method_configuration, mode, stream)`,
`allocate_state` / `allocate_control` / `allocate_parameters` / `allocate_step_cache` and their
tangent / adjoint forms, `copy_state`, `forward_step`, `jvp_step` and `vjp_step`.  SPH<Method>::State is a particle state plus the method's state
(DFSPH's warm-start pressures); SPH<Method>::Parameters the particle parameters plus the method's.
Every call goes to libphysica_pbf.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import dataclasses
import enum

import numpy as np
import torch

from . import pbf
from .pbf import ControlC, DomainConfigurationC, LaunchShape, LaunchShapeC, ParticleStateC, _ptr, _vf, check

PARAMETER_NAMES = ("masses", "rest_densities", "viscosities", "surface_tensions", "speed_of_sound", "tait_exponent",
                   "boundary_surface_tension", "pressure_relaxation", "jacobi_relaxation", "divergence_relaxation",
                   "density_relaxation")

# Parameters each method reads besides the particle parameters (sph/sph.ixx:45-49, 111, 157, 214-217).
METHOD_PARAMETERS = {
    "wcsph": ("speed_of_sound", "tait_exponent", "boundary_surface_tension"),
    "pcisph": ("pressure_relaxation",),
    "iisph": ("jacobi_relaxation",),
    "dfsph": ("divergence_relaxation", "density_relaxation"),
}


class Method(enum.IntEnum):
    wcsph = 0
    pcisph = 1
    iisph = 2
    dfsph = 3


class CacheField(enum.IntEnum):
    DENSITIES = 0
    PRESSURES = 1
    PRESSURE_ACCELERATIONS = 2
    VISCOSITY_ACCELERATIONS = 3
    SURFACE_ACCELERATIONS = 4
    PREDICTED_DENSITIES = 5


class ConfigurationC(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("pressure_iterations", ctypes.c_uint32), ("divergence_iterations", ctypes.c_uint32),
                ("density_iterations", ctypes.c_uint32), ("checkpoint_interval", ctypes.c_uint32),
                ("pressure_warm_start", ctypes.c_uint32)]


class ParametersC(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in PARAMETER_NAMES]


class MethodStateC(ctypes.Structure):
    """sph_method_state and sph_method_state_adjoint: DFSPH's two warm-start pressure arrays as device
    pointers (float for a state or tangent, double for an adjoint)."""
    _fields_ = [("warm_divergence_pressure", ctypes.c_void_p), ("warm_density_pressure", ctypes.c_void_p)]


class ParameterAdjointC(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in PARAMETER_NAMES]


_bound = False


def library() -> ctypes.CDLL:
    """libphysica_pbf.so with the SPH entry points' signatures declared."""
    global _bound
    lib = pbf.library()
    if not _bound:
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        lib.sph_create.argtypes = [P(DomainConfigurationC), P(ConfigurationC), ctypes.c_int, vp, P(vp)]
        lib.sph_destroy.argtypes = [vp]
        lib.sph_allocate_step_cache.argtypes = [vp, P(vp)]
        lib.sph_free_step_cache.argtypes = [vp, vp]
        lib.sph_forward_step.argtypes = [vp, P(ParticleStateC), P(MethodStateC), P(ControlC), P(ParametersC),
                                         P(ParticleStateC), P(MethodStateC), vp]
        lib.sph_read_cache.argtypes = [vp, vp, ctypes.c_int, vp, vp, vp]
        lib.sph_jvp_step.argtypes = [vp, P(ParticleStateC), P(MethodStateC), P(ControlC), P(ParametersC), P(ParticleStateC), vp,
                                     P(pbf.StateTangentC), P(MethodStateC), P(ControlC), P(ParametersC), P(pbf.StateTangentC),
                                     P(MethodStateC)]
        lib.sph_vjp_step.argtypes = [vp, P(ParticleStateC), P(MethodStateC), P(ControlC), P(ParametersC), P(ParticleStateC), vp,
                                     P(pbf.StateAdjointC), P(MethodStateC), P(pbf.StateAdjointC), P(MethodStateC), P(ControlC),
                                     P(ParameterAdjointC)]
        lib.sph_copy_state.argtypes = [vp, P(ParticleStateC), P(MethodStateC), P(ParticleStateC), P(MethodStateC)]
        lib.sph_copy_state_tangent.argtypes = [vp, P(pbf.StateTangentC), P(MethodStateC), P(pbf.StateTangentC), P(MethodStateC)]
        lib.sph_copy_state_adjoint.argtypes = [vp, P(pbf.StateAdjointC), P(MethodStateC), P(pbf.StateAdjointC), P(MethodStateC)]
        lib.sph_accumulate_state_adjoint.argtypes = [vp, P(pbf.StateAdjointC), P(MethodStateC), P(pbf.StateAdjointC),
                                                     P(MethodStateC)]
        lib.sph_reference_gradient_norm.argtypes = [vp, P(ctypes.c_float)]
        lib.sph_set_launch_shape.argtypes = [vp, P(LaunchShapeC)]
        lib.sph_get_launch_shape.argtypes = [vp, P(LaunchShapeC)]
        lib.sph_synchronize.argtypes = [vp]
        lib.sph_stream.argtypes = [vp]
        lib.sph_stream.restype = vp
        _bound = True
    return lib


@dataclasses.dataclass
class Configuration:
    """Method::Configuration (sph/sph.ixx:104-107, 150-153, 196-201), reference defaults."""
    method: Method = Method.wcsph
    pressure_iterations: int = 6
    divergence_iterations: int = 4
    density_iterations: int = 6
    checkpoint_interval: int = 2
    pressure_warm_start: bool = True

    def to_c(self) -> ConfigurationC:
        return ConfigurationC(int(self.method), self.pressure_iterations, self.divergence_iterations, self.density_iterations,
                              self.checkpoint_interval, 1 if self.pressure_warm_start else 0)


@dataclasses.dataclass
class State:
    """SPH<Method>::State (sph/sph.ixx:275-278): positions / velocities (3, N) float32 and, for
    DFSPH, the warm-start pressures (N,) float32."""
    positions: torch.Tensor
    velocities: torch.Tensor
    step_index: int = 0
    warm_divergence_pressure: torch.Tensor | None = None
    warm_density_pressure: torch.Tensor | None = None

    def c(self) -> ParticleStateC:
        return ParticleStateC(_vf(self.positions), _vf(self.velocities), self.step_index)

    def method_c(self) -> MethodStateC:
        a, b = self.warm_divergence_pressure, self.warm_density_pressure
        return MethodStateC(_ptr(a) if a is not None and a.numel() else None, _ptr(b) if b is not None and b.numel() else None)


@dataclasses.dataclass
class StateTangent:
    """SPH<Method>::StateTangent (sph/sph.ixx:279-282): (3, N) float32 position / velocity tangents
    and, for DFSPH, the (N,) float32 tangents of the warm-start pressures."""
    positions: torch.Tensor
    velocities: torch.Tensor
    warm_divergence_pressure: torch.Tensor | None = None
    warm_density_pressure: torch.Tensor | None = None

    def c(self) -> pbf.StateTangentC:
        return pbf.StateTangentC(_vf(self.positions), _vf(self.velocities))

    def method_c(self) -> MethodStateC:
        a, b = self.warm_divergence_pressure, self.warm_density_pressure
        return MethodStateC(_ptr(a) if a is not None and a.numel() else None, _ptr(b) if b is not None and b.numel() else None)


@dataclasses.dataclass
class StateAdjoint:
    """SPH<Method>::StateAdjoint (sph/sph.ixx:283-286): (3, N) float64 position / velocity adjoints
    and, for DFSPH, the (N,) float64 adjoints of the warm-start pressures."""
    positions: torch.Tensor
    velocities: torch.Tensor
    warm_divergence_pressure: torch.Tensor | None = None
    warm_density_pressure: torch.Tensor | None = None

    def c(self) -> pbf.StateAdjointC:
        return pbf.StateAdjointC(_vf(self.positions), _vf(self.velocities))

    def method_c(self) -> MethodStateC:
        a, b = self.warm_divergence_pressure, self.warm_density_pressure
        return MethodStateC(_ptr(a) if a is not None and a.numel() else None, _ptr(b) if b is not None and b.numel() else None)


class Parameters:
    """SPH<Method>::Parameters (sph/sph.ixx:287-290): one (N,) float32 tensor per parameter."""

    def __init__(self, tensors: dict):
        self.tensors = tensors

    def __getattr__(self, name):
        if name in PARAMETER_NAMES:
            return self.tensors[name]
        raise AttributeError(name)

    def c(self) -> ParametersC:
        return ParametersC(*[_ptr(self.tensors[n]) if self.tensors.get(n) is not None and self.tensors[n].numel() else None
                             for n in PARAMETER_NAMES])


class StepCache:
    """SPH<Method>::StepCache (sph/sph.ixx:299-303), owned by the library."""

    def __init__(self, solver: "SPH"):
        self.solver = solver
        h = ctypes.c_void_p()
        check(library().sph_allocate_step_cache(solver.handle, ctypes.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None) and getattr(self.solver, "handle", None):
            library().sph_free_step_cache(self.solver.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read(self, field: CacheField) -> torch.Tensor:
        """A field of the cached step in original particle order."""
        s = self.solver
        scalar = field in (CacheField.DENSITIES, CacheField.PRESSURES, CacheField.PREDICTED_DENSITIES)
        out = torch.empty((s.count,) if scalar else (3, s.count), dtype=torch.float32, device=s.device)
        if s.count == 0:
            return out
        if scalar:
            ptrs = (out.data_ptr(), None, None)
        else:
            ptrs = (out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
        check(library().sph_read_cache(s.handle, self.handle, int(field), *ptrs))
        return out


class SPH:
    """The B200 SPH solver SPH<Method> (sph/sph.ixx:273-372), forward mode."""

    def __init__(self, domain_configuration: pbf.DomainConfiguration, configuration: Configuration = Configuration(),
                 mode: pbf.ExecutionMode = pbf.ExecutionMode.forward, stream: torch.cuda.Stream | None = None,
                 device: torch.device | str = "cuda"):
        lib = library()
        self.device = torch.device(device)
        if self.device.type != "cuda" or not torch.cuda.is_available():
            raise RuntimeError("the SPH solver needs a CUDA device")
        self.domain_configuration = domain_configuration
        self.configuration = configuration
        self.method = Method(configuration.method)
        self.mode = pbf.ExecutionMode(mode)
        self.stream = stream or torch.cuda.current_stream(self.device)
        self.count = int(domain_configuration.particle_count)
        self._dc = domain_configuration.to_c()
        cc = configuration.to_c()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(lib.sph_create(ctypes.byref(self._dc), ctypes.byref(cc), int(self.mode),
                                 ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            library().sph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _vec(self):
        return torch.zeros((3, self.count), dtype=torch.float32, device=self.device)

    def allocate_state(self) -> State:
        dfsph = self.method == Method.dfsph
        z = (lambda: torch.zeros(self.count, dtype=torch.float32, device=self.device)) if dfsph else (lambda: None)
        return State(self._vec(), self._vec(), 0, z(), z())

    def allocate_control(self) -> pbf.Control:
        return pbf.Control(self._vec())

    def allocate_parameters(self) -> Parameters:
        return Parameters({n: torch.zeros(self.count, dtype=torch.float32, device=self.device) for n in PARAMETER_NAMES})

    def allocate_step_cache(self) -> StepCache:
        return StepCache(self)

    def allocate_state_tangent(self) -> StateTangent:
        s = self.allocate_state()
        return StateTangent(s.positions, s.velocities, s.warm_divergence_pressure, s.warm_density_pressure)

    def allocate_parameter_tangent(self) -> Parameters:
        return self.allocate_parameters()

    def allocate_state_adjoint(self) -> StateAdjoint:
        z3 = lambda: torch.zeros((3, self.count), dtype=torch.float64, device=self.device)
        dfsph = self.method == Method.dfsph
        z = (lambda: torch.zeros(self.count, dtype=torch.float64, device=self.device)) if dfsph else (lambda: None)
        return StateAdjoint(z3(), z3(), z(), z())

    def allocate_control_adjoint(self) -> pbf.Control:
        return pbf.Control(torch.zeros((3, self.count), dtype=torch.float64, device=self.device))

    def allocate_parameter_adjoint(self) -> Parameters:
        return Parameters({n: torch.zeros(self.count, dtype=torch.float64, device=self.device) for n in PARAMETER_NAMES})

    def state_from_arrays(self, positions, velocities, step_index=0) -> State:
        s = self.allocate_state()
        s.positions.copy_(torch.as_tensor(np.ascontiguousarray(positions)))
        s.velocities.copy_(torch.as_tensor(np.ascontiguousarray(velocities)))
        s.step_index = step_index
        return s

    def parameters_from_arrays(self, arrays: dict) -> Parameters:
        p = self.allocate_parameters()
        for k, v in arrays.items():
            p.tensors[k].copy_(torch.as_tensor(np.ascontiguousarray(v)))
        return p

    def _copy(self, entry, source, destination):
        sc, dc = source.c(), destination.c()
        check(entry(self.handle, ctypes.byref(sc), ctypes.byref(source.method_c()), ctypes.byref(dc),
                    ctypes.byref(destination.method_c())))
        return dc

    def copy_state(self, source: State, destination: State):
        """SPH<Method>::copy_state (sph/sph.ixx:326-329): particles and DFSPH's warm starts."""
        destination.step_index = self._copy(library().sph_copy_state, source, destination).step_index

    def copy_state_tangent(self, source: StateTangent, destination: StateTangent):
        """SPH<Method>::copy_state_tangent (sph/sph.ixx:331-334)."""
        self._copy(library().sph_copy_state_tangent, source, destination)

    def copy_state_adjoint(self, source: StateAdjoint, destination: StateAdjoint):
        """SPH<Method>::copy_state_adjoint (sph/sph.ixx:336-339)."""
        self._copy(library().sph_copy_state_adjoint, source, destination)

    def accumulate_state_adjoint(self, source: StateAdjoint, destination: StateAdjoint):
        """SPH<Method>::accumulate_state_adjoint (sph/sph.ixx:341-344): destination += source."""
        self._copy(library().sph_accumulate_state_adjoint, source, destination)

    def forward_step(self, state: State, control: pbf.Control, parameters: Parameters, next_state: State, cache: StepCache):
        """SPH<Method>::forward_step (sph/sph.ixx:350-354)."""
        sc, ns = state.c(), next_state.c()
        ms, nms = state.method_c(), next_state.method_c()
        check(library().sph_forward_step(self.handle, ctypes.byref(sc), ctypes.byref(ms), ctypes.byref(control.c()),
                                          ctypes.byref(parameters.c()), ctypes.byref(ns), ctypes.byref(nms), cache.handle))
        next_state.step_index = ns.step_index

    def jvp_step(self, state: State, control: pbf.Control, parameters: Parameters, next_state: State, cache: StepCache,
                 state_tangent: StateTangent, control_tangent: pbf.Control, parameter_tangent: Parameters | None,
                 next_state_tangent: StateTangent):
        """SPH<Method>::jvp_step (sph/sph.ixx:356-359), FP32 tangents of the step held by `cache`."""
        pt = ctypes.byref(parameter_tangent.c()) if parameter_tangent is not None else None
        check(library().sph_jvp_step(self.handle, ctypes.byref(state.c()), ctypes.byref(state.method_c()),
                                     ctypes.byref(control.c()), ctypes.byref(parameters.c()), ctypes.byref(next_state.c()),
                                     cache.handle, ctypes.byref(state_tangent.c()), ctypes.byref(state_tangent.method_c()),
                                     ctypes.byref(control_tangent.c()), pt, ctypes.byref(next_state_tangent.c()),
                                     ctypes.byref(next_state_tangent.method_c())))

    def vjp_step(self, state: State, control: pbf.Control, parameters: Parameters, next_state: State, cache: StepCache,
                 next_state_adjoint: StateAdjoint, previous_state_adjoint: StateAdjoint, control_adjoint: pbf.Control,
                 parameter_adjoint: Parameters):
        """SPH<Method>::vjp_step (sph/sph.ixx:361-365); accumulates into the previous-state, control
        and parameter adjoints (DFSPH's previous warm-pressure adjoints are overwritten)."""
        pa = ParameterAdjointC(*[_ptr(parameter_adjoint.tensors[n]) if parameter_adjoint.tensors.get(n) is not None else None
                                 for n in PARAMETER_NAMES])
        check(library().sph_vjp_step(self.handle, ctypes.byref(state.c()), ctypes.byref(state.method_c()),
                                     ctypes.byref(control.c()), ctypes.byref(parameters.c()), ctypes.byref(next_state.c()),
                                     cache.handle, ctypes.byref(next_state_adjoint.c()),
                                     ctypes.byref(next_state_adjoint.method_c()), ctypes.byref(previous_state_adjoint.c()),
                                     ctypes.byref(previous_state_adjoint.method_c()), ctypes.byref(control_adjoint.c()),
                                     ctypes.byref(pa)))

    @property
    def reference_gradient_norm(self) -> float:
        v = ctypes.c_float()
        check(library().sph_reference_gradient_norm(self.handle, ctypes.byref(v)))
        return float(v.value)

    @property
    def launch_shape(self) -> LaunchShape:
        c = LaunchShapeC()
        check(library().sph_get_launch_shape(self.handle, ctypes.byref(c)))
        return LaunchShape.from_c(c)

    @launch_shape.setter
    def launch_shape(self, shape: LaunchShape):
        check(library().sph_set_launch_shape(self.handle, ctypes.byref(shape.to_c())))

    def synchronize(self):
        check(library().sph_synchronize(self.handle))


def solver_for_scene(scene, method: Method, *, configuration: Configuration | None = None,
                     mode: pbf.ExecutionMode = pbf.ExecutionMode.forward, device="cuda"):
    """A solver, state, control and parameters for a synthetic SPH scene (scenes.sph_dam_break)."""
    dc = pbf.DomainConfiguration.from_scene(scene)
    cfg = configuration or Configuration(method=Method(method))
    solver = SPH(dc, cfg, mode, device=device)
    state = solver.state_from_arrays(scene.positions, scene.velocities)
    control = solver.allocate_control()
    control.external_accelerations.copy_(torch.from_numpy(scene.controls))
    params = solver.parameters_from_arrays(scene.sph)
    return solver, state, control, params
