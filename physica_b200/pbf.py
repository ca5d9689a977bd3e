"""Python front end of the B200 PBF solver over the C ABI of include/physica_pbf.h.

Mirrors the reference's solver interface (fluids/liquid/particle/pbf/pbf.ixx:14-141 and
domain/domain.ixx:12-165): `PBF(domain_configuration, configuration, mode, stream)`,
the `allocate_*` family, `forward_step`, `jvp_step`, `vjp_step`, `copy_state`,
`copy_state_tangent`, `copy_state_adjoint`, `accumulate_state_adjoint`.  Device memory comes from torch
(tensors are the `VectorField` x/y/z buffers); every call goes to the CUDA library
libphysica_pbf.so.  There is no CPU fallback: importing works without a GPU, but
creating a solver without the built library or a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import dataclasses
import enum
import pathlib

import torch

LIB_PATH = pathlib.Path(__file__).resolve().parent / "lib" / "libphysica_pbf.so"

# ----------------------------------------------------------------------------- C types
c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)


class Vector3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class BoxBoundaryC(ctypes.Structure):
    _fields_ = [("minimum", Vector3), ("maximum", Vector3), ("velocity", Vector3), ("no_slip", ctypes.c_uint32)]


class BoundaryParticleC(ctypes.Structure):
    _fields_ = [("position", Vector3), ("velocity", Vector3), ("volume", ctypes.c_float)]


class DomainConfigurationC(ctypes.Structure):
    _fields_ = [
        ("particle_count", ctypes.c_uint32),
        ("time_step", ctypes.c_float),
        ("support_radius", ctypes.c_float),
        ("particle_radius", ctypes.c_float),
        ("gravity", Vector3),
        ("boundary", BoxBoundaryC),
        ("boundary_particles", ctypes.POINTER(BoundaryParticleC)),
        ("boundary_particle_count", ctypes.c_uint32),
    ]


class ConfigurationC(ctypes.Structure):
    _fields_ = [("pressure_iterations", ctypes.c_uint32), ("checkpoint_interval", ctypes.c_uint32)]


class VectorFieldC(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p)]


class ParticleStateC(ctypes.Structure):
    _fields_ = [("positions", VectorFieldC), ("velocities", VectorFieldC), ("step_index", ctypes.c_uint64)]


class ControlC(ctypes.Structure):
    _fields_ = [("external_accelerations", VectorFieldC)]


class StateFieldsC(ctypes.Structure):
    """pbf_particle_state_tangent and pbf_particle_state_adjoint: positions and velocities as three
    device pointers each (float arrays for a tangent, double arrays for an adjoint)."""
    _fields_ = [("positions", VectorFieldC), ("velocities", VectorFieldC)]


StateTangentC = StateFieldsC
StateAdjointC = StateFieldsC


PARAMETER_NAMES = ("masses", "rest_densities", "viscosities", "surface_tensions", "relaxation",
                   "artificial_pressure_strength", "artificial_pressure_exponent", "artificial_pressure_radius",
                   "xsph_viscosity", "vorticity_confinement")


class ParametersC(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in PARAMETER_NAMES]


class LaunchShapeC(ctypes.Structure):
    _fields_ = [("list_scan", ctypes.c_uint32), ("scan_block_size", ctypes.c_uint32), ("block_size", ctypes.c_uint32)]


@dataclasses.dataclass
class LaunchShape:
    """Launch shape of the neighbour-list and gather kernels (results are identical for every shape).
    list_scan: 0 = per-lane walk, 1 = warp-cooperative scan, 2 = shared-memory staged walk,
    3 = per-lane walk with each Jacobi iteration's density + lambda in the same kernel,
    4 = as 3 with hit-mask neighbour lists in forward mode;
    scan_block_size (list scan) and
    block_size (gather passes): 32, 64, 96 or 128."""
    list_scan: int = 0
    scan_block_size: int = 128
    block_size: int = 128

    def to_c(self) -> "LaunchShapeC":
        return LaunchShapeC(self.list_scan, self.scan_block_size, self.block_size)

    @staticmethod
    def from_c(c: "LaunchShapeC") -> "LaunchShape":
        return LaunchShape(int(c.list_scan), int(c.scan_block_size), int(c.block_size))


class HostStateC(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p * 3), ("velocities", ctypes.c_void_p * 3), ("step_index", ctypes.c_uint64)]


INPUT_NONFINITE_POSITION = 1
INPUT_NONFINITE_VELOCITY = 2
INPUT_NONFINITE_CONTROL = 4
INPUT_BAD_MASS = 8


class FrameC(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("velocities", ctypes.c_void_p), ("vorticity", ctypes.c_void_p)]


class CacheField(enum.IntEnum):
    SORTED_PARTICLE_INDICES = 0
    CELL_OFFSETS = 1
    SORTED_KEYS = 2
    PREDICTED_POSITIONS = 3
    CORRECTED_POSITIONS = 4
    RECONSTRUCTED_VELOCITIES = 5
    VORTICITIES = 6
    VORTICITY_MAGNITUDES = 7
    VORTICITY_NORMALS = 8
    VORTICITY_NORMALIZERS = 9
    CONFINED_VELOCITIES = 10
    FIRST_DENSITIES = 11
    FIRST_LAMBDAS = 12
    NEIGHBOR_COUNTS = 13
    GRID_RESOLUTION = 14


class IterationField(enum.IntEnum):
    POSITIONS = 0
    DENSITIES = 1
    LAMBDAS = 2
    GRADIENT_SUMS = 3
    DENOMINATORS = 4
    COLLISION_MASKS = 5


class ExecutionMode(enum.IntEnum):
    """domain/domain.ixx:231-234"""
    forward = 0
    differentiable = 1


class PBFError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None


def library() -> ctypes.CDLL:
    """Load libphysica_pbf.so; raises if it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA library {LIB_PATH} is missing: run `python -m physica_b200.build` "
                               "(or __graft_entry__.build()) first; there is no CPU fallback")
        lib = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        lib.pbf_create.argtypes = [P(DomainConfigurationC), P(ConfigurationC), ctypes.c_int, vp, P(vp)]
        lib.pbf_destroy.argtypes = [vp]
        lib.pbf_allocate_step_cache.argtypes = [vp, P(vp)]
        lib.pbf_free_step_cache.argtypes = [vp]
        lib.pbf_forward_step.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC), vp]
        lib.pbf_vjp_step.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC), vp,
                                     P(StateAdjointC), P(StateAdjointC), P(ControlC), P(ParametersC)]
        lib.pbf_jvp_step.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC), vp,
                                     P(StateTangentC), P(ControlC), P(ParametersC), P(StateTangentC)]
        lib.pbf_copy_state.argtypes = [vp, P(ParticleStateC), P(ParticleStateC)]
        lib.pbf_copy_state_adjoint.argtypes = [vp, P(StateAdjointC), P(StateAdjointC)]
        lib.pbf_copy_state_tangent.argtypes = [vp, P(StateTangentC), P(StateTangentC)]
        lib.pbf_accumulate_state_adjoint.argtypes = [vp, P(StateAdjointC), P(StateAdjointC)]
        lib.pbf_forward_step_host.argtypes = [vp, P(HostStateC), P(ControlC), P(ParametersC), P(HostStateC), vp]
        lib.pbf_step_cache_read.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_size_t]
        lib.pbf_step_cache_read_iteration.argtypes = [vp, vp, ctypes.c_int, ctypes.c_uint32, vp, ctypes.c_size_t]
        lib.pbf_grid_cell_count.argtypes = [vp, P(ctypes.c_uint64)]
        lib.pbf_synchronize.argtypes = [vp]
        lib.pbf_status_string.restype = ctypes.c_char_p
        lib.pbf_last_error.restype = ctypes.c_char_p
        lib.pbf_launch_count.restype = ctypes.c_uint64
        lib.pbf_batch_create.argtypes = [P(DomainConfigurationC), ctypes.c_uint32, P(ConfigurationC), ctypes.c_int, vp, P(vp)]
        lib.pbf_batch_destroy.argtypes = [vp]
        lib.pbf_batch_particle_offset.argtypes = [vp, ctypes.c_uint32, P(ctypes.c_uint32), P(ctypes.c_uint32)]
        lib.pbf_batch_forward_step.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC),
                                               ctypes.c_uint32]
        lib.pbf_batch_vjp_step.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC),
                                           ctypes.c_uint32, P(StateAdjointC), P(StateAdjointC), P(ControlC),
                                           P(ParametersC)]
        lib.pbf_batch_jvp_step.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC),
                                           ctypes.c_uint32, P(StateTangentC), P(ControlC), P(ParametersC), P(StateTangentC)]
        lib.pbf_batch_reserve_caches.argtypes = [vp, ctypes.c_uint32]
        lib.pbf_set_launch_shape.argtypes = [vp, P(LaunchShapeC)]
        lib.pbf_get_launch_shape.argtypes = [vp, P(LaunchShapeC)]
        lib.pbf_autotune.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC), vp,
                                     ctypes.c_uint32, P(LaunchShapeC), P(ctypes.c_float)]
        lib.pbf_export_frame.argtypes = [vp, P(ParticleStateC), vp, P(FrameC)]
        lib.pbf_set_input_checks.argtypes = [vp, ctypes.c_int]
        lib.pbf_read_input_checks.argtypes = [vp, P(ctypes.c_uint32)]
        lib.pbf_batch_set_input_checks.argtypes = [vp, ctypes.c_int]
        lib.pbf_batch_read_input_checks.argtypes = [vp, P(ctypes.c_uint32)]
        lib.pbf_batch_set_launch_shape.argtypes = [vp, P(LaunchShapeC)]
        lib.pbf_batch_get_launch_shape.argtypes = [vp, P(LaunchShapeC)]
        lib.pbf_batch_autotune.argtypes = [vp, P(ParticleStateC), P(ControlC), P(ParametersC), P(ParticleStateC),
                                           ctypes.c_uint32, ctypes.c_uint32, P(LaunchShapeC), P(ctypes.c_float)]
        lib.pbf_batch_synchronize.argtypes = [vp]
        lib.pbf_batch_scene_sums.argtypes = [vp, vp, vp]
        lib.pbf_batch_set_graph_mode.argtypes = [vp, ctypes.c_int]
        lib.pbf_set_graph_mode.argtypes = [vp, ctypes.c_int]
        lib.pbf_set_checkpoint_recompute.argtypes = [vp, ctypes.c_int]
        lib.pbf_batch_set_checkpoint_recompute.argtypes = [vp, ctypes.c_int]
        lib.pbf_sum_compensated.argtypes = [vp, vp, ctypes.c_uint32, vp]
        lib.pbf_profile_enable.argtypes = [vp, ctypes.c_int]
        lib.pbf_batch_profile_enable.argtypes = [vp, ctypes.c_int]
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != 0:
        lib = library()
        raise PBFError(status, f"{lib.pbf_status_string(status).decode()}: {lib.pbf_last_error().decode()}")


def launch_count() -> int:
    return int(library().pbf_launch_count())


# ------------------------------------------------------------------------- host types
@dataclasses.dataclass
class BoxBoundary:
    minimum: tuple = (0.0, 0.0, 0.0)
    maximum: tuple = (1.0, 1.0, 1.0)
    velocity: tuple = (0.0, 0.0, 0.0)
    no_slip: bool = True


@dataclasses.dataclass
class DomainConfiguration:
    """domain/domain.ixx:221-229"""
    particle_count: int
    time_step: float
    support_radius: float
    particle_radius: float
    gravity: tuple = (0.0, -9.81, 0.0)
    boundary: BoxBoundary = dataclasses.field(default_factory=BoxBoundary)
    boundary_particles: list = dataclasses.field(default_factory=list)

    def to_c(self) -> DomainConfigurationC:
        c = DomainConfigurationC()
        c.particle_count = self.particle_count
        c.time_step = self.time_step
        c.support_radius = self.support_radius
        c.particle_radius = self.particle_radius
        c.gravity = Vector3(*self.gravity)
        c.boundary = BoxBoundaryC(Vector3(*self.boundary.minimum), Vector3(*self.boundary.maximum),
                                  Vector3(*self.boundary.velocity), 1 if self.boundary.no_slip else 0)
        if self.boundary_particles:
            arr = (BoundaryParticleC * len(self.boundary_particles))()
            for k, (pos, vel, vol) in enumerate(self.boundary_particles):
                arr[k] = BoundaryParticleC(Vector3(*pos), Vector3(*vel), vol)
            c.boundary_particles = ctypes.cast(arr, ctypes.POINTER(BoundaryParticleC))
            c._keep = arr
        c.boundary_particle_count = len(self.boundary_particles)
        return c

    @staticmethod
    def from_scene(scene) -> "DomainConfiguration":
        particles = []
        b = getattr(scene, "boundary", None)
        if b is not None:
            particles = [(tuple(b["positions"][:, k].tolist()), tuple(b["velocities"][:, k].tolist()), float(b["volumes"][k]))
                         for k in range(len(b["volumes"]))]
        return DomainConfiguration(
            particle_count=scene.count, time_step=scene.time_step, support_radius=scene.support_radius,
            particle_radius=scene.particle_radius, gravity=tuple(scene.gravity),
            boundary=BoxBoundary(tuple(scene.box_min), tuple(scene.box_max), tuple(scene.box_velocity),
                                 bool(getattr(scene, "no_slip", True))),
            boundary_particles=particles)


@dataclasses.dataclass
class Configuration:
    """pbf/pbf.ixx:15-18"""
    pressure_iterations: int = 5
    checkpoint_interval: int = 2


def _ptr(t: torch.Tensor) -> int:
    assert t.is_cuda and t.is_contiguous(), "fields must be contiguous CUDA tensors"
    return t.data_ptr()


def _vf(t: torch.Tensor) -> VectorFieldC:
    """(3, N) tensor -> x/y/z device pointers."""
    return VectorFieldC(_ptr(t[0]), _ptr(t[1]), _ptr(t[2])) if t.shape[1] else VectorFieldC(_ptr(t), _ptr(t), _ptr(t))


@dataclasses.dataclass
class State:
    """PBF::State (pbf/pbf.ixx:20): positions and velocities as (3, N) float32 tensors."""
    positions: torch.Tensor
    velocities: torch.Tensor
    step_index: int = 0

    def c(self) -> ParticleStateC:
        return ParticleStateC(_vf(self.positions), _vf(self.velocities), self.step_index)


@dataclasses.dataclass
class Control:
    external_accelerations: torch.Tensor

    def c(self) -> ControlC:
        return ControlC(_vf(self.external_accelerations))


@dataclasses.dataclass
class StateAdjoint:
    """PBF::StateAdjoint: (3, N) float64 tensors."""
    positions: torch.Tensor
    velocities: torch.Tensor

    def c(self) -> StateAdjointC:
        return StateAdjointC(_vf(self.positions), _vf(self.velocities))


@dataclasses.dataclass
class StateTangent:
    positions: torch.Tensor
    velocities: torch.Tensor

    def c(self) -> StateTangentC:
        return StateTangentC(_vf(self.positions), _vf(self.velocities))


class Parameters:
    """PBF::Parameters (pbf/pbf.ixx:24-32): one (N,) tensor per parameter."""

    def __init__(self, tensors: dict):
        self.tensors = tensors

    def __getattr__(self, name):
        if name in PARAMETER_NAMES:
            return self.tensors[name]
        raise AttributeError(name)

    def c(self) -> ParametersC:
        return ParametersC(*[_ptr(self.tensors[n]) if self.tensors.get(n) is not None else None for n in PARAMETER_NAMES])


class StepCache:
    """PBF::StepCache (pbf/pbf.ixx:54-70), owned by the library."""

    def __init__(self, solver: "PBF"):
        self.solver = solver
        h = ctypes.c_void_p()
        check(library().pbf_allocate_step_cache(solver.handle, ctypes.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            library().pbf_free_step_cache(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read(self, field: CacheField) -> torch.Tensor:
        """Copy a cache field (original particle order) into a new tensor."""
        s = self.solver
        n = s.count
        dev = s.device
        if field == CacheField.GRID_RESOLUTION:
            dims = (ctypes.c_uint32 * 3)()
            check(library().pbf_step_cache_read(s.handle, self.handle, int(field), ctypes.cast(dims, ctypes.c_void_p), 12))
            return torch.tensor(list(dims), dtype=torch.int64)
        if field in (CacheField.SORTED_PARTICLE_INDICES, CacheField.NEIGHBOR_COUNTS):
            out = torch.empty(n, dtype=torch.int32, device=dev)
        elif field == CacheField.CELL_OFFSETS:
            out = torch.empty(s.cells + 1, dtype=torch.int32, device=dev)
        elif field == CacheField.SORTED_KEYS:
            out = torch.empty(n, dtype=torch.int64, device=dev)
        elif field in (CacheField.VORTICITY_MAGNITUDES, CacheField.VORTICITY_NORMALIZERS, CacheField.FIRST_DENSITIES,
                       CacheField.FIRST_LAMBDAS):
            out = torch.empty(n, dtype=torch.float32, device=dev)
        else:
            out = torch.empty((3, n), dtype=torch.float32, device=dev)
        check(library().pbf_step_cache_read(s.handle, self.handle, int(field), out.data_ptr() if out.numel() else None,
                                            out.numel() * out.element_size()))
        return out


    def read_iteration(self, field: IterationField, iteration: int) -> torch.Tensor:
        """Copy a per-iteration field (original particle order) into a new tensor."""
        s = self.solver
        if field in (IterationField.POSITIONS, IterationField.GRADIENT_SUMS):
            out = torch.empty((3, s.count), dtype=torch.float32, device=s.device)
        elif field == IterationField.COLLISION_MASKS:
            out = torch.empty(s.count, dtype=torch.int32, device=s.device)
        else:
            out = torch.empty(s.count, dtype=torch.float32, device=s.device)
        check(library().pbf_step_cache_read_iteration(s.handle, self.handle, int(field), iteration,
                                                      out.data_ptr() if out.numel() else None,
                                                      out.numel() * out.element_size()))
        return out


class PBF:
    """The B200 PBF solver (pbf/pbf.ixx:14-141)."""

    def __init__(self, domain_configuration: DomainConfiguration, configuration: Configuration = Configuration(),
                 mode: ExecutionMode = ExecutionMode.forward, stream: torch.cuda.Stream | None = None,
                 device: torch.device | str = "cuda"):
        lib = library()
        self.device = torch.device(device)
        if self.device.type != "cuda" or not torch.cuda.is_available():
            raise RuntimeError("the PBF solver needs a CUDA device")
        self.domain_configuration = domain_configuration
        self.configuration = configuration
        self.mode = ExecutionMode(mode)
        self.stream = stream or torch.cuda.current_stream(self.device)
        self.count = int(domain_configuration.particle_count)
        h = ctypes.c_void_p()
        self._dc = domain_configuration.to_c()
        cc = ConfigurationC(configuration.pressure_iterations, configuration.checkpoint_interval)
        with torch.cuda.device(self.device):
            check(lib.pbf_create(ctypes.byref(self._dc), ctypes.byref(cc), int(self.mode),
                                 ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self.handle = h
        cells = ctypes.c_uint64()
        check(lib.pbf_grid_cell_count(self.handle, ctypes.byref(cells)))
        self.cells = int(cells.value)

    def close(self):
        if getattr(self, "handle", None):
            library().pbf_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- allocation (pbf/pbf.cpp:79-160) --
    def _vec(self, dtype=torch.float32, zero=True):
        f = torch.zeros if zero else torch.empty
        return f((3, self.count), dtype=dtype, device=self.device)

    def allocate_state(self) -> State:
        return State(self._vec(), self._vec(), 0)

    def allocate_control(self) -> Control:
        return Control(self._vec())

    def allocate_parameters(self) -> Parameters:
        return Parameters({n: torch.zeros(self.count, dtype=torch.float32, device=self.device) for n in PARAMETER_NAMES})

    def allocate_step_cache(self) -> StepCache:
        return StepCache(self)

    def allocate_state_adjoint(self) -> StateAdjoint:
        return StateAdjoint(self._vec(torch.float64), self._vec(torch.float64))

    def allocate_control_adjoint(self) -> Control:
        return Control(self._vec(torch.float64))

    def allocate_parameter_adjoint(self) -> Parameters:
        return Parameters({n: torch.zeros(self.count, dtype=torch.float64, device=self.device) for n in PARAMETER_NAMES})

    def allocate_state_tangent(self) -> StateTangent:
        return StateTangent(self._vec(), self._vec())

    def allocate_parameter_tangent(self) -> Parameters:
        return self.allocate_parameters()

    def parameters_from_scene(self, scene) -> Parameters:
        p = self.allocate_parameters()
        for k, v in scene.parameter_arrays().items():
            p.tensors[k].copy_(torch.from_numpy(v))
        return p

    def state_from_arrays(self, positions, velocities, step_index=0) -> State:
        s = self.allocate_state()
        s.positions.copy_(torch.as_tensor(positions))
        s.velocities.copy_(torch.as_tensor(velocities))
        s.step_index = step_index
        return s

    # -- steps --
    def forward_step(self, state: State, control: Control, parameters: Parameters, next_state: State, cache: StepCache):
        """pbf/pbf.cpp:167-191; next_state.step_index becomes state.step_index + 1."""
        sc, nc = state.c(), next_state.c()
        check(library().pbf_forward_step(self.handle, ctypes.byref(sc), ctypes.byref(control.c()),
                                         ctypes.byref(parameters.c()), ctypes.byref(nc), cache.handle))
        next_state.step_index = int(nc.step_index)

    def vjp_step(self, state: State, control: Control, parameters: Parameters, next_state: State, cache: StepCache,
                 next_state_adjoint: StateAdjoint, previous_state_adjoint: StateAdjoint, control_adjoint: Control,
                 parameter_adjoint: Parameters):
        """pbf/pbf.cpp:217-258; accumulates into the previous-state, control and parameter adjoints."""
        check(library().pbf_vjp_step(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                     ctypes.byref(parameters.c()), ctypes.byref(next_state.c()), cache.handle,
                                     ctypes.byref(next_state_adjoint.c()), ctypes.byref(previous_state_adjoint.c()),
                                     ctypes.byref(control_adjoint.c()), ctypes.byref(parameter_adjoint.c())))

    def jvp_step(self, state, control, parameters, next_state, cache, state_tangent, control_tangent, parameter_tangent,
                 next_state_tangent):
        """pbf/pbf.cpp:193-215."""
        check(library().pbf_jvp_step(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                     ctypes.byref(parameters.c()), ctypes.byref(next_state.c()), cache.handle,
                                     ctypes.byref(state_tangent.c()), ctypes.byref(control_tangent.c()),
                                     ctypes.byref(parameter_tangent.c()), ctypes.byref(next_state_tangent.c())))

    def forward_step_host(self, positions, velocities, control: Control, parameters: Parameters, out_positions,
                          out_velocities, cache: StepCache, step_index: int = 0) -> int:
        """forward_step over host (CPU) float32 (3, N) tensors; copies in and out and waits."""
        def hs(p, v, step):
            h = HostStateC()
            for a in range(3):
                h.positions[a] = p[a].data_ptr()
                h.velocities[a] = v[a].data_ptr()
            h.step_index = step
            return h
        hin = hs(positions, velocities, step_index)
        hout = hs(out_positions, out_velocities, 0)
        check(library().pbf_forward_step_host(self.handle, ctypes.byref(hin), ctypes.byref(control.c()),
                                              ctypes.byref(parameters.c()), ctypes.byref(hout), cache.handle))
        return int(hout.step_index)

    def copy_state(self, source: State, destination: State):
        dc = destination.c()
        check(library().pbf_copy_state(self.handle, ctypes.byref(source.c()), ctypes.byref(dc)))
        destination.step_index = source.step_index

    def copy_state_tangent(self, source: StateTangent, destination: StateTangent):
        """PBF::copy_state_tangent (pbf/pbf.cpp:163)."""
        check(library().pbf_copy_state_tangent(self.handle, ctypes.byref(source.c()), ctypes.byref(destination.c())))

    def copy_state_adjoint(self, source: StateAdjoint, destination: StateAdjoint):
        check(library().pbf_copy_state_adjoint(self.handle, ctypes.byref(source.c()), ctypes.byref(destination.c())))

    def accumulate_state_adjoint(self, source: StateAdjoint, destination: StateAdjoint):
        check(library().pbf_accumulate_state_adjoint(self.handle, ctypes.byref(source.c()), ctypes.byref(destination.c())))

    def synchronize(self):
        check(library().pbf_synchronize(self.handle))

    def set_graph_mode(self, enable: bool = True):
        """Replay the forward launch sequence as a CUDA graph per buffer set."""
        check(library().pbf_set_graph_mode(self.handle, 1 if enable else 0))

    def set_checkpoint_recompute(self, enable: bool = True):
        """Step caches allocated afterwards keep every checkpoint_interval-th Jacobi iterate only;
        vjp_step / jvp_step recompute the rest (the reference's StepCache::checkpoints)."""
        check(library().pbf_set_checkpoint_recompute(self.handle, 1 if enable else 0))

    def export_frame(self, state: State, cache: "StepCache | None" = None) -> dict:
        """Frame of `state` for a viewer or a file dump: positions and velocities as (N, 3) float32,
        and, with the step cache that produced `state`, the vorticity magnitudes (N,)."""
        n = self.count
        out = {"positions": torch.empty((n, 3), dtype=torch.float32, device=self.device),
               "velocities": torch.empty((n, 3), dtype=torch.float32, device=self.device)}
        if cache is not None:
            out["vorticity"] = torch.empty(n, dtype=torch.float32, device=self.device)
        f = FrameC(out["positions"].data_ptr() if n else None, out["velocities"].data_ptr() if n else None,
                   out["vorticity"].data_ptr() if cache is not None and n else None)
        check(library().pbf_export_frame(self.handle, ctypes.byref(state.c()), cache.handle if cache is not None else None,
                                         ctypes.byref(f)))
        out["step"] = state.step_index
        return out

    def set_input_checks(self, enable: bool = True):
        """Test every forward step's inputs on the device (see read_input_checks)."""
        check(library().pbf_set_input_checks(self.handle, 1 if enable else 0))

    def read_input_checks(self) -> int:
        """PBF_INPUT_* bits seen since the last read (synchronises), then cleared."""
        v = ctypes.c_uint32()
        check(library().pbf_read_input_checks(self.handle, ctypes.byref(v)))
        return int(v.value)

    @property
    def launch_shape(self) -> LaunchShape:
        c = LaunchShapeC()
        check(library().pbf_get_launch_shape(self.handle, ctypes.byref(c)))
        return LaunchShape.from_c(c)

    @launch_shape.setter
    def launch_shape(self, shape: LaunchShape):
        check(library().pbf_set_launch_shape(self.handle, ctypes.byref(shape.to_c())))

    def autotune(self, state: State, control: Control, parameters: Parameters, repeats: int = 2):
        """Time every launch shape on forward steps from `state` and keep the fastest.
        Returns (shape, milliseconds per step)."""
        scratch = self.allocate_state()
        cache = self.allocate_step_cache()
        c, ms = LaunchShapeC(), ctypes.c_float()
        check(library().pbf_autotune(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                     ctypes.byref(parameters.c()), ctypes.byref(scratch.c()), cache.handle, repeats,
                                     ctypes.byref(c), ctypes.byref(ms)))
        return LaunchShape.from_c(c), float(ms.value)


class Batch:
    """Many independent scenes advanced together (pbf_batch_*).

    Particle arrays are the scenes' arrays concatenated in scene order; `particle_range(s)` gives a
    scene's slice.  Each scene evolves exactly as a separate PBF solver would.
    """

    def __init__(self, domain_configurations: list, configuration: Configuration = Configuration(),
                 mode: ExecutionMode = ExecutionMode.forward, stream: torch.cuda.Stream | None = None,
                 device: torch.device | str = "cuda"):
        lib = library()
        self.device = torch.device(device)
        self.mode = ExecutionMode(mode)
        self.stream = stream or torch.cuda.current_stream(self.device)
        self._dcs = [d.to_c() for d in domain_configurations]
        arr = (DomainConfigurationC * len(self._dcs))(*self._dcs)
        self._arr = arr
        cc = ConfigurationC(configuration.pressure_iterations, configuration.checkpoint_interval)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(lib.pbf_batch_create(arr, len(self._dcs), ctypes.byref(cc), int(self.mode),
                                       ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self.handle = h
        self.scene_count = len(self._dcs)
        self.ranges = []
        for s in range(self.scene_count):
            off, cnt = ctypes.c_uint32(), ctypes.c_uint32()
            check(lib.pbf_batch_particle_offset(self.handle, s, ctypes.byref(off), ctypes.byref(cnt)))
            self.ranges.append((int(off.value), int(cnt.value)))
        self.count = sum(c for _, c in self.ranges)

    def close(self):
        if getattr(self, "handle", None):
            library().pbf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def particle_range(self, scene: int) -> slice:
        off, cnt = self.ranges[scene]
        return slice(off, off + cnt)

    def _vec(self, dtype=torch.float32):
        return torch.zeros((3, self.count), dtype=dtype, device=self.device)

    def allocate_state(self) -> State:
        return State(self._vec(), self._vec(), 0)

    def allocate_state_adjoint(self) -> StateAdjoint:
        return StateAdjoint(self._vec(torch.float64), self._vec(torch.float64))

    def allocate_control_adjoint(self) -> Control:
        return Control(self._vec(torch.float64))

    def allocate_parameter_adjoint(self) -> Parameters:
        return Parameters({n: torch.zeros(self.count, dtype=torch.float64, device=self.device) for n in PARAMETER_NAMES})

    def reserve_caches(self, slots: int):
        check(library().pbf_batch_reserve_caches(self.handle, slots))

    def forward_step(self, state: State, control: Control, parameters: Parameters, next_state: State, cache_slot: int = 0):
        nc = next_state.c()
        check(library().pbf_batch_forward_step(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                               ctypes.byref(parameters.c()), ctypes.byref(nc), cache_slot))
        next_state.step_index = int(nc.step_index)

    def vjp_step(self, state, control, parameters, next_state, cache_slot, next_state_adjoint, previous_state_adjoint,
                 control_adjoint, parameter_adjoint):
        check(library().pbf_batch_vjp_step(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                           ctypes.byref(parameters.c()), ctypes.byref(next_state.c()), cache_slot,
                                           ctypes.byref(next_state_adjoint.c()), ctypes.byref(previous_state_adjoint.c()),
                                           ctypes.byref(control_adjoint.c()), ctypes.byref(parameter_adjoint.c())))

    def jvp_step(self, state, control, parameters, next_state, cache_slot, state_tangent, control_tangent,
                 parameter_tangent, next_state_tangent):
        check(library().pbf_batch_jvp_step(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                           ctypes.byref(parameters.c()), ctypes.byref(next_state.c()), cache_slot,
                                           ctypes.byref(state_tangent.c()), ctypes.byref(control_tangent.c()),
                                           ctypes.byref(parameter_tangent.c()), ctypes.byref(next_state_tangent.c())))

    def allocate_state_tangent(self) -> StateTangent:
        return StateTangent(self._vec(), self._vec())

    def scene_sums(self, values: torch.Tensor) -> torch.Tensor:
        """Compensated FP64 per-scene sums of a per-particle FP64 vector."""
        out = torch.empty(self.scene_count, dtype=torch.float64, device=self.device)
        check(library().pbf_batch_scene_sums(self.handle, ctypes.c_void_p(values.data_ptr()), ctypes.c_void_p(out.data_ptr())))
        return out

    def set_graph_mode(self, enable: bool = True):
        check(library().pbf_batch_set_graph_mode(self.handle, 1 if enable else 0))

    def set_checkpoint_recompute(self, enable: bool = True):
        """Cache slots reserved afterwards keep every checkpoint_interval-th Jacobi iterate only."""
        check(library().pbf_batch_set_checkpoint_recompute(self.handle, 1 if enable else 0))

    def set_input_checks(self, enable: bool = True):
        check(library().pbf_batch_set_input_checks(self.handle, 1 if enable else 0))

    def read_input_checks(self) -> int:
        v = ctypes.c_uint32()
        check(library().pbf_batch_read_input_checks(self.handle, ctypes.byref(v)))
        return int(v.value)

    @property
    def launch_shape(self) -> LaunchShape:
        c = LaunchShapeC()
        check(library().pbf_batch_get_launch_shape(self.handle, ctypes.byref(c)))
        return LaunchShape.from_c(c)

    @launch_shape.setter
    def launch_shape(self, shape: LaunchShape):
        check(library().pbf_batch_set_launch_shape(self.handle, ctypes.byref(shape.to_c())))

    def autotune(self, state: State, control: Control, parameters: Parameters, repeats: int = 2, cache_slot: int = 0):
        """Time every launch shape on batched forward steps from `state` and keep the fastest.
        Returns (shape, milliseconds per step)."""
        scratch = self.allocate_state()
        c, ms = LaunchShapeC(), ctypes.c_float()
        check(library().pbf_batch_autotune(self.handle, ctypes.byref(state.c()), ctypes.byref(control.c()),
                                           ctypes.byref(parameters.c()), ctypes.byref(scratch.c()), cache_slot, repeats,
                                           ctypes.byref(c), ctypes.byref(ms)))
        return LaunchShape.from_c(c), float(ms.value)

    def synchronize(self):
        check(library().pbf_batch_synchronize(self.handle))


def batch_for_scenes(scene_list, mode=ExecutionMode.forward, checkpoint_interval=2, device="cuda"):
    """A batch, its concatenated state, control and parameters for synthetic scenes (physica_b200.scenes)."""
    import numpy as np
    iters = {s.pressure_iterations for s in scene_list}
    if len(iters) != 1:
        raise ValueError("all scenes of a batch share the Jacobi iteration count")
    batch = Batch([DomainConfiguration.from_scene(s) for s in scene_list],
                  Configuration(iters.pop(), checkpoint_interval), mode, device=device)
    cat = lambda key: torch.from_numpy(np.concatenate([getattr(s, key) for s in scene_list], axis=-1)).to(batch.device)
    state = State(cat("positions").contiguous(), cat("velocities").contiguous(), 0)
    control = Control(cat("controls").contiguous())
    params = Parameters({n: torch.zeros(batch.count, dtype=torch.float32, device=batch.device) for n in PARAMETER_NAMES})
    for k in scene_list[0].parameter_arrays():
        params.tensors[k].copy_(torch.from_numpy(np.concatenate([s.parameter_arrays()[k] for s in scene_list])))
    return batch, state, control, params


def solver_for_scene(scene, mode=ExecutionMode.forward, checkpoint_interval=2, device="cuda"):
    """A solver, state, control and parameters for a synthetic scene (physica_b200.scenes)."""
    dc = DomainConfiguration.from_scene(scene)
    solver = PBF(dc, Configuration(scene.pressure_iterations, checkpoint_interval), mode, device=device)
    state = solver.state_from_arrays(scene.positions, scene.velocities)
    control = solver.allocate_control()
    control.external_accelerations.copy_(torch.from_numpy(scene.controls))
    params = solver.parameters_from_scene(scene)
    return solver, state, control, params
