"""ctypes front end of the FP64 host oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/lib/libpbf_oracle.so (built from oracle/pbf_oracle.c by
oracle/build.py).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use this module; the CUDA solver never imports it.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libpbf_oracle.so"

c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)


class OracleVec(ctypes.Structure):
    _fields_ = [("x", c_double_p), ("y", c_double_p), ("z", c_double_p)]


class OracleScene(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_uint32),
        ("iterations", ctypes.c_uint32),
        ("step_index", ctypes.c_uint64),
        ("time_step", ctypes.c_float),
        ("support_radius", ctypes.c_float),
        ("particle_radius", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("box_min", ctypes.c_float * 3),
        ("box_max", ctypes.c_float * 3),
        ("box_velocity", ctypes.c_float * 3),
        ("boundary_count", ctypes.c_uint32),
        ("boundary_position", c_double_p * 3),
        ("boundary_velocity", c_double_p * 3),
        ("boundary_volume", c_double_p),
    ]


class OracleParameters(ctypes.Structure):
    _fields_ = [(name, c_double_p) for name in (
        "masses", "rest_densities", "relaxation", "artificial_pressure_strength",
        "artificial_pressure_exponent", "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")]


class OracleTrace(ctypes.Structure):
    _fields_ = [
        ("predicted", OracleVec),
        ("density0", c_double_p),
        ("lambda0", c_double_p),
        ("corrected", OracleVec),
        ("vorticity", OracleVec),
        ("confined_velocity", OracleVec),
        ("neighbor_count0", c_u32_p),
    ]


class OracleAdjoint(ctypes.Structure):
    _fields_ = [
        ("next_position", OracleVec), ("next_velocity", OracleVec),
        ("position", OracleVec), ("velocity", OracleVec), ("control", OracleVec),
    ] + [(name, c_double_p) for name in (
        "masses", "rest_densities", "relaxation", "artificial_pressure_strength",
        "artificial_pressure_exponent", "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from oracle import build as _build  # noqa: PLC0415
            _build.build_oracle()
        lib = ctypes.CDLL(str(LIB_PATH))
        lib.oracle_forward_step.argtypes = [ctypes.POINTER(OracleScene), ctypes.POINTER(OracleParameters),
                                            OracleVec, OracleVec, OracleVec, OracleVec, OracleVec,
                                            ctypes.POINTER(OracleTrace)]
        lib.oracle_vjp_step.argtypes = [ctypes.POINTER(OracleScene), ctypes.POINTER(OracleParameters),
                                        OracleVec, OracleVec, OracleVec, ctypes.POINTER(OracleAdjoint)]
        lib.oracle_grid_dims.argtypes = [ctypes.c_float * 3, ctypes.c_float * 3, ctypes.c_float, ctypes.c_uint32 * 3]
        lib.oracle_grid_f32.argtypes = [ctypes.c_uint32, c_float_p, c_float_p, c_float_p, ctypes.c_float,
                                        ctypes.c_float * 3, ctypes.c_float * 3, ctypes.c_float * 3, ctypes.c_float,
                                        c_u32_p, c_u32_p, c_u32_p]
        lib.oracle_neighbor_counts_f32.argtypes = [ctypes.c_uint32, c_float_p * 3, c_float_p * 3, ctypes.c_float,
                                                   ctypes.c_float * 3, ctypes.c_float * 3, ctypes.c_float * 3,
                                                   ctypes.c_float, c_u32_p]
        lib.oracle_poly6.argtypes = [ctypes.c_double] * 4
        lib.oracle_poly6.restype = ctypes.c_double
        lib.oracle_spiky_gradient.argtypes = [ctypes.c_double] * 4 + [ctypes.c_double * 3]
        lib.oracle_thread_count.restype = ctypes.c_int
        _lib = lib
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(c_double_p)


def _vec(a: np.ndarray) -> OracleVec:
    """(3, N) float64 C-contiguous array -> OracleVec."""
    assert a.dtype == np.float64 and a.flags.c_contiguous and a.shape[0] == 3
    return OracleVec(_dp(a[0]), _dp(a[1]), _dp(a[2]))


def _f3(v):
    return (ctypes.c_float * 3)(*[float(np.float32(x)) for x in v])


def make_scene(scene, step_index=0) -> OracleScene:
    s = OracleScene()
    s.count = scene.count
    s.iterations = scene.pressure_iterations
    s.step_index = step_index
    s.time_step = scene.time_step
    s.support_radius = scene.support_radius
    s.particle_radius = scene.particle_radius
    s.gravity = _f3(scene.gravity)
    s.box_min = _f3(scene.box_min)
    s.box_max = _f3(scene.box_max)
    s.box_velocity = _f3(scene.box_velocity)
    s.boundary_count = 0
    return s


class Parameters:
    """FP64 copies of the per-particle parameter arrays, kept alive with their ctypes view."""

    def __init__(self, scene, xsph_override=None):
        arrays = scene.parameter_arrays()
        self.arrays = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in arrays.items()}
        if xsph_override is not None:
            self.arrays["xsph_viscosity"] = np.full(scene.count, float(xsph_override), dtype=np.float64)
        self.struct = OracleParameters(**{k: _dp(v) for k, v in self.arrays.items()})


def forward_step(scene, positions, velocities, controls=None, step_index=0, trace=False, params=None):
    """One FP64 substep; inputs are (3, N) arrays.  Returns (x1, v1[, trace dict])."""
    lib = load()
    n = scene.count
    x0 = np.ascontiguousarray(positions, dtype=np.float64)
    v0 = np.ascontiguousarray(velocities, dtype=np.float64)
    a0 = np.ascontiguousarray(controls if controls is not None else np.zeros((3, n)), dtype=np.float64)
    x1 = np.zeros((3, n)); v1 = np.zeros((3, n))
    sc = make_scene(scene, step_index)
    params = params or Parameters(scene)
    tr = None
    out = {}
    if trace:
        out = {"predicted": np.zeros((3, n)), "density0": np.zeros(n), "lambda0": np.zeros(n),
               "corrected": np.zeros((3, n)), "vorticity": np.zeros((3, n)), "confined_velocity": np.zeros((3, n)),
               "neighbor_count0": np.zeros(n, dtype=np.uint32)}
        tr = OracleTrace(predicted=_vec(out["predicted"]), density0=_dp(out["density0"]), lambda0=_dp(out["lambda0"]),
                         corrected=_vec(out["corrected"]), vorticity=_vec(out["vorticity"]),
                         confined_velocity=_vec(out["confined_velocity"]),
                         neighbor_count0=out["neighbor_count0"].ctypes.data_as(c_u32_p))
    rc = lib.oracle_forward_step(ctypes.byref(sc), ctypes.byref(params.struct), _vec(x0), _vec(v0), _vec(a0),
                                 _vec(x1), _vec(v1), ctypes.byref(tr) if tr is not None else None)
    if rc:
        raise RuntimeError(f"oracle_forward_step failed with status {rc}")
    return (x1, v1, out) if trace else (x1, v1)


def vjp_step(scene, positions, velocities, next_position_adjoint, next_velocity_adjoint, controls=None,
             step_index=0, params=None):
    """FP64 VJP of one substep.  Returns dict of adjoints (positions, velocities, controls, per-particle params)."""
    lib = load()
    n = scene.count
    x0 = np.ascontiguousarray(positions, dtype=np.float64)
    v0 = np.ascontiguousarray(velocities, dtype=np.float64)
    a0 = np.ascontiguousarray(controls if controls is not None else np.zeros((3, n)), dtype=np.float64)
    out = {k: np.zeros((3, n)) for k in ("position", "velocity", "control")}
    names = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
             "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")
    for k in names:
        out[k] = np.zeros(n)
    nx = np.ascontiguousarray(next_position_adjoint, dtype=np.float64)
    nv = np.ascontiguousarray(next_velocity_adjoint, dtype=np.float64)
    adj = OracleAdjoint(next_position=_vec(nx), next_velocity=_vec(nv), position=_vec(out["position"]),
                        velocity=_vec(out["velocity"]), control=_vec(out["control"]),
                        **{k: _dp(out[k]) for k in names})
    sc = make_scene(scene, step_index)
    params = params or Parameters(scene)
    rc = lib.oracle_vjp_step(ctypes.byref(sc), ctypes.byref(params.struct), _vec(x0), _vec(v0), _vec(a0),
                             ctypes.byref(adj))
    if rc:
        raise RuntimeError(f"oracle_vjp_step failed with status {rc}")
    return out


def grid_f32(scene, topology, time):
    """Reference-semantics FP32 grid of (3, N) float32 points: keys, stable sorted indices, cell offsets."""
    lib = load()
    dims = (ctypes.c_uint32 * 3)()
    if lib.oracle_grid_dims(_f3(scene.box_min), _f3(scene.box_max), ctypes.c_float(scene.support_radius), dims):
        raise ValueError("invalid grid")
    cells = int(dims[0]) * int(dims[1]) * int(dims[2])
    t = np.ascontiguousarray(topology, dtype=np.float32)
    n = t.shape[1]
    keys = np.zeros(n, dtype=np.uint32); srt = np.zeros(n, dtype=np.uint32); off = np.zeros(cells + 1, dtype=np.uint32)
    fp = lambda a: a.ctypes.data_as(c_float_p)
    up = lambda a: a.ctypes.data_as(c_u32_p)
    rc = lib.oracle_grid_f32(n, fp(t[0]), fp(t[1]), fp(t[2]), ctypes.c_float(scene.support_radius),
                             _f3(scene.box_min), _f3(scene.box_max), _f3(scene.box_velocity), ctypes.c_float(time),
                             up(keys), up(srt), up(off))
    if rc:
        raise RuntimeError(f"oracle_grid_f32 failed with status {rc}")
    return keys, srt, off, tuple(int(d) for d in dims)


def neighbor_counts_f32(scene, topology, positions, time):
    lib = load()
    t = np.ascontiguousarray(topology, dtype=np.float32)
    p = np.ascontiguousarray(positions, dtype=np.float32)
    n = t.shape[1]
    counts = np.zeros(n, dtype=np.uint32)
    tp = (c_float_p * 3)(*[t[a].ctypes.data_as(c_float_p) for a in range(3)])
    pp = (c_float_p * 3)(*[p[a].ctypes.data_as(c_float_p) for a in range(3)])
    rc = lib.oracle_neighbor_counts_f32(n, tp, pp, ctypes.c_float(scene.support_radius), _f3(scene.box_min),
                                        _f3(scene.box_max), _f3(scene.box_velocity), ctypes.c_float(time),
                                        counts.ctypes.data_as(c_u32_p))
    if rc:
        raise RuntimeError(f"oracle_neighbor_counts_f32 failed with status {rc}")
    return counts


def thread_count() -> int:
    return int(load().oracle_thread_count())


def poly6(d, h):
    return load().oracle_poly6(float(d[0]), float(d[1]), float(d[2]), float(h))


def spiky_gradient(d, h):
    out = (ctypes.c_double * 3)()
    load().oracle_spiky_gradient(float(d[0]), float(d[1]), float(d[2]), float(h), out)
    return np.array(out[:])
