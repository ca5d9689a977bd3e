"""ctypes front end of the reference's own CUDA PBF (oracle/_ref/libpbf_ref.so) -- TEST INFRASTRUCTURE ONLY.

The library is compiled from the reference sources by oracle/build.py and driven by
oracle/ref_harness.cu.  Tests use it to pin parity against the reference itself; bench.py
uses it as the reference arm.  Nothing in physica_b200 imports this module.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libpbf_ref.so"


class RefConfig(ctypes.Structure):
    _fields_ = [
        ("particle_count", ctypes.c_uint32),
        ("time_step", ctypes.c_float), ("support_radius", ctypes.c_float), ("particle_radius", ctypes.c_float),
        ("gravity", ctypes.c_float * 3), ("box_min", ctypes.c_float * 3), ("box_max", ctypes.c_float * 3),
        ("box_velocity", ctypes.c_float * 3), ("no_slip", ctypes.c_uint32),
        ("pressure_iterations", ctypes.c_uint32), ("checkpoint_interval", ctypes.c_uint32),
        ("differentiable", ctypes.c_int),
    ]


class RefStateIn(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("px", "py", "pz", "vx", "vy", "vz")]


RefStateOut = RefStateIn
RefAdjointState = RefStateIn


class RefParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("masses", "rest_densities", "relaxation", "strength", "exponent",
                                               "radius", "xsph", "vorticity")]


RefParamAdjoint = RefParams

FIELDS = {"sorted_keys": 0, "sorted_indices": 1, "cell_offsets": 2, "predicted": 3, "corrected": 4,
          "reconstructed": 5, "vorticities": 6, "magnitudes": 7, "normals": 8, "normalizers": 9, "confined": 10,
          "first_densities": 11, "first_lambdas": 12}

_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        P = ctypes.POINTER
        lib.ref_create.argtypes = [P(RefConfig), P(vp)]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_forward_step.argtypes = [vp, P(RefStateIn), P(vp), P(RefParams), P(RefStateOut), ctypes.c_uint64]
        lib.ref_set_boundary.argtypes = [vp, P(vp), P(vp), vp, ctypes.c_uint32]
        lib.ref_jvp_step.argtypes = [vp, P(RefStateIn), P(RefParams), P(RefStateIn), P(vp), P(RefParams), P(RefStateOut)]
        lib.ref_vjp_step.argtypes = [vp, P(RefStateIn), P(RefParams), P(RefAdjointState), P(RefAdjointState), P(vp),
                                     P(RefParamAdjoint)]
        lib.ref_read.argtypes = [vp, ctypes.c_int, vp]
        lib.ref_cells.argtypes = [vp, P(ctypes.c_uint32)]
        lib.ref_synchronize.argtypes = [vp]
        lib.ref_stream.argtypes = [vp]
        lib.ref_stream.restype = vp
        _lib = lib
    return _lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


class ReferencePBF:
    """The reference PBF kernels replayed by the harness, on device tensors."""

    def __init__(self, scene, checkpoint_interval=2, differentiable=False, device="cuda"):
        lib = load()
        self.scene = scene
        self.device = torch.device(device)
        c = RefConfig()
        c.particle_count = scene.count
        c.time_step = scene.time_step
        c.support_radius = scene.support_radius
        c.particle_radius = scene.particle_radius
        c.gravity = (ctypes.c_float * 3)(*scene.gravity)
        c.box_min = (ctypes.c_float * 3)(*scene.box_min)
        c.box_max = (ctypes.c_float * 3)(*scene.box_max)
        c.box_velocity = (ctypes.c_float * 3)(*scene.box_velocity)
        c.no_slip = 1 if getattr(scene, "no_slip", True) else 0
        c.pressure_iterations = scene.pressure_iterations
        c.checkpoint_interval = checkpoint_interval
        c.differentiable = 1 if differentiable else 0
        h = ctypes.c_void_p()
        torch.cuda.synchronize(self.device)
        rc = lib.ref_create(ctypes.byref(c), ctypes.byref(h))
        if rc:
            raise RuntimeError(f"ref_create failed: {rc}")
        self.handle = h
        dims = (ctypes.c_uint32 * 3)()
        lib.ref_cells(h, dims)
        self.dims = tuple(dims)
        self.cells = dims[0] * dims[1] * dims[2]
        n = scene.count
        f = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.device)
        self.params = {k: torch.from_numpy(v).to(self.device) for k, v in scene.parameter_arrays().items()}
        self.controls = torch.from_numpy(scene.controls).to(self.device).contiguous()
        self.n = n
        b = getattr(scene, "boundary", None)
        if b is not None and len(b["volumes"]):
            keep = [np.ascontiguousarray(b[k], dtype=np.float32) for k in ("positions", "velocities", "volumes")]
            pp = (ctypes.c_void_p * 3)(*[keep[0][a].ctypes.data for a in range(3)])
            vv = (ctypes.c_void_p * 3)(*[keep[1][a].ctypes.data for a in range(3)])
            rc = lib.ref_set_boundary(h, pp, vv, ctypes.c_void_p(keep[2].ctypes.data), len(b["volumes"]))
            if rc:
                raise RuntimeError(f"ref_set_boundary failed: {rc}")

    @property
    def stream(self):
        return load().ref_stream(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            load().ref_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _pstruct(self):
        p = self.params
        return RefParams(_p(p["masses"]), _p(p["rest_densities"]), _p(p["relaxation"]),
                         _p(p["artificial_pressure_strength"]), _p(p["artificial_pressure_exponent"]),
                         _p(p["artificial_pressure_radius"]), _p(p["xsph_viscosity"]), _p(p["vorticity_confinement"]))

    def forward_step(self, x, v, x_out, v_out, step_index, synchronize=True):
        """x, v, x_out, v_out: (3, N) float32 CUDA tensors."""
        lib = load()
        sin = RefStateIn(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]))
        sout = RefStateOut(_p(x_out[0]), _p(x_out[1]), _p(x_out[2]), _p(v_out[0]), _p(v_out[1]), _p(v_out[2]))
        ctrl = (ctypes.c_void_p * 3)(self.controls[0].data_ptr(), self.controls[1].data_ptr(), self.controls[2].data_ptr())
        self._keep = (sin, sout, ctrl)
        rc = lib.ref_forward_step(self.handle, ctypes.byref(sin), ctrl, ctypes.byref(self._pstruct()), ctypes.byref(sout),
                                  step_index)
        if rc:
            raise RuntimeError(f"ref_forward_step failed: {rc}")
        if synchronize:
            lib.ref_synchronize(self.handle)

    def vjp_step(self, x, v, next_adjoint, previous_adjoint, control_adjoint, param_adjoint):
        """Adjoints are dicts of float64 CUDA tensors; outputs are accumulated."""
        lib = load()
        sin = RefStateIn(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]))
        na = RefAdjointState(*[_p(next_adjoint[k][a]) for k in ("positions", "velocities") for a in range(3)])
        pa = RefAdjointState(*[_p(previous_adjoint[k][a]) for k in ("positions", "velocities") for a in range(3)])
        ca = (ctypes.c_void_p * 3)(*[control_adjoint[a].data_ptr() for a in range(3)])
        g = param_adjoint
        pp = RefParamAdjoint(_p(g["masses"]), _p(g["rest_densities"]), _p(g["relaxation"]),
                             _p(g["artificial_pressure_strength"]), _p(g["artificial_pressure_exponent"]),
                             _p(g["artificial_pressure_radius"]), _p(g["xsph_viscosity"]), _p(g["vorticity_confinement"]))
        torch.cuda.synchronize(self.device)
        rc = lib.ref_vjp_step(self.handle, ctypes.byref(sin), ctypes.byref(self._pstruct()), ctypes.byref(na),
                              ctypes.byref(pa), ca, ctypes.byref(pp))
        if rc:
            raise RuntimeError(f"ref_vjp_step failed: {rc}")
        lib.ref_synchronize(self.handle)

    def jvp_step(self, x, v, tangent, control_tangent, param_tangent, next_tangent, synchronize=True):
        """PBF::jvp_step after forward_step of (x, v).  tangent / next_tangent: dicts with (3, N)
        float32 CUDA tensors "positions" and "velocities"; param_tangent: dict of float32 (N,) tensors.
        synchronize=False leaves the launches queued on the harness's stream (inputs must be ready)."""
        lib = load()
        sin = RefStateIn(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]))
        tin = RefStateIn(*[_p(tangent[k][a]) for k in ("positions", "velocities") for a in range(3)])
        tout = RefStateOut(*[_p(next_tangent[k][a]) for k in ("positions", "velocities") for a in range(3)])
        ct = (ctypes.c_void_p * 3)(*[control_tangent[a].data_ptr() for a in range(3)])
        g = param_tangent
        pt = RefParams(_p(g["masses"]), _p(g["rest_densities"]), _p(g["relaxation"]),
                       _p(g["artificial_pressure_strength"]), _p(g["artificial_pressure_exponent"]),
                       _p(g["artificial_pressure_radius"]), _p(g["xsph_viscosity"]), _p(g["vorticity_confinement"]))
        if synchronize:
            torch.cuda.synchronize(self.device)
        self._keep_tangent = (sin, tin, tout, ct, pt)
        rc = lib.ref_jvp_step(self.handle, ctypes.byref(sin), ctypes.byref(self._pstruct()), ctypes.byref(tin), ct,
                              ctypes.byref(pt), ctypes.byref(tout))
        if rc:
            raise RuntimeError(f"ref_jvp_step failed: {rc}")
        if synchronize:
            lib.ref_synchronize(self.handle)

    def read(self, field: str) -> torch.Tensor:
        n = self.n
        code = FIELDS[field]
        if code == 0:
            out = torch.empty(n, dtype=torch.int64, device=self.device)
        elif code == 1:
            out = torch.empty(n, dtype=torch.int32, device=self.device)
        elif code == 2:
            out = torch.empty(self.cells + 1, dtype=torch.int32, device=self.device)
        elif code in (7, 9, 11, 12):
            out = torch.empty(n, dtype=torch.float32, device=self.device)
        else:
            out = torch.empty((3, n), dtype=torch.float32, device=self.device)
        torch.cuda.synchronize(self.device)
        rc = load().ref_read(self.handle, code, ctypes.c_void_p(out.data_ptr()))
        if rc:
            raise RuntimeError(f"ref_read failed: {rc}")
        return out


class RefSphConfig(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("pressure_iterations", ctypes.c_uint32), ("divergence_iterations", ctypes.c_uint32),
                ("density_iterations", ctypes.c_uint32), ("pressure_warm_start", ctypes.c_int),
                ("checkpoint_interval", ctypes.c_uint32), ("differentiable", ctypes.c_int)]


class RefSphParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("masses", "rest_densities", "viscosities", "surface_tensions", "method0",
                                               "method1", "method2")]


SPH_FIELDS = {"densities": 0, "pressures": 1, "pressure_accelerations": 2, "viscosity_accelerations": 3,
              "surface_accelerations": 4, "predicted_densities": 5, "total_accelerations": 6}
SPH_METHOD_PARAMETERS = {0: ("speed_of_sound", "tait_exponent", "boundary_surface_tension"), 1: ("pressure_relaxation",),
                         2: ("jacobi_relaxation",), 3: ("divergence_relaxation", "density_relaxation")}


def _load_sph():
    lib = load()
    if not getattr(lib, "_sph_bound", False):
        vp = ctypes.c_void_p
        P = ctypes.POINTER
        lib.ref_sph_create.argtypes = [vp, P(RefSphConfig), P(vp)]
        lib.ref_sph_destroy.argtypes = [vp]
        lib.ref_sph_forward_step.argtypes = [vp, P(RefStateIn), P(vp), P(RefSphParams), vp, vp, P(RefStateOut), vp, vp,
                                             ctypes.c_uint64]
        lib.ref_sph_read.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        lib.ref_sph_jvp_step.argtypes = [vp, P(RefStateIn), P(RefSphParams), P(RefStateIn), P(vp), P(vp), P(vp), P(vp),
                                         P(RefStateOut), P(vp), ctypes.c_uint64, vp, vp]
        lib.ref_sph_vjp_step.argtypes = [vp, P(RefStateIn), P(RefSphParams), P(vp), P(vp), P(vp), P(vp), P(vp), P(vp), P(vp),
                                         ctypes.c_uint64]
        lib.ref_sph_reference_gradient_norm.argtypes = [vp]
        lib.ref_sph_reference_gradient_norm.restype = ctypes.c_float
        lib._sph_bound = True
    return lib


class ReferenceSPH:
    """The reference SPH<Method>::forward_step replayed by the harness (ref_sph_* in
    oracle/ref_harness.cu) over the reference's own sph/*.cu kernels, on device tensors.
    method: 0 WCSPH, 1 PCISPH, 2 IISPH, 3 DFSPH; scene.sph holds the parameter arrays."""

    def __init__(self, scene, method, pressure_iterations=6, divergence_iterations=4, density_iterations=6,
                 pressure_warm_start=True, checkpoint_interval=2, differentiable=False, device="cuda"):
        self.base = ReferencePBF(scene, device=device)
        lib = _load_sph()
        self.method = int(method)
        c = RefSphConfig(self.method, pressure_iterations, divergence_iterations, density_iterations,
                         1 if pressure_warm_start else 0, checkpoint_interval, 1 if differentiable else 0)
        h = ctypes.c_void_p()
        rc = lib.ref_sph_create(self.base.handle, ctypes.byref(c), ctypes.byref(h))
        if rc:
            raise RuntimeError(f"ref_sph_create failed: {rc}")
        self.handle = h
        self.device = self.base.device
        self.n = scene.count
        self.params = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.device) for k, v in scene.sph.items()}
        self.controls = self.base.controls

    @property
    def stream(self):
        return self.base.stream

    @property
    def reference_gradient_norm(self) -> float:
        return float(_load_sph().ref_sph_reference_gradient_norm(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            _load_sph().ref_sph_destroy(self.handle)
            self.handle = None
        self.base.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _pstruct(self):
        p = self.params
        names = list(SPH_METHOD_PARAMETERS[self.method]) + [SPH_METHOD_PARAMETERS[self.method][0]] * 3
        return RefSphParams(_p(p["masses"]), _p(p["rest_densities"]), _p(p["viscosities"]), _p(p["surface_tensions"]),
                            _p(p[names[0]]), _p(p[names[1]]), _p(p[names[2]]))

    def forward_step(self, x, v, x_out, v_out, step_index, warm=None, warm_out=None, synchronize=True):
        """x, v, x_out, v_out: (3, N) float32 CUDA tensors; warm / warm_out: DFSPH's (divergence,
        density) warm-start pressure tensors (N,) float32."""
        lib = _load_sph()
        sin = RefStateIn(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]))
        sout = RefStateOut(_p(x_out[0]), _p(x_out[1]), _p(x_out[2]), _p(v_out[0]), _p(v_out[1]), _p(v_out[2]))
        ctrl = (ctypes.c_void_p * 3)(self.controls[0].data_ptr(), self.controls[1].data_ptr(), self.controls[2].data_ptr())
        w = warm if warm is not None else (None, None)
        wo = warm_out if warm_out is not None else (None, None)
        args = [ctypes.c_void_p(t.data_ptr()) if t is not None else None for t in (*w, *wo)]
        params = self._pstruct()
        self._keep = (sin, sout, ctrl, params)
        rc = lib.ref_sph_forward_step(self.handle, ctypes.byref(sin), ctrl, ctypes.byref(params), args[0], args[1],
                                      ctypes.byref(sout), args[2], args[3], step_index)
        if rc:
            raise RuntimeError(f"ref_sph_forward_step failed: {rc}")
        if synchronize:
            load().ref_synchronize(self.base.handle)

    def _method_names(self):
        names = list(SPH_METHOD_PARAMETERS[self.method])
        return names + [names[0]] * (3 - len(names))

    def jvp_step(self, x, v, tangent, control_tangent, param_tangent, next_tangent, step_index, warm=None, warm_tangent=None,
                 next_warm_tangent=None, synchronize=True):
        """SPH<Method>::jvp_step after forward_step of (x, v).  tangent / next_tangent: dicts of (3, N)
        float32 tensors "positions" / "velocities"; param_tangent: dict of (N,) float32 tensors keyed
        like scene.sph; warm / warm_tangent / next_warm_tangent: DFSPH pairs of (N,) float32.
        synchronize=False leaves the launches queued on the harness's stream (inputs must be ready)."""
        lib = _load_sph()
        if getattr(self, "_zero_tangent", None) is None or self._zero_tangent.numel() != self.n:
            self._zero_tangent = torch.zeros(self.n, dtype=torch.float32, device=self.device)
        z = self._zero_tangent
        sin = RefStateIn(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]))
        tin = RefStateIn(*[_p(tangent[k][a]) for k in ("positions", "velocities") for a in range(3)])
        tout = RefStateOut(*[_p(next_tangent[k][a]) for k in ("positions", "velocities") for a in range(3)])
        vp = ctypes.c_void_p
        ct = (vp * 3)(*[control_tangent[a].data_ptr() for a in range(3)])
        get = lambda k: param_tangent.get(k, z)
        pt = (vp * 4)(*[get(k).data_ptr() for k in ("masses", "rest_densities", "viscosities", "surface_tensions")])
        mt = (vp * 3)(*[get(k).data_ptr() for k in self._method_names()])
        wt = (vp * 2)(*[(warm_tangent[a] if warm_tangent is not None else z).data_ptr() for a in range(2)])
        nwt = (vp * 2)(*[(next_warm_tangent[a] if next_warm_tangent is not None else z).data_ptr() for a in range(2)])
        w = [vp(t.data_ptr()) if t is not None else None for t in (warm if warm is not None else (None, None))]
        params = self._pstruct()
        if synchronize:
            torch.cuda.synchronize(self.device)
        self._keep_tangent = (sin, tin, tout, ct, pt, mt, wt, nwt, w, params)
        rc = lib.ref_sph_jvp_step(self.handle, ctypes.byref(sin), ctypes.byref(params), ctypes.byref(tin), ct, pt, mt, wt,
                                  ctypes.byref(tout), nwt, step_index, w[0], w[1])
        if rc:
            raise RuntimeError(f"ref_sph_jvp_step failed: {rc}")
        if synchronize:
            load().ref_synchronize(self.base.handle)

    def vjp_step(self, x, v, next_adjoint, previous_adjoint, control_adjoint, param_adjoint, step_index, next_warm=None,
                 previous_warm=None):
        """SPH<Method>::vjp_step after forward_step of (x, v).  Adjoints are float64 CUDA tensors:
        next_adjoint / previous_adjoint dicts of (3, N) "positions" / "velocities"; control_adjoint
        (3, N); param_adjoint dict of (N,) keyed like scene.sph; next_warm / previous_warm: DFSPH
        pairs of (N,).  Outputs are accumulated (previous_warm is overwritten, as the reference does)."""
        lib = _load_sph()
        zd = lambda: torch.zeros(self.n, dtype=torch.float64, device=self.device)
        vp = ctypes.c_void_p
        sin = RefStateIn(_p(x[0]), _p(x[1]), _p(x[2]), _p(v[0]), _p(v[1]), _p(v[2]))
        na = (vp * 6)(*[next_adjoint[k][a].data_ptr() for k in ("positions", "velocities") for a in range(3)])
        pa = (vp * 6)(*[previous_adjoint[k][a].data_ptr() for k in ("positions", "velocities") for a in range(3)])
        ca = (vp * 3)(*[control_adjoint[a].data_ptr() for a in range(3)])
        keep = []

        def slot(d, k):
            if k in d:
                return d[k].data_ptr()
            t = zd()
            keep.append(t)
            return t.data_ptr()
        qa = (vp * 4)(*[slot(param_adjoint, k) for k in ("masses", "rest_densities", "viscosities", "surface_tensions")])
        names = list(SPH_METHOD_PARAMETERS[self.method])
        ma_ptrs = [slot(param_adjoint, k) for k in names]
        while len(ma_ptrs) < 3:
            t = zd()
            keep.append(t)
            ma_ptrs.append(t.data_ptr())
        ma = (vp * 3)(*ma_ptrs)
        nw = next_warm if next_warm is not None else (zd(), zd())
        pw = previous_warm if previous_warm is not None else (zd(), zd())
        keep.extend([nw, pw])
        nwp = (vp * 2)(nw[0].data_ptr(), nw[1].data_ptr())
        pwp = (vp * 2)(pw[0].data_ptr(), pw[1].data_ptr())
        params = self._pstruct()
        torch.cuda.synchronize(self.device)
        rc = lib.ref_sph_vjp_step(self.handle, ctypes.byref(sin), ctypes.byref(params), na, nwp, pa, ca, qa, ma, pwp, step_index)
        if rc:
            raise RuntimeError(f"ref_sph_vjp_step failed: {rc}")
        load().ref_synchronize(self.base.handle)

    def read(self, field: str) -> torch.Tensor:
        code = SPH_FIELDS[field]
        scalar = code in (0, 1, 5)
        out = torch.zeros((self.n,) if scalar else (3, self.n), dtype=torch.float32, device=self.device)
        torch.cuda.synchronize(self.device)
        ptrs = (out.data_ptr(), None, None) if scalar else (out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr())
        rc = _load_sph().ref_sph_read(self.handle, code, *[ctypes.c_void_p(p) if p else None for p in ptrs])
        if rc:
            raise RuntimeError(f"ref_sph_read failed: {rc}")
        return out
