"""The C++ front ends (include/physica_pbf.hpp and include/physica_sph.hpp), which mirror the
reference's PBF class (pbf/pbf.ixx:14-141) and SPH<Method> (sph/sph.ixx:273-372): they compile with
g++ against the library, and on a GPU programs written against them (tests/cpp/*_roundtrip.cpp) give
the same substeps, tangents and adjoints, bit for bit, as the same calls made through the Python
binding."""
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
SOURCE = ROOT / "tests" / "cpp" / "pbf_cpp_roundtrip.cpp"
BUILD = ROOT / "tests" / "cpp" / "_build"
PROGRAM = BUILD / "pbf_cpp_roundtrip"
LIBDIR = ROOT / "physica_b200" / "lib"
CUDA = pathlib.Path("/usr/local/cuda")


def build_program() -> pathlib.Path:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    if not (LIBDIR / "libphysica_pbf.so").exists():
        pytest.skip("libphysica_pbf.so not built")
    BUILD.mkdir(parents=True, exist_ok=True)
    deps = [SOURCE, ROOT / "include" / "physica_pbf.hpp", ROOT / "include" / "physica_pbf.h", LIBDIR / "libphysica_pbf.so"]
    if PROGRAM.exists() and all(PROGRAM.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return PROGRAM
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}",
           str(SOURCE), "-o", str(PROGRAM), f"-L{LIBDIR}", "-lphysica_pbf", f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return PROGRAM


def test_cpp_front_end_compiles_and_links():
    assert build_program().exists()


@pytest.mark.gpu
@pytest.mark.parametrize("recompute", [0, 1])
def test_cpp_front_end_matches_python_binding(tmp_path, cuda_lib, recompute):
    """recompute 1: the C++ solver keeps every second iterate only and recomputes the rest for the
    tangent and the adjoint; the Python solver keeps them all.  The results are the same bits."""
    import torch
    from physica_b200 import pbf, scenes

    program = build_program()
    sc = scenes.dam_break((10, 10, 10), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), 61, 3, velocity_sigma=0.2)
    sc.controls[:] = 0.0
    steps = 4
    n = sc.count
    params = sc.parameter_arrays()
    names = ("masses", "rest_densities", "viscosities", "surface_tensions", "relaxation", "artificial_pressure_strength",
             "artificial_pressure_exponent", "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([n, sc.pressure_iterations, steps, recompute], dtype=np.uint32).tofile(f)
        np.array([sc.time_step, sc.support_radius, sc.particle_radius, *sc.gravity, *sc.box_min, *sc.box_max,
                  *sc.box_velocity], dtype=np.float32).tofile(f)
        np.array([1 if sc.no_slip else 0], dtype=np.uint32).tofile(f)
        sc.positions.astype(np.float32).tofile(f)
        sc.velocities.astype(np.float32).tofile(f)
        for name in names:
            params.get(name, np.zeros(n, np.float32)).astype(np.float32).tofile(f)
    r = subprocess.run([str(program), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    f32 = np.frombuffer(raw[:9 * n * 4], dtype=np.float32)
    f64 = np.frombuffer(raw[9 * n * 4:], dtype=np.float64)
    assert f64.size == 7 * n
    cpp_x, cpp_v, cpp_t = f32[:3 * n].reshape(3, n), f32[3 * n:6 * n].reshape(3, n), f32[6 * n:].reshape(3, n)
    cpp_ax, cpp_av, cpp_am = f64[:3 * n].reshape(3, n), f64[3 * n:6 * n].reshape(3, n), f64[6 * n:]

    solver, state, control, prm = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    cur, nxt = state, solver.allocate_state()
    for _ in range(steps - 1):
        solver.forward_step(cur, control, prm, nxt, cache)
        cur, nxt = nxt, cur
    last = solver.allocate_state()
    solver.copy_state(cur, last)
    solver.forward_step(last, control, prm, nxt, cache)
    st, nt = solver.allocate_state_tangent(), solver.allocate_state_tangent()
    st.positions.fill_(1.0)
    solver.jvp_step(last, control, prm, nxt, cache, st, solver.allocate_control(), solver.allocate_parameter_tangent(), nt)
    na, pa = solver.allocate_state_adjoint(), solver.allocate_state_adjoint()
    na.positions.fill_(1.0)
    qa = solver.allocate_parameter_adjoint()
    solver.vjp_step(last, control, prm, nxt, cache, na, pa, solver.allocate_control_adjoint(), qa)
    torch.cuda.synchronize()

    assert np.array_equal(cpp_x.view(np.int32), nxt.positions.cpu().numpy().view(np.int32))
    assert np.array_equal(cpp_v.view(np.int32), nxt.velocities.cpu().numpy().view(np.int32))
    assert np.array_equal(cpp_t.view(np.int32), nt.positions.cpu().numpy().view(np.int32))
    assert np.array_equal(cpp_ax, pa.positions.cpu().numpy())
    assert np.array_equal(cpp_av, pa.velocities.cpu().numpy())
    assert np.array_equal(cpp_am, qa.tensors["masses"].cpu().numpy())
    assert np.isfinite(cpp_ax).all() and np.abs(cpp_ax).max() > 0


# ------------------------------------------------------------------------- SPH<Method>
SPH_SOURCE = ROOT / "tests" / "cpp" / "sph_cpp_roundtrip.cpp"
SPH_PROGRAM = BUILD / "sph_cpp_roundtrip"


def build_sph_program() -> pathlib.Path:
    build_program()   # the same checks
    deps = [SPH_SOURCE, ROOT / "include" / "physica_sph.hpp", ROOT / "include" / "physica_sph.h",
            ROOT / "include" / "physica_pbf.hpp", LIBDIR / "libphysica_pbf.so"]
    if SPH_PROGRAM.exists() and all(SPH_PROGRAM.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return SPH_PROGRAM
    cmd = [shutil.which("g++"), "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
           f"-I{CUDA / 'include'}", str(SPH_SOURCE), "-o", str(SPH_PROGRAM), f"-L{LIBDIR}", "-lphysica_pbf",
           f"-L{CUDA / 'lib64'}", "-lcudart", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return SPH_PROGRAM


def test_sph_cpp_front_end_compiles_and_links():
    assert build_sph_program().exists()


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["wcsph", "pcisph", "iisph", "dfsph"])
def test_sph_cpp_front_end_matches_python_binding(method, tmp_path, cuda_lib):
    import torch
    from physica_b200 import pbf, scenes, sph

    program = build_sph_program()
    sc = scenes.sph_dam_break((8, 8, 8), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), 71, method=method, velocity_sigma=0.2)
    sc.controls[:] = 0.0
    n, steps = sc.count, 3
    iterations = (3, 2, 3)
    rng = np.random.default_rng(19)
    warm = [rng.uniform(0, 50, n).astype(np.float32) for _ in range(2)]
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([int(sph.Method[method]), n, steps, *iterations], dtype=np.uint32).tofile(f)
        np.array([sc.time_step, sc.support_radius, sc.particle_radius, *sc.gravity, *sc.box_min, *sc.box_max,
                  *sc.box_velocity], dtype=np.float32).tofile(f)
        np.array([1 if sc.no_slip else 0], dtype=np.uint32).tofile(f)
        sc.positions.astype(np.float32).tofile(f)
        sc.velocities.astype(np.float32).tofile(f)
        for name in sph.PARAMETER_NAMES:
            np.asarray(sc.sph.get(name, np.zeros(n, np.float32)), dtype=np.float32).tofile(f)
        for w in warm:
            w.tofile(f)
    r = subprocess.run([str(program), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    f32 = np.frombuffer(raw[:9 * n * 4], dtype=np.float32)
    f64 = np.frombuffer(raw[9 * n * 4:], dtype=np.float64)
    assert f64.size == 7 * n

    cfg = sph.Configuration(method=sph.Method[method], pressure_iterations=iterations[0], divergence_iterations=iterations[1],
                            density_iterations=iterations[2])
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[method], configuration=cfg,
                                                          mode=pbf.ExecutionMode.differentiable)
    if method == "dfsph":
        state.warm_divergence_pressure.copy_(torch.from_numpy(warm[0]))
        state.warm_density_pressure.copy_(torch.from_numpy(warm[1]))
    cache = solver.allocate_step_cache()
    cur, nxt = state, solver.allocate_state()
    for _ in range(steps - 1):
        solver.forward_step(cur, control, params, nxt, cache)
        cur, nxt = nxt, cur
    last = solver.allocate_state()
    solver.copy_state(cur, last)
    solver.forward_step(last, control, params, nxt, cache)
    st, nt = solver.allocate_state_tangent(), solver.allocate_state_tangent()
    st.positions.fill_(1.0)
    solver.jvp_step(last, control, params, nxt, cache, st, solver.allocate_control(), solver.allocate_parameter_tangent(), nt)
    na, pa = solver.allocate_state_adjoint(), solver.allocate_state_adjoint()
    na.positions.fill_(1.0)
    qa = solver.allocate_parameter_adjoint()
    solver.vjp_step(last, control, params, nxt, cache, na, pa, solver.allocate_control_adjoint(), qa)
    torch.cuda.synchronize()

    assert np.array_equal(f32[:3 * n].view(np.int32), nxt.positions.cpu().numpy().reshape(-1).view(np.int32))
    assert np.array_equal(f32[3 * n:6 * n].view(np.int32), nxt.velocities.cpu().numpy().reshape(-1).view(np.int32))
    assert np.array_equal(f32[6 * n:].view(np.int32), nt.positions.cpu().numpy().reshape(-1).view(np.int32))
    assert np.array_equal(f64[:3 * n], pa.positions.cpu().numpy().reshape(-1))
    assert np.array_equal(f64[3 * n:6 * n], pa.velocities.cpu().numpy().reshape(-1))
    assert np.array_equal(f64[6 * n:], qa.tensors["masses"].cpu().numpy())
    assert np.isfinite(f64).all() and np.abs(f64[:3 * n]).max() > 0
