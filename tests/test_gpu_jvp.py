"""GPU tests of the forward-mode tangent (pbf_jvp_step, PBF::jvp_step pbf/pbf.cpp:193-215): against
the reference's own jvp_step kernels, against this library's FP64 adjoint through the identity
<J u, w> = <u, J^T w>, and against central differences of the FP64 oracle.  Tangents are FP32 like
the reference's, so the bars are relative (max-norm) FP32 tolerances written in each test."""
import numpy as np
import pytest
import torch

from physica_b200 import pbf, scenes

pytestmark = pytest.mark.gpu

NAMES = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
         "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")


@pytest.fixture(scope="module", autouse=True)
def _cuda(cuda_lib):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def _scene(lattice=(10, 10, 10), seed=41):
    return scenes.dam_break(lattice, (0, 0, 0), (1, 2, 1), seed, 4, velocity_sigma=0.1)


def _tangents(sc, seed, with_parameters=True):
    """Random tangents scaled to each input's magnitude (positions, velocities, controls, parameters)."""
    rng = np.random.default_rng(seed)
    n = sc.count
    t = {"positions": (rng.normal(size=(3, n)) * 1e-3).astype(np.float32),
         "velocities": (rng.normal(size=(3, n)) * 1e-2).astype(np.float32),
         "control": rng.normal(size=(3, n)).astype(np.float32)}
    scale = {"masses": 1e-5, "rest_densities": 1.0, "relaxation": 10.0, "artificial_pressure_strength": 1e-3,
             "artificial_pressure_exponent": 0.0, "artificial_pressure_radius": 0.0, "xsph_viscosity": 1e-8,
             "vorticity_confinement": 1e-10}
    pt = {k: ((rng.normal(size=n) * scale[k]) if with_parameters else np.zeros(n)).astype(np.float32) for k in NAMES}
    return t, pt


def my_jvp(sc, t, pt, solver=None):
    if solver is None:
        solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    else:
        solver, state, control, params = solver
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    st = pbf.StateTangent(torch.from_numpy(t["positions"]).cuda(), torch.from_numpy(t["velocities"]).cuda())
    ct = pbf.Control(torch.from_numpy(t["control"]).cuda())
    ptt = solver.allocate_parameter_tangent()
    for k in NAMES:
        ptt.tensors[k].copy_(torch.from_numpy(pt[k]))
    out = solver.allocate_state_tangent()
    solver.jvp_step(state, control, params, nxt, cache, st, ct, ptt, out)
    torch.cuda.synchronize()
    return out.positions.cpu().numpy(), out.velocities.cpu().numpy()


def test_jvp_matches_reference_jvp():
    """Tangents equal the reference's jvp_step kernels to FP32 rounding (max-norm relative 1e-4)."""
    from oracle import reference
    if not reference.available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    sc = _scene()
    t, pt = _tangents(sc, 1)
    mx, mv = my_jvp(sc, t, pt)
    ref = reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    ref.forward_step(x, v, xo, vo, 0)
    tin = {"positions": torch.from_numpy(t["positions"]).cuda(), "velocities": torch.from_numpy(t["velocities"]).cuda()}
    tout = {"positions": torch.zeros_like(x), "velocities": torch.zeros_like(v)}
    ctl = torch.from_numpy(t["control"]).cuda()
    ptd = {k: torch.from_numpy(pt[k]).cuda() for k in NAMES}
    ref.jvp_step(x, v, tin, ctl, ptd, tout)
    rx, rv = tout["positions"].cpu().numpy(), tout["velocities"].cpu().numpy()
    assert rel(mx, rx) < 1e-4, rel(mx, rx)
    assert rel(mv, rv) < 1e-4, rel(mv, rv)


def test_jvp_and_vjp_satisfy_the_adjoint_identity():
    """<J u, w> from the FP32 tangent equals <u, J^T w> from the FP64 adjoint (relative 1e-4)."""
    sc = _scene((9, 9, 9), 42)
    t, pt = _tangents(sc, 2)
    handles = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    solver, state, control, params = handles
    mx, mv = my_jvp(sc, t, pt, handles)
    rng = np.random.default_rng(3)
    wx, wv = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    na = pbf.StateAdjoint(torch.from_numpy(wx).cuda(), torch.from_numpy(wv).cuda())
    pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
    solver.vjp_step(state, control, params, nxt, cache, na, pa, ca, qa)
    torch.cuda.synchronize()
    lhs = float((wx * mx).sum() + (wv * mv).sum())
    rhs = float((pa.positions.cpu().numpy() * t["positions"]).sum() + (pa.velocities.cpu().numpy() * t["velocities"]).sum()
                + (ca.external_accelerations.cpu().numpy() * t["control"]).sum()
                + sum((qa.tensors[k].cpu().numpy() * pt[k]).sum() for k in NAMES))
    assert lhs == pytest.approx(rhs, rel=1e-4)


def test_jvp_matches_central_differences_of_the_fp64_oracle():
    """<J u, w> against the central difference of w . f(x + eps u) in FP64 (relative 1e-3)."""
    from oracle import oracle
    sc = _scene((8, 8, 8), 43)
    t, pt = _tangents(sc, 4, with_parameters=False)
    mx, mv = my_jvp(sc, t, pt)
    rng = np.random.default_rng(5)
    wx, wv = rng.normal(size=(3, sc.count)), rng.normal(size=(3, sc.count))
    x0, v0 = sc.positions.astype(np.float64), sc.velocities.astype(np.float64)
    a0 = sc.controls.astype(np.float64)

    def loss(e):
        x1, v1 = oracle.forward_step(sc, x0 + e * t["positions"], v0 + e * t["velocities"], a0 + e * t["control"])
        return float((wx * x1).sum() + (wv * v1).sum())

    eps = 1e-4
    fd = (loss(eps) - loss(-eps)) / (2 * eps)
    ad = float((wx * mx).sum() + (wv * mv).sum())
    assert ad == pytest.approx(fd, rel=1e-3)


def test_batched_jvp_equals_per_scene_jvp():
    scs = [scenes.batched_scene(c, 300 + k, 3, velocity_sigma=0.1) for k, c in enumerate((1200, 2500, 64))]
    batch, state, control, params = pbf.batch_for_scenes(scs, mode=pbf.ExecutionMode.differentiable)
    tangents = [_tangents(sc, 10 + k) for k, sc in enumerate(scs)]
    cat = lambda key: torch.from_numpy(np.concatenate([t[key] for t, _ in tangents], axis=-1)).cuda().contiguous()
    st = pbf.StateTangent(cat("positions"), cat("velocities"))
    ct = pbf.Control(cat("control"))
    ptt = pbf.Parameters({k: torch.from_numpy(np.concatenate([p[k] for _, p in tangents])).cuda() for k in NAMES})
    nxt = batch.allocate_state()
    batch.forward_step(state, control, params, nxt, 0)
    out = batch.allocate_state_tangent()
    batch.jvp_step(state, control, params, nxt, 0, st, ct, ptt, out)
    torch.cuda.synchronize()
    for s, sc in enumerate(scs):
        mx, mv = my_jvp(sc, *tangents[s])
        sl = batch.particle_range(s)
        assert np.array_equal(out.positions[:, sl].cpu().numpy(), mx), s
        assert np.array_equal(out.velocities[:, sl].cpu().numpy(), mv), s


def test_jvp_needs_a_differentiable_solver():
    sc = _scene((4, 4, 4), 44)
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    solver.forward_step(state, control, params, nxt, cache)
    st = solver.allocate_state_tangent()
    with pytest.raises(pbf.PBFError):
        solver.jvp_step(state, control, params, nxt, cache, st, solver.allocate_control(),
                        solver.allocate_parameter_tangent(), solver.allocate_state_tangent())


def test_copy_state_tangent_copies_all_six_fields():
    """PBF::copy_state_tangent (pbf/pbf.cpp:163): positions and velocities, bit for bit."""
    sc = _scene((5, 5, 5), 45)
    solver, _, _, _ = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    src, dst = solver.allocate_state_tangent(), solver.allocate_state_tangent()
    g = torch.Generator(device="cuda").manual_seed(7)
    src.positions.copy_(torch.randn(src.positions.shape, generator=g, device="cuda"))
    src.velocities.copy_(torch.randn(src.velocities.shape, generator=g, device="cuda"))
    solver.copy_state_tangent(src, dst)
    torch.cuda.synchronize()
    assert torch.equal(dst.positions, src.positions) and torch.equal(dst.velocities, src.velocities)
