"""Generate the golden fixtures of tests/golden/ by running the reference's own CUDA PBF.

The reference kernels are compiled from the reference sources into oracle/_ref/libpbf_ref.so
(oracle/build.py) and replayed by oracle/ref_harness.cu.  This script needs a CUDA device; run

    python tests/golden/make_golden.py [output_dir]

and copy the .npz files into tests/golden/.  The fixtures are small seeded scenes; the same
seeds regenerate the inputs byte for byte (physica_b200/scenes.py).
"""
from __future__ import annotations

import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from oracle import reference  # noqa: E402
from physica_b200 import scenes  # noqa: E402

STEP = dict(lattice=(12, 12, 12), box_min=(0.0, 0.0, 0.0), box_max=(1.0, 2.0, 1.0), seed=11, iterations=4)
VJP = dict(lattice=(8, 8, 8), box_min=(0.0, 0.0, 0.0), box_max=(1.0, 2.0, 1.0), seed=12, iterations=4, velocity_sigma=0.1)
TRAJ_STEPS = 10


def _scene(spec):
    kw = dict(spec)
    sigma = kw.pop("velocity_sigma", 0.0)
    return scenes.dam_break(kw["lattice"], kw["box_min"], kw["box_max"], kw["seed"], kw["iterations"],
                            velocity_sigma=sigma)


def make_step(out_dir: pathlib.Path):
    sc = _scene(STEP)
    ref = reference.ReferencePBF(sc)
    dev = "cuda"
    x = torch.from_numpy(sc.positions).to(dev).contiguous()
    v = torch.from_numpy(sc.velocities).to(dev).contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    ref.forward_step(x, v, xo, vo, 0)
    fields = {k: ref.read(k).cpu().numpy() for k in ("sorted_keys", "sorted_indices", "cell_offsets", "predicted",
                                                     "first_densities", "first_lambdas", "corrected", "vorticities",
                                                     "normals", "confined")}
    x1, v1 = xo.cpu().numpy(), vo.cpu().numpy()
    # a short trajectory
    xa, va, xb, vb = x.clone(), v.clone(), torch.zeros_like(x), torch.zeros_like(v)
    for k in range(TRAJ_STEPS):
        ref.forward_step(xa, va, xb, vb, k)
        xa, xb, va, vb = xb, xa, vb, va
    np.savez_compressed(out_dir / "reference_step_small.npz", x0=sc.positions, v0=sc.velocities, x1=x1, v1=v1,
                        x10=xa.cpu().numpy(), v10=va.cpu().numpy(), **fields,
                        **{k: np.asarray(v) for k, v in STEP.items()})


def make_vjp(out_dir: pathlib.Path):
    sc = _scene(VJP)
    dev = "cuda"
    ref = reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True)
    x = torch.from_numpy(sc.positions).to(dev).contiguous()
    v = torch.from_numpy(sc.velocities).to(dev).contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    ref.forward_step(x, v, xo, vo, 0)
    rng = np.random.default_rng(99)
    nxa = rng.normal(size=(3, sc.count))
    nva = rng.normal(size=(3, sc.count))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    z3 = lambda: torch.zeros((3, sc.count), dtype=torch.float64, device=dev)
    nxt = {"positions": d(nxa), "velocities": d(nva)}
    prev = {"positions": z3(), "velocities": z3()}
    ctrl = z3()
    names = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
             "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")
    padj = {k: torch.zeros(sc.count, dtype=torch.float64, device=dev) for k in names}
    ref.vjp_step(x, v, nxt, prev, ctrl, padj)
    np.savez_compressed(out_dir / "reference_vjp_small.npz", x0=sc.positions, v0=sc.velocities, x1=xo.cpu().numpy(),
                        v1=vo.cpu().numpy(), next_position_adjoint=nxa, next_velocity_adjoint=nva,
                        adj_position=prev["positions"].cpu().numpy(), adj_velocity=prev["velocities"].cpu().numpy(),
                        adj_control=ctrl.cpu().numpy(), **{f"adj_{k}": padj[k].cpu().numpy() for k in names},
                        **{k: np.asarray(v) for k, v in VJP.items()})


if __name__ == "__main__":
    out = pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else pathlib.Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    make_step(out)
    make_vjp(out)
    print("wrote", sorted(p.name for p in out.glob("*.npz")))
