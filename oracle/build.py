"""Build recipe for the oracle -- TEST INFRASTRUCTURE ONLY.

* oracle/lib/libpbf_oracle.so : the FP64 host restatement (gcc + OpenMP).
* oracle/_ref/libpbf_ref.so   : the reference's own CUDA PBF and SPH kernels, compiled from
  the reference sources (pbf/pbf.cu, density/density.cu, neighborhood/neighborhood.cu,
  domain/domain.cu, sph/{common,wcsph,pcisph,iisph,dfsph}.cu of fluids/liquid/particle) with
  nvcc for sm_100a, plus oracle/ref_harness.cu, which replays PBF::forward_step /
  PBF::vjp_step (pbf/pbf.cpp:167-258) and SPH<Method>::forward_step (sph/sph.ixx:337-341)
  over the reference's own launch_* functions.  The
  reference's C++23 module host layer (import std) cannot be compiled by this
  toolchain, so the harness stands in for it.  Built only where the reference
  tree exists ($PHYSICA_REFERENCE, or a checkout named `reference` beside this repository's
  directory); the .so then travels with the repository copy.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent


def reference_root() -> pathlib.Path:
    """The reference checkout: $PHYSICA_REFERENCE, else a checkout named `reference` beside this
    repository's directory."""
    env = os.environ.get("PHYSICA_REFERENCE")
    return pathlib.Path(env) if env else HERE.parent.parent / "reference"


def particle_root() -> pathlib.Path:
    return reference_root() / "fluids" / "liquid" / "particle"

REF_SOURCES = ["pbf/pbf.cu", "density/density.cu", "neighborhood/neighborhood.cu", "domain/domain.cu",
               "sph/common.cu", "sph/wcsph.cu", "sph/pcisph.cu", "sph/iisph.cu", "sph/dfsph.cu"]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def _cccl_root() -> pathlib.Path | None:
    try:
        import flashinfer  # noqa: F401,PLC0415
    except Exception:  # pragma: no cover - optional
        pass
    for base in sys.path:
        cand = pathlib.Path(base) / "flashinfer" / "data" / "cccl"
        if (cand / "libcudacxx" / "include" / "cuda" / "buffer").exists():
            return cand
    return None


def _run(cmd):
    subprocess.run(cmd, check=True)


def build_oracle(force: bool = False) -> pathlib.Path:
    out = HERE / "lib" / "libpbf_oracle.so"
    src = HERE / "pbf_oracle.c"
    if not force and out.exists() and out.stat().st_mtime >= max(src.stat().st_mtime, (HERE / "pbf_oracle.h").stat().st_mtime):
        return out
    out.parent.mkdir(exist_ok=True)
    tmp = out.with_suffix(f".so.tmp{os.getpid()}")
    _run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-std=c11", "-Wall",
          "-o", str(tmp), str(src), "-lm"])
    os.replace(tmp, out)
    return out


def reference_available() -> bool:
    particle = particle_root()
    return all((particle / s).exists() for s in REF_SOURCES) and _cccl_root() is not None


def build_reference(force: bool = False) -> pathlib.Path | None:
    """Compile the reference kernels + replay harness into oracle/_ref/libpbf_ref.so."""
    out = HERE / "_ref" / "libpbf_ref.so"
    harness = HERE / "ref_harness.cu"
    if not reference_available():
        return out if out.exists() else None
    if not force and out.exists() and out.stat().st_mtime >= harness.stat().st_mtime:
        return out
    particle = particle_root()
    cccl = _cccl_root()
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    objdir = HERE / "_ref" / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    inc = [f"-I{cccl / 'libcudacxx' / 'include'}", f"-I{cccl / 'cub'}", f"-I{cccl / 'thrust'}"]
    # Flags of the reference build (CMakeLists.txt:22-27): C++20 CUDA, default fmad/prec-div/prec-sqrt.
    common = [nvcc, "-std=c++20", ARCH, "-O3", "-Xcompiler", "-fPIC", *inc]
    objs = []
    procs = []
    for rel in REF_SOURCES:
        obj = objdir / (rel.replace("/", "_") + ".o")
        procs.append(subprocess.Popen([*common, "-c", str(particle / rel), "-o", str(obj)]))
        objs.append(obj)
    hobj = objdir / "ref_harness.o"
    procs.append(subprocess.Popen([*common, f"-I{particle}", "-c", str(harness), "-o", str(hobj)]))
    objs.append(hobj)
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("reference build failed")
    tmp = out.with_suffix(f".so.tmp{os.getpid()}")
    _run([nvcc, ARCH, "-shared", "-o", str(tmp), *map(str, objs)])
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference(force="--force" in sys.argv))
