"""CPU tests of the C ABI library: it loads, exports every declared entry point, and rejects
invalid configurations before touching the device."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s+((?:pbf|sph)_[a-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("pbf_create", "pbf_destroy", "pbf_allocate_step_cache", "pbf_forward_step", "pbf_vjp_step",
                     "pbf_jvp_step", "pbf_batch_create", "pbf_batch_forward_step", "pbf_forward_step_host",
                     "sph_create", "sph_forward_step", "sph_allocate_step_cache", "sph_read_cache"):
        assert required in names


def test_library_exports_every_declared_symbol(cuda_lib):
    lib = cuda_lib.library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version(cuda_lib):
    lib = cuda_lib.library()
    assert lib.pbf_abi_version() == 1
    for status in range(8):
        assert lib.pbf_status_string(status)
    assert lib.pbf_status_string(999) == b"unknown status"


def _domain(cuda_lib, **overrides):
    from physica_b200 import scenes
    dc = cuda_lib.DomainConfiguration.from_scene(scenes.plain_small(lattice=(4, 4, 4)))
    for k, v in overrides.items():
        setattr(dc, k, v)
    return dc


@pytest.mark.parametrize("field,value", [("time_step", -1.0), ("time_step", float("nan")), ("support_radius", 0.0)])
def test_create_rejects_invalid_domain(cuda_lib, field, value):
    lib = cuda_lib.library()
    dc = _domain(cuda_lib, **{field: value}).to_c()
    cc = cuda_lib.ConfigurationC(4, 2)
    h = ctypes.c_void_p()
    assert lib.pbf_create(ctypes.byref(dc), ctypes.byref(cc), 0, None, ctypes.byref(h)) == 1
    assert not h.value
    assert lib.pbf_last_error()


def test_create_rejects_bad_configuration(cuda_lib):
    lib = cuda_lib.library()
    dc = _domain(cuda_lib).to_c()
    h = ctypes.c_void_p()
    assert lib.pbf_create(ctypes.byref(dc), ctypes.byref(cuda_lib.ConfigurationC(4, 0)), 0, None, ctypes.byref(h)) == 1
    assert lib.pbf_create(ctypes.byref(dc), ctypes.byref(cuda_lib.ConfigurationC(1000, 1)), 0, None, ctypes.byref(h)) == 7
    assert lib.pbf_create(ctypes.byref(dc), ctypes.byref(cuda_lib.ConfigurationC(4, 1)), 7, None, ctypes.byref(h)) == 1
    assert lib.pbf_create(None, None, 0, None, ctypes.byref(h)) == 1
    # a degenerate box (max <= min) has no cells
    bad = _domain(cuda_lib)
    bad.boundary.maximum = bad.boundary.minimum
    assert lib.pbf_create(ctypes.byref(bad.to_c()), ctypes.byref(cuda_lib.ConfigurationC(4, 1)), 0, None, ctypes.byref(h)) == 1


def test_null_handles_are_rejected(cuda_lib):
    lib = cuda_lib.library()
    assert lib.pbf_forward_step(None, None, None, None, None, None) == 1
    assert lib.pbf_vjp_step(None, None, None, None, None, None, None, None, None, None) == 1
    assert lib.pbf_destroy(None) == 0
    assert lib.pbf_free_step_cache(None) == 0
    assert lib.pbf_batch_destroy(None) == 0


def test_scenes_are_deterministic():
    from physica_b200 import scenes
    a = scenes.plain_small(lattice=(8, 8, 8))
    b = scenes.plain_small(lattice=(8, 8, 8))
    assert np.array_equal(a.positions, b.positions)
    c = scenes.plain_small(seed=2, lattice=(8, 8, 8))
    assert not np.array_equal(a.positions, c.positions)
    d = scenes.differentiable(lattice=(4, 8, 4))
    assert d.targets is not None and d.targets.shape == (3, 128)
    assert abs(float(d.velocities.std()) - 0.1) < 0.03
    counts = scenes.batched_counts(4, 256, 2048, 65536, True)
    assert min(counts) >= 2048 and max(counts) <= 65536 and len(counts) == 256
    s = scenes.batched_scene(3000, 1, 4)
    assert s.count == 3000


def test_lattice_counts_of_the_workloads():
    from physica_b200 import scenes
    assert scenes.plain_small().count == 32768
    big = scenes.dam_break((128, 64, 128), (0, 0, 0), (4, 4, 4), 2, 8)
    assert big.count == 1048576 and big.grid_dims() == (160, 160, 160)
    assert scenes.plain_small().grid_dims() == (40, 80, 40)
