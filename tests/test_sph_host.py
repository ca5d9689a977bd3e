"""CPU tests of the SPH front end: the C entry points reject invalid configurations before any
device work."""
import ctypes

import numpy as np
import pytest

from physica_b200 import pbf, scenes, sph


def _create(cuda_lib, configuration, mode=0, **domain):
    lib = sph.library()
    sc = scenes.sph_dam_break((4, 4, 4), (0.0, 0.0, 0.0), (1.0, 2.0, 1.0), 1)
    dc = pbf.DomainConfiguration.from_scene(sc)
    for k, v in domain.items():
        setattr(dc, k, v)
    c = dc.to_c()
    h = ctypes.c_void_p()
    rc = lib.sph_create(ctypes.byref(c), ctypes.byref(configuration.to_c()), mode, None, ctypes.byref(h))
    return rc, h


def test_create_rejects_unknown_mode(cuda_lib):
    rc, h = _create(cuda_lib, sph.Configuration(), mode=7)
    assert rc == 1 and not h.value


@pytest.mark.parametrize("field,value", [("time_step", 0.0), ("support_radius", float("nan"))])
def test_create_rejects_invalid_domain(cuda_lib, field, value):
    rc, h = _create(cuda_lib, sph.Configuration(), **{field: value})
    assert rc == 1 and not h.value


def test_create_rejects_invalid_configuration(cuda_lib):
    assert _create(cuda_lib, sph.Configuration(checkpoint_interval=0))[0] == 1
    assert _create(cuda_lib, sph.Configuration(pressure_iterations=65))[0] == 7
    bad = sph.Configuration()
    c = bad.to_c()
    c.method = 9
    lib = sph.library()
    dc = pbf.DomainConfiguration.from_scene(scenes.sph_dam_break((4, 4, 4), (0, 0, 0), (1, 2, 1), 1)).to_c()
    h = ctypes.c_void_p()
    assert lib.sph_create(ctypes.byref(dc), ctypes.byref(c), 0, None, ctypes.byref(h)) == 1


def test_null_arguments(cuda_lib):
    lib = sph.library()
    h = ctypes.c_void_p()
    assert lib.sph_create(None, None, 0, None, ctypes.byref(h)) == 1
    assert lib.sph_forward_step(None, None, None, None, None, None, None, None) == 1
    assert lib.sph_destroy(None) == 0
