"""CPU checks of the C ABI: the library builds, loads, and exports every symbol that
include/cellgpu_b200.h declares (no compute calls: there is no GPU here)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", f)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(cg_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(cglib):
    missing = [n for n in sorted(declared_functions()) if not hasattr(cglib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_declarations(cglib):
    from cellgpu_b200 import _lib
    assert set(_lib.SIGNATURES) <= declared_functions()


def test_version(cglib):
    assert cglib.cg_version() >= 100


def test_error_string_roundtrip(cglib):
    import ctypes as C
    h = C.c_void_p()
    # invalid arguments are rejected on the host before any CUDA call
    rc = cglib.cg_voronoi_create(0, None, None, 16, 0, C.byref(h))
    assert rc == -2
    assert b"bad" in cglib.cg_last_error_string()


def test_restore_rejects_a_foreign_buffer():
    """cg_restore validates the snapshot header before touching the device."""
    import ctypes as C
    from cellgpu_b200._lib import CG_ERR_ARG, load
    lib = load()
    junk = C.create_string_buffer(b"definitely not a snapshot" * 8)
    h = C.c_void_p()
    assert lib.cg_restore(junk, len(junk.raw), C.byref(h)) == CG_ERR_ARG
    assert b"snapshot" in lib.cg_last_error_string()


def test_strided_buffers_are_refused():
    """The library reads every buffer row-major: a strided numpy view or torch tensor (a transpose,
    an index along the second axis) is refused instead of being read in the wrong order, and noise
    tensors must be float64 CUDA tensors of the right size."""
    import numpy as np
    import pytest
    import torch

    from cellgpu_b200._lib import device_noise, ptr
    a = np.zeros((6, 4))
    assert ptr(a) is not None and ptr(None) is None
    with pytest.raises(ValueError):
        ptr(a[:, ::2])
    with pytest.raises(ValueError):
        ptr(a[:, [0, 2, 1]])  # numpy lays an index along axis 1 out column-major
    t = torch.zeros(6, 4, dtype=torch.float64)
    assert ptr(t) is not None
    with pytest.raises(ValueError):
        ptr(t.t())
    assert device_noise(None, 10) is None
    with pytest.raises(ValueError):
        device_noise(t, 24)  # host tensor
