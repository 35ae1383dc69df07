"""ctypes binding of the C ABI declared in ``include/cellgpu_b200.h``.

The library is the in-tree ``cellgpu_b200/libcellgpu_b200.so`` (built by ``cellgpu_b200.build``).
There is no fallback: if the library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcellgpu_b200.so")

CG_OK = 0
CG_ERR_CUDA = -1
CG_ERR_ARG = -2
CG_ERR_CAPACITY = -3
CG_ERR_TOPOLOGY = -4
CG_ERR_TIMEOUT = -5
CG_ERR_STATE = -6
CG_FP64 = 0
CG_MIXED = 1

_vp = C.c_void_p
_i = C.c_int
_d = C.c_double
_u64 = C.c_uint64
_u32 = C.c_uint32
_sz = C.c_size_t

# name -> (restype, argtypes); every symbol here is declared in include/cellgpu_b200.h
SIGNATURES = {
    "cg_last_error_string": (C.c_char_p, []),
    "cg_version": (_i, []),
    "cg_voronoi_geometry": (_i, [_vp, _vp, _vp, _i, _i, _d, _d, _vp, _vp]),
    "cg_voronoi_forces": (_i, [_vp, _vp, _vp, _i, _i, _d, _d, _vp, _d, _d, _vp, _vp, _vp]),
    "cg_voronoi_test_triangulation": (_i, [_vp, _vp, _vp, _i, _i, _d, _d, _vp, _vp, _vp]),
    "cg_spp_step": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _d, _d, _d, _d, _u64, _u32, _vp]),
    "cg_voronoi_triangulate": (_i, [_vp, _i, _d, _d, _i, _vp, _vp, _vp]),
    "cg_voronoi_triangulate_noalloc": (_i, [_vp, _i, _d, _d, _i, _vp, _vp, _vp]),
    "cg_voronoi_create": (_i, [_i, _vp, _vp, _i, _i, C.POINTER(_vp)]),
    "cg_destroy": (_i, [_vp]),
    "cg_num_cells": (_i, [_vp]),
    "cg_num_dofs": (_i, [_vp]),
    "cg_num_instances": (_i, [_vp]),
    "cg_neighbor_capacity": (_i, [_vp]),
    "cg_device_bytes": (_sz, [_vp]),
    "cg_voronoi_footprint": (_sz, [_i, _vp, _i]),
    "cg_set_positions": (_i, [_vp, _vp]),
    "cg_get_positions": (_i, [_vp, _vp]),
    "cg_set_cell_preferences": (_i, [_vp, _vp]),
    "cg_set_moduli": (_i, [_vp, _d, _d]),
    "cg_set_motility": (_i, [_vp, _vp]),
    "cg_set_directors": (_i, [_vp, _vp]),
    "cg_get_directors": (_i, [_vp, _vp]),
    "cg_get_forces": (_i, [_vp, _vp]),
    "cg_get_area_perimeter": (_i, [_vp, _vp]),
    "cg_get_topology": (_i, [_vp, _vp, _vp]),
    "cg_set_topology": (_i, [_vp, _vp, _vp]),
    "cg_get_energies": (_i, [_vp, _vp]),
    "cg_set_stream": (_i, [_vp, _vp]),
    "cg_synchronize": (_i, [_vp]),
    "cg_triangulate": (_i, [_vp]),
    "cg_compute_forces": (_i, [_vp]),
    "cg_enforce_topology": (_i, [_vp]),
    "cg_set_seed": (_i, [_vp, _u64]),
    "cg_set_deterministic": (_i, [_vp, _i]),
    "cg_get_deterministic": (_i, [_vp]),
    "cg_set_instance_seeds": (_i, [_vp, _vp]),
    "cg_spp_run": (_i, [_vp, _i, _d, _d, _vp]),
    "cg_counters": (_i, [_vp, C.POINTER(C.c_longlong), _i]),
    "cg_get_stream": (_vp, [_vp]),
    "cg_spp_enqueue": (_i, [_vp, _i, _d, _d]),
    "cg_poll": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), _i]),
    "cg_spp_step_host": (_i, [_vp, _vp, _d, _d, _vp]),
    "cg_spp_enqueue_host": (_i, [_vp, _vp, _d, _d, _vp]),
    "cg_launch_force_pass": (_i, [_vp, _i]),
    "cg_kernels_launched": (C.c_longlong, [_vp]),
    "cg_vertex_create": (_i, [_i, _vp, _vp, _i, _i, C.POINTER(_vp)]),
    "cg_vertex_footprint": (_sz, [_i, _vp, _i]),
    "cg_device_memory": (_i, [_vp, _vp]),
    "cg_snapshot_size": (_sz, [_vp]),
    "cg_snapshot": (_i, [_vp, _vp, _sz]),
    "cg_restore": (_i, [_vp, _sz, _vp]),
    "cg_get_instances": (_i, [_vp, _vp, _vp]),
    "cg_model_kind": (_i, [_vp]),
    "cg_precision": (_i, [_vp]),
    "cg_set_reference_positions": (_i, [_vp]),
    "cg_observables": (_i, [_vp, _d, _vp]),
    "cg_spatial_sort": (_i, [_vp]),
    "cg_autotune": (_i, [_vp, _vp, _vp]),
    "cg_autotune_repair": (_i, [_vp, _i, _d, _d, _vp, _vp]),
    "cg_set_cell_types": (_i, [_vp, _vp]),
    "cg_set_tension": (_i, [_vp, _d]),
    "cg_set_tension_matrix": (_i, [_vp, _i, _vp]),
    "cg_set_exclusions": (_i, [_vp, _vp]),
    "cg_get_external_forces": (_i, [_vp, _vp]),
    "cg_get_tags": (_i, [_vp, _vp]),
    "cg_get_vertex_topology": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cg_set_vertex_topology": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cg_vertex_from_voronoi": (_i, [_vp, _vp]),
    "cg_brownian_run": (_i, [_vp, _i, _d, _d, _d, _vp]),
    "cg_vertex_spp_run": (_i, [_vp, _i, _d, _d, _vp]),
    "cg_set_t1_threshold": (_i, [_vp, _d]),
    "cg_fire_minimize": (_i, [_vp, _vp]),
    "cg_fire_begin": (_i, [_vp, _vp]),
    "cg_fire_advance": (_i, [_vp, _vp, _i, _vp]),
    "cg_fire_begin_instances": (_i, [_vp, _vp, _i, _i]),
    "cg_copy_instances": (_i, [_vp, _i, _vp, _i, _i]),
    "cg_fire_state": (_i, [_vp, _vp, _vp, _vp]),
}

class FireParams(C.Structure):
    """cg_fire_params; defaults of EnergyMinimizerFIRE::initializeParameters
    (src/updaters/EnergyMinimizerFIRE2D.cpp:24-41)."""

    _fields_ = [("dt", _d), ("dt_max", _d), ("dt_min", _d), ("dt_inc", _d), ("dt_dec", _d),
                ("alpha_start", _d), ("alpha_dec", _d), ("force_cutoff", _d), ("n_min", _i),
                ("max_iterations", _i)]

    @classmethod
    def defaults(cls, **kw):
        p = cls(dt=0.01, dt_max=0.1, dt_min=1e-4, dt_inc=1.05, dt_dec=0.95, alpha_start=0.99, alpha_dec=0.9,
                force_cutoff=1e-7, n_min=5, max_iterations=1000)
        for k, v in kw.items():
            setattr(p, k, v)
        if "dt" in kw and "dt_min" not in kw:
            p.dt_min = 0.01 * kw["dt"]  # setDeltaT: deltaTMin = 0.01 dt (EnergyMinimizerFIRE2D.h:42)
        return p


_lib = None


class CellGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cellgpu_b200 error {code}: {msg}")
        self.code = code


def load():
    """Load the in-tree library (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m cellgpu_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(code):
    if code != CG_OK:
        raise CellGPUError(code, load().cg_last_error_string().decode())
    return code


def ptr(a):
    """Device or host pointer of a torch tensor / numpy array (None -> NULL). The library reads
    buffers in row-major order, so a strided view (a transpose, an index along the second axis)
    is refused rather than read in the wrong order."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor is not contiguous (row-major); pass .contiguous()")
        return C.c_void_p(a.data_ptr())
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array is not C-contiguous; pass np.ascontiguousarray(...)")
    return a.ctypes.data_as(C.c_void_p)


def device_noise(noise, count):
    """A caller's noise tensor as the library reads it: float64 on the GPU, at least `count` values,
    row-major (a strided view is copied into order). Work queued on the caller's current stream,
    such as the copy that filled the tensor, is finished first: the library reads it from its own
    stream. None passes through (device noise)."""
    if noise is None:
        return None
    import torch
    if not isinstance(noise, torch.Tensor) or not noise.is_cuda:
        raise ValueError("noise must be a CUDA tensor")
    if noise.dtype != torch.float64:
        raise ValueError("noise must be float64")
    if noise.numel() < count:
        raise ValueError(f"noise holds {noise.numel()} values, {count} needed")
    noise = noise.contiguous()
    torch.cuda.current_stream(noise.device).synchronize()
    return noise
