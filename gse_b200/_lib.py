"""ctypes binding of libgse_b200.so (the C ABI declared in include/gse_b200.h).

The library is loaded from the package directory.  There is no fallback: if
the CUDA library is missing or no B200 is present, calls raise GseError.
"""
from __future__ import annotations

import ctypes
import os
from typing import Any

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgse_b200.so")

GSE_OK = 0
STATUS_NAMES = {
    0: "GSE_OK", 1: "GSE_ERR_INVALID_ARG", 2: "GSE_ERR_STENCIL_TOO_LARGE", 3: "GSE_ERR_CUDA",
    4: "GSE_ERR_OOM", 5: "GSE_ERR_TIMEOUT", 6: "GSE_ERR_NOT_READY", 7: "GSE_ERR_UNSUPPORTED",
    8: "GSE_ERR_NONFINITE", 9: "GSE_ERR_RANGE",
}
PRECISION = {"fp64": 0, "mixed": 1}
PATH_TILED, PATH_GREEN_IN_FFT, PATH_GRAPH = 1, 2, 4
GRID_RHO = 0
GRID_PHI = 1


class GseError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{self.name}: {message}")


class gse_params_t(ctypes.Structure):
    _fields_ = [
        ("size_x", ctypes.c_int), ("size_y", ctypes.c_int), ("size_z", ctypes.c_int),
        ("sigma", ctypes.c_double), ("kappa", ctypes.c_double),
        ("lambda_sigma", ctypes.c_double), ("lambda_sigma1", ctypes.c_double),
        ("box_x", ctypes.c_double), ("box_y", ctypes.c_double), ("box_z", ctypes.c_double),
        ("ccelec", ctypes.c_double), ("precision", ctypes.c_int), ("device", ctypes.c_int),
    ]


class gse_system_t(ctypes.Structure):
    _fields_ = [
        ("size_x", ctypes.c_int), ("size_y", ctypes.c_int), ("size_z", ctypes.c_int),
        ("box_x", ctypes.c_double), ("box_y", ctypes.c_double), ("box_z", ctypes.c_double),
        ("n", ctypes.c_int),
    ]


class gse_batch_info_t(ctypes.Structure):
    _fields_ = [
        ("n_total", ctypes.c_int), ("n_systems", ctypes.c_int), ("n_size_classes", ctypes.c_int),
        ("grid_points", ctypes.c_longlong),
        ("scatter_items", ctypes.c_int), ("gather_items", ctypes.c_int),
        ("scatter_ctas", ctypes.c_int), ("gather_ctas", ctypes.c_int),
        ("largest_first", ctypes.c_int),
        ("xyzq", ctypes.c_void_p), ("energies", ctypes.c_void_p), ("forces", ctypes.c_void_p),
        ("dLdE", ctypes.c_void_p), ("grad_forces", ctypes.c_void_p), ("grad_out", ctypes.c_void_p),
        ("fused", ctypes.c_int), ("gather_lanes", ctypes.c_int), ("fused_ctas", ctypes.c_int),
        ("graph_kernels", ctypes.c_int), ("fused_available", ctypes.c_int),
    ]


# Every exported symbol with (restype, argtypes); used both to bind and by
# the CPU test that checks the library exports what the header declares.
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "gse_params_default": (None, [ctypes.POINTER(gse_params_t)]),
    "gse_status_string": (ctypes.c_char_p, [_i]),
    "gse_last_error": (ctypes.c_char_p, []),
    "gse_abi_version": (_i, []),
    "gse_create": (_i, [ctypes.POINTER(gse_params_t), ctypes.POINTER(_vp)]),
    "gse_destroy": (_i, [_vp]),
    "gse_set_stream": (_i, [_vp, _vp]),
    "gse_set_box": (_i, [_vp, _d, _d, _d]),
    "gse_synchronize": (_i, [_vp]),
    "gse_spread_charge": (_i, [_vp, _i, _vp]),
    "gse_solve_poisson": (_i, [_vp]),
    "gse_calculate_energy": (_i, [_vp, _vp]),
    "gse_interpolate_force": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "gse_forward": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "gse_get_grid": (_i, [_vp, _i, _vp]),
    "gse_set_grid": (_i, [_vp, _i, _vp]),
    "gse_gauss_spread": (_i, [_vp, _d, _d, _i, _vp, _d, _d, _d, _i, _vp]),
    "gse_gauss_interpolate": (_i, [_vp, _d, _d, _i, _vp, _d, _d, _d, _vp, _vp, _vp, _vp]),
    "gse_green_mul": (_i, [_vp, _d, _d, _d, _d, _vp]),
    "gse_fft_solve": (_i, [_vp, _d, _d, _d, _d, _vp, _vp]),
    "gse_gauss_spread_on_grid": (_i, [_vp, _d, _d, _d, _d, _d, _vp, _vp]),
    "gse_gauss_efield_on_grid": (_i, [_vp, _d, _d, _d, _vp, _vp, _vp, _vp]),
    "gse_gauss_dipole_sum": (_i, [_vp, _d, _d, _d, _vp, _vp]),
    "gse_virial": (_i, [_vp, _vp]),
    "gse_interpolate_field": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "gse_set_timing": (_i, [_vp, _i]),
    "gse_get_timing": (_i, [_vp, _vp, _vp, _i]),
    "gse_get_launch_count": (_i, [_vp, _vp]),
    "gse_spread_mixed_noalloc": (_i, [_i, _i, _i, _d, _d, _i, _vp, _d, _d, _d, _vp, _vp]),
    "gse_adjoint": (_i, [_vp, _i, _vp, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gse_ewald_recip": (_i, [_i, _vp, _d, _i, _d, _d, _d, _d, _i, _vp, _vp, _vp, _vp, _vp]),
    "gse_ewald_direct": (_i, [_i, _vp, _d, _d, _d, _d, _d, _d, _i, _vp, _i, _vp, _vp, _vp, _vp,
                              _vp, _vp]),
    "gse_get_paths": (_i, [_vp, ctypes.POINTER(_i)]),
    "gse_measure_fp32_rate": (_i, [_i, _vp, _vp, _vp]),
    "gse_batch_create": (_i, [ctypes.POINTER(gse_params_t), _i, ctypes.POINTER(gse_system_t),
                              ctypes.POINTER(_vp)]),
    "gse_batch_destroy": (_i, [_vp]),
    "gse_batch_set_stream": (_i, [_vp, _vp]),
    "gse_batch_info": (_i, [_vp, ctypes.POINTER(gse_batch_info_t)]),
    "gse_batch_forward": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "gse_batch_adjoint": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gse_batch_capture": (_i, [_vp, _i]),
    "gse_batch_launch": (_i, [_vp]),
    "gse_batch_autotune": (_i, [_vp, ctypes.c_char_p, _i]),
    "gse_batch_set_schedule": (_i, [_vp, _i, _i, _i, _i, _i]),
    "gse_build_info": (ctypes.c_char_p, []),
}
STAGES = ["bin", "spread", "fft_forward", "green", "fft_backward", "gather"]

_lib = None


def load(build_if_missing: bool = True):
    global _lib
    if _lib is not None:
        return _lib
    from . import build
    fresh = build.built_hash(LIB_PATH) == build.source_hash()
    if not fresh:
        # missing, or built from other sources than the ones beside it
        if not build_if_missing:
            raise GseError(7, f"{LIB_PATH} is not built from the current sources")
        build.build_lib(force=True)
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != GSE_OK:
        msg = _lib.gse_last_error().decode() if _lib is not None else ""
        raise GseError(status, msg)


def ptr_f64(obj: Any, n: int, name: str):
    """Address of a per-atom float64 array (numpy or torch) holding at least n
    contiguous values; GseError (invalid argument) for any other dtype, a
    strided view or a shorter array, where the library would otherwise write
    or read doubles past its end.  None and raw integer addresses pass
    through unchecked."""
    if obj is None or isinstance(obj, int):
        return obj
    if hasattr(obj, "data_ptr"):  # torch.Tensor
        import torch
        ok = obj.dtype == torch.float64 and obj.is_contiguous() and obj.numel() >= n
    elif hasattr(obj, "ctypes") and hasattr(obj, "dtype"):  # numpy.ndarray
        import numpy as np
        ok = obj.dtype == np.float64 and obj.flags.c_contiguous and obj.size >= n
    else:
        return ptr(obj)
    if not ok:
        raise GseError(1, f"{name} must hold at least {n} contiguous float64 values "
                          f"(got {getattr(obj, 'dtype', type(obj))}, "
                          f"{getattr(obj, 'size', None) if not hasattr(obj, 'numel') else obj.numel()} values)")
    return ptr(obj)


def ptr_records(obj: Any, n: int, itemsize: int, name: str = "xyzq"):
    """Address of n position records {x, y, z, q} of the calculation type
    (itemsize 4: float32, 8: float64), as numpy or torch.  GseError (invalid
    argument) for another dtype, a strided view, fewer than 4n values or -- for
    CUDA tensors, which the kernels read in place as float4/double4 records --
    a start that is not 4*itemsize-byte aligned.  None and raw integer
    addresses pass through unchecked (the library checks device addresses
    itself)."""
    if obj is None or isinstance(obj, int):
        return obj
    if hasattr(obj, "data_ptr"):  # torch.Tensor
        import torch
        want = torch.float32 if itemsize == 4 else torch.float64
        ok = obj.dtype == want and obj.is_contiguous() and obj.numel() >= 4 * n
        if ok and getattr(obj, "is_cuda", False) and obj.data_ptr() % (4 * itemsize) != 0:
            raise GseError(1, f"{name} is device memory that is not {4 * itemsize}-byte aligned "
                              "(its records are read as 16/32-byte vectors)")
    elif hasattr(obj, "ctypes") and hasattr(obj, "dtype"):  # numpy.ndarray
        import numpy as np
        want = np.float32 if itemsize == 4 else np.float64
        ok = obj.dtype == want and obj.flags.c_contiguous and obj.size >= 4 * n
    else:
        return ptr(obj)
    if not ok:
        raise GseError(1, f"{name} must hold at least {n} contiguous {{x, y, z, q}} records of "
                          f"float{8 * itemsize} (got {getattr(obj, 'dtype', type(obj))})")
    return ptr(obj)


def ptr(obj: Any):
    """Address of a numpy array, a torch tensor, a ctypes object or an int."""
    if obj is None:
        return None
    if isinstance(obj, int):
        return obj
    if hasattr(obj, "data_ptr"):          # torch.Tensor
        return obj.data_ptr()
    if hasattr(obj, "ctypes"):            # numpy.ndarray
        return obj.ctypes.data
    if isinstance(obj, ctypes._SimpleCData) or isinstance(obj, ctypes.Array):
        return ctypes.addressof(obj)
    raise TypeError(f"cannot take the address of {type(obj)}")
