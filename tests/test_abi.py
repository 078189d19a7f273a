"""The C-ABI library: it loads on a CPU-only host, exports every symbol the
header declares, and fails cleanly (a status, never a crash) without a GPU."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(gse_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    from gse_b200 import _lib, build
    build.build_lib()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    for name in sorted(header_functions()):
        assert hasattr(lib, name), name


def test_binding_covers_header():
    from gse_b200 import _lib
    assert set(_lib.SIGNATURES) == header_functions()


def test_params_default_and_strings(lib):
    from gse_b200 import _lib
    p = _lib.gse_params_t()
    lib.gse_params_default(ctypes.byref(p))
    assert p.kappa == 0.4 and p.lambda_sigma == 3.0 and p.lambda_sigma1 == 3.0
    assert p.ccelec == 332.0716 and p.precision == 0 and p.device == 0
    for code, name in _lib.STATUS_NAMES.items():
        assert lib.gse_status_string(code).decode() == name
    assert lib.gse_abi_version() == 1


def test_create_rejects_bad_params_before_touching_a_gpu(lib):
    from gse_b200 import _lib
    p = _lib.gse_params_t()
    lib.gse_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    # sizes unset
    assert lib.gse_create(ctypes.byref(p), ctypes.byref(h)) == 1
    p.size_x = p.size_y = p.size_z = 8
    p.sigma, p.box_x, p.box_y, p.box_z = 2.0, 8.0, 8.0, 8.0
    p.kappa = 0.7  # CpuGSE::setParam asserts kappa <= 0.5
    assert lib.gse_create(ctypes.byref(p), ctypes.byref(h)) == 1
    assert "kappa" in lib.gse_last_error().decode()
    assert not h.value


def test_create_without_gpu_reports_unsupported(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gse_b200 import _lib
    p = _lib.gse_params_t()
    lib.gse_params_default(ctypes.byref(p))
    p.size_x = p.size_y = p.size_z = 8
    p.sigma, p.box_x, p.box_y, p.box_z = 2.0, 8.0, 8.0, 8.0
    h = ctypes.c_void_p()
    assert lib.gse_create(ctypes.byref(p), ctypes.byref(h)) == 7
    assert not h.value


def test_null_context_is_an_error(lib):
    assert lib.gse_solve_poisson(None) == 1
    assert lib.gse_destroy(None) == 0
    assert lib.gse_batch_forward(None, None, None, None, None, None) == 1
    assert lib.gse_batch_launch(None) == 1
    assert lib.gse_batch_destroy(None) == 0


def test_batch_create_checks_arguments_before_touching_a_gpu(lib):
    import torch
    from gse_b200 import _lib
    p = _lib.gse_params_t()
    lib.gse_params_default(ctypes.byref(p))
    p.sigma = 2.0
    systems = (_lib.gse_system_t * 2)()
    for s in systems:
        s.size_x = s.size_y = s.size_z = 16
        s.box_x = s.box_y = s.box_z = 16.0
        s.n = 30
    h = ctypes.c_void_p()
    assert lib.gse_batch_create(ctypes.byref(p), 0, systems, ctypes.byref(h)) == 1
    # the FP64 form has no batched path
    assert lib.gse_batch_create(ctypes.byref(p), 2, systems, ctypes.byref(h)) == 7
    assert "mixed" in lib.gse_last_error().decode()
    p.precision = _lib.PRECISION["mixed"]
    p.kappa = 0.6
    assert lib.gse_batch_create(ctypes.byref(p), 2, systems, ctypes.byref(h)) == 1
    p.kappa = 0.4
    if not torch.cuda.is_available():
        assert lib.gse_batch_create(ctypes.byref(p), 2, systems, ctypes.byref(h)) == 7
    assert not h.value


def test_python_mirror_has_reference_methods():
    from gse_b200 import gse
    for cls, methods in {
        gse.CpuGSEk: ["spreadCharge1", "solvePoisson", "calculateEnergy", "interpolateForce",
                      "getRhoS", "getPhi", "getSigma1", "getSigma2", "getLambdaSigma1",
                      "setBoxSize", "printInfo"],
        gse.CpuGaussCharge: ["spreadChargeToGrid", "interpolateForce", "calcSupportSize"],
        gse.CpuGreensFuncGSE: ["mul"],
        gse.CpuFFTSolver: ["run"],
        gse.CpuGrid: ["clear", "add", "sub", "copy", "scale", "sum", "maxAbsValue",
                      "getDataValue", "save", "getPos", "getDataPointer"],
    }.items():
        for m in methods:
            assert callable(getattr(cls, m)), (cls, m)


def test_support_size_matches_reference_formula():
    """calcSupportSize (CpuGaussCharge.cpp:28-56) is host arithmetic."""
    from gse_b200 import gse
    import numpy as np
    g = gse.CpuGaussCharge.__new__(gse.CpuGaussCharge)
    g.sizeX = g.sizeY = g.sizeZ = 20
    # brute force the reference's loop
    h = 1.0
    rcut = 3 * np.sqrt(2.0) * 2.121320344 * np.sqrt(0.4)
    n = int(np.ceil(rcut / h))
    cnt = 0
    for tz in range(-n, n + 1):
        for ty in range(-n, n + 1):
            for tx in range(-n, n + 1):
                dx, dy, dz = (abs(tx) - 1) * h, (abs(ty) - 1) * h, (abs(tz) - 1) * h
                cnt += (dx * dx + dy * dy + dz * dz) < rcut * rcut
    assert g.calcSupportSize(rcut, 20.0, 20.0, 20.0) == cnt
    # the mixed instance forms the distances in float32, as CT = float does
    g.dtype = np.float32
    rc2 = np.float32(rcut * rcut)
    cnt32 = 0
    for tz in range(-n, n + 1):
        for ty in range(-n, n + 1):
            for tx in range(-n, n + 1):
                dx, dy, dz = (np.float32(abs(t) - 1) * np.float32(h) for t in (tx, ty, tz))
                cnt32 += (dx * dx + dy * dy) + dz * dz < rc2
    assert g.calcSupportSize(rcut, 20.0, 20.0, 20.0) == cnt32


def test_library_is_stamped_with_its_sources():
    """The library carries the hash of the sources it was built from; the
    loader rebuilds a library whose stamp differs from the sources beside it,
    and gse_build_info reports the stamp."""
    from gse_b200 import _lib, build
    h = build.source_hash()
    assert len(h) == 16 and build.built_hash() == h
    info = _lib.load().gse_build_info().decode()
    assert info.startswith(f"sources {h}, nvcc ") and info.endswith("sm_100a")
